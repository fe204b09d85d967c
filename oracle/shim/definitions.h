/* Oracle shim (test infrastructure only): a single-process stand-in for the
 * parts of the Corsair platform API that RHybrid's hot-path sources include.
 * Corsair/ParGrid are not vendored with the reference; this file restates the
 * few definitions those sources need so that they compile unmodified.
 *
 * Corsair block layout: RHybrid requires 1x1x1 blocks (src/user.cpp:163-167),
 * so a block is one cell and the 3x3x3 neighbourhood array has side 3.
 */
#ifndef RHSHIM_DEFINITIONS_H
#define RHSHIM_DEFINITIONS_H

#include <cstddef>
#include <cstdint>

typedef double Real;

namespace block {
   const int WIDTH_X = 1;
   const int WIDTH_Y = 1;
   const int WIDTH_Z = 1;
   const int SIZE = WIDTH_X*WIDTH_Y*WIDTH_Z;
   /* index of cell (i,j,k) inside a block */
   inline int index(int i,int j,int k) { return i + WIDTH_X*(j + WIDTH_Y*k); }
   /* index inside the (WIDTH+2)^3 neighbourhood array used by fetchData and
    * the accumulator (src/hybrid_propagator.cpp:1894-2094) */
   inline int arrayIndex(int i,int j,int k) { return i + (WIDTH_X+2)*(j + (WIDTH_Y+2)*k); }
}

#endif
