/* Oracle (test infrastructure only): rules that the reference leaves to the
 * Corsair platform (not vendored), stated once and shared by the reference
 * build driver (ref_driver.cpp) and the C restatement (rh_oracle.c). The GPU
 * library implements the same rules in rhybrid_b200/csrc/rh_device.cuh.
 *
 * Block origin: Corsair's block coordinate array holds the minimum corner of
 * each 1x1x1 block; restated as x_min + i*dx.
 *
 * Migration: after the drift x += dt*v (boris.h:191-193) a particle whose
 * local coordinate left [0,dx) on an axis moves to the neighbour cell on that
 * axis and its local coordinate shifts by exactly dx:
 *   x <  0  -> x += dx, cell index -1 (if rounding gives x == dx, x becomes
 *              the largest double below dx so that x stays in [0,dx));
 *   x >= dx -> x -= dx, cell index +1 (exact by Sterbenz' lemma).
 * A particle still outside [0,dx) after one shift moved more than one cell in
 * a step; it is removed and counted (the maximum ion speed of 0.9 dx/dt,
 * src/user.cpp:1774-1777, keeps accelerated particles below one cell).
 * In the destination cell, the particles that stayed come first, in their
 * previous order; then the arrivals, grouped by the direction they came from
 * (dir = (dz+1)*9 + (dy+1)*3 + (dx+1) with (dx,dy,dz) = source cell -
 * destination cell; stayers have dir 13) in increasing dir, each group in its
 * order inside the source cell. rh_dir_rank() gives the position of a dir in
 * that sequence.
 */
#ifndef RH_ORACLE_COMMON_H
#define RH_ORACLE_COMMON_H

#include <stdint.h>

static inline int rh_wrap(int* i,int n,int periodic) {
   if (*i >= 0 && *i < n) return 1;
   if (!periodic) return 0;
   *i = (*i + n) % n;
   return 1;
}

static inline double rh_block_origin(double xmin,int i,double dx) { return xmin + (double)i*dx; }

static inline int rh_dir_from_offset(int dxs,int dys,int dzs) { return (dzs+1)*9 + (dys+1)*3 + (dxs+1); }

/* order of a direction group inside the destination cell: stayers (dir 13)
 * first, then dir 0..12, 14..26 */
static inline int rh_dir_rank(int dir) { return dir == 13 ? 0 : (dir < 13 ? dir + 1 : dir); }

/* shifts r into [0,dx) by at most one cell per axis; off[a] in {-1,0,1};
 * returns nonzero if the particle moved more than one cell */
static inline int rh_migrate_canonical(double r[3],double dx,double dx_below,int off[3]) {
   int st = 0;
   for (int a=0;a<3;++a) {
      double x = r[a];
      int o = 0;
      if (x < 0.0) {
         x += dx; o = -1;
         if (x >= dx) x = dx_below;
         if (x < 0.0) st = 1;
      } else if (x >= dx) {
         x -= dx; o = 1;
         if (x >= dx) st = 1;
      }
      r[a] = x; off[a] = o;
   }
   return st;
}

#endif
