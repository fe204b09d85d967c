// Device-side definitions shared by the rhgpu kernels (sm_100a).
//
// Grid: nx*ny*nz cells (Corsair 1x1x1 blocks), linear index n = i + nx*(j + ny*k).
// Field arrays are stored component-planar in HBM: component l of cell n of a
// vector array lives at a[l*N + n], so that neighbouring threads (cells) read
// neighbouring addresses. The C ABI converts from/to ParGrid's interleaved
// layout on upload/download.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/rhgpu.h"

namespace rh {

struct GridInfo {
   int nx, ny, nz;
   int per[3];
   long long N;
   double dx, dt, dV, dx_below;
   double rdx;   // 1/dx, correctly rounded
   double x_min, y_min, z_min;
};

__host__ __device__ inline bool wrapc(int& i, int n, int per) {
   if (i >= 0 && i < n) return true;
   if (!per) return false;
   i = (i + n) % n;
   return true;
}

__host__ __device__ inline long long cidx(const GridInfo& g, int i, int j, int k) {
   return (long long)i + (long long)g.nx * ((long long)j + (long long)g.ny * (long long)k);
}

// neighbour (di,dj,dk) of cell (i,j,k), or -1 where the box has no neighbour
__host__ __device__ inline long long nbr(const GridInfo& g, int i, int j, int k, int di, int dj, int dk) {
   int a = i + di, b = j + dj, c = k + dk;
   if (!wrapc(a, g.nx, g.per[0]) || !wrapc(b, g.ny, g.per[1]) || !wrapc(c, g.nz, g.per[2])) return -1;
   return cidx(g, a, b, c);
}

// ParGrid's ALL_NEIGHBOURS_EXIST test for a cell
__host__ __device__ inline bool allNb(const GridInfo& g, int i, int j, int k) {
   return (g.per[0] || (i > 0 && i < g.nx - 1)) && (g.per[1] || (j > 0 && j < g.ny - 1)) &&
          (g.per[2] || (k > 0 && k < g.nz - 1));
}
__host__ __device__ inline bool xPos(const GridInfo& g, int i) { return g.per[0] || i < g.nx - 1; }
__host__ __device__ inline bool yPos(const GridInfo& g, int j) { return g.per[1] || j < g.ny - 1; }
__host__ __device__ inline bool zPos(const GridInfo& g, int k) { return g.per[2] || k < g.nz - 1; }
__host__ __device__ inline bool xNeg(const GridInfo& g, int i) { return g.per[0] || i > 0; }
__host__ __device__ inline bool yNeg(const GridInfo& g, int j) { return g.per[1] || j > 0; }
__host__ __device__ inline bool zNeg(const GridInfo& g, int k) { return g.per[2] || k > 0; }
// + neighbours exist (required by cell2Node, calcNodeJ, calcNodeUe,
// upwindNodeB, calcNodeE, faceCurl: hybrid_propagator.cpp:1064-1067 etc.)
__host__ __device__ inline bool plusOk(const GridInfo& g, int i, int j, int k) {
   return xPos(g, i) && yPos(g, j) && zPos(g, k);
}

// missing-wall mask of an exterior cell: 1=-x 2=+y 4=-y 8=+z 16=-z 32=+x
__host__ __device__ inline int missingMask(const GridInfo& g, int i, int j, int k) {
   int m = 0;
   if (!xNeg(g, i)) m |= 1;
   if (!yPos(g, j)) m |= 2;
   if (!yNeg(g, j)) m |= 4;
   if (!zPos(g, k)) m |= 8;
   if (!zNeg(g, k)) m |= 16;
   if (!xPos(g, i)) m |= 32;
   return m;
}

__host__ __device__ inline double blockOrigin(double xmin, int i, double dx) { return xmin + (double)i * dx; }

__host__ __device__ inline int dirFromOffset(int dxs, int dys, int dzs) { return (dzs + 1) * 9 + (dys + 1) * 3 + (dxs + 1); }
// stayers first, then arrivals in direction order
__host__ __device__ inline int dirRank(int dir) { return dir == 13 ? 0 : (dir < 13 ? dir + 1 : dir); }
__host__ __device__ inline int rankToDir(int r) { return r == 0 ? 13 : (r <= 13 ? r - 1 : r); }

// Particle migration (Corsair's particle list is not vendored; this is the
// rule the oracle restates too): a local coordinate that left [0,dx) shifts
// by exactly one cell, x + dx rounding up to dx becomes the largest double
// below dx. Returns nonzero when the particle moved more than one cell.
__host__ __device__ inline int migrateAxis(double& x, int& off, double dx, double dx_below) {
   int st = 0;
   off = 0;
   if (x < 0.0) {
      x += dx;
      off = -1;
      if (x >= dx) x = dx_below;
      if (x < 0.0) st = 1;
   } else if (x >= dx) {
      x -= dx;
      off = 1;
      if (x >= dx) st = 1;
   }
   return st;
}

// x / dx, correctly rounded, without a division: Markstein's method (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000 processor",
// IBM J. Res. Dev. 34(1), 1990). With r = RN(1/dx) and q = RN(x r), the residual
// e = x - q dx is exact in one fused multiply-add and RN(q + e r) = RN(x / dx).
// The method needs no overflow or underflow on the way: quotients outside
// [2^-500, 2^500] in magnitude (zeros, NaN and infinities included) take the
// IEEE division; rhgpu_create keeps dx within [2^-200, 2^200].
__device__ inline double divDx(double x, const GridInfo& g) {
   const double q = x * g.rdx;
   const double aq = fabs(q);
   if (!(aq >= 0x1p-500 && aq <= 0x1p+500)) return x / g.dx;
   const double e = fma(-q, g.dx, x);
   return fma(e, g.rdx, q);
}

#ifdef __CUDACC__
// ---- per-thread asynchronous global -> shared copies (cp.async) ----------------------------------
// bytes = 0 copies nothing and writes zeros (the source address is not read)
__device__ __forceinline__ void cpAsync8(void* sdst, const void* gsrc, int bytes) {
   const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
   asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gsrc), "r"(bytes) : "memory");
}
// 4-byte form (both addresses 4-byte aligned)
__device__ __forceinline__ void cpAsync4(void* sdst, const void* gsrc) {
   const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
   asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
// 16-byte form (both addresses 16-byte aligned)
__device__ __forceinline__ void cpAsync16(void* sdst, const void* gsrc, int bytes) {
   const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
   asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpAsyncWaitAll() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
// every group but the newest N of this thread complete
template <int N>
__device__ __forceinline__ void cpAsyncWaitGroup() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
#endif

}  // namespace rh
