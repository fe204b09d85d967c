// Initial fill of a population on the GPU: InjectorUniform::injectParticles
// (particle_injector.cpp:188-255) for the segment storage of the fast path and
// of the FP32 form, without host records.
//
// Every cell whose centre lies in the injector's region draws probRound(ppc)
// macroparticles (particle_injector.cpp:41-48), uniform in the central
// (1 - epsCell) of the cell, velocity U + vth N(0,1) per component (the polar
// Gaussian, as sampleGaussian), weight n dx^3 / ppc. Particle k of cell c
// draws from its own Philox stream keyed by (seed, c, k) (count: k = ~0), so
// the fill does not depend on launch shape or order.
//
// One block per storage segment: each thread takes one of the cells whose
// particles can fall in the segment's dual cells (at most 34 x 2 x 2), in a
// fixed order (z, then y, then x), regenerates their positions and keeps those
// whose dual cell is in the segment. k_fill_count gives the segment's count;
// after the layout, k_fill_write stores them in (cell order, k) order.
#pragma once

#include "rh_device.cuh"
#include "rh_rng.cuh"
#include "k_fast.cuh"
#include "k_f32.cuh"

namespace rh {

struct FillSpec {
   unsigned long long seed;
   double ppc;              // macroparticles per cell (probRound)
   double w;                // weight
   double vth;              // sqrt(k_B T / m)
   double U[3];             // bulk velocity
   double lo[3], hi[3];     // region of the cell centres (global coordinates)
   int species;
};

constexpr double FILL_EPS_CELL = 1e-4;   // epsCell of the injectors
constexpr int FILL_MAX_CELLS = (SEG + 2) * 4;
constexpr int FILL_THREADS = 256;
static_assert(FILL_MAX_CELLS <= FILL_THREADS, "one thread per candidate cell");

__device__ inline void fillStream(RngStream& r, const FillSpec& F, long long c, unsigned k) {
   r.init(F.seed, (uint32_t)c, (uint32_t)((unsigned long long)c >> 32) ^ (0x5A000000u | (uint32_t)F.species), k);
}

// probRound(ppc) for cell c whose centre is in the region, else 0
__device__ inline int fillCount(const FillSpec& F, const GridInfo& g, int i, int j, int k) {
   const double xc = g.x_min + (i + 0.5) * g.dx, yc = g.y_min + (j + 0.5) * g.dx, zc = g.z_min + (k + 0.5) * g.dx;
   if (xc < F.lo[0] || xc > F.hi[0] || yc < F.lo[1] || yc > F.hi[1] || zc < F.lo[2] || zc > F.hi[2]) return 0;
   const double f = floor(F.ppc);
   RngStream r;
   fillStream(r, F, cidx(g, i, j, k), 0xffffffffu);
   return (int)f + (r.uniform() < F.ppc - f ? 1 : 0);
}

// the cell-local position of particle k (the first three draws of its stream)
__device__ inline void fillPosition(RngStream& r, const GridInfo& g, double x[3]) {
   const double xc = 0.5 * g.dx;
   for (int a = 0; a < 3; ++a) x[a] = xc + (1.0 - FILL_EPS_CELL) * g.dx * (r.uniform() - 0.5);
}

// the candidate cell t of segment S: false if t is past the candidates or the
// cell is outside a non-periodic box
__device__ inline bool fillCell(const GridInfo& g, const FastGeom& fg, long long S, int t, int& i, int& j, int& k,
                                int& uy, int& uz, int& u0, int& u1) {
   const long long row = S / fg.nseg;
   const int gseg = (int)(S % fg.nseg);
   uy = (int)(row % fg.nd[1]);
   uz = (int)(row / fg.nd[1]);
   u0 = gseg * SEG;
   u1 = min(u0 + SEG, fg.nd[0]);
   // cells b and b + 1 of each dual cell b + 1 (b on a periodic axis): x from the
   // first dual cell's b to the last one's b + 1, y and z two cells; a periodic
   // axis shorter than the range (one segment along x, or ny or nz = 1) takes
   // each of its cells once
   const int x0 = dualB(u0, g.per[0]);
   int nxc = dualB(u1 - 1, g.per[0]) + 2 - x0;
   if (g.per[0] && nxc > g.nx) nxc = g.nx;
   const int nyc = (g.per[1] && g.ny < 2) ? 1 : 2, nzc = (g.per[2] && g.nz < 2) ? 1 : 2;
   if (t >= nxc * nyc * nzc) return false;
   i = x0 + t % nxc;
   j = dualB(uy, g.per[1]) + (t / nxc) % nyc;
   k = dualB(uz, g.per[2]) + t / (nxc * nyc);
   return wrapc(i, g.nx, g.per[0]) && wrapc(j, g.ny, g.per[1]) && wrapc(k, g.nz, g.per[2]);
}

// dual cell of a cell-local position: FP64 storage (halfS of the position) or
// the FP32 form (halfS of its FP32 offset, as the FP32 upload stores it)
template <bool F32>
__device__ inline void fillDual(const GridInfo& g, int i, int j, int k, const double x[3], float below1, int u[3]) {
   const int c[3] = {i, j, k};
   const int n[3] = {g.nx, g.ny, g.nz};
   for (int a = 0; a < 3; ++a) {
      const int h = F32 ? halfSf(offsetOf(x[a], g.rdx, below1)) : halfS(x[a], g.dx);
      u[a] = dualU(c[a] + h - 1, n[a], g.per[a]);
   }
}

// particles of candidate cell t that belong to segment S
template <bool F32>
__device__ inline int fillInSegment(const FillSpec& F, const GridInfo& g, const FastGeom& fg, long long S, int t,
                                    float below1) {
   int i, j, k, uy, uz, u0, u1;
   if (!fillCell(g, fg, S, t, i, j, k, uy, uz, u0, u1)) return 0;
   const int n = fillCount(F, g, i, j, k);
   const long long c = cidx(g, i, j, k);
   int m = 0;
   for (int p = 0; p < n; ++p) {
      RngStream r;
      fillStream(r, F, c, (unsigned)p);
      double x[3];
      fillPosition(r, g, x);
      int u[3];
      fillDual<F32>(g, i, j, k, x, below1, u);
      m += (u[1] == uy && u[2] == uz && u[0] >= u0 && u[0] < u1) ? 1 : 0;
   }
   return m;
}

template <bool F32>
__global__ void __launch_bounds__(FILL_THREADS) k_fill_count(GridInfo g, FastGeom fg, FillSpec F, float below1, int* cnt) {
   __shared__ int s_sum[FILL_THREADS / 32];
   const long long S = blockIdx.x;
   const int t = threadIdx.x;
   int m = fillInSegment<F32>(F, g, fg, S, t, below1);
   for (int o = 16; o > 0; o >>= 1) m += __shfl_xor_sync(0xffffffffu, m, o);
   if ((t & 31) == 0) s_sum[t >> 5] = m;
   __syncthreads();
   if (t == 0) {
      int a = 0;
      for (int w = 0; w < FILL_THREADS / 32; ++w) a += s_sum[w];
      cnt[S] = a;
   }
}

// the segment's particles in (candidate cell, k) order from slot base[S]; the
// FP64 storage (B64, 7 components + dual x in the segment) or the FP32 form (B32)
template <bool F32>
__global__ void __launch_bounds__(FILL_THREADS) k_fill_write(GridInfo g, FastGeom fg, FillSpec F, float below1,
                                                             const long long* base, SegBuf B64, F32Buf B32) {
   __shared__ int s_off[FILL_THREADS / 32];
   const long long S = blockIdx.x;
   const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
   const int m = fillInSegment<F32>(F, g, fg, S, t, below1);
   int x = m;
   for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
   }
   if (lane == 31) s_off[warp] = x;
   __syncthreads();
   int before = 0;
   for (int w = 0; w < warp; ++w) before += s_off[w];
   if (m == 0) return;
   long long slot = base[S] + before + (x - m);
   int i, j, k, uy, uz, u0, u1;
   fillCell(g, fg, S, t, i, j, k, uy, uz, u0, u1);
   const int n = fillCount(F, g, i, j, k);
   const long long c = cidx(g, i, j, k);
   for (int p = 0; p < n; ++p) {
      RngStream r;
      fillStream(r, F, c, (unsigned)p);
      double st[6];
      fillPosition(r, g, st);
      int u[3];
      fillDual<F32>(g, i, j, k, st, below1, u);
      if (!(u[1] == uy && u[2] == uz && u[0] >= u0 && u[0] < u1)) continue;
      GaussSource gs;
      gs.has = false;
      gs.ok = true;
      for (int a = 0; a < 3; ++a) st[3 + a] = F.U[a] + F.vth * gs.next(r);
      if (F32) {
         B32.cell[slot] = (int)c;
         for (int a = 0; a < 3; ++a) {
            B32.o[a][slot] = offsetOf(st[a], g.rdx, below1);
            B32.v[a][slot] = (float)st[3 + a];
         }
      } else {
         for (int a = 0; a < 6; ++a) B64.a[a][slot] = st[a];
         B64.a[6][slot] = F.w;
         B64.lx[slot] = (unsigned char)(u[0] - u0);
      }
      ++slot;
   }
}

}  // namespace rh
