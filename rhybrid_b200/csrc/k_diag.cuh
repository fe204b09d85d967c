// Global FP64 diagnostic reductions: the population log (logCalcParticle,
// diagnostics.h:187-230) and the field log (logCalcField, diagnostics.h:246-404)
// of RHybrid. Each block reduces its share in a fixed tree and writes one
// partial row; the host adds the rows in block order, so the results are
// deterministic (they differ from the reference's sequential sums by
// round-off only).
#pragma once

#include "rh_device.cuh"
#include "k_fields.cuh"
#include "k_particles.cuh"
#include "k_fast.cuh"

namespace rh {

constexpr int DIAG_BLOCKS = 592;   // 4 per SM
constexpr int DIAG_THREADS = 256;
constexpr int DIAG_P = 8;          // per species
constexpr int DIAG_F = 30;         // field quantities of the log sums
constexpr int DIAG_FS = 35;        // + the five extremes behind the spatial, temporal and velocity scales

// sums, maxima (bit q of maxMask) or minima (bit q of minMask) of v over the
// block, into out[0..nv) (thread 0)
template <int NV>
__device__ inline void blockReduce(double (&v)[NV], const unsigned long long maxMask, double* sm, double* out,
                                   const unsigned long long minMask = 0ull) {
   const int tid = threadIdx.x;
   for (int q = 0; q < NV; ++q) {
      sm[tid] = v[q];
      __syncthreads();
      for (int h = DIAG_THREADS / 2; h > 0; h >>= 1) {
         if (tid < h)
            sm[tid] = ((maxMask >> q) & 1ull)   ? fmax(sm[tid], sm[tid + h])
                      : ((minMask >> q) & 1ull) ? fmin(sm[tid], sm[tid + h])
                                                : sm[tid] + sm[tid + h];
         __syncthreads();
      }
      if (tid == 0) out[q] = sm[0];
      __syncthreads();
   }
}

// per-particle terms of the population log
__device__ inline void particleTerms(const double* st, double (&v)[DIAG_P]) {
   const double w = st[6];
   v[0] += 1.0;
   v[1] += w;
   v[2] += w * st[3];
   v[3] += w * st[4];
   v[4] += w * st[5];
   const double v2 = sq(st[3]) + sq(st[4]) + sq(st[5]);
   const double vtot = sqrt(v2);
   v[5] += w * vtot;
   v[6] += w * v2;
   if (vtot > v[7]) v[7] = vtot;
}
constexpr unsigned long long DIAG_P_MAX = 1ull << 7;

// fast path: one species' particles of the segments blockIdx.x, +gridDim.x, ...
__global__ void __launch_bounds__(DIAG_THREADS)
k_diag_particles_seg(SegBuf B, const long long* base, long long NS, double* part);

// exact path: one species' particles of the cells blockIdx.x, +gridDim.x, ...
__global__ void __launch_bounds__(DIAG_THREADS)
k_diag_particles_cell(PStore P, long long N, double* part);

// field log over cells with all neighbours, without the inner-boundary cells
// unless includeInner (Hybrid.includeInnerCellsInFieldLog, false by default).
// Slots 30..34, formed where rhoM is given (the total ion mass density per
// cell, clamped): min and max of cellRhoQi over cells with cellRhoQi > 0, min
// and max of rhoM over cells with rhoM > 0, max Alfven speed |B| / sqrt(mu0 rhoM)
// (diagnostics.h:365-395; the inertial lengths and the Larmor period are
// monotone in these extremes and are formed from them on the host).
constexpr unsigned long long DIAG_F_MAX = (1ull << 5) | (1ull << 7) | (1ull << 8) | (1ull << 14) | (1ull << 19) |
                                          (1ull << 25) | (1ull << 28) | (1ull << 31) | (1ull << 33) | (1ull << 34);
constexpr unsigned long long DIAG_F_MIN = (1ull << 30) | (1ull << 32);
__global__ void __launch_bounds__(DIAG_THREADS)
k_diag_field(GridInfo g, Fields f, const double* rhoM, int includeInner, double* part);

// total ion mass density of logCalcParticle (diagnostics.h:223-238): every
// species' w*m summed into the particle's own cell, then /dV and the floor
// minIonChargeDensity*m_p/e.
// Exact path: one thread per cell, the species in order and each cell's
// particles in order, as the reference adds them.
struct MassSet {
   int ns;
   PStore P[8];
   double m[8];
};
__global__ void k_diag_rhom_cell(MassSet M, long long N, double dV, double minRhoM, double* rhoM);
// fast path: exact 128-bit fixed-point sums of w*m per cell (order-independent),
// the particle's cell from its segment, dual x index and half-cell side
__global__ void k_diag_rhom_seg(GridInfo g, FastGeom fg, SegBuf B, const long long* base, double m, double scale,
                                unsigned long long* lo, unsigned long long* hi);
__global__ void k_diag_rhom_finish(const unsigned long long* lo, const unsigned long long* hi, long long N, double hiScale,
                                   double loScale, double dV, double minRhoM, double* rhoM);

}  // namespace rh
