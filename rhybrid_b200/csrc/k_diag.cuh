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
k_diag_particles_seg(SegBuf B, const long long* base, long long NS, double* part) {
   __shared__ double sm[DIAG_THREADS];
   double v[DIAG_P] = {0, 0, 0, 0, 0, 0, 0, 0};
   for (long long S = blockIdx.x; S < NS; S += gridDim.x)
      for (int r = threadIdx.x; r < B.cnt[S]; r += blockDim.x) {
         double st[7];
         for (int e = 0; e < 7; ++e) st[e] = B.a[e][base[S] + r];
         particleTerms(st, v);
      }
   blockReduce(v, DIAG_P_MAX, sm, part + (long long)blockIdx.x * DIAG_P);
}

// exact path: one species' particles of the cells blockIdx.x, +gridDim.x, ...
__global__ void __launch_bounds__(DIAG_THREADS)
k_diag_particles_cell(PStore P, long long N, double* part) {
   __shared__ double sm[DIAG_THREADS];
   double v[DIAG_P] = {0, 0, 0, 0, 0, 0, 0, 0};
   for (long long c = blockIdx.x; c < N; c += gridDim.x)
      for (int r = threadIdx.x; r < P.alive[c]; r += blockDim.x) {
         double st[7];
         for (int e = 0; e < 7; ++e) st[e] = P.a[e][P.start[c] + r];
         particleTerms(st, v);
      }
   blockReduce(v, DIAG_P_MAX, sm, part + (long long)blockIdx.x * DIAG_P);
}

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
k_diag_field(GridInfo g, Fields f, const double* rhoM, int includeInner, double* part) {
   __shared__ double sm[DIAG_THREADS];
   double v[DIAG_FS];
   for (int q = 0; q < DIAG_FS; ++q) v[q] = ((DIAG_F_MIN >> q) & 1ull) ? INFINITY : 0.0;
   const long long N = g.N;
   for (long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += (long long)gridDim.x * blockDim.x) {
      const int i = (int)(n % g.nx), j = (int)((n / g.nx) % g.ny), k = (int)(n / ((long long)g.nx * g.ny));
      if (!allNb(g, i, j, k)) continue;
      if (!includeInner && (f.flags[n] & RHGPU_FLAG_INNER_FIELD)) continue;
      const double bx1 = f.faceB[n], bx0 = f.faceB[nbr(g, i, j, k, -1, 0, 0)];
      const double by1 = f.faceB[N + n], by0 = f.faceB[N + nbr(g, i, j, k, 0, -1, 0)];
      const double bz1 = f.faceB[2 * N + n], bz0 = f.faceB[2 * N + nbr(g, i, j, k, 0, 0, -1)];
      double divB = ((bx1 - bx0) + (by1 - by0) + (bz1 - bz0)) / g.dx;
      divB = fabs(divB);
      const double Bx = 0.5 * (bx1 + bx0), By = 0.5 * (by1 + by0), Bz = 0.5 * (bz1 + bz0);
      const double B2 = sq(Bx) + sq(By) + sq(Bz);
      const double Btot = sqrt(B2);
      const double divBPerB = Btot > 0.0 ? divB / Btot : 0.0;
      v[0] += 1.0;
      v[1] += Bx; v[2] += By; v[3] += Bz; v[4] += Btot;
      if (Btot > v[5]) v[5] = Btot;
      v[6] += divB;
      if (divB > v[7]) v[7] = divB;
      if (divBPerB > v[8]) v[8] = divBPerB;
      v[9] += B2;
      const double jx = f.cellJi[n], jy = f.cellJi[N + n], jz = f.cellJi[2 * N + n];
      const double jt = sqrt(sq(jx) + sq(jy) + sq(jz));
      v[10] += jx; v[11] += jy; v[12] += jz; v[13] += jt;
      if (jt > v[14]) v[14] = jt;
      const double ex = f.cellEp[n], ey = f.cellEp[N + n], ez = f.cellEp[2 * N + n];
      const double ep2 = sq(ex) + sq(ey) + sq(ez);
      const double ept = sqrt(ep2);
      v[15] += ex; v[16] += ey; v[17] += ez; v[18] += ept;
      if (ept > v[19]) v[19] = ept;
      v[20] += ep2;
      const double nx_ = f.nodeE[n], ny_ = f.nodeE[N + n], nz_ = f.nodeE[2 * N + n];
      const double ne2 = sq(nx_) + sq(ny_) + sq(nz_);
      const double net = sqrt(ne2);
      v[21] += nx_; v[22] += ny_; v[23] += nz_; v[24] += net;
      if (net > v[25]) v[25] = net;
      v[26] += ne2;
      const double ux = f.cellUe[n], uy = f.cellUe[N + n], uz = f.cellUe[2 * N + n];
      const double cex = -(uy * Bz - uz * By), cey = -(uz * Bx - ux * Bz), cez = -(ux * By - uy * Bx);
      v[27] += sq(cex) + sq(cey) + sq(cez);
      const double ut = sqrt(sq(ux) + sq(uy) + sq(uz));
      if (ut > v[28]) v[28] = ut;
      const double rq = f.cellRho[n];
      v[29] += rq;
      if (rq > 0.0) { v[30] = fmin(v[30], rq); v[31] = fmax(v[31], rq); }
      if (rhoM) {
         const double rm = rhoM[n];
         if (rm > 0.0) {
            v[32] = fmin(v[32], rm);
            v[33] = fmax(v[33], rm);
            const double vA = Btot / sqrt(RHGPU_PERMEABILITY * rm);
            if (vA > v[34]) v[34] = vA;
         }
      }
   }
   blockReduce(v, DIAG_F_MAX, sm, part + (long long)blockIdx.x * DIAG_FS, DIAG_F_MIN);
}

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
__global__ void k_diag_rhom_cell(MassSet M, long long N, double dV, double minRhoM, double* rhoM) {
   const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (n >= N) return;
   double a = 0.0;
   for (int s = 0; s < M.ns; ++s) {
      const PStore& P = M.P[s];
      if (!P.start) continue;
      const long long b = P.start[n];
      for (int r = 0; r < P.alive[n]; ++r) a += P.a[6][b + r] * M.m[s];
   }
   a /= dV;
   rhoM[n] = a < minRhoM ? minRhoM : a;
}
// fast path: exact 128-bit fixed-point sums of w*m per cell (order-independent),
// the particle's cell from its segment, dual x index and half-cell side
__global__ void k_diag_rhom_seg(GridInfo g, FastGeom fg, SegBuf B, const long long* base, double m, double scale,
                                unsigned long long* lo, unsigned long long* hi) {
   for (long long S = blockIdx.x; S < fg.NS; S += gridDim.x) {
      const long long row = S / fg.nseg;
      const int gs = (int)(S % fg.nseg);
      const int uy = (int)(row % fg.nd[1]), uz = (int)(row / fg.nd[1]);
      const int c = B.cnt[S];
      for (int r = threadIdx.x; r < c; r += blockDim.x) {
         const long long slot = base[S] + r;
         int ci = dualB(gs * SEG + B.lx[slot], g.per[0]) + 1 - halfS(B.a[0][slot], g.dx);
         int cj = dualB(uy, g.per[1]) + 1 - halfS(B.a[1][slot], g.dx);
         int ck = dualB(uz, g.per[2]) + 1 - halfS(B.a[2][slot], g.dx);
         wrapc(ci, g.nx, 1); wrapc(cj, g.ny, 1); wrapc(ck, g.nz, 1);
         const long long n = cidx(g, ci, cj, ck);
         add128(lo + n, hi + n, B.a[6][slot] * m, scale);
      }
   }
}
__global__ void k_diag_rhom_finish(const unsigned long long* lo, const unsigned long long* hi, long long N, double hiScale,
                                   double loScale, double dV, double minRhoM, double* rhoM) {
   const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (n >= N) return;
   const double a = fixedToDouble(lo[n], hi[n], hiScale, loScale) / dV;
   rhoM[n] = a < minRhoM ? minRhoM : a;
}

}  // namespace rh
