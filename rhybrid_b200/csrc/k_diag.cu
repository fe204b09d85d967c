// Definitions of the kernels declared in k_diag.cuh (each declaration there says
// what its kernel does); the template kernels stay in the header.
#include "k_diag.cuh"

namespace rh {

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
