// Definitions of the kernels declared in k_avg.cuh (each declaration there says
// what its kernel does); the template kernels stay in the header.
#include "k_avg.cuh"

namespace rh {

__global__ void k_deposit_gather_avg(GridInfo g, const double* S, double* nSum, double* vSum) {
   RH_CELL_PROLOGUE
   const Sources3 Q = sortedSources(g, i, j, k);
   double v[4];
   v[0] = nSum[n];
   for (int l = 0; l < 3; ++l) v[1 + l] = vSum[l * N + n];
   addSources(g, Q, S, N, v);
   nSum[n] = v[0];
   for (int l = 0; l < 3; ++l) vSum[l * N + n] = v[1 + l];
}

__global__ void k_fast_avg_movers(GridInfo g, FastGeom fg, FastSpecies FS, const Mover* mv, long long n, unsigned mask,
                                  FastBufs fb) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= n) return;
   const Mover& M = mv[t];
   if (!(M.lx & (MOVER_DEPOSIT | MOVER_AVG)) || !((mask >> M.species) & 1u)) return;
   moverAdd128<false>(g, fg, FS, M, fb.MMlo, fb.MMhi, fb.scaleR, fb.scaleJ, nullptr);
}

__global__ void k_fast_avg_gather(GridInfo g, FastGeom fg, FastBufs fb, double hiR, double loR, double hiJ, double loJ,
                                  double* nSum, double* vSum) {
   RH_CELL_PROLOGUE
   const bool bnd = g.per[0] ? (fg.nseg > 1 && i % SEG == 0) : ((i + 1) % SEG == 0);
   const int gb = g.per[0] ? i / SEG : (i + 1) / SEG;
   double v[4];
   for (int qq = 0; qq < 4; ++qq) {
      const int uyy = dualU(j - (qq & 1), g.ny, g.per[1]);
      const int uzz = dualU(k - (qq >> 1), g.nz, g.per[2]);
      const long long row = (long long)uyy + (long long)fg.nd[1] * uzz;
      const double* rp = fb.RP + (((long long)qq * fg.nrows + row) * g.nx + i) * 4;
      const double* rb = fb.RPB + (((long long)qq * fg.nrows + row) * fg.nseg + gb) * 4;
      for (int l = 0; l < 4; ++l) {
         double r = rp[l];
         if (bnd) r = r + rb[l];
         v[l] = qq == 0 ? r : v[l] + r;
      }
   }
   v[0] += fixedToDouble(fb.MMlo[n], fb.MMhi[n], hiR, loR);
   for (int l = 0; l < 3; ++l) v[1 + l] += fixedToDouble(fb.MMlo[(1 + l) * N + n], fb.MMhi[(1 + l) * N + n], hiJ, loJ);
   for (int l = 0; l < 4; ++l) { fb.MMlo[l * N + n] = 0ull; fb.MMhi[l * N + n] = 0ull; }
   nSum[n] += v[0];
   for (int l = 0; l < 3; ++l) vSum[l * N + n] += v[1 + l];
}

__global__ void k_avg_output(long long N, double* nSum, double* vSum, double q, double dV, double inv, double* nOut,
                             double* vOut) {
   const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (n >= N) return;
   const double a = nSum[n];
   if (nOut) nOut[n] = a / (q * dV) * inv;
   if (vOut)
      for (int l = 0; l < 3; ++l) vOut[3 * n + l] = a > 0 ? vSum[l * N + n] / a : 0.0;
   nSum[n] = 0.0;
   for (int l = 0; l < 3; ++l) vSum[l * N + n] = 0.0;
}

__global__ void k_avgB_output(long long N, double* sumB, double inv, double* out) {
   const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (n >= N) return;
   for (int l = 0; l < 3; ++l) {
      out[3 * n + l] = sumB[l * N + n] * inv;
      sumB[l * N + n] = 0.0;
   }
}

}  // namespace rh
