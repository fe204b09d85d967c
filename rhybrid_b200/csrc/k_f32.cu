// Definitions of the kernels declared in k_f32.cuh (each declaration there says
// what its kernel does); the template kernels stay in the header.
#include "k_f32.cuh"

namespace rh {

__global__ void k_f32_mig_place(F32Set FS, long long NS, long long nb, const Mover32* mv, const unsigned* order,
                                const unsigned* bkt, const long long* off, long long n) {
   const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (q >= n) return;
   const long long b = bkt[q];
   if (b >= nb) return;
   const int s = (int)(b / NS);
   const long long S = b % NS;
   const F32Species& SS = FS.st[s];
   const long long pos = SS.base[S] + SS.nxt.cnt[S] + (q - off[b]);
   const Mover32& M = mv[order[q]];
   SS.nxt.cell[pos] = M.cell;
   for (int e = 0; e < 3; ++e) { SS.nxt.o[e][pos] = M.o[e]; SS.nxt.v[e][pos] = M.v[e]; }
}

__global__ void k_f32_mover_deposit(GridInfo g, FastGeom fg, F32Set FS, F32Bufs fb, long long n) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= n) return;
   const Mover32& M = fb.movers[t];
   if (!(M.lx & MOVER_DEPOSIT)) return;
   const int s = M.species;
   const long long row = M.dest / fg.nseg;
   const int vx = (int)(M.dest % fg.nseg) * SEG + (M.lx & 0xff);
   const int vy = (int)(row % fg.nd[1]), vz = (int)(row / fg.nd[1]);
   const int bx = dualB(vx, g.per[0]), by = dualB(vy, g.per[1]), bz = dualB(vz, g.per[2]);
   float o[3] = {M.o[0], M.o[1], M.o[2]};
   float w8[8];
   cicWeightsF(o, FS.wqRel[s], w8);
   const long long N = g.N;
   for (int q = 0; q < 8; ++q) {
      int dxc = bx + (q & 1), dyc = by + ((q >> 1) & 1), dzc = bz + ((q >> 2) & 1);
      if (!wrapc(dxc, g.nx, g.per[0]) || !wrapc(dyc, g.ny, g.per[1]) || !wrapc(dzc, g.nz, g.per[2])) continue;
      const long long dc = cidx(g, dxc, dyc, dzc);
      add128(&fb.MMlo[dc], &fb.MMhi[dc], (double)w8[q], fb.scaleR);
      for (int l = 0; l < 3; ++l)
         add128(&fb.MMlo[(1 + l) * N + dc], &fb.MMhi[(1 + l) * N + dc], (double)(w8[q] * M.v[l]), fb.scaleJ);
      fb.touched[dc] = 1;
   }
}

__global__ void k_f32_cell_keys(FastGeom fg, F32Buf B, const long long* base, const long long* first, unsigned* key,
                                unsigned long long* slots) {
   const long long S = blockIdx.x;
   const int c = B.cnt[S];
   for (int r = threadIdx.x; r < c; r += blockDim.x) {
      const long long slot = base[S] + r;
      key[first[S] + r] = (unsigned)B.cell[slot];
      slots[first[S] + r] = (unsigned long long)slot;
   }
}

__global__ void k_f32_gather_records(F32Buf B, const unsigned long long* slots, const unsigned* idx, long long n,
                                     double dx, double w, double* aos) {
   const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (j >= n) return;
   const unsigned long long slot = slots[idx[j]];
   for (int a = 0; a < 3; ++a) {
      aos[7 * j + a] = (double)B.o[a][slot] * dx;
      aos[7 * j + 3 + a] = (double)B.v[a][slot];
   }
   aos[7 * j + 6] = w;
}

__global__ void k_f32_gather_records_f32(F32Buf B, const unsigned long long* slots, const unsigned* idx, long long n,
                                         float* rec) {
   const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (j >= n) return;
   const unsigned long long slot = slots[idx[j]];
   for (int a = 0; a < 3; ++a) {
      rec[6 * j + a] = B.o[a][slot];
      rec[6 * j + 3 + a] = B.v[a][slot];
   }
}

__global__ void k_f32_relayout(F32Buf from, const long long* fromBase, F32Buf to, const long long* toBase) {
   const long long S = blockIdx.x;
   const int c = from.cnt[S];
   const long long a0 = fromBase[S], b0 = toBase[S];
   for (int r = threadIdx.x; r < c; r += blockDim.x) {
      to.cell[b0 + r] = from.cell[a0 + r];
      for (int e = 0; e < 3; ++e) { to.o[e][b0 + r] = from.o[e][a0 + r]; to.v[e][b0 + r] = from.v[e][a0 + r]; }
   }
   if (threadIdx.x == 0) to.cnt[S] = c;
}

__global__ void k_weight_range(const double* aos, long long n, unsigned long long* mn, unsigned long long* mx) {
   __shared__ double slo[32], shi[32];
   double lo = 1e308, hi = 0.0;
   for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
      const double w = fabs(aos[7 * p + 6]);
      lo = fmin(lo, w);
      hi = fmax(hi, w);
   }
   for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
   }
   if ((threadIdx.x & 31) == 0) { slo[threadIdx.x >> 5] = lo; shi[threadIdx.x >> 5] = hi; }
   __syncthreads();
   if (threadIdx.x == 0) {
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { lo = fmin(lo, slo[w]); hi = fmax(hi, shi[w]); }
      atomicMin(mn, (unsigned long long)__double_as_longlong(lo));
      atomicMax(mx, (unsigned long long)__double_as_longlong(hi));
   }
}

__global__ void __launch_bounds__(DIAG_THREADS)
k_diag_particles_f32(F32Buf B, const long long* base, long long NS, double w, double* part) {
   __shared__ double sm[DIAG_THREADS];
   double v[DIAG_P] = {0, 0, 0, 0, 0, 0, 0, 0};
   for (long long S = blockIdx.x; S < NS; S += gridDim.x)
      for (int r = threadIdx.x; r < B.cnt[S]; r += blockDim.x) {
         double st[7];
         for (int e = 0; e < 3; ++e) { st[e] = 0.0; st[3 + e] = (double)B.v[e][base[S] + r]; }
         st[6] = w;
         particleTerms(st, v);
      }
   blockReduce(v, DIAG_P_MAX, sm, part + (long long)blockIdx.x * DIAG_P);
}

__global__ void k_diag_rhom_f32(F32Buf B, const long long* base, long long NS, double wm, double scale,
                                unsigned long long* lo, unsigned long long* hi) {
   for (long long S = blockIdx.x; S < NS; S += gridDim.x)
      for (int r = threadIdx.x; r < B.cnt[S]; r += blockDim.x) {
         const long long n = B.cell[base[S] + r];
         add128(lo + n, hi + n, wm, scale);
      }
}

}  // namespace rh
