// Definitions of the kernels declared in k_fast.cuh (each declaration there says
// what its kernel does); the template kernels stay in the header.
#include "k_fast.cuh"

namespace rh {

__global__ void k_fast_mover_deposit(GridInfo g, FastGeom fg, FastSpecies FS, FastBufs fb, long long n) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= n) return;
   const Mover& M = fb.movers[t];
   if (!(M.lx & MOVER_DEPOSIT)) return;
   moverAdd128<true>(g, fg, FS, M, fb.MMlo, fb.MMhi, fb.scaleR, fb.scaleJ, fb.touched);
}

__global__ void k_fast_fold_boundary(GridInfo g, FastGeom fg, FastBufs fb) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   const long long nrows = fg.nrows;
   if (t >= 16 * nrows * fg.nseg) return;
   const int m = (int)(t & 3);
   const long long e = t >> 2;                    // (qq, row, gseg)
   const int gseg = (int)(e % fg.nseg);
   const long long qr = e / fg.nseg;              // qq * nrows + row
   if (!(g.per[0] ? fg.nseg > 1 : gseg >= 1)) return;
   const int x = g.per[0] ? gseg * SEG : gseg * SEG - 1;
   if (x >= g.nx) return;
   double* rp = fb.RP + (qr * g.nx + x) * 4 + m;
   *rp = *rp + fb.RPB[e * 4 + m];
}

__global__ void k_fast_mig_place(FastSpecies FS, long long NS, long long nb, const Mover* mv, const unsigned* order,
                                 const unsigned* bkt, const long long* off, long long n) {
   const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (q >= n) return;
   const long long b = bkt[q];
   if (b >= nb) return;
   const int s = (int)(b / NS);
   const long long S = b % NS;
   const SegSpecies& SS = FS.st[s];
   const long long pos = SS.base[S] + SS.nxt.cnt[S] + (q - off[b]);
   const Mover& M = mv[order[q]];
   for (int e = 0; e < 7; ++e) SS.nxt.a[e][pos] = M.s[e];
   SS.nxt.lx[pos] = (unsigned char)(M.lx & 0xff);
}

__global__ void k_mig_large_list(const int* inc, long long nb, unsigned* large, int* nlarge) {
   const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (b < nb && inc[b] > MIG_SMALL) large[atomicAdd(nlarge, 1)] = (unsigned)b;
}

__global__ void k_fast_seg_of(GridInfo g, FastGeom fg, const double* aos, const int* pcell, long long n,
                              unsigned* key, unsigned char* lx) {
   const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (p >= n) return;
   const int c = pcell[p];
   const int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
   const double* st = aos + 7 * p;
   const int ux = dualU(i + halfS(st[0], g.dx) - 1, g.nx, g.per[0]);
   const int uy = dualU(j + halfS(st[1], g.dx) - 1, g.ny, g.per[1]);
   const int uz = dualU(k + halfS(st[2], g.dx) - 1, g.nz, g.per[2]);
   const int gs = ux / SEG;
   key[p] = (unsigned)(((long long)uy + (long long)fg.nd[1] * uz) * fg.nseg + gs);
   lx[p] = (unsigned char)(ux - gs * SEG);
}

__global__ void k_sorted_bounds(const unsigned* key, long long n, long long nkeys, long long* first) {
   const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (j > n) return;
   const long long lo = j == 0 ? 0 : (long long)key[j - 1] + 1;
   const long long hi = j == n ? nkeys : (long long)key[j];
   for (long long k = lo; k <= hi; ++k) first[k] = j;
}

__global__ void k_bounds_counts(const long long* first, long long nkeys, int* cnt) {
   const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (k < nkeys) cnt[k] = (int)(first[k + 1] - first[k]);
}

__global__ void k_fast_capacity(long long NS, const int* cnt, const int* extra, long long* cap) {
   const long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (d < NS) {
      const long long c = (long long)cnt[d] + (extra ? extra[d] : 0);
      cap[d] = c + max(32LL, c / 4);
   } else if (d == NS) {
      cap[d] = 0;
   }
}

__global__ void k_fast_scatter_sorted(const double* aos, const unsigned char* lxIn, const unsigned* key,
                                      const unsigned* idx, long long n, const long long* first, SegBuf B,
                                      const long long* base) {
   const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (j >= n) return;
   const unsigned S = key[j];
   const long long slot = base[S] + (j - first[S]);
   const unsigned src = idx[j];
   for (int a = 0; a < 7; ++a) B.a[a][slot] = aos[7LL * src + a];
   B.lx[slot] = lxIn[src];
}

__global__ void k_fast_cell_keys(GridInfo g, FastGeom fg, SegBuf B, const long long* base, const long long* first,
                                 unsigned* key, unsigned long long* slots) {
   const long long S = blockIdx.x;
   const long long row = S / fg.nseg;
   const int gs = (int)(S % fg.nseg);
   const int uy = (int)(row % fg.nd[1]), uz = (int)(row / fg.nd[1]);
   const int c = B.cnt[S];
   for (int r = threadIdx.x; r < c; r += blockDim.x) {
      const long long slot = base[S] + r;
      const int u = gs * SEG + B.lx[slot];
      int ci = dualB(u, g.per[0]) + 1 - halfS(B.a[0][slot], g.dx);
      int cj = dualB(uy, g.per[1]) + 1 - halfS(B.a[1][slot], g.dx);
      int ck = dualB(uz, g.per[2]) + 1 - halfS(B.a[2][slot], g.dx);
      wrapc(ci, g.nx, 1); wrapc(cj, g.ny, 1); wrapc(ck, g.nz, 1);
      key[first[S] + r] = (unsigned)cidx(g, ci, cj, ck);
      slots[first[S] + r] = (unsigned long long)slot;
   }
}

__global__ void k_fast_gather_records(SegBuf B, const unsigned long long* slots, const unsigned* idx, long long n,
                                      double* aos) {
   const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (j >= n) return;
   const unsigned long long slot = slots[idx[j]];
   for (int a = 0; a < 7; ++a) aos[7 * j + a] = B.a[a][slot];
}

__global__ void k_fast_relayout(SegBuf from, const long long* fromBase, SegBuf to, const long long* toBase) {
   const long long S = blockIdx.x;
   const int c = from.cnt[S];
   const long long a0 = fromBase[S], b0 = toBase[S];
   for (int r = threadIdx.x; r < c; r += blockDim.x) {
      for (int e = 0; e < 7; ++e) to.a[e][b0 + r] = from.a[e][a0 + r];
      to.lx[b0 + r] = from.lx[a0 + r];
   }
   if (threadIdx.x == 0) to.cnt[S] = c;
}

__global__ void k_fast_max_abs_w(SegBuf B, const long long* base, unsigned long long* out) {
   __shared__ double sm[32];
   const long long S = blockIdx.x;
   const int c = B.cnt[S];
   double m = 0.0;
   for (int r = threadIdx.x; r < c; r += blockDim.x) m = fmax(m, fabs(B.a[6][base[S] + r]));
   for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
   if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
   __syncthreads();
   if (threadIdx.x == 0) {
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, sm[w]);
      if (m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
   }
}

}  // namespace rh
