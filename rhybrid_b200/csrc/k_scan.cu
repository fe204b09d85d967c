// Definitions of the kernels declared in k_scan.cuh (each declaration there says
// what its kernel does); the template kernels stay in the header.
#include "k_scan.cuh"

namespace rh {

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tile(const long long* in, long long* out, long long n,
                                                            long long* sums) {
   __shared__ long long warpTot[SCAN_THREADS / 32];
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
   const long long base = (long long)blockIdx.x * SCAN_TILE + (long long)tid * SCAN_PER;
   long long v[SCAN_PER];
   long long t = 0;
#pragma unroll
   for (int k = 0; k < SCAN_PER; ++k) {
      v[k] = base + k < n ? in[base + k] : 0;
      t += v[k];
   }
   // inclusive scan of the thread totals within the warp, then over the warps
   long long x = t;
#pragma unroll
   for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
   }
   if (lane == 31) warpTot[warp] = x;
   __syncthreads();
   long long before = 0, all = 0;
#pragma unroll
   for (int w = 0; w < SCAN_THREADS / 32; ++w) {
      const long long wt = warpTot[w];
      if (w < warp) before += wt;
      all += wt;
   }
   long long run = before + x - t;   // exclusive prefix of this thread's first value
#pragma unroll
   for (int k = 0; k < SCAN_PER; ++k) {
      if (base + k < n) out[base + k] = run;
      run += v[k];
   }
   if (tid == 0 && sums) sums[blockIdx.x] = all;
}

__global__ void k_scan_add(long long* out, long long n, const long long* offs) {
   const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (i < n) out[i] += offs[i / SCAN_TILE];
}

__global__ void k_max_int(const int* a, long long n, int* mx) {
   __shared__ int wmax[8];
   int m = 0;
   for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      m = max(m, a[i]);
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
   if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
   __syncthreads();
   if (threadIdx.x == 0) {
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = max(m, wmax[w]);
      atomicMax(mx, m);
   }
}

}  // namespace rh
