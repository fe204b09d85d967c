// Definitions of the kernels declared in k_util.cuh.
#include "k_util.cuh"

namespace rh {

// per cell: slot range from the counts, cell index of every slot
__global__ void k_counts_in(long long N, const uint32_t* counts, long long* cnt64, int* alive) {
   const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (b < N) { cnt64[b] = counts[b]; alive[b] = (int)counts[b]; }
   if (b == N) cnt64[N] = 0;
}
__global__ void k_fill_pcell(long long N, const long long* start, int* pcell) {
   const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (b >= N) return;
   for (long long p = start[b]; p < start[b + 1]; ++p) pcell[p] = (int)b;
}

__global__ void k_iota(unsigned* v, long long n) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t < n) v[t] = (unsigned)t;
}
__global__ void k_int_to64(const int* in, long long n, long long* out) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t < n) out[t] = in[t];
   if (t == n) out[n] = 0;
}

__global__ void k_fill_u32(unsigned* a, long long n, unsigned v) {
   const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (p < n) a[p] = v;
}
__global__ void k_gather_u32(const unsigned* src, const unsigned* idx, long long n, unsigned* dst) {
   const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (p < n) dst[p] = src[idx[p]];
}

}  // namespace rh
