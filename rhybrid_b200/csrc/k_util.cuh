// Small kernels of the particle storage's bookkeeping (upload, download,
// migration), shared by the particle paths.
#pragma once

#include "rh_device.cuh"

namespace rh {

// per cell: the count as 64 bits and as the alive count; cnt64[N] = 0
__global__ void k_counts_in(long long N, const uint32_t* counts, long long* cnt64, int* alive);
// cell index of every slot, from the cells' first slots
__global__ void k_fill_pcell(long long N, const long long* start, int* pcell);
// v[t] = t
__global__ void k_iota(unsigned* v, long long n);
// out[t] = in[t] as 64 bits, out[n] = 0
__global__ void k_int_to64(const int* in, long long n, long long* out);
// a[p] = v
__global__ void k_fill_u32(unsigned* a, long long n, unsigned v);
// dst[p] = src[idx[p]]
__global__ void k_gather_u32(const unsigned* src, const unsigned* idx, long long n, unsigned* dst);

}  // namespace rh
