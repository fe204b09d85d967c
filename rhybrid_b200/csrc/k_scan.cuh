// Exclusive prefix sums of 64-bit counts and the maximum of 32-bit counts:
// the bookkeeping of the particle storage (cell and segment layouts, the
// migration's arrival offsets). Integer sums, so any order gives the same
// result; these replace library scans on the per-step path.
//
// A scan of n values in place: tiles of SCAN_TILE values (SCAN_THREADS threads
// x SCAN_PER consecutive values each) are scanned by one block each, their
// totals written to a sums array; the sums array is scanned the same way
// (recursively, until one tile holds it), and a last pass adds each tile's
// offset. Every thread reads its own values before it writes them, so in and
// out may be the same array.
#pragma once

#include "rh_device.cuh"

namespace rh {

constexpr int SCAN_THREADS = 256, SCAN_PER = 8, SCAN_TILE = SCAN_THREADS * SCAN_PER;

// per tile: out[i] = sum of in[tile start .. i - 1]; sums[tile] = tile total
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tile(const long long* in, long long* out, long long n,
                                                            long long* sums);

// out[i] += offs[tile of i]
__global__ void k_scan_add(long long* out, long long n, const long long* offs);

// *mx = max(*mx, a[0..n)) (*mx cleared by the caller)
__global__ void k_max_int(const int* a, long long n, int* mx);

}  // namespace rh
