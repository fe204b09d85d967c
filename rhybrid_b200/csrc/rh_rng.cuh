// Counter-based random numbers for the particle sources: Philox-4x32-10
// (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC'11). Each draw is a pure function of a
// 128-bit counter and a 64-bit key, so GPU threads draw independent streams
// in any order and a run is reproducible.
#pragma once

#include <stdint.h>

namespace rh {

struct Philox4 {
   uint32_t v[4];
};

// 10 rounds of the Philox-4x32 bijection (multipliers and Weyl key increments of the paper)
__host__ __device__ inline Philox4 philox4x32(const uint32_t ctr[4], const uint32_t key[2]) {
   uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
   uint32_t k0 = key[0], k1 = key[1];
   for (int r = 0; r < 10; ++r) {
      const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
      const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
      const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
      const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
      c0 = hi1 ^ c1 ^ k0;
      c1 = lo1;
      c2 = hi0 ^ c3 ^ k1;
      c3 = lo0;
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
   }
   Philox4 o;
   o.v[0] = c0; o.v[1] = c1; o.v[2] = c2; o.v[3] = c3;
   return o;
}

// a stream of uniform doubles in [0, 1) for one (key, stream id): draws 4 words
// per counter increment, 53-bit doubles from two words each
struct RngStream {
   uint32_t key[2];
   uint32_t ctr[4];
   Philox4 buf;
   int used;   // doubles taken from buf (2 per block)

   __host__ __device__ void init(uint64_t seed, uint32_t a, uint32_t b, uint32_t c) {
      key[0] = (uint32_t)seed;
      key[1] = (uint32_t)(seed >> 32);
      ctr[0] = 0; ctr[1] = a; ctr[2] = b; ctr[3] = c;
      used = 2;
   }
   __host__ __device__ double uniform() {
      if (used == 2) {
         buf = philox4x32(ctr, key);
         ++ctr[0];
         used = 0;
      }
      const uint32_t hi = buf.v[2 * used], lo = buf.v[2 * used + 1];
      ++used;
      // (27 high bits, 26 low bits) / 2^53
      return ((double)(hi >> 5) * 67108864.0 + (double)(lo >> 6)) * (1.0 / 9007199254740992.0);
   }
};

}  // namespace rh
