// Learned denoiser of the charge/current moments (sm_100a): a 3-layer 3D
// convolutional network, 3x3x3 kernels, 16 channels (4 in, 4 out, residual),
// leaky ReLU between layers, on BF16 activations with FP32 accumulation on the
// tensor cores, forward and backward written here: the convolutions (forward
// and data gradient) on tcgen05.mma with the accumulators in tensor memory
// (k_dn_conv_tc), the weight gradient on mma.sync m16n8k16 (k_dn_wgrad).
//
// Activations are channels-last, 16 BF16 channels per voxel (32 B), voxel
// index v = i + nx (j + ny k); padded channels are zero. A convolution is an
// implicit GEMM: for a tile of 16 consecutive voxels (rows) and the 16 output
// channels (two n8 tiles), the K dimension runs over 27 taps x 16 input
// channels. Outside a non-periodic box the input is zero; periodic axes wrap.
//
// Parameters (FP32 master copy): per layer W[27][16 cin][16 cout] then b[16];
// tap t = (dx+1) + 3 (dy+1) + 9 (dz+1). Layer 0 uses cin < 4, layer 2 cout < 4;
// the other entries stay zero (their gradients are masked).
#pragma once

#include <cuda_bf16.h>
#include "rh_device.cuh"
#include "k_fast.cuh"

namespace rh {

constexpr int DN_C = 16;                  // channels (padded)
constexpr int DN_TAPS = 27;
constexpr int DN_LAYER = DN_TAPS * DN_C * DN_C + DN_C;   // floats per layer
constexpr int DN_PARAMS = 3 * DN_LAYER;
constexpr int DN_WARPS = 4;               // warps per block of the convolution kernels
constexpr int DN_WGRAD_VOX = 1024;        // voxels per block of the weight-gradient kernel
constexpr float DN_LEAK = 0.125f;         // slope of the leaky ReLU below zero

struct DnGrid {
   int nx, ny, nz;
   int per[3];
   long long N;
};

__device__ inline unsigned packBf16(float lo, float hi) {
   const __nv_bfloat16 a = __float2bfloat16_rn(lo), b = __float2bfloat16_rn(hi);
   return (unsigned)__bfloat16_as_ushort(a) | ((unsigned)__bfloat16_as_ushort(b) << 16);
}
__device__ inline float bf16lo(unsigned u) { return __bfloat162float(__ushort_as_bfloat16((unsigned short)(u & 0xffffu))); }
__device__ inline float bf16hi(unsigned u) { return __bfloat162float(__ushort_as_bfloat16((unsigned short)(u >> 16))); }

__device__ inline void mma16816(float c[4], const unsigned a[4], unsigned b0, unsigned b1) {
   asm volatile(
       "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
       : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
       : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// (i, j, k) of voxel v (v < N < 2^31), -1 in i when v is outside
struct DnPos { int i, j, k; };
__device__ inline DnPos dnDecode(const DnGrid& g, long long v) {
   DnPos p;
   if (v < 0 || v >= g.N) { p.i = -1; p.j = 0; p.k = 0; return p; }
   const unsigned u = (unsigned)v, nx = (unsigned)g.nx, ny = (unsigned)g.ny;
   const unsigned r = u / nx;
   p.i = (int)(u - r * nx);
   p.k = (int)(r / ny);
   p.j = (int)(r - (unsigned)p.k * ny);
   return p;
}
// neighbour of a decoded voxel at tap t (sign sgn), -1 outside
__device__ inline int dnNb(const DnGrid& g, DnPos p, int t, int sgn) {
   if (p.i < 0) return -1;
   int i = p.i + sgn * (t % 3 - 1), j = p.j + sgn * ((t / 3) % 3 - 1), k = p.k + sgn * (t / 9 - 1);
   if (i < 0 || i >= g.nx) { if (!g.per[0]) return -1; i = i < 0 ? i + g.nx : i - g.nx; }
   if (j < 0 || j >= g.ny) { if (!g.per[1]) return -1; j = j < 0 ? j + g.ny : j - g.ny; }
   if (k < 0 || k >= g.nz) { if (!g.per[2]) return -1; k = k < 0 ? k + g.nz : k - g.nz; }
   return i + g.nx * (j + g.ny * k);
}

// the brick staging of a periodic or closed axis: coordinate x wrapped, or -1 outside
__device__ inline int dnWrap(int x, int n, int per) {
   if (x >= 0 && x < n) return x;
   if (!per) return -1;
   x %= n;
   return x < 0 ? x + n : x;
}

// inputs of the convolution read from the FP64 moments instead of an
// activation (the first layer inside a step), and written back in place (the
// last layer): rho (N) and J (3 x N, planar), their normalization and the rho floor
struct DnMoments {
   double* rho;    // N
   double* J;      // 3 x N
   double sr, sj, rsr, rsj, minRho;
   long long N;
   int vel;        // velocity form: the network sees rho and J / rho (sj the velocity scale)
   const unsigned char* keep;   // per cell, nonzero: the moments stay the deposit's (null: none)
};

// the factor that takes a current component to the network's input: 1 / sj,
// or in the velocity form 1 / (sj rho), the bulk velocity J / rho over its
// scale (0 where rho is not positive)
__host__ __device__ inline double dnJFactor(int vel, double rsj, double rho) {
   return vel ? (rho > 0.0 ? rsj / rho : 0.0) : rsj;
}

// ---- the convolution on the 5th-generation tensor cores (tcgen05) ----------------------------
// One convolution layer as an implicit GEMM on tcgen05.mma (kind::f16, BF16 x
// BF16 -> FP32 in tensor memory): the forward layer (bias, leaky ReLU, the
// residual or the moments written back in the epilogue, by `mode`), or
// TRANSPOSED, the data gradient with mirrored taps and W transposed, no bias,
// masked by the ReLU derivative.
//
// A block owns a column of 30 x 8 output voxels in (x, y) and TC_ZC of its
// z-slices. Input z-slices of 32 x-positions x 10 y-rows (one voxel of halo
// each side) stream through a ring of 4 slots in shared memory, one plane per
// 8-channel half with 16 bytes per voxel: any run of positions is a K-major,
// unswizzled UMMA operand (core matrices of 8 consecutive positions x 16 bytes,
// 128 B apart; the two channel halves one plane apart). An M-tile is 128
// consecutive positions = 4 x-rows of one slice. Positions 0 and 31 of a row
// are the x halo: their outputs are computed and dropped.
//
// The loop runs over input slices (input-stationary along z): input slice z'
// feeds output slices z' - 1, z', z' + 1 through the taps dz = +1, 0, -1 (the
// data gradient: -1, 0, +1). For each in-plane shift (sx, sy) one MMA of N = 48
// takes the slice shifted by sx + 32 sy positions as A and, as B, the three
// taps' 16 x 16 weights stacked along N (k_dn_bimage), so one read of A by the
// tensor core serves three output slices: per tile and input slice 9 MMAs of N
// 48 in place of 27 of N 16 per output slice, a third of the A operand reads
// from shared memory, which bound the narrow MMAs. The accumulators of output
// slice o live in column group (o + 2) mod 4 of the tile's 64 tensor-memory
// columns; where an MMA's three groups wrap past the last one it is issued as
// two (N 32 and N 16). A group is zeroed (tcgen05.st) after its slice's
// epilogue, before the first MMA of the output slice that reuses it.
//
// Per input slice: one thread issues the MMAs of both tiles and commits them
// to an mbarrier; the warps wait for the previous input slice's MMAs, which
// complete output slice z' - 2, take its accumulators through the epilogue
// (tcgen05.ld, warp w its 32 lanes = one x-row, one voxel per thread, 16
// channels), zero them, and copy input slice z' + 3 (cp.async) into the slot
// that slice z' - 1 held, while the tensor cores work on slice z'. Every
// mbarrier wait is bounded: on expiry the kernel raises RHGPU_DEVERR_DENOISER
// in `err`, stops issuing, waits (bounded again) for the last commit of the
// MMAs it issued, and still frees its tensor memory.
constexpr int TC_HX = 32, TC_BY = 8, TC_ZC = 8;
constexpr int TC_HY = TC_BY + 2;
constexpr int TC_BX = TC_HX - 2;                             // output voxels per x-row
constexpr int TC_SPOS = TC_HX * TC_HY;                       // positions of one staged slice
constexpr int TC_PAD = 1;                                    // zero positions before and after a slice
constexpr int TC_SLOT = (TC_SPOS + 2 * TC_PAD) * 16;         // bytes of one slice in one plane
constexpr int TC_RING = 4;                                   // slices in shared memory
// bytes per channel-half plane; the extra 16 put a position's two halves on different banks
constexpr int TC_PLANE = TC_RING * TC_SLOT + 16;
constexpr int TC_TILES = TC_BY / 4;                          // M-tiles of 128 positions per slice
constexpr int TC_GROUPS = 4;                                 // accumulator groups (output slices) per tile
constexpr int TC_TCOLS = TC_GROUPS * 16;                     // tensor-memory columns per tile
constexpr int TC_COLS = TC_TILES * TC_TCOLS;                 // tensor-memory columns of a block
constexpr int TC_NB = 3 * DN_C;                              // N of a stacked B image: 3 taps x 16 channels
constexpr int TC_QIMG = TC_NB * DN_C * 2;                    // bytes of one shift's B image
constexpr int TC_BIMG = 9 * TC_QIMG;                         // bytes of one layer's B images
constexpr int TC_THREADS = 128;
constexpr long long TC_WAIT_LIMIT = 1LL << 22;               // mbarrier polls before giving up
static_assert(TC_BIMG == DN_TAPS * DN_C * DN_C * 2, "the stacked images hold every tap once");
static_assert(TC_COLS == 128 && TC_BY % 4 == 0, "the allocation is a power of two; 4 blocks fill the 512 columns");
// a tile starts at row 1 + 4j; shifts reach one row and one position either side
static_assert(TC_HX * 0 - 1 >= -TC_PAD && TC_HX * (TC_HY - 1) + TC_HX - 1 + 1 < TC_SPOS + TC_PAD,
              "shifted operands stay inside the slice and its padding");

struct TcShared {
   alignas(16) unsigned char plane[2][TC_PLANE];
   alignas(16) unsigned char bimg[TC_BIMG];
   alignas(8) unsigned long long bar[2];
   unsigned tmemBase;
};
constexpr size_t TC_SMEM = sizeof(TcShared);
static_assert(TC_SMEM < (1u << 18), "operand addresses fit the descriptors' 14-bit start field");
static_assert(TC_PLANE % 16 == 0 && TC_QIMG % 16 == 0, "descriptor strides are multiples of 16 bytes");

// UMMA B images of one layer from FP32 W[27][16 cin][16 cout]. For each
// in-plane shift q = (sx + 1) + 3 (sy + 1), an N 48 x K 16 BF16 image, element
// (n, k) at byte q * TC_QIMG + (k / 8) * 768 + (n / 8) * 128 + (n % 8) * 16 +
// (k % 8) * 2 (K-major core matrices). N block b = n / 16 is the tap that takes
// input slice z' to output slice z' - 1 + b: forward the tap (sx, sy, 1 - b)
// with B(n, k) = W[t][k][n % 16]; the data gradient the tap (-sx, -sy, b - 1)
// with B(n, k) = W[t][n % 16][k]. Tap t = (dx + 1) + 3 (dy + 1) + 9 (dz + 1).
__global__ void k_dn_bimage(const float* W, __nv_bfloat16* img, int transposed);

__device__ __forceinline__ unsigned long long umma_desc(unsigned addr, unsigned lbo, unsigned sbo) {
   // start >> 4 [0,14), LBO >> 4 [16,30), SBO >> 4 [32,46), version 1 [46,48), no swizzle
   return (unsigned long long)((addr >> 4) & 0x3fffu) | ((unsigned long long)((lbo >> 4) & 0x3fffu) << 16) |
          ((unsigned long long)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}
// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N as given
__host__ __device__ constexpr unsigned tcIdesc(unsigned n) { return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24); }

__device__ __forceinline__ bool tcWait(unsigned bar, unsigned parity) {
   for (long long i = 0; i < TC_WAIT_LIMIT; ++i) {
      unsigned ok;
      asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                   "selp.b32 %0, 1, 0, P1;\n\t}\n"
                   : "=r"(ok)
                   : "r"(bar), "r"(parity)
                   : "memory");
      if (ok) return true;
   }
   return false;
}

// input slice zz into ring slot `slot`: 32 x 10 positions from (x0 - 1, y0 - 1),
// zeros outside a non-periodic box, wrapped on periodic axes
__device__ __forceinline__ void tcStageSlice(TcShared& sh, const DnGrid& g, const unsigned* in, const DnMoments& mom,
                                             int x0, int y0, int zz, int slot) {
   const int z = dnWrap(zz, g.nz, g.per[2]);
   for (int e = threadIdx.x; e < 2 * TC_SPOS; e += TC_THREADS) {
      const int p = e >> 1, h = e & 1;
      const int hx = p % TC_HX, hy = p / TC_HX;
      const int x = dnWrap(x0 - 1 + hx, g.nx, g.per[0]), y = dnWrap(y0 - 1 + hy, g.ny, g.per[1]);
      unsigned char* dst = &sh.plane[h][slot * TC_SLOT + 16 * (TC_PAD + p)];
      const bool ok = x >= 0 && y >= 0 && z >= 0;
      const long long gv = ok ? (long long)x + (long long)g.nx * ((long long)y + (long long)g.ny * z) : 0;
      if (in) {
         cpAsync16(dst, reinterpret_cast<const uint4*>(in) + (gv * 2 + h), ok ? 16 : 0);
      } else {
         uint4 v = make_uint4(0u, 0u, 0u, 0u);
         if (ok && h == 0) {
            const double r = mom.rho[gv], fj = dnJFactor(mom.vel, mom.rsj, r);
            v = make_uint4(packBf16((float)(r * mom.rsr), (float)(mom.J[gv] * fj)),
                           packBf16((float)(mom.J[mom.N + gv] * fj), (float)(mom.J[2 * mom.N + gv] * fj)), 0u, 0u);
         }
         *reinterpret_cast<uint4*>(dst) = v;
      }
   }
}

// the staged data (generic-proxy and cp.async writes) made visible to the
// tensor cores and to every thread; PENDING: cp.async groups of this thread
// that may stay in flight (the newest ones)
template <int PENDING>
__device__ __forceinline__ void tcPublish() {
   asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
   asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
   asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
   __syncthreads();
   asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

template <bool TRANSPOSED>
__device__ __forceinline__ void tcEpilogue(const DnGrid& g, unsigned tmem, int group, int x0, int y0, int z,
                                           const float* bias, int mode, unsigned* out, const unsigned* mask,
                                           float* out32, const float* res, const DnMoments& mom) {
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   unsigned rr[TC_TILES][16];
#pragma unroll
   for (int j = 0; j < TC_TILES; ++j) {
      unsigned* r = rr[j];
      const unsigned taddr = tmem + ((unsigned)(32 * warp) << 16) + (unsigned)(j * TC_TCOLS + 16 * group);
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
                   : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                     "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                   : "r"(taddr));
   }
   asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
   for (int j = 0; j < TC_TILES; ++j) {
      const unsigned* r = rr[j];
      const int x = x0 - 1 + lane, y = y0 + 4 * j + warp;
      if (lane < 1 || lane > TC_BX || x >= g.nx || y >= g.ny) continue;
      const long long v = (long long)x + (long long)g.nx * ((long long)y + (long long)g.ny * z);
      float c[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) c[k] = __uint_as_float(r[k]);
      if (!TRANSPOSED && bias)
#pragma unroll
         for (int k = 0; k < 16; ++k) c[k] += bias[k];
      if (mode == 0)
#pragma unroll
         for (int k = 0; k < 16; ++k) c[k] = c[k] > 0.f ? c[k] : DN_LEAK * c[k];
      if (mode == 2) {
         const uint4 m0 = reinterpret_cast<const uint4*>(mask)[v * 2], m1 = reinterpret_cast<const uint4*>(mask)[v * 2 + 1];
         const unsigned mw[8] = {m0.x, m0.y, m0.z, m0.w, m1.x, m1.y, m1.z, m1.w};
#pragma unroll
         for (int k = 0; k < 8; ++k) {
            if (!(bf16lo(mw[k]) > 0.f)) c[2 * k] *= DN_LEAK;
            if (!(bf16hi(mw[k]) > 0.f)) c[2 * k + 1] *= DN_LEAK;
         }
      }
      if (mode == 3) {
#pragma unroll
         for (int k = 0; k < 4; ++k) out32[v * 4 + k] = c[k] + res[v * 4 + k];
         continue;
      }
      if (mode == 4) {
         if (mom.keep && mom.keep[v]) continue;
         // the velocity form writes back J = rho' u' from the denoised density and velocity
         const double rin = mom.rho[v], fj = dnJFactor(mom.vel, mom.rsj, rin);
         double r0 = (double)(c[0] + (float)(rin * mom.rsr)) * mom.sr;
         if (r0 < mom.minRho) r0 = mom.minRho;
         double j0 = (double)(c[1] + (float)(mom.J[v] * fj)) * mom.sj;
         double j1 = (double)(c[2] + (float)(mom.J[mom.N + v] * fj)) * mom.sj;
         double j2 = (double)(c[3] + (float)(mom.J[2 * mom.N + v] * fj)) * mom.sj;
         if (mom.vel) { j0 *= r0; j1 *= r0; j2 *= r0; }
         mom.rho[v] = r0;
         mom.J[v] = j0;
         mom.J[mom.N + v] = j1;
         mom.J[2 * mom.N + v] = j2;
         continue;
      }
      uint4* o = reinterpret_cast<uint4*>(out) + v * 2;
      o[0] = make_uint4(packBf16(c[0], c[1]), packBf16(c[2], c[3]), packBf16(c[4], c[5]), packBf16(c[6], c[7]));
      o[1] = make_uint4(packBf16(c[8], c[9]), packBf16(c[10], c[11]), packBf16(c[12], c[13]), packBf16(c[14], c[15]));
   }
}

// zeros into 16 tensor-memory columns of this warp's 32 lanes
__device__ __forceinline__ void tcZero16(unsigned taddr) {
   asm volatile("tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};\n"
                ::"r"(taddr), "r"(0u)
                : "memory");
}

__device__ __forceinline__ void tcMma(unsigned d, unsigned long long ad, unsigned long long bd, unsigned idesc) {
   asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                :
                : "r"(d), "l"(ad), "l"(bd), "r"(idesc), "r"(1), "r"(0), "r"(0), "r"(0), "r"(0));
}

// the MMAs of one input slice (both tiles, 9 shifts): A from the slice's slot
// (descriptor words aHi:aLo), B from the stacked images (bHi:bLo), output
// slices z' - 1, z', z' + 1 into groups A0, A0 + 1, A0 + 2 (mod 4) of each tile
template <int A0>
__device__ __forceinline__ void tcIssue(unsigned tmem, unsigned aHi, unsigned aLo, unsigned bHi, unsigned bLo) {
#pragma unroll
   for (int j = 0; j < TC_TILES; ++j) {
      const unsigned dT = tmem + (unsigned)(j * TC_TCOLS);
#pragma unroll
      for (int q = 0; q < 9; ++q) {
         const int sx = q % 3 - 1, sy = q / 3 - 1;
         const int pos = TC_PAD + TC_HX * (1 + 4 * j + sy) + sx;   // compile-time, 16-byte units
         const unsigned long long ad = ((unsigned long long)aHi << 32) | (aLo + (unsigned)pos);
         const unsigned bq = bLo + (unsigned)(q * (TC_QIMG >> 4));
         const unsigned long long b0 = ((unsigned long long)bHi << 32) | bq;
         if (A0 <= 1) {
            tcMma(dT + 16u * A0, ad, b0, tcIdesc(48));
         } else if (A0 == 2) {   // groups 2, 3 | 0
            tcMma(dT + 32u, ad, b0, tcIdesc(32));
            tcMma(dT, ad, ((unsigned long long)bHi << 32) | (bq + (512u >> 4)), tcIdesc(16));
         } else {                // groups 3 | 0, 1
            tcMma(dT + 48u, ad, b0, tcIdesc(16));
            tcMma(dT, ad, ((unsigned long long)bHi << 32) | (bq + (256u >> 4)), tcIdesc(32));
         }
      }
   }
}

template <bool TRANSPOSED>
__global__ void __launch_bounds__(TC_THREADS)
k_dn_conv_tc(DnGrid g, const unsigned* in, const __nv_bfloat16* bimg, const float* bias, int mode, unsigned* out,
             const unsigned* mask, float* out32, const float* res, DnMoments mom, unsigned* err) {
   extern __shared__ __align__(16) unsigned char tcSmemRaw[];
   TcShared& sh = *reinterpret_cast<TcShared*>(tcSmemRaw);
   const int tid = threadIdx.x, warp = tid >> 5;
   const int x0 = blockIdx.x * TC_BX, y0 = blockIdx.y * TC_BY, z0 = blockIdx.z * TC_ZC;
   const int nzc = min(TC_ZC, g.nz - z0);
   const int nin = nzc + 2;   // input slices z0 - 1 .. z0 + nzc; input i is slice z0 - 1 + i, in slot i % 4
   const unsigned planeBase = (unsigned)__cvta_generic_to_shared(&sh.plane[0][0]);
   const unsigned bimgBase = (unsigned)__cvta_generic_to_shared(&sh.bimg[0]);
   // tensor memory (one warp), mbarriers (one thread)
   if (warp == 0) {
      const unsigned dst = (unsigned)__cvta_generic_to_shared(&sh.tmemBase);
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(TC_COLS));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
   }
   if (tid == 0) {
      for (int j = 0; j < 2; ++j) {
         const unsigned b = (unsigned)__cvta_generic_to_shared(&sh.bar[j]);
         asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(b), "r"(1));
      }
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   // the weights, the slices' zero padding, and input slices 0-2 (slots 0-2)
   {
      const uint4* src = reinterpret_cast<const uint4*>(bimg);
      for (int e = tid; e < TC_BIMG / 16; e += TC_THREADS) cpAsync16(&sh.bimg[16 * e], src + e, 16);
      for (int e = tid; e < 2 * TC_RING * 2 * TC_PAD; e += TC_THREADS) {
         const int h = e / (TC_RING * 2 * TC_PAD), q = e % (TC_RING * 2 * TC_PAD);
         const int slot = q / (2 * TC_PAD), k = q % (2 * TC_PAD);
         const int pos = k < TC_PAD ? k : TC_PAD + TC_SPOS + (k - TC_PAD);
         *reinterpret_cast<uint4*>(&sh.plane[h][slot * TC_SLOT + 16 * pos]) = make_uint4(0u, 0u, 0u, 0u);
      }
      for (int k = 0; k < 3; ++k) tcStageSlice(sh, g, in, mom, x0, y0, z0 - 1 + k, k);
      cpAsyncCommit();
   }
   tcPublish<0>();
   const unsigned tmem = sh.tmemBase;
   const unsigned lanes = (unsigned)(32 * warp) << 16;
   // every accumulator group starts at zero
#pragma unroll
   for (int c = 0; c < TC_COLS; c += 16) tcZero16(tmem + lanes + (unsigned)c);
   asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
   tcPublish<0>();
   // descriptors: the low word holds the start address >> 4 (14 bits, no carry into LBO for
   // shared addresses below 256 KB), so an operand's descriptor is a base plus a constant
   const unsigned long long a0 = umma_desc(planeBase, TC_PLANE, 128);
   const unsigned long long b0 = umma_desc(bimgBase, TC_NB * 16, 128);
   const unsigned aHi = (unsigned)(a0 >> 32), aLo0 = (unsigned)a0, bHi = (unsigned)(b0 >> 32), bLo = (unsigned)b0;
   bool timedOut = false;
   int lastCommit = -1;   // the input slice whose commit covers every MMA issued so far
   for (int i = 0; i < nin && !timedOut; ++i) {
      lastCommit = i;
      if (tid == 0) {
         const unsigned aLo = aLo0 + (unsigned)((i % TC_RING) * (TC_SLOT >> 4));
         switch (i & 3) {   // output slice o of input i's N block b is i - 2 + b, in group (o + 2) & 3
         case 0: tcIssue<0>(tmem, aHi, aLo, bHi, bLo); break;
         case 1: tcIssue<1>(tmem, aHi, aLo, bHi, bLo); break;
         case 2: tcIssue<2>(tmem, aHi, aLo, bHi, bLo); break;
         default: tcIssue<3>(tmem, aHi, aLo, bHi, bLo); break;
         }
         const unsigned b = (unsigned)__cvta_generic_to_shared(&sh.bar[i & 1]);
         asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(b) : "memory");
      }
      if (i > 0) {
         // input i - 1's MMAs done: output slice i - 3 is complete, slot (i - 1) % 4 is free
         const int pb = (i - 1) & 1;
         // warp-uniform outcome: the epilogue's tcgen05.ld / .st are warp-collective
         if (!__all_sync(0xffffffffu, tcWait((unsigned)__cvta_generic_to_shared(&sh.bar[pb]), (unsigned)(((i - 1) >> 1) & 1)))) {
            timedOut = true;
         } else {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (i + 3 < nin) tcStageSlice(sh, g, in, mom, x0, y0, z0 + 2 + i, (i + 3) % TC_RING);
            const int o = i - 3, grp = (i + 3) & 3;   // (o + 2) & 3
            if (o >= 0) tcEpilogue<TRANSPOSED>(g, tmem, grp, x0, y0, z0 + o, bias, mode, out, mask, out32, res, mom);
            if (i + 1 < nin) {   // the group's next output slice, o + 4, takes its first MMA from input i + 1
#pragma unroll
               for (int j = 0; j < TC_TILES; ++j) tcZero16(tmem + lanes + (unsigned)(j * TC_TCOLS + 16 * grp));
               asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
            }
         }
      } else if (3 < nin) {
         tcStageSlice(sh, g, in, mom, x0, y0, z0 + 2, 3);   // slot 3 is still free
      }
      cpAsyncCommit();   // one group per iteration, empty or not
      timedOut = __syncthreads_or(timedOut);
      tcPublish<1>();    // the copies issued now may stay in flight: their slice is read 3 iterations on
   }
   if (!timedOut) {
      const int lb = (nin - 1) & 1;
      if (!__all_sync(0xffffffffu, tcWait((unsigned)__cvta_generic_to_shared(&sh.bar[lb]), (unsigned)(((nin - 1) >> 1) & 1)))) {
         timedOut = true;
      } else {
         asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
         tcEpilogue<TRANSPOSED>(g, tmem, (nzc + 1) & 3, x0, y0, z0 + nzc - 1, bias, mode, out, mask, out32, res, mom);
      }
   }
   if (timedOut) {
      // the MMAs issued so far may still run: wait (bounded again) for the last commit
      // before the tensor memory is freed
      if (tid == 0) raiseError(err, RHGPU_DEVERR_DENOISER);
      if (lastCommit >= 0)
         tcWait((unsigned)__cvta_generic_to_shared(&sh.bar[lastCommit & 1]), (unsigned)((lastCommit >> 1) & 1));
   }
   asm volatile("cp.async.wait_group 0;\n" ::: "memory");
   asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
   __syncthreads();
   if (warp == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_COLS));
   }
}

// Weight gradient of one layer: dW[t][ci][co] = sum_v X[nb(v,t)][ci] dY[v][co].
// Block (blockIdx.x, tap blockIdx.y) covers DN_WGRAD_VOX voxels, each warp a
// quarter in k-steps of 16 voxels: C[ci][co] += A[ci][vox] B[vox][co] (mma),
// then the 4 warps are added in order and the block's partial row written.
__global__ void __launch_bounds__(32 * DN_WARPS)
k_dn_wgrad(DnGrid g, const unsigned* X, const unsigned* dY, float* part);

// bias gradient partials: sum over the block's voxels of dY[v][co]
__global__ void k_dn_bgrad(DnGrid g, const unsigned* dY, float* part);

// sum of the block partials in block order -> grad (n values per row)
__global__ void k_dn_reduce_rows(const float* part, long long rows, int n, float* out);

// MSE loss over the 4 real channels and its gradient (BF16, 16 channels)
// border: voxels within `border` of a non-periodic face are left out of the
// loss (zero gradient): for training on crops of a larger grid, whose outer
// voxels see the zero halo of the crop instead of their neighbours
__global__ void k_dn_loss(DnGrid g, const float* pred, const float* target, double inv, unsigned* dY, double* part,
                          int border);

// Adam (Kingma & Ba 2015) on the FP32 master parameters; mask 0 keeps padding at zero
__global__ void k_dn_adam(float* p, const float* gr, float* m, float* v, const unsigned char* mask, int n, float lr,
                          float b1, float b2, float eps, float c1, float c2);

// normalized FP32 copy (N x 4) of planar FP64 moments: rho / sr and J / sj as
// products with the reciprocals rsr = 1 / sr, rsj = 1 / sj (velocity form:
// J / (sj rho), dnJFactor)
__global__ void k_dn_norm(long long N, const double* rho, const double* J, double rsr, double rsj, int vel, float* out);

// FP32 normalized moments (N x 4) -> BF16 network input (16 channels)
__global__ void k_dn_res_to_act(long long N, const float* res, unsigned* act);

// CIC deposit of one in `factor` particles of the fast-path store (index in the
// segment = offset mod factor), weights times factor, into FP64 sums (4 x N,
// atomics: training data only). One block per segment.
__global__ void k_dn_subsample_deposit(GridInfo g, FastGeom fg, SegBuf B, const long long* base, double q, int factor,
                                       int offset, double* acc);
// one crop of a normalized (N x 4) moment grid: the crop's voxel (x, y, z) is
// the full grid's (x0 + x, y0 + y, z0 + z)
__global__ void k_dn_crop(const float* full, int fnx, int fny, DnGrid c, int x0, int y0, int z0, float* out);

// the deposit's finalize on the subsample sums: /dV, rho clamp, then normalized
// FP32 (N x 4) as k_dn_norm
__global__ void k_dn_subsample_finish(long long N, const double* acc, double dV, double minRho, double rsr, double rsj,
                                      int vel, float* out);

// squared-error sums for the relative L2 errors of one pair: per block
// {sum |a-t|^2 rho, sum |t|^2 rho, sum |a-t|^2 J, sum |t|^2 J}
__global__ void k_dn_err(long long N, const float* a, const float* t, double* part);

}  // namespace rh
