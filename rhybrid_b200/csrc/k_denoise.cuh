// Learned denoiser of the charge/current moments (sm_100a): a 3-layer 3D
// convolutional network, 3x3x3 kernels, 16 channels (4 in, 4 out, residual),
// leaky ReLU between layers, on BF16 activations with FP32 accumulation on the
// tensor cores (mma.sync m16n8k16 bf16, A fragments by ldmatrix from a
// shared-memory brick), forward and backward written here.
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

// B fragments of one layer for mma.m16n8k16 (.col): [tap][ntile][lane][2] u32,
// b0 = W[k = 2q, 2q+1][n = g], b1 = W[k = 2q+8, 2q+9][n = g] (g = lane/4, q = lane%4)
constexpr int DN_FRAG = DN_TAPS * 2 * 32 * 2;   // u32 per layer

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

// B fragments from FP32 weights W[27][16][16] (cin, cout); transposed: use W[t][cout][cin]
__global__ void k_dn_frags(const float* W, unsigned* frag, int transposed) {
   const int e = blockIdx.x * blockDim.x + threadIdx.x;   // (t, nt, lane)
   if (e >= DN_TAPS * 2 * 32) return;
   const int lane = e & 31, nt = (e >> 5) & 1, t = e >> 6;
   const int g = lane >> 2, q = lane & 3;
   const int n = nt * 8 + g;
   auto w = [&](int k) {
      return transposed ? W[(t * DN_C + n) * DN_C + k] : W[(t * DN_C + k) * DN_C + n];
   };
   frag[e * 2 + 0] = packBf16(w(2 * q), w(2 * q + 1));
   frag[e * 2 + 1] = packBf16(w(2 * q + 8), w(2 * q + 9));
}

// One convolution layer (transposed: the data-gradient convolution, taps
// mirrored and W transposed, no bias). A block covers a brick of DN_BX x DN_BY
// x DN_BZ output voxels: the input brick with a one-voxel halo (zero outside a
// non-periodic box, wrapped on periodic axes) is staged in shared memory with
// 16-byte copies, and each warp runs 4 x-rows of 16 voxels (M) x 16 output
// channels (two n8 tiles) over the 27 taps (K = 16 input channels per tap),
// the A fragments read with ldmatrix. Voxel lv = hx + DN_HX (hy + DN_HY hz) of
// the brick keeps its two 16-byte channel halves h at 16-byte slots
// 2 lv + (h ^ bit 2 of hx): the 8 rows of an ldmatrix phase (8 consecutive hx)
// fall on 8 different bank groups, and a tap's y/z shift keeps each lane's
// swizzle, so the taps' addresses are a per-lane x part plus constants.
// mode 0: out = lrelu(conv + b) as BF16; mode 1: out = conv + b as BF16;
// mode 2: out = conv * (mask > 0 ? 1 : 1/8) as BF16 (leaky ReLU backward, mask
// = that layer's input activation); mode 3: FP32 out (4 channels) = conv + b +
// residual (the first 4 channels of res, FP32); mode 4: the moments mom.rho,
// mom.J (FP64, planar) overwritten in place by (conv + b + their normalized
// FP32 values) times the scales, rho clamped at mom.minRho. With `in` null,
// the input is read from the moments mom: channels 0-3 = BF16(FP32(rho rsr)),
// BF16(FP32(J rsj)), the rest zero (rsr = 1 / sr, rsj = 1 / sj, as k_dn_norm).
struct DnMoments {
   double* rho;    // N
   double* J;      // 3 x N
   double sr, sj, rsr, rsj, minRho;
   long long N;
};
constexpr int DN_BX = 16, DN_BY = 8, DN_BZ = 4;                 // output brick
constexpr int DN_HX = DN_BX + 2, DN_HY = DN_BY + 2, DN_HZ = DN_BZ + 2;
constexpr int DN_HV = DN_HX * DN_HY * DN_HZ;                    // staged voxels
constexpr int DN_TWARPS = 8;                                    // warps of k_dn_conv
constexpr int DN_ROWS = DN_BY * DN_BZ / DN_TWARPS;              // x-rows per warp
constexpr int DN_STAGE = (2 * DN_HV + 32 * DN_TWARPS - 1) / (32 * DN_TWARPS);   // 16-byte copies per thread
static_assert(DN_BX == 16 && DN_BY * DN_BZ % DN_TWARPS == 0, "one m16 tile per brick x-row");

__device__ inline int dnSlot(int hx, int lv, int h) { return 2 * lv + (h ^ ((hx >> 2) & 1)); }
__device__ inline int dnWrap(int x, int n, int per) {
   if (x >= 0 && x < n) return x;
   if (!per) return -1;
   x %= n;
   return x < 0 ? x + n : x;
}

template <bool TRANSPOSED>
__global__ void __launch_bounds__(32 * DN_TWARPS)
k_dn_conv(DnGrid g, const unsigned* in, const unsigned* frag, const float* bias, int mode, unsigned* out,
          const unsigned* mask, float* out32, const float* res, DnMoments mom) {
   constexpr bool transposed = TRANSPOSED;
   __shared__ __align__(16) uint4 sin[2 * DN_HV];
   __shared__ __align__(16) unsigned sfrag[DN_FRAG];
   const int tid = threadIdx.x;
   const int x0 = blockIdx.x * DN_BX, y0 = blockIdx.y * DN_BY, z0 = blockIdx.z * DN_BZ;
   {
      const uint4* f4 = reinterpret_cast<const uint4*>(frag);
      uint4* s4 = reinterpret_cast<uint4*>(sfrag);
      for (int e = tid; e < DN_FRAG / 4; e += blockDim.x) s4[e] = f4[e];
      uint4 v[DN_STAGE];
      int slot[DN_STAGE];
#pragma unroll
      for (int k = 0; k < DN_STAGE; ++k) {
         const int e = tid + 32 * DN_TWARPS * k;
         v[k] = make_uint4(0u, 0u, 0u, 0u);
         slot[k] = -1;
         if (e >= 2 * DN_HV) continue;
         const int lv = e >> 1, h = e & 1;
         const int hx = lv % DN_HX, r = lv / DN_HX, hy = r % DN_HY, hz = r / DN_HY;
         slot[k] = dnSlot(hx, lv, h);
         const int x = dnWrap(x0 - 1 + hx, g.nx, g.per[0]), y = dnWrap(y0 - 1 + hy, g.ny, g.per[1]),
                   z = dnWrap(z0 - 1 + hz, g.nz, g.per[2]);
         if (x < 0 || y < 0 || z < 0) continue;
         const long long gv = (long long)x + (long long)g.nx * ((long long)y + (long long)g.ny * z);
         if (!in) {
            if (h == 0)
               v[k] = make_uint4(packBf16((float)(mom.rho[gv] * mom.rsr), (float)(mom.J[gv] * mom.rsj)),
                                 packBf16((float)(mom.J[mom.N + gv] * mom.rsj), (float)(mom.J[2 * mom.N + gv] * mom.rsj)),
                                 0u, 0u);
         } else {
            v[k] = reinterpret_cast<const uint4*>(in)[gv * 2 + h];
         }
      }
#pragma unroll
      for (int k = 0; k < DN_STAGE; ++k)
         if (slot[k] >= 0) sin[slot[k]] = v[k];
   }
   __syncthreads();
   const int lane = tid & 31, warp = tid >> 5;
   const int gq = lane >> 2, q = lane & 3;
   const int lr = lane & 15, lh = lane >> 4;   // ldmatrix: this lane's row and channel half
   const unsigned sbase = (unsigned)__cvta_generic_to_shared(sin);
   constexpr int sgn = TRANSPOSED ? -1 : 1;
   // byte offsets: x part of this lane at hx = lr + dx + 1 (dx = -1, 0, 1), and of each row
   unsigned xo[3];
#pragma unroll
   for (int d = 0; d < 3; ++d) {
      const int hx = lr + d;
      xo[d] = sbase + 16u * (unsigned)(2 * hx + (lh ^ ((hx >> 2) & 1)));
   }
   unsigned ro[DN_ROWS];
#pragma unroll
   for (int r = 0; r < DN_ROWS; ++r) {
      const int row = warp * DN_ROWS + r, ry = row % DN_BY, rz = row / DN_BY;
      ro[r] = 32u * (unsigned)(DN_HX * ((ry + 1) + DN_HY * (rz + 1)));
   }
   float c[DN_ROWS][2][4];
#pragma unroll
   for (int r = 0; r < DN_ROWS; ++r)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) c[r][nt][0] = c[r][nt][1] = c[r][nt][2] = c[r][nt][3] = 0.f;
#pragma unroll
   for (int t = 0; t < DN_TAPS; ++t) {
      const int dx = sgn * (t % 3 - 1), dy = sgn * ((t / 3) % 3 - 1), dz = sgn * (t / 9 - 1);
      const int tyz = 32 * DN_HX * (dy + DN_HY * dz);   // byte offset of the tap's y/z shift
      const unsigned* f = sfrag + (t * 2) * 64;
      const uint2 bf0 = *reinterpret_cast<const uint2*>(f + lane * 2);
      const uint2 bf1 = *reinterpret_cast<const uint2*>(f + 64 + lane * 2);
#pragma unroll
      for (int r = 0; r < DN_ROWS; ++r) {
         const unsigned addr = xo[dx + 1] + ro[r] + (unsigned)tyz;
         unsigned a[4];
         asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                      : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
                      : "r"(addr));
         mma16816(c[r][0], a, bf0.x, bf0.y);
         mma16816(c[r][1], a, bf1.x, bf1.y);
      }
   }
   // c[r][nt][0,1]: voxel x = gq, channels nt*8 + 2q, +1; c[r][nt][2,3]: x = gq + 8
#pragma unroll
   for (int r = 0; r < DN_ROWS; ++r) {
      const int row = warp * DN_ROWS + r, y = y0 + row % DN_BY, z = z0 + row / DN_BY;
      if (y >= g.ny || z >= g.nz) continue;
      const long long rowv = (long long)g.nx * ((long long)y + (long long)g.ny * z);
      const bool oka = x0 + gq < g.nx, okb = x0 + gq + 8 < g.nx;
      const long long va = rowv + x0 + gq, vb = va + 8;
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) {
         const int ch = nt * 8 + 2 * q;
         float x0v = c[r][nt][0], x1v = c[r][nt][1], x2v = c[r][nt][2], x3v = c[r][nt][3];
         if (!transposed && bias) { x0v += bias[ch]; x1v += bias[ch + 1]; x2v += bias[ch]; x3v += bias[ch + 1]; }
         if (mode == 0) {
            x0v = x0v > 0.f ? x0v : DN_LEAK * x0v; x1v = x1v > 0.f ? x1v : DN_LEAK * x1v;
            x2v = x2v > 0.f ? x2v : DN_LEAK * x2v; x3v = x3v > 0.f ? x3v : DN_LEAK * x3v;
         }
         if (mode == 2) {
            // leaky ReLU backward: the activation's sign is its input's sign
            if (oka) { const unsigned m = mask[va * 8 + nt * 4 + q]; if (!(bf16lo(m) > 0.f)) x0v *= DN_LEAK; if (!(bf16hi(m) > 0.f)) x1v *= DN_LEAK; }
            if (okb) { const unsigned m = mask[vb * 8 + nt * 4 + q]; if (!(bf16lo(m) > 0.f)) x2v *= DN_LEAK; if (!(bf16hi(m) > 0.f)) x3v *= DN_LEAK; }
         }
         if (mode == 3) {
            if (nt == 0 && q < 2) {
               if (oka) { out32[va * 4 + ch] = x0v + res[va * 4 + ch]; out32[va * 4 + ch + 1] = x1v + res[va * 4 + ch + 1]; }
               if (okb) { out32[vb * 4 + ch] = x2v + res[vb * 4 + ch]; out32[vb * 4 + ch + 1] = x3v + res[vb * 4 + ch + 1]; }
            }
            continue;
         }
         if (mode == 4) {
            // channels ch, ch + 1 of voxels va, vb: (rho, Jx) for q = 0, (Jy, Jz) for q = 1
            if (nt == 0 && q < 2) {
               double* p0 = q == 0 ? mom.rho : mom.J + mom.N;
               double* p1 = q == 0 ? mom.J : mom.J + 2 * mom.N;
               const double s0 = q == 0 ? mom.sr : mom.sj, rs0 = q == 0 ? mom.rsr : mom.rsj;
               auto put = [&](long long v, float y0, float y1) {
                  double r0 = (double)(y0 + (float)(p0[v] * rs0)) * s0;
                  const double r1 = (double)(y1 + (float)(p1[v] * mom.rsj)) * mom.sj;
                  if (q == 0 && r0 < mom.minRho) r0 = mom.minRho;
                  p0[v] = r0;
                  p1[v] = r1;
               };
               if (oka) put(va, x0v, x1v);
               if (okb) put(vb, x2v, x3v);
            }
            continue;
         }
         if (oka) out[va * 8 + nt * 4 + q] = packBf16(x0v, x1v);
         if (okb) out[vb * 8 + nt * 4 + q] = packBf16(x2v, x3v);
      }
   }
}

// Weight gradient of one layer: dW[t][ci][co] = sum_v X[nb(v,t)][ci] dY[v][co].
// Block (blockIdx.x, tap blockIdx.y) covers DN_WGRAD_VOX voxels, each warp a
// quarter in k-steps of 16 voxels: C[ci][co] += A[ci][vox] B[vox][co] (mma),
// then the 4 warps are added in order and the block's partial row written.
__global__ void __launch_bounds__(32 * DN_WARPS)
k_dn_wgrad(DnGrid g, const unsigned* X, const unsigned* dY, float* part) {
   __shared__ float sacc[DN_WARPS][DN_C * DN_C];
   const unsigned short* x16 = reinterpret_cast<const unsigned short*>(X);
   const unsigned short* y16 = reinterpret_cast<const unsigned short*>(dY);
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   const int gq = lane >> 2, q = lane & 3;
   const int t = blockIdx.y;
   float c[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
   const long long vw = (long long)blockIdx.x * DN_WGRAD_VOX + warp * (DN_WGRAD_VOX / DN_WARPS);
   auto yv = [&](long long v, int ch) -> unsigned { return (v < g.N) ? (unsigned)y16[v * DN_C + ch] : 0u; };
   for (int ks = 0; ks < DN_WGRAD_VOX / DN_WARPS; ks += 16) {
      const long long vk = vw + ks;
      if (vk >= g.N) break;
      // the input voxels (at tap t) of this thread's four k indices
      const int n0 = dnNb(g, dnDecode(g, vk + 2 * q), t, 1), n1 = dnNb(g, dnDecode(g, vk + 2 * q + 1), t, 1);
      const int n8 = dnNb(g, dnDecode(g, vk + 2 * q + 8), t, 1), n9 = dnNb(g, dnDecode(g, vk + 2 * q + 9), t, 1);
      auto xv = [&](int n, int ch) -> unsigned { return n >= 0 ? (unsigned)x16[(long long)n * DN_C + ch] : 0u; };
      unsigned a[4];
      a[0] = xv(n0, gq) | (xv(n1, gq) << 16);
      a[1] = xv(n0, gq + 8) | (xv(n1, gq + 8) << 16);
      a[2] = xv(n8, gq) | (xv(n9, gq) << 16);
      a[3] = xv(n8, gq + 8) | (xv(n9, gq + 8) << 16);
      for (int nt = 0; nt < 2; ++nt) {
         const int co = nt * 8 + gq;
         const unsigned b0 = yv(vk + 2 * q, co) | (yv(vk + 2 * q + 1, co) << 16);
         const unsigned b1 = yv(vk + 2 * q + 8, co) | (yv(vk + 2 * q + 9, co) << 16);
         mma16816(c[nt], a, b0, b1);
      }
   }
   // c[nt][0,1]: ci = gq, co = nt*8 + 2q, +1; c[nt][2,3]: ci = gq + 8
   for (int nt = 0; nt < 2; ++nt) {
      const int co = nt * 8 + 2 * q;
      sacc[warp][gq * DN_C + co] = c[nt][0];
      sacc[warp][gq * DN_C + co + 1] = c[nt][1];
      sacc[warp][(gq + 8) * DN_C + co] = c[nt][2];
      sacc[warp][(gq + 8) * DN_C + co + 1] = c[nt][3];
   }
   __syncthreads();
   for (int e = threadIdx.x; e < DN_C * DN_C; e += blockDim.x) {
      float a = 0.f;
      for (int w = 0; w < DN_WARPS; ++w) a += sacc[w][e];
      part[((long long)blockIdx.x * DN_TAPS + t) * DN_C * DN_C + e] = a;
   }
}

// bias gradient partials: sum over the block's voxels of dY[v][co]
__global__ void k_dn_bgrad(DnGrid g, const unsigned* dY, float* part) {
   __shared__ float s[256][DN_C];
   const unsigned short* y16 = reinterpret_cast<const unsigned short*>(dY);
   float a[DN_C];
   for (int c = 0; c < DN_C; ++c) a[c] = 0.f;
   for (long long v = (long long)blockIdx.x * DN_WGRAD_VOX + threadIdx.x;
        v < min(g.N, (long long)(blockIdx.x + 1) * DN_WGRAD_VOX); v += blockDim.x)
      for (int c = 0; c < DN_C; ++c) a[c] += __bfloat162float(__ushort_as_bfloat16(y16[v * DN_C + c]));
   for (int c = 0; c < DN_C; ++c) s[threadIdx.x][c] = a[c];
   __syncthreads();
   if (threadIdx.x < DN_C) {
      float t = 0.f;
      for (int r = 0; r < (int)blockDim.x; ++r) t += s[r][threadIdx.x];
      part[(long long)blockIdx.x * DN_C + threadIdx.x] = t;
   }
}

// sum of the block partials in block order -> grad (n values per row)
__global__ void k_dn_reduce_rows(const float* part, long long rows, int n, float* out) {
   const int e = blockIdx.x * blockDim.x + threadIdx.x;
   if (e >= n) return;
   float a = 0.f;
   for (long long r = 0; r < rows; ++r) a += part[r * n + e];
   out[e] = a;
}

// MSE loss over the 4 real channels and its gradient (BF16, 16 channels)
// border: voxels within `border` of a non-periodic face are left out of the
// loss (zero gradient): for training on crops of a larger grid, whose outer
// voxels see the zero halo of the crop instead of their neighbours
__global__ void k_dn_loss(DnGrid g, const float* pred, const float* target, double inv, unsigned* dY, double* part,
                          int border) {
   __shared__ double s[256];
   double l = 0.0;
   for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < g.N; v += (long long)gridDim.x * blockDim.x) {
      const int x = (int)(v % g.nx), y = (int)((v / g.nx) % g.ny), z = (int)(v / ((long long)g.nx * g.ny));
      const bool in = (g.per[0] || (x >= border && x < g.nx - border)) && (g.per[1] || (y >= border && y < g.ny - border)) &&
                      (g.per[2] || (z >= border && z < g.nz - border));
      float d[4];
      for (int c = 0; c < 4; ++c) {
         d[c] = in ? pred[v * 4 + c] - target[v * 4 + c] : 0.0f;
         l += (double)d[c] * d[c];
      }
      const float k = (float)(2.0 * inv);
      dY[v * 8 + 0] = packBf16(k * d[0], k * d[1]);
      dY[v * 8 + 1] = packBf16(k * d[2], k * d[3]);
      for (int u = 2; u < 8; ++u) dY[v * 8 + u] = 0u;
   }
   s[threadIdx.x] = l;
   __syncthreads();
   if (threadIdx.x == 0) {
      double a = 0.0;
      for (int r = 0; r < (int)blockDim.x; ++r) a += s[r];
      part[blockIdx.x] = a;
   }
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters; mask 0 keeps padding at zero
__global__ void k_dn_adam(float* p, const float* gr, float* m, float* v, const unsigned char* mask, int n, float lr,
                          float b1, float b2, float eps, float c1, float c2) {
   const int e = blockIdx.x * blockDim.x + threadIdx.x;
   if (e >= n || !mask[e]) return;
   const float g = gr[e];
   m[e] = b1 * m[e] + (1.f - b1) * g;
   v[e] = b2 * v[e] + (1.f - b2) * g * g;
   p[e] -= lr * (m[e] / c1) / (sqrtf(v[e] / c2) + eps);
}

// planar FP64 moments (rho N, J 3N) -> normalized FP32 residual copy (N x 4) + BF16 input (16 channels)
// normalized FP32 copy (N x 4) of planar FP64 moments: rho / sr and J / sj as
// products with the reciprocals rsr = 1 / sr, rsj = 1 / sj
__global__ void k_dn_norm(long long N, const double* rho, const double* J, double rsr, double rsj, float* out) {
   const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (v >= N) return;
   out[v * 4] = (float)(rho[v] * rsr);
   for (int l = 0; l < 3; ++l) out[v * 4 + 1 + l] = (float)(J[l * N + v] * rsj);
}

// FP32 normalized moments (N x 4) -> BF16 network input (16 channels)
__global__ void k_dn_res_to_act(long long N, const float* res, unsigned* act) {
   const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (v >= N) return;
   act[v * 8 + 0] = packBf16(res[v * 4], res[v * 4 + 1]);
   act[v * 8 + 1] = packBf16(res[v * 4 + 2], res[v * 4 + 3]);
   for (int u = 2; u < 8; ++u) act[v * 8 + u] = 0u;
}

// CIC deposit of one in `factor` particles of the fast-path store (index in the
// segment = offset mod factor), weights times factor, into FP64 sums (4 x N,
// atomics: training data only). One block per segment.
__global__ void k_dn_subsample_deposit(GridInfo g, FastGeom fg, SegBuf B, const long long* base, double q, int factor,
                                       int offset, double* acc) {
   const long long S = blockIdx.x;
   const long long row = S / fg.nseg;
   const int gs = (int)(S % fg.nseg);
   const int uy = (int)(row % fg.nd[1]), uz = (int)(row / fg.nd[1]);
   const long long N = g.N;
   for (int r = threadIdx.x; r < B.cnt[S]; r += blockDim.x) {
      if (r % factor != offset) continue;
      const long long slot = base[S] + r;
      double st[7];
      for (int a = 0; a < 7; ++a) st[a] = B.a[a][slot];
      const int u = gs * SEG + B.lx[slot];
      const int bx = dualB(u, g.per[0]), by = dualB(uy, g.per[1]), bz = dualB(uz, g.per[2]);
      double w8[8];
      cicWeightsDx(st[0], st[1], st[2], st[6] * q * factor, g, w8);
      for (int o = 0; o < 8; ++o) {
         int x = bx + (o & 1), y = by + ((o >> 1) & 1), z = bz + ((o >> 2) & 1);
         if (!wrapc(x, g.nx, g.per[0]) || !wrapc(y, g.ny, g.per[1]) || !wrapc(z, g.nz, g.per[2])) continue;
         const long long c = cidx(g, x, y, z);
         atomicAdd(&acc[c], w8[o]);
         for (int l = 0; l < 3; ++l) atomicAdd(&acc[(1 + l) * N + c], w8[o] * st[3 + l]);
      }
   }
}
// the deposit's finalize on the subsample sums: /dV, rho clamp, then normalized FP32 (N x 4)
// one crop of a normalized (N x 4) moment grid: the crop's voxel (x, y, z) is
// the full grid's (x0 + x, y0 + y, z0 + z)
__global__ void k_dn_crop(const float* full, int fnx, int fny, DnGrid c, int x0, int y0, int z0, float* out) {
   const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (v >= c.N) return;
   const int x = (int)(v % c.nx), y = (int)((v / c.nx) % c.ny), z = (int)(v / ((long long)c.nx * c.ny));
   const long long f = (long long)(x0 + x) + (long long)fnx * ((long long)(y0 + y) + (long long)fny * (z0 + z));
   const float4 q = *reinterpret_cast<const float4*>(full + 4 * f);
   *reinterpret_cast<float4*>(out + 4 * v) = q;
}

__global__ void k_dn_subsample_finish(long long N, const double* acc, double dV, double minRho, double rsr, double rsj,
                                      float* out) {
   const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (v >= N) return;
   double r = acc[v] / dV;
   if (r < minRho) r = minRho;
   out[v * 4] = (float)(r * rsr);
   for (int l = 0; l < 3; ++l) out[v * 4 + 1 + l] = (float)(acc[(1 + l) * N + v] / dV * rsj);
}

// squared-error sums for the relative L2 errors of one pair: per block
// {sum |a-t|^2 rho, sum |t|^2 rho, sum |a-t|^2 J, sum |t|^2 J}
__global__ void k_dn_err(long long N, const float* a, const float* t, double* part) {
   __shared__ double s[256][4];
   double e[4] = {0, 0, 0, 0};
   for (long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x; v < N; v += (long long)gridDim.x * blockDim.x) {
      const double d0 = (double)a[v * 4] - t[v * 4];
      e[0] += d0 * d0;
      e[1] += (double)t[v * 4] * t[v * 4];
      for (int l = 1; l < 4; ++l) {
         const double d = (double)a[v * 4 + l] - t[v * 4 + l];
         e[2] += d * d;
         e[3] += (double)t[v * 4 + l] * t[v * 4 + l];
      }
   }
   for (int q = 0; q < 4; ++q) s[threadIdx.x][q] = e[q];
   __syncthreads();
   if (threadIdx.x < 4) {
      double a2 = 0.0;
      for (int r = 0; r < (int)blockDim.x; ++r) a2 += s[r][threadIdx.x];
      part[blockIdx.x * 4 + threadIdx.x] = a2;
   }
}

}  // namespace rh
