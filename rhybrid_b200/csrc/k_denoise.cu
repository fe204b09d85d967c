// Definitions of the kernels declared in k_denoise.cuh (each declaration there says
// what its kernel does); the template kernels stay in the header.
#include "k_denoise.cuh"

namespace rh {

__global__ void k_dn_bimage(const float* W, __nv_bfloat16* img, int transposed) {
   const int e = blockIdx.x * blockDim.x + threadIdx.x;   // (q, n, k)
   if (e >= 9 * TC_NB * DN_C) return;
   const int k = e % DN_C, n = (e / DN_C) % TC_NB, q = e / (DN_C * TC_NB);
   const int b = n / DN_C, c = n % DN_C;
   const int sx = q % 3 - 1, sy = q / 3 - 1;
   const int dx = transposed ? -sx : sx, dy = transposed ? -sy : sy, dz = transposed ? b - 1 : 1 - b;
   const int t = (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1);
   const float w = transposed ? W[(t * DN_C + c) * DN_C + k] : W[(t * DN_C + k) * DN_C + c];
   img[q * (TC_QIMG / 2) + (k / 8) * (TC_NB * 8) + (n / 8) * 64 + (n % 8) * 8 + (k % 8)] = __float2bfloat16_rn(w);
}

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

__global__ void k_dn_reduce_rows(const float* part, long long rows, int n, float* out) {
   const int e = blockIdx.x * blockDim.x + threadIdx.x;
   if (e >= n) return;
   float a = 0.f;
   for (long long r = 0; r < rows; ++r) a += part[r * n + e];
   out[e] = a;
}

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

__global__ void k_dn_adam(float* p, const float* gr, float* m, float* v, const unsigned char* mask, int n, float lr,
                          float b1, float b2, float eps, float c1, float c2) {
   const int e = blockIdx.x * blockDim.x + threadIdx.x;
   if (e >= n || !mask[e]) return;
   const float g = gr[e];
   m[e] = b1 * m[e] + (1.f - b1) * g;
   v[e] = b2 * v[e] + (1.f - b2) * g * g;
   p[e] -= lr * (m[e] / c1) / (sqrtf(v[e] / c2) + eps);
}

__global__ void k_dn_norm(long long N, const double* rho, const double* J, double rsr, double rsj, int vel, float* out) {
   const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (v >= N) return;
   const double fj = dnJFactor(vel, rsj, rho[v]);
   out[v * 4] = (float)(rho[v] * rsr);
   for (int l = 0; l < 3; ++l) out[v * 4 + 1 + l] = (float)(J[l * N + v] * fj);
}

__global__ void k_dn_res_to_act(long long N, const float* res, unsigned* act) {
   const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (v >= N) return;
   act[v * 8 + 0] = packBf16(res[v * 4], res[v * 4 + 1]);
   act[v * 8 + 1] = packBf16(res[v * 4 + 2], res[v * 4 + 3]);
   for (int u = 2; u < 8; ++u) act[v * 8 + u] = 0u;
}

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

__global__ void k_dn_crop(const float* full, int fnx, int fny, DnGrid c, int x0, int y0, int z0, float* out) {
   const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (v >= c.N) return;
   const int x = (int)(v % c.nx), y = (int)((v / c.nx) % c.ny), z = (int)(v / ((long long)c.nx * c.ny));
   const long long f = (long long)(x0 + x) + (long long)fnx * ((long long)(y0 + y) + (long long)fny * (z0 + z));
   const float4 q = *reinterpret_cast<const float4*>(full + 4 * f);
   *reinterpret_cast<float4*>(out + 4 * v) = q;
}

__global__ void k_dn_subsample_finish(long long N, const double* acc, double dV, double minRho, double rsr, double rsj,
                                      int vel, float* out) {
   const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (v >= N) return;
   double r = acc[v] / dV;
   if (r < minRho) r = minRho;
   const double fj = dnJFactor(vel, rsj, r);
   out[v * 4] = (float)(r * rsr);
   for (int l = 0; l < 3; ++l) out[v * 4 + 1 + l] = (float)(acc[(1 + l) * N + v] / dV * fj);
}

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
