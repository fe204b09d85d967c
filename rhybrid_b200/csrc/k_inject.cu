// Definitions of the kernels declared in k_inject.cuh (each declaration there says
// what its kernel does); the template kernels stay in the header.
#include "k_inject.cuh"

namespace rh {

__global__ void k_inject_select(InjDev J, long long step, int* list, int* count) {
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   const int lane = threadIdx.x & 31;
   bool any = false;
   if (t < J.ncells) {
      RngStream r;
      r.init(J.seed, (uint32_t)step, (uint32_t)(step >> 32), (uint32_t)t);
      const double x = J.rates[t];
      if (x > 0) {
         int n = (int)floor(x);
         if (r.uniform() < x - n) ++n;
         any = n > 0;
      }
   }
   const unsigned m = __ballot_sync(0xffffffffu, any);
   int base = 0;
   if (lane == 0 && m) base = atomicAdd(count, __popc(m));
   base = __shfl_sync(0xffffffffu, base, 0);
   if (any) list[base + __popc(m & ((1u << lane) - 1u))] = t;
}

__global__ void k_np_eval(NeutralProfile P, long long n, const double* xyz, double* out) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= n) return;
   out[t] = neutralDensityAt(P, xyz[3 * t], xyz[3 * t + 1], xyz[3 * t + 2]);
}

__global__ void k_exo_density(GridInfo g, NeutralProfile P, double R2exo, unsigned long long seed, double* out) {
   const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (n >= g.N) return;
   const int i = (int)(n % g.nx), j = (int)((n / g.nx) % g.ny), k = (int)(n / ((long long)g.nx * g.ny));
   const double xc = g.x_min + (i + 0.5) * g.dx, yc = g.y_min + (j + 0.5) * g.dx, zc = g.z_min + (k + 0.5) * g.dx;
   RngStream r;
   r.init(seed, 0xE705u, (uint32_t)n, (uint32_t)(n >> 32));
   double sum = 0.0;
   for (int s = 0; s < INJ_MC_POINTS; ++s) {
      const double x = xc + (1.0 - INJ_EPS_CELL) * g.dx * (r.uniform() - 0.5);
      const double y = yc + (1.0 - INJ_EPS_CELL) * g.dx * (r.uniform() - 0.5);
      const double z = zc + (1.0 - INJ_EPS_CELL) * g.dx * (r.uniform() - 0.5);
      const double r2 = x * x + y * y + z * z;
      if (r2 < R2exo) continue;
      sum += neutralDensityAt(P, x, y, z);
   }
   out[n] = sum / INJ_MC_POINTS * g.dV;
}

__global__ void k_chapman_shell(GridInfo g, double R, double noon, double night, double H, unsigned long long seed,
                                double* out) {
   const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (n >= g.N) return;
   const int i = (int)(n % g.nx), j = (int)((n / g.nx) % g.ny), k = (int)(n / ((long long)g.nx * g.ny));
   const double xc = g.x_min + (i + 0.5) * g.dx, yc = g.y_min + (j + 0.5) * g.dx, zc = g.z_min + (k + 0.5) * g.dx;
   RngStream r;
   r.init(seed, 0xC4A9u, (uint32_t)n, (uint32_t)(n >> 32));
   double inside = 0.0;
   for (int s = 0; s < INJ_MC_POINTS; ++s) {
      const double x = xc + (1.0 - INJ_EPS_CELL) * g.dx * (r.uniform() - 0.5);
      const double y = yc + (1.0 - INJ_EPS_CELL) * g.dx * (r.uniform() - 0.5);
      const double z = zc + (1.0 - INJ_EPS_CELL) * g.dx * (r.uniform() - 0.5);
      const double a0 = chapmanAccept(x, y, z, R, noon, night, H);
      if (r.uniform() < a0) inside += 1.0;
   }
   out[n] = inside < 10 ? 0.0 : inside;   // cells with fewer than 10 kept points emit nothing
}

__global__ void k_iono_shell(GridInfo g, double R, int profile, double noon, double night, unsigned long long seed,
                             double* out) {
   const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (n >= g.N) return;
   const int i = (int)(n % g.nx), j = (int)((n / g.nx) % g.ny), k = (int)(n / ((long long)g.nx * g.ny));
   const double xc = g.x_min + (i + 0.5) * g.dx, yc = g.y_min + (j + 0.5) * g.dx, zc = g.z_min + (k + 0.5) * g.dx;
   const double lo[3] = {xc - 0.5 * g.dx, yc - 0.5 * g.dx, zc - 0.5 * g.dx};
   const double hi[3] = {xc + 0.5 * g.dx, yc + 0.5 * g.dx, zc + 0.5 * g.dx};
   RngStream r;
   r.init(seed, 0x10705u, (uint32_t)n, (uint32_t)(n >> 32));
   double inside = 0.0;
   for (int s = 0; s < INJ_MC_POINTS; ++s) {
      double p[3];
      p[0] = xc + (1.0 - INJ_EPS_CELL) * g.dx * (r.uniform() - 0.5);
      p[1] = yc + (1.0 - INJ_EPS_CELL) * g.dx * (r.uniform() - 0.5);
      p[2] = zc + (1.0 - INJ_EPS_CELL) * g.dx * (r.uniform() - 0.5);
      const double norm = R / sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
      bool in = true;
      for (int a = 0; a < 3; ++a) {
         p[a] *= norm;
         in = in && p[a] > lo[a] && p[a] < hi[a];
      }
      if (in) inside += 1.0;
   }
   out[n] = inside * ionoFactor(profile, noon, night, xc, yc, zc);
}

}  // namespace rh
