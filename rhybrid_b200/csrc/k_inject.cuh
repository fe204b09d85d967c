// Particle sources (sm_100a): the reference's solar wind, flow and exosphere
// injectors (particle_injector.cpp:517-730 InjectorSolarWind, :734-945
// InjectorFlow, :1491-1840 InjectorExosphere),
// run after the boundary conditions of every step (user.cpp:119-122), on the
// GPU. One thread per injection cell draws its particles from a counter-based
// stream (Philox, keyed by the injector's seed, the step and the cell), so the
// result does not depend on thread order. New particles enter the step's mover
// list as placement-only movers (no deposit in this step, as in the reference)
// with keys after every real mover, and the migration stores them.
#pragma once

#include "rh_device.cuh"
#include "rh_rng.cuh"
#include "k_fast.cuh"
#include "k_f32.cuh"

namespace rh {

constexpr int INJ_SOLARWIND = 1;   // RHGPU_INJECT_SOLARWIND
constexpr int INJ_FLOW = 2;        // RHGPU_INJECT_FLOW
constexpr int INJ_EXOSPHERE = 3;   // RHGPU_INJECT_EXOSPHERE
constexpr int INJ_IONOSPHERE = 4;  // RHGPU_INJECT_IONOSPHERE
constexpr int INJ_CHAPMAN = 5;     // RHGPU_INJECT_CHAPMAN_IONOSPHERE
constexpr double INJ_EPS_CELL = 1.0e-4;   // margin of a cell's random points (particle_injector.cpp:31)
constexpr int INJ_MC_POINTS = 1000;       // Monte Carlo points per cell (particle_injector.cpp:33)
constexpr int INJ_MAX_TRIES = 1000;   // bound of every rejection loop (failures raise a device error)

struct InjDev {
   int species;
   int type;
   int wall;             // solar wind: axis * 2 + (1 if it enters at the positive wall)
   int ncells;           // injection cells
   const int* cells;     // their cell indices
   double U;             // solar wind speed |U|
   double vel[3];        // flow bulk velocity
   double vth;           // thermal speed sqrt(k T / m)
   double perCellPerDt;  // macroparticles per injection cell per step
   double w;             // macroparticle weight
   unsigned long long seed;
   long long keyBase;    // first mover key source id (above every real segment)
   const double* rates;  // exosphere: expected macroparticles per step of each injection cell
   double R2exo;         // exosphere: squared exobase radius
   double R, noon, night, H;   // Chapman ionosphere: emission radius, day/night factors, scale height
   const int* list;            // rate-based sources: the cells that draw particles this step (k_inject_select), or null
   const int* listCount;
};

// rate-based sources (exosphere, ionospheres): draw every injection cell's
// count as k_inject does and list the cells that get at least one particle,
// so that k_inject runs over those only (most cells draw none)
__global__ void k_inject_select(InjDev J, long long step, int* list, int* count);

// neutral density of an exospheric profile at radius r (neutral_profiles.h:36-87):
// 1 ChamberlainH, 2 ChamberlainT (a[i] = G M m / (k_B T0[i])), 3 Exponential, 4 PowerLaw
struct NeutralProfile {
   int type, n;
   double r0;
   double n0[4], b[4];   // b: H0, a, H0 or k0 per component
};
__device__ inline double neutralDensity(const NeutralProfile& P, double r) {
   double d = 0.0;
   for (int i = 0; i < P.n; ++i) {
      if (P.type == 1 || P.type == 2) d += P.n0[i] * exp(-P.b[i] * (1.0 / P.r0 - 1.0 / r));
      else if (P.type == 3) d += P.n0[i] * exp(-(r - P.r0) / P.b[i]);
      else d += P.n0[i] * pow(P.r0 / r, P.b[i]);
   }
   return d;
}

// Planetary neutral models of neutral_profiles.h:79-214. Corsair's planetary
// constants are not vendored with the reference; these are the IAU nominal
// radii and masses and 15.999 u for oxygen.
constexpr double NP_VENUS_RADIUS = 6051.8e3;
constexpr double NP_VENUS_MASS = 4.8675e24;
constexpr double NP_MASS_OXYGEN = 15.999 * 1.66053906660e-27;
constexpr double NP_MERCURY_RADIUS = 2439.7e3;

// solar zenith angle (the Sun on +x)
__device__ inline double sza(double x, double r) { return acos(x / r); }

// Venus hydrogen: thermal day/night Chamberlain-like terms blended by the solar
// zenith angle, plus the hot corona (exp(a1 r + a2 + a3 / r)) at noon, the
// terminator and midnight (neutral_profiles.h:79-112)
__device__ inline double venusHydrogen(double x, double y, double z) {
   const double r = sqrt(x * x + y * y + z * z);
   const double chi = sza(x, r);
   const double exoR = NP_VENUS_RADIUS + 170e3;
   const double GM = RHGPU_GRAVITY * NP_VENUS_MASS;
   const double bDay = GM * RHGPU_MASS_PROTON / (RHGPU_BOLTZMANN * 285);
   const double bNight = GM * RHGPU_MASS_PROTON / (RHGPU_BOLTZMANN * 110);
   const double nDay = 1.32e11 * exp(-bDay * (1 / exoR - 1.0 / r));
   const double nNight = 2.59e12 * exp(-bNight * (1.0 / exoR - 1.0 / r));
   const double thermal = (1.0 - (chi / M_PI)) * nDay + (chi / M_PI) * nNight;
   // hot corona fits: (a1 [1/m], a2, a3 [m]) at noon, terminator, midnight
   const double hot[3][3] = {{-6.2625e-5 / 1e3, 15.4817, 3.6414e4 * 1e3},
                             {-8.4607e-5 / 1e3, 15.9944, 2.9743e4 * 1e3},
                             {-6.2309e-5 / 1e3, 15.2723, 4.3781e4 * 1e3}};
   double h[3];
   for (int q = 0; q < 3; ++q) h[q] = exp(hot[q][0] * r + hot[q][1] + hot[q][2] / r);
   const double u = chi / (M_PI / 2);
   const double hotN = chi <= M_PI / 2 ? (1.0 - u) * h[0] + u * h[1] : (1.0 - (u - 1)) * h[1] + (u - 1) * h[2];
   return thermal + hotN;
}

// Venus oxygen: day and night Chamberlain-like profiles from their base radii,
// blended by the solar zenith angle (neutral_profiles.h:114-138)
__device__ inline double venusOxygen(double x, double y, double z) {
   const double r = sqrt(x * x + y * y + z * z);
   const double chi = sza(x, r);
   const double GMm = RHGPU_GRAVITY * NP_VENUS_MASS * NP_MASS_OXYGEN;
   const double r0Day = NP_VENUS_RADIUS + 200e3, r0Night = NP_VENUS_RADIUS + 300e3;
   const double bDay = GMm / (RHGPU_BOLTZMANN * 6400), bNight = GMm / (RHGPU_BOLTZMANN * 4847);
   const double nDay = r < r0Day ? 0.0 : 7.5e10 * exp(-bDay * (1.0 / r0Day - 1.0 / r));
   const double nNight = r < r0Night ? 0.0 : 2e9 * exp(-bNight * (1.0 / r0Night - 1.0 / r));
   return (1.0 - (chi / M_PI)) * nDay + (chi / M_PI) * nNight;
}

// one component of the Mercury sodium model: exponential in altitude times a
// Gaussian in the great-circle angle from its maximum (neutral_profiles.h:141-147)
__device__ inline double expexpNa(double x, double y, double z, double r, double Rp, double n0, double Hr, double Ht,
                                  double latMax, double lonMax) {
   const double lat = atan2(z, sqrt(x * x + y * y));
   const double lon = atan2(y, x);
   const double dth = acos(sin(lat) * sin(latMax) + cos(lat) * cos(latMax) * cos(lonMax - lon));
   return n0 * exp(-(r - Rp) / Hr) * exp(-((dth / Ht) * (dth / Ht)));
}

// Mercury sodium, Exner et al. (2020, J. Geophys. Res. 125, e2019JA027691):
// micro-meteoroid vaporisation, thermal desorption, two photon-stimulated
// desorption lobes and four sputtering lobes, times (Rp / r)^2
// (neutral_profiles.h:150-213)
__device__ inline double mercurySodium(double x, double y, double z) {
   const double Rp = NP_MERCURY_RADIUS;
   const double r = sqrt(x * x + y * y + z * z);
   const double d = M_PI / 180.0;
   // {n0 [m^-3], Hr [m], angular width, latitude, longitude of the maximum}
   const double lobes[7][5] = {{8.86e9, 100e3, 15 * d, 0 * d, 0 * d},        // thermal desorption
                               {5.67e6, 748e3, 15 * d, 80 * d, 0 * d},       // sputtering, day
                               {5.67e6, 748e3, 15 * d, -80 * d, 0 * d},
                               {5.67e6, 748e3, 10 * d, 15 * d, 180 * d},     // sputtering, night
                               {5.67e6, 748e3, 10 * d, -15 * d, 180 * d},
                               {4.06e10, 232e3, 20 * d, 50 * d, 0 * d},      // photon-stimulated desorption
                               {4.06e10, 232e3, 20 * d, -50 * d, 0 * d}};
   double sum = 7.84e6 * exp(-(r - Rp) / 431e3);   // micro-meteoroid vaporisation
   for (int q = 0; q < 7; ++q)
      sum = sum + expexpNa(x, y, z, r, Rp, lobes[q][0], lobes[q][1], lobes[q][2], lobes[q][3], lobes[q][4]);
   return ((Rp / r) * (Rp / r)) * sum;
}

// neutral density at (x, y, z): the planetary models (types 5-7) or a radial profile
__device__ inline double neutralDensityAt(const NeutralProfile& P, double x, double y, double z) {
   if (P.type == 5) return venusHydrogen(x, y, z);
   if (P.type == 6) return venusOxygen(x, y, z);
   if (P.type == 7) return mercurySodium(x, y, z);
   return neutralDensity(P, sqrt(x * x + y * y + z * z));
}

// the neutral density at n points (x, y, z interleaved)
__global__ void k_np_eval(NeutralProfile P, long long n, const double* xyz, double* out);

// each cell's mean neutral density times its volume by Monte Carlo over
// INJ_MC_POINTS points (zero below the exobase), particle_injector.cpp:1718-1736
__global__ void k_exo_density(GridInfo g, NeutralProfile P, double R2exo, unsigned long long seed, double* out);

// a Gaussian deviate pair by the polar method (G. Marsaglia, T. A. Bray, SIAM Rev. 6, 1964),
// the reference's sampleGaussian; false if no pair is accepted in INJ_MAX_TRIES
__device__ inline bool gaussianPair(RngStream& r, double& a, double& b) {
   for (int t = 0; t < INJ_MAX_TRIES; ++t) {
      const double x = 2.0 * r.uniform() - 1.0, y = 2.0 * r.uniform() - 1.0;
      const double r2 = x * x + y * y;
      if (r2 < 1.0 && r2 > 0.0) {
         const double fac = sqrt(-2.0 * log(r2) / r2);
         a = x * fac;
         b = y * fac;
         return true;
      }
   }
   a = b = 0.0;
   return false;
}

struct GaussSource {
   double saved;
   bool has;
   bool ok;
   __device__ double next(RngStream& r) {
      if (has) { has = false; return saved; }
      double a, b;
      ok = gaussianPair(r, a, b) && ok;
      saved = b;
      has = true;
      return a;
   }
};

// f(x) = c max(0, x) exp(-(x - x0)^2 / 2): the reference's sampleDerivGaussian
// (particle_injector.cpp:83-106), rejection from the unit Gaussian around the
// maximum xm = (x0 + sqrt(x0^2 + 4)) / 2; the normal speed of a drifting
// Maxwellian's flux through a wall, in thermal units
__device__ inline double derivGaussian(double x0, RngStream& r, GaussSource& g) {
   const double xm = 0.5 * (x0 + sqrt(x0 * x0 + 4.0));
   const double d = (x0 - xm) * (x0 - xm);
   for (int t = 0; t < INJ_MAX_TRIES; ++t) {
      const double x = xm + g.next(r);
      if (x < 0) continue;
      // pdf / majorant = x exp(-(x - x0)^2 / 2) / (xm exp(-((x - xm)^2 + d) / 2))
      const double ratio = (x / xm) * exp(-0.5 * ((x - x0) * (x - x0)) + 0.5 * ((x - xm) * (x - xm) + d));
      if (r.uniform() <= ratio) return x;
   }
   g.ok = false;
   return xm;
}

// the new particle's cell-local state (x, y, z, vx, vy, vz) in a cell of side dx
__device__ inline void injState(const InjDev& J, double dx, RngStream& r, GaussSource& g, double st[6]) {
   if (J.type == INJ_SOLARWIND) {
      const int ax = J.wall >> 1;
      const bool pos = J.wall & 1;   // enters through the positive wall, moving to -ax
      for (int a = 0; a < 3; ++a) st[a] = a == ax ? (pos ? 0.0 : dx) : r.uniform() * dx;
      for (int a = 0; a < 3; ++a) {
         if (a == ax) {
            const double s = J.vth * derivGaussian(J.U / J.vth, r, g);
            st[3 + a] = pos ? -s : s;
         } else {
            st[3 + a] = J.vth * g.next(r);
         }
      }
   } else if (J.type == INJ_FLOW) {
      for (int a = 0; a < 3; ++a) st[a] = r.uniform() * dx;
      for (int a = 0; a < 3; ++a) st[3 + a] = J.vel[a] + J.vth * g.next(r);
   } else {   // exosphere, ionospheres (particle_injector.cpp:1538-1564, 985-1018, 1285-1318)
      for (int a = 0; a < 3; ++a) st[a] = 0.5 * dx + (1.0 - INJ_EPS_CELL) * dx * (r.uniform() - 0.5);
      for (int a = 0; a < 3; ++a) st[3 + a] = J.vth * g.next(r);
   }
}

// ionosphere: each cell's share of the emission shell r = R, by Monte Carlo
// over INJ_MC_POINTS points of the cell projected on the shell, times the
// emission profile at the cell centre (InjectorIonosphere::initialize,
// particle_injector.cpp:1114-1210); profile 1..4 as RHGPU_IONO_*
__device__ inline double ionoFactor(int profile, double noon, double night, double xc, double yc, double zc) {
   if (profile == 3) return 1.0;
   if (profile == 4) {   // polar caps: rotated toward noon by `noon` degrees, half angle `night` degrees
      const double t = fabs(noon) * M_PI / 180.0, cap = fabs(night) * M_PI / 180.0;
      const double s = zc > 0.0 ? -t : t;
      const double x = xc * cos(s) + zc * sin(s), z = xc * sin(s) + zc * cos(s);
      const double rr = sqrt(x * x + yc * yc + z * z);
      const double colat = fabs(M_PI / 2.0 - acos(x / rr));
      return colat <= cap ? 1.0 : 0.0;
   }
   const double rr = sqrt(xc * xc + yc * yc + zc * zc);
   const double chi = acos(xc / rr);
   if (profile == 1) return chi < M_PI / 2 ? noon + (night - noon) * (1 - cos(chi)) : night;
   return chi < M_PI / 2 ? noon : night;   // 2: constant day, constant night
}
// Chapman ionosphere: acceptance a0 = a exp(1 - h - exp(-h)) of a point at
// (x, y, z) with h = (r - R) / H - log(1 / a), a the cos(SZA)-day / constant-night
// factor there (particle_injector.cpp:1299-1312, 1444-1456). The scale height
// uses Mars' surface gravity (Corsair's constants are not vendored: IAU
// nominal mass 6.4171e23 kg and radius 3389.5 km).
constexpr double NP_MARS_MASS = 6.4171e23;
constexpr double NP_MARS_RADIUS = 3389.5e3;
__device__ inline double chapmanAccept(double x, double y, double z, double R, double noon, double night, double H) {
   const double r = sqrt(x * x + y * y + z * z);
   const double chi = acos(x / r);
   const double a = chi < M_PI / 2 ? noon + (night - noon) * (1 - cos(chi)) : night;
   const double h = (r - R) / H - log(1.0 / a);
   return a * exp(1 - h - exp(-1 * h));
}
__global__ void k_chapman_shell(GridInfo g, double R, double noon, double night, double H, unsigned long long seed,
                                double* out);

__global__ void k_iono_shell(GridInfo g, double R, int profile, double noon, double night, unsigned long long seed,
                             double* out);

// migration of an injected position that sits on the far face of its cell
// (x == dx): to the next cell, as the push's migration does
__device__ inline void injCell(const GridInfo& g, int& i, int& j, int& k, double st[3]) {
   int c[3] = {i, j, k};
   const int n[3] = {g.nx, g.ny, g.nz};
   for (int a = 0; a < 3; ++a) {
      if (st[a] >= g.dx) {
         st[a] -= g.dx;
         if (++c[a] >= n[a]) c[a] = g.per[a] ? 0 : n[a] - 1;
      }
   }
   i = c[0]; j = c[1]; k = c[2];
}

// one thread per injection cell: probRound(perCellPerDt) particles (particle_injector.cpp:41-47)
template <class MV>
__global__ void k_inject(GridInfo g, FastGeom fg, InjDev J, long long step, MV* movers,
                         unsigned long long* nmovers, long long moverCap, double* injCnt, unsigned* err);

__device__ inline void writeMover(Mover& M, const GridInfo& g, const FastGeom& fg, const double st[7], int i, int j,
                                  int k, int species, unsigned long long key) {
   const int ux = dualU(i + halfS(st[0], g.dx) - 1, g.nx, g.per[0]);
   const int uy = dualU(j + halfS(st[1], g.dx) - 1, g.ny, g.per[1]);
   const int uz = dualU(k + halfS(st[2], g.dx) - 1, g.nz, g.per[2]);
   for (int a = 0; a < 7; ++a) M.s[a] = st[a];
   M.key = key;
   const int gd = ux / SEG;
   M.dest = ((long long)uy + (long long)fg.nd[1] * uz) * fg.nseg + gd;
   M.species = species;
   M.lx = (ux - gd * SEG) | MOVER_PLACE;
}

// FP32 form: offsets in cell units (as k_f32_seg_of stores an uploaded particle)
__device__ inline void writeMover(Mover32& M, const GridInfo& g, const FastGeom& fg, const double st[7], int i, int j,
                                  int k, int species, unsigned long long key) {
   const float below1 = 0x1.fffffep-1f;
   float o[3];
   for (int a = 0; a < 3; ++a) {
      o[a] = (float)(st[a] / g.dx);
      if (o[a] >= 1.0f) o[a] = below1;
   }
   const int ux = dualU(i + halfSf(o[0]) - 1, g.nx, g.per[0]);
   const int uy = dualU(j + halfSf(o[1]) - 1, g.ny, g.per[1]);
   const int uz = dualU(k + halfSf(o[2]) - 1, g.nz, g.per[2]);
   for (int a = 0; a < 3; ++a) { M.o[a] = o[a]; M.v[a] = (float)st[3 + a]; }
   M.cell = (int)cidx(g, i, j, k);
   M.species = species;
   M.key = key;
   const int gd = ux / SEG;
   M.dest = ((long long)uy + (long long)fg.nd[1] * uz) * fg.nseg + gd;
   M.lx = (ux - gd * SEG) | MOVER_PLACE;
}

// one injection cell t (or none, t < 0) per thread of a full warp
template <class MV>
__device__ void injectCell(const GridInfo& g, const FastGeom& fg, const InjDev& J, long long step, int t, MV* movers,
                           unsigned long long* nmovers, long long moverCap, double* injCnt, unsigned* err);

// grid-stride over the injection cells (or over the listed ones), whole blocks per round
template <class MV>
__global__ void k_inject(GridInfo g, FastGeom fg, InjDev J, long long step, MV* movers,
                         unsigned long long* nmovers, long long moverCap, double* injCnt, unsigned* err) {
   const int total = J.list ? *J.listCount : J.ncells;
   for (int b0 = blockIdx.x * blockDim.x; b0 < total; b0 += gridDim.x * blockDim.x) {
      const int idx = b0 + threadIdx.x;
      const int t = idx < total ? (J.list ? J.list[idx] : idx) : -1;
      injectCell(g, fg, J, step, t, movers, nmovers, moverCap, injCnt, err);
   }
}

template <class MV>
__device__ void injectCell(const GridInfo& g, const FastGeom& fg, const InjDev& J, long long step, int t, MV* movers,
                           unsigned long long* nmovers, long long moverCap, double* injCnt, unsigned* err) {
   const int lane = threadIdx.x & 31;
   RngStream r;
   int n = 0;
   if (t >= 0) {
      r.init(J.seed, (uint32_t)step, (uint32_t)(step >> 32), (uint32_t)t);
      // probRound: floor(x) + 1 with probability x - floor(x)
      const double x = (J.type == INJ_EXOSPHERE || J.type == INJ_IONOSPHERE || J.type == INJ_CHAPMAN) ? J.rates[t]
                                                                                                    : J.perCellPerDt;
      if (x > 0) {
         n = (int)floor(x);
         if (r.uniform() < x - n) ++n;
      }
   }
   // mover slots: one reservation per warp (inclusive scan of the counts)
   int incl = n;
   for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
   }
   const int wtotal = __shfl_sync(0xffffffffu, incl, 31);
   unsigned long long base = 0;
   if (lane == 31 && wtotal > 0) base = atomicAdd(nmovers, (unsigned long long)wtotal);
   base = __shfl_sync(0xffffffffu, base, 31);
   const unsigned long long m0 = base + (unsigned long long)(incl - n);
   double sw = 0.0, ske = 0.0;
   int placed = 0;
   GaussSource gs;
   gs.has = false;
   gs.ok = true;
   const int cell = n > 0 ? J.cells[t] : 0;
   const int ci = cell % g.nx, cj = (cell / g.nx) % g.ny, ck = cell / (g.nx * g.ny);
   for (int p = 0; p < n; ++p) {
      double st[7];
      injState(J, g.dx, r, gs, st);
      st[6] = J.w;
      int i = ci, j = cj, k = ck;
      if (J.type == INJ_CHAPMAN) {   // positions redrawn until accepted (particle_injector.cpp:1285-1318)
         bool acc = false;
         for (int tr = 0; tr < INJ_MAX_TRIES && !acc; ++tr) {
            if (tr > 0)
               for (int a = 0; a < 3; ++a) st[a] = 0.5 * g.dx + (1.0 - INJ_EPS_CELL) * g.dx * (r.uniform() - 0.5);
            const double a0 = chapmanAccept(g.x_min + ci * g.dx + st[0], g.y_min + cj * g.dx + st[1],
                                            g.z_min + ck * g.dx + st[2], J.R, J.noon, J.night, J.H);
            acc = r.uniform() < a0;
         }
         if (!acc) gs.ok = false;
      }
      if (J.type == INJ_IONOSPHERE || J.type == INJ_CHAPMAN) {   // upward (particle_injector.cpp:1008-1013)
         const double xg = g.x_min + ci * g.dx + st[0], yg = g.y_min + cj * g.dx + st[1], zg = g.z_min + ck * g.dx + st[2];
         if (st[3] * xg + st[4] * yg + st[5] * zg < 0)
            for (int a = 3; a < 6; ++a) st[a] = -st[a];
      }
      // exosphere: only above the exobase, no redraw (particle_injector.cpp:1547-1549)
      bool keep = true;
      if (J.type == INJ_EXOSPHERE) {
         const double xg = g.x_min + ci * g.dx + st[0], yg = g.y_min + cj * g.dx + st[1], zg = g.z_min + ck * g.dx + st[2];
         keep = xg * xg + yg * yg + zg * zg >= J.R2exo;
      }
      if (keep) injCell(g, i, j, k, st);
      const unsigned long long m = m0 + p;
      if ((long long)m >= moverCap) {
         raiseError(err, RHGPU_DEVERR_CAPACITY);
         continue;
      }
      if (!keep) {   // the reserved slot carries no flags: neither placed nor deposited
         movers[m].lx = 0;
         movers[m].species = J.species;
         movers[m].key = ~0ull;
         continue;
      }
      ++placed;
      sw += J.w;
      ske += J.w * (st[3] * st[3] + st[4] * st[4] + st[5] * st[5]);
      const unsigned long long key = ((unsigned long long)(J.keyBase + t) << 32) | (unsigned long long)p;
      writeMover(movers[m], g, fg, st, i, j, k, J.species, key);
   }
   if (!gs.ok) raiseError(err, RHGPU_DEVERR_INJECT);
   // the injection counters: one atomic per warp
   for (int o = 16; o > 0; o >>= 1) {
      sw += __shfl_xor_sync(0xffffffffu, sw, o);
      ske += __shfl_xor_sync(0xffffffffu, ske, o);
      placed += __shfl_xor_sync(0xffffffffu, placed, o);
   }
   if (lane == 0 && placed > 0) {
      atomicAdd(&injCnt[3 * J.species + 0], sw);
      atomicAdd(&injCnt[3 * J.species + 1], (double)placed);
      atomicAdd(&injCnt[3 * J.species + 2], ske);
   }
}

}  // namespace rh
