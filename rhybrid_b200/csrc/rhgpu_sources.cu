// Particle sources of the C ABI: the injectors' device form (solar wind,
// flow, exosphere and ionosphere sources with their neutral and production
// profiles), their counters, and the uniform fill of a species.
#include "rhgpu_host.h"

namespace rhh {

// the device buffers of one particle source
void freeInjector(InjHost& h) {
   cudaFree(h.cells);
   cudaFree(h.rates);
   cudaFree(h.list);
   h.cells = nullptr;
   h.rates = nullptr;
   h.list = nullptr;
}

}  // namespace rhh

namespace {
// InjectorExosphere::initialize (particle_injector.cpp:1610-1797): each cell's
// expected exospheric ion macroparticles per step, the weight and the cells
// that get any
// the device form of a neutral profile (per-component parameters of the radial profiles)
int neutralProfile(const rhgpu_injector& J, double m, NeutralProfile& P) {
   std::memset(&P, 0, sizeof P);
   const bool planet = J.profile >= RHGPU_NEUTRAL_VENUS_HYDROGEN && J.profile <= RHGPU_NEUTRAL_MERCURY_SODIUM_EXNER20;
   if (!planet && (J.profile < 1 || J.profile > 4 || J.n_components < 1 || J.n_components > RHGPU_NEUTRAL_MAX_COMPONENTS))
      return fail(RHGPU_ERR_ARG, "neutral profile type or its number of components");
   P.type = J.profile;
   P.n = planet ? 0 : J.n_components;
   P.r0 = J.r0;
   for (int i = 0; i < P.n; ++i) {
      P.n0[i] = J.n0[i];
      P.b[i] = J.profile == RHGPU_NEUTRAL_CHAMBERLAIN_H || J.profile == RHGPU_NEUTRAL_EXPONENTIAL ? J.H0[i]
               : J.profile == RHGPU_NEUTRAL_CHAMBERLAIN_T ? J.gm_object * m / (1.380649e-23 * J.T0[i])
                                                          : J.k0[i];
   }
   return RHGPU_OK;
}

int exoRates(rhgpu_ctx* c, const rhgpu_injector& J, InjHost& h, std::vector<int>& cells, std::vector<double>& rates) {
   const GridInfo& g = c->g;
   if (!(J.upstream_macro_ratio > 0)) return fail(RHGPU_ERR_ARG, "set_injectors: exosphere needs upstream_macro_ratio > 0");
   const bool ionGiven = J.ionization_rate >= 0, totalGiven = J.total_production_rate >= 0;
   if (ionGiven == totalGiven)
      return fail(RHGPU_ERR_ARG, "set_injectors: exosphere needs exactly one of ionization_rate, total_production_rate");
   const double m = c->sp[J.species].m;
   NeutralProfile P;
   {
      const int rc = neutralProfile(J, m, P);
      if (rc) return rc;
   }
   const double Rexo = std::max(J.exobase_radius, 0.0), Rsh = std::max(J.shadow_radius, 0.0);
   h.d.R2exo = Rexo * Rexo;
   double* dens = nullptr;
   RH_CUDA(cudaMalloc(&dens, sizeof(double) * g.N));
   k_exo_density<<<blocks1d(g.N, 128), 128, 0, c->stream>>>(g, P, h.d.R2exo, J.seed, dens);
   std::vector<double> cellExo(g.N);
   cudaError_t e = cudaGetLastError();
   if (e == cudaSuccess) e = cudaMemcpyAsync(cellExo.data(), dens, sizeof(double) * g.N, cudaMemcpyDeviceToHost, c->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
   cudaFree(dens);
   if (e != cudaSuccess) return fail(RHGPU_ERR_CUDA, std::string("set_injectors: exosphere density: ") + cudaGetErrorString(e));
   double total = 0.0;
   for (double v : cellExo) {
      if (v < 0) return fail(RHGPU_ERR_ARG, "set_injectors: negative neutral density");
      total += v;
   }
   if (!(total > 0)) return fail(RHGPU_ERR_ARG, "set_injectors: no neutrals in the box");
   const double rel = J.macroparticles_per_cell_relative >= 0 ? J.macroparticles_per_cell_relative : 1.0;
   const double perDt = rel * J.upstream_macro_ratio;
   if (!(perDt > 0)) return fail(RHGPU_ERR_ARG, "set_injectors: exosphere macroparticles per step must be positive");
   const double ionRate = ionGiven ? J.ionization_rate : J.total_production_rate / total;
   const double totalRate = ionGiven ? total * J.ionization_rate : J.total_production_rate;
   if (!(totalRate > 0)) return fail(RHGPU_ERR_ARG, "set_injectors: exosphere total production rate must be positive");
   const double shadow = std::max(J.ionization_factor_shadow, 0.0);
   for (long long n = 0; n < g.N; ++n) {
      const int i = (int)(n % g.nx), j = (int)((n / g.nx) % g.ny), k = (int)(n / ((long long)g.nx * g.ny));
      const double xc = g.x_min + (i + 0.5) * g.dx, yc = g.y_min + (j + 0.5) * g.dx, zc = g.z_min + (k + 0.5) * g.dx;
      const double f = (xc < 0 && yc * yc + zc * zc < Rsh * Rsh) ? shadow : 1.0;
      const double r = perDt * cellExo[n] * f * ionRate / totalRate;
      if (r > 0) {
         cells.push_back((int)n);
         rates.push_back(r);
      }
   }
   h.d.w = totalRate * g.dt / perDt;
   h.d.vth = J.temperature > 0 ? std::sqrt(1.380649e-23 * J.temperature / m) : 0.0;
   return RHGPU_OK;
}
// ionosphere: expected macroparticles per step of every cell on the emission
// shell (InjectorIonosphere::initialize, particle_injector.cpp:1059-1229)
int ionoRates(rhgpu_ctx* c, const rhgpu_injector& J, InjHost& h, std::vector<int>& cells, std::vector<double>& rates) {
   const GridInfo& g = c->g;
   const bool chapman = J.type == RHGPU_INJECT_CHAPMAN_IONOSPHERE;
   if (!chapman && (J.iono_profile < RHGPU_IONO_COS_SZA_DAY_CONSTANT_NIGHT || J.iono_profile > RHGPU_IONO_POLAR_CAP))
      return fail(RHGPU_ERR_ARG, "set_injectors: unknown ionospheric emission profile");
   if (!(J.emission_radius > 0)) return fail(RHGPU_ERR_ARG, "set_injectors: ionosphere needs emission_radius > 0");
   const double rel = J.macroparticles_per_cell_relative >= 0 ? J.macroparticles_per_cell_relative : 1.0;
   const double perDt = rel * (J.upstream_macro_ratio > 0 ? J.upstream_macro_ratio : 100.0);
   const double totalRate = J.total_production_rate;
   const double m = c->sp[J.species].m;
   h.d.vth = J.temperature > 0 ? std::sqrt(1.380649e-23 * J.temperature / m) : 0.0;
   if (!(perDt > 0 && totalRate > 0)) { h.d.w = 0.0; return RHGPU_OK; }   // no emission
   double* shell = nullptr;
   RH_CUDA(cudaMalloc(&shell, sizeof(double) * g.N));
   if (chapman) {
      // scale heights with Mars' surface gravity: 150 K for the cells' shares,
      // the source's temperature for the new particles (particle_injector.cpp:1306-1307, 1450-1451)
      const double gs = RHGPU_GRAVITY * NP_MARS_MASS / (NP_MARS_RADIUS * NP_MARS_RADIUS);
      h.d.R = J.emission_radius;
      h.d.noon = J.noon_factor;
      h.d.night = J.night_factor;
      h.d.H = (1.380649e-23 * J.temperature) / (m * gs);
      k_chapman_shell<<<blocks1d(g.N, 128), 128, 0, c->stream>>>(g, J.emission_radius, J.noon_factor, J.night_factor,
                                                                 (1.380649e-23 * 150) / (m * gs), J.seed, shell);
   } else {
      k_iono_shell<<<blocks1d(g.N, 128), 128, 0, c->stream>>>(g, J.emission_radius, J.iono_profile, J.noon_factor,
                                                               J.night_factor, J.seed, shell);
   }
   std::vector<double> inside(g.N);
   cudaError_t e = cudaGetLastError();
   if (e == cudaSuccess) e = cudaMemcpyAsync(inside.data(), shell, sizeof(double) * g.N, cudaMemcpyDeviceToHost, c->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
   cudaFree(shell);
   if (e != cudaSuccess) return fail(RHGPU_ERR_CUDA, std::string("set_injectors: ionosphere shell: ") + cudaGetErrorString(e));
   double total = 0.0;
   for (double v : inside) total += v;
   if (total > 0.0)
      for (long long n = 0; n < g.N; ++n) {
         const double r = perDt * inside[n] / total;
         if (r > 0) {
            cells.push_back((int)n);
            rates.push_back(r);
         }
      }
   h.d.w = totalRate * g.dt / perDt;
   return RHGPU_OK;
}
}  // namespace

extern "C" {

int rhgpu_fill_uniform(rhgpu_ctx* c, int32_t s, const rhgpu_injector* J, const double* region) {
   if (!c || s < 0 || s >= c->ns || !J) return fail(RHGPU_ERR_ARG, "fill_uniform: bad arguments");
   if (c->path != RHGPU_PATH_FAST && c->path != RHGPU_PATH_FP32)
      return fail(RHGPU_ERR_STATE, "fill_uniform: the fast path or the FP32 form only (the exact path takes host records)");
   if (!(J->density >= 0) || !(J->temperature >= 0) || !(J->macroparticles_per_cell >= 0) ||
       !(J->macroparticles_per_cell < 2e9))
      return fail(RHGPU_ERR_ARG, "fill_uniform: density, temperature and macroparticles_per_cell must be >= 0");
   RH_CUDA(cudaSetDevice(c->device));
   const GridInfo& g = c->g;
   FillSpec F;
   F.seed = J->seed;
   F.ppc = J->density > 0 ? J->macroparticles_per_cell : 0.0;
   F.w = (F.ppc > 0) ? J->density * g.dV / F.ppc : 0.0;
   F.vth = J->temperature > 0 ? std::sqrt(1.380649e-23 * J->temperature / c->sp[s].m) : 0.0;
   for (int a = 0; a < 3; ++a) {
      F.U[a] = J->velocity[a];
      F.lo[a] = region ? region[2 * a] : -HUGE_VAL;
      F.hi[a] = region ? region[2 * a + 1] : HUGE_VAL;
   }
   F.species = s;
   const long long NS = c->fg.NS;
   const bool f32 = c->path == RHGPU_PATH_FP32;
   const float below1 = std::nextafter(1.0f, 0.0f);
   int rc = RHGPU_OK;
   int* cnt;
   long long* base;
   if (f32) {
      rc = f32Init(c);
      if (rc) return rc;
      cnt = c->f32[s].cnt[c->f32[s].cur];
      base = c->f32[s].base;
   } else {
      cnt = c->seg[s].cnt[c->seg[s].cur];
      base = c->seg[s].base;
   }
   if (f32)
      k_fill_count<true><<<(unsigned)NS, FILL_THREADS, 0, c->stream>>>(g, c->fg, F, below1, cnt);
   else
      k_fill_count<false><<<(unsigned)NS, FILL_THREADS, 0, c->stream>>>(g, c->fg, F, below1, cnt);
   RH_CUDA(cudaGetLastError());
   long long n = 0;
   rc = segPrefix(c, cnt, &n);
   if (rc) return rc;
   if (c->capHint[s] > 0 && n > c->capHint[s]) return fail(RHGPU_ERR_CAPACITY, "fill_uniform: more particles than capacity");
   long long slots = 0;
   rc = fastLayout(c, cnt, nullptr, base, &slots);
   if (rc) return rc;
   if (f32) {
      F32Host& h = c->f32[s];
      rc = f32Reserve(h, 0, slots);
      if (!rc) rc = f32Reserve(h, 1, slots);
      if (rc) return rc;
      h.w = F.w;
      SegBuf none{};
      k_fill_write<true><<<(unsigned)NS, FILL_THREADS, 0, c->stream>>>(g, c->fg, F, below1, base, none, f32View(h, h.cur));
   } else {
      SegHost& h = c->seg[s];
      rc = segReserve(h, 0, slots);
      if (!rc) rc = segReserve(h, 1, slots);
      if (rc) return rc;
      F32Buf none{};
      k_fill_write<false><<<(unsigned)NS, FILL_THREADS, 0, c->stream>>>(g, c->fg, F, below1, base, segView(h, h.cur), none);
   }
   RH_CUDA(cudaGetLastError());
   RH_CUDA(cudaStreamSynchronize(c->stream));
   c->uploaded = true;
   if (f32) {
      f32Exponents(c);
      return f32MoverBuffers(c);
   }
   rc = fastExponents(c);
   if (rc) return rc;
   return fastMoverBuffers(c);
}

// the device form of one particle source (cells, rates and lists allocated on
// the device); on failure h holds whatever was allocated, for freeInjector
int buildInjector(rhgpu_ctx* c, const rhgpu_injector& J, long long& keyBase, InjHost& h) {
   const GridInfo& g = c->g;
   const int nn[3] = {g.nx, g.ny, g.nz};
   if (J.species < 0 || J.species >= c->ns) return fail(RHGPU_ERR_ARG, "set_injectors: bad species");
   if (!(J.density >= 0) || !(J.temperature >= 0) || !(J.macroparticles_per_cell >= 0))
      return fail(RHGPU_ERR_ARG, "set_injectors: density, temperature and macroparticles_per_cell must be >= 0");
   std::memset(&h.d, 0, sizeof h.d);
   h.d.species = J.species;
   h.d.type = J.type;
   h.d.seed = J.seed;
   const double m = c->sp[J.species].m;
   h.d.vth = J.temperature > 0 ? std::sqrt(1.380649e-23 * J.temperature / m) : 0.0;
   const double ppc = J.macroparticles_per_cell;
   h.d.w = (ppc > 0 && J.density > 0) ? J.density * g.dV / ppc : 0.0;
   std::vector<int> cells;
   // (i, j, k) has its neighbour along axis a on the side sgn
   auto hasNb = [&](const int p[3], int a, int sgn) {
      if (g.per[a]) return true;
      return sgn > 0 ? p[a] < nn[a] - 1 : p[a] > 0;
   };
   if (J.type == RHGPU_INJECT_SOLARWIND) {
      int ax = -1;
      for (int a = 0; a < 3; ++a)
         if (J.velocity[a] != 0.0) { if (ax >= 0) ax = 3; else ax = a; }
      if (ax < 0 || ax > 2)
         return fail(RHGPU_ERR_ARG, "set_injectors: solar wind velocity must have exactly one non-zero component");
      const bool pos = J.velocity[ax] < 0;   // flows toward -ax: enters through the +ax wall
      h.d.wall = 2 * ax + (pos ? 1 : 0);
      h.d.U = std::fabs(J.velocity[ax]);
      h.d.perCellPerDt = ppc > 0 && J.density > 0 ? ppc * h.d.U * g.dt / g.dx : 0.0;
      if (h.d.vth <= 0) return fail(RHGPU_ERR_ARG, "set_injectors: solar wind needs a temperature > 0");
      // InjectorSolarWind::checkIfInjectionCell{X,Y,Z}{Pos,Neg} (particle_injector.cpp:392-446)
      for (int k = 0; k < g.nz; ++k)
         for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
               const int p[3] = {i, j, k};
               if (hasNb(p, ax, pos ? 1 : -1)) continue;
               bool edge = false;
               for (int a = 0; a < 3; ++a)
                  if (a != ax && (!hasNb(p, a, 1) || !hasNb(p, a, -1))) edge = true;
               if (!edge) cells.push_back(i + g.nx * (j + g.ny * k));
            }
   } else if (J.type == RHGPU_INJECT_FLOW) {
      for (int a = 0; a < 3; ++a) h.d.vel[a] = J.velocity[a];
      h.d.perCellPerDt = ppc > 0 && J.density > 0 ? ppc : 0.0;
      // ghost cells of the selected inflow walls (InjectorFlow::inject, particle_injector.cpp:749-760)
      for (int k = 0; k < g.nz; ++k)
         for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i) {
               const int p[3] = {i, j, k};
               bool in = false;
               for (int b = 0; b < 6; ++b)
                  if ((J.inflow_walls >> b & 1) && !hasNb(p, b >> 1, (b & 1) ? -1 : 1)) in = true;
               if (in) cells.push_back(i + g.nx * (j + g.ny * k));
            }
   } else if (J.type == RHGPU_INJECT_EXOSPHERE || J.type == RHGPU_INJECT_IONOSPHERE ||
              J.type == RHGPU_INJECT_CHAPMAN_IONOSPHERE) {
      std::vector<double> rates;
      int rc = J.type == RHGPU_INJECT_EXOSPHERE ? exoRates(c, J, h, cells, rates) : ionoRates(c, J, h, cells, rates);
      if (rc) return rc;
      if (!rates.empty()) {
         RH_CUDA(cudaMalloc(&h.rates, sizeof(double) * rates.size()));
         RH_CUDA(cudaMemcpy(h.rates, rates.data(), sizeof(double) * rates.size(), cudaMemcpyHostToDevice));
      }
      h.rateCells = cells;
      h.rateValues = rates;
      h.d.rates = h.rates;
      if (!cells.empty()) {
         // the selected cells (ncells ints) and their count (one int after them)
         RH_CUDA(cudaMalloc(&h.list, sizeof(int) * (cells.size() + 1)));
         h.d.list = h.list;
         h.d.listCount = h.list + cells.size();
      }
   } else {
      return fail(RHGPU_ERR_ARG, "set_injectors: unknown type");
   }
   h.d.ncells = (int)cells.size();
   h.d.keyBase = keyBase;
   keyBase += (long long)cells.size();
   if (!cells.empty()) {
      RH_CUDA(cudaMalloc(&h.cells, sizeof(int) * cells.size()));
      RH_CUDA(cudaMemcpy(h.cells, cells.data(), sizeof(int) * cells.size(), cudaMemcpyHostToDevice));
   }
   h.d.cells = h.cells;
   return RHGPU_OK;
}

// the new source set is built aside and replaces the old one only when every
// source was built; on failure the previous sources stay in force and what was
// built is freed
int rhgpu_set_injectors(rhgpu_ctx* c, int32_t n, const rhgpu_injector* inj) {
   if (!c || n < 0 || (n > 0 && !inj)) return fail(RHGPU_ERR_ARG, "set_injectors: bad arguments");
   RH_CUDA(cudaSetDevice(c->device));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   if (!c->injCnt) {
      RH_CUDA(cudaMalloc(&c->injCnt, sizeof(double) * 3 * MAX_SPECIES));
      RH_CUDA(cudaMemset(c->injCnt, 0, sizeof(double) * 3 * MAX_SPECIES));
   }
   long long keyBase = c->fg.NS > 0 ? c->fg.NS : 1;
   std::vector<InjHost> built;
   for (int q = 0; q < n; ++q) {
      InjHost h;
      const int rc = buildInjector(c, inj[q], keyBase, h);
      if (rc) {
         freeInjector(h);
         for (auto& b : built) freeInjector(b);
         return rc;
      }
      built.push_back(h);
   }
   for (auto& h : c->inj) freeInjector(h);
   c->inj = std::move(built);
   c->injKeyMax = keyBase;
   return RHGPU_OK;
}

int rhgpu_source_rates(rhgpu_ctx* c, int32_t injector, double* out) {
   if (!c || !out) return fail(RHGPU_ERR_ARG, "source_rates: bad arguments");
   if (injector < 0 || injector >= (int)c->inj.size()) return fail(RHGPU_ERR_ARG, "source_rates: no such source");
   const InjHost& h = c->inj[injector];
   std::fill(out, out + c->g.N, 0.0);
   for (size_t q = 0; q < h.rateCells.size(); ++q) out[h.rateCells[q]] = h.rateValues[q];
   return RHGPU_OK;
}

int rhgpu_neutral_density(const rhgpu_injector* profile, double mass, int64_t n, const double* xyz, double* out,
                          int32_t device) {
   if (!profile || n < 0 || (n > 0 && (!xyz || !out))) return fail(RHGPU_ERR_ARG, "neutral_density: bad arguments");
   NeutralProfile P;
   int rc = neutralProfile(*profile, mass, P);
   if (rc) return rc;
   if (n == 0) return RHGPU_OK;
   RH_CUDA(cudaSetDevice(device));
   double *dx = nullptr, *dout = nullptr;
   RH_CUDA(cudaMalloc(&dx, sizeof(double) * 3 * n));
   cudaError_t e = cudaMalloc(&dout, sizeof(double) * n);
   if (e == cudaSuccess) e = cudaMemcpy(dx, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice);
   if (e == cudaSuccess) {
      k_np_eval<<<blocks1d(n, 128), 128>>>(P, n, dx, dout);
      e = cudaGetLastError();
   }
   if (e == cudaSuccess) e = cudaMemcpy(out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost);
   cudaFree(dx);
   cudaFree(dout);
   if (e != cudaSuccess) return fail(RHGPU_ERR_CUDA, std::string("neutral_density: ") + cudaGetErrorString(e));
   return RHGPU_OK;
}

int rhgpu_get_injection_counters(rhgpu_ctx* c, double* out, int32_t n) {
   if (!c || !out || n < 3 * c->ns) return fail(RHGPU_ERR_ARG, "get_injection_counters: bad arguments");
   RH_CUDA(cudaSetDevice(c->device));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   std::vector<double> v(3 * (size_t)c->ns, 0.0);
   if (c->injCnt) RH_CUDA(cudaMemcpy(v.data(), c->injCnt, sizeof(double) * v.size(), cudaMemcpyDeviceToHost));
   std::memcpy(out, v.data(), sizeof(double) * v.size());
   return RHGPU_OK;
}

void rhgpu_philox4x32(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
   const Philox4 r = philox4x32(ctr, key);
   for (int a = 0; a < 4; ++a) out[a] = r.v[a];
}

}  // extern "C"
