// Diagnostics of the C ABI: the log sums (rhgpu_reduce_diagnostics), the log
// files and the max-B stop, the temporal averages of the output populations,
// and the per-cell grid constraint counters.
#include "rhgpu_host.h"

extern "C" {

namespace {
// adds the DIAG_BLOCKS partial rows of width w in block order (sums, or maxima where maxMask has the bit)
void diagCombine(const std::vector<double>& h, int w, unsigned long long maxMask, double* out,
                 unsigned long long minMask = 0ull) {
   for (int q = 0; q < w; ++q) {
      double a = ((minMask >> q) & 1ull) ? INFINITY : 0.0;
      for (int b = 0; b < DIAG_BLOCKS; ++b) {
         const double x = h[(size_t)b * w + q];
         a = ((maxMask >> q) & 1ull) ? std::max(a, x) : ((minMask >> q) & 1ull) ? std::min(a, x) : a + x;
      }
      out[q] = a;
   }
}

// total ion mass density per cell into c->rhoM (logCalcParticle, diagnostics.h:223-238)
int massDensity(rhgpu_ctx* c) {
   const long long N = c->g.N;
   if (!c->rhoM) {
      RH_CUDA(cudaMalloc(&c->rhoM, sizeof(double) * N));
      RH_CUDA(cudaMalloc(&c->rhoMfix, sizeof(unsigned long long) * 2 * N));
   }
   const double minRhoM = c->P.min_ion_charge_density * RHGPU_MASS_PROTON / RHGPU_CHARGE_ELEMENTARY;
   if (c->path == RHGPU_PATH_EXACT) {
      MassSet M;
      std::memset(&M, 0, sizeof M);
      M.ns = c->ns;
      for (int s = 0; s < c->ns; ++s) { M.P[s] = c->ps[s]; M.m[s] = c->sp[s].m; }
      k_diag_rhom_cell<<<blocks1d(N, 256), 256, 0, c->stream>>>(M, N, c->g.dV, minRhoM, c->rhoM);
      RH_CUDA(cudaGetLastError());
      return RHGPU_OK;
   }
   // fixed-point scale from the largest w*m: every addend below 2^62
   double wm[MAX_SPECIES] = {};
   double big = 0.0;
   for (int s = 0; s < c->ns; ++s) {
      double w = 0.0;
      if (c->path == RHGPU_PATH_FAST) {
         const SegHost& h = c->seg[s];
         if (!h.a[h.cur][0]) continue;
         unsigned long long* mw = (unsigned long long*)c->fover;
         RH_CUDA(cudaMemsetAsync(mw, 0, sizeof(unsigned long long), c->stream));
         k_fast_max_abs_w<<<(unsigned)c->fg.NS, 128, 0, c->stream>>>(segView(h, h.cur), h.base, mw);
         RH_CUDA(cudaGetLastError());
         unsigned long long bits = 0;
         RH_CUDA(cudaMemcpyAsync(&bits, mw, sizeof bits, cudaMemcpyDeviceToHost, c->stream));
         RH_CUDA(cudaStreamSynchronize(c->stream));
         std::memcpy(&w, &bits, sizeof w);
      } else {
         if (!c->f32ready || !c->f32[s].cell[c->f32[s].cur]) continue;
         w = std::fabs(c->f32[s].w);
      }
      wm[s] = w * c->sp[s].m;
      big = std::max(big, wm[s]);
   }
   int e;
   std::frexp(big > 0 ? big : 1.0, &e);
   const int k = 62 - e;
   const double scale = std::ldexp(1.0, k);
   unsigned long long *lo = c->rhoMfix, *hi = c->rhoMfix + N;
   RH_CUDA(cudaMemsetAsync(c->rhoMfix, 0, sizeof(unsigned long long) * 2 * N, c->stream));
   for (int s = 0; s < c->ns; ++s) {
      if (wm[s] == 0.0) continue;
      if (c->path == RHGPU_PATH_FAST) {
         const SegHost& h = c->seg[s];
         k_diag_rhom_seg<<<DIAG_BLOCKS, DIAG_THREADS, 0, c->stream>>>(c->g, c->fg, segView(h, h.cur), h.base, c->sp[s].m,
                                                                      scale, lo, hi);
      } else {
         const F32Host& h = c->f32[s];
         k_diag_rhom_f32<<<DIAG_BLOCKS, DIAG_THREADS, 0, c->stream>>>(f32View(h, h.cur), h.base, c->fg.NS,
                                                                      h.w * c->sp[s].m, scale, lo, hi);
      }
      RH_CUDA(cudaGetLastError());
   }
   k_diag_rhom_finish<<<blocks1d(N, 256), 256, 0, c->stream>>>(lo, hi, N, std::ldexp(1.0, 64 - k), std::ldexp(1.0, -k),
                                                                c->g.dV, minRhoM, c->rhoM);
   RH_CUDA(cudaGetLastError());
   return RHGPU_OK;
}

// the population and field reductions into out (8 ns + 30 values, + 6 scales when withScales)
int diagnostics(rhgpu_ctx* c, double* out, bool withScales) {
   RH_CUDA(cudaSetDevice(c->device));
   std::vector<double> h((size_t)DIAG_BLOCKS * DIAG_FS);
   for (int s = 0; s < c->ns; ++s) {
      double* o = out + DIAG_P * s;
      bool launched = false;
      if (c->path == RHGPU_PATH_FAST) {
         const SegHost& sh = c->seg[s];
         if (sh.a[sh.cur][0]) {
            k_diag_particles_seg<<<DIAG_BLOCKS, DIAG_THREADS, 0, c->stream>>>(segView(sh, sh.cur), sh.base, c->fg.NS, c->diagPart);
            launched = true;
         }
      } else if (c->path == RHGPU_PATH_FP32) {
         const F32Host& fh = c->f32[s];
         if (c->f32ready && fh.cell[fh.cur]) {
            k_diag_particles_f32<<<DIAG_BLOCKS, DIAG_THREADS, 0, c->stream>>>(f32View(fh, fh.cur), fh.base, c->fg.NS,
                                                                            fh.w, c->diagPart);
            launched = true;
         }
      } else if (c->ps[s].start) {
         k_diag_particles_cell<<<DIAG_BLOCKS, DIAG_THREADS, 0, c->stream>>>(c->ps[s], c->g.N, c->diagPart);
         launched = true;
      }
      if (!launched) {
         for (int q = 0; q < DIAG_P; ++q) o[q] = 0.0;
         continue;
      }
      RH_CUDA(cudaGetLastError());
      RH_CUDA(cudaMemcpyAsync(h.data(), c->diagPart, sizeof(double) * DIAG_BLOCKS * DIAG_P, cudaMemcpyDeviceToHost, c->stream));
      RH_CUDA(cudaStreamSynchronize(c->stream));
      diagCombine(h, DIAG_P, DIAG_P_MAX, o);
   }
   if (withScales) {
      const int rc = massDensity(c);
      if (rc) return rc;
   }
   k_diag_field<<<DIAG_BLOCKS, DIAG_THREADS, 0, c->stream>>>(c->g, c->f, withScales ? c->rhoM : nullptr, c->logInner,
                                                             c->diagPart);
   RH_CUDA(cudaGetLastError());
   RH_CUDA(cudaMemcpyAsync(h.data(), c->diagPart, sizeof(double) * DIAG_BLOCKS * DIAG_FS, cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   double f[DIAG_FS];
   diagCombine(h, DIAG_FS, DIAG_F_MAX, f, DIAG_F_MIN);
   double* o = out + DIAG_P * c->ns;
   for (int q = 0; q < DIAG_F; ++q) o[q] = f[q];
   if (withScales) {
      // min/max de, min/max di, min Larmor period, max Alfven speed
      logScales(f[30], f[31], f[32], f[33], f[5], RHGPU_MASS_ELECTRON, RHGPU_MASS_PROTON, RHGPU_CHARGE_ELEMENTARY,
                RHGPU_PERMEABILITY, o + DIAG_F);
      o[DIAG_F + 5] = f[34];
   }
   return RHGPU_OK;
}

// the log counters back to zero (logWriteParticleField, diagnostics.h:777-800)
int zeroLogCounters(rhgpu_ctx* c) {
   RH_CUDA(cudaMemsetAsync(c->cntU, 0, sizeof(unsigned long long) * NCNT_U, c->stream));
   RH_CUDA(cudaMemsetAsync(c->cntD, 0, sizeof(double) * 4 * MAX_SPECIES, c->stream));
   if (c->injCnt) RH_CUDA(cudaMemsetAsync(c->injCnt, 0, sizeof(double) * 3 * MAX_SPECIES, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   return RHGPU_OK;
}
}  // namespace

int rhgpu_reduce_diagnostics(rhgpu_ctx* c, double* out, int32_t n) {
   if (!c || !out) return fail(RHGPU_ERR_ARG, "bad arguments");
   if (n < DIAG_P * c->ns + DIAG_F) return fail(RHGPU_ERR_ARG, "reduce_diagnostics: out needs 8*n_species + 30 doubles");
   return diagnostics(c, out, n >= DIAG_P * c->ns + DIAG_F + 6);
}

int rhgpu_log_open(rhgpu_ctx* c, const rhgpu_log_config* cfg) {
   if (!c || !cfg || !cfg->directory || !cfg->species_names) return fail(RHGPU_ERR_ARG, "log_open: bad arguments");
   std::vector<LogSpecies> sp(c->ns);
   for (int s = 0; s < c->ns; ++s) {
      if (!cfg->species_names[s]) return fail(RHGPU_ERR_ARG, "log_open: a species name is NULL");
      sp[s].name = cfg->species_names[s];
      sp[s].m = c->sp[s].m;
      sp[s].q = c->sp[s].q;
   }
   if (!c->logs) c->logs = new LogFiles();
   std::string err;
   if (!c->logs->open(cfg->directory, sp, cfg->precision > 0 ? cfg->precision : 10, err)) return fail(RHGPU_ERR_ARG, "log_open: " + err);
   c->logInner = cfg->include_inner_cells ? 1 : 0;
   c->logMaxB = cfg->max_B_stop_run;
   c->logTStart = c->t;
   RH_CUDA(cudaSetDevice(c->device));
   return zeroLogCounters(c);
}

int rhgpu_log_write(rhgpu_ctx* c, int32_t main_log_diagnostics, int32_t* stop_run, char* messages, int32_t messages_cap) {
   if (!c) return fail(RHGPU_ERR_ARG, "null context");
   if (!c->logs || !c->logs->isOpen()) return fail(RHGPU_ERR_STATE, "log_write: rhgpu_log_open first");
   const int ns = c->ns;
   std::vector<double> d(DIAG_P * ns + DIAG_F + 6);
   int rc = diagnostics(c, d.data(), true);
   if (rc) return rc;
   std::vector<double> cnt(RHGPU_NUM_FIELD_COUNTERS + RHGPU_CNT_PER_SPECIES * ns);
   rc = rhgpu_get_counters(c, cnt.data(), (int32_t)cnt.size());
   if (rc) return rc;
   std::vector<double> inj(3 * ns, 0.0);
   if (c->injCnt) RH_CUDA(cudaMemcpy(inj.data(), c->injCnt, sizeof(double) * 3 * ns, cudaMemcpyDeviceToHost));
   LogStep L;
   L.t = c->t;
   L.dt = c->P.dt;
   L.dx = c->P.dx;
   L.dV = c->g.dV;
   L.tStart = c->logTStart;
   L.timestep = c->timestep;
   L.permeability = RHGPU_PERMEABILITY;
   L.permittivity = RHGPU_PERMITTIVITY;
   L.pop.resize(ns);
   L.pc.assign(ns, std::vector<double>(LPC_COUNT, 0.0));
   for (int s = 0; s < ns; ++s) {
      const double* p = &d[DIAG_P * s];
      L.pop[s] = LogPopulation{p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7]};
      const double* q = &cnt[RHGPU_NUM_FIELD_COUNTERS + RHGPU_CNT_PER_SPECIES * s];
      std::vector<double>& pc = L.pc[s];
      pc[LPC_MAXVI] = q[0];
      pc[LPC_ESCAPE] = q[1];
      pc[LPC_ESCAPE_KE] = q[2];
      pc[LPC_IMPACT] = q[3];
      pc[LPC_IMPACT_KE] = q[4];
      pc[LPC_INJECT] = inj[3 * s + 0];
      pc[LPC_INJECT_MACRO] = inj[3 * s + 1];
      pc[LPC_INJECT_KE] = inj[3 * s + 2];
   }
   const double* f = &d[DIAG_P * ns];
   LogField& F = L.f;
   F.nCells = f[0];
   F.sumBx = f[1]; F.sumBy = f[2]; F.sumBz = f[3]; F.sumB = f[4]; F.maxB = f[5];
   F.sumDivB = f[6]; F.maxDivB = f[7]; F.maxDivBPerB = f[8]; F.sumB2 = f[9];
   F.sumJx = f[10]; F.sumJy = f[11]; F.sumJz = f[12]; F.sumJ = f[13]; F.maxJ = f[14];
   F.sumEpx = f[15]; F.sumEpy = f[16]; F.sumEpz = f[17]; F.sumEp = f[18]; F.maxEp = f[19]; F.sumEp2 = f[20];
   F.sumEx = f[21]; F.sumEy = f[22]; F.sumEz = f[23]; F.sumE = f[24]; F.maxE = f[25]; F.sumE2 = f[26];
   F.sumCellE2 = f[27]; F.maxUe = f[28];
   F.minDe = f[30]; F.maxDe = f[31]; F.minDi = f[32]; F.maxDi = f[33]; F.minTLarmor = f[34]; F.maxVA = f[35];
   L.fc[LFC_MAX_CELL_UE] = cnt[RHGPU_CNT_FIELD_MAX_CELL_UE];
   L.fc[LFC_MAX_NODE_UE] = cnt[RHGPU_CNT_FIELD_MAX_NODE_UE];
   L.fc[LFC_MAX_VW] = cnt[RHGPU_CNT_FIELD_MAX_NODE_UE];   // the reference's writer reports this counter here
   L.fc[LFC_MAX_E] = cnt[RHGPU_CNT_FIELD_MAX_E];
   L.fc[LFC_MIN_CELL_RHOQI] = cnt[RHGPU_CNT_FIELD_MIN_CELL_RHOQI];
   L.fc[LFC_MIN_NODE_RHOQI] = cnt[RHGPU_CNT_FIELD_MIN_NODE_RHOQI];
   std::string msg;
   const bool ok = c->logs->write(L, c->logMaxB, main_log_diagnostics != 0, msg);
   if (stop_run) *stop_run = ok ? 0 : 1;
   if (messages && messages_cap > 0) {
      const size_t k = std::min(msg.size(), (size_t)messages_cap - 1);
      std::memcpy(messages, msg.data(), k);
      messages[k] = 0;
   }
   c->logTStart = c->t;
   return zeroLogCounters(c);
}

int rhgpu_set_population_averages(rhgpu_ctx* c, int32_t n_groups, const int32_t* group_of_species) {
   if (!c || n_groups < 0 || (n_groups > 0 && !group_of_species)) return fail(RHGPU_ERR_ARG, "set_population_averages: bad arguments");
   if (n_groups > 0 && c->path == RHGPU_PATH_FP32)
      return fail(RHGPU_ERR_STATE, "population averages run on the fast and exact paths");
   for (int s = 0; s < c->ns && n_groups > 0; ++s)
      if (group_of_species[s] < -1 || group_of_species[s] >= n_groups)
         return fail(RHGPU_ERR_ARG, "set_population_averages: group index out of range");
   RH_CUDA(cudaSetDevice(c->device));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   cudaFree(c->avgN); cudaFree(c->avgV); cudaFree(c->avgOut);
   c->avgN = c->avgV = c->avgOut = nullptr;
   c->avgGroups = 0;
   if (n_groups == 0) return RHGPU_OK;
   const long long N = c->g.N;
   RH_CUDA(cudaMalloc(&c->avgN, sizeof(double) * n_groups * N));
   RH_CUDA(cudaMalloc(&c->avgV, sizeof(double) * 3 * n_groups * N));
   RH_CUDA(cudaMalloc(&c->avgOut, sizeof(double) * 4 * N));
   RH_CUDA(cudaMemset(c->avgN, 0, sizeof(double) * n_groups * N));
   RH_CUDA(cudaMemset(c->avgV, 0, sizeof(double) * 3 * n_groups * N));
   for (int s = 0; s < c->ns; ++s) c->avgGroupOf[s] = group_of_species[s];
   c->avgGroups = n_groups;
   return RHGPU_OK;
}

int rhgpu_output_averages(rhgpu_ctx* c, double* cellB_average, double* n_average, double* v_average) {
   if (!c) return fail(RHGPU_ERR_ARG, "null context");
   if ((n_average || v_average) && !c->avgGroups)
      return fail(RHGPU_ERR_STATE, "output_averages: no population averages (rhgpu_set_population_averages)");
   RH_CUDA(cudaSetDevice(c->device));
   const long long N = c->g.N;
   const double inv = c->gridAvgCounter > 0 ? 1.0 / c->gridAvgCounter : 0.0;
   if (!c->avgOut && cellB_average) {
      RH_CUDA(cudaMalloc(&c->avgOut, sizeof(double) * 4 * N));
   }
   if (cellB_average) {
      k_avgB_output<<<blocks1d(N, 256), 256, 0, c->stream>>>(N, c->arr[RHGPU_CELL_AVERAGE_B], inv, c->avgOut);
      RH_CUDA(cudaGetLastError());
      RH_CUDA(cudaMemcpyAsync(cellB_average, c->avgOut, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, c->stream));
      RH_CUDA(cudaStreamSynchronize(c->stream));
   }
   if (n_average || v_average) {
      for (int grp = 0; grp < c->avgGroups; ++grp) {
         // the charge of the population's first species (operator_userdata.cpp:186-187)
         int first = -1;
         for (int s = 0; s < c->ns && first < 0; ++s)
            if (c->avgGroupOf[s] == grp) first = s;
         const double q = first >= 0 ? c->sp[first].q : 1.0;
         k_avg_output<<<blocks1d(N, 256), 256, 0, c->stream>>>(N, c->avgN + (long long)grp * N, c->avgV + 3LL * grp * N, q,
                                                               c->g.dV, inv, n_average ? c->avgOut : nullptr,
                                                               v_average ? c->avgOut + N : nullptr);
         RH_CUDA(cudaGetLastError());
         if (n_average)
            RH_CUDA(cudaMemcpyAsync(n_average + (long long)grp * N, c->avgOut, sizeof(double) * N, cudaMemcpyDeviceToHost,
                                    c->stream));
         if (v_average)
            RH_CUDA(cudaMemcpyAsync(v_average + 3LL * grp * N, c->avgOut + N, sizeof(double) * 3 * N,
                                    cudaMemcpyDeviceToHost, c->stream));
         RH_CUDA(cudaStreamSynchronize(c->stream));
      }
   }
   c->gridAvgCounter = 0;
   return RHGPU_OK;
}

int rhgpu_set_grid_counters(rhgpu_ctx* c, int32_t enable) {
   if (!c) return fail(RHGPU_ERR_ARG, "null context");
   RH_CUDA(cudaSetDevice(c->device));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   const long long N = c->g.N;
   if (!enable) {
      cudaFree(c->gridCnt);
      c->gridCnt = nullptr;
      c->f.gc = nullptr;
      return RHGPU_OK;
   }
   if (!c->gridCnt) RH_CUDA(cudaMalloc(&c->gridCnt, sizeof(double) * GC_PLANES * N));
   RH_CUDA(cudaMemset(c->gridCnt, 0, sizeof(double) * GC_PLANES * N));
   c->f.gc = c->gridCnt;
   return RHGPU_OK;
}

int rhgpu_download_grid_counters(rhgpu_ctx* c, double* out) {
   if (!c || !out) return fail(RHGPU_ERR_ARG, "download_grid_counters: bad arguments");
   if (!c->gridCnt) return fail(RHGPU_ERR_STATE, "download_grid_counters: grid counters are off (rhgpu_set_grid_counters)");
   RH_CUDA(cudaSetDevice(c->device));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   RH_CUDA(cudaMemcpy(out, c->gridCnt, sizeof(double) * GC_PLANES * c->g.N, cudaMemcpyDeviceToHost));
   return RHGPU_OK;
}

int rhgpu_log_close(rhgpu_ctx* c) {
   if (!c) return fail(RHGPU_ERR_ARG, "null context");
   if (c->logs) c->logs->close();
   return RHGPU_OK;
}

}  // extern "C"
