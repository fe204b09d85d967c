// The FP32 precision form of the C ABI (RHGPU_PATH_FP32): its particle
// storage (cell index, FP32 offsets and velocities), upload and download, the
// push and deposit, the movers' deposit and placement, the gather.
#include <cub/device/device_radix_sort.cuh>

#include "rhgpu_host.h"

namespace rhh {

F32Buf f32View(const F32Host& h, int which) {
   F32Buf b;
   b.cell = h.cell[which];
   for (int a = 0; a < 3; ++a) { b.o[a] = h.o[which][a]; b.v[a] = h.v[which][a]; }
   b.cnt = h.cnt[which];
   return b;
}

int f32Reserve(F32Host& h, int which, long long slots) {
   if (slots <= h.capOf[which] && h.cell[which]) return RHGPU_OK;
   const long long had = h.capOf[which];
   auto release = [&]() {
      cudaFree(h.cell[which]);
      h.cell[which] = nullptr;
      for (int a = 0; a < 3; ++a) {
         cudaFree(h.o[which][a]); cudaFree(h.v[which][a]);
         h.o[which][a] = nullptr; h.v[which][a] = nullptr;
      }
      h.capOf[which] = 0;
   };
   auto alloc = [&](long long n) {
      cudaError_t e = cudaMalloc(&h.cell[which], sizeof(int) * n);
      for (int a = 0; a < 3 && e == cudaSuccess; ++a) {
         e = cudaMalloc(&h.o[which][a], sizeof(float) * n);
         if (e == cudaSuccess) e = cudaMalloc(&h.v[which][a], sizeof(float) * n);
      }
      return e;
   };
   release();
   long long n = growSlots(had, slots);
   if (alloc(n) != cudaSuccess && had > 0) {   // no room for the growth margin: the slots alone
      release();
      cudaGetLastError();
      n = growSlots(0, slots);
      alloc(n);
   }
   const cudaError_t e = cudaGetLastError();
   if (e != cudaSuccess || !h.v[which][2]) {
      release();
      return fail(RHGPU_ERR_CUDA, std::string("FP32 particle storage: ") + cudaGetErrorString(e));
   }
   h.capOf[which] = n;
   return RHGPU_OK;
}

// buffers of the FP32 form, allocated when a context chooses it
int f32Init(rhgpu_ctx* c) {
   if (c->f32ready) return RHGPU_OK;
   const long long NS = c->fg.NS;
   for (int s = 0; s < c->ns; ++s) {
      F32Host& h = c->f32[s];
      for (int b = 0; b < 2; ++b) {
         RH_CUDA(cudaMalloc(&h.cnt[b], sizeof(int) * NS));
         RH_CUDA(cudaMemset(h.cnt[b], 0, sizeof(int) * NS));
      }
      RH_CUDA(cudaMalloc(&h.base, sizeof(long long) * (NS + 1)));
      RH_CUDA(cudaMemset(h.base, 0, sizeof(long long) * (NS + 1)));
      RH_CUDA(cudaMalloc(&h.baseAlt, sizeof(long long) * (NS + 1)));
   }
   RH_CUDA(cudaMalloc(&c->f32b.RP, sizeof(float) * 16 * c->fg.nrows * c->g.nx));
   RH_CUDA(cudaMalloc(&c->f32b.RPB, sizeof(float) * 16 * c->fg.nrows * c->fg.nseg));
   RH_CUDA(cudaMemset(c->f32b.RPB, 0, sizeof(float) * 16 * c->fg.nrows * c->fg.nseg));
   c->f32b.MMlo = c->fb.MMlo;
   c->f32b.MMhi = c->fb.MMhi;
   c->f32b.touched = c->fb.touched;
   c->f32b.segInner = c->fb.segInner;
   c->f32b.nmovers = c->fb.nmovers;
   RH_CUDA(cudaDeviceSynchronize());   // the clears above run on the default stream
   c->f32ready = true;
   return RHGPU_OK;
}

// (w q) of the first species that deposits anything: the unit of the FP32 sums
double f32WqRef(const rhgpu_ctx* c) {
   for (int s = 0; s < c->ns; ++s) {
      const double wq = c->f32[s].w * c->sp[s].q;
      if (wq != 0.0) return wq;
   }
   return 1.0;
}

F32Set f32Set(rhgpu_ctx* c) {
   F32Set F;
   std::memset(&F, 0, sizeof F);
   F.ns = c->ns;
   const double ref = f32WqRef(c);
   for (int s = 0; s < c->ns; ++s) {
      const F32Host& h = c->f32[s];
      F.st[s].cur = f32View(h, h.cur);
      F.st[s].nxt = f32View(h, h.cur ^ 1);
      F.st[s].base = h.base;
      F.accumulate[s] = c->sp[s].accumulate;
      F.accelerate[s] = c->sp[s].accelerate;
      F.qm[s] = (float)(0.5 * c->sp[s].q * c->P.dt / c->sp[s].m);
      F.wqRel[s] = (float)(h.w * c->sp[s].q / ref);
      F.R2obs[s] = (float)c->sp[s].R2_obstacle;
      F.w[s] = h.w;
   }
   return F;
}

F32Params f32Params(rhgpu_ctx* c) {
   F32Params pp;
   pp.dtdx = (float)(c->P.dt / c->P.dx);
   pp.dt = (float)c->P.dt;
   pp.dx = (float)c->P.dx;
   pp.below1 = std::nextafter(1.0f, 0.0f);
   pp.maxVi2 = (float)c->P.max_ion_speed2;
   pp.GMdt = (float)c->P.GMdt;
   pp.useIFT = c->useIFT;
   pp.use_ep = c->P.use_electron_pressure;
   pp.use_gravity = c->P.use_gravity;
   return pp;
}

// fixed-point exponents of the out-of-segment sums, in units of the reference (w q)
void f32Exponents(rhgpu_ctx* c) {
   const double ref = f32WqRef(c);
   double bR = 0.0;
   for (int s = 0; s < c->ns; ++s) bR = std::max(bR, std::fabs(c->f32[s].w * c->sp[s].q / ref));
   // FP32 weights and velocities: allow the rounding of a float above the bound
   bR *= 1.0 + 1e-6;
   const double bJ = bR * (2.0 * c->P.dx / c->P.dt);
   int e;
   std::frexp(bR > 0 ? bR : 1.0, &e);
   c->kR = 62 - e;
   std::frexp(bJ > 0 ? bJ : 1.0, &e);
   c->kJ = 62 - e;
   c->f32b.scaleR = std::ldexp(1.0, c->kR);
   c->f32b.scaleJ = std::ldexp(1.0, c->kJ);
}

int f32MoverBuffers(rhgpu_ctx* c) {
   long long tot = 0;
   for (int s = 0; s < c->ns; ++s) tot += c->f32[s].capOf[c->f32[s].cur];
   const long long want = moverListSize(tot);
   if (want > c->f32b.moverCap) {
      cudaFree(c->f32b.movers);
      c->f32b.movers = nullptr;
      c->f32b.moverCap = 0;
      RH_CUDA(cudaMalloc(&c->f32b.movers, sizeof(Mover32) * want));
      c->f32b.moverCap = want;
   }
   return ensureMigBuffers(c, want);
}

// particles: 7 doubles per record, or (particles32, with weight32) the FP32
// form's own 6-float records
int f32Upload(rhgpu_ctx* c, int s, const uint32_t* counts, const double* particles, long long n,
              const float* particles32, double weight32) {
   int rc = f32Init(c);
   if (rc) return rc;
   const long long N = c->g.N, NS = c->fg.NS;
   const size_t recBytes = particles32 ? sizeof(float) * 6 : sizeof(double) * 7;
   const size_t recAll = recBytes * (size_t)(n > 0 ? n : 1);
   rc = ensureStaging(c, recAll + sizeof(uint32_t) * (size_t)N + 64);
   if (rc) return rc;
   rc = ensureKeyCapacity(c, 2 * n + 2);
   if (rc) return rc;
   double* aos = (double*)c->staging;
   float* aos32 = (float*)c->staging;
   uint32_t* dcounts = (uint32_t*)((char*)c->staging + ((recAll + 15) / 16) * 16);
   RH_CUDA(cudaMemcpyAsync(dcounts, counts, sizeof(uint32_t) * N, cudaMemcpyHostToDevice, c->stream));
   if (n) RH_CUDA(cudaMemcpyAsync(c->staging, particles32 ? (const void*)particles32 : (const void*)particles,
                                  recBytes * n, cudaMemcpyHostToDevice, c->stream));
   F32Host& h = c->f32[s];
   // one weight per species
   if (particles32) {
      h.w = n ? weight32 : 0.0;
   } else if (n) {
      unsigned long long* mm = (unsigned long long*)c->fover;   // [0] min, [1] max
      const unsigned long long init[2] = {~0ull, 0ull};
      RH_CUDA(cudaMemcpyAsync(mm, init, sizeof init, cudaMemcpyHostToDevice, c->stream));
      k_weight_range<<<DIAG_BLOCKS, 256, 0, c->stream>>>(aos, n, mm, mm + 1);
      RH_CUDA(cudaGetLastError());
      unsigned long long r[2];
      RH_CUDA(cudaMemcpyAsync(r, mm, sizeof r, cudaMemcpyDeviceToHost, c->stream));
      RH_CUDA(cudaStreamSynchronize(c->stream));
      double lo, hi;
      std::memcpy(&lo, &r[0], 8);
      std::memcpy(&hi, &r[1], 8);
      if (lo != hi) return fail(RHGPU_ERR_ARG, "upload_particles: the FP32 form stores one weight per species");
      h.w = hi;
   } else {
      h.w = 0.0;
   }
   int* pcell = c->rank;
   long long* cstart = c->ftmpCellStart;
   k_counts_in<<<blocks1d(N + 1, 256), 256, 0, c->stream>>>(N, dcounts, c->newCount, c->outCount);
   RH_CUDA(cudaGetLastError());
   if (int rc_ = scanExclusive64(c, c->newCount, cstart, N + 1)) return rc_;
   long long total = 0;
   RH_CUDA(cudaMemcpyAsync(&total, cstart + N, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   if (total != n) return fail(RHGPU_ERR_ARG, "upload_particles: sum(counts) != n_particles");
   k_fill_pcell<<<blocks1d(N, 128), 128, 0, c->stream>>>(N, cstart, pcell);
   RH_CUDA(cudaGetLastError());
   rc = growBuffer(c->fsort, c->fsortCap, 2 * n + 2);
   if (rc) return rc;
   unsigned* keyIn = (unsigned*)c->key;
   unsigned* keyOut = keyIn + (n + 1);
   unsigned* idxIn = (unsigned*)c->fsort;
   unsigned* idxOut = idxIn + (n + 1);
   const float below1 = std::nextafter(1.0f, 0.0f);
   if (n) {
      if (particles32)
         k_f32_seg_of<<<blocks1d(n, 256), 256, 0, c->stream>>>(c->g, c->fg, RecordsF{aos32}, pcell, n, below1, keyIn);
      else
         k_f32_seg_of<<<blocks1d(n, 256), 256, 0, c->stream>>>(c->g, c->fg, RecordsD{aos}, pcell, n, below1, keyIn);
      k_iota<<<blocks1d(n, 256), 256, 0, c->stream>>>(idxIn, n);
      RH_CUDA(cudaGetLastError());
      size_t sb = 0;
      cub::DeviceRadixSort::SortPairs(nullptr, sb, keyIn, keyOut, idxIn, idxOut, (int)n, 0, 32, c->stream);
      rc = ensureSortTmp(c, sb);
      if (rc) return rc;
      sb = c->sortTmpBytes;
      RH_CUDA(cub::DeviceRadixSort::SortPairs(c->sortTmp, sb, keyIn, keyOut, idxIn, idxOut, (int)n, 0, 32, c->stream));
   }
   k_sorted_bounds<<<blocks1d(n + 1, 256), 256, 0, c->stream>>>(keyOut, n, NS, c->ffirst);
   k_bounds_counts<<<blocks1d(NS, 256), 256, 0, c->stream>>>(c->ffirst, NS, h.cnt[h.cur]);
   RH_CUDA(cudaGetLastError());
   long long slots = 0;
   rc = fastLayout(c, h.cnt[h.cur], nullptr, h.base, &slots);
   if (rc) return rc;
   rc = f32Reserve(h, 0, slots);
   if (rc) return rc;
   rc = f32Reserve(h, 1, slots);
   if (rc) return rc;
   if (n) {
      if (particles32)
         k_f32_scatter_sorted<<<blocks1d(n, 256), 256, 0, c->stream>>>(c->g, RecordsF{aos32}, pcell, keyOut, idxOut, n,
                                                                       c->ffirst, f32View(h, h.cur), h.base, below1);
      else
         k_f32_scatter_sorted<<<blocks1d(n, 256), 256, 0, c->stream>>>(c->g, RecordsD{aos}, pcell, keyOut, idxOut, n,
                                                                       c->ffirst, f32View(h, h.cur), h.base, below1);
      RH_CUDA(cudaGetLastError());
   }
   RH_CUDA(cudaStreamSynchronize(c->stream));
   f32Exponents(c);
   return f32MoverBuffers(c);
}

int f32NumParticles(rhgpu_ctx* c, int s, long long* n) {
   if (!c->f32ready) { *n = 0; return RHGPU_OK; }
   return segPrefix(c, c->f32[s].cnt[c->f32[s].cur], n);
}

// particles: 7 doubles per record, or (particles32) the FP32 form's own 6-float records
int f32Download(rhgpu_ctx* c, int s, uint32_t* counts, double* particles, long long capacity, long long* n_out,
                float* particles32) {
   const long long N = c->g.N, NS = c->fg.NS;
   int rc = f32Init(c);
   if (rc) return rc;
   long long tot = 0;
   rc = f32NumParticles(c, s, &tot);
   if (rc) return rc;
   if (tot > capacity) return fail(RHGPU_ERR_ARG, "download_particles: capacity too small");
   rc = ensureKeyCapacity(c, 2 * tot + 2);
   if (rc) return rc;
   rc = growBuffer(c->fsortSlots, c->fsortSlotsCap, tot + 1);
   if (rc) return rc;
   rc = growBuffer(c->fsort, c->fsortCap, 2 * tot + 2);
   if (rc) return rc;
   rc = ensureStaging(c, sizeof(double) * 7 * (size_t)(tot > 0 ? tot : 1) + sizeof(uint32_t) * (size_t)N + 64);
   if (rc) return rc;
   unsigned* keyIn = (unsigned*)c->key;
   unsigned* keyOut = keyIn + (tot + 1);
   unsigned* idxIn = (unsigned*)c->fsort;
   unsigned* idxOut = idxIn + (tot + 1);
   double* aos = (double*)c->staging;
   int* cellCnt = c->outCount;
   const F32Host& h = c->f32[s];
   if (tot) {
      k_f32_cell_keys<<<(unsigned)NS, 128, 0, c->stream>>>(c->fg, f32View(h, h.cur), h.base, c->ffirst, keyIn, c->fsortSlots);
      k_iota<<<blocks1d(tot, 256), 256, 0, c->stream>>>(idxIn, tot);
      RH_CUDA(cudaGetLastError());
      size_t sb = 0;
      cub::DeviceRadixSort::SortPairs(nullptr, sb, keyIn, keyOut, idxIn, idxOut, (int)tot, 0, 32, c->stream);
      rc = ensureSortTmp(c, sb);
      if (rc) return rc;
      sb = c->sortTmpBytes;
      RH_CUDA(cub::DeviceRadixSort::SortPairs(c->sortTmp, sb, keyIn, keyOut, idxIn, idxOut, (int)tot, 0, 32, c->stream));
      k_sorted_bounds<<<blocks1d(tot + 1, 256), 256, 0, c->stream>>>(keyOut, tot, N, c->ftmpCellStart);
      k_bounds_counts<<<blocks1d(N, 256), 256, 0, c->stream>>>(c->ftmpCellStart, N, cellCnt);
      if (particles32)
         k_f32_gather_records_f32<<<blocks1d(tot, 256), 256, 0, c->stream>>>(f32View(h, h.cur), c->fsortSlots, idxOut,
                                                                              tot, (float*)aos);
      else
         k_f32_gather_records<<<blocks1d(tot, 256), 256, 0, c->stream>>>(f32View(h, h.cur), c->fsortSlots, idxOut, tot,
                                                                         c->P.dx, h.w, aos);
      RH_CUDA(cudaGetLastError());
   } else {
      RH_CUDA(cudaMemsetAsync(cellCnt, 0, sizeof(int) * N, c->stream));
   }
   RH_CUDA(cudaMemcpyAsync(counts, cellCnt, sizeof(uint32_t) * N, cudaMemcpyDeviceToHost, c->stream));
   if (tot && particles32)
      RH_CUDA(cudaMemcpyAsync(particles32, aos, sizeof(float) * 6 * tot, cudaMemcpyDeviceToHost, c->stream));
   else if (tot && particles)
      RH_CUDA(cudaMemcpyAsync(particles, aos, sizeof(double) * 7 * tot, cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   *n_out = tot;
   return RHGPU_OK;
}

// relays out the "next" buffers of the species in `mask` (bit s: species s)
// with room for their pending arrivals; the other species keep their layout
int f32RelayoutNext(rhgpu_ctx* c, unsigned mask) {
   RH_TIME(c, "f32_relayout");
   const long long NS = c->fg.NS;
   for (int s = 0; s < c->ns; ++s) {
      if (!((mask >> s) & 1u)) continue;
      F32Host& h = c->f32[s];
      const int nx = h.cur ^ 1;
      long long total = 0;
      int rc = fastLayout(c, h.cnt[nx], c->finc + (long long)s * NS, h.baseAlt, &total);
      if (rc) return rc;
      rc = f32Reserve(h, h.cur, total);
      if (rc) return rc;
      k_f32_relayout<<<(unsigned)NS, 128, 0, c->stream>>>(f32View(h, nx), h.base, f32View(h, h.cur), h.baseAlt);
      RH_CUDA(cudaGetLastError());
      std::swap(h.base, h.baseAlt);
      h.cur ^= 1;
      rc = f32Reserve(h, h.cur, total);
      if (rc) return rc;
   }
   RH_CUDA(cudaStreamSynchronize(c->stream));
   return f32MoverBuffers(c);
}

int f32Push(rhgpu_ctx* c) {
   int rc = f32Init(c);
   if (rc) return rc;
   c->timestep += 1;
   if (c->P.initial_flow_through_period < c->t && c->useIFT) c->useIFT = 0;
   const long long N = c->g.N, NS = c->fg.NS;
   RH_CUDA(cudaMemsetAsync(c->fb.touched, 0, (size_t)N + 16, c->stream));
   RH_CUDA(cudaMemsetAsync(c->fb.nmovers, 0, sizeof(unsigned long long), c->stream));
   {
      RH_TIME(c, "f32_push_deposit");
      const F32Set FS = f32Set(c);
      const F32Params FP = f32Params(c);
      switch (perMask(c->g)) {
#define RH_F32_PD(M)                                                                                            \
   case M:                                                                                                        \
      if (c->f.gc)                                                                                                \
         k_f32_push_deposit<M, true><<<(unsigned)NS, FT, 0, c->stream>>>(c->g, c->f, c->fg, FS, FP, c->f32b, c->cntD,  \
                                                                         c->cntU, c->err);                         \
      else                                                                                                        \
         k_f32_push_deposit<M, false><<<(unsigned)NS, FT, 0, c->stream>>>(c->g, c->f, c->fg, FS, FP, c->f32b,          \
                                                                          c->cntD, c->cntU, c->err);               \
      break;
         RH_F32_PD(0) RH_F32_PD(1) RH_F32_PD(2) RH_F32_PD(3) RH_F32_PD(4) RH_F32_PD(5) RH_F32_PD(6) RH_F32_PD(7)
#undef RH_F32_PD
      }
      RH_LAUNCHED(c);
   }
   {
      const int rc = injectAll(c, c->f32b.movers, c->f32b.moverCap);
      if (rc) return rc;
   }
   unsigned long long nm = 0;
   RH_CUDA(cudaMemcpyAsync(&nm, c->fb.nmovers, sizeof nm, cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   if ((long long)nm > c->f32b.moverCap) return fail(RHGPU_ERR_CAPACITY, "mover list overflow");
   if (nm > 0) {
      {
         RH_TIME(c, "f32_mover_deposit");
         k_f32_mover_deposit<<<blocks1d(nm, 128), 128, 0, c->stream>>>(c->g, c->fg, f32Set(c), c->f32b, nm);
         RH_LAUNCHED(c);
      }
      const long long nb = (long long)c->ns * NS;
      int over = 0;
      {
         RH_TIME(c, "f32_migrate");
         unsigned *order = nullptr, *bkt = nullptr;
         int rc = migSort(c, c->f32b.movers, (long long)nm, f32Set(c), &order, &bkt, &over);
         if (rc) return rc;
         if (over) {
            // some segments lack room for their arrivals: relayout with room for them
            rc = f32RelayoutNext(c, (unsigned)over);
            if (rc) return rc;
            RH_CUDA(cudaMemsetAsync(c->fover, 0, sizeof(int), c->stream));
            k_mig_check<<<blocks1d(nb, 256), 256, 0, c->stream>>>(f32Set(c), NS, c->finc, c->fover);
            RH_LAUNCHED(c);
            RH_CUDA(cudaMemcpyAsync(&over, c->fover, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
            RH_CUDA(cudaStreamSynchronize(c->stream));
            if (over) return fail(RHGPU_ERR_CAPACITY, "segment relayout did not make room");
         }
         k_f32_mig_place<<<blocks1d(nm, 256), 256, 0, c->stream>>>(f32Set(c), NS, nb, c->f32b.movers, order, bkt, c->foffInc,
                                                                 (long long)nm);
         RH_LAUNCHED(c);
         k_mig_counts<<<blocks1d(nb, 256), 256, 0, c->stream>>>(f32Set(c), NS, c->finc);
         RH_LAUNCHED(c);
      }
   }
   for (int s = 0; s < c->ns; ++s) c->f32[s].cur ^= 1;
   return RHGPU_OK;
}

int f32Gather(rhgpu_ctx* c) {
   int rc = f32Init(c);
   if (rc) return rc;
   RH_TIME(c, "f32_gather");
   const double hiR = std::ldexp(1.0, 64 - c->kR), loR = std::ldexp(1.0, -c->kR);
   const double hiJ = std::ldexp(1.0, 64 - c->kJ), loJ = std::ldexp(1.0, -c->kJ);
   const double scale = f32WqRef(c) / c->g.dV;
   if (c->f.gc)
      k_f32_gather<true><<<cellGrid(c->g), cellBlock(), 0, c->stream>>>(c->g, c->f, c->fg, c->f32b, hiR, loR, hiJ, loJ,
                                                                       scale, c->P.min_ion_charge_density, c->cntU);
   else
      k_f32_gather<false><<<cellGrid(c->g), cellBlock(), 0, c->stream>>>(c->g, c->f, c->fg, c->f32b, hiR, loR, hiJ,
                                                                        loJ, scale, c->P.min_ion_charge_density, c->cntU);
   RH_LAUNCHED(c);
   return RHGPU_OK;
}

}  // namespace rhh
