// The fast particle path of the C ABI (RHGPU_PATH_FAST): row-segment storage,
// upload and download in the reference's per-cell layout, the fused push and
// deposit, the movers' deposit and placement, the gather of the moments, and
// the particle sources of a step.
#include <cub/device/device_radix_sort.cuh>

#include "rhgpu_host.h"

namespace rhh {

// sort scratch of at least `bytes`; it grows by at least a quarter at a time,
// since the migration's radix sorts ask for more with every new largest mover
// count and each reallocation synchronises inside the step
int ensureSortTmp(rhgpu_ctx* c, size_t bytes) {
   if (bytes <= c->sortTmpBytes) return RHGPU_OK;
   const size_t want = std::max(bytes, c->sortTmpBytes + c->sortTmpBytes / 4) + 256;
   cudaFree(c->sortTmp);
   c->sortTmp = nullptr;
   c->sortTmpBytes = 0;
   RH_CUDA(cudaMalloc(&c->sortTmp, want));
   c->sortTmpBytes = want;
   return RHGPU_OK;
}

SegBuf segView(const SegHost& h, int which) {
   SegBuf b;
   for (int a = 0; a < 7; ++a) b.a[a] = h.a[which][a];
   b.lx = h.lx[which];
   b.cnt = h.cnt[which];
   return b;
}

// particle arrays of buffer `which` with room for `slots` slots
int segReserve(SegHost& h, int which, long long slots) {
   if (slots <= h.capOf[which] && h.a[which][0]) return RHGPU_OK;
   const long long had = h.capOf[which];
   auto release = [&]() {
      for (int a = 0; a < 7; ++a) { cudaFree(h.a[which][a]); h.a[which][a] = nullptr; }
      cudaFree(h.lx[which]);
      h.lx[which] = nullptr;
      h.capOf[which] = 0;
   };
   auto alloc = [&](long long n) {
      cudaError_t e = cudaSuccess;
      for (int a = 0; a < 7 && e == cudaSuccess; ++a) e = cudaMalloc(&h.a[which][a], sizeof(double) * n);
      if (e == cudaSuccess) e = cudaMalloc(&h.lx[which], n);
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
   if (e != cudaSuccess || !h.lx[which]) {
      release();
      return fail(RHGPU_ERR_CUDA, std::string("particle storage: ") + cudaGetErrorString(e));
   }
   h.capOf[which] = n;
   return RHGPU_OK;
}

// segment layout with slack from per-segment counts (+ pending arrivals): base, total slots
int fastLayout(rhgpu_ctx* c, const int* cnt, const int* extra, long long* base, long long* total) {
   const long long NS = c->fg.NS;
   k_fast_capacity<<<blocks1d(NS + 1, 256), 256, 0, c->stream>>>(NS, cnt, extra, c->fcap);
   RH_CUDA(cudaGetLastError());
   if (int rc_ = scanExclusive64(c, c->fcap, base, NS + 1)) return rc_;
   RH_CUDA(cudaMemcpyAsync(total, base + NS, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   return RHGPU_OK;
}

FastSpecies fastSpecies(rhgpu_ctx* c) {
   FastSpecies F;
   std::memset(&F, 0, sizeof F);
   F.ns = c->ns;
   for (int s = 0; s < c->ns; ++s) {
      const SegHost& h = c->seg[s];
      F.st[s].cur = segView(h, h.cur);
      F.st[s].nxt = segView(h, h.cur ^ 1);
      F.st[s].base = h.base;
      F.sp[s] = speciesDev(c, s);
   }
   return F;
}

// fixed-point exponents of the out-of-segment deposit from the largest |w q| (oracle: fixedPointExponents)
int fastExponents(rhgpu_ctx* c) {
   double bR = 0.0;
   for (int s = 0; s < c->ns; ++s) {
      unsigned long long* mw = (unsigned long long*)c->fover;
      RH_CUDA(cudaMemsetAsync(mw, 0, sizeof(unsigned long long), c->stream));
      k_fast_max_abs_w<<<(unsigned)c->fg.NS, 128, 0, c->stream>>>(segView(c->seg[s], c->seg[s].cur), c->seg[s].base, mw);
      RH_CUDA(cudaGetLastError());
      unsigned long long bits = 0;
      RH_CUDA(cudaMemcpyAsync(&bits, mw, sizeof bits, cudaMemcpyDeviceToHost, c->stream));
      RH_CUDA(cudaStreamSynchronize(c->stream));
      double w;
      std::memcpy(&w, &bits, sizeof w);
      const double b = w * std::fabs(c->sp[s].q);
      if (b > bR) bR = b;
   }
   const double bJ = bR * (2.0 * c->P.dx / c->P.dt);
   int e;
   std::frexp(bR > 0 ? bR : 1.0, &e);
   c->kR = 62 - e;
   std::frexp(bJ > 0 ? bJ : 1.0, &e);
   c->kJ = 62 - e;
   c->fb.scaleR = std::ldexp(1.0, c->kR);
   c->fb.scaleJ = std::ldexp(1.0, c->kJ);
   return RHGPU_OK;
}

// sort buffers of the migration for up to `want` movers
int ensureMigBuffers(rhgpu_ctx* c, long long want) {
   if (want <= c->mcap) return RHGPU_OK;
   cudaFree(c->mkey); cudaFree(c->mval); cudaFree(c->mbkt);
   c->mkey = nullptr; c->mval = nullptr; c->mbkt = nullptr;
   c->mcap = 0;
   RH_CUDA(cudaMalloc(&c->mkey, sizeof(unsigned long long) * 2 * want));
   RH_CUDA(cudaMalloc(&c->mval, sizeof(unsigned) * 2 * want));
   RH_CUDA(cudaMalloc(&c->mbkt, sizeof(unsigned) * 2 * want));
   c->mcap = want;
   return RHGPU_OK;
}

// entries of the mover list for `slots` particle slots: a quarter of them (at
// least 2^20); past 2^29 slots a sixteenth, but at least 2^27 (movers are
// about 1-3 % of the particles per step in the workloads, more in hot plasmas
// of small test boxes; a step whose movers exceed the list fails with
// RHGPU_ERR_CAPACITY)
long long moverListSize(long long slots) {
   return std::max(1LL << 20, std::min(slots / 4, std::max(slots / 16, 1LL << 27)));
}

// mover list: moverListSize of all slots
int fastMoverBuffers(rhgpu_ctx* c) {
   long long tot = 0;
   for (int s = 0; s < c->ns; ++s) tot += c->seg[s].capOf[c->seg[s].cur];
   const long long want = moverListSize(tot);
   if (want > c->fb.moverCap) {
      cudaFree(c->fb.movers);
      c->fb.movers = nullptr;
      c->fb.moverCap = 0;
      RH_CUDA(cudaMalloc(&c->fb.movers, sizeof(Mover) * want));
      c->fb.moverCap = want;
   }
   return ensureMigBuffers(c, want);
}

int bitsFor(long long x) {
   int b = 1;
   while (b < 63 && (x >> b) != 0) ++b;
   return b;
}

// the arrivals of the nm movers: per destination (species, segment) bucket the
// count (c->finc) and first position (c->foffInc), the movers sorted by bucket
// and within it by key (*order, *bucket; bucket ns*NS = not placed), and
// whether some bucket lacks room (*over). Buckets of at most MIG_SMALL arrivals
// (the usual case) are ordered one thread per bucket, those of up to
// MIG_LARGE one block per bucket; past that two stable radix sorts over all
// movers (by key, then by bucket) give the same order.
template <class MV, class SET>
int migSort(rhgpu_ctx* c, const MV* mv, long long nm, const SET& FS, unsigned** order, unsigned** bucket, int* over) {
   const long long NS = c->fg.NS, nb = (long long)c->ns * NS;
   if (nm > c->mcap) return fail(RHGPU_ERR_CAPACITY, "mover list larger than its sort buffers");
   RH_CUDA(cudaMemsetAsync(c->finc, 0, sizeof(int) * nb, c->stream));
   RH_CUDA(cudaMemsetAsync(c->fover, 0, sizeof(int), c->stream));
   k_fast_mig_count<<<blocks1d(nm, 256), 256, 0, c->stream>>>(mv, nm, NS, c->finc);
   RH_LAUNCHED(c);
   k_int_to64<<<blocks1d(nb + 1, 256), 256, 0, c->stream>>>(c->finc, nb, c->ftmpInc64);
   RH_LAUNCHED(c);
   if (int rc_ = scanExclusive64(c, c->ftmpInc64, c->foffInc, nb + 1)) return rc_;
   unsigned long long *kA = c->mkey, *kB = c->mkey + c->mcap;
   unsigned *vA = c->mval, *vB = c->mval + c->mcap, *bA = c->mbkt, *bB = c->mbkt + c->mcap;
   RH_CUDA(cudaMemsetAsync(c->fmaxInc, 0, sizeof(int), c->stream));
   k_max_int<<<(unsigned)std::min<long long>(blocks1d(nb, 256), 4 * 148), 256, 0, c->stream>>>(c->finc, nb, c->fmaxInc);
   RH_LAUNCHED(c);
   int rc = RHGPU_OK;
   int maxInc = 0;
   RH_CUDA(cudaMemcpyAsync(&maxInc, c->fmaxInc, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   if (maxInc <= MIG_LARGE) {
      // buckets past the placed movers stay at nb (not placed)
      RH_CUDA(cudaMemsetAsync(c->ffill, 0, sizeof(int) * nb, c->stream));
      k_fill_u32<<<blocks1d(nm, 256), 256, 0, c->stream>>>(bA, nm, (unsigned)nb);
      k_mig_bucket<<<blocks1d(nm, 256), 256, 0, c->stream>>>(mv, nm, NS, c->foffInc, c->ffill, vA);
      RH_LAUNCHED(c);
      k_mig_order_small<<<blocks1d(nb, 256), 256, 0, c->stream>>>(mv, nb, c->finc, c->foffInc, vA, bA);
      RH_LAUNCHED(c);
      if (maxInc > MIG_SMALL) {
         // the large buckets (each holds more than MIG_SMALL movers, so fewer
         // than nm / MIG_SMALL of them) listed in bB, their count in fmaxInc
         RH_CUDA(cudaMemsetAsync(c->fmaxInc, 0, sizeof(int), c->stream));
         k_mig_large_list<<<blocks1d(nb, 256), 256, 0, c->stream>>>(c->finc, nb, bB, c->fmaxInc);
         RH_LAUNCHED(c);
         const unsigned grid = (unsigned)std::min<long long>(nm / MIG_SMALL + 1, 4 * 148);
         k_mig_order_large<<<grid, MIG_LARGE_THREADS, 0, c->stream>>>(mv, c->finc, c->foffInc, vA, bA, bB, c->fmaxInc);
         RH_LAUNCHED(c);
      }
      k_mig_check<<<blocks1d(nb, 256), 256, 0, c->stream>>>(FS, NS, c->finc, c->fover);
      RH_LAUNCHED(c);
      RH_CUDA(cudaMemcpyAsync(over, c->fover, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      RH_CUDA(cudaStreamSynchronize(c->stream));
      *order = vA;
      *bucket = bA;
      return RHGPU_OK;
   }
   RH_TIME(c, "mig_radix_order");   // the fallback: a bucket with more than MIG_SMALL arrivals
   k_mig_sort_keys<<<blocks1d(nm, 256), 256, 0, c->stream>>>(mv, nm, NS, nb, kA, vA, bA);
   RH_LAUNCHED(c);
   const int kbits = 32 + bitsFor(std::max(NS > 1 ? NS - 1 : 1, c->injKeyMax)), bbits = bitsFor(nb);
   size_t s1 = 0, s2 = 0;
   cub::DeviceRadixSort::SortPairs(nullptr, s1, kA, kB, vA, vB, (int)nm, 0, kbits, c->stream);
   cub::DeviceRadixSort::SortPairs(nullptr, s2, bB, bA, vB, vA, (int)nm, 0, bbits, c->stream);
   rc = ensureSortTmp(c, std::max(s1, s2));
   if (rc) return rc;
   size_t sb = c->sortTmpBytes;
   RH_CUDA(cub::DeviceRadixSort::SortPairs(c->sortTmp, sb, kA, kB, vA, vB, (int)nm, 0, kbits, c->stream));
   k_gather_u32<<<blocks1d(nm, 256), 256, 0, c->stream>>>(bA, vB, nm, bB);
   RH_LAUNCHED(c);
   sb = c->sortTmpBytes;
   RH_CUDA(cub::DeviceRadixSort::SortPairs(c->sortTmp, sb, bB, bA, vB, vA, (int)nm, 0, bbits, c->stream));
   k_mig_check<<<blocks1d(nb, 256), 256, 0, c->stream>>>(FS, NS, c->finc, c->fover);
   RH_LAUNCHED(c);
   RH_CUDA(cudaMemcpyAsync(over, c->fover, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   *order = vA;
   *bucket = bA;
   return RHGPU_OK;
}

// exclusive prefix of a per-segment count array (NS+1 entries into c->ffirst); returns the total
int segPrefix(rhgpu_ctx* c, const int* cnt, long long* total) {
   const long long NS = c->fg.NS;
   k_int_to64<<<blocks1d(NS + 1, 256), 256, 0, c->stream>>>(cnt, NS, c->ftmp64);
   RH_CUDA(cudaGetLastError());
   if (int rc_ = scanExclusive64(c, c->ftmp64, c->ffirst, NS + 1)) return rc_;
   RH_CUDA(cudaMemcpyAsync(total, c->ffirst + NS, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   return RHGPU_OK;
}

// relayout of every species' next buffer with room for its pending arrivals (finc), order kept
// relays out the "next" buffers of the species in `mask` (bit s: species s)
// with room for their pending arrivals; the other species keep their layout
int fastRelayoutNext(rhgpu_ctx* c, unsigned mask) {
   RH_TIME(c, "fast_relayout");
   const long long NS = c->fg.NS;
   for (int s = 0; s < c->ns; ++s) {
      if (!((mask >> s) & 1u)) continue;
      SegHost& h = c->seg[s];
      const int nx = h.cur ^ 1;   // holds the step's particles; h.cur is free
      long long total = 0;
      int rc = fastLayout(c, h.cnt[nx], c->finc + (long long)s * NS, h.baseAlt, &total);
      if (rc) return rc;
      rc = segReserve(h, h.cur, total);
      if (rc) return rc;
      k_fast_relayout<<<(unsigned)NS, 128, 0, c->stream>>>(segView(h, nx), h.base, segView(h, h.cur), h.baseAlt);
      RH_CUDA(cudaGetLastError());
      std::swap(h.base, h.baseAlt);
      h.cur ^= 1;   // the relaid buffer takes the "next" role
      rc = segReserve(h, h.cur, total);
      if (rc) return rc;
   }
   RH_CUDA(cudaStreamSynchronize(c->stream));
   return fastMoverBuffers(c);
}

int fastUpload(rhgpu_ctx* c, int s, const uint32_t* counts, const double* particles, long long n) {
   const long long N = c->g.N, NS = c->fg.NS;
   int rc = ensureStaging(c, sizeof(double) * 7 * (size_t)(n > 0 ? n : 1) + sizeof(uint32_t) * (size_t)N + 64);
   if (rc) return rc;
   rc = ensureKeyCapacity(c, 2 * n + 2);
   if (rc) return rc;
   double* aos = (double*)c->staging;
   uint32_t* dcounts = (uint32_t*)((char*)c->staging + sizeof(double) * 7 * (size_t)(n > 0 ? n : 1));
   RH_CUDA(cudaMemcpyAsync(dcounts, counts, sizeof(uint32_t) * N, cudaMemcpyHostToDevice, c->stream));
   if (n) RH_CUDA(cudaMemcpyAsync(aos, particles, sizeof(double) * 7 * n, cudaMemcpyHostToDevice, c->stream));
   // cell of every record
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
   // segment of every record, stable sort by it
   rc = growBuffer(c->fsort, c->fsortCap, 2 * n + 2);
   if (rc) return rc;
   rc = growBuffer(c->flxTmp, c->flxTmpCap, n + 1);
   if (rc) return rc;
   unsigned* keyIn = (unsigned*)c->key;
   unsigned* keyOut = keyIn + (n + 1);
   unsigned* idxIn = (unsigned*)c->fsort;
   unsigned* idxOut = idxIn + (n + 1);
   if (n) {
      k_fast_seg_of<<<blocks1d(n, 256), 256, 0, c->stream>>>(c->g, c->fg, aos, pcell, n, keyIn, c->flxTmp);
      k_iota<<<blocks1d(n, 256), 256, 0, c->stream>>>(idxIn, n);
      RH_CUDA(cudaGetLastError());
      size_t sb = 0;
      cub::DeviceRadixSort::SortPairs(nullptr, sb, keyIn, keyOut, idxIn, idxOut, (int)n, 0, 32, c->stream);
      rc = ensureSortTmp(c, sb);
      if (rc) return rc;
      sb = c->sortTmpBytes;
      RH_CUDA(cub::DeviceRadixSort::SortPairs(c->sortTmp, sb, keyIn, keyOut, idxIn, idxOut, (int)n, 0, 32, c->stream));
   }
   SegHost& h = c->seg[s];
   // first sorted record of every segment and the counts, from the sorted keys
   k_sorted_bounds<<<blocks1d(n + 1, 256), 256, 0, c->stream>>>(keyOut, n, NS, c->ffirst);
   k_bounds_counts<<<blocks1d(NS, 256), 256, 0, c->stream>>>(c->ffirst, NS, h.cnt[h.cur]);
   RH_CUDA(cudaGetLastError());
   long long slots = 0;
   rc = fastLayout(c, h.cnt[h.cur], nullptr, h.base, &slots);
   if (rc) return rc;
   rc = segReserve(h, 0, slots);
   if (rc) return rc;
   rc = segReserve(h, 1, slots);
   if (rc) return rc;
   if (n) {
      k_fast_scatter_sorted<<<blocks1d(n, 256), 256, 0, c->stream>>>(aos, c->flxTmp, keyOut, idxOut, n, c->ffirst,
                                                                     segView(h, h.cur), h.base);
      RH_CUDA(cudaGetLastError());
   }
   RH_CUDA(cudaStreamSynchronize(c->stream));
   rc = fastExponents(c);
   if (rc) return rc;
   return fastMoverBuffers(c);
}

int fastNumParticles(rhgpu_ctx* c, int s, long long* n) {
   return segPrefix(c, c->seg[s].cnt[c->seg[s].cur], n);
}

int fastDownload(rhgpu_ctx* c, int s, uint32_t* counts, double* particles, long long capacity, long long* n_out) {
   const long long N = c->g.N, NS = c->fg.NS;
   long long tot = 0;
   int rc = fastNumParticles(c, s, &tot);   // leaves the segment offsets in c->ffirst
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
   const SegHost& h = c->seg[s];
   if (tot) {
      k_fast_cell_keys<<<(unsigned)NS, 128, 0, c->stream>>>(c->g, c->fg, segView(h, h.cur), h.base, c->ffirst, keyIn,
                                                           c->fsortSlots);
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
      k_fast_gather_records<<<blocks1d(tot, 256), 256, 0, c->stream>>>(segView(h, h.cur), c->fsortSlots, idxOut, tot, aos);
      RH_CUDA(cudaGetLastError());
   } else {
      RH_CUDA(cudaMemsetAsync(cellCnt, 0, sizeof(int) * N, c->stream));
   }
   RH_CUDA(cudaMemcpyAsync(counts, cellCnt, sizeof(uint32_t) * N, cudaMemcpyDeviceToHost, c->stream));
   if (tot && particles) RH_CUDA(cudaMemcpyAsync(particles, aos, sizeof(double) * 7 * tot, cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   *n_out = tot;
   return RHGPU_OK;
}

// fused push + deposit, then placement of the particles that left their segment
// the particle sources of this step, appended to the mover list
template <class MV>
int injectAll(rhgpu_ctx* c, MV* movers, long long moverCap) {
   for (const InjHost& h : c->inj) {
      if (h.d.ncells == 0) continue;
      RH_TIME(c, h.d.type == INJ_EXOSPHERE                                  ? "inject_exosphere"
                 : (h.d.type == INJ_IONOSPHERE || h.d.type == INJ_CHAPMAN) ? "inject_ionosphere"
                                                                            : "inject_inflow");
      unsigned grid = blocks1d(h.d.ncells, 128);
      if (h.d.list) {   // most cells of a rate-based source draw nothing: list the others first
         RH_CUDA(cudaMemsetAsync(h.list + h.d.ncells, 0, sizeof(int), c->stream));
         k_inject_select<<<grid, 128, 0, c->stream>>>(h.d, c->timestep, h.list, h.list + h.d.ncells);
         RH_LAUNCHED(c);
         grid = std::min(grid, 2u * 148u);
      }
      k_inject<MV><<<grid, 128, 0, c->stream>>>(c->g, c->fg, h.d, c->timestep, movers, c->fb.nmovers, moverCap,
                                                c->injCnt, c->err);
      RH_LAUNCHED(c);
   }
   return RHGPU_OK;
}

// fast path: each output population's share of this step's deposit added to
// its averages: the stayers (the next buffer before the arrivals are placed)
// by segment, then every deposited mover (left its segment, or deposited in it
// and removed by a boundary)
int fastAverages(rhgpu_ctx* c, long long nm) {
   const long long N = c->g.N;
   FastBufs& A = c->avgFB;
   if (!A.RP) {
      RH_CUDA(cudaMalloc(&A.RP, sizeof(double) * 16 * c->fg.nrows * c->g.nx));
      RH_CUDA(cudaMalloc(&A.RPB, sizeof(double) * 16 * c->fg.nrows * c->fg.nseg));
      RH_CUDA(cudaMalloc(&A.MMlo, sizeof(unsigned long long) * 4 * N));
      RH_CUDA(cudaMalloc(&A.MMhi, sizeof(unsigned long long) * 4 * N));
      RH_CUDA(cudaMemset(A.RPB, 0, sizeof(double) * 16 * c->fg.nrows * c->fg.nseg));
      RH_CUDA(cudaMemset(A.MMlo, 0, sizeof(unsigned long long) * 4 * N));
      RH_CUDA(cudaMemset(A.MMhi, 0, sizeof(unsigned long long) * 4 * N));
   }
   A.scaleR = c->fb.scaleR;
   A.scaleJ = c->fb.scaleJ;
   const double hiR = std::ldexp(1.0, 64 - c->kR), loR = std::ldexp(1.0, -c->kR);
   const double hiJ = std::ldexp(1.0, 64 - c->kJ), loJ = std::ldexp(1.0, -c->kJ);
   FastSpecies FS = fastSpecies(c);
   FastSpecies stay = FS;
   for (int s = 0; s < c->ns; ++s) stay.st[s].cur = FS.st[s].nxt;
   for (int grp = 0; grp < c->avgGroups; ++grp) {
      unsigned mask = 0;
      for (int s = 0; s < c->ns; ++s)
         if (c->avgGroupOf[s] == grp && c->sp[s].accumulate && c->seg[s].a[c->seg[s].cur][0]) mask |= 1u << s;
      if (!mask) continue;
      RH_TIME(c, "population_averages");
      switch (perMask(c->g)) {
#define RH_FAST_AVG(M)                                                                                         \
   case M:                                                                                                      \
      k_fast_avg_deposit<M><<<(unsigned)c->fg.NS, FT, 0, c->stream>>>(c->g, c->fg, stay, mask, A);              \
      break;
         RH_FAST_AVG(0) RH_FAST_AVG(1) RH_FAST_AVG(2) RH_FAST_AVG(3) RH_FAST_AVG(4) RH_FAST_AVG(5) RH_FAST_AVG(6)
         RH_FAST_AVG(7)
#undef RH_FAST_AVG
      }
      RH_LAUNCHED(c);
      if (nm > 0) {
         k_fast_avg_movers<<<blocks1d(nm, 128), 128, 0, c->stream>>>(c->g, c->fg, FS, c->fb.movers, nm, mask, A);
         RH_LAUNCHED(c);
      }
      k_fast_avg_gather<<<cellGrid(c->g), cellBlock(), 0, c->stream>>>(c->g, c->fg, A, hiR, loR, hiJ, loJ,
                                                                      c->avgN + (long long)grp * N, c->avgV + 3LL * grp * N);
      RH_LAUNCHED(c);
   }
   return RHGPU_OK;
}

// k_fast_push_deposit uses more than the 48 KB of static shared memory: its
// limit is raised once per instantiation (and device) before the launch
template <int PER, bool EXTRA>
int launchPushDeposit(rhgpu_ctx* c, const FastSpecies& FS, const PushParams& pp) {
   static bool raised[64] = {};
   int dev = 0;
   RH_CUDA(cudaGetDevice(&dev));
   if (dev < 0 || dev >= 64) return fail(RHGPU_ERR_CUDA, "device index out of range");
   if (!raised[dev]) {
      RH_CUDA(cudaFuncSetAttribute(k_fast_push_deposit<PER, EXTRA>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)PUSH_DEPOSIT_SMEM));
      raised[dev] = true;
   }
   k_fast_push_deposit<PER, EXTRA><<<(unsigned)c->fg.NS, FT, PUSH_DEPOSIT_SMEM, c->stream>>>(
       c->g, c->f, c->fg, FS, pp, c->fb, c->cntD, c->cntU, c->err);
   return RHGPU_OK;
}

int fastPush(rhgpu_ctx* c) {
   c->timestep += 1;
   if (c->P.initial_flow_through_period < c->t && c->useIFT) c->useIFT = 0;
   PushParams pp;
   pp.useIFT = c->useIFT;
   pp.use_ep = c->P.use_electron_pressure;
   pp.use_gravity = c->P.use_gravity;
   pp.GMdt = c->P.GMdt;
   pp.maxVi2 = c->P.max_ion_speed2;
   pp.avgList = c->avgGroups > 0;
   const long long N = c->g.N, NS = c->fg.NS;
   RH_CUDA(cudaMemsetAsync(c->fb.touched, 0, (size_t)N + 16, c->stream));
   RH_CUDA(cudaMemsetAsync(c->fb.nmovers, 0, sizeof(unsigned long long), c->stream));
   {
      RH_TIME(c, "fast_push_deposit");
      const FastSpecies FS = fastSpecies(c);
      int rc = RHGPU_OK;
      switch (perMask(c->g)) {
#define RH_FAST_PD(M)                                                                                           \
   case M:                                                                                                        \
      if (c->avgGroups || c->f.gc)                                                                                \
         rc = launchPushDeposit<M, true>(c, FS, pp);                                                              \
      else                                                                                                        \
         rc = launchPushDeposit<M, false>(c, FS, pp);                                                             \
      break;
         RH_FAST_PD(0) RH_FAST_PD(1) RH_FAST_PD(2) RH_FAST_PD(3) RH_FAST_PD(4) RH_FAST_PD(5) RH_FAST_PD(6) RH_FAST_PD(7)
#undef RH_FAST_PD
      }
      if (rc) return rc;
      RH_LAUNCHED(c);
   }
   {
      const int rc = injectAll(c, c->fb.movers, c->fb.moverCap);
      if (rc) return rc;
   }
   unsigned long long nm = 0;
   RH_CUDA(cudaMemcpyAsync(&nm, c->fb.nmovers, sizeof nm, cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   if ((long long)nm > c->fb.moverCap) return fail(RHGPU_ERR_CAPACITY, "mover list overflow");
   if (nm > 0) {
      RH_TIME(c, "fast_mover_deposit");
      k_fast_mover_deposit<<<blocks1d(nm, 128), 128, 0, c->stream>>>(c->g, c->fg, fastSpecies(c), c->fb, nm);
      RH_LAUNCHED(c);
   }
   if (c->avgGroups) {
      const int rc = fastAverages(c, (long long)nm);
      if (rc) return rc;
   }
   if (nm > 0) {
      const long long nb = (long long)c->ns * NS;
      int over = 0;
      {
         RH_TIME(c, "fast_migrate");
         unsigned *order = nullptr, *bkt = nullptr;
         int rc = migSort(c, c->fb.movers, (long long)nm, fastSpecies(c), &order, &bkt, &over);
         if (rc) return rc;
         if (over) {
            // some segments lack room for their arrivals: relayout with room for them
            rc = fastRelayoutNext(c, (unsigned)over);
            if (rc) return rc;
            RH_CUDA(cudaMemsetAsync(c->fover, 0, sizeof(int), c->stream));
            k_mig_check<<<blocks1d(nb, 256), 256, 0, c->stream>>>(fastSpecies(c), NS, c->finc, c->fover);
            RH_LAUNCHED(c);
            RH_CUDA(cudaMemcpyAsync(&over, c->fover, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
            RH_CUDA(cudaStreamSynchronize(c->stream));
            if (over) return fail(RHGPU_ERR_CAPACITY, "segment relayout did not make room");
         }
         k_fast_mig_place<<<blocks1d(nm, 256), 256, 0, c->stream>>>(fastSpecies(c), NS, nb, c->fb.movers, order, bkt, c->foffInc,
                                                                 (long long)nm);
         RH_LAUNCHED(c);
         k_mig_counts<<<blocks1d(nb, 256), 256, 0, c->stream>>>(fastSpecies(c), NS, c->finc);
         RH_LAUNCHED(c);
      }
   }
   for (int s = 0; s < c->ns; ++s) c->seg[s].cur ^= 1;
   return RHGPU_OK;
}

int fastGather(rhgpu_ctx* c) {
   RH_TIME(c, "fast_gather");
   k_fast_fold_boundary<<<blocks1d(16 * c->fg.nrows * c->fg.nseg, 256), 256, 0, c->stream>>>(c->g, c->fg, c->fb);
   RH_LAUNCHED(c);
   const double hiR = std::ldexp(1.0, 64 - c->kR), loR = std::ldexp(1.0, -c->kR);
   const double hiJ = std::ldexp(1.0, 64 - c->kJ), loJ = std::ldexp(1.0, -c->kJ);
   if (c->f.gc)
      k_fast_gather<true><<<cellGrid(c->g), cellBlock(), 0, c->stream>>>(c->g, c->f, c->fg, c->fb, hiR, loR, hiJ, loJ,
                                                                        c->P.min_ion_charge_density, c->cntU);
   else
      k_fast_gather<false><<<cellGrid(c->g), cellBlock(), 0, c->stream>>>(c->g, c->f, c->fg, c->fb, hiR, loR, hiJ, loJ,
                                                                         c->P.min_ion_charge_density, c->cntU);
   RH_LAUNCHED(c);
   return RHGPU_OK;
}

template int migSort<Mover, FastSpecies>(rhgpu_ctx*, const Mover*, long long, const FastSpecies&, unsigned**, unsigned**,
                                         int*);
template int migSort<Mover32, F32Set>(rhgpu_ctx*, const Mover32*, long long, const F32Set&, unsigned**, unsigned**, int*);
template int injectAll<Mover>(rhgpu_ctx*, Mover*, long long);
template int injectAll<Mover32>(rhgpu_ctx*, Mover32*, long long);

}  // namespace rhh
