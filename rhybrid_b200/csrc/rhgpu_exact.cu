// The exact particle path of the C ABI: per-cell particle storage in the
// reference's order, the push, migration, deposit and particle boundary
// conditions launched in the reference's order (src/user.cpp:118-134), and the
// allocation-free deposit entry point rhgpu_accumulate_noalloc.
#include "rhgpu_host.h"

namespace rhh {

// Scratch of rhgpu_accumulate_noalloc: the exact-path deposit's 108 per-cell
// sums (S[e*N + c]) for grids of up to RHGPU_NOALLOC_MAX_CELLS cells, in the
// module's static device memory; every entry of a cell is written before it
// is read, so nothing needs clearing. Its device address is looked up once
// per device.
__device__ __align__(256) double g_noallocScratch[108 * (size_t)RHGPU_NOALLOC_MAX_CELLS];
constexpr int NOALLOC_MAX_DEVICES = 64;
// host threads may make their first call on a device at the same time: each
// looks the address up and stores the same value
std::atomic<double*> g_noallocPtr[NOALLOC_MAX_DEVICES] = {};

int allocStore(PStore& s, long long cap, long long N) {
   s.cap = cap;
   s.nslots = 0;
   for (int a = 0; a < 7; ++a) RH_CUDA(cudaMalloc(&s.a[a], sizeof(double) * (cap > 0 ? cap : 1)));
   RH_CUDA(cudaMalloc(&s.pcell, sizeof(int) * (cap > 0 ? cap : 1)));
   RH_CUDA(cudaMalloc(&s.start, sizeof(long long) * (N + 1)));
   RH_CUDA(cudaMalloc(&s.alive, sizeof(int) * N));
   RH_CUDA(cudaMemset(s.start, 0, sizeof(long long) * (N + 1)));
   RH_CUDA(cudaMemset(s.alive, 0, sizeof(int) * N));
   return RHGPU_OK;
}

void freeStore(PStore& s) {
   for (int a = 0; a < 7; ++a) cudaFree(s.a[a]);
   cudaFree(s.pcell);
   cudaFree(s.start);
   cudaFree(s.alive);
   std::memset(&s, 0, sizeof s);
}

int migrate(rhgpu_ctx* c, int s) {
   PStore& P = c->ps[s];
   PStore& Q = c->alt[s];
   const GridInfo& g = c->g;
   {
      RH_TIME(c, "mig_count");
      k_mig_count<<<blocks1d(g.N, 128), 128, 0, c->stream>>>(g, P, c->key, c->outCount, c->rank);
      RH_LAUNCHED(c);
   }
   {
      RH_TIME(c, "mig_incount");
      k_mig_incount<<<cellGrid(g), cellBlock(), 0, c->stream>>>(g, c->outCount, c->inPrefix, c->newCount);
      RH_LAUNCHED(c);
   }
   // exclusive scan of the new counts into Q.start[0..N], Q.start[N] = total
   RH_CUDA(cudaMemsetAsync(c->newCount + g.N, 0, sizeof(long long), c->stream));
   {
      RH_TIME(c, "mig_scan");
      if (int rc_ = scanExclusive64(c, c->newCount, Q.start, g.N + 1)) return rc_;
   }
   long long total = 0;
   RH_CUDA(cudaMemcpyAsync(&total, Q.start + g.N, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   if (total > Q.cap) return fail(RHGPU_ERR_CAPACITY, "particle capacity exceeded in migration");
   Q.nslots = total;
   {
      RH_TIME(c, "mig_scatter");
      k_mig_scatter<<<blocks1d(P.nslots > 0 ? P.nslots : 1, 256), 256, 0, c->stream>>>(g, P, Q, c->key, c->rank,
                                                                                      c->inPrefix, Q.start, c->err);
      RH_LAUNCHED(c);
   }
   {
      RH_TIME(c, "mig_alive");
      k_set_alive_from_count<<<blocks1d(g.N, 256), 256, 0, c->stream>>>(g.N, c->newCount, Q.alive);
      RH_LAUNCHED(c);
   }
   std::swap(c->ps[s], c->alt[s]);
   return RHGPU_OK;
}

int pushAll(rhgpu_ctx* c) {
   c->timestep += 1;
   // initial flow-through switch-off (user.cpp:52-59)
   if (c->P.initial_flow_through_period < c->t && c->useIFT) c->useIFT = 0;
   PushParams pp;
   pp.useIFT = c->useIFT;
   pp.use_ep = c->P.use_electron_pressure;
   pp.use_gravity = c->P.use_gravity;
   pp.GMdt = c->P.GMdt;
   pp.maxVi2 = c->P.max_ion_speed2;
   pp.avgList = c->avgGroups > 0;
   for (int s = 0; s < c->ns; ++s) {
      PStore& P = c->ps[s];
      if (!P.start) continue;   // species without uploaded particles
      int rc = ensureKeyCapacity(c, P.nslots);
      if (rc) return rc;
      if (P.nslots > 0) {
         RH_TIME(c, "push");
         k_push<<<blocks1d(P.nslots, 256), 256, 0, c->stream>>>(c->g, c->f, P, speciesDev(c, s), pp, c->key,
                                                                c->cntU, c->cntD, c->err, s);
         RH_LAUNCHED(c);
      }
      rc = migrate(c, s);
      if (rc) return rc;
   }
   return RHGPU_OK;
}

// exact-path deposit with the 108 per-cell sums in S (108 * N doubles)
int depositExact(rhgpu_ctx* c, double* S) {
   int last = -1, first = -1;
   for (int s = 0; s < c->ns; ++s)
      if (deposits(c, s)) { if (first < 0) first = s; last = s; }
   const GridInfo& g = c->g;
   if (last < 0) {
      RH_TIME(c, "deposit_gather");
      k_deposit_finalize_only<<<cellGrid(g), cellBlock(), 0, c->stream>>>(g, c->f, c->P.min_ion_charge_density, c->cntU);
      RH_LAUNCHED(c);
   }
   for (int s = 0; s < c->ns; ++s) {
      if (!deposits(c, s)) continue;
      {
         RH_TIME(c, "deposit_cell");
         const unsigned nblk = (unsigned)std::min<long long>(blocks1d(g.N, DEP_WARPS), DEP_GRID);
         k_deposit_cell<<<nblk, 32 * DEP_WARPS, 0, c->stream>>>(g, c->ps[s], c->sp[s].q, S, c->err);
         RH_LAUNCHED(c);
      }
      {
         RH_TIME(c, "deposit_gather");
         k_deposit_gather<<<cellGrid(g), cellBlock(), 0, c->stream>>>(g, c->f, S, s == first, s == last,
                                                                      c->P.min_ion_charge_density, c->cntU);
         RH_LAUNCHED(c);
      }
      const int grp = c->avgGroups ? c->avgGroupOf[s] : -1;
      if (grp >= 0) {
         RH_TIME(c, "population_averages");
         k_deposit_gather_avg<<<cellGrid(g), cellBlock(), 0, c->stream>>>(g, S, c->avgN + (long long)grp * g.N,
                                                                          c->avgV + 3LL * grp * g.N);
         RH_LAUNCHED(c);
      }
   }
   return RHGPU_OK;
}

int accumulateAll(rhgpu_ctx* c) {
   if (!c->S) RH_CUDA(cudaMalloc(&c->S, sizeof(double) * 108 * c->g.N));
   return depositExact(c, c->S);
}

int boundariesAll(rhgpu_ctx* c) {
   for (int s = 0; s < c->ns; ++s) {
      if (!c->ps[s].start) continue;
      if (c->next > 0) {
         RH_TIME(c, "bc_exterior");
         k_bc_exterior<<<blocks1d(c->next, 128), 128, 0, c->stream>>>(c->g, c->ps[s], c->ext, c->next, c->cntD, s);
         RH_LAUNCHED(c);
      }
      if (c->nobst > 0) {
         RH_TIME(c, "bc_obstacle");
         k_bc_obstacle<<<blocks1d(c->nobst, 64), 64, 0, c->stream>>>(c->g, c->ps[s], c->obst, c->nobst,
                                                                     c->sp[s].R2_obstacle, c->cntD, s);
         RH_LAUNCHED(c);
      }
   }
   return RHGPU_OK;
}

}  // namespace rhh

extern "C" {

int rhgpu_accumulate_noalloc(rhgpu_ctx* c) {
   if (!c) return fail(RHGPU_ERR_ARG, "null context");
   if (c->path != RHGPU_PATH_EXACT) return fail(RHGPU_ERR_STATE, "accumulate_noalloc: the context must use RHGPU_PATH_EXACT");
   if (c->g.N > RHGPU_NOALLOC_MAX_CELLS)
      return fail(RHGPU_ERR_ARG, "accumulate_noalloc: the grid has more cells than RHGPU_NOALLOC_MAX_CELLS (" +
                                     std::to_string(RHGPU_NOALLOC_MAX_CELLS) + ")");
   if (c->device < 0 || c->device >= NOALLOC_MAX_DEVICES) return fail(RHGPU_ERR_ARG, "accumulate_noalloc: device index out of range");
   RH_CUDA(cudaSetDevice(c->device));
   double* S = g_noallocPtr[c->device].load();
   if (!S) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noallocScratch);
      if (e != cudaSuccess || !p)
         return fail(RHGPU_ERR_CUDA, std::string("accumulate_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      S = (double*)p;
      g_noallocPtr[c->device].store(S);
   }
   // the kernel timer creates events on demand: off for this call
   const bool timing = c->timing;
   c->timing = false;
   const int rc = depositExact(c, S);
   c->timing = timing;
   if (rc) return rc;
   return checkDeviceError(c);
}

}  // extern "C"
