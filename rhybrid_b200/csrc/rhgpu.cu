// rhgpu: C ABI (include/rhgpu.h) of the B200 hybrid-PIC hot path.
//
// Host side of the library: context and device memory, the per-step launch
// sequence replaying RHybrid's propagate() (src/user.cpp:118-134), upload /
// download with the ParGrid layout, counters, timing and reductions. The
// device code is in k_particles.cuh (push, migration, deposit, particle
// boundary conditions) and k_fields.cuh (propagateB).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_reduce.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <atomic>

#include "../../include/rhgpu.h"
#include "k_fields.cuh"
#include "k_particles.cuh"
#include "k_fast.cuh"
#include "k_diag.cuh"
#include "k_f32.cuh"
#include "k_denoise.cuh"
#include "k_inject.cuh"
#include "k_avg.cuh"
#include "k_fill.cuh"
#include "k_scan.cuh"
#include "rh_logs.h"

using namespace rh;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
   g_err = msg;
   return code;
}

#define RH_CUDA(call)                                                                     \
   do {                                                                                   \
      cudaError_t e_ = (call);                                                            \
      if (e_ != cudaSuccess) return fail(RHGPU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
   } while (0)

const int MAX_SPECIES = 8;
const int NCNT_U = 32;   // field counters 0..15, species MaxVi at 16+s

int arrayDim(int id) {
   return (id == RHGPU_CELL_RHOQI || id == RHGPU_NODE_RHOQI || id == RHGPU_NODE_ETA) ? 1 : 3;
}

// neumannCell rules (hybrid_propagator.cpp:456-652) in the reference's order:
// missing-wall mask (1=-x 2=+y 4=-y 8=+z 16=-z 32=+x) and source offset
const int NEU_CELL[26][4] = {
   {1, +1, 0, 0}, {2, 0, -1, 0}, {4, 0, +1, 0}, {8, 0, 0, -1}, {16, 0, 0, +1}, {32, -1, 0, 0},
   {1 | 4, +1, +1, 0}, {1 | 2, +1, -1, 0}, {32 | 4, -1, +1, 0}, {32 | 2, -1, -1, 0},
   {1 | 16, +1, 0, +1}, {1 | 8, +1, 0, -1}, {32 | 16, -1, 0, +1}, {32 | 8, -1, 0, -1},
   {4 | 16, 0, +1, +1}, {4 | 8, 0, +1, -1}, {2 | 16, 0, -1, +1}, {2 | 8, 0, -1, -1},
   {1 | 4 | 16, +1, +1, +1}, {1 | 4 | 8, +1, +1, -1}, {1 | 2 | 16, +1, -1, +1}, {1 | 2 | 8, +1, -1, -1},
   {32 | 4 | 16, -1, +1, +1}, {32 | 4 | 8, -1, +1, -1}, {32 | 2 | 16, -1, -1, +1}, {32 | 2 | 8, -1, -1, -1}};

// neumannFace rules (hybrid_propagator.cpp:673-901): per component, source offset (use flag)
struct FaceRule { int mask; int src[3][3]; int use[3]; };
const FaceRule NEU_FACE[] = {
   {1, {{0, 0, 0}, {+1, 0, 0}, {+1, 0, 0}}, {0, 1, 1}},
   {2, {{0, -1, 0}, {0, 0, 0}, {0, -1, 0}}, {1, 0, 1}},
   {4, {{0, +1, 0}, {0, 0, 0}, {0, +1, 0}}, {1, 0, 1}},
   {8, {{0, 0, -1}, {0, 0, -1}, {0, 0, 0}}, {1, 1, 0}},
   {16, {{0, 0, +1}, {0, 0, +1}, {0, 0, 0}}, {1, 1, 0}},
   {32, {{0, 0, 0}, {-1, 0, 0}, {-1, 0, 0}}, {0, 1, 1}},
   {1 | 4, {{0, +1, 0}, {+1, 0, 0}, {+1, +1, 0}}, {1, 1, 1}},
   {1 | 2, {{0, -1, 0}, {0, 0, 0}, {+1, -1, 0}}, {1, 0, 1}},
   {32 | 4, {{0, 0, 0}, {-1, 0, 0}, {-1, +1, 0}}, {0, 1, 1}},
   {32 | 2, {{0, 0, 0}, {0, 0, 0}, {-1, -1, 0}}, {0, 0, 1}},
   {1 | 16, {{0, 0, +1}, {+1, 0, +1}, {+1, 0, 0}}, {1, 1, 1}},
   {1 | 8, {{0, 0, -1}, {+1, 0, -1}, {0, 0, 0}}, {1, 1, 0}},
   {32 | 16, {{0, 0, 0}, {-1, 0, +1}, {-1, 0, 0}}, {0, 1, 1}},
   {32 | 8, {{0, 0, 0}, {-1, 0, -1}, {0, 0, 0}}, {0, 1, 0}},
   {4 | 16, {{0, +1, +1}, {0, 0, +1}, {0, +1, 0}}, {1, 1, 1}},
   {4 | 8, {{0, +1, -1}, {0, 0, -1}, {0, 0, 0}}, {1, 1, 0}},
   {2 | 16, {{0, -1, +1}, {0, 0, 0}, {0, -1, 0}}, {1, 0, 1}},
   {2 | 8, {{0, -1, -1}, {0, 0, 0}, {0, 0, 0}}, {1, 0, 0}},
   {1 | 4 | 16, {{0, +1, +1}, {+1, 0, +1}, {+1, +1, 0}}, {1, 1, 1}},
   {1 | 4 | 8, {{0, +1, -1}, {+1, 0, -1}, {0, 0, 0}}, {1, 1, 0}},
   {1 | 2 | 16, {{0, -1, +1}, {0, 0, 0}, {+1, -1, 0}}, {1, 0, 1}},
   {1 | 2 | 8, {{0, -1, -1}, {0, 0, 0}, {0, 0, 0}}, {1, 0, 0}},
   {32 | 4 | 16, {{0, 0, 0}, {-1, 0, +1}, {-1, +1, 0}}, {0, 1, 1}},
   {32 | 4 | 8, {{0, 0, 0}, {-1, 0, -1}, {0, 0, 0}}, {0, 1, 0}},
   {32 | 2 | 16, {{0, 0, 0}, {0, 0, 0}, {-1, -1, 0}}, {0, 0, 1}},
};

NeumannTables buildNeumannTables() {
   NeumannTables t;
   std::memset(&t, 0, sizeof t);
   for (int m = 0; m < 64; ++m) {
      for (int r = 0; r < 26; ++r) {
         if ((m & NEU_CELL[r][0]) != NEU_CELL[r][0]) continue;
         for (int a = 0; a < 3; ++a) t.cellSrc[m][a] = (signed char)NEU_CELL[r][1 + a];
      }
      for (const FaceRule& fr : NEU_FACE) {
         if ((m & fr.mask) != fr.mask) continue;
         for (int l = 0; l < 3; ++l) {
            if (!fr.use[l]) continue;
            t.faceUse[m][l] = 1;
            for (int a = 0; a < 3; ++a) t.faceSrc[m][l][a] = (signed char)fr.src[l][a];
         }
      }
   }
   return t;
}

struct TimerRec { int cls; int ea, eb; };

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

// one species' FP32-form storage: cell index, FP32 offsets and velocities
struct F32Host {
   int* cell[2] = {};
   float* o[2][3] = {};
   float* v[2][3] = {};
   int* cnt[2] = {};
   long long capOf[2] = {0, 0};
   long long* base = nullptr;
   long long* baseAlt = nullptr;
   int cur = 0;
   double w = 0.0;   // macroparticle weight of the species
};

// one species' row-segment storage: two particle buffers sharing the layout `base`
struct SegHost {
   double* a[2][7] = {};
   unsigned char* lx[2] = {};
   int* cnt[2] = {};
   long long capOf[2] = {0, 0};   // slots allocated in each buffer
   long long* base = nullptr;      // NS+1 slot offsets
   long long* baseAlt = nullptr;   // NS+1, relayout target
   int cur = 0;                    // buffer holding the current particles
};

}  // namespace

struct InjHost {
   InjDev d;
   int* cells = nullptr;     // device copy of d.cells
   double* rates = nullptr;  // device copy of d.rates (exosphere, ionospheres)
   int* list = nullptr;      // rate-based sources: cells drawing particles this step, then their count
   // rate-based sources, host copy: the cells with a positive expected
   // number of macroparticles per step, and that number
   std::vector<int> rateCells;
   std::vector<double> rateValues;
};

struct rhgpu_ctx {
   rhgpu_params P;
   GridInfo g;
   int device = 0;
   std::vector<InjHost> inj;      // particle sources
   double* injCnt = nullptr;      // 3 x ns: injected weight, macroparticles, weight v^2
   long long injKeyMax = 0;       // largest mover key source id of the sources
   cudaStream_t stream = nullptr;
   int ns = 0;
   rhgpu_species sp[MAX_SPECIES];
   Fields f;
   FieldParams fp;
   double* arr[RHGPU_NUM_ARRAYS] = {};
   double* tmp3 = nullptr;
   uint8_t* flags = nullptr;
   int* ext = nullptr;
   int next = 0;
   int* obst = nullptr;
   int nobst = 0;
   PStore ps[MAX_SPECIES];
   PStore alt[MAX_SPECIES];   // migration target buffers
   int* key = nullptr;
   int* rank = nullptr;
   long long keyCap = 0;
   int* outCount = nullptr;
   int* inPrefix = nullptr;
   long long* newCount = nullptr;
   void* scanTmp = nullptr;
   size_t scanTmpBytes = 0;
   double* S = nullptr;
   unsigned long long* cntU = nullptr;
   double* cntD = nullptr;
   unsigned* err = nullptr;
   double t = 0;
   long long timestep = 0;
   int useIFT = 0;
   double gridAvgCounter = 0;
   bool timing = false;
   std::vector<cudaEvent_t> evPool;   // per-launch event pairs of the last rhgpu_step
   size_t evUsed = 0;
   std::vector<TimerRec> recs;
   std::vector<std::string> clsNames;
   long long launches = 0;
   long long launchesStep = 0;
   void* staging = nullptr;      // particle record staging for upload/download
   size_t stagingBytes = 0;
   // fast path (row-segment storage)
   int path = RHGPU_PATH_FAST;
   bool uploaded = false;
   FastGeom fg;
   SegHost seg[MAX_SPECIES];
   FastBufs fb = {};
   unsigned char* segInnerDev = nullptr;   // fb.segInner: per segment, an obstacle cell within one step
   int* finc = nullptr;                 // arrivals per (species, segment)
   unsigned long long* mkey = nullptr;  // migration sort: 2 x mcap mover keys
   unsigned* mval = nullptr;            // 2 x mcap mover indices
   unsigned* mbkt = nullptr;            // 2 x mcap destination buckets
   long long mcap = 0;
   int* ffill = nullptr;                // ns*NS fill counters of the small-bucket placement
   int* fmaxInc = nullptr;              // largest arrivals of a bucket
   int* fover = nullptr;                // 16 bytes
   int kR = 0, kJ = 0;
   void* sortTmp = nullptr;
   size_t sortTmpBytes = 0;
   long long* fcap = nullptr;           // NS+1
   long long* ffirst = nullptr;         // NS+1
   long long* ftmp64 = nullptr;         // NS+1
   long long* ftmpCellStart = nullptr;  // N+1
   long long* ftmpInc64 = nullptr;      // ns*NS+1
   long long* foffInc = nullptr;        // ns*NS+1
   unsigned* fsort = nullptr;
   long long fsortCap = 0;
   unsigned long long* fsortSlots = nullptr;
   long long fsortSlotsCap = 0;
   unsigned char* flxTmp = nullptr;
   long long flxTmpCap = 0;
   long long capHint[MAX_SPECIES] = {};
   double* diagPart = nullptr;          // DIAG_BLOCKS x DIAG_FS partial rows of rhgpu_reduce_diagnostics
   double* rhoM = nullptr;              // N: total ion mass density of the field log
   unsigned long long* rhoMfix = nullptr;   // 2N: its fixed-point sums (lo, hi)
   // temporal averages of the output populations (rhgpu_set_population_averages)
   int avgGroups = 0;
   int avgGroupOf[MAX_SPECIES] = {};
   double* avgN = nullptr;              // avgGroups x N charge sums
   double* avgV = nullptr;              // avgGroups x 3N current sums (component planes)
   double* avgOut = nullptr;            // 4N output staging
   FastBufs avgFB = {};                 // fast path: row partials and fixed-point sums of one population
   double* gridCnt = nullptr;           // GC_PLANES x N grid constraint counters (c->f.gc when on)
   // log files (rhgpu_log_*)
   LogFiles* logs = nullptr;
   int logInner = 0;
   double logTStart = 0.0;
   double logMaxB = 0.0;
   // FP32 precision form
   bool f32ready = false;
   F32Host f32[MAX_SPECIES];
   F32Bufs f32b = {};
   // learned denoiser applied to the moments before the field update
   struct rhgpu_dn* dn = nullptr;
   bool dnOn = false;
};

// learned denoiser: parameters, optimiser state, activations and the training pairs
struct rhgpu_dn {
   int device = 0;
   cudaStream_t stream = nullptr;
   DnGrid g;
   double sr = 1.0, sj = 1.0;            // normalization of rho and J
   float* params = nullptr;              // DN_PARAMS, FP32 master copy
   float* grad = nullptr;                // DN_PARAMS
   float* m = nullptr;                   // Adam moments
   float* v = nullptr;
   unsigned char* mask = nullptr;        // trainable entries
   __nv_bfloat16* bimg = nullptr;        // UMMA B images: 3 layers forward + 3 transposed, TC_BIMG bytes each
   unsigned* err = nullptr;              // device error word of the convolutions (RHGPU_DEVERR_DENOISER)
   unsigned* act[3] = {};                // BF16 inputs of layers 0..2 (16 channels)
   unsigned* dY[3] = {};                 // BF16 output gradients of layers 0..2
   float* res = nullptr;                 // normalized FP32 input (N x 4)
   float* out32 = nullptr;               // network output (N x 4)
   float* part = nullptr;                // weight-gradient partials
   long long partRows = 0;
   double* lossPart = nullptr;
   double* acc = nullptr;                // subsample deposit sums (4 x N)
   float* pairIn = nullptr;              // ring of training pairs: inputs (N x 4 each)
   float* pairOut = nullptr;             // targets
   int pairCap = 0, pairCount = 0, pairNext = 0;
   long long adamStep = 0;
   int border = 0;                       // loss mask width at non-periodic faces (crop training)
   long long fullN = 0;                  // crop pairs: the source grid's deposits (normalized, 4 x fullN)
   double* fullAcc = nullptr;
   float* fullIn = nullptr;
   float* fullOut = nullptr;
   unsigned long long rng = 0x9e3779b97f4a7c15ull;
};

namespace {

dim3 cellBlock() { return dim3(32, 4, 1); }
dim3 cellGrid(const GridInfo& g) { return dim3((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz); }
unsigned blocks1d(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// Kernel timing: with timing on, every launch is bracketed by a pair of CUDA
// events recorded on the context's stream (no synchronisation); the elapsed
// times are summed per kernel class by rhgpu_get_timing.
int timerBegin(rhgpu_ctx* c, const char* name) {
   if (!c->timing) return -1;
   int cls = -1;
   for (size_t q = 0; q < c->clsNames.size(); ++q)
      if (c->clsNames[q] == name) { cls = (int)q; break; }
   if (cls < 0) { c->clsNames.push_back(name); cls = (int)c->clsNames.size() - 1; }
   while (c->evPool.size() < c->evUsed + 2) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      c->evPool.push_back(e);
   }
   TimerRec r{cls, (int)c->evUsed, (int)c->evUsed + 1};
   c->evUsed += 2;
   cudaEventRecord(c->evPool[r.ea], c->stream);
   c->recs.push_back(r);
   return (int)c->recs.size() - 1;
}
void timerEnd(rhgpu_ctx* c, int r) {
   if (r >= 0) cudaEventRecord(c->evPool[c->recs[r].eb], c->stream);
}
struct KScope {
   rhgpu_ctx* c;
   int r;
   KScope(rhgpu_ctx* c_, const char* n) : c(c_), r(timerBegin(c_, n)) {}
   ~KScope() { timerEnd(c, r); }
};
#define RH_TIME(c, name) KScope rh_scope_(c, name)

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

int checkLaunch(rhgpu_ctx* c) {
   c->launches++;
   c->launchesStep++;
   cudaError_t e = cudaGetLastError();
   if (e != cudaSuccess) return fail(RHGPU_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
   return RHGPU_OK;
}
#define RH_LAUNCHED(c) do { int rc_ = checkLaunch(c); if (rc_) return rc_; } while (0)

// ---- prefix sums (k_scan.cuh) ---------------------------------------------------------------
// scratch of a scan of n values: the tile sums of every level
long long scanScratchLongs(long long n) {
   long long tot = 16;
   for (long long m = n; m > SCAN_TILE;) {
      m = (m + SCAN_TILE - 1) / SCAN_TILE;
      tot += m;
   }
   return tot;
}

int scanLevel(rhgpu_ctx* c, const long long* in, long long* out, long long n, long long* scratch) {
   const long long nb = (n + SCAN_TILE - 1) / SCAN_TILE;
   if (nb <= 1) {
      k_scan_tile<<<1, SCAN_THREADS, 0, c->stream>>>(in, out, n, nullptr);
      RH_LAUNCHED(c);
      return RHGPU_OK;
   }
   k_scan_tile<<<(unsigned)nb, SCAN_THREADS, 0, c->stream>>>(in, out, n, scratch);
   RH_LAUNCHED(c);
   if (int rc = scanLevel(c, scratch, scratch, nb, scratch + nb)) return rc;
   k_scan_add<<<blocks1d(n, 256), 256, 0, c->stream>>>(out, n, scratch);
   RH_LAUNCHED(c);
   return RHGPU_OK;
}

// exclusive prefix sum of n 64-bit values on the context's stream (in and out
// may be the same array); the context's scan scratch holds the tile sums
int scanExclusive64(rhgpu_ctx* c, const long long* in, long long* out, long long n) {
   if (n <= 0) return RHGPU_OK;
   if (sizeof(long long) * (size_t)scanScratchLongs(n) > c->scanTmpBytes)
      return fail(RHGPU_ERR_CAPACITY, "prefix sum larger than its scratch");
   return scanLevel(c, in, out, n, (long long*)c->scanTmp);
}


SpeciesDev speciesDev(const rhgpu_ctx* c, int s) {
   SpeciesDev d;
   d.q = c->sp[s].q;
   d.m = c->sp[s].m;
   d.R2obs = c->sp[s].R2_obstacle;
   // qmideltT2 = 0.5*species.q*sim->dt/species.m (boris.h:112)
   d.qmideltT2 = 0.5 * c->sp[s].q * c->P.dt / c->sp[s].m;
   d.accelerate = c->sp[s].accelerate;
   d.accumulate = c->sp[s].accumulate;
   return d;
}

int ensureKeyCapacity(rhgpu_ctx* c, long long n) {
   if (n <= c->keyCap) return RHGPU_OK;
   cudaFree(c->key);
   cudaFree(c->rank);
   c->keyCap = n + n / 8 + 1024;
   RH_CUDA(cudaMalloc(&c->key, sizeof(int) * c->keyCap));
   RH_CUDA(cudaMalloc(&c->rank, sizeof(int) * c->keyCap));
   return RHGPU_OK;
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

// species whose particles the exact-path deposit adds (accumulating, particles uploaded)
bool deposits(const rhgpu_ctx* c, int s) { return c->sp[s].accumulate && c->ps[s].start; }

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
         k_deposit_cell<<<blocks1d(g.N, DEP_WARPS), 32 * DEP_WARPS, 0, c->stream>>>(g, c->ps[s], c->sp[s].q, S, c->err);
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

#define RH_FIELD_LAUNCH(name, grid, block, ...)              \
   do {                                                      \
      RH_TIME(c, #name);                                     \
      name<<<grid, block, 0, c->stream>>>(__VA_ARGS__);      \
      RH_LAUNCHED(c);                                        \
   } while (0)

// propagateB (hybrid_propagator.cpp:42-440) in five passes when E is not
// smoothed: face2Cell, the exterior boundary rules, the node pass, the cell
// pass with Faraday, the cellUe Neumann rule (k_fields.cuh: the fused kernels)
int fieldsAll(rhgpu_ctx* c) {
   const GridInfo& g = c->g;
   const dim3 G = cellGrid(g), B = cellBlock();
   const unsigned EB = blocks1d(c->next > 0 ? c->next : 1, 128);
   const bool smooth = c->P.n_linear_smoothings_nodeE > 0 || c->P.use_gaussian_smoothing_nodeE;
   RH_FIELD_LAUNCH(k_face2cell, G, B, g, c->f);
   if (c->next > 0) RH_FIELD_LAUNCH(k_ext_bc, EB, 128, g, c->f, c->fp, c->ext, c->next);
   RH_FIELD_LAUNCH(k_node_fused, G, B, g, c->f, c->fp, c->cntU);
   c->gridAvgCounter += 1;
   {
      RH_TIME(c, "k_cell_tiled");
      const dim3 NG((g.nx + NT_X - 1) / NT_X, (g.ny + NT_Y - 1) / NT_Y, (g.nz + NT_Z - 1) / NT_Z);
      if (smooth)
         k_cell_tiled<false><<<NG, dim3(NT_X, NT_Y), CT_SMEM, c->stream>>>(g, c->f, c->fp, c->P.use_electron_pressure,
                                                                          c->cntU);
      else
         k_cell_tiled<true><<<NG, dim3(NT_X, NT_Y), CT_SMEM, c->stream>>>(g, c->f, c->fp, c->P.use_electron_pressure,
                                                                         c->cntU);
      RH_LAUNCHED(c);
   }
   if (c->next > 0) RH_FIELD_LAUNCH(k_ext_cell_neumann3, EB, 128, g, c->f.cellUe, c->ext, c->next);
   if (smooth) {
      for (int it = 0; it < c->P.n_linear_smoothings_nodeE; ++it) {
         RH_FIELD_LAUNCH(k_node2cell3, G, B, g, c->f.nodeE, c->f.cellJ);
         if (c->next > 0) RH_FIELD_LAUNCH(k_ext_cell_neumann3, EB, 128, g, c->f.cellJ, c->ext, c->next);
         RH_FIELD_LAUNCH(k_cell2node3, G, B, g, c->f.cellJ, c->f.nodeE);
         RH_CUDA(cudaMemsetAsync(c->f.cellJ, 0, sizeof(double) * 3 * g.N, c->stream));
      }
      if (c->P.use_gaussian_smoothing_nodeE) {
         RH_CUDA(cudaMemcpyAsync(c->tmp3, c->f.nodeE, sizeof(double) * 3 * g.N, cudaMemcpyDeviceToDevice, c->stream));
         RH_FIELD_LAUNCH(k_node_avg, G, B, g, c->tmp3, c->f.nodeE, c->fp);
      }
      RH_FIELD_LAUNCH(k_faraday, G, B, g, c->f);
   }
   c->t += c->P.dt;
   return RHGPU_OK;
}

int checkDeviceError(rhgpu_ctx* c) {
   unsigned w = 0;
   RH_CUDA(cudaMemcpyAsync(&w, c->err, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   if (w) return fail(RHGPU_ERR_DEVICE, "device error word " + std::to_string(w));
   return RHGPU_OK;
}

// per cell: slot range from the counts, cell index of every slot
__global__ void k_counts_in(long long N, const uint32_t* counts, long long* cnt64, int* alive) {
   const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (b < N) { cnt64[b] = counts[b]; alive[b] = (int)counts[b]; }
   if (b == N) cnt64[N] = 0;
}
__global__ void k_fill_pcell(long long N, const long long* start, int* pcell) {
   const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (b >= N) return;
   for (long long p = start[b]; p < start[b + 1]; ++p) pcell[p] = (int)b;
}

int ensureStaging(rhgpu_ctx* c, size_t bytes) {
   if (bytes <= c->stagingBytes) return RHGPU_OK;
   cudaFree(c->staging);
   c->staging = nullptr;
   c->stagingBytes = 0;
   RH_CUDA(cudaMalloc(&c->staging, bytes));
   c->stagingBytes = bytes;
   return RHGPU_OK;
}

// ---------------------------------------------------------------------------
// fast path, host side

template <class T> int growBuffer(T*& p, long long& have, long long need) {
   if (need <= have) return RHGPU_OK;
   cudaFree(p);
   p = nullptr;
   have = 0;
   const long long n = need + need / 8 + 64;
   RH_CUDA(cudaMalloc(&p, sizeof(T) * n));
   have = n;
   return RHGPU_OK;
}

int ensureSortTmp(rhgpu_ctx* c, size_t bytes) {
   if (bytes <= c->sortTmpBytes) return RHGPU_OK;
   cudaFree(c->sortTmp);
   c->sortTmp = nullptr;
   RH_CUDA(cudaMalloc(&c->sortTmp, bytes + 256));
   c->sortTmpBytes = bytes + 256;
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
   for (int a = 0; a < 7; ++a) { cudaFree(h.a[which][a]); h.a[which][a] = nullptr; }
   cudaFree(h.lx[which]);
   h.lx[which] = nullptr;
   h.capOf[which] = 0;
   const long long n = slots + slots / 16 + 1024;
   for (int a = 0; a < 7; ++a) RH_CUDA(cudaMalloc(&h.a[which][a], sizeof(double) * n));
   RH_CUDA(cudaMalloc(&h.lx[which], n));
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

// the periodic axes of a grid as a 3-bit mask (bit a = axis a)
int perMask(const GridInfo& g) { return (g.per[0] ? 1 : 0) | (g.per[1] ? 2 : 0) | (g.per[2] ? 4 : 0); }

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

__global__ void k_iota(unsigned* v, long long n) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t < n) v[t] = (unsigned)t;
}
__global__ void k_int_to64(const int* in, long long n, long long* out) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t < n) out[t] = in[t];
   if (t == n) out[n] = 0;
}

__global__ void k_fill_u32(unsigned* a, long long n, unsigned v) {
   const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (p < n) a[p] = v;
}
__global__ void k_gather_u32(const unsigned* src, const unsigned* idx, long long n, unsigned* dst) {
   const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (p < n) dst[p] = src[idx[p]];
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
// (the usual case) are ordered one thread per bucket; otherwise two stable
// radix sorts over all movers (by key, then by bucket) give the same order.
const int MIG_SMALL = 64;
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
   if (maxInc <= MIG_SMALL) {
      // buckets past the placed movers stay at nb (not placed)
      RH_CUDA(cudaMemsetAsync(c->ffill, 0, sizeof(int) * nb, c->stream));
      k_fill_u32<<<blocks1d(nm, 256), 256, 0, c->stream>>>(bA, nm, (unsigned)nb);
      k_mig_bucket<<<blocks1d(nm, 256), 256, 0, c->stream>>>(mv, nm, NS, c->foffInc, c->ffill, vA);
      RH_LAUNCHED(c);
      k_mig_order_small<<<blocks1d(nb, 256), 256, 0, c->stream>>>(mv, nb, c->finc, c->foffInc, vA, bA);
      RH_LAUNCHED(c);
      k_mig_check<<<blocks1d(nb, 256), 256, 0, c->stream>>>(FS, NS, c->finc, c->fover);
      RH_LAUNCHED(c);
      RH_CUDA(cudaMemcpyAsync(over, c->fover, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      RH_CUDA(cudaStreamSynchronize(c->stream));
      *order = vA;
      *bucket = bA;
      return RHGPU_OK;
   }
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


// ---------------------------------------------------------------------------
// FP32 precision form, host side

F32Buf f32View(const F32Host& h, int which) {
   F32Buf b;
   b.cell = h.cell[which];
   for (int a = 0; a < 3; ++a) { b.o[a] = h.o[which][a]; b.v[a] = h.v[which][a]; }
   b.cnt = h.cnt[which];
   return b;
}

int f32Reserve(F32Host& h, int which, long long slots) {
   if (slots <= h.capOf[which] && h.cell[which]) return RHGPU_OK;
   cudaFree(h.cell[which]);
   h.cell[which] = nullptr;
   for (int a = 0; a < 3; ++a) {
      cudaFree(h.o[which][a]); cudaFree(h.v[which][a]);
      h.o[which][a] = nullptr; h.v[which][a] = nullptr;
   }
   h.capOf[which] = 0;
   const long long n = slots + slots / 16 + 1024;
   RH_CUDA(cudaMalloc(&h.cell[which], sizeof(int) * n));
   for (int a = 0; a < 3; ++a) {
      RH_CUDA(cudaMalloc(&h.o[which][a], sizeof(float) * n));
      RH_CUDA(cudaMalloc(&h.v[which][a], sizeof(float) * n));
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
              const float* particles32 = nullptr, double weight32 = 0.0) {
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
                float* particles32 = nullptr) {
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

}  // namespace

// ---------------------------------------------------------------------------
// learned denoiser, host side

namespace {

const int DN_LOSS_BLOCKS = 296;

// the UMMA B images of every layer (forward and transposed) from the FP32 parameters
int dnRebuildImages(rhgpu_dn* d) {
   for (int l = 0; l < 3; ++l)
      for (int tr = 0; tr < 2; ++tr)
         k_dn_bimage<<<(DN_TAPS * DN_C * DN_C + 255) / 256, 256, 0, d->stream>>>(
             d->params + (size_t)l * DN_LAYER, d->bimg + (size_t)(3 * tr + l) * (TC_BIMG / 2), tr);
   RH_CUDA(cudaGetLastError());
   return RHGPU_OK;
}

// one convolution layer on the tensor cores (k_dn_conv_tc): layer l, forward or
// transposed (the data gradient); `err` receives RHGPU_DEVERR_DENOISER
int dnConv(rhgpu_dn* d, cudaStream_t st, bool transposed, int l, const unsigned* in, const float* bias, int mode,
           unsigned* out, const unsigned* mask, float* out32, const float* res, const DnMoments& mom, unsigned* err) {
   static bool raised[64][2] = {};
   if (d->device < 0 || d->device >= 64) return fail(RHGPU_ERR_CUDA, "denoiser: device index out of range");
   if (!raised[d->device][transposed]) {
      RH_CUDA(cudaFuncSetAttribute(transposed ? k_dn_conv_tc<true> : k_dn_conv_tc<false>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
      raised[d->device][transposed] = true;
   }
   const dim3 grid((unsigned)((d->g.nx + TC_BX - 1) / TC_BX), (unsigned)((d->g.ny + TC_BY - 1) / TC_BY),
                   (unsigned)((d->g.nz + TC_ZC - 1) / TC_ZC));
   const __nv_bfloat16* img = d->bimg + (size_t)((transposed ? 3 : 0) + l) * (TC_BIMG / 2);
   if (transposed)
      k_dn_conv_tc<true><<<grid, TC_THREADS, TC_SMEM, st>>>(d->g, in, img, bias, mode, out, mask, out32, res, mom, err);
   else
      k_dn_conv_tc<false><<<grid, TC_THREADS, TC_SMEM, st>>>(d->g, in, img, bias, mode, out, mask, out32, res, mom, err);
   RH_CUDA(cudaGetLastError());
   return RHGPU_OK;
}

// the convolutions' device error word, read and cleared (after a synchronisation of d->stream)
int dnCheckError(rhgpu_dn* d) {
   unsigned w = 0;
   RH_CUDA(cudaMemcpyAsync(&w, d->err, sizeof w, cudaMemcpyDeviceToHost, d->stream));
   RH_CUDA(cudaStreamSynchronize(d->stream));
   if (w) {
      RH_CUDA(cudaMemsetAsync(d->err, 0, sizeof w, d->stream));
      return fail(RHGPU_ERR_DEVICE, "denoiser: a convolution's wait on its tensor-core work ran out");
   }
   return RHGPU_OK;
}

// forward of the network on d->res (normalized FP32 input) into d->out32
int dnForward(rhgpu_dn* d) {
   const long long N = d->g.N;
   k_dn_res_to_act<<<blocks1d(N, 256), 256, 0, d->stream>>>(N, d->res, d->act[0]);
   const float* b0 = d->params + DN_TAPS * DN_C * DN_C;
   const float* b1 = d->params + DN_LAYER + DN_TAPS * DN_C * DN_C;
   const float* b2 = d->params + 2 * DN_LAYER + DN_TAPS * DN_C * DN_C;
   int rc = dnConv(d, d->stream, false, 0, d->act[0], b0, 0, d->act[1], nullptr, nullptr, nullptr, DnMoments{}, d->err);
   if (!rc) rc = dnConv(d, d->stream, false, 1, d->act[1], b1, 0, d->act[2], nullptr, nullptr, nullptr, DnMoments{}, d->err);
   if (!rc) rc = dnConv(d, d->stream, false, 2, d->act[2], b2, 3, nullptr, nullptr, d->out32, d->res, DnMoments{}, d->err);
   return rc;
}

// loss against target (normalized FP32, N x 4) and the gradient of all parameters into d->grad
int dnBackward(rhgpu_dn* d, const float* target, double* loss) {
   const long long N = d->g.N;
   // voxels in the loss: all but the masked border of the non-periodic faces
   long long in = 1;
   const int nn[3] = {d->g.nx, d->g.ny, d->g.nz};
   for (int a = 0; a < 3; ++a) in *= d->g.per[a] ? nn[a] : std::max(0, nn[a] - 2 * d->border);
   if (in < 1) return fail(RHGPU_ERR_STATE, "dn_train: the loss border leaves no voxel");
   k_dn_loss<<<DN_LOSS_BLOCKS, 256, 0, d->stream>>>(d->g, d->out32, target, 1.0 / (4.0 * (double)in), d->dY[2], d->lossPart,
                                                   d->border);
   const unsigned wb = (unsigned)((N + DN_WGRAD_VOX - 1) / DN_WGRAD_VOX);
   for (int l = 2; l >= 0; --l) {
      k_dn_wgrad<<<dim3(wb, DN_TAPS), 32 * DN_WARPS, 0, d->stream>>>(d->g, d->act[l], d->dY[l], d->part);
      k_dn_reduce_rows<<<(DN_TAPS * DN_C * DN_C + 255) / 256, 256, 0, d->stream>>>(d->part, wb, DN_TAPS * DN_C * DN_C,
                                                                                  d->grad + (size_t)l * DN_LAYER);
      k_dn_bgrad<<<wb, 256, 0, d->stream>>>(d->g, d->dY[l], d->part);
      k_dn_reduce_rows<<<1, DN_C, 0, d->stream>>>(d->part, wb, DN_C, d->grad + (size_t)l * DN_LAYER + DN_TAPS * DN_C * DN_C);
      if (l > 0)
         if (int rc = dnConv(d, d->stream, true, l, d->dY[l], nullptr, 2, d->dY[l - 1], d->act[l], nullptr, nullptr,
                             DnMoments{}, d->err))
            return rc;
   }
   RH_CUDA(cudaGetLastError());
   std::vector<double> lp(DN_LOSS_BLOCKS);
   RH_CUDA(cudaMemcpyAsync(lp.data(), d->lossPart, sizeof(double) * DN_LOSS_BLOCKS, cudaMemcpyDeviceToHost, d->stream));
   RH_CUDA(cudaStreamSynchronize(d->stream));
   double a = 0.0;
   for (double x : lp) a += x;
   if (loss) *loss = a / (4.0 * (double)in);
   return RHGPU_OK;
}

// host moments in the ABI layout (rho N, Ji interleaved 3N) -> device planar scratch (acc)
int dnUploadMoments(rhgpu_dn* d, const double* rho, const double* ji, double* planar) {
   const long long N = d->g.N;
   std::vector<double> h(4 * (size_t)N);
   for (long long n = 0; n < N; ++n) {
      h[n] = rho[n];
      for (int l = 0; l < 3; ++l) h[(1 + l) * N + n] = ji[3 * n + l];
   }
   RH_CUDA(cudaMemcpyAsync(planar, h.data(), sizeof(double) * 4 * N, cudaMemcpyHostToDevice, d->stream));
   RH_CUDA(cudaStreamSynchronize(d->stream));
   return RHGPU_OK;
}


// the network on planar device moments (rho N, J 3 x N), in place: the first layer
// reads and normalizes them, the last adds its output to their normalized values
// and scales back (rho clamped at minRho), in three launches
int dnApplyMoments(rhgpu_dn* d, cudaStream_t st, double* rho, double* J, double minRho, unsigned* err) {
   const long long N = d->g.N;
   const DnMoments mom{rho, J, d->sr, d->sj, 1.0 / d->sr, 1.0 / d->sj, minRho, N};
   const float* b0 = d->params + DN_TAPS * DN_C * DN_C;
   const float* b1 = d->params + DN_LAYER + DN_TAPS * DN_C * DN_C;
   const float* b2 = d->params + 2 * DN_LAYER + DN_TAPS * DN_C * DN_C;
   int rc = dnConv(d, st, false, 0, nullptr, b0, 0, d->act[1], nullptr, nullptr, nullptr, mom, err);
   if (!rc) rc = dnConv(d, st, false, 1, d->act[1], b1, 0, d->act[2], nullptr, nullptr, nullptr, DnMoments{}, err);
   if (!rc) rc = dnConv(d, st, false, 2, d->act[2], b2, 4, nullptr, nullptr, nullptr, nullptr, mom, err);
   return rc;
}

// the denoiser on the context's moments (device, on the context's stream), before the field update
int dnApplyCtx(rhgpu_ctx* c) {
   RH_TIME(c, "dn_apply");
   return dnApplyMoments(c->dn, c->stream, c->f.cellRho, c->f.cellJi, c->P.min_ion_charge_density, c->err);
}

}  // namespace

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

const char* rhgpu_last_error(void) { return g_err.c_str(); }

const char* rhgpu_version(void) {
   return "rhgpu 0.1 sm_100a fp64 (--fmad=false, IEEE div/sqrt), paths: fast (dual-cell order, default), exact (reference order)";
}

int rhgpu_create(const rhgpu_params* params, int32_t n_species, const rhgpu_species* species,
                 const int64_t* capacity, int32_t device, rhgpu_ctx** out) {
   if (!params || !species || !out || n_species < 1 || n_species > MAX_SPECIES)
      return fail(RHGPU_ERR_ARG, "rhgpu_create: bad arguments");
   if (params->nx < 3 || params->ny < 3 || params->nz < 3) return fail(RHGPU_ERR_ARG, "rhgpu_create: at least 3 cells per axis");
   const long long N = (long long)params->nx * params->ny * params->nz;
   if (N * 27 >= (1LL << 31)) return fail(RHGPU_ERR_ARG, "rhgpu_create: grid too large (27*cells must fit int32)");
   if (!(params->dx >= std::ldexp(1.0, -200) && params->dx <= std::ldexp(1.0, 200)) || !(params->dt > 0))
      return fail(RHGPU_ERR_ARG, "rhgpu_create: dx must lie in [2^-200, 2^200] and dt must be positive");
   RH_CUDA(cudaSetDevice(device));
   rhgpu_ctx* c = new rhgpu_ctx();
   c->P = *params;
   c->device = device;
   c->ns = n_species;
   std::memcpy(c->sp, species, sizeof(rhgpu_species) * n_species);
   GridInfo& g = c->g;
   g.nx = params->nx; g.ny = params->ny; g.nz = params->nz;
   for (int a = 0; a < 3; ++a) g.per[a] = params->periodic[a] ? 1 : 0;
   g.N = N;
   g.dx = params->dx;
   g.dt = params->dt;
   g.dV = params->dx * params->dx * params->dx;
   g.dx_below = std::nextafter(params->dx, 0.0);
   g.rdx = 1.0 / params->dx;   // correctly rounded reciprocal, for divDx
   g.x_min = params->x_min; g.y_min = params->y_min; g.z_min = params->z_min;
   c->t = params->t_initial;
   c->useIFT = params->use_initial_flow_through;
   FieldParams& fp = c->fp;
   fp.use_hall = params->use_hall;
   fp.use_ep = params->use_electron_pressure;
   fp.isothermal = params->isothermal_electrons;
   fp.ep_coeff = params->electron_pressure_coeff;
   for (int l = 0; l < 3; ++l) fp.obstacleUe[l] = params->field_obstacle_Ue[l];
   fp.maxUe2 = params->max_electron_speed2;
   fp.minRho = params->min_ion_charge_density;
   fp.maxE2 = params->max_electric_field2;
   fp.maxVw = params->max_whistler_speed;
   for (int l = 0; l < 4; ++l) fp.gauss[l] = params->gaussian_coeffs[l];
   for (int l = 0; l < 3; ++l) fp.imf[l] = params->imf_B[l];
   for (int w = 0; w < 6; ++w) { fp.imfCell[w] = params->imf_boundary_cellB[w]; fp.imfFace[w] = params->imf_boundary_faceB[w]; }

   int rc = RHGPU_OK;
   auto alloc = [&](void** p, size_t bytes) {
      if (rc) return;
      cudaError_t e = cudaMalloc(p, bytes);
      if (e != cudaSuccess) rc = fail(RHGPU_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
      else cudaMemset(*p, 0, bytes);
   };
   if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete c;
      return fail(RHGPU_ERR_CUDA, "stream create failed");
   }
   for (int a = 0; a < RHGPU_NUM_ARRAYS; ++a) alloc((void**)&c->arr[a], sizeof(double) * N * arrayDim(a));
   alloc((void**)&c->tmp3, sizeof(double) * 3 * N);
   alloc((void**)&c->flags, N);
   alloc((void**)&c->outCount, sizeof(int) * 27 * N);
   alloc((void**)&c->inPrefix, sizeof(int) * 27 * N);
   alloc((void**)&c->newCount, sizeof(long long) * (N + 1));
   alloc((void**)&c->cntU, sizeof(unsigned long long) * NCNT_U);
   alloc((void**)&c->cntD, sizeof(double) * 4 * MAX_SPECIES);
   alloc((void**)&c->err, sizeof(unsigned));
   // fast-path geometry and buffers
   FastGeom& fg = c->fg;
   for (int a = 0; a < 3; ++a) fg.nd[a] = (a == 0 ? g.nx : a == 1 ? g.ny : g.nz) + (g.per[a] ? 0 : 1);
   fg.nseg = (fg.nd[0] + SEG - 1) / SEG;
   fg.nrows = (long long)fg.nd[1] * fg.nd[2];
   fg.NS = fg.nrows * fg.nseg;
   const long long NS = fg.NS, nb = (long long)n_species * fg.NS;
   for (int s = 0; s < n_species; ++s) {
      SegHost& h = c->seg[s];
      alloc((void**)&h.cnt[0], sizeof(int) * NS);
      alloc((void**)&h.cnt[1], sizeof(int) * NS);
      alloc((void**)&h.base, sizeof(long long) * (NS + 1));
      alloc((void**)&h.baseAlt, sizeof(long long) * (NS + 1));
      c->capHint[s] = capacity ? (long long)capacity[s] : 0;
   }
   alloc((void**)&c->fb.RP, sizeof(double) * 16 * fg.nrows * g.nx);
   alloc((void**)&c->fb.RPB, sizeof(double) * 16 * fg.nrows * fg.nseg);
   alloc((void**)&c->fb.MMlo, sizeof(unsigned long long) * 4 * N);
   alloc((void**)&c->fb.MMhi, sizeof(unsigned long long) * 4 * N);
   alloc((void**)&c->fb.touched, (size_t)N + 16);
   alloc((void**)&c->segInnerDev, (size_t)NS + 16);
   c->fb.segInner = c->segInnerDev;
   alloc((void**)&c->fb.nmovers, sizeof(unsigned long long));
   alloc((void**)&c->finc, sizeof(int) * nb);
   alloc((void**)&c->ffill, sizeof(int) * nb);
   alloc((void**)&c->fmaxInc, sizeof(int));
   alloc((void**)&c->fcap, sizeof(long long) * (NS + 1));
   alloc((void**)&c->ffirst, sizeof(long long) * (NS + 1));
   alloc((void**)&c->ftmp64, sizeof(long long) * (NS + 1));
   alloc((void**)&c->ftmpCellStart, sizeof(long long) * (N + 1));
   alloc((void**)&c->ftmpInc64, sizeof(long long) * (nb + 1));
   alloc((void**)&c->foffInc, sizeof(long long) * (nb + 1));
   alloc((void**)&c->fover, 2 * sizeof(unsigned long long));
   alloc((void**)&c->diagPart, sizeof(double) * DIAG_BLOCKS * DIAG_FS);
   if (!rc) {
      // MM starts at zero; the gather clears it after reading
      if (cudaMemset(c->fb.MMlo, 0, sizeof(unsigned long long) * 4 * N) != cudaSuccess ||
          cudaMemset(c->fb.MMhi, 0, sizeof(unsigned long long) * 4 * N) != cudaSuccess ||
          cudaMemset(c->fb.RPB, 0, sizeof(double) * 16 * fg.nrows * fg.nseg) != cudaSuccess ||
          cudaMemset(c->segInnerDev, 0, (size_t)NS + 16) != cudaSuccess)
         rc = fail(RHGPU_ERR_CUDA, "create: clear fast-path sums");
   }
   if (!rc) {
      // scan scratch for the largest scan (cells, dual cells, species x dual cells)
      const long long mx = std::max(N, nb) + 1;
      c->scanTmpBytes = sizeof(long long) * (size_t)scanScratchLongs(mx);
      alloc(&c->scanTmp, c->scanTmpBytes);
   }
   // exterior cells (missing a neighbour) and obstacle-flagged cells are
   // listed after upload_cell_flags; exterior list now
   if (!rc) {
      std::vector<int> ext;
      for (int k = 0; k < g.nz; ++k)
         for (int j = 0; j < g.ny; ++j)
            for (int i = 0; i < g.nx; ++i)
               if (!allNb(g, i, j, k)) ext.push_back((int)cidx(g, i, j, k));
      c->next = (int)ext.size();
      alloc((void**)&c->ext, sizeof(int) * (ext.size() + 1));
      if (!rc && !ext.empty()) {
         if (cudaMemcpy(c->ext, ext.data(), sizeof(int) * ext.size(), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = fail(RHGPU_ERR_CUDA, "copy exterior list");
      }
   }
   if (!rc) {
      NeumannTables t = buildNeumannTables();
      if (cudaMemcpyToSymbol(c_neu, &t, sizeof t) != cudaSuccess) rc = fail(RHGPU_ERR_CUDA, "neumann tables");
   }
   if (!rc) {
      Fields& f = c->f;
      f.faceB = c->arr[RHGPU_FACE_B]; f.cellB = c->arr[RHGPU_CELL_B]; f.cellUe = c->arr[RHGPU_CELL_UE];
      f.cellEp = c->arr[RHGPU_CELL_EP]; f.cellRho = c->arr[RHGPU_CELL_RHOQI]; f.cellJi = c->arr[RHGPU_CELL_JI];
      f.cellJ = c->arr[RHGPU_CELL_J]; f.nodeRho = c->arr[RHGPU_NODE_RHOQI]; f.nodeJi = c->arr[RHGPU_NODE_JI];
      f.nodeJ = c->arr[RHGPU_NODE_J]; f.nodeUe = c->arr[RHGPU_NODE_UE]; f.nodeB = c->arr[RHGPU_NODE_B];
      f.nodeE = c->arr[RHGPU_NODE_E]; f.nodeEta = c->arr[RHGPU_NODE_ETA]; f.cellAvgB = c->arr[RHGPU_CELL_AVERAGE_B];
      f.tmp3 = c->tmp3;
      f.flags = c->flags;
      f.gc = nullptr;   // grid constraint counters off until rhgpu_set_grid_counters
   }
   if (rc) {
      rhgpu_destroy(c);
      return rc;
   }
   if (cudaDeviceSynchronize() != cudaSuccess) return fail(RHGPU_ERR_CUDA, "create: sync failed");
   *out = c;
   return RHGPU_OK;
}

int rhgpu_destroy(rhgpu_ctx* c) {
   if (!c) return RHGPU_OK;
   cudaSetDevice(c->device);
   if (c->stream) cudaStreamSynchronize(c->stream);
   for (int a = 0; a < RHGPU_NUM_ARRAYS; ++a) cudaFree(c->arr[a]);
   cudaFree(c->tmp3); cudaFree(c->flags); cudaFree(c->ext); cudaFree(c->obst);
   cudaFree(c->key); cudaFree(c->rank); cudaFree(c->outCount); cudaFree(c->inPrefix);
   cudaFree(c->newCount); cudaFree(c->scanTmp); cudaFree(c->S); cudaFree(c->cntU); cudaFree(c->cntD); cudaFree(c->err);
   cudaFree(c->staging);
   for (int s = 0; s < c->ns; ++s) {
      SegHost& h = c->seg[s];
      for (int b = 0; b < 2; ++b) {
         for (int a = 0; a < 7; ++a) cudaFree(h.a[b][a]);
         cudaFree(h.lx[b]);
         cudaFree(h.cnt[b]);
      }
      cudaFree(h.base);
      cudaFree(h.baseAlt);
   }
   cudaFree(c->fb.RP); cudaFree(c->fb.RPB); cudaFree(c->fb.MMlo); cudaFree(c->fb.MMhi); cudaFree(c->fb.touched); cudaFree(c->segInnerDev);
   cudaFree(c->fb.nmovers); cudaFree(c->fb.movers);
   for (auto& h : c->inj) { cudaFree(h.cells); cudaFree(h.rates); cudaFree(h.list); }
   cudaFree(c->injCnt);
   cudaFree(c->finc); cudaFree(c->fover); cudaFree(c->ffill); cudaFree(c->fmaxInc);
   cudaFree(c->mkey); cudaFree(c->mval); cudaFree(c->mbkt);
   cudaFree(c->sortTmp); cudaFree(c->fcap); cudaFree(c->ffirst); cudaFree(c->ftmp64); cudaFree(c->ftmpCellStart);
   cudaFree(c->ftmpInc64); cudaFree(c->foffInc); cudaFree(c->fsort); cudaFree(c->fsortSlots); cudaFree(c->flxTmp);
   cudaFree(c->diagPart);
   cudaFree(c->rhoM);
   cudaFree(c->rhoMfix);
   cudaFree(c->avgN); cudaFree(c->avgV); cudaFree(c->avgOut);
   cudaFree(c->avgFB.RP); cudaFree(c->avgFB.RPB); cudaFree(c->avgFB.MMlo); cudaFree(c->avgFB.MMhi);
   cudaFree(c->gridCnt);
   if (c->logs) { c->logs->close(); delete c->logs; c->logs = nullptr; }
   for (int s = 0; s < c->ns; ++s) {
      F32Host& h = c->f32[s];
      for (int b = 0; b < 2; ++b) {
         cudaFree(h.cell[b]);
         for (int a = 0; a < 3; ++a) { cudaFree(h.o[b][a]); cudaFree(h.v[b][a]); }
         cudaFree(h.cnt[b]);
      }
      cudaFree(h.base);
      cudaFree(h.baseAlt);
   }
   cudaFree(c->f32b.RP); cudaFree(c->f32b.RPB); cudaFree(c->f32b.movers);
   for (int s = 0; s < c->ns; ++s) { freeStore(c->ps[s]); freeStore(c->alt[s]); }
   for (cudaEvent_t e : c->evPool) cudaEventDestroy(e);
   if (c->stream) cudaStreamDestroy(c->stream);
   delete c;
   return RHGPU_OK;
}

// ----------------------------------------------------------------------------
// grid arrays: ParGrid interleaved layout <-> component planes

namespace {
__global__ void k_interleaved_to_planes(const double* in, double* out, long long N, int dim) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= N * dim) return;
   const long long n = t / dim;
   const int l = (int)(t % dim);
   out[(long long)l * N + n] = in[t];
}
__global__ void k_planes_to_interleaved(const double* in, double* out, long long N, int dim) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= N * dim) return;
   const long long n = t / dim;
   const int l = (int)(t % dim);
   out[t] = in[(long long)l * N + n];
}
}  // namespace

int rhgpu_upload_array(rhgpu_ctx* c, int32_t id, const double* host) {
   if (!c || !host || id < 0 || id >= RHGPU_NUM_ARRAYS) return fail(RHGPU_ERR_ARG, "upload_array: bad arguments");
   RH_CUDA(cudaSetDevice(c->device));
   const int dim = arrayDim(id);
   const long long N = c->g.N;
   RH_CUDA(cudaMemcpyAsync(c->tmp3, host, sizeof(double) * N * dim, cudaMemcpyHostToDevice, c->stream));
   k_interleaved_to_planes<<<blocks1d(N * dim, 256), 256, 0, c->stream>>>(c->tmp3, c->arr[id], N, dim);
   RH_CUDA(cudaGetLastError());
   RH_CUDA(cudaStreamSynchronize(c->stream));
   return RHGPU_OK;
}

int rhgpu_download_array(rhgpu_ctx* c, int32_t id, double* host) {
   if (!c || !host || id < 0 || id >= RHGPU_NUM_ARRAYS) return fail(RHGPU_ERR_ARG, "download_array: bad arguments");
   RH_CUDA(cudaSetDevice(c->device));
   const int dim = arrayDim(id);
   const long long N = c->g.N;
   k_planes_to_interleaved<<<blocks1d(N * dim, 256), 256, 0, c->stream>>>(c->arr[id], c->tmp3, N, dim);
   RH_CUDA(cudaGetLastError());
   RH_CUDA(cudaMemcpyAsync(host, c->tmp3, sizeof(double) * N * dim, cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   return RHGPU_OK;
}

int rhgpu_upload_cell_flags(rhgpu_ctx* c, const uint8_t* host) {
   if (!c || !host) return fail(RHGPU_ERR_ARG, "upload_cell_flags: bad arguments");
   RH_CUDA(cudaSetDevice(c->device));
   RH_CUDA(cudaMemcpy(c->flags, host, c->g.N, cudaMemcpyHostToDevice));
   std::vector<int> ob;
   for (long long n = 0; n < c->g.N; ++n)
      if (host[n] & RHGPU_FLAG_INNER_PARTICLE) ob.push_back((int)n);
   {
      // per row segment: can a particle of it land, within one step, in a cell
      // flagged RHGPU_FLAG_INNER_PARTICLE? The cells it can reach are those of
      // its dual cells one cell out on every side (x from xs0 - 1 to
      // xs0 + SEG + 1, y and z from the base - 1 to the base + 2, wrapped on
      // periodic axes); the push kernels test the obstacle only where one is
      const FastGeom& fg = c->fg;
      const GridInfo& g = c->g;
      std::vector<unsigned char> si((size_t)fg.NS, 0);
      if (!ob.empty()) {
         for (long long S = 0; S < fg.NS; ++S) {
            const long long row = S / fg.nseg;
            const int gseg = (int)(S % fg.nseg);
            const int uy = (int)(row % fg.nd[1]), uz = (int)(row / fg.nd[1]);
            const int xs0 = dualB(gseg * SEG, g.per[0]), ys0 = dualB(uy, g.per[1]), zs0 = dualB(uz, g.per[2]);
            bool hit = false;
            for (int dz = -1; dz <= 2 && !hit; ++dz)
               for (int dy = -1; dy <= 2 && !hit; ++dy) {
                  int y = ys0 + dy, z = zs0 + dz;
                  if (!wrapc(y, g.ny, g.per[1]) || !wrapc(z, g.nz, g.per[2])) continue;
                  for (int dx = -1; dx <= SEG + 1 && !hit; ++dx) {
                     int x = xs0 + dx;
                     if (wrapc(x, g.nx, g.per[0])) hit = (host[cidx(g, x, y, z)] & RHGPU_FLAG_INNER_PARTICLE) != 0;
                  }
               }
            si[(size_t)S] = hit ? 1 : 0;
         }
      }
      RH_CUDA(cudaMemcpy(c->segInnerDev, si.data(), (size_t)fg.NS, cudaMemcpyHostToDevice));
   }
   cudaFree(c->obst);
   c->obst = nullptr;
   c->nobst = (int)ob.size();
   RH_CUDA(cudaMalloc(&c->obst, sizeof(int) * (ob.size() + 1)));
   if (!ob.empty()) RH_CUDA(cudaMemcpy(c->obst, ob.data(), sizeof(int) * ob.size(), cudaMemcpyHostToDevice));
   return RHGPU_OK;
}

namespace {
// particle records (7 doubles) -> 7 component planes
__global__ void k_aos_to_soa(const double* aos, PStore P, long long n) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= 7 * n) return;
   const long long p = t / 7;
   const int a = (int)(t % 7);
   P.a[a][p] = aos[t];
}
// alive particles of each cell -> records at the cell's output offset
__global__ void k_soa_to_aos(PStore P, long long N, const long long* outStart, double* aos, uint32_t* counts) {
   const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (b >= N) return;
   const long long s = P.start[b], o = outStart[b];
   const int na = P.alive[b];
   counts[b] = (uint32_t)na;
   for (int t = 0; t < na; ++t)
      for (int a = 0; a < 7; ++a) aos[7 * (o + t) + a] = P.a[a][s + t];
}
__global__ void k_alive_to64(long long N, const int* alive, long long* out) {
   const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (b < N) out[b] = alive[b];
   if (b == N) out[N] = 0;
}
}  // namespace

int rhgpu_upload_particles(rhgpu_ctx* c, int32_t s, const uint32_t* counts, const double* particles, int64_t n) {
   if (!c || s < 0 || s >= c->ns || !counts || (n > 0 && !particles) || n < 0)
      return fail(RHGPU_ERR_ARG, "upload_particles: bad arguments");
   RH_CUDA(cudaSetDevice(c->device));
   if (c->capHint[s] > 0 && n > c->capHint[s]) return fail(RHGPU_ERR_CAPACITY, "upload_particles: more particles than capacity");
   c->uploaded = true;
   if (c->path == RHGPU_PATH_FAST) return fastUpload(c, s, counts, particles, n);
   if (c->path == RHGPU_PATH_FP32) return f32Upload(c, s, counts, particles, n);
   const long long N = c->g.N;
   PStore& P = c->ps[s];
   if (n > P.cap || !P.start) {
      // bit-exact path storage, allocated on first use (also for an empty upload)
      const long long cap = std::max<long long>(c->capHint[s], (long long)n + n / 8 + 1024);
      freeStore(c->ps[s]);
      freeStore(c->alt[s]);
      int rc0 = allocStore(c->ps[s], cap, N);
      if (!rc0) rc0 = allocStore(c->alt[s], cap, N);
      if (rc0) return rc0;
   }
   int rc = ensureStaging(c, sizeof(double) * 7 * (size_t)(n > 0 ? n : 1) + sizeof(uint32_t) * (size_t)N + 64);
   if (rc) return rc;
   double* aos = (double*)c->staging;
   uint32_t* dcounts = (uint32_t*)((char*)c->staging + sizeof(double) * 7 * (size_t)(n > 0 ? n : 1));
   RH_CUDA(cudaMemcpyAsync(dcounts, counts, sizeof(uint32_t) * N, cudaMemcpyHostToDevice, c->stream));
   if (n) RH_CUDA(cudaMemcpyAsync(aos, particles, sizeof(double) * 7 * n, cudaMemcpyHostToDevice, c->stream));
   k_counts_in<<<blocks1d(N + 1, 256), 256, 0, c->stream>>>(N, dcounts, c->newCount, P.alive);
   RH_CUDA(cudaGetLastError());
   if (int rc_ = scanExclusive64(c, c->newCount, P.start, N + 1)) return rc_;
   long long total = 0;
   RH_CUDA(cudaMemcpyAsync(&total, P.start + N, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   if (total != n) return fail(RHGPU_ERR_ARG, "upload_particles: sum(counts) != n_particles");
   k_fill_pcell<<<blocks1d(N, 128), 128, 0, c->stream>>>(N, P.start, P.pcell);
   RH_CUDA(cudaGetLastError());
   if (n) {
      k_aos_to_soa<<<blocks1d(7 * n, 256), 256, 0, c->stream>>>(aos, P, n);
      RH_CUDA(cudaGetLastError());
   }
   RH_CUDA(cudaStreamSynchronize(c->stream));
   P.nslots = n;
   return ensureKeyCapacity(c, n);
}

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

int rhgpu_num_particles(rhgpu_ctx* c, int32_t s, int64_t* n_out) {
   if (!c || s < 0 || s >= c->ns || !n_out) return fail(RHGPU_ERR_ARG, "num_particles: bad arguments");
   RH_CUDA(cudaSetDevice(c->device));
   if (c->path == RHGPU_PATH_FAST || c->path == RHGPU_PATH_FP32) {
      long long t = 0;
      int rc = c->path == RHGPU_PATH_FAST ? fastNumParticles(c, s, &t) : f32NumParticles(c, s, &t);
      *n_out = t;
      return rc;
   }
   if (!c->ps[s].alive) { *n_out = 0; return RHGPU_OK; }
   std::vector<int> alive(c->g.N);
   RH_CUDA(cudaStreamSynchronize(c->stream));
   RH_CUDA(cudaMemcpy(alive.data(), c->ps[s].alive, sizeof(int) * c->g.N, cudaMemcpyDeviceToHost));
   long long t = 0;
   for (int a : alive) t += a;
   *n_out = t;
   return RHGPU_OK;
}

int rhgpu_download_particles(rhgpu_ctx* c, int32_t s, uint32_t* counts, double* particles, int64_t capacity,
                             int64_t* n_out) {
   if (!c || s < 0 || s >= c->ns || !counts || !n_out) return fail(RHGPU_ERR_ARG, "download_particles: bad arguments");
   RH_CUDA(cudaSetDevice(c->device));
   if (c->path == RHGPU_PATH_FAST || c->path == RHGPU_PATH_FP32) {
      long long t = 0;
      int rc = c->path == RHGPU_PATH_FAST ? fastDownload(c, s, counts, particles, capacity, &t)
                                          : f32Download(c, s, counts, particles, capacity, &t);
      *n_out = t;
      return rc;
   }
   if (!c->ps[s].alive) {
      std::memset(counts, 0, sizeof(uint32_t) * c->g.N);
      *n_out = 0;
      return RHGPU_OK;
   }
   const long long N = c->g.N;
   PStore& P = c->ps[s];
   // output offsets: exclusive scan of the alive counts (scratch: newCount, alt.start)
   k_alive_to64<<<blocks1d(N + 1, 256), 256, 0, c->stream>>>(N, P.alive, c->newCount);
   RH_CUDA(cudaGetLastError());
   long long* outStart = c->alt[s].start;
   if (int rc_ = scanExclusive64(c, c->newCount, outStart, N + 1)) return rc_;
   long long tot = 0;
   RH_CUDA(cudaMemcpyAsync(&tot, outStart + N, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   if (tot > capacity) return fail(RHGPU_ERR_ARG, "download_particles: capacity too small");
   int rc = ensureStaging(c, sizeof(double) * 7 * (size_t)(tot > 0 ? tot : 1) + sizeof(uint32_t) * (size_t)N + 64);
   if (rc) return rc;
   double* aos = (double*)c->staging;
   uint32_t* dcounts = (uint32_t*)((char*)c->staging + sizeof(double) * 7 * (size_t)(tot > 0 ? tot : 1));
   k_soa_to_aos<<<blocks1d(N, 128), 128, 0, c->stream>>>(P, N, outStart, aos, dcounts);
   RH_CUDA(cudaGetLastError());
   RH_CUDA(cudaMemcpyAsync(counts, dcounts, sizeof(uint32_t) * N, cudaMemcpyDeviceToHost, c->stream));
   if (tot && particles) RH_CUDA(cudaMemcpyAsync(particles, aos, sizeof(double) * 7 * tot, cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   *n_out = tot;
   return RHGPU_OK;
}

int rhgpu_upload_particles_f32(rhgpu_ctx* c, int32_t s, const uint32_t* counts, const float* particles, int64_t n,
                               double weight) {
   if (!c || s < 0 || s >= c->ns || !counts || (n > 0 && !particles) || n < 0 || !std::isfinite(weight))
      return fail(RHGPU_ERR_ARG, "upload_particles_f32: bad arguments");
   if (c->path != RHGPU_PATH_FP32) return fail(RHGPU_ERR_ARG, "upload_particles_f32: the context is not on the FP32 form");
   RH_CUDA(cudaSetDevice(c->device));
   if (c->capHint[s] > 0 && n > c->capHint[s])
      return fail(RHGPU_ERR_CAPACITY, "upload_particles_f32: more particles than capacity");
   c->uploaded = true;
   return f32Upload(c, s, counts, nullptr, n, particles, weight);
}

int rhgpu_download_particles_f32(rhgpu_ctx* c, int32_t s, uint32_t* counts, float* particles, int64_t capacity,
                                 int64_t* n_out, double* weight_out) {
   if (!c || s < 0 || s >= c->ns || !counts || !n_out) return fail(RHGPU_ERR_ARG, "download_particles_f32: bad arguments");
   if (c->path != RHGPU_PATH_FP32) return fail(RHGPU_ERR_ARG, "download_particles_f32: the context is not on the FP32 form");
   RH_CUDA(cudaSetDevice(c->device));
   long long t = 0;
   const int rc = f32Download(c, s, counts, nullptr, capacity, &t, particles);
   *n_out = t;
   if (!rc && weight_out) *weight_out = c->f32ready ? c->f32[s].w : 0.0;
   return rc;
}

namespace {
int phasePush(rhgpu_ctx* c) {
   if (!c->inj.empty() && c->path == RHGPU_PATH_EXACT)
      return fail(RHGPU_ERR_STATE, "particle sources run on the fast and FP32 paths, not the exact path");
   if (!c->inj.empty() && c->path == RHGPU_PATH_FP32) {
      // the FP32 form stores one weight per species: a source must inject that weight
      for (const InjHost& h : c->inj) {
         if (h.d.ncells == 0 || !(h.d.w > 0)) continue;
         double& ws = c->f32[h.d.species].w;
         if (ws == 0.0) {   // a species uploaded without particles takes its source's weight
            ws = h.d.w;
            f32Exponents(c);
         } else if (std::fabs(h.d.w - ws) > 1e-12 * ws) {
            return fail(RHGPU_ERR_STATE, "FP32 form: a particle source's weight differs from its species' weight");
         }
      }
   }
   return c->path == RHGPU_PATH_FAST ? fastPush(c) : c->path == RHGPU_PATH_FP32 ? f32Push(c) : pushAll(c);
}
int phaseAccumulate(rhgpu_ctx* c) {
   if (c->path == RHGPU_PATH_FAST) return fastGather(c);
   if (c->path == RHGPU_PATH_FP32) {
      if (c->avgGroups) return fail(RHGPU_ERR_STATE, "population averages run on the fast and exact paths");
      return f32Gather(c);
   }
   return accumulateAll(c);
}
// the fast path removes boundary particles inside its push kernel
int phaseBoundaries(rhgpu_ctx* c) { return c->path == RHGPU_PATH_EXACT ? boundariesAll(c) : RHGPU_OK; }
}  // namespace

int rhgpu_set_path(rhgpu_ctx* c, int32_t path) {
   if (!c || (path != RHGPU_PATH_FAST && path != RHGPU_PATH_EXACT && path != RHGPU_PATH_FP32))
      return fail(RHGPU_ERR_ARG, "set_path: bad arguments");
   if (c->uploaded && path != c->path) return fail(RHGPU_ERR_STATE, "set_path: particles already uploaded");
   c->path = path;
   return RHGPU_OK;
}

int rhgpu_push(rhgpu_ctx* c) {
   if (!c) return fail(RHGPU_ERR_ARG, "null context");
   RH_CUDA(cudaSetDevice(c->device));
   int rc = phasePush(c);
   if (rc) return rc;
   return checkDeviceError(c);
}

int rhgpu_accumulate(rhgpu_ctx* c) {
   if (!c) return fail(RHGPU_ERR_ARG, "null context");
   RH_CUDA(cudaSetDevice(c->device));
   int rc = phaseAccumulate(c);
   if (rc) return rc;
   return checkDeviceError(c);
}

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

int rhgpu_apply_boundaries(rhgpu_ctx* c) {
   if (!c) return fail(RHGPU_ERR_ARG, "null context");
   RH_CUDA(cudaSetDevice(c->device));
   int rc = phaseBoundaries(c);
   if (rc) return rc;
   return checkDeviceError(c);
}

int rhgpu_propagate_fields(rhgpu_ctx* c) {
   if (!c) return fail(RHGPU_ERR_ARG, "null context");
   RH_CUDA(cudaSetDevice(c->device));
   int rc = fieldsAll(c);
   if (rc) return rc;
   return checkDeviceError(c);
}

int rhgpu_step(rhgpu_ctx* c, int32_t nsteps) {
   if (!c || nsteps < 0) return fail(RHGPU_ERR_ARG, "step: bad arguments");
   RH_CUDA(cudaSetDevice(c->device));
   c->launchesStep = 0;
   c->recs.clear();
   c->evUsed = 0;
   for (int n = 0; n < nsteps; ++n) {
      int rc = phasePush(c);
      if (!rc) rc = phaseAccumulate(c);
      if (!rc && c->dnOn) rc = dnApplyCtx(c);
      if (!rc) rc = phaseBoundaries(c);
      if (!rc) rc = fieldsAll(c);
      if (rc) return rc;
   }
   return checkDeviceError(c);
}

int rhgpu_device_errors(rhgpu_ctx* c, uint32_t* word_out) {
   if (!c || !word_out) return fail(RHGPU_ERR_ARG, "device_errors: bad arguments");
   RH_CUDA(cudaSetDevice(c->device));
   RH_CUDA(cudaMemcpyAsync(word_out, c->err, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   return RHGPU_OK;
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

void freeInjector(InjHost& h) {
   cudaFree(h.cells);
   cudaFree(h.rates);
   cudaFree(h.list);
   h.cells = nullptr;
   h.rates = nullptr;
   h.list = nullptr;
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

int rhgpu_get_counters(rhgpu_ctx* c, double* out, int32_t n) {
   if (!c || !out) return fail(RHGPU_ERR_ARG, "get_counters: bad arguments");
   RH_CUDA(cudaSetDevice(c->device));
   unsigned long long u[NCNT_U];
   double d[4 * MAX_SPECIES];
   RH_CUDA(cudaStreamSynchronize(c->stream));
   RH_CUDA(cudaMemcpy(u, c->cntU, sizeof u, cudaMemcpyDeviceToHost));
   RH_CUDA(cudaMemcpy(d, c->cntD, sizeof d, cudaMemcpyDeviceToHost));
   std::vector<double> v(RHGPU_NUM_FIELD_COUNTERS + RHGPU_CNT_PER_SPECIES * c->ns, 0.0);
   for (int i = 0; i < RHGPU_NUM_FIELD_COUNTERS; ++i) v[i] = (double)u[i];
   v[RHGPU_CNT_GRID_AVERAGE_COUNTER] = c->gridAvgCounter;
   for (int s = 0; s < c->ns; ++s) {
      double* q = &v[RHGPU_NUM_FIELD_COUNTERS + RHGPU_CNT_PER_SPECIES * s];
      q[0] = (double)u[CNT_SPECIES_MAXVI + s];
      q[1] = d[4 * s + 0];
      q[2] = d[4 * s + 1];
      q[3] = d[4 * s + 2];
      q[4] = d[4 * s + 3];
   }
   for (int i = 0; i < n && i < (int)v.size(); ++i) out[i] = v[i];
   return RHGPU_OK;
}

int rhgpu_get_time(rhgpu_ctx* c, double* t_out, int64_t* ts_out) {
   if (!c || !t_out || !ts_out) return fail(RHGPU_ERR_ARG, "get_time: bad arguments");
   *t_out = c->t;
   *ts_out = c->timestep;
   return RHGPU_OK;
}

void* rhgpu_stream(rhgpu_ctx* c) { return c ? (void*)c->stream : nullptr; }

int rhgpu_set_timing(rhgpu_ctx* c, int32_t enable) {
   if (!c) return fail(RHGPU_ERR_ARG, "null context");
   c->timing = enable != 0;
   return RHGPU_OK;
}

int rhgpu_get_timing(rhgpu_ctx* c, char* names, int32_t name_cap, double* ms, int32_t n, int32_t* n_out) {
   if (!c || !names || !ms || !n_out) return fail(RHGPU_ERR_ARG, "get_timing: bad arguments");
   RH_CUDA(cudaStreamSynchronize(c->stream));
   std::vector<double> tot(c->clsNames.size(), 0.0);
   for (const TimerRec& r : c->recs) {
      float x = 0;
      if (cudaEventElapsedTime(&x, c->evPool[r.ea], c->evPool[r.eb]) == cudaSuccess) tot[r.cls] += x;
   }
   std::string s;
   int m = 0;
   for (size_t q = 0; q < tot.size() && (int)q < n; ++q, ++m) {
      if (q) s += ",";
      s += c->clsNames[q];
      ms[q] = tot[q];
   }
   std::snprintf(names, name_cap, "%s", s.c_str());
   *n_out = m;
   return RHGPU_OK;
}

int rhgpu_last_launch_count(rhgpu_ctx* c, int64_t* out) {
   if (!c || !out) return fail(RHGPU_ERR_ARG, "bad arguments");
   *out = c->launchesStep;
   return RHGPU_OK;
}

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


int rhgpu_dn_create(int32_t nx, int32_t ny, int32_t nz, const int32_t* periodic, int32_t pair_capacity, int32_t device,
                    rhgpu_dn** out) {
   if (!out || !periodic || nx < 1 || ny < 1 || nz < 1 || pair_capacity < 0) return fail(RHGPU_ERR_ARG, "dn_create: bad arguments");
   RH_CUDA(cudaSetDevice(device));
   rhgpu_dn* d = new rhgpu_dn();
   d->device = device;
   d->g.nx = nx; d->g.ny = ny; d->g.nz = nz;
   for (int a = 0; a < 3; ++a) d->g.per[a] = periodic[a] ? 1 : 0;
   d->g.N = (long long)nx * ny * nz;
   const long long N = d->g.N;
   d->pairCap = pair_capacity;
   d->partRows = (N + DN_WGRAD_VOX - 1) / DN_WGRAD_VOX;
   int rc = RHGPU_OK;
   auto alloc = [&](void** p, size_t bytes) {
      if (rc) return;
      if (cudaMalloc(p, bytes) != cudaSuccess) rc = fail(RHGPU_ERR_NOMEM, "dn_create: cudaMalloc");
      else cudaMemset(*p, 0, bytes);
   };
   if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess) rc = fail(RHGPU_ERR_CUDA, "dn_create: stream");
   alloc((void**)&d->params, sizeof(float) * DN_PARAMS);
   alloc((void**)&d->grad, sizeof(float) * DN_PARAMS);
   alloc((void**)&d->m, sizeof(float) * DN_PARAMS);
   alloc((void**)&d->v, sizeof(float) * DN_PARAMS);
   alloc((void**)&d->mask, DN_PARAMS);
   alloc((void**)&d->bimg, 6 * (size_t)TC_BIMG);
   alloc((void**)&d->err, sizeof(unsigned));
   for (int l = 0; l < 3; ++l) {
      alloc((void**)&d->act[l], sizeof(unsigned) * 8 * N);
      alloc((void**)&d->dY[l], sizeof(unsigned) * 8 * N);
   }
   alloc((void**)&d->res, sizeof(float) * 4 * N);
   alloc((void**)&d->out32, sizeof(float) * 4 * N);
   alloc((void**)&d->part, sizeof(float) * d->partRows * DN_TAPS * DN_C * DN_C);
   alloc((void**)&d->lossPart, sizeof(double) * DN_LOSS_BLOCKS);
   alloc((void**)&d->acc, sizeof(double) * std::max(4 * N, 4LL * 64));   // also k_dn_err's 64 x 4 partials
   if (pair_capacity > 0) {
      alloc((void**)&d->pairIn, sizeof(float) * 4 * N * pair_capacity);
      alloc((void**)&d->pairOut, sizeof(float) * 4 * N * pair_capacity);
   }
   if (!rc) {
      // trainable entries: layer 0 reads 4 channels, layer 2 writes 4 channels
      std::vector<unsigned char> mk(DN_PARAMS, 0);
      for (int l = 0; l < 3; ++l)
         for (int t = 0; t < DN_TAPS; ++t)
            for (int ci = 0; ci < DN_C; ++ci)
               for (int co = 0; co < DN_C; ++co)
                  mk[(size_t)l * DN_LAYER + (t * DN_C + ci) * DN_C + co] = (l == 0 ? ci < 4 : true) && (l == 2 ? co < 4 : true);
      for (int l = 0; l < 3; ++l)
         for (int co = 0; co < DN_C; ++co) mk[(size_t)l * DN_LAYER + DN_TAPS * DN_C * DN_C + co] = l == 2 ? co < 4 : 1;
      if (cudaMemcpy(d->mask, mk.data(), DN_PARAMS, cudaMemcpyHostToDevice) != cudaSuccess) rc = fail(RHGPU_ERR_CUDA, "dn_create: mask");
   }
   if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = fail(RHGPU_ERR_CUDA, "dn_create: sync");
   if (rc) {
      rhgpu_dn_destroy(d);
      return rc;
   }
   *out = d;
   return RHGPU_OK;
}

int rhgpu_dn_destroy(rhgpu_dn* d) {
   if (!d) return RHGPU_OK;
   cudaSetDevice(d->device);
   if (d->stream) cudaStreamSynchronize(d->stream);
   cudaFree(d->params); cudaFree(d->grad); cudaFree(d->m); cudaFree(d->v); cudaFree(d->mask); cudaFree(d->bimg); cudaFree(d->err);
   for (int l = 0; l < 3; ++l) { cudaFree(d->act[l]); cudaFree(d->dY[l]); }
   cudaFree(d->res); cudaFree(d->out32); cudaFree(d->part); cudaFree(d->lossPart); cudaFree(d->acc);
   cudaFree(d->pairIn); cudaFree(d->pairOut);
   cudaFree(d->fullAcc); cudaFree(d->fullIn); cudaFree(d->fullOut);
   if (d->stream) cudaStreamDestroy(d->stream);
   delete d;
   return RHGPU_OK;
}

int rhgpu_dn_set_params(rhgpu_dn* d, const float* p, int64_t n) {
   if (!d || !p || n != DN_PARAMS) return fail(RHGPU_ERR_ARG, "dn_set_params: needs RHGPU_DN_PARAMS floats");
   RH_CUDA(cudaSetDevice(d->device));
   std::vector<unsigned char> mk(DN_PARAMS);
   RH_CUDA(cudaMemcpy(mk.data(), d->mask, DN_PARAMS, cudaMemcpyDeviceToHost));
   std::vector<float> h(p, p + n);
   for (int64_t e = 0; e < n; ++e) if (!mk[e]) h[e] = 0.f;
   RH_CUDA(cudaMemcpyAsync(d->params, h.data(), sizeof(float) * n, cudaMemcpyHostToDevice, d->stream));
   RH_CUDA(cudaMemsetAsync(d->m, 0, sizeof(float) * n, d->stream));
   RH_CUDA(cudaMemsetAsync(d->v, 0, sizeof(float) * n, d->stream));
   d->adamStep = 0;
   int rc = dnRebuildImages(d);
   if (rc) return rc;
   RH_CUDA(cudaStreamSynchronize(d->stream));
   return RHGPU_OK;
}

int rhgpu_dn_get_params(rhgpu_dn* d, float* p, int64_t n) {
   if (!d || !p || n != DN_PARAMS) return fail(RHGPU_ERR_ARG, "dn_get_params: needs RHGPU_DN_PARAMS floats");
   RH_CUDA(cudaSetDevice(d->device));
   RH_CUDA(cudaMemcpyAsync(p, d->params, sizeof(float) * n, cudaMemcpyDeviceToHost, d->stream));
   RH_CUDA(cudaStreamSynchronize(d->stream));
   return RHGPU_OK;
}

int rhgpu_dn_set_scales(rhgpu_dn* d, double rho_scale, double j_scale) {
   if (!d || !(rho_scale > 0) || !(j_scale > 0)) return fail(RHGPU_ERR_ARG, "dn_set_scales: scales must be positive");
   d->sr = rho_scale;
   d->sj = j_scale;
   return RHGPU_OK;
}

int rhgpu_dn_apply(rhgpu_dn* d, const double* rho_in, const double* ji_in, double* rho_out, double* ji_out, double min_rho) {
   if (!d || !rho_in || !ji_in || !rho_out || !ji_out) return fail(RHGPU_ERR_ARG, "dn_apply: bad arguments");
   RH_CUDA(cudaSetDevice(d->device));
   const long long N = d->g.N;
   int rc = dnUploadMoments(d, rho_in, ji_in, d->acc);
   if (rc) return rc;
   rc = dnApplyMoments(d, d->stream, d->acc, d->acc + N, min_rho, d->err);
   if (!rc) rc = dnCheckError(d);
   if (rc) return rc;
   std::vector<double> h(4 * (size_t)N);
   RH_CUDA(cudaMemcpyAsync(h.data(), d->acc, sizeof(double) * 4 * N, cudaMemcpyDeviceToHost, d->stream));
   RH_CUDA(cudaStreamSynchronize(d->stream));
   for (long long v = 0; v < N; ++v) {
      rho_out[v] = h[v];
      for (int l = 0; l < 3; ++l) ji_out[3 * v + l] = h[(1 + l) * N + v];
   }
   return RHGPU_OK;
}

int rhgpu_dn_loss_grad(rhgpu_dn* d, const double* rho_in, const double* ji_in, const double* rho_t, const double* ji_t,
                       double* loss, float* grad) {
   if (!d || !rho_in || !ji_in || !rho_t || !ji_t) return fail(RHGPU_ERR_ARG, "dn_loss_grad: bad arguments");
   RH_CUDA(cudaSetDevice(d->device));
   const long long N = d->g.N;
   int rc = dnUploadMoments(d, rho_t, ji_t, d->acc);
   if (rc) return rc;
   k_dn_norm<<<blocks1d(N, 256), 256, 0, d->stream>>>(N, d->acc, d->acc + N, 1.0 / d->sr, 1.0 / d->sj, d->out32);
   // target kept in dY[0]'s storage as FP32 (N x 4 floats fit in 8 u32 per voxel)
   float* target = reinterpret_cast<float*>(d->dY[0]);
   RH_CUDA(cudaMemcpyAsync(target, d->out32, sizeof(float) * 4 * N, cudaMemcpyDeviceToDevice, d->stream));
   rc = dnUploadMoments(d, rho_in, ji_in, d->acc);
   if (rc) return rc;
   k_dn_norm<<<blocks1d(N, 256), 256, 0, d->stream>>>(N, d->acc, d->acc + N, 1.0 / d->sr, 1.0 / d->sj, d->res);
   rc = dnForward(d);
   if (rc) return rc;
   // the loss kernel reads the target before the backward overwrites dY[0]
   float* tcopy = reinterpret_cast<float*>(d->acc);
   RH_CUDA(cudaMemcpyAsync(tcopy, target, sizeof(float) * 4 * N, cudaMemcpyDeviceToDevice, d->stream));
   rc = dnBackward(d, tcopy, loss);
   if (!rc) rc = dnCheckError(d);
   if (rc) return rc;
   if (grad) {
      RH_CUDA(cudaMemcpyAsync(grad, d->grad, sizeof(float) * DN_PARAMS, cudaMemcpyDeviceToHost, d->stream));
      RH_CUDA(cudaStreamSynchronize(d->stream));
   }
   return RHGPU_OK;
}

// the normalized moments of a fast-path context (4 x N floats, voxel-major):
// one in `factor` of its particles (from `offset`) with weights times factor,
// or all (factor 1); acc is 4 x N doubles of scratch
int dnDepositSample(rhgpu_dn* d, rhgpu_ctx* c, int factor, int offset, double* acc, float* out) {
   const long long N = c->g.N;
   RH_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * 4 * N, d->stream));
   for (int s = 0; s < c->ns; ++s) {
      if (!c->sp[s].accumulate) continue;
      const SegHost& h = c->seg[s];
      if (!h.a[h.cur][0]) continue;
      k_dn_subsample_deposit<<<(unsigned)c->fg.NS, 128, 0, d->stream>>>(c->g, c->fg, segView(h, h.cur), h.base,
                                                                       c->sp[s].q, factor, offset, acc);
   }
   k_dn_subsample_finish<<<blocks1d(N, 256), 256, 0, d->stream>>>(N, acc, c->g.dV, c->P.min_ion_charge_density,
                                                                 1.0 / d->sr, 1.0 / d->sj, out);
   RH_CUDA(cudaGetLastError());
   return RHGPU_OK;
}

int rhgpu_dn_add_crops(rhgpu_dn* d, rhgpu_ctx* c, int32_t factor, int32_t offset, int32_t ncrops, const int32_t* origins) {
   if (!d || !c || factor < 1 || offset < 0 || offset >= factor || ncrops < 1 || !origins)
      return fail(RHGPU_ERR_ARG, "dn_add_crops: bad arguments");
   if (d->pairCap < 1) return fail(RHGPU_ERR_STATE, "dn_add_crops: created without pair capacity");
   if (c->path != RHGPU_PATH_FAST) return fail(RHGPU_ERR_STATE, "dn_add_crops: the context must use RHGPU_PATH_FAST");
   if (c->device != d->device) return fail(RHGPU_ERR_ARG, "dn_add_crops: the device differs");
   for (int q = 0; q < ncrops; ++q) {
      const int* o = origins + 3 * q;
      if (o[0] < 0 || o[1] < 0 || o[2] < 0 || o[0] + d->g.nx > c->g.nx || o[1] + d->g.ny > c->g.ny ||
          o[2] + d->g.nz > c->g.nz)
         return fail(RHGPU_ERR_ARG, "dn_add_crops: a crop leaves the context's grid");
   }
   RH_CUDA(cudaSetDevice(d->device));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   const long long NF = c->g.N;
   if (d->fullN != NF) {
      cudaFree(d->fullAcc); cudaFree(d->fullIn); cudaFree(d->fullOut);
      d->fullAcc = nullptr; d->fullIn = nullptr; d->fullOut = nullptr;
      d->fullN = 0;
      RH_CUDA(cudaMalloc(&d->fullAcc, sizeof(double) * 4 * NF));
      RH_CUDA(cudaMalloc(&d->fullIn, sizeof(float) * 4 * NF));
      RH_CUDA(cudaMalloc(&d->fullOut, sizeof(float) * 4 * NF));
      d->fullN = NF;
   }
   int rc = dnDepositSample(d, c, factor, offset, d->fullAcc, d->fullIn);
   if (!rc) rc = dnDepositSample(d, c, 1, 0, d->fullAcc, d->fullOut);
   if (rc) return rc;
   const long long N = d->g.N;
   for (int q = 0; q < ncrops; ++q) {
      const int* o = origins + 3 * q;
      float* in = d->pairIn + (size_t)d->pairNext * 4 * N;
      float* tg = d->pairOut + (size_t)d->pairNext * 4 * N;
      k_dn_crop<<<blocks1d(N, 256), 256, 0, d->stream>>>(d->fullIn, c->g.nx, c->g.ny, d->g, o[0], o[1], o[2], in);
      k_dn_crop<<<blocks1d(N, 256), 256, 0, d->stream>>>(d->fullOut, c->g.nx, c->g.ny, d->g, o[0], o[1], o[2], tg);
      d->pairNext = (d->pairNext + 1) % d->pairCap;
      d->pairCount = std::min(d->pairCount + 1, d->pairCap);
   }
   RH_CUDA(cudaGetLastError());
   RH_CUDA(cudaStreamSynchronize(d->stream));
   return RHGPU_OK;
}

int rhgpu_dn_set_loss_border(rhgpu_dn* d, int32_t border) {
   if (!d || border < 0) return fail(RHGPU_ERR_ARG, "dn_set_loss_border: bad arguments");
   d->border = border;
   return RHGPU_OK;
}

int rhgpu_dn_add_pair(rhgpu_dn* d, rhgpu_ctx* c, int32_t factor, int32_t offset) {
   if (!d || !c || factor < 1 || offset < 0 || offset >= factor) return fail(RHGPU_ERR_ARG, "dn_add_pair: bad arguments");
   if (d->pairCap < 1) return fail(RHGPU_ERR_STATE, "dn_add_pair: created without pair capacity");
   if (c->path != RHGPU_PATH_FAST) return fail(RHGPU_ERR_STATE, "dn_add_pair: the context must use RHGPU_PATH_FAST");
   if (c->g.nx != d->g.nx || c->g.ny != d->g.ny || c->g.nz != d->g.nz || c->device != d->device)
      return fail(RHGPU_ERR_ARG, "dn_add_pair: grid or device differs");
   RH_CUDA(cudaSetDevice(d->device));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   const long long N = d->g.N;
   float* in = d->pairIn + (size_t)d->pairNext * 4 * N;
   float* tg = d->pairOut + (size_t)d->pairNext * 4 * N;
   // input: one in `factor` particles, weights times factor; target: all particles,
   // by the same deposit of the same state
   int rc = dnDepositSample(d, c, factor, offset, d->acc, in);
   if (!rc) rc = dnDepositSample(d, c, 1, 0, d->acc, tg);
   if (rc) return rc;
   RH_CUDA(cudaStreamSynchronize(d->stream));
   d->pairNext = (d->pairNext + 1) % d->pairCap;
   d->pairCount = std::min(d->pairCount + 1, d->pairCap);
   return RHGPU_OK;
}

int rhgpu_dn_train(rhgpu_dn* d, int32_t iterations, float lr, double* mean_loss) {
   if (!d || iterations < 0 || !(lr > 0)) return fail(RHGPU_ERR_ARG, "dn_train: bad arguments");
   if (d->pairCount < 1) return fail(RHGPU_ERR_STATE, "dn_train: no training pairs");
   RH_CUDA(cudaSetDevice(d->device));
   const long long N = d->g.N;
   double tot = 0.0;
   const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
   for (int it = 0; it < iterations; ++it) {
      d->rng = d->rng * 6364136223846793005ull + 1442695040888963407ull;
      const int p = (int)((d->rng >> 33) % (unsigned long long)d->pairCount);
      RH_CUDA(cudaMemcpyAsync(d->res, d->pairIn + (size_t)p * 4 * N, sizeof(float) * 4 * N, cudaMemcpyDeviceToDevice, d->stream));
      int rc = dnForward(d);
      if (rc) return rc;
      double l = 0.0;
      rc = dnBackward(d, d->pairOut + (size_t)p * 4 * N, &l);
      if (rc) return rc;
      tot += l;
      d->adamStep += 1;
      const float c1 = 1.f - std::pow(b1, (float)d->adamStep), c2 = 1.f - std::pow(b2, (float)d->adamStep);
      k_dn_adam<<<(DN_PARAMS + 255) / 256, 256, 0, d->stream>>>(d->params, d->grad, d->m, d->v, d->mask, DN_PARAMS, lr, b1, b2,
                                                               eps, c1, c2);
      rc = dnRebuildImages(d);
      if (rc) return rc;
   }
   RH_CUDA(cudaStreamSynchronize(d->stream));
   if (int rc = dnCheckError(d)) return rc;
   if (mean_loss) *mean_loss = iterations ? tot / iterations : 0.0;
   return RHGPU_OK;
}

int rhgpu_set_denoiser(rhgpu_ctx* c, rhgpu_dn* d, int32_t enabled) {
   if (!c) return fail(RHGPU_ERR_ARG, "set_denoiser: null context");
   if (d && (c->g.nx != d->g.nx || c->g.ny != d->g.ny || c->g.nz != d->g.nz || c->device != d->device ||
             c->g.per[0] != d->g.per[0] || c->g.per[1] != d->g.per[1] || c->g.per[2] != d->g.per[2]))
      return fail(RHGPU_ERR_ARG, "set_denoiser: grid or device differs");
   c->dn = d;
   c->dnOn = d && enabled;
   return RHGPU_OK;
}


int rhgpu_dn_pair_error(rhgpu_dn* d, int32_t pair, double* out4) {
   if (!d || !out4 || pair < 0 || pair >= d->pairCount) return fail(RHGPU_ERR_ARG, "dn_pair_error: bad arguments");
   RH_CUDA(cudaSetDevice(d->device));
   const long long N = d->g.N;
   const float* in = d->pairIn + (size_t)pair * 4 * N;
   const float* tg = d->pairOut + (size_t)pair * 4 * N;
   RH_CUDA(cudaMemcpyAsync(d->res, in, sizeof(float) * 4 * N, cudaMemcpyDeviceToDevice, d->stream));
   int rc = dnForward(d);
   if (rc) return rc;
   std::vector<double> h(4 * 64);
   double r[2][4];
   for (int which = 0; which < 2; ++which) {
      k_dn_err<<<64, 256, 0, d->stream>>>(N, which ? d->out32 : in, tg, d->acc);
      RH_CUDA(cudaGetLastError());
      RH_CUDA(cudaMemcpyAsync(h.data(), d->acc, sizeof(double) * 4 * 64, cudaMemcpyDeviceToHost, d->stream));
      RH_CUDA(cudaStreamSynchronize(d->stream));
      for (int q = 0; q < 4; ++q) {
         r[which][q] = 0.0;
         for (int b = 0; b < 64; ++b) r[which][q] += h[b * 4 + q];
      }
   }
   out4[0] = std::sqrt(r[0][0] / r[0][1]);   // raw rho
   out4[1] = std::sqrt(r[0][2] / r[0][3]);   // raw J
   out4[2] = std::sqrt(r[1][0] / r[1][1]);   // denoised rho
   out4[3] = std::sqrt(r[1][2] / r[1][3]);   // denoised J
   return RHGPU_OK;
}

int rhgpu_dn_num_pairs(rhgpu_dn* d, int32_t* n_out, int32_t* newest) {
   if (!d || !n_out || !newest) return fail(RHGPU_ERR_ARG, "dn_num_pairs: bad arguments");
   *n_out = d->pairCount;
   *newest = d->pairCount ? (d->pairNext + d->pairCap - 1) % d->pairCap : -1;
   return RHGPU_OK;
}

}  // extern "C"
