// Host side of the library, shared by its translation units: the context
// (rhgpu_ctx) and the denoiser (rhgpu_dn) with their device storage, error
// reporting, kernel timing, and the helpers that one part calls in another.
//   rhgpu.cu          context, grid arrays, particle upload / download, the
//                     per-step launch sequence replaying RHybrid's propagate()
//                     (src/user.cpp:118-134), the field update, counters, timing
//   rhgpu_exact.cu    the exact particle path (the reference's order) and the
//                     allocation-free deposit
//   rhgpu_fast.cu     the fast particle path (row-segment storage)
//   rhgpu_f32.cu      the FP32 precision form
//   rhgpu_sources.cu  particle sources and the uniform fill
//   rhgpu_diag.cu     log sums and files, temporal averages, grid counters
//   rhgpu_denoise.cu  the learned moment denoiser
// The kernels are declared in k_*.cuh and defined in k_*.cu (template kernels
// in the headers).
#pragma once

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

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
#include "k_util.cuh"
#include "rh_logs.h"

using namespace rh;

namespace rhh {

// the message of the last error of this host thread (rhgpu_last_error)
extern thread_local std::string g_err;
int fail(int code, const std::string& msg);

#define RH_CUDA(call)                                                                     \
   do {                                                                                   \
      cudaError_t e_ = (call);                                                            \
      if (e_ != cudaSuccess) return fail(RHGPU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
   } while (0)

const int MAX_SPECIES = 8;
const int NCNT_U = 32;   // field counters 0..15, species MaxVi at 16+s

struct TimerRec { int cls; int ea, eb; };

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

}  // namespace rhh

using namespace rhh;

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
   int vel = 0;                          // velocity form (rhgpu_dn_set_velocity_form)
   unsigned char* keep = nullptr;        // per cell: moments left as deposited (rhgpu_dn_set_keep_mask)
};

namespace rhh {

inline dim3 cellBlock() { return dim3(32, 4, 1); }
inline dim3 cellGrid(const GridInfo& g) { return dim3((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz); }
inline unsigned blocks1d(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// kernel timing (rhgpu_get_timing): one launch bracketed by CUDA events of its class
int timerBegin(rhgpu_ctx* c, const char* name);
void timerEnd(rhgpu_ctx* c, int r);
struct KScope {
   rhgpu_ctx* c;
   int r;
   KScope(rhgpu_ctx* c_, const char* n) : c(c_), r(timerBegin(c_, n)) {}
   ~KScope() { timerEnd(c, r); }
};
#define RH_TIME(c, name) KScope rh_scope_(c, name)

#define RH_LAUNCHED(c) do { int rc_ = checkLaunch(c); if (rc_) return rc_; } while (0)

template <class T>
inline int growBuffer(T*& p, long long& have, long long need) {
   if (need <= have) return RHGPU_OK;
   cudaFree(p);
   p = nullptr;
   have = 0;
   const long long n = need + need / 8 + 64;
   RH_CUDA(cudaMalloc(&p, sizeof(T) * n));
   have = n;
   return RHGPU_OK;
}

// slots to allocate for `slots` particles in a buffer of `have` slots (0: a
// first allocation): 1/16 more, and when a buffer grows again at least a
// quarter more than it had, so that a run whose particle count keeps rising
// reallocates (a synchronous free and allocation inside a step) rarely
inline long long growSlots(long long have, long long slots) {
   const long long n = slots + slots / 16 + 1024;
   return have > 0 ? std::max(n, have + have / 4) : n;
}

// the periodic axes of a grid as a 3-bit mask (bit a = axis a)
inline int perMask(const GridInfo& g) { return (g.per[0] ? 1 : 0) | (g.per[1] ? 2 : 0) | (g.per[2] ? 4 : 0); }

// ---- context, storage and the step (rhgpu.cu)
int checkLaunch(rhgpu_ctx* c);
long long scanScratchLongs(long long n);
int scanExclusive64(rhgpu_ctx* c, const long long* in, long long* out, long long n);
SpeciesDev speciesDev(const rhgpu_ctx* c, int s);
int ensureKeyCapacity(rhgpu_ctx* c, long long n);
int ensureStaging(rhgpu_ctx* c, size_t bytes);
int checkDeviceError(rhgpu_ctx* c);
int fieldsAll(rhgpu_ctx* c);

// ---- exact path (rhgpu_exact.cu)
int allocStore(PStore& s, long long cap, long long N);
void freeStore(PStore& s);
int pushAll(rhgpu_ctx* c);
// species whose particles the exact-path deposit adds (accumulating, particles uploaded)
inline bool deposits(const rhgpu_ctx* c, int s) { return c->sp[s].accumulate && c->ps[s].start; }
// exact-path deposit with the 108 per-cell sums in S (108 * N doubles)
int depositExact(rhgpu_ctx* c, double* S);
int accumulateAll(rhgpu_ctx* c);
int boundariesAll(rhgpu_ctx* c);

// ---- fast path (rhgpu_fast.cu)
int ensureSortTmp(rhgpu_ctx* c, size_t bytes);
SegBuf segView(const SegHost& h, int which);
int segReserve(SegHost& h, int which, long long slots);
int fastLayout(rhgpu_ctx* c, const int* cnt, const int* extra, long long* base, long long* total);
int fastExponents(rhgpu_ctx* c);
int ensureMigBuffers(rhgpu_ctx* c, long long want);
long long moverListSize(long long slots);
int fastMoverBuffers(rhgpu_ctx* c);
int bitsFor(long long x);
int segPrefix(rhgpu_ctx* c, const int* cnt, long long* total);
int fastUpload(rhgpu_ctx* c, int s, const uint32_t* counts, const double* particles, long long n);
int fastNumParticles(rhgpu_ctx* c, int s, long long* n);
int fastDownload(rhgpu_ctx* c, int s, uint32_t* counts, double* particles, long long capacity, long long* n_out);
int fastPush(rhgpu_ctx* c);
int fastGather(rhgpu_ctx* c);

// ---- FP32 form (rhgpu_f32.cu)
F32Buf f32View(const F32Host& h, int which);
int f32Reserve(F32Host& h, int which, long long slots);
int f32Init(rhgpu_ctx* c);
void f32Exponents(rhgpu_ctx* c);
int f32MoverBuffers(rhgpu_ctx* c);
int f32Upload(rhgpu_ctx* c, int s, const uint32_t* counts, const double* particles, long long n,
              const float* particles32 = nullptr, double weight32 = 0.0);
int f32NumParticles(rhgpu_ctx* c, int s, long long* n);
int f32Download(rhgpu_ctx* c, int s, uint32_t* counts, double* particles, long long capacity, long long* n_out,
                float* particles32 = nullptr);
int f32Push(rhgpu_ctx* c);
int f32Gather(rhgpu_ctx* c);

// ---- denoiser (rhgpu_denoise.cu) and particle sources (rhgpu_sources.cu)
int dnApplyCtx(rhgpu_ctx* c);
void freeInjector(InjHost& h);

// the movers' placement order (rhgpu_fast.cu; instantiated for the fast path's
// and the FP32 form's movers) and the particle sources of a step appended to
// a mover list
template <class MV, class SET>
int migSort(rhgpu_ctx* c, const MV* mv, long long nm, const SET& FS, unsigned** order, unsigned** bucket, int* over);
template <class MV>
int injectAll(rhgpu_ctx* c, MV* movers, long long moverCap);

}  // namespace rhh
