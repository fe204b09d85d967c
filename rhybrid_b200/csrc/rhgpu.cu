// rhgpu: C ABI (include/rhgpu.h) of the B200 hybrid-PIC hot path. This part:
// the context and its device memory, grid arrays in the ParGrid layout,
// particle upload / download (dispatched to the path's storage), the per-step
// launch sequence replaying RHybrid's propagate() (src/user.cpp:118-134), the
// field update propagateB, counters and kernel timing. rhgpu_host.h lists the
// other parts.
#include "rhgpu_host.h"

namespace rhh {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
   g_err = msg;
   return code;
}

}  // namespace rhh

namespace {

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

}  // namespace

namespace rhh {

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

int checkLaunch(rhgpu_ctx* c) {
   c->launches++;
   c->launchesStep++;
   cudaError_t e = cudaGetLastError();
   if (e != cudaSuccess) return fail(RHGPU_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
   return RHGPU_OK;
}

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

int ensureStaging(rhgpu_ctx* c, size_t bytes) {
   if (bytes <= c->stagingBytes) return RHGPU_OK;
   cudaFree(c->staging);
   c->staging = nullptr;
   c->stagingBytes = 0;
   RH_CUDA(cudaMalloc(&c->staging, bytes));
   c->stagingBytes = bytes;
   return RHGPU_OK;
}

}  // namespace rhh

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
      if (setNeumannTables(t) != cudaSuccess) rc = fail(RHGPU_ERR_CUDA, "neumann tables");
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

}  // extern "C"
