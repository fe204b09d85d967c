// Field update propagateB (RHybrid src/hybrid_propagator.cpp:42-440) as
// FP64 stencil kernels for sm_100a. Each kernel restates one or more of the
// reference's per-block routines with the reference's operation order, so
// that with --fmad=false the results are bitwise identical:
//   k_face2cell          face2Cell                        (:1043-1056)
//   k_ext_bc             neumannCell x3 + setIMFCell, neumannFace + setIMFFace
//                        (:443-908, :910-1040)
//   k_node_fused         cell2Node of B, rhoq, Ji + cellAverageB, calcNodeJ
//                        (USE_EDGE_J), calcNodeUe, upwindNodeB, calcNodeE
//                        (:1059-1089, :157-167, :1449-1522, :1524-1584, :1268-1339, :1392-1446)
//   k_cell_tiled         node2Cell(J) + calcCellUe, calcCellEp, faceCurl
//                        (:1092-1112, :1342-1387, :1674-1737, :1587-1671)
//   k_ext_cell_neumann3  neumannCell of one 3-vector      (:443-655)
//   k_node2cell3, k_cell2node3, k_node_avg, k_faraday   nodeE smoothing and the
//                        Faraday step after it (:354-404, :1115-1265, :1587-1671)
// Exterior-cell kernels run over the list of cells missing a neighbour. In
// the reference those loops are sequential, but every value an exterior cell
// receives comes from a cell (or a component) that the same loop does not
// write, so running them in parallel gives the same result (checked bitwise
// against the reference on closed boxes by tests/test_gpu_parity.py).
#pragma once

#include "rh_device.cuh"

namespace rh {

struct Fields {
   double* faceB;   double* cellB;   double* cellUe;  double* cellEp;
   double* cellRho; double* cellJi;  double* cellJ;   double* nodeRho;
   double* nodeJi;  double* nodeJ;   double* nodeUe;  double* nodeB;
   double* nodeE;   double* nodeEta; double* cellAvgB;
   double* tmp3;    // scratch 3-vector (Gaussian smoothing)
   const uint8_t* flags;
   double* gc;      // per-cell grid constraint counters, GC_PLANES planes of N, or null (off)
};

// per-cell grid constraint counters (USE_GRID_CONSTRAINT_COUNTERS): how often
// each cell (node) hit a limit; the node Ue limit counts in the cell plane, as
// the reference does (hybrid_propagator.cpp:1579)
enum GridCounterPlane { GC_CELL_MAX_UE = 0, GC_CELL_MAX_VI, GC_CELL_MIN_RHOQI, GC_NODE_MAX_E, GC_NODE_MAX_VW, GC_PLANES };
__device__ inline void gridCount(const Fields& f, int plane, long long N, long long n, bool hit) {
   if (hit && f.gc) f.gc[plane * N + n] += 1.0;
}
__device__ inline void gridCountAtomic(const Fields& f, int plane, long long N, long long n, bool hit) {
   if (hit && f.gc) atomicAdd(&f.gc[plane * N + n], 1.0);
}

struct FieldParams {
   int use_hall, use_ep, isothermal;
   double ep_coeff;
   double obstacleUe[3];
   double maxUe2, minRho, maxE2, maxVw;
   double gauss[4];
   double imf[3];
   int imfCell[6], imfFace[6];
};

// neumann source tables, indexed by missing-wall mask (64 entries):
// cell: offset of the last matching rule (all components); face: per component
struct NeumannTables {
   signed char cellSrc[64][3];
   signed char faceSrc[64][3][3];
   unsigned char faceUse[64][3];
};
// the tables in constant memory (k_fields.cu), read by k_ext_cell_neumann3 and k_ext_bc
cudaError_t setNeumannTables(const NeumannTables& t);

// counter slots in the device counter array
enum {
   CNT_MIN_CELL_RHO = RHGPU_CNT_FIELD_MIN_CELL_RHOQI,
   CNT_MAX_CELL_UE = RHGPU_CNT_FIELD_MAX_CELL_UE,
   CNT_MAX_NODE_UE = RHGPU_CNT_FIELD_MAX_NODE_UE,
   CNT_MAX_VW = RHGPU_CNT_FIELD_MAX_VW,
   CNT_MAX_E = RHGPU_CNT_FIELD_MAX_E,
   CNT_MIN_NODE_RHO = RHGPU_CNT_FIELD_MIN_NODE_RHOQI,
   CNT_SPECIES_MAXVI = 16   // + species
};

__device__ inline void countIf(bool pred, unsigned long long* c) {
   const unsigned act = __activemask();
   const unsigned m = __ballot_sync(act, pred);
   if (m && (threadIdx.x & 31) == (unsigned)(__ffs(act) - 1)) atomicAdd(c, (unsigned long long)__popc(m));
}

__device__ inline double sq(double x) { return x * x; }

#define RH_CELL_PROLOGUE                                          \
   const int i = blockIdx.x * blockDim.x + threadIdx.x;           \
   const int j = blockIdx.y * blockDim.y + threadIdx.y;           \
   const int k = blockIdx.z;                                      \
   if (i >= g.nx || j >= g.ny) return;                            \
   const long long n = cidx(g, i, j, k);                          \
   const long long N = g.N;                                       \
   (void)N;

__global__ void k_face2cell(GridInfo g, Fields f);

__device__ inline void extCellIJK(const GridInfo& g, int c, int& i, int& j, int& k) {
   i = c % g.nx;
   j = (c / g.nx) % g.ny;
   k = c / (g.nx * g.ny);
}

// neumannCell of one 3-vector (cellUe, or cellJ during smoothing)
__global__ void k_ext_cell_neumann3(GridInfo g, double* a, const int* ext, int next);

// cell2Node of a 3-vector (smoothing: cellJ -> nodeE)
__global__ void k_cell2node3(GridInfo g, const double* src, double* dst);

// node2Cell of a 3-vector (smoothing: nodeE -> cellJ)
__global__ void k_node2cell3(GridInfo g, const double* src, double* dst);

// nodeAvg: 27-point Gaussian of nodeE. Neighbours that do not exist read 0,
// except the (-,-,-) corner x component, which reads the exclusion marker
// (the reference's temp array has only its first element set to max()).
__global__ void k_node_avg(GridInfo g, const double* old, double* out, FieldParams fp);

// faceCurl(nodeE -> faceB, Faraday): faceB += dt curl(E)
__global__ void k_faraday(GridInfo g, Fields f);

// ---- the field update in fewer passes ------------------------------------------------------
// The reference's propagateB steps, fused where one pass can form the values
// the next one reads, each expression in the reference's order (bit for bit):
//   k_ext_bc      neumannCell(cellB, cellJi, cellRhoQi) / setIMFCell and
//                 neumannFace / setIMFFace(faceB) of the exterior cells
//                 (hybrid_propagator.cpp:443-908; disjoint arrays)
//   k_node_fused  per node: cellAverageB += cellB, cell2Node (nodeB, nodeRhoQi,
//                 nodeJi), calcNodeJ (edge curls of faceB / (2 dx mu0 d), the
//                 whistler limiter d), then calcNodeUe, upwindNodeB and calcNodeE;
//                 the averaged nodeB that the whistler limiter reads stays in
//                 registers, the upwind weights re-read the same eight cells
//   k_cell_tiled  per cell: node2Cell of nodeJ and calcCellUe, calcCellEp (the
//                 gradient of face-averaged nodeRhoQi), and (FARADAY: no E
//                 smoothing) faceCurl, faceB += dt curl E; none of them reads
//                 what another writes
// k_cell_tiled reads its eight-point stencils from node layers staged in shared
// memory. The node pass reads its cells directly: its FP64 work per node (eight
// square roots and divisions) keeps it issue-bound, and a staged version with
// fewer resident warps took 0.42 ms against 0.33 ms for this one.
// The cellUe Neumann pass (k_ext_cell_neumann3) follows k_cell_tiled; calcNodeUe
// and calcNodeE do not read cellUe, so its place before them in the reference's
// order does not matter.
__global__ void k_ext_bc(GridInfo g, Fields f, FieldParams fp, const int* ext, int next);

__global__ void __launch_bounds__(128, 8) k_node_fused(GridInfo g, Fields f, FieldParams fp, unsigned long long* cnt);

// ---- the cell pass, its node stencil in shared memory ------------------------------------------
// A block of 32 x 4 cells marches NT_Z planes along z; the node layers k - 1
// and k that a plane of cells reads (nodeJ, nodeRhoQi, nodeE over 33 x 5 nodes
// from (i0 - 1, j0 - 1)) sit in a ring of three layer slots, the next one
// copied in with cp.async while the current plane is computed, so every node
// value is loaded once per block instead of once per cell reading it.
constexpr int NT_X = 32, NT_Y = 4, NT_Z = 8;
constexpr int NT_LX = NT_X + 1, NT_LY = NT_Y + 1;
constexpr int CT_ARR = 7;    // nodeJ x 3, nodeRhoQi, nodeE x 3
constexpr int CT_LAYER = CT_ARR * NT_LY * NT_LX;
constexpr size_t CT_SMEM = 3 * CT_LAYER * sizeof(double);

// node (dx, dy, dz) in {-1, 0}^3 of a cell's stencil, o = (dx + 1) + 2 (dy + 1) + 4 (dz + 1)
struct CellStencil {
   const double* L;   // node layer k - 1
   const double* U;   // node layer k
   int off;           // this cell's (x, y) in a layer
   __device__ __forceinline__ double at(int a, int o) const {
      return ((o & 4) ? U : L)[a * (NT_LY * NT_LX) + off + ((o >> 1) & 1) * NT_LX + (o & 1)];
   }
   __device__ __forceinline__ double nj(int l, int o) const { return at(l, o); }
   __device__ __forceinline__ double nr(int o) const { return at(3, o); }
   __device__ __forceinline__ double ne(int l, int o) const { return at(4 + l, o); }
};

__device__ __forceinline__ void ctStage(const GridInfo& g, const Fields& f, double* dst, int i0, int j0, int kz) {
   int z = kz;
   const bool zok = wrapc(z, g.nz, g.per[2]);
   const long long N = g.N;
   for (int e = threadIdx.x + NT_X * threadIdx.y; e < CT_LAYER; e += NT_X * NT_Y) {
      const int a = e / (NT_LY * NT_LX), r = e - a * (NT_LY * NT_LX), jj = r / NT_LX, ii = r - jj * NT_LX;
      int x = i0 - 1 + ii, y = j0 - 1 + jj;
      const bool ok = zok && wrapc(x, g.nx, g.per[0]) && wrapc(y, g.ny, g.per[1]);
      const double* arr = a < 3 ? f.nodeJ + a * N : a == 3 ? f.nodeRho : f.nodeE + (a - 4) * N;
      cpAsync8(dst + e, ok ? arr + cidx(g, x, y, z) : f.faceB, ok ? 8 : 0);
   }
}

template <bool FARADAY>
__device__ __forceinline__ void cellFromStencil(const GridInfo& g, const Fields& f, const FieldParams& fp, int useEp,
                                                unsigned long long* cnt, int i, int j, int k, long long n,
                                                const CellStencil& st) {
   const long long N = g.N;
   const bool inner = allNb(g, i, j, k);
   bool clamp = false;
   if (inner) {
      constexpr int a0 = 7, a1 = 6, a2 = 4, a3 = 5, a4 = 3, a5 = 1, a6 = 2, a7 = 0;
      // node2Cell(nodeJ -> cellJ), calcCellUe
      double J[3];
      for (int l = 0; l < 3; ++l) {
         J[l] = 0.125 * (st.nj(l, a0) + st.nj(l, a1) + st.nj(l, a2) + st.nj(l, a3) + st.nj(l, a4) + st.nj(l, a5) +
                         st.nj(l, a6) + st.nj(l, a7));
         f.cellJ[l * N + n] = J[l];
      }
      double Ue[3];
      const unsigned char fl = f.flags[n];
      if (fl & RHGPU_FLAG_INNER_FIELD) {
         for (int l = 0; l < 3; ++l) Ue[l] = fp.obstacleUe[l];
      } else {
         const double rho = f.cellRho[n];
         for (int l = 0; l < 3; ++l) {
            if (fabs(rho) > 0) {
               if (fp.use_hall) Ue[l] = -(J[l] - f.cellJi[l * N + n]) / rho;
               else Ue[l] = f.cellJi[l * N + n] / rho;
            } else {
               Ue[l] = 0.0;
            }
         }
         const double Ue2 = sq(Ue[0]) + sq(Ue[1]) + sq(Ue[2]);
         if (Ue2 > fp.maxUe2) {
            const double norm = sqrt(fp.maxUe2 / Ue2);
            Ue[0] *= norm; Ue[1] *= norm; Ue[2] *= norm;
            clamp = true;
         }
      }
      for (int l = 0; l < 3; ++l) f.cellUe[l * N + n] = Ue[l];
      // calcCellEp (reads the clamped nodeRhoQi)
      if (useEp) {
         double Ep[3] = {0.0, 0.0, 0.0};
         if (!(fl & RHGPU_FLAG_INNER_CELLEP)) {
            constexpr int o000 = a0, o00m = a4, o0mm = a5, o0m0 = a3, om00 = a1, om0m = a6, ommm = a7, omm0 = a2;
            const double xPos = 0.25 * (st.nr(o000) + st.nr(o00m) + st.nr(o0mm) + st.nr(o0m0));
            const double xNeg = 0.25 * (st.nr(om00) + st.nr(om0m) + st.nr(ommm) + st.nr(omm0));
            const double yPos = 0.25 * (st.nr(o000) + st.nr(o00m) + st.nr(om0m) + st.nr(om00));
            const double yNeg = 0.25 * (st.nr(o0m0) + st.nr(o0mm) + st.nr(ommm) + st.nr(omm0));
            const double zPos = 0.25 * (st.nr(o000) + st.nr(o0m0) + st.nr(omm0) + st.nr(om00));
            const double zNeg = 0.25 * (st.nr(o00m) + st.nr(o0mm) + st.nr(ommm) + st.nr(om0m));
            const double gx = (xPos - xNeg) / g.dx, gy = (yPos - yNeg) / g.dx, gz = (zPos - zNeg) / g.dx;
            const double C = fp.ep_coeff;
            if (!fp.isothermal) {
               Ep[0] = -C * gx; Ep[1] = -C * gy; Ep[2] = -C * gz;
            } else if (fabs(f.cellRho[n]) > 0) {
               const double rho = f.cellRho[n];
               Ep[0] = -C * gx / rho; Ep[1] = -C * gy / rho; Ep[2] = -C * gz / rho;
            }
         }
         for (int l = 0; l < 3; ++l) f.cellEp[l * N + n] = Ep[l];
      }
   }
   countIf(clamp, &cnt[CNT_MAX_CELL_UE]);
   gridCount(f, GC_CELL_MAX_UE, N, n, clamp);
   if (!FARADAY) return;
   // faceCurl(nodeE -> faceB)
   bool doX = true, doY = true, doZ = true;
   if (!inner) {
      if (!plusOk(g, i, j, k)) return;
      if (!xNeg(g, i)) { doY = doZ = false; }
      if (!yNeg(g, j)) { doX = doZ = false; }
      if (!zNeg(g, k)) { doX = doY = false; }
   }
   const double dx = g.dx, dt = g.dt;
   if (doX) {
      constexpr int s5 = 5, s6 = 1, s7 = 3, s8 = 7;
      const double n5y = st.ne(1, s5), n5z = st.ne(2, s5), n6y = st.ne(1, s6), n6z = st.ne(2, s6);
      const double n7y = st.ne(1, s7), n7z = st.ne(2, s7), n8y = st.ne(1, s8), n8z = st.ne(2, s8);
      const double curlX = 0.5 * (+n5z + n6z - n6y - n7y - n7z - n8z + n8y + n5y) / dx;
      f.faceB[0 * N + n] += dt * curlX;
   }
   if (doY) {
      constexpr int s3 = 2, s4 = 6, s7 = 3, s8 = 7;
      const double n3x = st.ne(0, s3), n3z = st.ne(2, s3), n4x = st.ne(0, s4), n4z = st.ne(2, s4);
      const double n7x = st.ne(0, s7), n7z = st.ne(2, s7), n8x = st.ne(0, s8), n8z = st.ne(2, s8);
      const double curlY = 0.5 * (-n4x - n8x + n8z + n7z + n7x + n3x - n3z - n4z) / dx;
      f.faceB[1 * N + n] += dt * curlY;
   }
   if (doZ) {
      constexpr int s1 = 4, s4 = 6, s5 = 5, s8 = 7;
      const double n1x = st.ne(0, s1), n1y = st.ne(1, s1), n4x = st.ne(0, s4), n4y = st.ne(1, s4);
      const double n5x = st.ne(0, s5), n5y = st.ne(1, s5), n8x = st.ne(0, s8), n8y = st.ne(1, s8);
      const double curlZ = 0.5 * (-n1x - n5x - n5y - n8y + n8x + n4x + n4y + n1y) / dx;
      f.faceB[2 * N + n] += dt * curlZ;
   }
}

template <bool FARADAY>
__global__ void __launch_bounds__(NT_X * NT_Y) k_cell_tiled(GridInfo g, Fields f, FieldParams fp, int useEp,
                                                            unsigned long long* cnt) {
   extern __shared__ __align__(16) double ctLayers[];
   const int tx = threadIdx.x, ty = threadIdx.y;
   const int i0 = blockIdx.x * NT_X, j0 = blockIdx.y * NT_Y, k0 = blockIdx.z * NT_Z;
   const int i = i0 + tx, j = j0 + ty;
   const int nk = min(NT_Z, g.nz - k0);
   const bool mine = i < g.nx && j < g.ny;
   ctStage(g, f, ctLayers, i0, j0, k0 - 1);
   ctStage(g, f, ctLayers + CT_LAYER, i0, j0, k0);
   cpAsyncCommit();
   if (nk > 1) ctStage(g, f, ctLayers + 2 * CT_LAYER, i0, j0, k0 + 1);
   cpAsyncCommit();
   for (int t = 0; t < nk; ++t) {
      cpAsyncWaitGroup<1>();   // node layers k - 1 and k are in
      __syncthreads();
      CellStencil st;
      st.L = ctLayers + (t % 3) * CT_LAYER;
      st.U = ctLayers + ((t + 1) % 3) * CT_LAYER;
      st.off = ty * NT_LX + tx;
      const int k = k0 + t;
      if (mine) cellFromStencil<FARADAY>(g, f, fp, useEp, cnt, i, j, k, cidx(g, i, j, k), st);
      __syncthreads();         // layer k - 1 is read by every thread: its slot takes layer k + 2
      if (t + 3 <= nk) ctStage(g, f, ctLayers + (t % 3) * CT_LAYER, i0, j0, k0 + t + 2);
      cpAsyncCommit();
   }
}

}  // namespace rh
