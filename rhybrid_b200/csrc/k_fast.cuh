// Fast path (sm_100a, FP64): fused push + CIC deposit over particles binned
// by row segment. Same per-particle and per-cell arithmetic as the bit-exact
// path (boris.h:64-194, particle_accumulator.cpp:65-333); the deposit sums are
// formed in a different, fixed order, restated bit for bit by the oracle's
// RHO_DEPOSIT_GPU mode (oracle/rh_oracle.c).
//
// Dual cells: the 2x2x2 block of cells whose centres surround a particle
// (base b = c + s - 1 per axis, s = 0 if x < 0.5 dx else 1, the index shift of
// accumulateCell, particle_accumulator.cpp:78-84). Dual index u = b + 1 on a
// non-periodic axis (n + 1 dual cells), b mod n on a periodic one.
//
// Storage (per species, structure of arrays): a dual row (uy, uz) is cut into
// segments of RHGPU_FAST_SEGMENT dual cells along x; segment S = row * nseg + g
// owns the slots [base[S], base[S+1]) (slack included), the first cnt[S] hold
// its particles with their dual x index within the segment (lx, one byte).
// Two buffers per species (current, next) share the layout.
//
//   k_fast_push_deposit  one block per segment, one thread per particle:
//                        push + migration + CIC weights of the new position +
//                        boundary removal (particle_boundary_cond_hybrid.h:112-185).
//                        The field stencil and each chunk of particles are
//                        copied to shared memory with per-thread cp.async, the
//                        next chunk while the current one is processed.
//                        Particles that stay in the segment are written to the
//                        next buffer in order; their deposit records go to
//                        shared memory counting-sorted by target dual cell
//                        (stable) and are summed sequentially per (dual cell,
//                        corner, moment) in FP64, one thread per (dual cell,
//                        corner). Particles that leave the segment go to the
//                        mover list.
//   k_fast_mover_deposit the movers' CIC contributions as exact 128-bit
//                        fixed-point sums (order-independent)
//   k_mig_*, k_fast_mig_place  placement of the movers after the stayers of their
//                        destination segment, in (source segment, index) order
//   k_fast_gather        cell moments from the four row partials (+ the segment
//                        boundary partial) + the fixed-point part, then /dV and
//                        the rho clamp (particle_accumulator.cpp:319-333)
#pragma once

#include "rh_device.cuh"
#include "k_fields.cuh"
#include "k_particles.cuh"

namespace rh {

constexpr int FAST_MAX_SPECIES = 8;
constexpr int SEG = RHGPU_FAST_SEGMENT;   // dual cells per segment
constexpr int FT = 256;                   // threads of k_fast_push_deposit (one chunk of particles)
constexpr int FW = FT / 32;
constexpr int REC = 11;                   // doubles per deposit record: w8[8], v[3]
static_assert(SEG == 32 && SEG * 8 == FT, "the deposit sums map (dual cell, corner) to one thread");

struct SegBuf {
   double* a[7];        // x, y, z (cell-local), vx, vy, vz, weight
   unsigned char* lx;   // dual x index within the segment
   int* cnt;            // particles per segment
};
struct SegSpecies {
   SegBuf cur, nxt;
   const long long* base;   // NS+1 slot offsets
};
struct FastSpecies {
   int ns;
   SegSpecies st[FAST_MAX_SPECIES];
   SpeciesDev sp[FAST_MAX_SPECIES];
};
struct FastGeom {
   int nd[3];        // dual cells per axis
   int nseg;         // segments per dual row
   long long nrows;  // dual rows
   long long NS;     // segments
};

// a particle leaving its segment: key orders the arrivals of a destination
// segment, (source segment << 32) | index in the source segment
struct Mover {
   double s[7];
   unsigned long long key;
   long long dest;   // destination segment
   int species;
   int lx;           // dual x in the destination segment | MOVER_* flags
};
constexpr int MOVER_DEPOSIT = 1 << 8;   // deposits its CIC contributions (fixed point)
constexpr int MOVER_PLACE = 1 << 9;     // is stored in the destination segment
constexpr int MOVER_AVG = 1 << 10;      // removed after its in-segment deposit: population averages only

struct FastBufs {
   double* RP;                 // row partials: 4 planes x nrows x nx x 4
   double* RPB;                // segment-boundary partials: 4 planes x nrows x nseg x 4
   unsigned long long* MMlo;   // 4 x N
   unsigned long long* MMhi;   // 4 x N
   unsigned char* touched;     // byte per cell: MM nonzero this step
   const unsigned char* segInner;   // per segment: an obstacle (RHGPU_FLAG_INNER_PARTICLE) cell within reach
   Mover* movers;
   unsigned long long* nmovers;
   long long moverCap;
   double scaleR, scaleJ;      // 2^kR, 2^kJ
};

// b in [-n, 2n)
__host__ __device__ inline int dualU(int b, int n, int per) { return per ? (b < 0 ? b + n : (b >= n ? b - n : b)) : b + 1; }
__host__ __device__ inline int dualB(int u, int per) { return per ? u : u - 1; }
__host__ __device__ inline int halfS(double x, double dx) { return (x < (0 + 0.5) * dx) ? 0 : 1; }

// exact 128-bit fixed-point accumulation of v * scale (rounded to an integer, |.| < 2^62)
__device__ inline void add128(unsigned long long* lo, unsigned long long* hi, double v, double scale) {
   const long long iv = __double2ll_rn(v * scale);
   const unsigned long long ulo = (unsigned long long)iv;
   const unsigned long long sext = iv < 0 ? ~0ull : 0ull;
   const unsigned long long old = atomicAdd(lo, ulo);
   const unsigned long long carry = (old + ulo < old) ? 1ull : 0ull;
   const unsigned long long h = sext + carry;
   if (h) atomicAdd(hi, h);
}

__device__ inline double fixedToDouble(unsigned long long lo, unsigned long long hi, double hiScale, double loScale) {
   return __ll2double_rn((long long)hi) * hiScale + __ull2double_rn(lo) * loScale;
}

// cicWeights (particle_accumulator.cpp:68-110) with the divisions by dx done by divDx
__device__ inline void cicWeightsDx(double x, double y, double z, double wq, const GridInfo& g, double w8[8]) {
   const double dx = g.dx;
   int i = (int)floor(divDx(x, g)), j = (int)floor(divDx(y, g)), k = (int)floor(divDx(z, g));
   if (x < (i + 0.5) * dx) { --i; }
   if (y < (j + 0.5) * dx) { --j; }
   if (z < (k + 0.5) * dx) { --k; }
   ++i; ++j; ++k;
   const double x0 = (i - 1 + 0.5) * dx, y0 = (j - 1 + 0.5) * dx, z0 = (k - 1 + 0.5) * dx;
   const double w_x = divDx(x - x0, g), w_y = divDx(y - y0, g), w_z = divDx(z - z0, g);
   w8[0] = (1 - w_x) * (1 - w_y) * (1 - w_z) * wq;
   w8[1] = w_x * (1 - w_y) * (1 - w_z) * wq;
   w8[2] = (1 - w_x) * w_y * (1 - w_z) * wq;
   w8[3] = w_x * w_y * (1 - w_z) * wq;
   w8[4] = (1 - w_x) * (1 - w_y) * w_z * wq;
   w8[5] = w_x * (1 - w_y) * w_z * wq;
   w8[6] = (1 - w_x) * w_y * w_z * wq;
   w8[7] = w_x * w_y * w_z * wq;
}

// cicWeightsDx for a cell-local position in [0, dx), as every particle has
// after its migration: there floor(x / dx) = 0 (x / dx rounds below 1), so the
// dual base of each axis is the half-cell shift alone and the weights are
// those of cicWeightsDx, bit for bit
__device__ inline void cicWeightsLocal(double x, double y, double z, double wq, const GridInfo& g, double w8[8]) {
   const double dx = g.dx;
   const int i = halfS(x, dx), j = halfS(y, dx), k = halfS(z, dx);
   const double x0 = (i - 1 + 0.5) * dx, y0 = (j - 1 + 0.5) * dx, z0 = (k - 1 + 0.5) * dx;
   const double w_x = divDx(x - x0, g), w_y = divDx(y - y0, g), w_z = divDx(z - z0, g);
   w8[0] = (1 - w_x) * (1 - w_y) * (1 - w_z) * wq;
   w8[1] = w_x * (1 - w_y) * (1 - w_z) * wq;
   w8[2] = (1 - w_x) * w_y * (1 - w_z) * wq;
   w8[3] = w_x * w_y * (1 - w_z) * wq;
   w8[4] = (1 - w_x) * (1 - w_y) * w_z * wq;
   w8[5] = w_x * (1 - w_y) * w_z * wq;
   w8[6] = (1 - w_x) * w_y * w_z * wq;
   w8[7] = w_x * w_y * w_z * wq;
}

// stayers of a chunk in the chunk positions [p0, p1), from the warps' stayer ballots
__device__ inline int stayersIn(const unsigned* bs, int p0, int p1) {
   int n = 0;
   for (int w = 0; w < FW; ++w) {
      const int lo = max(p0 - 32 * w, 0), hi = min(p1 - 32 * w, 32);
      if (lo >= hi) continue;
      const unsigned m = (hi == 32 ? ~0u : ((1u << hi) - 1u)) & (~0u << lo);
      n += __popc(bs[w] & m);
   }
   return n;
}

// the field stencil of one segment's cells in shared memory: local cell
// (lc, ly, lz) = global (xs0 + lc, ys0 + ly, zs0 + lz), lc in [0, SEG],
// ly, lz in {0, 1}; faceB also holds the -x / -y / -z neighbour faces
template <class T>
struct SegFieldsT {
   T bx[2][2][SEG + 2];    // [lz][ly][lc + 1]
   T by[2][3][SEG + 1];    // [lz][ly + 1][lc]
   T bz[3][2][SEG + 1];    // [lz + 1][ly][lc]
   T ue[3][2][2][SEG + 1]; // [l][lz][ly][lc]
   T ep[3][2][2][SEG + 1];
};
using SegFields = SegFieldsT<double>;
constexpr int SF_ROWS_B = 4 + 6 + 6;    // x-rows of faceB components in the stencil
constexpr int SF_ROWS_C = 12;           // x-rows of one cell vector field (3 components x 2 x 2)

// one x-row of the stencil: its shared-memory start, length, first global x,
// and the global array, component and (y, z)
template <class T>
__device__ inline T* stencilRow(SegFieldsT<T>& F, const Fields& f, int r, int& len, int& dxs, const double*& arr,
                                int& l, int& dy, int& dz) {
   if (r < 4) {   // faceB x: ly, lz in {0, 1}, lc from -1
      const int lz = r >> 1, ly = r & 1;
      len = SEG + 2; dxs = -1; arr = f.faceB; l = 0; dy = ly; dz = lz;
      return &F.bx[lz][ly][0];
   }
   if (r < 10) {  // faceB y: ly from -1
      const int q = r - 4, lz = q / 3, lyp = q - 3 * lz;
      len = SEG + 1; dxs = 0; arr = f.faceB; l = 1; dy = lyp - 1; dz = lz;
      return &F.by[lz][lyp][0];
   }
   if (r < 16) {  // faceB z: lz from -1
      const int q = r - 10, lzp = q >> 1, ly = q & 1;
      len = SEG + 1; dxs = 0; arr = f.faceB; l = 2; dy = ly; dz = lzp - 1;
      return &F.bz[lzp][ly][0];
   }
   const int q = (r - 16) % SF_ROWS_C, c = q >> 2, lz = (q >> 1) & 1, ly = q & 1;
   len = SEG + 1; dxs = 0; l = c; dy = ly; dz = lz;
   if (r < 16 + SF_ROWS_C) {
      arr = f.cellUe;
      return &F.ue[c][lz][ly][0];
   }
   arr = f.cellEp;
   return &F.ep[c][lz][ly][0];
}

// the stencil in two passes: threads 0..nrows-1 describe one x-row each
// (source row or none outside a non-periodic box in y/z, first global x,
// shared-memory offset), then all threads copy the rows' elements, SF_ROW_W
// slots per row (values 0 outside a non-periodic box; the push accelerates
// only particles of cells with all neighbours, so those are never read); all
// loads of a thread are issued before its shared-memory stores
constexpr int SF_ROW_W = SEG + 2;                               // slots per row (bx rows use all)
constexpr int SF_MAX_ROWS = SF_ROWS_B + 2 * SF_ROWS_C;
constexpr int SF_PER_THREAD = (SF_MAX_ROWS * SF_ROW_W + FT - 1) / FT;
struct StencilRow {
   const double* src;   // global x = 0 of the row, or nullptr (zeros)
   int dst;             // element offset of the row in the stencil
   int xs;              // global x of the row's first element
   int len;             // elements of the row
};

template <class T>
__device__ inline void stageSegRows(const GridInfo& g, const Fields& f, bool useEp, int xs0, int ys0, int zs0,
                                    SegFieldsT<T>& F, StencilRow* rows) {
   const int nrows = SF_ROWS_B + SF_ROWS_C * (useEp ? 2 : 1);
   const int tid = threadIdx.x;
   if (tid < nrows) {
      int len, dxs, l, dy, dz;
      const double* arr;
      T* dst = stencilRow(F, f, tid, len, dxs, arr, l, dy, dz);
      int y = ys0 + dy, z = zs0 + dz;
      if (g.per[1]) { if (y < 0) y += g.ny; else if (y >= g.ny) y -= g.ny; }
      if (g.per[2]) { if (z < 0) z += g.nz; else if (z >= g.nz) z -= g.nz; }
      StencilRow r;
      r.src = (y >= 0 && y < g.ny && z >= 0 && z < g.nz)
                  ? arr + (long long)l * g.N + (long long)g.nx * ((long long)y + (long long)g.ny * z)
                  : nullptr;
      r.dst = (int)(dst - (T*)&F);
      r.xs = xs0 + dxs;
      r.len = len;
      rows[tid] = r;
   }
   __syncthreads();
   double v[SF_PER_THREAD];
   int d[SF_PER_THREAD];
#pragma unroll
   for (int k = 0; k < SF_PER_THREAD; ++k) {
      const int e = tid + FT * k;
      const int ri = e / SF_ROW_W, c = e - ri * SF_ROW_W;
      v[k] = 0.0;
      d[k] = -1;
      if (ri >= nrows) continue;
      const StencilRow r = rows[ri];
      if (c >= r.len) continue;
      d[k] = r.dst + c;
      int x = r.xs + c;
      if (g.per[0]) { if (x < 0) x += g.nx; else if (x >= g.nx) x -= g.nx; }
      if (r.src && x >= 0 && x < g.nx) v[k] = r.src[x];
   }
   T* const base = (T*)&F;
#pragma unroll
   for (int k = 0; k < SF_PER_THREAD; ++k)
      if (d[k] >= 0) base[d[k]] = (T)v[k];
}

// pushOne with the fields from the segment's staged stencil and divDx; the
// same arithmetic in the same order
__device__ inline bool pushStaged(const GridInfo& g, const SegFields& F, const SpeciesDev& sp, const PushParams& pp,
                                  int i, int j, int k, int lc, int ly, int lz, double st[7]) {
   bool clamp = false;
   const bool accelerate = sp.accelerate && !pp.useIFT && allNb(g, i, j, k);
   double vx = st[3], vy = st[4], vz = st[5];
   if (accelerate) {
      const double dx = g.dx;
      double B[3], Ue[3], E[3];
      const double xs = divDx(st[0], g), ys = divDx(st[1], g), zs = divDx(st[2], g);
      B[0] = (xs - 0.0) * F.bx[lz][ly][lc + 1] + (1.0 - xs) * F.bx[lz][ly][lc];
      B[1] = (ys - 0.0) * F.by[lz][ly + 1][lc] + (1.0 - ys) * F.by[lz][ly][lc];
      B[2] = (zs - 0.0) * F.bz[lz + 1][ly][lc] + (1.0 - zs) * F.bz[lz][ly][lc];
      for (int l = 0; l < 3; ++l) Ue[l] = F.ue[l][lz][ly][lc];
      E[0] = B[1] * Ue[2] - B[2] * Ue[1];
      E[1] = B[2] * Ue[0] - B[0] * Ue[2];
      E[2] = B[0] * Ue[1] - B[1] * Ue[0];
      if (pp.use_ep) for (int l = 0; l < 3; ++l) E[l] += F.ep[l][lz][ly][lc];
      const double qm = sp.qmideltT2;
      const double dvx = qm * E[0], dvy = qm * E[1], dvz = qm * E[2];
      const double tx = qm * B[0], ty = qm * B[1], tz = qm * B[2];
      const double t2 = tx * tx + ty * ty + tz * tz;
      const double b2 = 2. / (1. + t2);
      const double sx = b2 * tx, sy = b2 * ty, sz = b2 * tz;
      const double vmx = vx + dvx, vmy = vy + dvy, vmz = vz + dvz;
      const double v0x = vmx + vmy * tz - vmz * ty;
      const double v0y = vmy + vmz * tx - vmx * tz;
      const double v0z = vmz + vmx * ty - vmy * tx;
      const double vpx = vmx + v0y * sz - v0z * sy;
      const double vpy = vmy + v0z * sx - v0x * sz;
      const double vpz = vmz + v0x * sy - v0y * sx;
      vx = vpx + dvx; vy = vpy + dvy; vz = vpz + dvz;
      if (pp.use_gravity) {
         const double xg = st[0] + blockOrigin(g.x_min, i, dx), yg = st[1] + blockOrigin(g.y_min, j, dx),
                      zg = st[2] + blockOrigin(g.z_min, k, dx);
         const double rr = sqrt(sq(xg) + sq(yg) + sq(zg));
         const double r3 = rr * rr * rr;
         if (r3 > 0) {
            const double s = -pp.GMdt / r3;
            vx += s * xg; vy += s * yg; vz += s * zg;
         }
      }
      const double v2 = sq(vx) + sq(vy) + sq(vz);
      if (v2 > pp.maxVi2) {
         const double norm = sqrt(pp.maxVi2 / v2);
         vx *= norm; vy *= norm; vz *= norm;
         clamp = true;
      }
   }
   st[3] = vx; st[4] = vy; st[5] = vz;
   st[0] += g.dt * vx;
   st[1] += g.dt * vy;
   st[2] += g.dt * vz;
   return clamp;
}

// push of one particle at local position st[0..2] in cell (i,j,k); returns true if clamped
__device__ inline bool pushOne(const GridInfo& g, const Fields& f, const SpeciesDev& sp, const PushParams& pp,
                               int i, int j, int k, double st[7]) {
   const long long N = g.N;
   const long long c = cidx(g, i, j, k);
   bool clamp = false;
   const bool accelerate = sp.accelerate && !pp.useIFT && allNb(g, i, j, k);
   double vx = st[3], vy = st[4], vz = st[5];
   if (accelerate) {
      const double dx = g.dx;
      double B[3], Ue[3], E[3];
      const double xs = st[0] / dx, ys = st[1] / dx, zs = st[2] / dx;
      B[0] = (xs - 0.0) * f.faceB[0 * N + c] + (1.0 - xs) * f.faceB[0 * N + nbr(g, i, j, k, -1, 0, 0)];
      B[1] = (ys - 0.0) * f.faceB[1 * N + c] + (1.0 - ys) * f.faceB[1 * N + nbr(g, i, j, k, 0, -1, 0)];
      B[2] = (zs - 0.0) * f.faceB[2 * N + c] + (1.0 - zs) * f.faceB[2 * N + nbr(g, i, j, k, 0, 0, -1)];
      for (int l = 0; l < 3; ++l) Ue[l] = f.cellUe[l * N + c];
      E[0] = B[1] * Ue[2] - B[2] * Ue[1];
      E[1] = B[2] * Ue[0] - B[0] * Ue[2];
      E[2] = B[0] * Ue[1] - B[1] * Ue[0];
      if (pp.use_ep) for (int l = 0; l < 3; ++l) E[l] += f.cellEp[l * N + c];
      const double qm = sp.qmideltT2;
      const double dvx = qm * E[0], dvy = qm * E[1], dvz = qm * E[2];
      const double tx = qm * B[0], ty = qm * B[1], tz = qm * B[2];
      const double t2 = tx * tx + ty * ty + tz * tz;
      const double b2 = 2. / (1. + t2);
      const double sx = b2 * tx, sy = b2 * ty, sz = b2 * tz;
      const double vmx = vx + dvx, vmy = vy + dvy, vmz = vz + dvz;
      const double v0x = vmx + vmy * tz - vmz * ty;
      const double v0y = vmy + vmz * tx - vmx * tz;
      const double v0z = vmz + vmx * ty - vmy * tx;
      const double vpx = vmx + v0y * sz - v0z * sy;
      const double vpy = vmy + v0z * sx - v0x * sz;
      const double vpz = vmz + v0x * sy - v0y * sx;
      vx = vpx + dvx; vy = vpy + dvy; vz = vpz + dvz;
      if (pp.use_gravity) {
         const double xg = st[0] + blockOrigin(g.x_min, i, dx), yg = st[1] + blockOrigin(g.y_min, j, dx),
                      zg = st[2] + blockOrigin(g.z_min, k, dx);
         const double rr = sqrt(sq(xg) + sq(yg) + sq(zg));
         const double r3 = rr * rr * rr;
         if (r3 > 0) {
            const double s = -pp.GMdt / r3;
            vx += s * xg; vy += s * yg; vz += s * zg;
         }
      }
      const double v2 = sq(vx) + sq(vy) + sq(vz);
      if (v2 > pp.maxVi2) {
         const double norm = sqrt(pp.maxVi2 / v2);
         vx *= norm; vy *= norm; vz *= norm;
         clamp = true;
      }
   }
   st[3] = vx; st[4] = vy; st[5] = vz;
   st[0] += g.dt * vx;
   st[1] += g.dt * vy;
   st[2] += g.dt * vz;
   return clamp;
}

// PER: the periodic axes (bit a = axis a), fixed at compile time; the host
// launches the instantiation that matches the grid
// the block's sums per (dual cell, corner) -> the segment's row partials (corner
// ox = 1 of each dual cell plus ox = 0 of the next) and, where the first dual
// cell's partner is in another segment, its boundary partial. s_rec is free.
__device__ __forceinline__ void segPartialsOut(const GridInfo& g, const FastGeom& fg, const FastBufs& fb, double* s_rec,
                                               long long row, int gseg, int u0, int u1, double a0, double a1,
                                               double a2, double a3) {
   const int tid = threadIdx.x, myDual = tid >> 3, myCorner = tid & 7;
   {
      double* q = s_rec + myDual * 32 + myCorner * 4;
      q[0] = a0; q[1] = a1; q[2] = a2; q[3] = a3;
   }
   __syncthreads();
   const int nx = g.nx;
   const long long nrows = fg.nrows;
   for (int e = tid; e < SEG * 16; e += FT) {
      const int dl = e >> 4, qq = (e >> 2) & 3, m = e & 3;
      const int lo = u0 + dl;   // the dual cell giving corner ox = 1 to cell x
      if (lo >= u1) continue;
      int x, hi;
      if (g.per[0]) {
         x = lo + 1 == nx ? 0 : lo + 1;
         hi = lo + 1 < u1 ? dl + 1 : (fg.nseg == 1 ? 0 : -1);
      } else {
         x = lo;
         if (x >= nx) continue;
         hi = lo + 1 < u1 ? dl + 1 : -1;
      }
      double v = s_rec[dl * 32 + ((1 + 2 * qq) << 2) + m];
      if (hi >= 0) v = v + s_rec[hi * 32 + ((2 * qq) << 2) + m];
      fb.RP[(((long long)qq * nrows + row) * nx + x) * 4 + m] = v;
   }
   // corner ox = 0 of the first dual cell, when the cell's other dual cell is in another segment
   if (tid < 16 && (g.per[0] ? fg.nseg > 1 : gseg >= 1)) {
      const int qq = tid >> 2, m = tid & 3;
      fb.RPB[(((long long)qq * nrows + row) * fg.nseg + gseg) * 4 + m] = s_rec[((2 * qq) << 2) + m];
   }
}

// one species' arrays offset to the block's segment: current x..w (0-6), next
// x..w (7-13), current lx (14), next lx (15)
constexpr int SEG_PTRS = 16;

// shared memory of k_fast_push_deposit (dynamic: more than the 48 KB static limit)
struct PushDepositShared {
   double rec[FT * REC];                  // deposit records of a chunk; at the end acc[SEG][32]
   double pf[7][FT];                      // the next chunk's particles, one plane per component
   SegFields f;                           // field stencil of the segment
   void* ptr[FAST_MAX_SPECIES][SEG_PTRS];
   StencilRow rows[SF_MAX_ROWS];
   alignas(8) unsigned char wd[SEG][FW];  // records per (dual cell, warp)
   int rank[FT];                          // stayers of the chunk before each chunk position
   int wcnt[FW];                          // stayers per warp
   int prefix[FAST_MAX_SPECIES + 1];      // first particle of each species in the segment
   int stay[FAST_MAX_SPECIES];            // stayers of each species so far
};
constexpr size_t PUSH_DEPOSIT_SMEM = sizeof(PushDepositShared);

// the segment's first chunk and the field stencil requested with cp.async: the
// stencil rows (see stageSegRows) with zeros outside a non-periodic box, the
// particles of chunk positions tid into pf
template <int PER>
__device__ __forceinline__ void pdStage(const GridInfo& g, const Fields& f, bool useEp, PushDepositShared& sh,
                                        int total, int ns, int& lxNext) {
   const int tid = threadIdx.x;
   if (tid < total) {
      int s = 0;
      while (s + 1 < ns && tid >= sh.prefix[s + 1]) ++s;
      const int p = tid - sh.prefix[s];
#pragma unroll
      for (int a = 0; a < 7; ++a) cpAsync8(&sh.pf[a][tid], (const double*)sh.ptr[s][a] + p, 8);
      lxNext = ((const unsigned char*)sh.ptr[s][14])[p];
   }
   const int nrows = SF_ROWS_B + SF_ROWS_C * (useEp ? 2 : 1);
   double* const base = (double*)&sh.f;
   for (int e = tid; e < nrows * SF_ROW_W; e += FT) {
      const int ri = e / SF_ROW_W, c = e - ri * SF_ROW_W;
      const StencilRow r = sh.rows[ri];
      if (c >= r.len) continue;
      int x = r.xs + c;
      if (PER & 1) { if (x < 0) x += g.nx; else if (x >= g.nx) x -= g.nx; }
      const bool ok = r.src != nullptr && x >= 0 && x < g.nx;
      cpAsync8(base + r.dst + c, ok ? r.src + x : f.faceB, ok ? 8 : 0);
   }
   cpAsyncCommit();
}

// cicWeightsLocal with the dual cell's lower centre (i - 1 + 0.5) dx = -dx/2 or
// +dx/2 selected (both exact), the same weights bit for bit
__device__ __forceinline__ void cicWeightsHalf(double x, double y, double z, double wq, const GridInfo& g, double hdx,
                                               double w8[8]) {
   const double x0 = x < hdx ? -hdx : hdx, y0 = y < hdx ? -hdx : hdx, z0 = z < hdx ? -hdx : hdx;
   const double w_x = divDx(x - x0, g), w_y = divDx(y - y0, g), w_z = divDx(z - z0, g);
   w8[0] = (1 - w_x) * (1 - w_y) * (1 - w_z) * wq;
   w8[1] = w_x * (1 - w_y) * (1 - w_z) * wq;
   w8[2] = (1 - w_x) * w_y * (1 - w_z) * wq;
   w8[3] = w_x * w_y * (1 - w_z) * wq;
   w8[4] = (1 - w_x) * (1 - w_y) * w_z * wq;
   w8[5] = w_x * (1 - w_y) * w_z * wq;
   w8[6] = (1 - w_x) * w_y * w_z * wq;
   w8[7] = w_x * w_y * w_z * wq;
}

// EXTRA: the variant with the optional outputs (the removed in-segment deposits
// listed for the population averages, the per-cell maxVi constraint counter);
// the default instantiation carries neither.
//
// One block per segment, one thread per particle, chunks of FT particles in
// storage order (species after species). The particles of chunk k+1 are copied
// to shared memory (cp.async, each thread its own position) while chunk k is
// processed; per chunk two barriers order the records and the stayers. A
// particle leaving the segment reserves its mover slot before the second
// barrier and is written after the deposit sums, so the reservation's round
// trip overlaps the chunk's remaining work.
template <int PER, bool EXTRA>
__global__ void __launch_bounds__(FT, 4)
k_fast_push_deposit(GridInfo gIn, Fields f, FastGeom fg, FastSpecies FS, PushParams pp, FastBufs fb,
                    double* cntd, unsigned long long* cntu, unsigned* err) {
   extern __shared__ __align__(16) unsigned char pdSmem[];
   PushDepositShared& sh = *reinterpret_cast<PushDepositShared*>(pdSmem);
   GridInfo g = gIn;
   g.per[0] = PER & 1;
   g.per[1] = (PER >> 1) & 1;
   g.per[2] = (PER >> 2) & 1;
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
   const unsigned below = (1u << lane) - 1u;
   const int S = (int)blockIdx.x;
   const int nseg = fg.nseg;
   const int row = S / nseg, gseg = S - row * nseg;
   const int uy = row % fg.nd[1], uz = row / fg.nd[1];
   const int u0 = gseg * SEG, u1 = min(u0 + SEG, fg.nd[0]);
   const int ns = FS.ns;
   const double dx = g.dx, hdx = 0.5 * dx;
   const int xs0 = dualB(u0, g.per[0]), ys0 = dualB(uy, g.per[1]), zs0 = dualB(uz, g.per[2]);
   // no obstacle cell within one step of the segment: the obstacle test is skipped
   const bool segInner = fb.segInner[S] != 0;

   // ---- set-up: species prefix (warp 0), segment pointers (warps 1-4), stencil rows (warps 5-6)
   if (warp == 0) {
      const int cnt = lane < ns ? FS.st[lane].cur.cnt[S] : 0;
      int x = cnt;
#pragma unroll
      for (int o = 1; o < 16; o <<= 1) {
         const int y = __shfl_up_sync(0xffffffffu, x, o);
         if (lane >= o) x += y;
      }
      if (lane <= ns) sh.prefix[lane] = x - cnt;
      if (lane < FAST_MAX_SPECIES) sh.stay[lane] = 0;
   } else if (tid < 32 + SEG_PTRS * ns) {
      const int q = tid - 32, s = q / SEG_PTRS, k = q - s * SEG_PTRS;
      const SegSpecies& SS = FS.st[s];
      const long long b = SS.base[S];
      void* v;
      if (k < 7) v = SS.cur.a[k] + b;
      else if (k < 14) v = SS.nxt.a[k - 7] + b;
      else if (k == 14) v = SS.cur.lx + b;
      else v = SS.nxt.lx + b;
      sh.ptr[s][k] = v;
   } else if (tid >= 160 && tid < 160 + SF_ROWS_B + SF_ROWS_C * (pp.use_ep ? 2 : 1)) {
      const int r = tid - 160;
      int len, dxs, l, dy, dz;
      const double* arr;
      double* dst = stencilRow(sh.f, f, r, len, dxs, arr, l, dy, dz);
      int y = ys0 + dy, z = zs0 + dz;
      if (PER & 2) { if (y < 0) y += g.ny; else if (y >= g.ny) y -= g.ny; }
      if (PER & 4) { if (z < 0) z += g.nz; else if (z >= g.nz) z -= g.nz; }
      StencilRow sr;
      sr.src = (y >= 0 && y < g.ny && z >= 0 && z < g.nz)
                   ? arr + (long long)l * g.N + (long long)g.nx * ((long long)y + (long long)g.ny * z)
                   : nullptr;
      sr.dst = (int)(dst - (double*)&sh.f);
      sr.xs = xs0 + dxs;
      sr.len = len;
      sh.rows[r] = sr;
   }
   __syncthreads();
   const int total = sh.prefix[ns];
   int lxNext = 0;
   pdStage<PER>(g, f, pp.use_ep, sh, total, ns, lxNext);
   cpAsyncWaitAll();
   __syncthreads();

   const int myDual = tid >> 3, myCorner = tid & 7;   // this thread's sums: (dual cell, corner) x 4 moments
   double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;

   for (int c0 = 0; c0 < total; c0 += FT) {
      const int i = c0 + tid;
      const bool active = i < total;
      int s = 0;
      if (active)
         while (s + 1 < ns && i >= sh.prefix[s + 1]) ++s;
      double st[7];
      bool stay = false, rec = false, leave = false, clamp = false;
      int mflags = 0;
      int vx = 0, vy = 0, vz = 0;
      int p = 0;
      const int lu = lxNext;
      if (c0 > 0) cpAsyncWaitAll();   // this thread's copies of the chunk
      if (active) {
         p = i - sh.prefix[s];
#pragma unroll
         for (int a = 0; a < 7; ++a) st[a] = sh.pf[a][tid];
         const int hx = halfS(st[0], dx), hy = halfS(st[1], dx), hz = halfS(st[2], dx);
         const int lc = lu + 1 - hx, ly = 1 - hy, lz = 1 - hz;
         int ci = xs0 + lu + 1 - hx;
         int cj = ys0 + ly;
         int ck = zs0 + lz;
         if (ci >= g.nx) ci -= g.nx;   // periodic axes: dual cell 0 holds the upper half of the last cell
         if (cj >= g.ny) cj -= g.ny;
         if (ck >= g.nz) ck -= g.nz;
         clamp = pushStaged(g, sh.f, FS.sp[s], pp, ci, cj, ck, lc, ly, lz, st);
         if (EXTRA) gridCountAtomic(f, GC_CELL_MAX_VI, g.N, cidx(g, ci, cj, ck), clamp);
         if (isnan(st[0]) || isnan(st[1]) || isnan(st[2])) raiseError(err, RHGPU_DEVERR_NAN_PARTICLE);
         int ox, oy, oz;
         int bad = migrateAxis(st[0], ox, dx, g.dx_below);
         bad |= migrateAxis(st[1], oy, dx, g.dx_below);
         bad |= migrateAxis(st[2], oz, dx, g.dx_below);
         int ti = ci + ox, tj = cj + oy, tk = ck + oz;
         const bool inside = wrapc(ti, g.nx, g.per[0]) && wrapc(tj, g.ny, g.per[1]) && wrapc(tk, g.nz, g.per[2]);
         if (bad || !inside) {
            const double ke = st[6] * (sq(st[3]) + sq(st[4]) + sq(st[5]));
            atomicAdd(&cntd[4 * s + 0], st[6]);
            atomicAdd(&cntd[4 * s + 1], ke);
         } else {
            vx = dualU(ti + halfS(st[0], dx) - 1, g.nx, g.per[0]);
            vy = dualU(tj + halfS(st[1], dx) - 1, g.ny, g.per[1]);
            vz = dualU(tk + halfS(st[2], dx) - 1, g.nz, g.per[2]);
            const bool inSeg = vy == uy && vz == uz && vx >= u0 && vx < u1;
            if (FS.sp[s].accumulate) {
               if (inSeg) {
                  rec = true;   // its CIC weights are formed just before the record is written
               } else {
                  mflags |= MOVER_DEPOSIT;   // deposited by k_fast_mover_deposit
               }
            }
            // boundary conditions of the step
            bool removed = false;
            if (!allNb(g, ti, tj, tk)) {
               removed = true;
               const double ke = st[6] * (sq(st[3]) + sq(st[4]) + sq(st[5]));
               atomicAdd(&cntd[4 * s + 0], st[6]);
               atomicAdd(&cntd[4 * s + 1], ke);
            } else {
               const unsigned cn = (unsigned)ti + (unsigned)g.nx * ((unsigned)tj + (unsigned)g.ny * (unsigned)tk);
               if (segInner && (f.flags[cn] & RHGPU_FLAG_INNER_PARTICLE)) {
                  const double xp = blockOrigin(g.x_min, ti, dx) + st[0];
                  const double yp = blockOrigin(g.y_min, tj, dx) + st[1];
                  const double zp = blockOrigin(g.z_min, tk, dx) + st[2];
                  if (sq(xp) + sq(yp) + sq(zp) < FS.sp[s].R2obs) {
                     removed = true;
                     const double ke = st[6] * (sq(st[3]) + sq(st[4]) + sq(st[5]));
                     atomicAdd(&cntd[4 * s + 2], st[6]);
                     atomicAdd(&cntd[4 * s + 3], ke);
                  }
               }
            }
            if (!removed) {
               stay = inSeg;
               if (!inSeg) mflags |= MOVER_PLACE;
            } else if (EXTRA && rec && pp.avgList) {
               mflags |= MOVER_AVG;   // population averages: its in-segment deposit is listed
            }
            leave = mflags != 0;
         }
      }
      if (clamp) atomicAdd(&cntu[CNT_SPECIES_MAXVI + s], 1ull);

      // ---- order of the chunk's stayers and records --------------------------------------
      // warp-local first: stayer/record ballots and the records per (warp, dual cell)
      const unsigned bs = __ballot_sync(0xffffffffu, stay), br = __ballot_sync(0xffffffffu, rec);
      if (lane == 0) sh.wcnt[warp] = __popc(bs);
      sh.wd[lane][warp] = 0;
      __syncwarp();
      const int rd = rec ? vx - u0 : 0;
      int rrank = 0;
      if (rec) {
         const unsigned mm = __match_any_sync(br, rd);
         rrank = __popc(mm & below);
         if (rrank == 0) sh.wd[rd][warp] = (unsigned char)__popc(mm);
      }
      __syncthreads();
      // every shared-memory read of this chunk's particles is done: request the next chunk's
      {
         const int i2 = i + FT;
         if (i2 < total) {
            int s2 = s;
            while (s2 + 1 < ns && i2 >= sh.prefix[s2 + 1]) ++s2;
            const int p2 = i2 - sh.prefix[s2];
#pragma unroll
            for (int a = 0; a < 7; ++a) cpAsync8(&sh.pf[a][tid], (const double*)sh.ptr[s2][a] + p2, 8);
            lxNext = ((const unsigned char*)sh.ptr[s2][14])[p2];
         }
         cpAsyncCommit();
      }
      // every warp, per dual cell (lane): the first sorted record of the dual cell
      // (bin) and of this warp's records for it (off)
      int binD, offD, nrec;
      {
         // the eight per-warp counts of dual cell `lane` are bytes (each at most 32):
         // byte sums by one multiply per 32-bit half
         const uint2 c8 = *reinterpret_cast<const uint2*>(&sh.wd[lane][0]);
         const int t = (int)(((c8.x * 0x01010101u) >> 24) + ((c8.y * 0x01010101u) >> 24));
         const unsigned mlo = warp >= 4 ? 0xffffffffu : (1u << (8 * warp)) - 1u;
         const unsigned mhi = warp <= 4 ? 0u : (1u << (8 * (warp - 4))) - 1u;
         const int before = (int)((((c8.x & mlo) * 0x01010101u) >> 24) + (((c8.y & mhi) * 0x01010101u) >> 24));
         int x = t;
         for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
         }
         binD = x - t;
         offD = binD + before;
         nrec = __shfl_sync(0xffffffffu, x, 31);
      }
      const int recPos = __shfl_sync(0xffffffffu, offD, rd) + rrank;
      const int sumLo = __shfl_sync(0xffffffffu, binD, myDual);
      const int sumHiN = __shfl_sync(0xffffffffu, binD, (myDual + 1) & 31);
      const int sumHi = myDual == SEG - 1 ? nrec : sumHiN;
      // stayers of the chunk before this position (and in all), and this species' count so far
      const int wc = lane < FW ? sh.wcnt[lane] : 0;
      const int myRank = (int)__reduce_add_sync(0xffffffffu, (unsigned)(lane < warp ? wc : 0)) + __popc(bs & below);
      const int chunkStay = (int)__reduce_add_sync(0xffffffffu, (unsigned)wc);
      sh.rank[tid] = myRank;
      const int stayBase = stay ? sh.stay[s] : 0;
      // mover slots reserved now, written after the sums
      const unsigned lm = __ballot_sync(0xffffffffu, leave);
      const int leader = lm ? __ffs(lm) - 1 : 0;
      unsigned long long mb = 0;
      if (lm && lane == leader) mb = atomicAdd(fb.nmovers, (unsigned long long)__popc(lm));
      if (rec) {
         double w8[8];
         cicWeightsHalf(st[0], st[1], st[2], st[6] * FS.sp[s].q, g, hdx, w8);
         double* r = sh.rec + recPos * REC;
#pragma unroll
         for (int o = 0; o < 8; ++o) r[o] = w8[o];
         r[8] = st[3]; r[9] = st[4]; r[10] = st[5];
      }
      __syncthreads();
      if (stay) {
         const int p0 = sh.prefix[s] - c0;   // chunk position of the species' first particle
         const int q = stayBase + myRank - (p0 > 0 ? sh.rank[p0] : 0);
         double* const* nx = (double* const*)&sh.ptr[s][7];
#pragma unroll
         for (int a = 0; a < 7; ++a) nx[a][q] = st[a];
         ((unsigned char*)sh.ptr[s][15])[q] = (unsigned char)(vx - u0);
      }
      // running stayer count of each species
      if (tid < ns) {
         const int lo = min(max(sh.prefix[tid] - c0, 0), FT), hi = min(max(sh.prefix[tid + 1] - c0, 0), FT);
         const int rlo = lo < FT ? sh.rank[lo] : chunkStay, rhi = hi < FT ? sh.rank[hi] : chunkStay;
         sh.stay[tid] += rhi - rlo;
      }
      // ---- sums of this thread's (dual cell, corner), records in list order ----------------
#pragma unroll 2
      for (int r = sumLo; r < sumHi; ++r) {
         const double* rr = sh.rec + r * REC;
         const double w = rr[myCorner];
         a0 += w;
         a1 += w * rr[8];
         a2 += w * rr[9];
         a3 += w * rr[10];
      }
      // ---- particles that left the segment -----------------------------------------------
      if (lm) {
         mb = __shfl_sync(0xffffffffu, mb, leader);
         if (leave) {
            const unsigned long long m = mb + __popc(lm & below);
            if ((long long)m < fb.moverCap) {
               Mover& M = fb.movers[m];
#pragma unroll
               for (int a = 0; a < 7; ++a) M.s[a] = st[a];
               M.key = ((unsigned long long)S << 32) | (unsigned long long)p;
               const int gd = vx / SEG;
               M.dest = ((long long)vy + (long long)fg.nd[1] * vz) * nseg + gd;
               M.species = s;
               M.lx = (vx - gd * SEG) | mflags;
            } else {
               raiseError(err, RHGPU_DEVERR_CAPACITY);
            }
         }
      }
      // no barrier here: the next chunk's first barrier orders the reads of rec,
      // rank and stay before their next writes
   }

   // ---- outputs: stayer counts, row partials, segment-boundary partial ---------------------
   __syncthreads();
   if (tid < ns) FS.st[tid].nxt.cnt[S] = sh.stay[tid];
   segPartialsOut(g, fg, fb, sh.rec, row, gseg, u0, u1, a0, a1, a2, a3);
}

// CIC contributions of the particles that left their segment, as exact fixed-point sums (MM)
// one mover's CIC contributions as exact fixed-point sums into lo/hi (4 x N),
// marking the touched cells (TOUCH)
template <bool TOUCH>
__device__ __forceinline__ void moverAdd128(const GridInfo& g, const FastGeom& fg, const FastSpecies& FS, const Mover& M,
                                            unsigned long long* lo, unsigned long long* hi, double scaleR, double scaleJ,
                                            unsigned char* touched) {
   const int s = M.species;
   const long long row = M.dest / fg.nseg;
   const int vx = (int)(M.dest % fg.nseg) * SEG + (M.lx & 0xff);
   const int vy = (int)(row % fg.nd[1]), vz = (int)(row / fg.nd[1]);
   const int bx = dualB(vx, g.per[0]), by = dualB(vy, g.per[1]), bz = dualB(vz, g.per[2]);
   double st[7];
   for (int a = 0; a < 7; ++a) st[a] = M.s[a];
   double w8[8];
   cicWeightsLocal(st[0], st[1], st[2], st[6] * FS.sp[s].q, g, w8);
   const long long N = g.N;
   for (int o = 0; o < 8; ++o) {
      int dxc = bx + (o & 1), dyc = by + ((o >> 1) & 1), dzc = bz + ((o >> 2) & 1);
      if (!wrapc(dxc, g.nx, g.per[0]) || !wrapc(dyc, g.ny, g.per[1]) || !wrapc(dzc, g.nz, g.per[2])) continue;
      const long long dc = cidx(g, dxc, dyc, dzc);
      add128(&lo[dc], &hi[dc], w8[o], scaleR);
      for (int l = 0; l < 3; ++l) add128(&lo[(1 + l) * N + dc], &hi[(1 + l) * N + dc], w8[o] * st[3 + l], scaleJ);
      if (TOUCH) touched[dc] = 1;   // a plain byte store: every writer stores the same value
   }
}

__global__ void k_fast_mover_deposit(GridInfo g, FastGeom fg, FastSpecies FS, FastBufs fb, long long n);

// the segment-boundary partials folded into the row partials of their cells
// (RP += RPB, the addition the gather would make): the gather then reads four
// row partials per cell and nothing else
__global__ void k_fast_fold_boundary(GridInfo g, FastGeom fg, FastBufs fb);

// destination moments: four row partials (boundary partials folded in) +
// fixed-point part, then finalize. The touched mark, the four row partials
// (16-byte loads) and the fixed-point sums are all requested before any sum:
// most cells are touched by some mover, and waiting for the touched mark
// before loading the sums would add a second dependent round trip.
template <bool GC>   // GC: also count the rho clamp per cell (grid counters on)
__global__ void k_fast_gather(GridInfo g, Fields f, FastGeom fg, FastBufs fb, double hiR, double loR, double hiJ,
                              double loJ, double minRho, unsigned long long* cnt) {
   RH_CELL_PROLOGUE
   const unsigned tw = fb.touched[n];
   double2 rp[4][2];
#pragma unroll
   for (int qq = 0; qq < 4; ++qq) {
      const int uyy = dualU(j - (qq & 1), g.ny, g.per[1]);
      const int uzz = dualU(k - (qq >> 1), g.nz, g.per[2]);
      const long long row = (long long)uyy + (long long)fg.nd[1] * uzz;
      const double2* p2 = reinterpret_cast<const double2*>(fb.RP + (((long long)qq * fg.nrows + row) * g.nx + i) * 4);
      rp[qq][0] = p2[0];
      rp[qq][1] = p2[1];
   }
   double v[4] = {rp[0][0].x, rp[0][0].y, rp[0][1].x, rp[0][1].y};
#pragma unroll
   for (int qq = 1; qq < 4; ++qq) {
      v[0] = v[0] + rp[qq][0].x;
      v[1] = v[1] + rp[qq][0].y;
      v[2] = v[2] + rp[qq][1].x;
      v[3] = v[3] + rp[qq][1].y;
   }
   unsigned long long mlo[4], mhi[4];
#pragma unroll
   for (int l = 0; l < 4; ++l) {
      mlo[l] = fb.MMlo[l * N + n];
      mhi[l] = fb.MMhi[l * N + n];
   }
   if (tw) {
      v[0] += fixedToDouble(mlo[0], mhi[0], hiR, loR);
      for (int l = 0; l < 3; ++l) v[1 + l] += fixedToDouble(mlo[1 + l], mhi[1 + l], hiJ, loJ);
   }
   // every cell's sums cleared for the next step, touched or not: whole sectors
   // written (a warp writing only its touched cells leaves partly written
   // sectors, which cost a read-modify-write each; 0.48 -> 0.17 ms per step)
   for (int l = 0; l < 4; ++l) { fb.MMlo[l * N + n] = 0ull; fb.MMhi[l * N + n] = 0ull; }
   double rho = v[0] / g.dV;
   bool clamp = false;
   if (rho < minRho) { rho = minRho; clamp = true; }
   countIf(clamp, &cnt[CNT_MIN_CELL_RHO]);
   if (GC) gridCount(f, GC_CELL_MIN_RHOQI, N, n, clamp);
   f.cellRho[n] = rho;
   for (int l = 0; l < 3; ++l) f.cellJi[l * N + n] = v[1 + l] / g.dV;
}

// ---- mover placement ------------------------------------------------------------------------
template <class MV>
__global__ void k_fast_mig_count(const MV* mv, long long n, long long NS, int* inc) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= n || !(mv[t].lx & MOVER_PLACE)) return;
   atomicAdd(&inc[(long long)mv[t].species * NS + mv[t].dest], 1);
}
// Placement order of the arrivals of a destination (species, segment) bucket:
// by mover key (source segment, index in it). The movers are sorted by key and
// then, stably, by bucket (radix sorts on the host side); these kernels prepare
// the sort keys, check the room of every bucket, place the movers (one thread
// each) after the bucket's stayers, and add the arrivals to the counts.
template <class MV>
__global__ void k_mig_sort_keys(const MV* mv, long long n, long long NS, long long nb, unsigned long long* key,
                                unsigned* val, unsigned* bkt) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= n) return;
   key[t] = mv[t].key;
   val[t] = (unsigned)t;
   bkt[t] = (mv[t].lx & MOVER_PLACE) ? (unsigned)((long long)mv[t].species * NS + mv[t].dest) : (unsigned)nb;
}
template <class SET>
__global__ void k_mig_check(SET FS, long long NS, const int* inc, int* overflow) {
   const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (b >= (long long)FS.ns * NS || inc[b] == 0) return;
   const int s = (int)(b / NS);
   const long long S = b % NS;
   // one bit per species whose arrivals do not fit (relaid alone)
   if (FS.st[s].base[S] + FS.st[s].nxt.cnt[S] + inc[b] > FS.st[s].base[S + 1]) atomicOr((unsigned*)overflow, 1u << s);
}
template <class SET>
__global__ void k_mig_counts(SET FS, long long NS, int* inc) {
   const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (b >= (long long)FS.ns * NS || inc[b] == 0) return;
   FS.st[(int)(b / NS)].nxt.cnt[b % NS] += inc[b];
   inc[b] = 0;
}
// small buckets: the arrivals of each bucket listed (in any order) at off[b] by
// k_mig_bucket, then one thread per bucket orders them by key (insertion sort)
// into order[], the same order as the sorts
template <class MV>
__global__ void k_mig_bucket(const MV* mv, long long n, long long NS, const long long* off, int* fill,
                             unsigned* list) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= n || !(mv[t].lx & MOVER_PLACE)) return;
   const long long b = (long long)mv[t].species * NS + mv[t].dest;
   const int k = atomicAdd(&fill[b], 1);
   list[off[b] + k] = (unsigned)t;
}
constexpr int MIG_SMALL = 64;     // arrivals a bucket's own thread orders
constexpr int MIG_LARGE = 2048;   // arrivals one block orders in shared memory (k_mig_order_large)
template <class MV>
__global__ void k_mig_order_small(const MV* mv, long long nb, const int* inc, const long long* off, unsigned* list,
                                  unsigned* bkt) {
   const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (b >= nb) return;
   const int k = inc[b];
   if (k > MIG_SMALL) return;   // k_mig_order_large
   unsigned* bk = list + off[b];
   for (int a = 1; a < k; ++a) {
      const unsigned t = bk[a];
      const unsigned long long key = mv[t].key;
      int c = a;
      for (; c > 0 && mv[bk[c - 1]].key > key; --c) bk[c] = bk[c - 1];
      bk[c] = t;
   }
   for (int a = 0; a < k; ++a) bkt[off[b] + a] = (unsigned)b;
}

// the buckets with more than MIG_SMALL arrivals, appended to large[] (count in *nlarge)
__global__ void k_mig_large_list(const int* inc, long long nb, unsigned* large, int* nlarge);

// each bucket of large[] (at most MIG_LARGE arrivals) ordered by one block: its
// arrivals' (key, mover index) sorted bitonically in shared memory, the order
// the radix sorts give (by key; equal keys by mover index)
constexpr int MIG_LARGE_THREADS = 256;
template <class MV>
__global__ void __launch_bounds__(MIG_LARGE_THREADS) k_mig_order_large(const MV* mv, const int* inc, const long long* off,
                                                                        unsigned* list, unsigned* bkt,
                                                                        const unsigned* large, const int* nlarge) {
   __shared__ unsigned long long skey[MIG_LARGE];
   __shared__ unsigned sval[MIG_LARGE];
   const int n = *nlarge;
   for (int q = blockIdx.x; q < n; q += gridDim.x) {
      const unsigned b = large[q];
      const int k = inc[b];
      unsigned* bk = list + off[b];
      int m = 1;
      while (m < k) m <<= 1;
      for (int i = threadIdx.x; i < m; i += MIG_LARGE_THREADS) {
         if (i < k) {
            skey[i] = mv[bk[i]].key;
            sval[i] = bk[i];
         } else {
            skey[i] = ~0ull;
            sval[i] = ~0u;
         }
      }
      __syncthreads();
      for (int size = 2; size <= m; size <<= 1) {
         for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < m; i += MIG_LARGE_THREADS) {
               const int j = i ^ stride;
               if (j > i) {
                  const bool up = (i & size) == 0;
                  const unsigned long long ki = skey[i], kj = skey[j];
                  const unsigned vi = sval[i], vj = sval[j];
                  const bool gt = ki > kj || (ki == kj && vi > vj);
                  if (gt == up) {
                     skey[i] = kj; skey[j] = ki;
                     sval[i] = vj; sval[j] = vi;
                  }
               }
            }
            __syncthreads();
         }
      }
      for (int i = threadIdx.x; i < k; i += MIG_LARGE_THREADS) {
         bk[i] = sval[i];
         bkt[off[b] + i] = b;
      }
      __syncthreads();
   }
}

// mover order[q] to slot q - off[bucket] after its bucket's stayers (bucket nb: not placed)
__global__ void k_fast_mig_place(FastSpecies FS, long long NS, long long nb, const Mover* mv, const unsigned* order,
                                 const unsigned* bkt, const long long* off, long long n);

// ---- upload / download / relayout support -----------------------------------------------------
// segment and dual x (in the segment) of each uploaded particle (records grouped by cell)
__global__ void k_fast_seg_of(GridInfo g, FastGeom fg, const double* aos, const int* pcell, long long n,
                              unsigned* key, unsigned char* lx);
// for keys sorted ascending: first[k] = first position with key >= k, k in [0, nkeys]
// (every k written exactly once, no atomics)
__global__ void k_sorted_bounds(const unsigned* key, long long n, long long nkeys, long long* first);
// counts from the bounds
__global__ void k_bounds_counts(const long long* first, long long nkeys, int* cnt);
// segment capacity with slack: c + max(32, c/4); entry NS is 0 (for the scan's total)
__global__ void k_fast_capacity(long long NS, const int* cnt, const int* extra, long long* cap);
// sorted upload records -> segment slots
__global__ void k_fast_scatter_sorted(const double* aos, const unsigned char* lxIn, const unsigned* key,
                                      const unsigned* idx, long long n, const long long* first, SegBuf B,
                                      const long long* base);
// one block per segment: cell key and slot of every particle, in storage order
__global__ void k_fast_cell_keys(GridInfo g, FastGeom fg, SegBuf B, const long long* base, const long long* first,
                                 unsigned* key, unsigned long long* slots);
__global__ void k_fast_gather_records(SegBuf B, const unsigned long long* slots, const unsigned* idx, long long n,
                                      double* aos);
// one block per segment: copy the particles of a segment to another layout
__global__ void k_fast_relayout(SegBuf from, const long long* fromBase, SegBuf to, const long long* toBase);
// one block per segment: largest |weight|
// (non-negative doubles order like their bit patterns; one atomic per block)
__global__ void k_fast_max_abs_w(SegBuf B, const long long* base, unsigned long long* out);

}  // namespace rh
