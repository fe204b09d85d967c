// FP32 precision form (sm_100a): particles stored as an int32 cell index, FP32
// offsets in the cell (cell units, [0,1)) and FP32 velocities (28 B per
// particle, one macroparticle weight per species), pushed and deposited in FP32
// with FP32 accumulation. The grid fields stay FP64 in HBM; a segment's field
// stencil is staged as FP32 in shared memory, and the moments are handed to the
// FP64 field update after the gather.
//
// The structure is the fast path's (k_fast.cuh): row segments of
// RHGPU_FAST_SEGMENT CIC dual cells, one block per segment and one thread per
// particle, stayers kept in order, deposit records counting-sorted by target
// dual cell and summed per (dual cell, corner) x 4 moments, particles leaving
// their segment deposited as exact fixed-point sums and placed afterwards.
// The arithmetic follows the reference's push (boris.h:64-194) and CIC weights
// (particle_accumulator.cpp:68-110) rewritten in cell units:
//   B = xs B(c) + (1 - xs) B(c - 1) with xs the offset (face2r);
//   w_x = off + 0.5 - s, s = (off >= 0.5) (accumulateCell's x0 shift);
//   drift off += v dt/dx; migration by exactly one cell.
// Deposit weights are geometric weights times w q / (w q of species 0), so the
// FP32 sums stay O(ppc); the gather scales by (w q)_0 / dV in FP64.
#pragma once

#include "rh_device.cuh"
#include "k_fields.cuh"
#include "k_particles.cuh"
#include "k_fast.cuh"
#include "k_diag.cuh"

namespace rh {

struct F32Buf {
   int* cell;        // cell index
   float* o[3];      // offsets in the cell, cell units
   float* v[3];      // velocity [m/s]
   int* cnt;         // particles per segment
};
struct F32Species {
   F32Buf cur, nxt;
   const long long* base;
};
struct F32Set {
   int ns;
   F32Species st[FAST_MAX_SPECIES];
   int accumulate[FAST_MAX_SPECIES];
   int accelerate[FAST_MAX_SPECIES];
   float qm[FAST_MAX_SPECIES];       // q dt / (2 m)
   float wqRel[FAST_MAX_SPECIES];    // (w q)_s / (w q)_0
   float R2obs[FAST_MAX_SPECIES];
   double w[FAST_MAX_SPECIES];       // macroparticle weight
};
struct F32Params {
   float dtdx;        // dt / dx
   float dt;
   float dx;
   float below1;      // largest float below 1
   float maxVi2;
   float GMdt;
   int useIFT, use_ep, use_gravity;
};

// a particle leaving its segment (FP32 form)
struct Mover32 {
   float o[3], v[3];
   int cell;
   int species;
   unsigned long long key;   // (source segment << 32) | index in the source segment
   long long dest;           // destination segment
   int lx;                   // dual x in the destination segment | MOVER_* flags
   int pad;
};

struct F32Bufs {
   float* RP;                  // 4 planes x nrows x nx x 4
   float* RPB;                 // 4 planes x nrows x nseg x 4
   unsigned long long* MMlo;   // 4 x N (shared with the FP64 fast path)
   unsigned long long* MMhi;
   unsigned* touched;
   Mover32* movers;
   unsigned long long* nmovers;
   long long moverCap;
   double scaleR, scaleJ;
};

__device__ inline int halfSf(float o) { return o < 0.5f ? 0 : 1; }

// the segment's field stencil as FP32 (staged by stageSegRows<float>)
using SegFields32 = SegFieldsT<float>;

// Boris-Buneman push in FP32 (boris.h:64-194 in cell units); o: offsets, v: velocity
__device__ inline bool pushF32(const GridInfo& g, const SegFields32& F, const F32Set& FS, int s, const F32Params& pp,
                               int i, int j, int k, int lc, int ly, int lz, float o[3], float v[3]) {
   bool clamp = false;
   const bool accelerate = FS.accelerate[s] && !pp.useIFT && allNb(g, i, j, k);
   float vx = v[0], vy = v[1], vz = v[2];
   if (accelerate) {
      float B[3], Ue[3], E[3];
      const float xs = o[0], ys = o[1], zs = o[2];
      B[0] = xs * F.bx[lz][ly][lc + 1] + (1.0f - xs) * F.bx[lz][ly][lc];
      B[1] = ys * F.by[lz][ly + 1][lc] + (1.0f - ys) * F.by[lz][ly][lc];
      B[2] = zs * F.bz[lz + 1][ly][lc] + (1.0f - zs) * F.bz[lz][ly][lc];
      for (int l = 0; l < 3; ++l) Ue[l] = F.ue[l][lz][ly][lc];
      E[0] = B[1] * Ue[2] - B[2] * Ue[1];
      E[1] = B[2] * Ue[0] - B[0] * Ue[2];
      E[2] = B[0] * Ue[1] - B[1] * Ue[0];
      if (pp.use_ep) for (int l = 0; l < 3; ++l) E[l] += F.ep[l][lz][ly][lc];
      const float qm = FS.qm[s];
      const float dvx = qm * E[0], dvy = qm * E[1], dvz = qm * E[2];
      const float tx = qm * B[0], ty = qm * B[1], tz = qm * B[2];
      const float t2 = tx * tx + ty * ty + tz * tz;
      const float b2 = 2.0f / (1.0f + t2);
      const float sx = b2 * tx, sy = b2 * ty, sz = b2 * tz;
      const float vmx = vx + dvx, vmy = vy + dvy, vmz = vz + dvz;
      const float v0x = vmx + vmy * tz - vmz * ty;
      const float v0y = vmy + vmz * tx - vmx * tz;
      const float v0z = vmz + vmx * ty - vmy * tx;
      const float vpx = vmx + v0y * sz - v0z * sy;
      const float vpy = vmy + v0z * sx - v0x * sz;
      const float vpz = vmz + v0x * sy - v0y * sx;
      vx = vpx + dvx; vy = vpy + dvy; vz = vpz + dvz;
      if (pp.use_gravity) {
         const float xg = (float)blockOrigin(g.x_min, i, g.dx) + o[0] * pp.dx;
         const float yg = (float)blockOrigin(g.y_min, j, g.dx) + o[1] * pp.dx;
         const float zg = (float)blockOrigin(g.z_min, k, g.dx) + o[2] * pp.dx;
         const float rr = sqrtf(xg * xg + yg * yg + zg * zg);
         const float r3 = rr * rr * rr;
         if (r3 > 0.0f) {
            const float sg = -pp.GMdt / r3;
            vx += sg * xg; vy += sg * yg; vz += sg * zg;
         }
      }
      const float v2 = vx * vx + vy * vy + vz * vz;
      if (v2 > pp.maxVi2) {
         const float norm = sqrtf(pp.maxVi2 / v2);
         vx *= norm; vy *= norm; vz *= norm;
         clamp = true;
      }
   }
   v[0] = vx; v[1] = vy; v[2] = vz;
   o[0] += pp.dtdx * vx;
   o[1] += pp.dtdx * vy;
   o[2] += pp.dtdx * vz;
   return clamp;
}

// migration of one offset by exactly one cell; nonzero if it moved further
__device__ inline int migrateAxisF(float& o, int& off, float below1) {
   int st = 0;
   off = 0;
   if (o < 0.0f) {
      o += 1.0f;
      off = -1;
      if (o >= 1.0f) o = below1;
      if (o < 0.0f) st = 1;
   } else if (o >= 1.0f) {
      o -= 1.0f;
      off = 1;
      if (o >= 1.0f) st = 1;
   }
   return st;
}

// CIC weights in cell units (accumulateCell's weights), times wq
__device__ inline void cicWeightsF(const float o[3], float wq, float w8[8]) {
   const float wx = o[0] + 0.5f - (float)halfSf(o[0]);
   const float wy = o[1] + 0.5f - (float)halfSf(o[1]);
   const float wz = o[2] + 0.5f - (float)halfSf(o[2]);
   w8[0] = (1.0f - wx) * (1.0f - wy) * (1.0f - wz) * wq;
   w8[1] = wx * (1.0f - wy) * (1.0f - wz) * wq;
   w8[2] = (1.0f - wx) * wy * (1.0f - wz) * wq;
   w8[3] = wx * wy * (1.0f - wz) * wq;
   w8[4] = (1.0f - wx) * (1.0f - wy) * wz * wq;
   w8[5] = wx * (1.0f - wy) * wz * wq;
   w8[6] = (1.0f - wx) * wy * wz * wq;
   w8[7] = wx * wy * wz * wq;
}

constexpr int REC32 = 11;   // floats per deposit record: w8[8], v[3]

// PER: the periodic axes (bit a = axis a), fixed at compile time; the host
// launches the instantiation that matches the grid
// GC: the variant that also counts the per-cell maxVi constraint (grid counters on)
template <int PER, bool GC>
__global__ void __launch_bounds__(FT, 4)
k_f32_push_deposit(GridInfo gIn, Fields f, FastGeom fg, F32Set FS, F32Params pp, F32Bufs fb, double* cntd,
                   unsigned long long* cntu, unsigned* err) {
   GridInfo g = gIn;
   g.per[0] = PER & 1;
   g.per[1] = (PER >> 1) & 1;
   g.per[2] = (PER >> 2) & 1;
   __shared__ float s_rec[FT * REC32];            // deposit records of a chunk; at the end acc[SEG][32]
   __shared__ int s_wd[FW][SEG];                  // records per (warp, dual cell), then their first sorted slot
   __shared__ int s_bin[SEG + 1];                 // first sorted record of each dual cell
   __shared__ int s_wcnt[FW];                     // stayers per warp, then the stayers of the warps before
   __shared__ unsigned s_bs[FW];
   __shared__ int s_prefix[FAST_MAX_SPECIES + 1];
   __shared__ int s_stay[FAST_MAX_SPECIES];
   __shared__ SegFields32 s_f;
   __shared__ StencilRow s_rows[SF_MAX_ROWS];
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
   const unsigned below = (1u << lane) - 1u;
   const long long S = blockIdx.x;
   const long long row = S / fg.nseg;
   const int gseg = (int)(S % fg.nseg);
   const int uy = (int)(row % fg.nd[1]), uz = (int)(row / fg.nd[1]);
   const int ndx = fg.nd[0];
   const int u0 = gseg * SEG, u1 = min(u0 + SEG, ndx);
   const int ns = FS.ns;
   if (tid == 0) {
      int a = 0;
      for (int s = 0; s < ns; ++s) {
         s_prefix[s] = a;
         a += FS.st[s].cur.cnt[S];
      }
      s_prefix[ns] = a;
   }
   if (tid < FAST_MAX_SPECIES) s_stay[tid] = 0;
   const int by0 = dualB(uy, g.per[1]), bz0 = dualB(uz, g.per[2]);
   stageSegRows(g, f, pp.use_ep, dualB(u0, g.per[0]), by0, bz0, s_f, s_rows);
   __syncthreads();
   const int total = s_prefix[ns];
   const int myDual = tid >> 3, myCorner = tid & 7;
   float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;

   for (int c0 = 0; c0 < total; c0 += FT) {
      const int i = c0 + tid;
      const bool active = i < total;
      int s = 0;
      if (active)
         while (s + 1 < ns && i >= s_prefix[s + 1]) ++s;
      float o[3], v[3];
      int cell = 0;
      long long p = 0;
      bool stay = false, rec = false, leave = false, clamp = false;
      int mflags = 0, vx = 0, vy = 0, vz = 0, ti = 0, tj = 0, tk = 0;
      if (active) {
         const F32Species& SS = FS.st[s];
         p = i - s_prefix[s];
         const long long slot = SS.base[S] + p;
         cell = SS.cur.cell[slot];
         for (int a = 0; a < 3; ++a) { o[a] = SS.cur.o[a][slot]; v[a] = SS.cur.v[a][slot]; }
         const int sx = halfSf(o[0]), sy = halfSf(o[1]), sz = halfSf(o[2]);
         int cj = by0 + 1 - sy, ck = bz0 + 1 - sz;
         if (cj >= g.ny) cj -= g.ny;
         if (ck >= g.nz) ck -= g.nz;
         const int ci = cell - g.nx * (cj + g.ny * ck);
         const int lu = dualU(ci + sx - 1, g.nx, g.per[0]) - u0;
         const int lc = lu + 1 - sx, ly = 1 - sy, lz = 1 - sz;
         clamp = pushF32(g, s_f, FS, s, pp, ci, cj, ck, lc, ly, lz, o, v);
         if (isnan(o[0]) || isnan(o[1]) || isnan(o[2])) raiseError(err, RHGPU_DEVERR_NAN_PARTICLE);
         int ox, oy, oz;
         int bad = migrateAxisF(o[0], ox, pp.below1);
         bad |= migrateAxisF(o[1], oy, pp.below1);
         bad |= migrateAxisF(o[2], oz, pp.below1);
         ti = ci + ox; tj = cj + oy; tk = ck + oz;
         const bool inside = wrapc(ti, g.nx, g.per[0]) && wrapc(tj, g.ny, g.per[1]) && wrapc(tk, g.nz, g.per[2]);
         const double w = FS.w[s];
         const double ke = w * ((double)v[0] * v[0] + (double)v[1] * v[1] + (double)v[2] * v[2]);
         if (bad || !inside) {
            atomicAdd(&cntd[4 * s + 0], w);
            atomicAdd(&cntd[4 * s + 1], ke);
         } else {
            vx = dualU(ti + halfSf(o[0]) - 1, g.nx, g.per[0]);
            vy = dualU(tj + halfSf(o[1]) - 1, g.ny, g.per[1]);
            vz = dualU(tk + halfSf(o[2]) - 1, g.nz, g.per[2]);
            const bool inSeg = vy == uy && vz == uz && vx >= u0 && vx < u1;
            if (FS.accumulate[s]) {
               if (inSeg) {
                  rec = true;   // its CIC weights are formed just before the record is written
               } else {
                  mflags |= MOVER_DEPOSIT;
               }
            }
            bool removed = false;
            if (!allNb(g, ti, tj, tk)) {
               removed = true;
               atomicAdd(&cntd[4 * s + 0], w);
               atomicAdd(&cntd[4 * s + 1], ke);
            } else if (f.flags[cidx(g, ti, tj, tk)] & RHGPU_FLAG_INNER_PARTICLE) {
               const float xp = (float)blockOrigin(g.x_min, ti, g.dx) + o[0] * pp.dx;
               const float yp = (float)blockOrigin(g.y_min, tj, g.dx) + o[1] * pp.dx;
               const float zp = (float)blockOrigin(g.z_min, tk, g.dx) + o[2] * pp.dx;
               if (xp * xp + yp * yp + zp * zp < FS.R2obs[s]) {
                  removed = true;
                  atomicAdd(&cntd[4 * s + 2], w);
                  atomicAdd(&cntd[4 * s + 3], ke);
               }
            }
            if (!removed) {
               stay = inSeg;
               if (!inSeg) mflags |= MOVER_PLACE;
            }
            leave = mflags != 0;
         }
      }
      if (clamp) atomicAdd(&cntu[CNT_SPECIES_MAXVI + s], 1ull);
      if (GC) gridCountAtomic(f, GC_CELL_MAX_VI, g.N, cell, clamp);

      const unsigned bs = __ballot_sync(0xffffffffu, stay), br = __ballot_sync(0xffffffffu, rec);
      if (lane == 0) {
         s_wcnt[warp] = __popc(bs);
         s_bs[warp] = bs;
      }
      s_wd[warp][lane] = 0;
      __syncwarp();
      const int rd = rec ? vx - u0 : 0;
      int rrank = 0;
      if (rec) {
         const unsigned mm = __match_any_sync(br, rd);
         rrank = __popc(mm & below);
         if (rrank == 0) s_wd[warp][rd] = __popc(mm);
      }
      __syncthreads();
      if (warp == 0) {
         int t = 0;
         int c[FW];
         for (int w = 0; w < FW; ++w) { c[w] = s_wd[w][lane]; t += c[w]; }
         int x = t;
         for (int q = 1; q < 32; q <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, q);
            if (lane >= q) x += y;
         }
         int b = x - t;
         s_bin[lane] = b;
         if (lane == 31) s_bin[SEG] = x;
         for (int w = 0; w < FW; ++w) { s_wd[w][lane] = b; b += c[w]; }
         const int sw = lane < FW ? s_wcnt[lane] : 0;
         int xs = sw;
         for (int q = 1; q < FW; q <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, xs, q);
            if (lane >= q) xs += y;
         }
         __syncwarp();
         if (lane < FW) s_wcnt[lane] = xs - sw;
      }
      {
         const unsigned lm = __ballot_sync(0xffffffffu, leave);
         if (lm) {
            const int leader = __ffs(lm) - 1;
            unsigned long long b0 = 0;
            if (lane == leader) b0 = atomicAdd(fb.nmovers, (unsigned long long)__popc(lm));
            b0 = __shfl_sync(0xffffffffu, b0, leader);
            if (leave) {
               const unsigned long long m = b0 + __popc(lm & below);
               if ((long long)m < fb.moverCap) {
                  Mover32& M = fb.movers[m];
                  for (int a = 0; a < 3; ++a) { M.o[a] = o[a]; M.v[a] = v[a]; }
                  M.cell = (int)cidx(g, ti, tj, tk);
                  M.species = s;
                  M.key = ((unsigned long long)S << 32) | (unsigned long long)p;
                  const int gd = vx / SEG;
                  M.dest = ((long long)vy + (long long)fg.nd[1] * vz) * fg.nseg + gd;
                  M.lx = (vx - gd * SEG) | mflags;
               } else {
                  raiseError(err, RHGPU_DEVERR_CAPACITY);
               }
            }
         }
      }
      __syncthreads();
      if (stay) {
         const int stayIdx = s_wcnt[warp] + __popc(bs & below);
         // (zero unless the species starts inside this chunk)
         const int p0 = s_prefix[s] - c0;
         const int firstIdx = p0 > 0 ? stayersIn(s_bs, 0, p0) : 0;
         const F32Species& SS = FS.st[s];
         const long long slot = SS.base[S] + s_stay[s] + (stayIdx - firstIdx);
         SS.nxt.cell[slot] = (int)cidx(g, ti, tj, tk);
         for (int a = 0; a < 3; ++a) { SS.nxt.o[a][slot] = o[a]; SS.nxt.v[a][slot] = v[a]; }
      }
      const int stayAdd = tid < ns ? stayersIn(s_bs, max(s_prefix[tid], c0) - c0, min(s_prefix[tid + 1], c0 + FT) - c0) : 0;
      if (rec) {
         float w8[8];
         cicWeightsF(o, FS.wqRel[s], w8);
         float* r = s_rec + (s_wd[warp][rd] + rrank) * REC32;
         for (int q = 0; q < 8; ++q) r[q] = w8[q];
         r[8] = v[0]; r[9] = v[1]; r[10] = v[2];
      }
      __syncthreads();
      if (tid < ns) s_stay[tid] += stayAdd;
      {
         const int r1 = s_bin[myDual + 1];
#pragma unroll 2
         for (int r = s_bin[myDual]; r < r1; ++r) {
            const float* rr = s_rec + r * REC32;
            const float w = rr[myCorner];
            a0 += w;
            a1 += w * rr[8];
            a2 += w * rr[9];
            a3 += w * rr[10];
         }
      }
   }

   __syncthreads();
   if (tid < ns) FS.st[tid].nxt.cnt[S] = s_stay[tid];
   {
      float* q = s_rec + myDual * 32 + myCorner * 4;
      q[0] = a0; q[1] = a1; q[2] = a2; q[3] = a3;
   }
   __syncthreads();
   const int nx = g.nx;
   const long long nrows = fg.nrows;
   for (int e = tid; e < SEG * 16; e += FT) {
      const int dl = e >> 4, qq = (e >> 2) & 3, m = e & 3;
      const int lo = u0 + dl;
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
      float val = s_rec[dl * 32 + ((1 + 2 * qq) << 2) + m];
      if (hi >= 0) val = val + s_rec[hi * 32 + ((2 * qq) << 2) + m];
      fb.RP[(((long long)qq * nrows + row) * nx + x) * 4 + m] = val;
   }
   if (tid < 16 && (g.per[0] ? fg.nseg > 1 : gseg >= 1)) {
      const int qq = tid >> 2, m = tid & 3;
      fb.RPB[(((long long)qq * nrows + row) * fg.nseg + gseg) * 4 + m] = s_rec[((2 * qq) << 2) + m];
   }
}

// mover order[q] to slot q - off[bucket] after its bucket's stayers (bucket nb: not placed)
__global__ void k_f32_mig_place(F32Set FS, long long NS, long long nb, const Mover32* mv, const unsigned* order,
                                const unsigned* bkt, const long long* off, long long n) {
   const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (q >= n) return;
   const long long b = bkt[q];
   if (b >= nb) return;
   const int s = (int)(b / NS);
   const long long S = b % NS;
   const F32Species& SS = FS.st[s];
   const long long pos = SS.base[S] + SS.nxt.cnt[S] + (q - off[b]);
   const Mover32& M = mv[order[q]];
   SS.nxt.cell[pos] = M.cell;
   for (int e = 0; e < 3; ++e) { SS.nxt.o[e][pos] = M.o[e]; SS.nxt.v[e][pos] = M.v[e]; }
}

// CIC contributions of the particles that left their segment, exact fixed-point sums
__global__ void k_f32_mover_deposit(GridInfo g, FastGeom fg, F32Set FS, F32Bufs fb, long long n) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= n) return;
   const Mover32& M = fb.movers[t];
   if (!(M.lx & MOVER_DEPOSIT)) return;
   const int s = M.species;
   const long long row = M.dest / fg.nseg;
   const int vx = (int)(M.dest % fg.nseg) * SEG + (M.lx & 0xff);
   const int vy = (int)(row % fg.nd[1]), vz = (int)(row / fg.nd[1]);
   const int bx = dualB(vx, g.per[0]), by = dualB(vy, g.per[1]), bz = dualB(vz, g.per[2]);
   float o[3] = {M.o[0], M.o[1], M.o[2]};
   float w8[8];
   cicWeightsF(o, FS.wqRel[s], w8);
   const long long N = g.N;
   for (int q = 0; q < 8; ++q) {
      int dxc = bx + (q & 1), dyc = by + ((q >> 1) & 1), dzc = bz + ((q >> 2) & 1);
      if (!wrapc(dxc, g.nx, g.per[0]) || !wrapc(dyc, g.ny, g.per[1]) || !wrapc(dzc, g.nz, g.per[2])) continue;
      const long long dc = cidx(g, dxc, dyc, dzc);
      add128(&fb.MMlo[dc], &fb.MMhi[dc], (double)w8[q], fb.scaleR);
      for (int l = 0; l < 3; ++l)
         add128(&fb.MMlo[(1 + l) * N + dc], &fb.MMhi[(1 + l) * N + dc], (double)(w8[q] * M.v[l]), fb.scaleJ);
      atomicOr(&fb.touched[dc >> 5], 1u << (dc & 31));
   }
}

// cell moments: four row partials (+ boundary partials) + fixed-point part, times (w q)_0 / dV
template <bool GC>   // GC: also count the rho clamp per cell (grid counters on)
__global__ void k_f32_gather(GridInfo g, Fields f, FastGeom fg, F32Bufs fb, double hiR, double loR, double hiJ,
                             double loJ, double scale, double minRho, unsigned long long* cnt) {
   RH_CELL_PROLOGUE
   const bool bnd = g.per[0] ? (fg.nseg > 1 && i % SEG == 0) : ((i + 1) % SEG == 0);
   const int gb = g.per[0] ? i / SEG : (i + 1) / SEG;
   // every load first (one wait for memory), the same sums in the same order
   float4 rp[4];
   float rb[4][4];
#pragma unroll
   for (int qq = 0; qq < 4; ++qq) {
      const int uyy = dualU(j - (qq & 1), g.ny, g.per[1]);
      const int uzz = dualU(k - (qq >> 1), g.nz, g.per[2]);
      const long long row = (long long)uyy + (long long)fg.nd[1] * uzz;
      rp[qq] = *reinterpret_cast<const float4*>(fb.RP + (((long long)qq * fg.nrows + row) * g.nx + i) * 4);
      if (bnd) {
         const float* pb = fb.RPB + (((long long)qq * fg.nrows + row) * fg.nseg + gb) * 4;
#pragma unroll
         for (int l = 0; l < 4; ++l) rb[qq][l] = pb[l];
      }
   }
   const unsigned tw = fb.touched[n >> 5];
   unsigned long long mlo[4], mhi[4];
#pragma unroll
   for (int l = 0; l < 4; ++l) { mlo[l] = fb.MMlo[l * N + n]; mhi[l] = fb.MMhi[l * N + n]; }
   double v[4];
#pragma unroll
   for (int qq = 0; qq < 4; ++qq) {
      const float rv[4] = {rp[qq].x, rp[qq].y, rp[qq].z, rp[qq].w};
#pragma unroll
      for (int l = 0; l < 4; ++l) {
         float r = rv[l];
         if (bnd) r = r + rb[qq][l];
         v[l] = qq == 0 ? (double)r : v[l] + (double)r;
      }
   }
   if (tw & (1u << (n & 31))) {
      v[0] += fixedToDouble(mlo[0], mhi[0], hiR, loR);
      for (int l = 0; l < 3; ++l) v[1 + l] += fixedToDouble(mlo[1 + l], mhi[1 + l], hiJ, loJ);
      for (int l = 0; l < 4; ++l) { fb.MMlo[l * N + n] = 0ull; fb.MMhi[l * N + n] = 0ull; }
   }
   double rho = v[0] * scale;
   bool clamp = false;
   if (rho < minRho) { rho = minRho; clamp = true; }
   countIf(clamp, &cnt[CNT_MIN_CELL_RHO]);
   if (GC) gridCount(f, GC_CELL_MIN_RHOQI, N, n, clamp);
   f.cellRho[n] = rho;
   for (int l = 0; l < 3; ++l) f.cellJi[l * N + n] = v[1 + l] * scale;
}

// ---- upload / download / relayout ----------------------------------------------------------
__device__ inline float offsetOf(double x, double rdx, float below1) {
   float o = (float)(x * rdx);
   if (o >= 1.0f) o = below1;
   if (o < 0.0f) o = 0.0f;
   return o;
}
// segment and dual x of each uploaded particle, from its FP32 offsets
__global__ void k_f32_seg_of(GridInfo g, FastGeom fg, const double* aos, const int* pcell, long long n, float below1,
                             unsigned* key) {
   const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (p >= n) return;
   const int c = pcell[p];
   const int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
   const double* st = aos + 7 * p;
   const int ux = dualU(i + halfSf(offsetOf(st[0], g.rdx, below1)) - 1, g.nx, g.per[0]);
   const int uy = dualU(j + halfSf(offsetOf(st[1], g.rdx, below1)) - 1, g.ny, g.per[1]);
   const int uz = dualU(k + halfSf(offsetOf(st[2], g.rdx, below1)) - 1, g.nz, g.per[2]);
   key[p] = (unsigned)(((long long)uy + (long long)fg.nd[1] * uz) * fg.nseg + ux / SEG);
}
__global__ void k_f32_scatter_sorted(GridInfo g, const double* aos, const int* pcell, const unsigned* key,
                                     const unsigned* idx, long long n, const long long* first, F32Buf B,
                                     const long long* base, float below1) {
   const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (j >= n) return;
   const unsigned S = key[j];
   const long long slot = base[S] + (j - first[S]);
   const unsigned src = idx[j];
   const double* st = aos + 7LL * src;
   B.cell[slot] = pcell[src];
   for (int a = 0; a < 3; ++a) {
      B.o[a][slot] = offsetOf(st[a], g.rdx, below1);
      B.v[a][slot] = (float)st[3 + a];
   }
}
__global__ void k_f32_cell_keys(FastGeom fg, F32Buf B, const long long* base, const long long* first, unsigned* key,
                                unsigned long long* slots) {
   const long long S = blockIdx.x;
   const int c = B.cnt[S];
   for (int r = threadIdx.x; r < c; r += blockDim.x) {
      const long long slot = base[S] + r;
      key[first[S] + r] = (unsigned)B.cell[slot];
      slots[first[S] + r] = (unsigned long long)slot;
   }
}
__global__ void k_f32_gather_records(F32Buf B, const unsigned long long* slots, const unsigned* idx, long long n,
                                     double dx, double w, double* aos) {
   const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (j >= n) return;
   const unsigned long long slot = slots[idx[j]];
   for (int a = 0; a < 3; ++a) {
      aos[7 * j + a] = (double)B.o[a][slot] * dx;
      aos[7 * j + 3 + a] = (double)B.v[a][slot];
   }
   aos[7 * j + 6] = w;
}
__global__ void k_f32_relayout(F32Buf from, const long long* fromBase, F32Buf to, const long long* toBase) {
   const long long S = blockIdx.x;
   const int c = from.cnt[S];
   const long long a0 = fromBase[S], b0 = toBase[S];
   for (int r = threadIdx.x; r < c; r += blockDim.x) {
      to.cell[b0 + r] = from.cell[a0 + r];
      for (int e = 0; e < 3; ++e) { to.o[e][b0 + r] = from.o[e][a0 + r]; to.v[e][b0 + r] = from.v[e][a0 + r]; }
   }
   if (threadIdx.x == 0) to.cnt[S] = c;
}
// min and max |weight| of uploaded particles, grid-stride with one atomic pair per block
// (bit patterns of non-negative doubles order like the values)
__global__ void k_weight_range(const double* aos, long long n, unsigned long long* mn, unsigned long long* mx) {
   __shared__ double slo[32], shi[32];
   double lo = 1e308, hi = 0.0;
   for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
      const double w = fabs(aos[7 * p + 6]);
      lo = fmin(lo, w);
      hi = fmax(hi, w);
   }
   for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
   }
   if ((threadIdx.x & 31) == 0) { slo[threadIdx.x >> 5] = lo; shi[threadIdx.x >> 5] = hi; }
   __syncthreads();
   if (threadIdx.x == 0) {
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { lo = fmin(lo, slo[w]); hi = fmax(hi, shi[w]); }
      atomicMin(mn, (unsigned long long)__double_as_longlong(lo));
      atomicMax(mx, (unsigned long long)__double_as_longlong(hi));
   }
}
// population log sums of one FP32-form species in FP64 (see k_diag.cuh)
__global__ void __launch_bounds__(DIAG_THREADS)
k_diag_particles_f32(F32Buf B, const long long* base, long long NS, double w, double* part) {
   __shared__ double sm[DIAG_THREADS];
   double v[DIAG_P] = {0, 0, 0, 0, 0, 0, 0, 0};
   for (long long S = blockIdx.x; S < NS; S += gridDim.x)
      for (int r = threadIdx.x; r < B.cnt[S]; r += blockDim.x) {
         double st[7];
         for (int e = 0; e < 3; ++e) { st[e] = 0.0; st[3 + e] = (double)B.v[e][base[S] + r]; }
         st[6] = w;
         particleTerms(st, v);
      }
   blockReduce(v, DIAG_P_MAX, sm, part + (long long)blockIdx.x * DIAG_P);
}

// total ion mass density (logCalcParticle, diagnostics.h:223-238) on the FP32
// form: every particle adds its species' w*m to its cell as an exact fixed-point sum
__global__ void k_diag_rhom_f32(F32Buf B, const long long* base, long long NS, double wm, double scale,
                                unsigned long long* lo, unsigned long long* hi) {
   for (long long S = blockIdx.x; S < NS; S += gridDim.x)
      for (int r = threadIdx.x; r < B.cnt[S]; r += blockDim.x) {
         const long long n = B.cell[base[S] + r];
         add128(lo + n, hi + n, wm, scale);
      }
}

}  // namespace rh
