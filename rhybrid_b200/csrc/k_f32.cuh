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
   unsigned char* touched;
   const unsigned char* segInner;   // per segment: an obstacle cell within reach (shared with the fast path)
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
      // (fused multiply-adds: the FP32 form is not held to the FP64 operation order)
      B[0] = fmaf(xs, F.bx[lz][ly][lc + 1], (1.0f - xs) * F.bx[lz][ly][lc]);
      B[1] = fmaf(ys, F.by[lz][ly + 1][lc], (1.0f - ys) * F.by[lz][ly][lc]);
      B[2] = fmaf(zs, F.bz[lz + 1][ly][lc], (1.0f - zs) * F.bz[lz][ly][lc]);
      for (int l = 0; l < 3; ++l) Ue[l] = F.ue[l][lz][ly][lc];
      E[0] = fmaf(B[1], Ue[2], -(B[2] * Ue[1]));
      E[1] = fmaf(B[2], Ue[0], -(B[0] * Ue[2]));
      E[2] = fmaf(B[0], Ue[1], -(B[1] * Ue[0]));
      if (pp.use_ep) for (int l = 0; l < 3; ++l) E[l] += F.ep[l][lz][ly][lc];
      const float qm = FS.qm[s];
      const float dvx = qm * E[0], dvy = qm * E[1], dvz = qm * E[2];
      const float tx = qm * B[0], ty = qm * B[1], tz = qm * B[2];
      const float t2 = fmaf(tx, tx, fmaf(ty, ty, tz * tz));
      const float b2 = 2.0f / (1.0f + t2);
      const float sx = b2 * tx, sy = b2 * ty, sz = b2 * tz;
      const float vmx = vx + dvx, vmy = vy + dvy, vmz = vz + dvz;
      const float v0x = fmaf(-vmz, ty, fmaf(vmy, tz, vmx));
      const float v0y = fmaf(-vmx, tz, fmaf(vmz, tx, vmy));
      const float v0z = fmaf(-vmy, tx, fmaf(vmx, ty, vmz));
      const float vpx = fmaf(-v0z, sy, fmaf(v0y, sz, vmx));
      const float vpy = fmaf(-v0x, sz, fmaf(v0z, sx, vmy));
      const float vpz = fmaf(-v0y, sx, fmaf(v0x, sy, vmz));
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
      const float v2 = fmaf(vx, vx, fmaf(vy, vy, vz * vz));
      if (v2 > pp.maxVi2) {
         const float norm = sqrtf(pp.maxVi2 / v2);
         vx *= norm; vy *= norm; vz *= norm;
         clamp = true;
      }
   }
   v[0] = vx; v[1] = vy; v[2] = vz;
   o[0] = fmaf(pp.dtdx, vx, o[0]);
   o[1] = fmaf(pp.dtdx, vy, o[1]);
   o[2] = fmaf(pp.dtdx, vz, o[2]);
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

// shared memory of k_f32_push_deposit
constexpr int F32_PTRS = 14;   // one species' arrays offset to the segment: current cell, o, v (0-6), next (7-13)
struct F32PushShared {
   float rec[FT * REC32];                   // deposit records of a chunk; at the end acc[SEG][32]
   float pf[7][FT];                         // the next chunk's particles: cell (int bits), o[3], v[3]
   SegFields32 f;                           // field stencil of the segment
   void* ptr[FAST_MAX_SPECIES][F32_PTRS];
   StencilRow rows[SF_MAX_ROWS];
   alignas(8) unsigned char wd[SEG][FW];    // records per (dual cell, warp)
   int rank[FT];                            // stayers of the chunk before each chunk position
   int wcnt[FW];                            // stayers per warp
   int prefix[FAST_MAX_SPECIES + 1];        // first particle of each species in the segment
   int stay[FAST_MAX_SPECIES];              // stayers of each species so far
};

// chunk position tid of the chunk starting at c0 requested into pf (cp.async)
__device__ __forceinline__ void f32Prefetch(F32PushShared& sh, int i, int total, int ns, int s0) {
   const int tid = threadIdx.x;
   if (i < total) {
      int s = s0;
      while (s + 1 < ns && i >= sh.prefix[s + 1]) ++s;
      const int p = i - sh.prefix[s];
#pragma unroll
      for (int a = 0; a < 7; ++a) cpAsync4(&sh.pf[a][tid], (const float*)sh.ptr[s][a] + p);
   }
   cpAsyncCommit();
}

// PER: the periodic axes (bit a = axis a), fixed at compile time; the host
// launches the instantiation that matches the grid
// GC: the variant that also counts the per-cell maxVi constraint (grid counters on)
//
// One block per segment, one thread per particle, chunks of FT particles in
// storage order (species after species), as k_fast_push_deposit: the next
// chunk's particles are copied to shared memory (cp.async) while the current
// one is processed, two barriers per chunk, per-warp record counts packed in
// bytes, a leaving particle's mover slot reserved before the second barrier
// and written after the deposit sums.
template <int PER, bool GC>
__global__ void __launch_bounds__(FT, 4)
k_f32_push_deposit(GridInfo gIn, Fields f, FastGeom fg, F32Set FS, F32Params pp, F32Bufs fb, double* cntd,
                   unsigned long long* cntu, unsigned* err) {
   GridInfo g = gIn;
   g.per[0] = PER & 1;
   g.per[1] = (PER >> 1) & 1;
   g.per[2] = (PER >> 2) & 1;
   __shared__ F32PushShared sh;
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
   const unsigned below = (1u << lane) - 1u;
   const long long S = blockIdx.x;
   const long long row = S / fg.nseg;
   const int gseg = (int)(S % fg.nseg);
   const int uy = (int)(row % fg.nd[1]), uz = (int)(row / fg.nd[1]);
   const int ndx = fg.nd[0];
   const int u0 = gseg * SEG, u1 = min(u0 + SEG, ndx);
   const int ns = FS.ns;
   // set-up: species prefix (warp 0), segment pointers (warps 1-4)
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
   } else if (tid < 32 + F32_PTRS * ns) {
      const int q = tid - 32, s = q / F32_PTRS, k = q - s * F32_PTRS;
      const F32Species& SS = FS.st[s];
      const long long b = SS.base[S];
      const F32Buf& B = k < 7 ? SS.cur : SS.nxt;
      const int kk = k < 7 ? k : k - 7;
      void* v;
      if (kk == 0) v = B.cell + b;
      else if (kk < 4) v = B.o[kk - 1] + b;
      else v = B.v[kk - 4] + b;
      sh.ptr[s][k] = v;
   }
   const int by0 = dualB(uy, g.per[1]), bz0 = dualB(uz, g.per[2]);
   const bool segInner = fb.segInner[S] != 0;   // an obstacle cell within one step of the segment
   // (stageSegRows' own barrier publishes the prefix and the pointers)
   stageSegRows(g, f, pp.use_ep, dualB(u0, g.per[0]), by0, bz0, sh.f, sh.rows);
   __syncthreads();
   const int total = sh.prefix[ns];
   f32Prefetch(sh, tid, total, ns, 0);
   const int myDual = tid >> 3, myCorner = tid & 7;
   float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;

   for (int c0 = 0; c0 < total; c0 += FT) {
      const int i = c0 + tid;
      const bool active = i < total;
      int s = 0;
      if (active)
         while (s + 1 < ns && i >= sh.prefix[s + 1]) ++s;
      float o[3], v[3];
      int cell = 0, p = 0;
      bool stay = false, rec = false, leave = false, clamp = false;
      int mflags = 0, vx = 0, vy = 0, vz = 0, ti = 0, tj = 0, tk = 0;
      cpAsyncWaitAll();   // this thread's copies of the chunk
      if (active) {
         p = i - sh.prefix[s];
         cell = __float_as_int(sh.pf[0][tid]);
         for (int a = 0; a < 3; ++a) { o[a] = sh.pf[1 + a][tid]; v[a] = sh.pf[4 + a][tid]; }
         const int sx = halfSf(o[0]), sy = halfSf(o[1]), sz = halfSf(o[2]);
         int cj = by0 + 1 - sy, ck = bz0 + 1 - sz;
         if (cj >= g.ny) cj -= g.ny;
         if (ck >= g.nz) ck -= g.nz;
         const int ci = cell - g.nx * (cj + g.ny * ck);
         const int lu = dualU(ci + sx - 1, g.nx, g.per[0]) - u0;
         const int lc = lu + 1 - sx, ly = 1 - sy, lz = 1 - sz;
         clamp = pushF32(g, sh.f, FS, s, pp, ci, cj, ck, lc, ly, lz, o, v);
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
            } else if (segInner && (f.flags[cidx(g, ti, tj, tk)] & RHGPU_FLAG_INNER_PARTICLE)) {
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

      // ---- order of the chunk's stayers and records (warp-local first) ---------------------
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
      f32Prefetch(sh, i + FT, total, ns, s);
      // every warp, per dual cell (lane): the first sorted record of the dual cell
      // (bin) and of this warp's records for it (off)
      int binD, offD, nrec;
      {
         const uint2 c8 = *reinterpret_cast<const uint2*>(&sh.wd[lane][0]);
         const int t = (int)(((c8.x * 0x01010101u) >> 24) + ((c8.y * 0x01010101u) >> 24));
         const unsigned mlo = warp >= 4 ? 0xffffffffu : (1u << (8 * warp)) - 1u;
         const unsigned mhi = warp <= 4 ? 0u : (1u << (8 * (warp - 4))) - 1u;
         const int before = (int)((((c8.x & mlo) * 0x01010101u) >> 24) + (((c8.y & mhi) * 0x01010101u) >> 24));
         int x = t;
         for (int q = 1; q < 32; q <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, q);
            if (lane >= q) x += y;
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
         float w8[8];
         cicWeightsF(o, FS.wqRel[s], w8);
         float* r = sh.rec + recPos * REC32;
         for (int q = 0; q < 8; ++q) r[q] = w8[q];
         r[8] = v[0]; r[9] = v[1]; r[10] = v[2];
      }
      __syncthreads();
      if (stay) {
         const int p0 = sh.prefix[s] - c0;   // chunk position of the species' first particle
         const int q = stayBase + myRank - (p0 > 0 ? sh.rank[p0] : 0);
         ((int*)sh.ptr[s][7])[q] = (int)cidx(g, ti, tj, tk);
         for (int a = 0; a < 3; ++a) {
            ((float*)sh.ptr[s][8 + a])[q] = o[a];
            ((float*)sh.ptr[s][11 + a])[q] = v[a];
         }
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
         const float* rr = sh.rec + r * REC32;
         const float w = rr[myCorner];
         a0 += w;
         a1 = fmaf(w, rr[8], a1);
         a2 = fmaf(w, rr[9], a2);
         a3 = fmaf(w, rr[10], a3);
      }
      // ---- particles that left the segment -----------------------------------------------
      if (lm) {
         mb = __shfl_sync(0xffffffffu, mb, leader);
         if (leave) {
            const unsigned long long m = mb + __popc(lm & below);
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
      // no barrier here: the next chunk's first barrier orders the reads of rec,
      // rank and stay before their next writes
   }

   __syncthreads();
   if (tid < ns) FS.st[tid].nxt.cnt[S] = sh.stay[tid];
   {
      float* q = sh.rec + myDual * 32 + myCorner * 4;
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
      float val = sh.rec[dl * 32 + ((1 + 2 * qq) << 2) + m];
      if (hi >= 0) val = val + sh.rec[hi * 32 + ((2 * qq) << 2) + m];
      fb.RP[(((long long)qq * nrows + row) * nx + x) * 4 + m] = val;
   }
   if (tid < 16 && (g.per[0] ? fg.nseg > 1 : gseg >= 1)) {
      const int qq = tid >> 2, m = tid & 3;
      fb.RPB[(((long long)qq * nrows + row) * fg.nseg + gseg) * 4 + m] = sh.rec[((2 * qq) << 2) + m];
   }
}

// mover order[q] to slot q - off[bucket] after its bucket's stayers (bucket nb: not placed)
__global__ void k_f32_mig_place(F32Set FS, long long NS, long long nb, const Mover32* mv, const unsigned* order,
                                const unsigned* bkt, const long long* off, long long n);

// CIC contributions of the particles that left their segment, exact fixed-point sums
__global__ void k_f32_mover_deposit(GridInfo g, FastGeom fg, F32Set FS, F32Bufs fb, long long n);

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
   const unsigned tw = fb.touched[n];
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
   if (tw) {
      v[0] += fixedToDouble(mlo[0], mhi[0], hiR, loR);
      for (int l = 0; l < 3; ++l) v[1 + l] += fixedToDouble(mlo[1 + l], mhi[1 + l], hiJ, loJ);
   }
   // every cell's sums cleared for the next step, touched or not: whole sectors
   // written (a warp writing only its touched cells leaves partly written
   // sectors, which cost a read-modify-write each; 0.48 -> 0.17 ms per step)
   for (int l = 0; l < 4; ++l) { fb.MMlo[l * N + n] = 0ull; fb.MMhi[l * N + n] = 0ull; }
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
// uploaded records: 7 doubles (cell-local position [m], velocity, weight), or
// the FP32 form's own 6 floats (offsets in the cell in units of dx, velocity)
struct RecordsD {
   const double* a;
   __device__ float off(long long p, int k, double rdx, float below1) const { return offsetOf(a[7 * p + k], rdx, below1); }
   __device__ float vel(long long p, int k) const { return (float)a[7 * p + 3 + k]; }
};
struct RecordsF {
   const float* a;
   __device__ float off(long long p, int k, double, float below1) const {
      float o = a[6 * p + k];
      if (o >= 1.0f) o = below1;
      if (o < 0.0f) o = 0.0f;
      return o;
   }
   __device__ float vel(long long p, int k) const { return a[6 * p + 3 + k]; }
};

// segment and dual x of each uploaded particle, from its FP32 offsets
template <class R>
__global__ void k_f32_seg_of(GridInfo g, FastGeom fg, R rec, const int* pcell, long long n, float below1,
                             unsigned* key) {
   const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (p >= n) return;
   const int c = pcell[p];
   const int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
   const int ux = dualU(i + halfSf(rec.off(p, 0, g.rdx, below1)) - 1, g.nx, g.per[0]);
   const int uy = dualU(j + halfSf(rec.off(p, 1, g.rdx, below1)) - 1, g.ny, g.per[1]);
   const int uz = dualU(k + halfSf(rec.off(p, 2, g.rdx, below1)) - 1, g.nz, g.per[2]);
   key[p] = (unsigned)(((long long)uy + (long long)fg.nd[1] * uz) * fg.nseg + ux / SEG);
}
template <class R>
__global__ void k_f32_scatter_sorted(GridInfo g, R rec, const int* pcell, const unsigned* key,
                                     const unsigned* idx, long long n, const long long* first, F32Buf B,
                                     const long long* base, float below1) {
   const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (j >= n) return;
   const unsigned S = key[j];
   const long long slot = base[S] + (j - first[S]);
   const unsigned src = idx[j];
   B.cell[slot] = pcell[src];
   for (int a = 0; a < 3; ++a) {
      B.o[a][slot] = rec.off(src, a, g.rdx, below1);
      B.v[a][slot] = rec.vel(src, a);
   }
}
__global__ void k_f32_cell_keys(FastGeom fg, F32Buf B, const long long* base, const long long* first, unsigned* key,
                                unsigned long long* slots);
__global__ void k_f32_gather_records(F32Buf B, const unsigned long long* slots, const unsigned* idx, long long n,
                                     double dx, double w, double* aos);
// the FP32 form's own records: 6 floats per particle, offsets and velocity as stored
__global__ void k_f32_gather_records_f32(F32Buf B, const unsigned long long* slots, const unsigned* idx, long long n,
                                         float* rec);
__global__ void k_f32_relayout(F32Buf from, const long long* fromBase, F32Buf to, const long long* toBase);
// min and max |weight| of uploaded particles, grid-stride with one atomic pair per block
// (bit patterns of non-negative doubles order like the values)
__global__ void k_weight_range(const double* aos, long long n, unsigned long long* mn, unsigned long long* mx);
// population log sums of one FP32-form species in FP64 (see k_diag.cuh)
__global__ void __launch_bounds__(DIAG_THREADS)
k_diag_particles_f32(F32Buf B, const long long* base, long long NS, double w, double* part);

// total ion mass density (logCalcParticle, diagnostics.h:223-238) on the FP32
// form: every particle adds its species' w*m to its cell as an exact fixed-point sum
__global__ void k_diag_rhom_f32(F32Buf B, const long long* base, long long NS, double wm, double scale,
                                unsigned long long* lo, unsigned long long* hi);

}  // namespace rh
