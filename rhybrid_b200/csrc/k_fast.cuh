// Fast path (sm_100a, FP64): fused push + CIC deposit over particles grouped
// by CIC dual cell. Same per-particle and per-cell arithmetic as the bit-exact
// path; the deposit sums are formed in a different (fixed) order, restated
// bit for bit by the oracle's RHO_DEPOSIT_GPU mode (oracle/rh_oracle.c).
//
// Storage (per species): particles grouped by dual cell, the 2x2x2 block of
// cells whose centres surround the particle (base b = c + s - 1 per axis,
// s = 0 if x < 0.5 dx else 1, as accumulateCell's index shift,
// particle_accumulator.cpp:78-84). Dual index u = b + 1 on a non-periodic axis,
// b mod n on a periodic one. Dual cell D owns slots [start[D], start[D+1]);
// the first cnt[D] hold particles.
//
//   k_fast_push_deposit  one warp per dual row (uy, uz): push (boris.h:64-194)
//                        + migration + CIC weights of the new position; the
//                        contributions go to a 3-dual-cell window of running sums
//                        held across the lanes (lane q = corner*4 + moment) and
//                        leave as row partials; off-row movers are deposited as
//                        exact 128-bit fixed-point sums; boundary removals
//                        (particle_boundary_cond_hybrid.h:112-185) happen here
//   k_fast_mig_*         placement of off-row movers, in a fixed order
//   k_fast_gather        cell moments from the 4 row partials + fixed-point
//                        part, then /dV and the rho clamp (particle_accumulator.cpp:319-333)
#pragma once

#include "rh_device.cuh"
#include "k_fields.cuh"
#include "k_particles.cuh"

namespace rh {

constexpr int FAST_MAX_SPECIES = 8;
constexpr int FAST_WARPS = 4;

struct DStore {
   double* a[7];
   long long* start;   // Nd+1 slot offsets
   int* cnt;           // particles per dual cell
   long long cap;
};

struct FastGeom {
   int nd[3];
   long long Nd;
   long long nrows;
};

struct FastSpecies {
   int ns;
   DStore st[FAST_MAX_SPECIES];
   SpeciesDev sp[FAST_MAX_SPECIES];
};

// off-row mover record: key orders the arrivals of a destination dual cell:
// (class << 62) | (source dual index << 24) | rank in the source
struct Mover {
   double s[7];
   unsigned long long key;
   long long dest;      // destination dual index
   int species;
   int pad;
};

struct FastBufs {
   double* RP;                 // 4 planes x nrows x nx x 4
   unsigned long long* MMlo;   // 4 x N
   unsigned long long* MMhi;   // 4 x N
   unsigned* touched;          // bit per cell: MM nonzero this step
   Mover* movers;
   unsigned long long* nmovers;
   long long moverCap;
   double* pend;               // per row: ns x 2 x pendCap records of 8 doubles
   int pendCap;
   double scaleR, scaleJ;      // 2^kR, 2^kJ
};

__host__ __device__ inline int dualU(int b, int n, int per) { return per ? ((b % n) + n) % n : b + 1; }
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

// per-warp state of the storage placement, one entry per species
struct PlaceState {
   int fill;      // particles placed in the previous dual cell of the row (u-1)
   int full;      // the previous dual cell stopped taking in-row arrivals
   int stay;      // stayers of the current dual cell placed so far
   int npPrev;    // +x movers from u-1 waiting for the current dual cell
   int npCur;     // +x movers from the current dual cell waiting for u+1
   int pendSel;   // which of the two pending buffers is "prev"
};

__device__ inline void warpSumAtomic(double v, double* dst) {
   for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
   if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(dst, v);
}

__global__ void __launch_bounds__(32 * FAST_WARPS)
k_fast_push_deposit(GridInfo g, Fields f, FastGeom fg, FastSpecies FS, PushParams pp, FastBufs fb,
                    double* cntd, unsigned long long* cntu, unsigned* err) {
   __shared__ double s_w[FAST_WARPS][32][12];   // w8[8], v[3] of the batch's particles
   __shared__ int s_tgt[FAST_WARPS][32];        // target dual x of the window, -1: none
   __shared__ PlaceState s_ps[FAST_WARPS][FAST_MAX_SPECIES];
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const long long row = (long long)blockIdx.x * FAST_WARPS + warp;
   if (row >= fg.nrows) return;
   const int ndx = fg.nd[0];
   const int uy = (int)(row % fg.nd[1]), uz = (int)(row / fg.nd[1]);
   const int ns = FS.ns;
   const long long N = g.N;
   const int nx = g.nx;
   const double dx = g.dx;
   const int q = lane, qo = q >> 2, ql = q & 3;   // corner and moment of this lane's window sums
   if (lane < ns) {
      PlaceState z;
      z.fill = 0; z.full = 0; z.stay = 0; z.npPrev = 0; z.npCur = 0; z.pendSel = 0;
      s_ps[warp][lane] = z;
   }
   __syncwarp();
   // deposit window over dual x = wb, wb+1, wb+2
   int wb = -1;
   double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
   double pend = 0.0, wrap0 = 0.0;
   int nextFlush = 0;       // dual cells < nextFlush have been flushed
   const int perx = g.per[0];
   const long long nrows = fg.nrows;
   double* RP = fb.RP;

   // flush dual cell u: destination row partial of x = base(u)
   auto flush = [&](int u) {
      // window slot of u
      const int sl = u - wb;
      const double a = sl == 0 ? acc0 : (sl == 1 ? acc1 : acc2);
      const double partner = __shfl_xor_sync(0xffffffffu, pend, 4);
      const bool ox0 = ((qo & 1) == 0);
      if (ox0) {
         const double out = partner + a;
         const int x = dualB(u, perx);
         const int qq = qo >> 1;
         if (perx && u == 0) {
            wrap0 = a;
         } else if (x >= 0 && x < nx) {
            RP[(((long long)qq * nrows + row) * nx + x) * 4 + ql] = out;
         }
      } else {
         pend = a;
      }
   };
   auto slide = [&](int newWb) {
      while (wb < newWb) {
         if (wb >= 0 && wb >= nextFlush) { flush(wb); nextFlush = wb + 1; }
         acc0 = acc1; acc1 = acc2; acc2 = 0.0;
         ++wb;
      }
   };

   const int ngroups = ndx * ns;
   int G = 0, r0 = 0;
   while (G < ngroups) {
      // ---- form a batch from groups G .. G+31 --------------------------------
      const int gl = G + lane;
      int rem = 0;
      long long gstart = 0;
      if (gl < ngroups) {
         const int u = gl / ns, s = gl % ns;
         const long long D = (long long)u + (long long)ndx * row;
         rem = FS.st[s].cnt[D] - (lane == 0 ? r0 : 0);
         gstart = FS.st[s].start[D] + (lane == 0 ? r0 : 0);
      }
      int cum = rem;
      for (int o = 1; o < 32; o <<= 1) {
         const int t = __shfl_up_sync(0xffffffffu, cum, o);
         if (lane >= o) cum += t;
      }
      const int total = __shfl_sync(0xffffffffu, cum, 31);
      const int nb = total < 32 ? total : 32;
      // group of this lane's particle: number of groups whose cumulative count is <= lane
      int gidx = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
         const int cm = __shfl_sync(0xffffffffu, cum, gidx + step - 1);
         if (cm <= lane) gidx += step;
      }
      if (gidx > 31) gidx = 31;
      const int cumPrev = __shfl_sync(0xffffffffu, cum, gidx > 0 ? gidx - 1 : 0);
      const long long gst = __shfl_sync(0xffffffffu, gstart, gidx);
      const int within = lane - (gidx > 0 ? cumPrev : 0);
      const int myG = G + gidx;
      const int u = myG / ns, s = myG % ns;
      const int rank = within + (gidx == 0 ? r0 : 0);
      const bool active = lane < nb;
      // ---- lane-parallel push, migration, classification ------------------------
      double st[7];
      int cls = -1;         // 0 stay, 1 -x in-row, 2 +x in-row, 3 off-row, -1 removed/none
      int tgt = -1;         // window target dual x
      long long Dn = -1;
      int ti = 0, tj = 0, tk = 0;
      bool clamp = false;
      if (active) {
         const DStore& S = FS.st[s];
         const long long p = gst + within;
         for (int a = 0; a < 7; ++a) st[a] = S.a[a][p];
         int ci = dualB(u, g.per[0]) + 1 - halfS(st[0], dx);
         int cj = dualB(uy, g.per[1]) + 1 - halfS(st[1], dx);
         int ck = dualB(uz, g.per[2]) + 1 - halfS(st[2], dx);
         wrapc(ci, g.nx, 1); wrapc(cj, g.ny, 1); wrapc(ck, g.nz, 1);
         clamp = pushOne(g, f, FS.sp[s], pp, ci, cj, ck, st);
         if (isnan(st[0]) || isnan(st[1]) || isnan(st[2])) raiseError(err, RHGPU_DEVERR_NAN_PARTICLE);
         int ox, oy, oz;
         int bad = migrateAxis(st[0], ox, dx, g.dx_below);
         bad |= migrateAxis(st[1], oy, dx, g.dx_below);
         bad |= migrateAxis(st[2], oz, dx, g.dx_below);
         ti = ci + ox; tj = cj + oy; tk = ck + oz;
         const bool inside = wrapc(ti, g.nx, g.per[0]) && wrapc(tj, g.ny, g.per[1]) && wrapc(tk, g.nz, g.per[2]);
         const double ke = st[6] * (sq(st[3]) + sq(st[4]) + sq(st[5]));
         if (bad || !inside) {
            atomicAdd(&cntd[4 * s + 0], st[6]);
            atomicAdd(&cntd[4 * s + 1], ke);
         } else {
            const int sx = halfS(st[0], dx), sy = halfS(st[1], dx), sz = halfS(st[2], dx);
            const int bx = ti + sx - 1, by = tj + sy - 1, bz = tk + sz - 1;
            const int vx = dualU(bx, g.nx, g.per[0]), vy = dualU(by, g.ny, g.per[1]), vz = dualU(bz, g.nz, g.per[2]);
            Dn = (long long)vx + (long long)ndx * ((long long)vy + (long long)fg.nd[1] * vz);
            const bool inRow = vy == uy && vz == uz && abs(vx - u) <= 1;
            if (FS.sp[s].accumulate) {
               double w8[8];
               int ind[8];
               cicWeights(st[0], st[1], st[2], st[6] * FS.sp[s].q, dx, w8, ind);
               if (inRow) {
                  for (int o = 0; o < 8; ++o) s_w[warp][lane][o] = w8[o];
                  s_w[warp][lane][8] = st[3]; s_w[warp][lane][9] = st[4]; s_w[warp][lane][10] = st[5];
                  tgt = vx;
               } else {
                  for (int o = 0; o < 8; ++o) {
                     int dxc = bx + (o & 1), dyc = by + ((o >> 1) & 1), dzc = bz + ((o >> 2) & 1);
                     if (!wrapc(dxc, g.nx, g.per[0]) || !wrapc(dyc, g.ny, g.per[1]) || !wrapc(dzc, g.nz, g.per[2])) continue;
                     const long long dc = cidx(g, dxc, dyc, dzc);
                     add128(&fb.MMlo[dc], &fb.MMhi[dc], w8[o], fb.scaleR);
                     for (int l = 0; l < 3; ++l)
                        add128(&fb.MMlo[(1 + l) * N + dc], &fb.MMhi[(1 + l) * N + dc], w8[o] * st[3 + l], fb.scaleJ);
                     atomicOr(&fb.touched[dc >> 5], 1u << (dc & 31));
                  }
               }
            }
            // boundary conditions of the step
            const long long cn = cidx(g, ti, tj, tk);
            bool removed = false;
            if (!allNb(g, ti, tj, tk)) {
               removed = true;
               atomicAdd(&cntd[4 * s + 0], st[6]);
               atomicAdd(&cntd[4 * s + 1], ke);
            } else if (f.flags[cn] & RHGPU_FLAG_INNER_PARTICLE) {
               const double xp = blockOrigin(g.x_min, ti, dx) + st[0];
               const double yp = blockOrigin(g.y_min, tj, dx) + st[1];
               const double zp = blockOrigin(g.z_min, tk, dx) + st[2];
               if (sq(xp) + sq(yp) + sq(zp) < FS.sp[s].R2obs) {
                  removed = true;
                  atomicAdd(&cntd[4 * s + 2], st[6]);
                  atomicAdd(&cntd[4 * s + 3], ke);
               }
            }
            if (!removed) {
               if (vx == u && vy == uy && vz == uz) cls = 0;
               else if (inRow && vx == u - 1) cls = 1;
               else if (inRow && vx == u + 1) cls = 2;
               else cls = 3;
            }
         }
      }
      s_tgt[warp][lane] = active ? tgt : -1;
      if (clamp) atomicAdd(&cntu[CNT_SPECIES_MAXVI + s], 1ull);
      __syncwarp();
      // ---- transposed deposit of the batch, in particle order --------------------
      for (int jj = 0; jj < nb; ++jj) {
         const int tv = s_tgt[warp][jj];
         if (tv < 0) continue;
         const int uj = __shfl_sync(0xffffffffu, u, jj);
         if (uj - 1 > wb) slide(uj - 1);
         const double w = s_w[warp][jj][qo];
         const double val = ql == 0 ? w : w * s_w[warp][jj][8 + ql - 1];
         const int sl = tv - wb;
         if (sl == 0) acc0 += val;
         else if (sl == 1) acc1 += val;
         else acc2 += val;
      }
      // ---- advance the group cursor ------------------------------------------------------
      // groups G .. gEnd-1 are finished by this batch; group G+lastIdx may continue
      int gEnd, lastIdx, r0n;
      {
         lastIdx = __shfl_sync(0xffffffffu, gidx, nb > 0 ? nb - 1 : 0);
         const int lastCum = __shfl_sync(0xffffffffu, cum, lastIdx);
         // groups after lastIdx (within the 32 read) with nothing left are finished too
         const unsigned emptyAfter = __ballot_sync(0xffffffffu, lane > lastIdx && G + lane < ngroups && cum == nb);
         if (nb == 0) {
            gEnd = min(G + 32, ngroups);
            r0n = 0;
         } else if (nb == lastCum) {
            int e = lastIdx + 1;
            while (e < 32 && ((emptyAfter >> e) & 1u)) ++e;
            gEnd = G + e;
            r0n = 0;
         } else {
            gEnd = G + lastIdx;
            const int lastPrevCum = lastIdx > 0 ? __shfl_sync(0xffffffffu, cum, lastIdx - 1) : 0;
            r0n = (lastIdx == 0 ? r0 : 0) + (nb - lastPrevCum);
         }
      }
      // ---- storage, one group at a time in group order: stayers in place, in-row
      //      movers after the neighbour's stayers, off-row movers to the global list;
      //      then the exit of every finished group --------------------------------------
      const int gLoopEnd = max(gEnd, G + (nb > 0 ? lastIdx + 1 : 0));
      const unsigned below = (1u << lane) - 1u;
      for (int gg = G; gg < gLoopEnd; ++gg) {
         const int ug = gg / ns, sg = gg % ns;
         PlaceState& P = s_ps[warp][sg];
         const DStore& S = FS.st[sg];
         const long long Du = (long long)ug + (long long)ndx * row;
         const bool mine = active && myG == gg;
         const unsigned mStay = __ballot_sync(0xffffffffu, mine && cls == 0);
         const unsigned mMinus = __ballot_sync(0xffffffffu, mine && cls == 1);
         const unsigned mPlus = __ballot_sync(0xffffffffu, mine && cls == 2);
         if (mine && cls >= 0) {
            bool toSlow = cls == 3;
            int slowClass = 2;
            if (cls == 0) {
               const long long pos = S.start[Du] + P.stay + __popc(mStay & below);
               for (int a = 0; a < 7; ++a) S.a[a][pos] = st[a];
            } else if (cls == 1) {
               const int k = P.fill + __popc(mMinus & below);
               const long long pos = S.start[Du - 1] + k;
               if (!P.full && pos < S.start[Du]) {
                  for (int a = 0; a < 7; ++a) S.a[a][pos] = st[a];
               } else {
                  toSlow = true;
                  slowClass = 1;
               }
            } else if (cls == 2) {
               const int k = P.npCur + __popc(mPlus & below);
               if (k < fb.pendCap) {
                  double* pb = fb.pend + (((row * ns + sg) * 2 + (P.pendSel ^ 1)) * (long long)fb.pendCap + k) * 8;
                  for (int a = 0; a < 7; ++a) pb[a] = st[a];
                  pb[7] = (double)rank;
               } else {
                  raiseError(err, RHGPU_DEVERR_CAPACITY);
               }
            }
            if (toSlow) {
               const unsigned long long m = atomicAdd(fb.nmovers, 1ull);
               if ((long long)m < fb.moverCap) {
                  Mover& M = fb.movers[m];
                  for (int a = 0; a < 7; ++a) M.s[a] = st[a];
                  M.key = ((unsigned long long)slowClass << 62) | ((unsigned long long)Du << 24) | (unsigned long long)rank;
                  M.dest = Dn;
                  M.species = sg;
               } else {
                  raiseError(err, RHGPU_DEVERR_CAPACITY);
               }
            }
         }
         __syncwarp();
         if (lane == 0) {
            P.stay += __popc(mStay);
            const int nm = __popc(mMinus);
            if (nm) {
               // once the previous dual cell is full, its -x arrivals keep going to the slow path
               const int cap = (int)(S.start[Du] - S.start[Du - 1]);
               if (P.full || P.fill + nm > cap) { P.fill = min(P.fill + nm, cap); P.full = 1; }
               else P.fill += nm;
            }
            P.npCur += __popc(mPlus);
         }
         __syncwarp();
         if (gg >= gEnd) continue;   // the last group continues in the next batch
         // exit of group (ug, sg): the previous dual cell of this species is final
         if (ug >= 1 && lane == 0) S.cnt[Du - 1] = P.fill;
         // +x movers from ug-1 go after the stayers of ug
         const int np = P.npPrev;
         const long long base = S.start[Du] + P.stay;
         const long long capEnd = S.start[Du + 1];
         double* pb = fb.pend + (((row * ns + sg) * 2 + P.pendSel) * (long long)fb.pendCap) * 8;
         const int fit = (int)max(0LL, min((long long)np, capEnd - base));
         for (int k = lane; k < np; k += 32) {
            const double* rec = pb + (long long)k * 8;
            if (k < fit) {
               for (int a = 0; a < 7; ++a) S.a[a][base + k] = rec[a];
            } else {
               const unsigned long long m = atomicAdd(fb.nmovers, 1ull);
               if ((long long)m < fb.moverCap) {
                  Mover& M = fb.movers[m];
                  for (int a = 0; a < 7; ++a) M.s[a] = rec[a];
                  const long long Dsrc = Du - 1;
                  M.key = (1ull << 62) | ((unsigned long long)Dsrc << 24) | (unsigned long long)rec[7];
                  M.dest = Du;
                  M.species = sg;
               } else {
                  raiseError(err, RHGPU_DEVERR_CAPACITY);
               }
            }
         }
         __syncwarp();
         if (lane == 0) {
            P.fill = P.stay + fit;
            P.full = fit < np ? 1 : 0;
            P.stay = 0;
            P.npPrev = P.npCur;
            P.npCur = 0;
            P.pendSel ^= 1;
         }
         __syncwarp();
      }
      G = gEnd;
      r0 = r0n;
   }
   // ---- end of row: finalize the last dual cell of every species, flush the window -----
   if (lane < ns) {
      const PlaceState& P = s_ps[warp][lane];
      const long long Dl = (long long)(ndx - 1) + (long long)ndx * row;
      FS.st[lane].cnt[Dl] = P.fill;
   }
   slide(ndx);
   if (perx) {
      // destination 0: corner 1 of the last dual cell + corner 0 of dual cell 0
      const double partner = __shfl_xor_sync(0xffffffffu, pend, 4);
      if ((qo & 1) == 0) RP[(((long long)(qo >> 1) * nrows + row) * nx + 0) * 4 + ql] = partner + wrap0;
   }
}

// destination moments: four row partials + fixed-point part, then finalize
__global__ void k_fast_gather(GridInfo g, Fields f, FastGeom fg, FastBufs fb, double hiR, double loR, double hiJ,
                              double loJ, double minRho, unsigned long long* cnt) {
   RH_CELL_PROLOGUE
   double v[4];
   for (int qq = 0; qq < 4; ++qq) {
      const int uyy = dualU(j - (qq & 1), g.ny, g.per[1]);
      const int uzz = dualU(k - (qq >> 1), g.nz, g.per[2]);
      const long long row = (long long)uyy + (long long)fg.nd[1] * uzz;
      const double* rp = fb.RP + (((long long)qq * fg.nrows + row) * g.nx + i) * 4;
      for (int l = 0; l < 4; ++l) v[l] = qq == 0 ? rp[l] : v[l] + rp[l];
   }
   if (fb.touched[n >> 5] & (1u << (n & 31))) {
      v[0] += fixedToDouble(fb.MMlo[n], fb.MMhi[n], hiR, loR);
      for (int l = 0; l < 3; ++l) v[1 + l] += fixedToDouble(fb.MMlo[(1 + l) * N + n], fb.MMhi[(1 + l) * N + n], hiJ, loJ);
      for (int l = 0; l < 4; ++l) { fb.MMlo[l * N + n] = 0ull; fb.MMhi[l * N + n] = 0ull; }
   }
   double rho = v[0] / g.dV;
   bool clamp = false;
   if (rho < minRho) { rho = minRho; clamp = true; }
   countIf(clamp, &cnt[CNT_MIN_CELL_RHO]);
   f.cellRho[n] = rho;
   for (int l = 0; l < 3; ++l) f.cellJi[l * N + n] = v[1 + l] / g.dV;
}

// ---- off-row mover placement ------------------------------------------------------
__global__ void k_fast_mig_count(const Mover* mv, long long n, long long Nd, int* inc) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= n) return;
   atomicAdd(&inc[(long long)mv[t].species * Nd + mv[t].dest], 1);
}
__global__ void k_fast_mig_bucket(const Mover* mv, long long n, long long Nd, const long long* off, int* fill, int* bucket) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= n) return;
   const long long b = (long long)mv[t].species * Nd + mv[t].dest;
   const int k = atomicAdd(&fill[b], 1);
   bucket[off[b] + k] = (int)t;
}
// per destination (species, dual cell): arrivals sorted by key, appended after
// the in-row placements; sets *overflow and places nothing if they do not fit
__global__ void k_fast_mig_place(FastSpecies FS, long long Nd, const Mover* mv, int* inc, const long long* off,
                                 int* bucket, int* overflow) {
   const long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (b >= (long long)FS.ns * Nd) return;
   const int k = inc[b];
   if (k == 0) return;
   const int s = (int)(b / Nd);
   const long long D = b % Nd;
   int* bk = bucket + off[b];
   for (int a = 1; a < k; ++a)
      for (int c = a; c > 0 && mv[bk[c - 1]].key > mv[bk[c]].key; --c) { int t = bk[c]; bk[c] = bk[c - 1]; bk[c - 1] = t; }
   const DStore& S = FS.st[s];
   const long long base = S.start[D] + S.cnt[D];
   if (base + k > S.start[D + 1]) { atomicOr((unsigned*)overflow, 1u); return; }
   for (int a = 0; a < k; ++a) {
      const Mover& M = mv[bk[a]];
      for (int e = 0; e < 7; ++e) S.a[e][base + a] = M.s[e];
   }
   S.cnt[D] += k;
   inc[b] = 0;
}

// ---- upload / download / repack support ------------------------------------------------
// dual index of each uploaded particle (records grouped by cell)
__global__ void k_fast_dual_of(GridInfo g, FastGeom fg, const double* aos, const int* pcell, long long n, unsigned* key) {
   const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (p >= n) return;
   const int c = pcell[p];
   const int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
   const double* st = aos + 7 * p;
   const int ux = dualU(i + halfS(st[0], g.dx) - 1, g.nx, g.per[0]);
   const int uy = dualU(j + halfS(st[1], g.dx) - 1, g.ny, g.per[1]);
   const int uz = dualU(k + halfS(st[2], g.dx) - 1, g.nz, g.per[2]);
   key[p] = (unsigned)((long long)ux + (long long)fg.nd[0] * ((long long)uy + (long long)fg.nd[1] * uz));
}
__global__ void k_fast_histogram(const unsigned* key, long long n, int* cnt) {
   const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (p < n) atomicAdd(&cnt[key[p]], 1);
}
// capacity with slack: cnt + max(8, cnt/2)
__global__ void k_fast_capacity(long long Nd, const int* cnt, const int* extra, long long* cap) {
   const long long d = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (d < Nd) {
      const long long c = (long long)cnt[d] + (extra ? extra[d] : 0);
      cap[d] = c + max(8LL, c / 2);
   }
   if (d == Nd) cap[Nd] = 0;
}
// sorted particle i (dual key[i], original index idx[i]) -> slot start[D] + (i - first[D])
__global__ void k_fast_scatter_sorted(const double* aos, const unsigned* key, const unsigned* idx, long long n,
                                      const long long* first, DStore S) {
   const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= n) return;
   const unsigned D = key[i];
   const long long pos = S.start[D] + (i - first[D]);
   const double* st = aos + 7 * (long long)idx[i];
   for (int a = 0; a < 7; ++a) S.a[a][pos] = st[a];
}
// cell index and storage sequence of every stored particle (download)
__global__ void k_fast_cell_keys(GridInfo g, FastGeom fg, DStore S, const long long* seqStart, unsigned* key,
                                 unsigned long long* slot) {
   const long long D = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (D >= fg.Nd) return;
   const int ux = (int)(D % fg.nd[0]), uy = (int)((D / fg.nd[0]) % fg.nd[1]), uz = (int)(D / ((long long)fg.nd[0] * fg.nd[1]));
   const long long s0 = S.start[D], o = seqStart[D];
   for (int t = 0; t < S.cnt[D]; ++t) {
      const long long p = s0 + t;
      int i = dualB(ux, g.per[0]) + 1 - halfS(S.a[0][p], g.dx);
      int j = dualB(uy, g.per[1]) + 1 - halfS(S.a[1][p], g.dx);
      int k = dualB(uz, g.per[2]) + 1 - halfS(S.a[2][p], g.dx);
      wrapc(i, g.nx, 1); wrapc(j, g.ny, 1); wrapc(k, g.nz, 1);
      key[o + t] = (unsigned)cidx(g, i, j, k);
      slot[o + t] = (unsigned long long)p;
   }
}
__global__ void k_fast_gather_records(DStore S, const unsigned long long* slot, const unsigned* order, long long n, double* aos) {
   const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= n) return;
   const long long p = (long long)slot[order[t]];
   for (int a = 0; a < 7; ++a) aos[7 * t + a] = S.a[a][p];
}
__global__ void k_fast_repack_copy(long long Nd, DStore from, DStore to) {
   const long long D = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (D >= Nd) return;
   const long long a = from.start[D], b = to.start[D];
   const int c = from.cnt[D];
   for (int t = 0; t < c; ++t)
      for (int e = 0; e < 7; ++e) to.a[e][b + t] = from.a[e][a + t];
   to.cnt[D] = c;
}
__global__ void k_fast_max_abs_w(DStore S, long long Nd, unsigned long long* out) {
   const long long D = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (D >= Nd) return;
   double m = 0.0;
   for (int t = 0; t < S.cnt[D]; ++t) m = fmax(m, fabs(S.a[6][S.start[D] + t]));
   atomicMax(out, (unsigned long long)__double_as_longlong(m));
}
__global__ void k_fast_max_int(const long long* start, long long Nd, int* out) {
   const long long D = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (D < Nd) atomicMax(out, (int)(start[D + 1] - start[D]));
}

}  // namespace rh
