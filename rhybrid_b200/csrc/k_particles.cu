// Definitions of the kernels declared in k_particles.cuh (each declaration there says
// what its kernel does); the template kernels stay in the header.
#include "k_particles.cuh"

namespace rh {

__global__ void k_push(GridInfo g, Fields f, PStore P, SpeciesDev sp, PushParams pp, int* key,
                       unsigned long long* cnt, double* cntd, unsigned* err, int sidx) {
   const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (p >= P.nslots) return;
   const int c = P.pcell[p];
   if (c < 0) { key[p] = -1; return; }
   const long long N = g.N;
   const int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
   double x = P.a[0][p], y = P.a[1][p], z = P.a[2][p];
   double vx = P.a[3][p], vy = P.a[4][p], vz = P.a[5][p];
   bool clamp = false;
   const bool accelerate = sp.accelerate && !pp.useIFT && allNb(g, i, j, k);
   if (accelerate) {
      const double dx = g.dx;
      double B[3], Ue[3], E[3];
      {
         const double xs = x / dx, ys = y / dx, zs = z / dx;
         // positions in [0,dx) give floor()==0 (see oracle: the quotient never rounds up to 1)
         const double w111x = xs - 0.0, w111y = ys - 0.0, w111z = zs - 0.0;
         const double w011x = 1.0 - xs, w101y = 1.0 - ys, w110z = 1.0 - zs;
         B[0] = w111x * f.faceB[0 * N + c] + w011x * f.faceB[0 * N + nbr(g, i, j, k, -1, 0, 0)];
         B[1] = w111y * f.faceB[1 * N + c] + w101y * f.faceB[1 * N + nbr(g, i, j, k, 0, -1, 0)];
         B[2] = w111z * f.faceB[2 * N + c] + w110z * f.faceB[2 * N + nbr(g, i, j, k, 0, 0, -1)];
      }
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
         const double xg = x + blockOrigin(g.x_min, i, dx), yg = y + blockOrigin(g.y_min, j, dx),
                      zg = z + blockOrigin(g.z_min, k, dx);
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
   countIf(clamp, &cnt[CNT_SPECIES_MAXVI + sidx]);
   gridCountAtomic(f, GC_CELL_MAX_VI, g.N, c, clamp);
   x += g.dt * vx;
   y += g.dt * vy;
   z += g.dt * vz;
   if (isnan(x) || isnan(y) || isnan(z)) raiseError(err, RHGPU_DEVERR_NAN_PARTICLE);
   int ox, oy, oz;
   int st = migrateAxis(x, ox, g.dx, g.dx_below);
   st |= migrateAxis(y, oy, g.dx, g.dx_below);
   st |= migrateAxis(z, oz, g.dx, g.dx_below);
   int ti = i + ox, tj = j + oy, tk = k + oz;
   const bool inside = wrapc(ti, g.nx, g.per[0]) && wrapc(tj, g.ny, g.per[1]) && wrapc(tk, g.nz, g.per[2]);
   P.a[0][p] = x; P.a[1][p] = y; P.a[2][p] = z;
   P.a[3][p] = vx; P.a[4][p] = vy; P.a[5][p] = vz;
   if (st || !inside) {
      const double w = P.a[6][p];
      atomicAdd(&cntd[4 * sidx + 0], w);
      atomicAdd(&cntd[4 * sidx + 1], w * (sq(vx) + sq(vy) + sq(vz)));
      key[p] = -1;
      return;
   }
   const long long d = cidx(g, ti, tj, tk);
   key[p] = (int)(d * 27 + dirRank(dirFromOffset(-ox, -oy, -oz)));
}

__global__ void k_mig_count(GridInfo g, PStore P, const int* key, int* outCount, int* rank) {
   const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (c >= g.N) return;
   int run[27];
   for (int r = 0; r < 27; ++r) run[r] = 0;
   const long long a = P.start[c], e = P.start[c + 1];
   for (long long p = a; p < e; ++p) {
      const int kk = key[p];
      if (kk < 0) continue;
      const int r = kk % 27;
      rank[p] = run[r]++;
   }
   for (int r = 0; r < 27; ++r) outCount[(long long)r * g.N + c] = run[r];
}

__global__ void k_mig_incount(GridInfo g, const int* outCount, int* inPrefix, long long* newCount) {
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   const int j = blockIdx.y * blockDim.y + threadIdx.y;
   const int k = blockIdx.z;
   if (i >= g.nx || j >= g.ny) return;
   const long long d = cidx(g, i, j, k);
   int run = 0;
   for (int r = 0; r < 27; ++r) {
      const int dir = rankToDir(r);
      const int sx = dir % 3 - 1, sy = (dir / 3) % 3 - 1, sz = dir / 9 - 1;
      const long long s = nbr(g, i, j, k, sx, sy, sz);
      inPrefix[(long long)r * g.N + d] = run;
      if (s >= 0) run += outCount[(long long)r * g.N + s];
   }
   newCount[d] = run;
}

__global__ void k_mig_scatter(GridInfo g, PStore P, PStore Q, const int* key, const int* rank,
                              const int* inPrefix, const long long* newStart, unsigned* err) {
   const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (p >= P.nslots) return;
   const int kk = key[p];
   if (kk < 0) return;
   const long long d = kk / 27;
   const int r = kk % 27;
   const long long pos = newStart[d] + inPrefix[(long long)r * g.N + d] + rank[p];
   if (pos < 0 || pos >= Q.cap) { raiseError(err, RHGPU_DEVERR_CAPACITY); return; }
   for (int a = 0; a < 7; ++a) Q.a[a][pos] = P.a[a][p];
   Q.pcell[pos] = (int)d;
}

__global__ void k_set_alive_from_count(long long N, const long long* cnt, int* alive) {
   const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
   if (c < N) alive[c] = (int)cnt[c];
}

__global__ void __launch_bounds__(32 * DEP_WARPS, 4) k_deposit_cell(GridInfo g, PStore P, double q, double* S, unsigned* err) {
   __shared__ double sw[DEP_WARPS][32][11];                // w8[0..7], v[0..2] of a batch's particles
   __shared__ int soct[DEP_WARPS][32];                     // octant (i + 2j + 4k) of the corner-000 entry, 8 if invalid
   __shared__ double stage[DEP_WARPS][DEP_ENTRIES + 1];    // the group's sums, per cell
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   // per entry t: its value (-1 charge, 0..2 current) and its corner map,
   // nibble o = the corner of a particle of octant o landing on the entry, 8
   // for none (nibble 8: a particle without a valid octant)
   unsigned long long cmap[4];
   int el[4];
   const int ne = lane < 12 ? 4 : 3;
#pragma unroll
   for (int t = 0; t < 4; ++t) {
      const int e = lane + 32 * t;
      int ind, l;
      if (e < 27) { ind = e; l = -1; } else { ind = (e - 27) / 3; l = (e - 27) % 3; }
      const int ea = ind % 3, eb = (ind / 3) % 3, ec = ind / 9;
      unsigned long long m = 8ull << 32;
      for (int o = 0; o < 8; ++o) {
         const int ox = ea - (o & 1), oy = eb - ((o >> 1) & 1), oz = ec - (o >> 2);
         const bool on = (unsigned)ox <= 1u && (unsigned)oy <= 1u && (unsigned)oz <= 1u;
         m |= (unsigned long long)(on ? ox + 2 * oy + 4 * oz : 8) << (4 * o);
      }
      cmap[t] = m;
      el[t] = l;
   }
   const long long groups = (g.N + DEP_WARPS - 1) / DEP_WARPS;
   for (long long grp = blockIdx.x; grp < groups; grp += gridDim.x) {
      const long long c = grp * DEP_WARPS + warp;
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      if (c < g.N) {
         const long long a0 = P.start[c];
         const int na = P.alive[c];
         for (int b0 = 0; b0 < na; b0 += 32) {
            const int nb = min(32, na - b0);
            if (lane < nb) {
               const long long p = a0 + b0 + lane;
               const double x = P.a[0][p], y = P.a[1][p], z = P.a[2][p];
               const double wq = P.a[6][p] * q;
               double w8[8];
               int ind[8];
               cicWeights(x, y, z, wq, g, w8, ind);
               int oct = 8;
               const int i0 = ind[0] % 3, j0 = (ind[0] / 3) % 3, k0 = ind[0] / 9;
               if (ind[0] >= 0 && ind[0] < 27 && i0 <= 1 && j0 <= 1 && k0 <= 1) oct = i0 + 2 * j0 + 4 * k0;
               else raiseError(err, RHGPU_DEVERR_NAN_PARTICLE);
#pragma unroll
               for (int o = 0; o < 8; ++o) sw[warp][lane][o] = w8[o];
               sw[warp][lane][8] = P.a[3][p];
               sw[warp][lane][9] = P.a[4][p];
               sw[warp][lane][10] = P.a[5][p];
               soct[warp][lane] = oct;
            }
            __syncwarp();
#pragma unroll 2
            for (int j = 0; j < nb; ++j) {
               const int sh = 4 * soct[warp][j];
               const double* r = sw[warp][j];
#pragma unroll
               for (int t = 0; t < 4; ++t) {
                  if (t >= ne) break;
                  const unsigned corner = (unsigned)(cmap[t] >> sh) & 15u;
                  const double w = r[corner & 7u];
                  const double v = el[t] < 0 ? w : w * r[8 + (el[t] < 0 ? 0 : el[t])];
                  acc[t] += corner < 8u ? v : 0.0;
               }
            }
            __syncwarp();
         }
      }
#pragma unroll
      for (int t = 0; t < 4; ++t)
         if (t < ne) stage[warp][lane + 32 * t] = acc[t];
      __syncthreads();
      for (int idx = threadIdx.x; idx < DEP_ENTRIES * DEP_WARPS; idx += 32 * DEP_WARPS) {
         const int e = idx / DEP_WARPS, w = idx - e * DEP_WARPS;
         const long long cc = grp * DEP_WARPS + w;
         if (cc < g.N) S[(long long)e * g.N + cc] = stage[w][e];
      }
      __syncthreads();
   }
}

__global__ void k_deposit_gather(GridInfo g, Fields f, const double* S, int first, int last, double minRho,
                                 unsigned long long* cnt) {
   RH_CELL_PROLOGUE
   const Sources3 Q = sortedSources(g, i, j, k);
   double v[4];
   v[0] = first ? 0.0 : f.cellRho[n];
   for (int l = 0; l < 3; ++l) v[1 + l] = first ? 0.0 : f.cellJi[l * N + n];
   addSources(g, Q, S, N, v);
   double rho = v[0], J0 = v[1], J1 = v[2], J2 = v[3];
   bool clamp = false;
   if (last) {
      rho /= g.dV;
      if (rho < minRho) { rho = minRho; clamp = true; }
      J0 /= g.dV; J1 /= g.dV; J2 /= g.dV;
   }
   countIf(clamp, &cnt[CNT_MIN_CELL_RHO]);
   gridCount(f, GC_CELL_MIN_RHOQI, N, n, clamp);
   f.cellRho[n] = rho;
   f.cellJi[0 * N + n] = J0;
   f.cellJi[1 * N + n] = J1;
   f.cellJi[2 * N + n] = J2;
}

__global__ void k_deposit_finalize_only(GridInfo g, Fields f, double minRho, unsigned long long* cnt) {
   RH_CELL_PROLOGUE
   double rho = 0.0 / g.dV;
   bool clamp = false;
   if (rho < minRho) { rho = minRho; clamp = true; }
   countIf(clamp, &cnt[CNT_MIN_CELL_RHO]);
   gridCount(f, GC_CELL_MIN_RHOQI, N, n, clamp);
   f.cellRho[n] = rho;
   for (int l = 0; l < 3; ++l) f.cellJi[l * N + n] = 0.0 / g.dV;
}

__global__ void k_bc_exterior(GridInfo g, PStore P, const int* ext, int next, double* cntd, int sidx) {
   const int e = blockIdx.x * blockDim.x + threadIdx.x;
   if (e >= next) return;
   const int c = ext[e];
   const long long a = P.start[c];
   const int na = P.alive[c];
   double sw = 0.0, se = 0.0;
   for (int t = 0; t < na; ++t) {
      const long long p = a + t;
      const double w = P.a[6][p];
      sw += w;
      se += w * (sq(P.a[3][p]) + sq(P.a[4][p]) + sq(P.a[5][p]));
      P.pcell[p] = -1;
   }
   if (na > 0) {
      atomicAdd(&cntd[4 * sidx + 0], sw);
      atomicAdd(&cntd[4 * sidx + 1], se);
   }
   P.alive[c] = 0;
}

__global__ void k_bc_obstacle(GridInfo g, PStore P, const int* cells, int ncells, double R2, double* cntd, int sidx) {
   const int e = blockIdx.x * blockDim.x + threadIdx.x;
   if (e >= ncells) return;
   const int c = cells[e];
   const int i = c % g.nx, j = (c / g.nx) % g.ny, k = c / (g.nx * g.ny);
   const double xB = blockOrigin(g.x_min, i, g.dx), yB = blockOrigin(g.y_min, j, g.dx), zB = blockOrigin(g.z_min, k, g.dx);
   const long long a = P.start[c];
   int cur = 0, end = P.alive[c] - 1;
   double sw = 0.0, se = 0.0;
   while (cur <= end) {
      const long long p = a + cur;
      const double xp = xB + P.a[0][p], yp = yB + P.a[1][p], zp = zB + P.a[2][p];
      const double r2 = sq(xp) + sq(yp) + sq(zp);
      if (r2 < R2) {
         const double w = P.a[6][p];
         sw += w;
         se += w * (sq(P.a[3][p]) + sq(P.a[4][p]) + sq(P.a[5][p]));
         const long long q = a + end;
         for (int s = 0; s < 7; ++s) P.a[s][p] = P.a[s][q];
         --end;
         continue;
      }
      ++cur;
   }
   for (int t = cur; t < P.alive[c]; ++t) P.pcell[a + t] = -1;
   if (sw != 0.0 || se != 0.0) {
      atomicAdd(&cntd[4 * sidx + 2], sw);
      atomicAdd(&cntd[4 * sidx + 3], se);
   }
   P.alive[c] = cur;
}

}  // namespace rh
