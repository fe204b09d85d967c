// Particle kernels of the bit-exact path (sm_100a, FP64):
//   k_push            BorisBuneman::propagate + getFields (particle_propagator_boris_buneman.h:64-194,
//                     hybrid_propagator.cpp:1740-1891) and the migration decision
//   k_mig_count / k_mig_incount / k_mig_scatter
//                     stable counting sort of the particles into their new cells
//   k_deposit_cell    Accumulator::accumulateCell (particle_accumulator.cpp:44-156): per cell, the
//                     3x3x3 CIC sums in particle order
//   k_deposit_gather  block::addValues3D in increasing source-cell order + finalize (:319-333)
//   k_bc_exterior / k_bc_obstacle   ParticleBoundaryCondHybrid::apply (particle_boundary_cond_hybrid.h:112-185)
// Particle storage per species, structure of arrays in HBM (7 doubles), grouped
// by cell: cell c owns slots [start[c], start[c+1]); the first alive[c] of them
// hold particles, pcell[p] is the cell of slot p or -1 for an empty slot.
#pragma once

#include "rh_device.cuh"
#include "k_fields.cuh"

namespace rh {

struct PStore {
   double* a[7];        // x, y, z (cell-local), vx, vy, vz, weight
   int* pcell;          // cell of each slot, -1 if empty
   long long* start;    // N+1 slot offsets
   int* alive;          // alive particles per cell (a prefix of its slots)
   long long nslots;
   long long cap;
};

struct SpeciesDev {
   double q, m, R2obs, qmideltT2;
   int accelerate, accumulate;
};

struct PushParams {
   int useIFT, use_ep, use_gravity;
   double GMdt, maxVi2;
   int avgList;   // fast path, EXTRA variant: list the removed in-segment deposits for the population averages
};

// device error word bits
__device__ inline void raiseError(unsigned* err, unsigned bit) { atomicOr(err, bit); }

__global__ void k_push(GridInfo g, Fields f, PStore P, SpeciesDev sp, PushParams pp, int* key,
                       unsigned long long* cnt, double* cntd, unsigned* err, int sidx);

// per source cell: counts per destination-direction rank, and the rank of
// each particle inside its (source, direction) group
__global__ void k_mig_count(GridInfo g, PStore P, const int* key, int* outCount, int* rank);

// per destination cell: arrivals per direction rank (exclusive prefix) and total
__global__ void k_mig_incount(GridInfo g, const int* outCount, int* inPrefix, long long* newCount);

__global__ void k_mig_scatter(GridInfo g, PStore P, PStore Q, const int* key, const int* rank,
                              const int* inPrefix, const long long* newStart, unsigned* err);

__global__ void k_set_alive_from_count(long long N, const long long* cnt, int* alive);

// CIC weights of one particle (particle_accumulator.cpp:68-110), corners in
// the order 000,100,010,110,001,101,011,111 with their 3x3x3 indices; the
// divisions by dx are divDx, the same correctly rounded quotients
__device__ inline void cicWeights(double x, double y, double z, double wq, const GridInfo& g, double w8[8],
                                  int ind[8]) {
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
   for (int o = 0; o < 8; ++o) {
      const int a = i + (o & 1), b = j + ((o >> 1) & 1), cc = k + ((o >> 2) & 1);
      ind[o] = a + 3 * (b + 3 * cc);
   }
}

// Per cell, the 3x3x3 CIC sums of accumulateCell in particle order, one warp
// per cell: lane L owns the accumulator entries e = L, L+32, L+64, L+96
// (e < 27: charge of 3x3x3 entry e; e = 27 + 3*entry + l: current l). The
// particles of the cell are taken 32 at a time, each lane computing one
// particle's CIC weights into shared memory; then every lane walks those
// particles in order and adds the contribution that falls on its entries, so
// each entry is the same sequential sum as in the reference. Each entry keeps
// a map from the particle's octant (the 3x3x3 index of its corner 000 is one
// of the 8 of {0,1}^3) to the corner landing on the entry, or none; an entry
// no corner lands on adds +0.0, which leaves every sum unchanged (a sum that
// starts at +0.0 is never -0.0, so x + 0.0 == x for each of its values), so
// the walk has no branches and each sum is still the reference's sequence.
// S[e*N + c] receives the 108 sums of cell c. A block takes DEP_WARPS
// consecutive cells at a time (one per warp) and writes their sums row by row
// through shared memory, DEP_WARPS cells contiguous per row; the blocks, one
// resident wave of DEP_GRID, stride over the groups of cells, so each warp
// builds its corner maps once.
constexpr int DEP_WARPS = 8;
constexpr int DEP_ENTRIES = 108;
constexpr int DEP_GRID = 148 * 4;   // 4 blocks of 256 threads at 64 registers per SM
__global__ void __launch_bounds__(32 * DEP_WARPS, 4) k_deposit_cell(GridInfo g, PStore P, double q, double* S, unsigned* err);

// destination sums over the 27 source cells in increasing source index
// The up to 3 source coordinates per axis of the 27-neighbourhood of cell
// (i,j,k), each with its offset source - destination, in increasing coordinate:
// looping z, y, x over them visits the sources in increasing cell ID, the order
// in which addValues3D reaches the destination when cells are accumulated in ID
// order.
struct Sources3 {
   int c[3][3], o[3][3], n[3];
};
__device__ inline Sources3 sortedSources(const GridInfo& g, int i, int j, int k) {
   Sources3 Q;
   const int at[3] = {i, j, k}, nn[3] = {g.nx, g.ny, g.nz};
   for (int a = 0; a < 3; ++a) {
      Q.n[a] = 0;
      for (int d = -1; d <= 1; ++d) {
         int x = at[a] + d;
         if (wrapc(x, nn[a], g.per[a])) { Q.c[a][Q.n[a]] = x; Q.o[a][Q.n[a]] = d; ++Q.n[a]; }
      }
      for (int u = 1; u < Q.n[a]; ++u)
         for (int w = u; w > 0 && Q.c[a][w - 1] > Q.c[a][w]; --w) {
            const int t1 = Q.c[a][w]; Q.c[a][w] = Q.c[a][w - 1]; Q.c[a][w - 1] = t1;
            const int t2 = Q.o[a][w]; Q.o[a][w] = Q.o[a][w - 1]; Q.o[a][w - 1] = t2;
         }
   }
   return Q;
}

// adds the 27 per-source contributions of one species' sums S to cell n, in
// the sources' ID order, onto v[0..3] (rho, Ji)
__device__ inline void addSources(const GridInfo& g, const Sources3& Q, const double* S, long long N, double v[4]) {
   for (int c3 = 0; c3 < Q.n[2]; ++c3)
      for (int b3 = 0; b3 < Q.n[1]; ++b3)
         for (int a3 = 0; a3 < Q.n[0]; ++a3) {
            const long long s = cidx(g, Q.c[0][a3], Q.c[1][b3], Q.c[2][c3]);
            // destination seen from the source: offset -o, array index -o+1
            const int e = (1 - Q.o[0][a3]) + 3 * ((1 - Q.o[1][b3]) + 3 * (1 - Q.o[2][c3]));
            v[0] += S[(long long)e * N + s];
            v[1] += S[(long long)(27 + 3 * e + 0) * N + s];
            v[2] += S[(long long)(27 + 3 * e + 1) * N + s];
            v[3] += S[(long long)(27 + 3 * e + 2) * N + s];
         }
}

__global__ void k_deposit_gather(GridInfo g, Fields f, const double* S, int first, int last, double minRho,
                                 unsigned long long* cnt);

// finalize without deposit (no accumulating species): rho = 0/dV clamped
__global__ void k_deposit_finalize_only(GridInfo g, Fields f, double minRho, unsigned long long* cnt);

__global__ void k_bc_exterior(GridInfo g, PStore P, const int* ext, int next, double* cntd, int sidx);

// swap-remove of particles inside the obstacle, in the reference's order
__global__ void k_bc_obstacle(GridInfo g, PStore P, const int* cells, int ncells, double R2, double* cntd, int sidx);

}  // namespace rh
