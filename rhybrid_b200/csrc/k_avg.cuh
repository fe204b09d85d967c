// Temporal averages of the output populations (WRITE_GRID_TEMPORAL_AVERAGES,
// the reference's default build):
//   every step, each accumulating species adds its CIC charge and current sums
//   (before /dV) to the sums of its output population
//     (particle_accumulator.cpp:148-150, 208-215)
//   at an output step, n_<pop>_ave = sum / (q dV) / count, v_<pop>_ave =
//   current sum / charge sum, cellBAverage = sum / count, and the sums restart
//     (operator_userdata.cpp:155-223)
//
//   k_deposit_gather_avg   exact path: one species' 27 per-source sums added to
//                          its population's sums in the reference's order
//   fast path, right after the step's deposit (the same particles it deposits):
//   k_fast_avg_deposit     one block per row segment over the population's
//                          species' particles that stayed in their segment:
//                          CIC records counting-sorted by dual cell and summed
//                          per (dual cell, corner) as the push kernel does,
//                          out as row partials
//   k_fast_avg_movers      the population's deposits that went through the
//                          mover list (left their segment; or deposited in it
//                          and then removed by a boundary), as exact
//                          fixed-point sums
//   k_fast_avg_gather      per cell, row partials + fixed-point part added to
//                          the sums
//   k_avg_output           the output step's normalisation and restart
#pragma once

#include "rh_device.cuh"
#include "k_particles.cuh"
#include "k_fast.cuh"

namespace rh {

// exact path: v_sum of cell n += this species' contributions, sources in ID order
__global__ void k_deposit_gather_avg(GridInfo g, const double* S, double* nSum, double* vSum);

// fast path: the CIC sums of the species in `mask` (bit s) over the particles of
// FS.st[s].cur (the step's stayers), as row partials in fb.RP / fb.RPB
template <int PER>
__global__ void __launch_bounds__(FT, 4)
k_fast_avg_deposit(GridInfo gIn, FastGeom fg, FastSpecies FS, unsigned mask, FastBufs fb) {
   GridInfo g = gIn;
   g.per[0] = PER & 1;
   g.per[1] = (PER >> 1) & 1;
   g.per[2] = (PER >> 2) & 1;
   __shared__ double s_rec[FT * REC];
   __shared__ int s_wd[FW][SEG];
   __shared__ int s_prefix[FAST_MAX_SPECIES + 1];
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
   const unsigned below = (1u << lane) - 1u;
   const long long S = blockIdx.x;
   const long long row = S / fg.nseg;
   const int gseg = (int)(S % fg.nseg);
   const int u0 = gseg * SEG, u1 = min(u0 + SEG, fg.nd[0]);
   const int ns = FS.ns;
   if (tid == 0) {
      int a = 0;
      for (int s = 0; s < ns; ++s) {
         s_prefix[s] = a;
         if ((mask >> s) & 1u) a += FS.st[s].cur.cnt[S];
      }
      s_prefix[ns] = a;
   }
   __syncthreads();
   const int total = s_prefix[ns];
   const int myDual = tid >> 3, myCorner = tid & 7;
   double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
   for (int c0 = 0; c0 < total; c0 += FT) {
      const int i = c0 + tid;
      const bool rec = i < total;
      int s = 0;
      if (rec)
         while (s + 1 < ns && i >= s_prefix[s + 1]) ++s;
      double st[7];
      int rd = 0;
      if (rec) {
         const SegSpecies& SS = FS.st[s];
         const long long slot = SS.base[S] + (i - s_prefix[s]);
         for (int a = 0; a < 7; ++a) st[a] = SS.cur.a[a][slot];
         rd = SS.cur.lx[slot];
      }
      // records counting-sorted by dual cell: chunk, warp, lane order within a dual cell
      const unsigned br = __ballot_sync(0xffffffffu, rec);
      s_wd[warp][lane] = 0;
      __syncwarp();
      int rrank = 0;
      if (rec) {
         const unsigned mm = __match_any_sync(br, rd);
         rrank = __popc(mm & below);
         if (rrank == 0) s_wd[warp][rd] = __popc(mm);
      }
      __syncthreads();
      int binD, offD, tot;
      {
         int t = 0, before = 0;
#pragma unroll
         for (int w = 0; w < FW; ++w) {
            const int cw = s_wd[w][lane];
            t += cw;
            if (w < warp) before += cw;
         }
         int x = t;
         for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
         }
         binD = x - t;
         offD = binD + before;
         tot = __shfl_sync(0xffffffffu, x, 31);
      }
      const int recPos = __shfl_sync(0xffffffffu, offD, rd) + rrank;
      const int sumLo = __shfl_sync(0xffffffffu, binD, myDual);
      const int sumHiN = __shfl_sync(0xffffffffu, binD, (myDual + 1) & 31);
      const int sumHi = myDual == SEG - 1 ? tot : sumHiN;
      if (rec) {
         double w8[8];
         cicWeightsLocal(st[0], st[1], st[2], st[6] * FS.sp[s].q, g, w8);
         double* r = s_rec + recPos * REC;
         for (int o = 0; o < 8; ++o) r[o] = w8[o];
         r[8] = st[3]; r[9] = st[4]; r[10] = st[5];
      }
      __syncthreads();
#pragma unroll 2
      for (int r = sumLo; r < sumHi; ++r) {
         const double* rr = s_rec + r * REC;
         const double w = rr[myCorner];
         a0 += w;
         a1 += w * rr[8];
         a2 += w * rr[9];
         a3 += w * rr[10];
      }
      // the next chunk's first barrier orders these reads before its record writes
   }
   __syncthreads();
   segPartialsOut(g, fg, fb, s_rec, row, gseg, u0, u1, a0, a1, a2, a3);
}

// fast path: the movers of the species in `mask` that were deposited this step
__global__ void k_fast_avg_movers(GridInfo g, FastGeom fg, FastSpecies FS, const Mover* mv, long long n, unsigned mask,
                                  FastBufs fb);

// fast path: row partials + fixed-point part added to the population's sums;
// the fixed-point sums restart
__global__ void k_fast_avg_gather(GridInfo g, FastGeom fg, FastBufs fb, double hiR, double loR, double hiJ, double loJ,
                                  double* nSum, double* vSum);

// output step of one population (operator_userdata.cpp:182-211): n = sum/(q dV)*inv,
// v = current sum / charge sum where the charge sum is positive, else 0; the sums
// restart. Outputs interleaved per cell (ParGrid order), as the ABI's arrays.
__global__ void k_avg_output(long long N, double* nSum, double* vSum, double q, double dV, double inv, double* nOut,
                             double* vOut);

// cellBAverage = cellAverageB * inv, and the sum restarts (operator_userdata.cpp:162-176)
__global__ void k_avgB_output(long long N, double* sumB, double inv, double* out);

}  // namespace rh
