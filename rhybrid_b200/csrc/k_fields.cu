// Definitions of the kernels declared in k_fields.cuh (each declaration there says
// what its kernel does); the template kernels stay in the header.
#include "k_fields.cuh"

namespace rh {

__constant__ NeumannTables c_neu;

cudaError_t setNeumannTables(const NeumannTables& t) { return cudaMemcpyToSymbol(c_neu, &t, sizeof t); }

#define RH_C2N(dst, src, off)                                                                  \
   dst[off + n] = 0.125 * (src[off + c000] + src[off + c001] + src[off + c010] + src[off + c100] + \
                           src[off + c011] + src[off + c110] + src[off + c101] + src[off + c111]);

__global__ void k_face2cell(GridInfo g, Fields f) {
   RH_CELL_PROLOGUE
   if (!allNb(g, i, j, k)) return;
   const double* fb = f.faceB;
   f.cellB[0 * N + n] = 0.5 * (fb[0 * N + n] + fb[0 * N + nbr(g, i, j, k, -1, 0, 0)]);
   f.cellB[1 * N + n] = 0.5 * (fb[1 * N + n] + fb[1 * N + nbr(g, i, j, k, 0, -1, 0)]);
   f.cellB[2 * N + n] = 0.5 * (fb[2 * N + n] + fb[2 * N + nbr(g, i, j, k, 0, 0, -1)]);
}

__global__ void k_ext_cell_neumann3(GridInfo g, double* a, const int* ext, int next) {
   const int e = blockIdx.x * blockDim.x + threadIdx.x;
   if (e >= next) return;
   const int c = ext[e];
   int i, j, k;
   extCellIJK(g, c, i, j, k);
   const long long N = g.N, n = c;
   const int m = missingMask(g, i, j, k);
   const signed char* o = c_neu.cellSrc[m];
   const long long s = nbr(g, i, j, k, o[0], o[1], o[2]);
   if (s < 0) return;
   for (int l = 0; l < 3; ++l) a[l * N + n] = a[l * N + s];
}

__global__ void k_cell2node3(GridInfo g, const double* src, double* dst) {
   RH_CELL_PROLOGUE
   if (!plusOk(g, i, j, k)) return;
   const long long c000 = n, c001 = nbr(g, i, j, k, 0, 0, 1), c010 = nbr(g, i, j, k, 0, 1, 0),
                   c100 = nbr(g, i, j, k, 1, 0, 0), c011 = nbr(g, i, j, k, 0, 1, 1),
                   c110 = nbr(g, i, j, k, 1, 1, 0), c101 = nbr(g, i, j, k, 1, 0, 1),
                   c111 = nbr(g, i, j, k, 1, 1, 1);
   for (int l = 0; l < 3; ++l) { RH_C2N(dst, src, l * N) }
}
#undef RH_C2N

__global__ void k_node2cell3(GridInfo g, const double* src, double* dst) {
   RH_CELL_PROLOGUE
   if (!allNb(g, i, j, k)) return;
   const long long a0 = n, a1 = nbr(g, i, j, k, -1, 0, 0), a2 = nbr(g, i, j, k, -1, -1, 0),
                   a3 = nbr(g, i, j, k, 0, -1, 0), a4 = nbr(g, i, j, k, 0, 0, -1),
                   a5 = nbr(g, i, j, k, 0, -1, -1), a6 = nbr(g, i, j, k, -1, 0, -1),
                   a7 = nbr(g, i, j, k, -1, -1, -1);
   for (int l = 0; l < 3; ++l) {
      const long long o = l * N;
      dst[o + n] = 0.125 * (src[o + a0] + src[o + a1] + src[o + a2] + src[o + a3] + src[o + a4] +
                            src[o + a5] + src[o + a6] + src[o + a7]);
   }
}

__global__ void k_node_avg(GridInfo g, const double* old, double* out, FieldParams fp) {
   RH_CELL_PROLOGUE
   if (!plusOk(g, i, j, k)) return;
   const signed char ORD[27][3] = {
      {1,1,1},{1,1,0},{0,1,1},{1,2,1},{2,1,1},{1,0,1},{1,1,2},{0,1,0},{1,0,0},{1,2,0},{2,1,0},
      {0,0,1},{0,2,1},{2,2,1},{2,0,1},{0,1,2},{1,2,2},{2,1,2},{1,0,2},{0,0,2},{0,2,2},{2,0,2},
      {2,2,2},{0,0,0},{0,2,0},{2,0,0},{2,2,0}};
   const double initVal = 1.7976931348623157e308;
   for (int l = 0; l < 3; ++l) {
      double v[27], C[27];
      bool zeroFound = false;
      for (int q = 0; q < 27; ++q) {
         const int X = ORD[q][0], Y = ORD[q][1], Z = ORD[q][2];
         const long long s = nbr(g, i, j, k, X - 1, Y - 1, Z - 1);
         double val;
         if (s >= 0) val = old[l * N + s];
         else val = (X == 0 && Y == 0 && Z == 0 && l == 0) ? initVal : 0.0;
         const int dist = (X != 1) + (Y != 1) + (Z != 1);
         double Cq = fp.gauss[dist];
         if (val == initVal) { val = 0.0; Cq = 0.0; zeroFound = true; }
         v[q] = val; C[q] = Cq;
      }
      if (zeroFound) {
         double Cs = C[0];
         for (int q = 1; q < 27; ++q) Cs += C[q];
         if (Cs > 0.0) for (int q = 0; q < 27; ++q) C[q] /= Cs;
      }
      double s = C[0] * v[0];
      for (int q = 1; q < 27; ++q) s += C[q] * v[q];
      out[l * N + n] = s;
   }
}

__global__ void k_faraday(GridInfo g, Fields f) {
   RH_CELL_PROLOGUE
   bool doX = true, doY = true, doZ = true;
   if (!allNb(g, i, j, k)) {
      if (!plusOk(g, i, j, k)) return;
      if (!xNeg(g, i)) { doY = doZ = false; }
      if (!yNeg(g, j)) { doX = doZ = false; }
      if (!zNeg(g, k)) { doX = doY = false; }
   }
   const double* E = f.nodeE;
   const double dx = g.dx, dt = g.dt;
   if (doX) {
      const long long s5 = nbr(g, i, j, k, 0, -1, 0), s6 = nbr(g, i, j, k, 0, -1, -1), s7 = nbr(g, i, j, k, 0, 0, -1);
      const double n5y = E[1 * N + s5], n5z = E[2 * N + s5], n6y = E[1 * N + s6], n6z = E[2 * N + s6];
      const double n7y = E[1 * N + s7], n7z = E[2 * N + s7], n8y = E[1 * N + n], n8z = E[2 * N + n];
      const double curlX = 0.5 * (+n5z + n6z - n6y - n7y - n7z - n8z + n8y + n5y) / dx;
      f.faceB[0 * N + n] += dt * curlX;
   }
   if (doY) {
      const long long s3 = nbr(g, i, j, k, -1, 0, -1), s4 = nbr(g, i, j, k, -1, 0, 0), s7 = nbr(g, i, j, k, 0, 0, -1);
      const double n3x = E[0 * N + s3], n3z = E[2 * N + s3], n4x = E[0 * N + s4], n4z = E[2 * N + s4];
      const double n7x = E[0 * N + s7], n7z = E[2 * N + s7], n8x = E[0 * N + n], n8z = E[2 * N + n];
      const double curlY = 0.5 * (-n4x - n8x + n8z + n7z + n7x + n3x - n3z - n4z) / dx;
      f.faceB[1 * N + n] += dt * curlY;
   }
   if (doZ) {
      const long long s1 = nbr(g, i, j, k, -1, -1, 0), s4 = nbr(g, i, j, k, -1, 0, 0), s5 = nbr(g, i, j, k, 0, -1, 0);
      const double n1x = E[0 * N + s1], n1y = E[1 * N + s1], n4x = E[0 * N + s4], n4y = E[1 * N + s4];
      const double n5x = E[0 * N + s5], n5y = E[1 * N + s5], n8x = E[0 * N + n], n8y = E[1 * N + n];
      const double curlZ = 0.5 * (-n1x - n5x - n5y - n8y + n8x + n4x + n4y + n1y) / dx;
      f.faceB[2 * N + n] += dt * curlZ;
   }
}

__global__ void k_ext_bc(GridInfo g, Fields f, FieldParams fp, const int* ext, int next) {
   const int e = blockIdx.x * blockDim.x + threadIdx.x;
   if (e >= next) return;
   const int c = ext[e];
   int i, j, k;
   extCellIJK(g, c, i, j, k);
   const long long N = g.N, n = c;
   const int m = missingMask(g, i, j, k);
   const int wall[6] = {32, 1, 2, 4, 8, 16};  // +x -x +y -y +z -z
   {  // neumannCell(cellB, 3), neumannCell(cellJi, 3), neumannCell(cellRhoQi, 1), setIMFCell
      const signed char* o = c_neu.cellSrc[m];
      const long long s = nbr(g, i, j, k, o[0], o[1], o[2]);
      if (s >= 0) {
         for (int l = 0; l < 3; ++l) f.cellB[l * N + n] = f.cellB[l * N + s];
         for (int l = 0; l < 3; ++l) f.cellJi[l * N + n] = f.cellJi[l * N + s];
         f.cellRho[n] = f.cellRho[s];
      }
      for (int w = 0; w < 6; ++w)
         if ((m & wall[w]) && fp.imfCell[w])
            for (int l = 0; l < 3; ++l) f.cellB[l * N + n] = fp.imf[l];
   }
   {  // neumannFace(faceB), setIMFFace(faceB)
      double v[3];
      bool set[3] = {false, false, false};
      for (int l = 0; l < 3; ++l) {
         if (!c_neu.faceUse[m][l]) continue;
         const signed char* o = c_neu.faceSrc[m][l];
         const long long s = nbr(g, i, j, k, o[0], o[1], o[2]);
         if (s < 0) continue;
         v[l] = f.faceB[l * N + s];
         set[l] = true;
      }
      for (int l = 0; l < 3; ++l) if (set[l]) f.faceB[l * N + n] = v[l];
      for (int w = 0; w < 6; ++w) {
         if ((m & wall[w]) && fp.imfFace[w]) {
            const int axis = w / 2;
            for (int l = 0; l < 3; ++l) if (l != axis) f.faceB[l * N + n] = fp.imf[l];
         }
      }
   }
}

__global__ void __launch_bounds__(128, 8) k_node_fused(GridInfo g, Fields f, FieldParams fp, unsigned long long* cnt) {
   RH_CELL_PROLOGUE
   for (int l = 0; l < 3; ++l) f.cellAvgB[l * N + n] += f.cellB[l * N + n];
   if (!plusOk(g, i, j, k)) return;
   const long long c000 = n, c001 = nbr(g, i, j, k, 0, 0, 1), c010 = nbr(g, i, j, k, 0, 1, 0),
                   c100 = nbr(g, i, j, k, 1, 0, 0), c011 = nbr(g, i, j, k, 0, 1, 1),
                   c110 = nbr(g, i, j, k, 1, 1, 0), c101 = nbr(g, i, j, k, 1, 0, 1),
                   c111 = nbr(g, i, j, k, 1, 1, 1);
   // cell2Node
   double nodeBavg[3];
   for (int l = 0; l < 3; ++l) {
      const double* s = f.cellB + l * N;
      nodeBavg[l] = 0.125 * (s[c000] + s[c001] + s[c010] + s[c100] + s[c011] + s[c110] + s[c101] + s[c111]);
   }
   double rho;
   {
      const double* s = f.cellRho;
      rho = 0.125 * (s[c000] + s[c001] + s[c010] + s[c100] + s[c011] + s[c110] + s[c101] + s[c111]);
   }
   double Ji[3];
#pragma unroll
   for (int l = 0; l < 3; ++l) {
      const double* s = f.cellJi + l * N;
      Ji[l] = 0.125 * (s[c000] + s[c001] + s[c010] + s[c100] + s[c011] + s[c110] + s[c101] + s[c111]);
      f.nodeJi[l * N + n] = Ji[l];
   }
   // calcNodeJ (its whistler limiter reads the averaged nodeB and the unclamped nodeRhoQi)
   double Jn[3];
   {
      const double* fb = f.faceB;
      const long long a000 = n, a100 = c100, a010 = c010, a001 = c001, a110 = c110, a101 = c101, a011 = c011;
#define FB(a, l) fb[(l) * N + (a)]
      const double edgeJx1 = -FB(a000, 2) + FB(a000, 1) + FB(a010, 2) - FB(a001, 1);
      const double edgeJx2 = -FB(a100, 2) + FB(a100, 1) + FB(a110, 2) - FB(a101, 1);
      const double edgeJy1 = +FB(a000, 2) + FB(a001, 0) - FB(a100, 2) - FB(a000, 0);
      const double edgeJy2 = +FB(a010, 2) + FB(a011, 0) - FB(a110, 2) - FB(a010, 0);
      const double edgeJz1 = -FB(a000, 1) + FB(a000, 0) + FB(a100, 1) - FB(a010, 0);
      const double edgeJz2 = -FB(a001, 1) + FB(a001, 0) + FB(a101, 1) - FB(a011, 0);
#undef FB
      double d = 1.0;
      double vw = 0.0;
      const double ne = rho / RHGPU_CHARGE_ELEMENTARY;
      const double Btot = sqrt(sq(nodeBavg[0]) + sq(nodeBavg[1]) + sq(nodeBavg[2]));
      if (ne > 0.0 && g.dx > 0.0) {
         vw = 2.0 * Btot * 3.14159265358979323846 / (RHGPU_PERMEABILITY * ne * RHGPU_CHARGE_ELEMENTARY * g.dx);
      }
      const bool lim = vw > fp.maxVw && fp.maxVw > 0.0;
      if (lim) d = vw / fp.maxVw;
      countIf(lim, &cnt[CNT_MAX_VW]);
      gridCount(f, GC_NODE_MAX_VW, N, n, lim);
      const double a = 0.5 / (g.dx * RHGPU_PERMEABILITY * d);
      Jn[0] = (edgeJx1 + edgeJx2) * a;
      Jn[1] = (edgeJy1 + edgeJy2) * a;
      Jn[2] = (edgeJz1 + edgeJz2) * a;
      for (int l = 0; l < 3; ++l) f.nodeJ[l * N + n] = Jn[l];
   }
   // calcNodeUe
   double Ue[3];
   bool rhoClamp = false, ueClamp = false;
   if (f.flags[n] & RHGPU_FLAG_INNER_NODE) {
      for (int l = 0; l < 3; ++l) Ue[l] = fp.obstacleUe[l];
   } else {
      if (rho < fp.minRho) {
         rho = fp.minRho;
         rhoClamp = true;
      }
      for (int l = 0; l < 3; ++l) {
         if (fabs(rho) > 0) {
            if (fp.use_hall) Ue[l] = -(Jn[l] - Ji[l]) / rho;
            else Ue[l] = Ji[l] / rho;
         } else {
            Ue[l] = 0.0;
         }
      }
      const double Ue2 = sq(Ue[0]) + sq(Ue[1]) + sq(Ue[2]);
      if (Ue2 > fp.maxUe2) {
         const double norm = sqrt(fp.maxUe2 / Ue2);
         Ue[0] *= norm; Ue[1] *= norm; Ue[2] *= norm;
         ueClamp = true;
      }
   }
   f.nodeRho[n] = rho;
   countIf(rhoClamp, &cnt[CNT_MIN_NODE_RHO]);
   countIf(ueClamp, &cnt[CNT_MAX_NODE_UE]);
   gridCount(f, GC_CELL_MAX_UE, N, n, ueClamp);
   for (int l = 0; l < 3; ++l) f.nodeUe[l * N + n] = Ue[l];
   // upwindNodeB: the same eight cells as cell2Node (c111 ... c222 = c000 ... c111)
   double xU = -0.5, yU = 0, zU = 0;
   const double U = sqrt(sq(Ue[0]) + sq(Ue[1]) + sq(Ue[2]));
   if (U > 0) {
      const double a = -0.5 / U;
      xU = Ue[0] * a; yU = Ue[1] * a; zU = Ue[2] * a;
   }
   const double w111 = 1 / sqrt(sq(-0.5 - xU) + sq(-0.5 - yU) + sq(-0.5 - zU));
   const double w112 = 1 / sqrt(sq(-0.5 - xU) + sq(-0.5 - yU) + sq(+0.5 - zU));
   const double w121 = 1 / sqrt(sq(-0.5 - xU) + sq(+0.5 - yU) + sq(-0.5 - zU));
   const double w211 = 1 / sqrt(sq(+0.5 - xU) + sq(-0.5 - yU) + sq(-0.5 - zU));
   const double w122 = 1 / sqrt(sq(-0.5 - xU) + sq(+0.5 - yU) + sq(+0.5 - zU));
   const double w221 = 1 / sqrt(sq(+0.5 - xU) + sq(+0.5 - yU) + sq(-0.5 - zU));
   const double w212 = 1 / sqrt(sq(+0.5 - xU) + sq(-0.5 - yU) + sq(+0.5 - zU));
   const double w222 = 1 / sqrt(sq(+0.5 - xU) + sq(+0.5 - yU) + sq(+0.5 - zU));
   const double wsum = w111 + w112 + w121 + w211 + w122 + w221 + w212 + w222;
   double B[3];
   if (wsum > 0) {
      for (int l = 0; l < 3; ++l) {
         const double* cbl = f.cellB + l * N;
         B[l] = (w111 * cbl[c000] + w112 * cbl[c001] + w121 * cbl[c010] + w211 * cbl[c100] + w122 * cbl[c011] +
                 w221 * cbl[c110] + w212 * cbl[c101] + w222 * cbl[c111]) / wsum;
      }
   } else {
      B[0] = B[1] = B[2] = 0.0;
   }
   for (int l = 0; l < 3; ++l) f.nodeB[l * N + n] = B[l];
   // calcNodeE: E = -Ue x B + eta J
   double E[3];
   E[0] = -(Ue[1] * B[2] - Ue[2] * B[1]);
   E[1] = -(Ue[2] * B[0] - Ue[0] * B[2]);
   E[2] = -(Ue[0] * B[1] - Ue[1] * B[0]);
   const double eta = f.nodeEta[n];
   E[0] += eta * Jn[0];
   E[1] += eta * Jn[1];
   E[2] += eta * Jn[2];
   bool eClamp = false;
   if (fp.maxE2 > 0) {
      const double E2 = sq(E[0]) + sq(E[1]) + sq(E[2]);
      if (E2 > fp.maxE2) {
         const double scaling = sqrt(fp.maxE2 / E2);
         E[0] *= scaling; E[1] *= scaling; E[2] *= scaling;
         eClamp = true;
      }
   }
   countIf(eClamp, &cnt[CNT_MAX_E]);
   gridCount(f, GC_NODE_MAX_E, N, n, eClamp);
   for (int l = 0; l < 3; ++l) f.nodeE[l * N + n] = E[l];
}

}  // namespace rh
