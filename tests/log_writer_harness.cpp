// Test harness (CPU): drives the library's log writer (rhybrid_b200/csrc/rh_logs.h,
// header-only host code) with log-step values read from a text file, so that
// its files can be compared with the reference's own log writer on CPU.
//
// Input (whitespace separated):
//   directory nspecies precision maxBStop mainLog nsteps
//   nspecies x (name m q)
//   nsteps x (t dt dx dV tStart timestep permeability permittivity
//             nspecies x (8 population sums, 8 counters in LogParticleCounter order)
//             35 field values in LogField order, 6 field counters in LogFieldCounter order)
// Output: the log files in `directory`, and one line per step on stdout:
// "stop" or "ok".
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "../rhybrid_b200/csrc/rh_logs.h"

int main(int argc, char** argv) {
   if (argc != 2) {
      std::cerr << "usage: log_writer_harness input.txt\n";
      return 2;
   }
   std::ifstream in(argv[1]);
   std::string dir;
   int ns = 0, precision = 10, mainLog = 0, nsteps = 0;
   double maxB = 0.0;
   in >> dir >> ns >> precision >> maxB >> mainLog >> nsteps;
   std::vector<rh::LogSpecies> sp(ns);
   for (auto& s : sp) in >> s.name >> s.m >> s.q;
   rh::LogFiles files;
   std::string err;
   if (!files.open(dir, sp, precision, err)) {
      std::cerr << err << "\n";
      return 1;
   }
   for (int k = 0; k < nsteps; ++k) {
      rh::LogStep L;
      in >> L.t >> L.dt >> L.dx >> L.dV >> L.tStart >> L.timestep >> L.permeability >> L.permittivity;
      L.pop.resize(ns);
      L.pc.assign(ns, std::vector<double>(rh::LPC_COUNT, 0.0));
      for (int s = 0; s < ns; ++s) {
         rh::LogPopulation& P = L.pop[s];
         in >> P.nMacro >> P.nReal >> P.sumVx >> P.sumVy >> P.sumVz >> P.sumV >> P.sumWV2 >> P.maxVi;
         for (int c = 0; c < rh::LPC_COUNT; ++c) in >> L.pc[s][c];
      }
      rh::LogField& F = L.f;
      double* f[35] = {&F.nCells, &F.sumBx, &F.sumBy, &F.sumBz, &F.sumB, &F.maxB, &F.sumDivB, &F.maxDivB,
                       &F.maxDivBPerB, &F.sumB2, &F.sumJx, &F.sumJy, &F.sumJz, &F.sumJ, &F.maxJ, &F.sumEpx,
                       &F.sumEpy, &F.sumEpz, &F.sumEp, &F.maxEp, &F.sumEp2, &F.sumEx, &F.sumEy, &F.sumEz, &F.sumE,
                       &F.maxE, &F.sumE2, &F.sumCellE2, &F.minDe, &F.maxDe, &F.minDi, &F.maxDi, &F.minTLarmor,
                       &F.maxVA, &F.maxUe};
      for (int q = 0; q < 35; ++q) in >> *f[q];
      for (int c = 0; c < rh::LFC_COUNT; ++c) in >> L.fc[c];
      if (!in) {
         std::cerr << "short input at step " << k << "\n";
         return 1;
      }
      std::string msg;
      std::cout << (files.write(L, maxB, mainLog != 0, msg) ? "ok" : "stop") << "\n";
   }
   files.close();
   return 0;
}
