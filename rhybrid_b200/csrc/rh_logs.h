// Population and field log files of RHybrid, written on the host from the
// device-side reductions (rhgpu_reduce_diagnostics) and the log counters.
//
// File names, header lines, column order, number format and the arithmetic of
// each column follow the reference's log writer so that the files are a
// drop-in for its post-processing (tools/rhb_log2pdf.sh):
//   headers              src/user.cpp:2147-2231
//   one line per log step, counter rates, warnings and the max-B stop
//                        src/diagnostics.h:405-818 (logWriteParticleField)
// Column 31 ("maxVw rate") carries the maxNodeUe counter, as the reference's
// writer does (diagnostics.h:497), so that the columns match its files.
#pragma once

#include <cmath>
#include <fstream>
#include <limits>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

namespace rh {

struct LogSpecies {
   std::string name;
   double m = 0.0, q = 0.0;
};

// per-species log counters, in the order the particle log prints their rates
enum LogParticleCounter {
   LPC_ESCAPE = 0, LPC_IMPACT, LPC_INJECT, LPC_INJECT_MACRO, LPC_ESCAPE_KE, LPC_IMPACT_KE, LPC_INJECT_KE, LPC_MAXVI,
   LPC_COUNT
};
// field log counters, in the order the field log prints their rates
enum LogFieldCounter {
   LFC_MAX_CELL_UE = 0, LFC_MAX_NODE_UE, LFC_MAX_VW, LFC_MAX_E, LFC_MIN_CELL_RHOQI, LFC_MIN_NODE_RHOQI, LFC_COUNT
};

// the population sums of one species (logCalcParticle, diagnostics.h:187-222)
struct LogPopulation {
   double nMacro, nReal, sumVx, sumVy, sumVz, sumV, sumWV2, maxVi;
};
// the field sums and scales (logCalcField, diagnostics.h:246-404)
struct LogField {
   double nCells, sumBx, sumBy, sumBz, sumB, maxB, sumDivB, maxDivB, maxDivBPerB, sumB2;
   double sumJx, sumJy, sumJz, sumJ, maxJ;
   double sumEpx, sumEpy, sumEpz, sumEp, maxEp, sumEp2;
   double sumEx, sumEy, sumEz, sumE, maxE, sumE2, sumCellE2;
   double minDe, maxDe, minDi, maxDi, minTLarmor, maxVA, maxUe;
};

struct LogStep {
   double t, dt, dx, dV, tStart;
   long long timestep;
   double permeability, permittivity;
   std::vector<LogPopulation> pop;
   std::vector<std::vector<double>> pc;   // LPC_COUNT per species
   LogField f;
   double fc[LFC_COUNT];
};

class LogFiles {
 public:
   bool open(const std::string& dir, const std::vector<LogSpecies>& sp, int precision, std::string& err) {
      close();
      species_ = sp;
      for (size_t s = 0; s < sp.size(); ++s) {
         // pop<NNN>_<name>.log with the reference's zero padding (two zeros below 10 species)
         std::stringstream ss;
         ss << dir << "/pop" << (s < 10 ? "00" : (s < 100 ? "0" : "")) << s + 1 << "_" << sp[s].name << ".log";
         pop_.emplace_back(new std::ofstream(ss.str().c_str(), std::ios_base::out));
         std::ofstream& o = *pop_.back();
         if (!o) { err = "cannot open " + ss.str(); close(); return false; }
         o.precision(precision);
         o << std::scientific << std::showpos;
         o << "% " << sp[s].name << std::endl << "% m [kg] = " << sp[s].m << std::endl
           << "% q [C] = " << sp[s].q << std::endl << "% columns = 17" << std::endl;
         static const char* cols[17] = {
            "Time [s]", "Particles [#]", "Macroparticles [#]", "avg(Vx) [m/s]", "avg(Vy) [m/s]", "avg(Vz) [m/s]",
            "avg(|V|) [m/s]", "Kinetic energy [J]", "max(|V|) [m/s]", "Escape rate [#/s]", "Impact rate [#/s]",
            "Inject rate [#/s]", "Macroparticle inject rate [#/dt]", "Kinetic energy escape rate [J/s]",
            "Kinetic energy impact rate [J/s]", "Kinetic energy inject rate [J/s]", "Constraint maxVi rate [#/dt]"};
         for (int c = 0; c < 17; ++c) o << colLabel(c) << cols[c] << std::endl;
      }
      const std::string fn = dir + "/field.log";
      field_.open(fn.c_str(), std::ios_base::out);
      if (!field_) { err = "cannot open " + fn; close(); return false; }
      field_.precision(precision);
      field_ << std::scientific << std::showpos;
      static const char* fcols[41] = {
         "Time [s]", "avg(faceBx) [T]", "avg(faceBy) [T]", "avg(faceBz) [T]", "avg(|faceB|) [T]", "max(|faceB|) [T]",
         "avg(div(faceB)) [T/m]", "max(div(faceB)) [T/m]", "max(dx*div(faceB)/faceB) [-]",
         "energy(sum(dV*faceB^2/2*mu0)) [J]", "avg(cellJix) [A/m^2]", "avg(cellJiy) [A/m^2]", "avg(cellJiz) [A/m^2]",
         "avg(|cellJi|) [A/m^2]", "max(|cellJi|) [A/m^2]", "avg(cellEpx) [V/m]", "avg(cellEpy) [V/m]",
         "avg(cellEpz) [V/m]", "avg(|cellEp|) [V/m]", "max(|cellEp|) [V/m]", "energy(sum(dV*cellEp^2*eps0/2)) [J]",
         "avg(nodeEx) [V/m]", "avg(nodeEy) [V/m]", "avg(nodeEz) [V/m]", "avg(|nodeE|) [V/m]", "max(|nodeE|) [V/m]",
         "energy(sum(dV*nodeE^2*eps0/2)), nodeE = -Ue x B + eta*J [J]",
         "energy(sum(dV*cellE^2*eps0/2)), cellE = -Ue x B [J]", "Constraint maxUe rate (cell) [#/dt]",
         "Constraint maxUe rate (node) [#/dt]", "Constraint maxVw rate (node) [#/dt]",
         "Constraint maxE rate (node) [#/dt]", "Constraint minRhoQi rate (cell) [#/dt]",
         "Constraint minRhoQi rate (node) [#/dt]", "Minimum electron inertial length [m]",
         "Maximum electron inertial length [m]", "Minimum proton inertial length [m]",
         "Maximum proton inertial length [m]", "Minimum ion Larmor period [s]", "Maximum Alfven speed [m/s]",
         "Maximum electron fluid speed [m/s]"};
      field_ << "% field" << std::endl << "% columns = 41" << std::endl;
      for (int c = 0; c < 41; ++c) field_ << colLabel(c) << fcols[c] << std::endl;
      return true;
   }

   bool isOpen() const { return field_.is_open(); }

   void close() {
      for (auto& o : pop_) { o->flush(); o->close(); }
      pop_.clear();
      if (field_.is_open()) { field_.flush(); field_.close(); }
   }

   // one line per file; false when max |B| exceeds maxBStop (the run stops).
   // Warnings, the stop message and (mainLog) the diagnostics block go to msg.
   bool write(const LogStep& L, double maxBStop, bool mainLog, std::string& msg) {
      const double Dt = L.t - L.tStart;
      double maxViAll = 0.0;
      std::stringstream macro;
      for (size_t s = 0; s < pop_.size(); ++s) {
         std::ostream& o = *pop_[s];
         const LogPopulation& P = L.pop[s];
         const std::vector<double>& c = L.pc[s];
         const double m = species_[s].m;
         o << L.t << " " << P.nReal << " " << P.nMacro << " ";
         if (mainLog) macro << "\t Nmacroparticles(" << species_[s].name << ") = " << str15(P.nMacro) << " = "
                            << str15(P.nMacro / 1.0e9) << " x 10^9" << std::endl;
         if (P.nReal > 0.0) {
            o << P.sumVx / P.nReal << " " << P.sumVy / P.nReal << " " << P.sumVz / P.nReal << " " << P.sumV / P.nReal << " ";
         } else {
            zeros(o, 4);
         }
         o << 0.5 * m * P.sumWV2 << " " << P.maxVi << " ";
         if (maxViAll < P.maxVi) maxViAll = P.maxVi;
         if (Dt > 0) {
            o << c[LPC_ESCAPE] / Dt << " " << c[LPC_IMPACT] / Dt << " " << c[LPC_INJECT] / Dt << " "
              << c[LPC_INJECT_MACRO] / Dt * L.dt << " " << 0.5 * m * c[LPC_ESCAPE_KE] / Dt << " "
              << 0.5 * m * c[LPC_IMPACT_KE] / Dt << " " << 0.5 * m * c[LPC_INJECT_KE] / Dt << " "
              << c[LPC_MAXVI] / Dt * L.dt << " ";
         } else {
            zeros(o, 8);
         }
      }
      const LogField& F = L.f;
      std::ostream& o = field_;
      o << L.t << " ";
      avg4(o, F.nCells, F.sumBx, F.sumBy, F.sumBz, F.sumB);
      o << F.maxB << " ";
      if (F.nCells > 0) o << F.sumDivB / F.nCells << " ";
      else zeros(o, 1);
      o << F.maxDivB << " " << L.dx * F.maxDivBPerB << " " << F.sumB2 * L.dV / (2.0 * L.permeability) << " ";
      avg4(o, F.nCells, F.sumJx, F.sumJy, F.sumJz, F.sumJ);
      o << F.maxJ << " ";
      avg4(o, F.nCells, F.sumEpx, F.sumEpy, F.sumEpz, F.sumEp);
      o << F.maxEp << " " << F.sumEp2 * L.dV * L.permittivity / (2.0) << " ";
      avg4(o, F.nCells, F.sumEx, F.sumEy, F.sumEz, F.sumE);
      // the reference's writer puts two blanks before max(|nodeE|)
      o << " " << F.maxE << " " << F.sumE2 * L.dV * L.permittivity / (2.0) << " "
        << F.sumCellE2 * L.dV * L.permittivity / (2.0) << " ";
      if (Dt > 0) {
         for (int k = 0; k < LFC_COUNT; ++k) o << L.fc[k] / Dt * L.dt << " ";
      } else {
         zeros(o, LFC_COUNT);
      }
      o << F.minDe << " " << F.maxDe << " " << F.minDi << " " << F.maxDi << " " << F.minTLarmor << " " << F.maxVA << " "
        << F.maxUe << " ";
      for (auto& p : pop_) *p << std::endl;
      o << std::endl;

      const double tL_dt = F.minTLarmor / L.dt;
      const double vi_dxdt = maxViAll / (L.dx / L.dt);
      const double va_dxdt = F.maxVA / (L.dx / L.dt);
      const double ue_dxdt = F.maxUe / (L.dx / L.dt);
      std::stringstream m;
      const auto when = [&](std::ostream& s) -> std::ostream& {
         return s << " (time step = " << L.timestep << ", time = " << L.t << ")";
      };
      if (mainLog) {
         m << "(RHYBRID) Diagnostics (time step = " << L.timestep << ", time = " << L.t << "):" << std::endl
           << macro.str()
           << "\t Max. |Vion|             : Vi_max  = " << maxViAll / 1e3 << " km/s = " << vi_dxdt << " dx/dt" << std::endl
           << "\t Max. |Ue|               : Ue_max  = " << F.maxUe / 1e3 << " km/s = " << ue_dxdt << " dx/dt" << std::endl
           << "\t Max. |VAlfven|          : Va_max  = " << F.maxVA / 1e3 << " km/s = " << va_dxdt << " dx/dt" << std::endl
           << "\t Max. |faceB|            : B_max   = " << F.maxB / 1e-9 << " nT" << std::endl
           << "\t Min. ion Larmor period  : tL_min  = " << F.minTLarmor << " s = " << tL_dt << " dt" << std::endl
           << "\t Max. |cellJi|           : Ji_max  = " << F.maxJ << " A/m^2" << std::endl
           << "\t Max. |cellEp|           : Ep_max  = " << F.maxEp / 1e-3 << " mV/m" << std::endl
           << "\t Max. |nodeE|            : E_max   = " << F.maxE / 1e-3 << " mV/m" << std::endl
           << "\t Min. e- inertial length : de_min  = " << F.minDe / 1e3 << " km = " << F.minDe / L.dx << " dx" << std::endl
           << "\t Max. e- inertial length : de_max  = " << F.maxDe / 1e3 << " km = " << F.maxDe / L.dx << " dx" << std::endl
           << "\t Min. H+ inertial length : di_min  = " << F.minDi / 1e3 << " km = " << F.minDi / L.dx << " dx" << std::endl
           << "\t Max. H+ inertial length : di_max  = " << F.maxDi / 1e3 << " km = " << F.maxDi / L.dx << " dx" << std::endl;
      }
      if (tL_dt < 10) when(m << "(RHYBRID) WARNING: Minimum Larmor period: tL_min/dt < 10 (" << tL_dt << ")") << std::endl;
      if (vi_dxdt > 0.9) when(m << "(RHYBRID) WARNING: Maximum ion speed: Vi_max/(dx/dt) > 0.9 (" << vi_dxdt << ")") << std::endl;
      if (ue_dxdt > 0.9) when(m << "(RHYBRID) WARNING: Maximum ion speed: Ue_max/(dx/dt) > 0.9 (" << ue_dxdt << ")") << std::endl;
      if (va_dxdt > 0.9) when(m << "(RHYBRID) WARNING: Maximum Alfven speed: Va_max/(dx/dt) > 0.9 (" << va_dxdt << ")") << std::endl;
      bool ok = true;
      if (F.maxB > maxBStop) {
         ok = false;
         m << "(RHYBRID) CONSTRAINT: maximum B reached (" << F.maxB / 1e-9 << " nT >" << maxBStop / 1e-9
           << " nT) at time step = " << L.timestep << " (time = " << L.t << "), stopping run" << std::endl;
      }
      msg = m.str();
      return ok;
   }

 private:
   // "% 01. " .. "% 41. " (formed as text: the streams print numbers with a sign)
   static std::string colLabel(int c) { return std::string("% ") + (c < 9 ? "0" : "") + std::to_string(c + 1) + ". "; }
   static void zeros(std::ostream& o, int n) {
      for (int k = 0; k < n; ++k) o << 0.0 << " ";
   }
   static void avg4(std::ostream& o, double n, double a, double b, double c, double d) {
      if (n > 0) o << a / n << " " << b / n << " " << c / n << " " << d / n << " ";
      else zeros(o, 4);
   }
   static std::string str15(double x) {
      std::stringstream ss;
      ss.precision(15);
      ss << x;
      return ss.str();
   }
   std::vector<LogSpecies> species_;
   std::vector<std::unique_ptr<std::ofstream>> pop_;
   std::ofstream field_;
};

// spatial, temporal and velocity scales of the field log from the extremes the
// device reduction forms (each scale is monotone in its extreme, so the result
// equals the per-cell extreme of the reference, diagnostics.h:375-395); the
// reference's starting values where no cell qualifies
inline void logScales(double minRhoQ, double maxRhoQ, double minRhoM, double maxRhoM, double maxB, double me, double mp,
                      double e, double mu0, double* out6_minDe_maxDe_minDi_maxDi_minTL) {
   double* o = out6_minDe_maxDe_minDi_maxDi_minTL;
   const double big = std::numeric_limits<double>::max(), low = std::numeric_limits<double>::lowest();
   const auto de = [&](double r) { return std::sqrt(me / (mu0 * e * r)); };
   const auto di = [&](double r) { return std::sqrt((mp * mp) / (mu0 * (e * e) * r)); };
   o[0] = maxRhoQ > 0.0 ? de(maxRhoQ) : big;
   o[1] = minRhoQ > 0.0 && minRhoQ < INFINITY ? de(minRhoQ) : low;
   o[2] = maxRhoM > 0.0 ? di(maxRhoM) : big;
   o[3] = minRhoM > 0.0 && minRhoM < INFINITY ? di(minRhoM) : low;
   o[4] = maxB > 0.0 ? 2.0 * M_PI * mp / (e * maxB) : big;
}

}  // namespace rh
