/* Corsair-side adaptor of the B200 hot path (C++, header only).
 *
 * RHybrid is driven by Corsair through three plugins named in the run's .cfg
 * (src/register_objects.cpp:50-58: propagator "BorisBuneman", accumulator
 * "HybridAccumulator", boundary condition "HybridBoundaryCond") and the user
 * hook propagate() (src/user.cpp:49-158), which calls them cell by cell. This
 * header registers GPU plugins under the same names and gives the hook that
 * replaces propagate(): one rhgpu_step() runs the whole step (push, migration,
 * deposit, particle boundary conditions, propagateB) for every population on
 * the GPU, so the plugins' per-cell methods have nothing left to do and
 * return true.
 *
 * A Corsair build adds, in place of RHybrid's own registration and hook:
 *
 *   registerObjectMakers(objectFactories)   -> rhgpu_corsair::registerObjectMakers<PARTICLE>(objectFactories)
 *   userLateInitialization(...), at its end -> rhgpu_corsair::gpuSetup(sim, simClasses, lists, periodic, device)
 *   propagate(sim, simClasses, lists)       -> rhgpu_corsair::gpuPropagate(sim, simClasses, lists)
 *   before each data save step              -> rhgpu_corsair::gpuDownload(sim, simClasses, lists)
 *   at exit                                 -> rhgpu_corsair::gpuFinalize()
 *
 * Grid arrays and particle lists stay in Corsair's ParGrid containers, which
 * the adaptor uploads once and brings back on output steps (vector arrays
 * interleaved per cell, particles as {X,Y,Z,VX,VY,VZ,WEIGHT} per cell, the
 * layouts the C ABI takes). One block is one cell (RHybrid's block size 1).
 * The headers it needs are Corsair's plugin base classes, RHybrid's hybrid.h
 * and particle_species.h, and include/rhgpu.h; link with librhgpu.so.
 */
#ifndef RHGPU_CORSAIR_H
#define RHGPU_CORSAIR_H

#include <cstring>
#include <string>
#include <vector>

#include "base_class_particle_accumulator.h"
#include "base_class_particle_boundary_condition.h"
#include "base_class_particle_propagator.h"
#include "hybrid.h"
#include "particle_species.h"
#include "rhgpu.h"

namespace rhgpu_corsair {

/* the GPU context of the run, shared by the plugins and the hook */
struct GpuRun {
   rhgpu_ctx* ctx = nullptr;
   std::vector<pargrid::DataID> particleIDs;   // per population, in list order
   std::string error;
};
inline GpuRun& run() {
   static GpuRun r;
   return r;
}

/* BorisBuneman::propagateCell (src/particle_propagator_boris_buneman.h:197-207) */
class BorisBunemanGPU : public ParticlePropagatorBase {
 public:
   bool propagateCell(pargrid::CellID, pargrid::DataID, const double* const, unsigned int) override { return true; }
};

/* Accumulator (src/particle_accumulator.h:36-45) */
class HybridAccumulatorGPU : public ParticleAccumulatorBase {
 public:
   bool accumulateBoundaryCells(pargrid::DataID, const unsigned int*) override { return true; }
   bool accumulateInnerCells(pargrid::DataID, const unsigned int*) override { return true; }
   bool addRemoteUpdates() override { return true; }
   bool clearAccumulationArrays() override { return true; }
   bool sendUpdates() override { return true; }
   bool wait() override { return true; }
};

/* ParticleBoundaryCondHybrid::apply (src/particle_boundary_cond_hybrid.h:112-185) */
template <class SPECIES, class PARTICLE>
class HybridBoundaryCondGPU : public ParticleBoundaryCondBase {
 public:
   bool apply(pargrid::DataID, unsigned int*, const std::vector<pargrid::CellID>&) { return true; }
};

inline ParticlePropagatorBase* BBGPUMaker() { return new BorisBunemanGPU(); }
inline ParticleAccumulatorBase* AccumulatorGPUMaker() { return new HybridAccumulatorGPU(); }
template <class SPECIES, class PARTICLE>
ParticleBoundaryCondBase* HybridBoundaryCondGPUMaker() { return new HybridBoundaryCondGPU<SPECIES, PARTICLE>(); }

/* the plugins under RHybrid's .cfg names (src/register_objects.cpp:50-58) */
template <class PARTICLE, class FACTORIES>
bool registerObjectMakers(FACTORIES& f) {
   bool ok = true;
   if (!f.particleAccumulators.registerMaker("HybridAccumulator", AccumulatorGPUMaker)) ok = false;
   if (!f.particleBoundaryConditions.registerMaker("HybridBoundaryCond", HybridBoundaryCondGPUMaker<Species, PARTICLE>)) ok = false;
   if (!f.particlePropagators.registerMaker("BorisBuneman", BBGPUMaker)) ok = false;
   return ok;
}

inline bool fail(const std::string& where) {
   run().error = where + ": " + rhgpu_last_error();
   return false;
}

/* the ParGrid arrays the context keeps, by rhgpu array id */
inline pargrid::DataID arrayID(int id) {
   switch (id) {
      case RHGPU_FACE_B: return Hybrid::dataFaceBID;
      case RHGPU_CELL_B: return Hybrid::dataCellBID;
      case RHGPU_CELL_UE: return Hybrid::dataCellUeID;
      case RHGPU_CELL_EP: return Hybrid::dataCellEpID;
      case RHGPU_CELL_RHOQI: return Hybrid::dataCellRhoQiID;
      case RHGPU_CELL_JI: return Hybrid::dataCellJiID;
      case RHGPU_CELL_J: return Hybrid::dataCellJID;
      case RHGPU_NODE_RHOQI: return Hybrid::dataNodeRhoQiID;
      case RHGPU_NODE_JI: return Hybrid::dataNodeJiID;
      case RHGPU_NODE_J: return Hybrid::dataNodeJID;
      case RHGPU_NODE_UE: return Hybrid::dataNodeUeID;
      case RHGPU_NODE_B: return Hybrid::dataNodeBID;
      case RHGPU_NODE_E: return Hybrid::dataNodeEID;
      case RHGPU_NODE_ETA: return Hybrid::dataNodeEtaID;
      case RHGPU_CELL_AVERAGE_B: return Hybrid::dataCellAverageBID;
   }
   return pargrid::INVALID_DATAID;
}

/* the run's parameters from RHybrid's configuration (the Hybrid statics that
 * userLateInitialization sets, src/user.cpp:356-1807) and Corsair's grid */
inline rhgpu_params params(const Simulation& sim, const int periodic[3]) {
   rhgpu_params P;
   std::memset(&P, 0, sizeof P);
   P.nx = sim.x_blocks; P.ny = sim.y_blocks; P.nz = sim.z_blocks;
   for (int a = 0; a < 3; ++a) P.periodic[a] = periodic[a] ? 1 : 0;
   P.x_min = sim.x_min; P.y_min = sim.y_min; P.z_min = sim.z_min;
   P.dx = Hybrid::dx;
   P.dt = sim.dt;
   P.t_initial = sim.t;
   P.use_hall = Hybrid::useHallElectricField;
   P.use_electron_pressure = Hybrid::useElectronPressure;
   P.isothermal_electrons = Hybrid::useIsothermalElectrons;
   P.use_gravity = Hybrid::useGravity;
   P.use_initial_flow_through = Hybrid::useInitialFlowThrough;
   P.n_linear_smoothings_nodeE = Hybrid::N_linearSmoothingsNodeE;
   P.use_gaussian_smoothing_nodeE = Hybrid::useGaussianSmoothingNodeE;
   P.electron_pressure_coeff = Hybrid::electronPressureCoeff;
   for (int l = 0; l < 4; ++l) P.gaussian_coeffs[l] = Hybrid::gaussianSmoothingCoeffsNodeE[l];
   for (int l = 0; l < 3; ++l) P.field_obstacle_Ue[l] = Hybrid::fieldObstacleUe[l];
   P.GMdt = Hybrid::GMdt;
   P.max_ion_speed2 = Hybrid::maxIonSpeed2;
   P.max_electron_speed2 = Hybrid::maxElectronSpeed2;
   P.min_ion_charge_density = Hybrid::minIonChargeDensity;
   P.max_electric_field2 = Hybrid::maxElectricField2;
   P.max_whistler_speed = Hybrid::maxWhistlerSpeed;
   P.initial_flow_through_period = Hybrid::initialFlowThroughPeriod;
   P.imf_B[0] = Hybrid::IMFBx; P.imf_B[1] = Hybrid::IMFBy; P.imf_B[2] = Hybrid::IMFBz;
   for (int w = 0; w < 6; ++w) {
      P.imf_boundary_cellB[w] = Hybrid::IMFBoundaryCellB[w] ? 1 : 0;
      P.imf_boundary_faceB[w] = Hybrid::IMFBoundaryFaceB[w] ? 1 : 0;
   }
   return P;
}

/* Creates the GPU context (on `device`, particle path `path`, RHGPU_PATH_FAST
 * by default) and uploads the grid arrays, the cell flags and every
 * population's particles from Corsair's containers. */
template <class PARTICLE>
bool gpuSetup(Simulation& sim, SimulationClasses& sc, std::vector<ParticleListBase*>& lists, const int periodic[3],
              int device = 0, int path = RHGPU_PATH_FAST) {
   GpuRun& r = run();
   if (r.ctx) return true;
   const rhgpu_params P = params(sim, periodic);
   std::vector<rhgpu_species> sp(lists.size());
   std::vector<int64_t> cap(lists.size(), 0);
   r.particleIDs.assign(lists.size(), pargrid::INVALID_DATAID);
   pargrid::ParGrid& pg = sc.pargrid;
   const size_t N = pg.getNumberOfAllCells();
   for (size_t s = 0; s < lists.size(); ++s) {
      const Species* S = reinterpret_cast<const Species*>(lists[s]->getSpecies());
      sp[s].q = S->q;
      sp[s].m = S->m;
      sp[s].R2_obstacle = S->R2_obstacle;
      sp[s].accumulate = S->accumulate ? 1 : 0;
      sp[s].accelerate = S->accelerate ? 1 : 0;
      if (!lists[s]->getParticles(r.particleIDs[s])) {
         r.error = "gpuSetup: a population has no particle data";
         return false;
      }
   }
   if (rhgpu_create(&P, (int32_t)sp.size(), sp.data(), cap.data(), device, &r.ctx) != RHGPU_OK) return fail("rhgpu_create");
   if (rhgpu_set_path(r.ctx, path) != RHGPU_OK) return fail("rhgpu_set_path");
   for (int id = 0; id < RHGPU_NUM_ARRAYS; ++id) {
      const Real* a = pg.getUserDataStatic<Real>(arrayID(id));
      if (rhgpu_upload_array(r.ctx, id, a) != RHGPU_OK) return fail("rhgpu_upload_array");
   }
   std::vector<uint8_t> flags(N, 0);
   const bool* f0 = pg.getUserDataStatic<bool>(Hybrid::dataInnerFlagFieldID);
   const bool* f1 = pg.getUserDataStatic<bool>(Hybrid::dataInnerFlagNodeID);
   const bool* f2 = pg.getUserDataStatic<bool>(Hybrid::dataInnerFlagParticleID);
   const bool* f3 = pg.getUserDataStatic<bool>(Hybrid::dataInnerFlagCellEpID);
   for (size_t b = 0; b < N; ++b)
      flags[b] = (f0[b] ? RHGPU_FLAG_INNER_FIELD : 0) | (f1[b] ? RHGPU_FLAG_INNER_NODE : 0) |
                 (f2[b] ? RHGPU_FLAG_INNER_PARTICLE : 0) | (f3[b] ? RHGPU_FLAG_INNER_CELLEP : 0);
   if (rhgpu_upload_cell_flags(r.ctx, flags.data()) != RHGPU_OK) return fail("rhgpu_upload_cell_flags");
   for (size_t s = 0; s < lists.size(); ++s) {
      pargrid::DataWrapper<PARTICLE> w = pg.getUserDataDynamic<PARTICLE>(r.particleIDs[s]);
      std::vector<uint32_t> counts(N);
      size_t n = 0;
      for (size_t b = 0; b < N; ++b) n += counts[b] = (uint32_t)w.size()[b];
      std::vector<double> rec(7 * (n ? n : 1));
      size_t off = 0;
      for (size_t b = 0; b < N; ++b) {
         for (uint32_t p = 0; p < counts[b]; ++p)
            for (int a = 0; a < 7; ++a) rec[7 * (off + p) + a] = w.data()[b][p].state[a];
         off += counts[b];
      }
      if (rhgpu_upload_particles(r.ctx, (int32_t)s, counts.data(), rec.data(), (int64_t)n) != RHGPU_OK)
         return fail("rhgpu_upload_particles");
   }
   return true;
}

/* the propagate() hook (src/user.cpp:49-158): one step on the GPU */
inline bool gpuPropagate(Simulation&, SimulationClasses&, std::vector<ParticleListBase*>&) {
   GpuRun& r = run();
   if (!r.ctx) {
      r.error = "gpuPropagate: gpuSetup has not run";
      return false;
   }
   if (rhgpu_step(r.ctx, 1) != RHGPU_OK) return fail("rhgpu_step");
   return true;
}

/* The device state into Corsair's containers (output steps): every grid array
 * and every population's particle list. */
template <class PARTICLE>
bool gpuDownload(Simulation&, SimulationClasses& sc, std::vector<ParticleListBase*>& lists) {
   GpuRun& r = run();
   if (!r.ctx) return true;
   pargrid::ParGrid& pg = sc.pargrid;
   const size_t N = pg.getNumberOfAllCells();
   for (int id = 0; id < RHGPU_NUM_ARRAYS; ++id)
      if (rhgpu_download_array(r.ctx, id, pg.getUserDataStatic<Real>(arrayID(id))) != RHGPU_OK)
         return fail("rhgpu_download_array");
   for (size_t s = 0; s < lists.size() && s < r.particleIDs.size(); ++s) {
      int64_t n = 0;
      if (rhgpu_num_particles(r.ctx, (int32_t)s, &n) != RHGPU_OK) return fail("rhgpu_num_particles");
      std::vector<uint32_t> counts(N);
      std::vector<double> rec(7 * (n ? n : 1));
      int64_t got = 0;
      if (rhgpu_download_particles(r.ctx, (int32_t)s, counts.data(), rec.data(), n, &got) != RHGPU_OK)
         return fail("rhgpu_download_particles");
      pargrid::DataWrapper<PARTICLE> w = pg.getUserDataDynamic<PARTICLE>(r.particleIDs[s]);
      size_t off = 0;
      for (size_t b = 0; b < N; ++b) {
         w.resize((pargrid::CellID)b, counts[b]);
         for (uint32_t p = 0; p < counts[b]; ++p)
            for (int a = 0; a < 7; ++a) w.data()[b][p].state[a] = rec[7 * (off + p) + a];
         off += counts[b];
      }
   }
   return true;
}

inline void gpuFinalize() {
   GpuRun& r = run();
   if (r.ctx) rhgpu_destroy(r.ctx);
   r.ctx = nullptr;
   r.particleIDs.clear();
}

}  // namespace rhgpu_corsair

#endif
