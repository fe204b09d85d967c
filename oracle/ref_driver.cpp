/* Oracle (test infrastructure only): drives RHybrid's own, unmodified
 * hot-path sources (compiled from the reference tree against the
 * single-process shim in oracle/shim/) through the same C ABI as the GPU
 * library (include/rhgpu.h), with the prefix rhref_.
 *
 * Used only by tests/ and bench.py's CPU baseline as the checker; never part
 * of the product path.
 *
 * One time step replays propagate() (src/user.cpp:49-158) without logging,
 * detectors and injection:
 *   initial flow-through switch-off            user.cpp:52-59
 *   setupGetFields                             user.cpp:118
 *   BorisBuneman::propagateCell, all cells     user.cpp:120-121
 *   cell-to-cell migration                     (Corsair, restated: rh_migrate_canonical)
 *   clearAccumulationArrays                    user.cpp:122
 *   accumulateBoundaryCells/InnerCells         user.cpp:125-126
 *   addRemoteUpdates (finalize /dV, rho clamp) particle_accumulator.cpp:260-335
 *   applyBoundaryConditions                    user.cpp:128
 *   propagateB                                 user.cpp:134
 * rhref_log_open / rhref_log_write run the reference's own log writer
 * (diagnostics::logWriteParticleField, src/diagnostics.h:405-818) on the
 * current state into files opened here without headers (the headers come
 * from src/user.cpp, which is not built).
 * Only one rhref context may exist at a time: the reference keeps its state
 * in the static struct Hybrid (src/hybrid.h:161).
 */
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

#include "hybrid.h"
#include "hybrid_propagator.h"
#include "particle_definition.h"
#include "particle_species.h"
#include "particle_accumulator.h"
#include "particle_propagator_boris_buneman.h"
#include "particle_boundary_cond_hybrid.h"
#include "diagnostics.h"
#include "operator_userdata.h"

#include <fstream>

#include "oracle_common.h"

/* The boundary condition's initialize() asks the (not built) injector for the
 * macroparticle weight, used only by the after-restart filter. */
bool getInjectorParameters(ParticleInjectorBase*,InjectorParameters& p) {
   p.w = 0.0;
   return true;
}

namespace {

const int MAX_SPECIES = 8;
thread_local std::string g_err;

int fail(int code,const std::string& msg) { g_err = msg; return code; }

typedef Particle<Real> PARTICLE;

struct RefCtx {
   rhgpu_params P;
   Simulation sim;
   SimulationClasses sc;
   ConfigReader cr;
   int nspecies = 0;
   std::vector<Species> species;
   std::vector<ParticleListBase> plists;
   std::vector<pargrid::DataID> particleIDs;
   std::vector<std::vector<unsigned int> > counts;
   BorisBuneman<PARTICLE> bb[MAX_SPECIES];
   ParticleBoundaryCondHybrid<Species,PARTICLE> bc[MAX_SPECIES];
   pargrid::DataID arrayIDs[RHGPU_NUM_ARRAYS];
   Real dxBelow = 0;
   double escapeFast = 0;
};

/* Accumulator keeps a process-wide construction count that decides which
 * instance clears (order 0) and which finalizes (the last one); a fixed pool
 * constructed once keeps those roles stable across contexts. */
Accumulator* accumulatorPool() {
   static Accumulator pool[MAX_SPECIES];
   return pool;
}

RefCtx* g_active = nullptr;

void setHybridStatics(RefCtx& c) {
   const rhgpu_params& P = c.P;
   pargrid::ParGrid& pg = c.sc.pargrid;
   Hybrid::X_POS_EXISTS = (1u << pg.calcNeighbourTypeID(+1,+0,+0));
   Hybrid::X_NEG_EXISTS = (1u << pg.calcNeighbourTypeID(-1,+0,+0));
   Hybrid::Y_POS_EXISTS = (1u << pg.calcNeighbourTypeID(+0,+1,+0));
   Hybrid::Y_NEG_EXISTS = (1u << pg.calcNeighbourTypeID(+0,-1,+0));
   Hybrid::Z_POS_EXISTS = (1u << pg.calcNeighbourTypeID(+0,+0,+1));
   Hybrid::Z_NEG_EXISTS = (1u << pg.calcNeighbourTypeID(+0,+0,-1));
   Hybrid::dx = P.dx;
   Hybrid::dV = cube(Hybrid::dx);
   for (int l=0;l<3;++l) Hybrid::fieldObstacleUe[l] = P.field_obstacle_Ue[l];
   Hybrid::useHallElectricField = P.use_hall != 0;
   Hybrid::useElectronPressure = P.use_electron_pressure != 0;
   Hybrid::useIsothermalElectrons = P.isothermal_electrons != 0;
   Hybrid::electronPressureCoeff = P.electron_pressure_coeff;
   Hybrid::useGravity = P.use_gravity != 0;
   Hybrid::GMdt = P.GMdt;
   Hybrid::maxIonSpeed2 = P.max_ion_speed2;
   Hybrid::maxElectronSpeed2 = P.max_electron_speed2;
   Hybrid::minIonChargeDensity = P.min_ion_charge_density;
   Hybrid::maxElectricField2 = P.max_electric_field2;
   Hybrid::maxWhistlerSpeed = P.max_whistler_speed;
   Hybrid::useInitialFlowThrough = P.use_initial_flow_through != 0;
   Hybrid::initialFlowThroughPeriod = P.initial_flow_through_period;
   Hybrid::N_linearSmoothingsNodeE = P.n_linear_smoothings_nodeE;
   Hybrid::useGaussianSmoothingNodeE = P.use_gaussian_smoothing_nodeE != 0;
   for (int l=0;l<4;++l) Hybrid::gaussianSmoothingCoeffsNodeE[l] = P.gaussian_coeffs[l];
   Hybrid::IMFBx = P.imf_B[0]; Hybrid::IMFBy = P.imf_B[1]; Hybrid::IMFBz = P.imf_B[2];
   for (int l=0;l<6;++l) {
      Hybrid::IMFBoundaryCellB[l] = P.imf_boundary_cellB[l] != 0;
      Hybrid::IMFBoundaryFaceB[l] = P.imf_boundary_faceB[l] != 0;
   }
   Hybrid::N_populations = c.nspecies;
   Hybrid::N_outputPopVars = 0;
   Hybrid::outputPopVarId.assign(MAX_SPECIES,-1);
   Hybrid::logCounterParticleMaxVi.assign(MAX_SPECIES,0.0);
   Hybrid::logCounterParticleEscape.assign(MAX_SPECIES,0.0);
   Hybrid::logCounterParticleEscapeKineticEnergy.assign(MAX_SPECIES,0.0);
   Hybrid::logCounterParticleImpact.assign(MAX_SPECIES,0.0);
   Hybrid::logCounterParticleImpactKineticEnergy.assign(MAX_SPECIES,0.0);
   Hybrid::logCounterParticleInject.assign(MAX_SPECIES,0.0);
   Hybrid::logCounterParticleInjectMacroparticles.assign(MAX_SPECIES,0.0);
   Hybrid::logCounterParticleInjectKineticEnergy.assign(MAX_SPECIES,0.0);
   Hybrid::logCounterFieldMaxCellUe = 0;
   Hybrid::logCounterFieldMaxNodeUe = 0;
   Hybrid::logCounterFieldMaxVw = 0;
   Hybrid::logCounterFieldMaxE = 0;
   Hybrid::logCounterFieldMinCellRhoQi = 0;
   Hybrid::logCounterFieldMinNodeRhoQi = 0;
   Hybrid::gridTemporalAverageCounter = 0;
   Hybrid::filterParticlesAfterRestartDone = true;
   Hybrid::accumulationStencilID = pargrid::DEFAULT_STENCIL;
}

void migrate(RefCtx& c,int s) {
   /* the particle lists are rebuilt in the canonical order of
    * rh_migrate_canonical (oracle_common.h): destination cell, then
    * rh_dir_rank of the direction the particle came from (stayers first),
    * then the order inside the source cell */
   pargrid::DataWrapper<PARTICLE> w = c.sc.pargrid.getUserDataDynamic<PARTICLE>(c.particleIDs[s]);
   const int nx = c.P.nx, ny = c.P.ny, nz = c.P.nz;
   const size_t N = (size_t)nx*ny*nz;
   std::vector<unsigned int>& cnt = c.counts[s];
   std::vector<PARTICLE> all;
   std::vector<int64_t> key;
   for (size_t sb=0;sb<N;++sb) {
      const int si = (int)(sb % nx), sj = (int)((sb/nx) % ny), sk = (int)(sb/((size_t)nx*ny));
      for (unsigned int p=0;p<cnt[sb];++p) {
         PARTICLE q = w.data()[sb][p];
         Real r[3] = {q.state[particle::X],q.state[particle::Y],q.state[particle::Z]};
         int off[3];
         const int st = rh_migrate_canonical(r,c.P.dx,c.dxBelow,off);
         int ti = si+off[0], tj = sj+off[1], tk = sk+off[2];
         const bool inside = rh_wrap(&ti,nx,c.P.periodic[0]) && rh_wrap(&tj,ny,c.P.periodic[1]) && rh_wrap(&tk,nz,c.P.periodic[2]);
         if (st != 0 || !inside) {
            /* left a non-periodic box, or moved more than one cell: removed */
            const Real ww = q.state[particle::WEIGHT];
            Hybrid::logCounterParticleEscape[s] += ww;
            Hybrid::logCounterParticleEscapeKineticEnergy[s] += ww*( sqr(q.state[particle::VX]) + sqr(q.state[particle::VY]) + sqr(q.state[particle::VZ]) );
            if (st != 0) c.escapeFast += 1;
            continue;
         }
         q.state[particle::X] = r[0]; q.state[particle::Y] = r[1]; q.state[particle::Z] = r[2];
         const int dir = rh_dir_rank(rh_dir_from_offset(-off[0],-off[1],-off[2]));
         const size_t d = (size_t)ti + nx*((size_t)tj + ny*(size_t)tk);
         all.push_back(q);
         key.push_back((int64_t)d*27 + dir);
      }
   }
   /* stable counting sort by key */
   std::vector<int64_t> start(N*27+1,0);
   for (int64_t k: key) start[k+1]++;
   for (size_t i=0;i<N*27;++i) start[i+1] += start[i];
   std::vector<PARTICLE> sorted(all.size());
   std::vector<int64_t> pos(start.begin(),start.end()-1);
   for (size_t i=0;i<all.size();++i) sorted[pos[key[i]]++] = all[i];
   for (size_t b=0;b<N;++b) {
      const int64_t a = start[b*27], e = start[b*27+27];
      w.resize((pargrid::CellID)b,(size_t)(e-a));
      if (e > a) std::memcpy(w.data()[b],&sorted[a],(size_t)(e-a)*sizeof(PARTICLE));
      cnt[b] = (unsigned int)(e-a);
   }
}

int arrayDim(int id) {
   switch (id) {
      case RHGPU_CELL_RHOQI: case RHGPU_NODE_RHOQI: case RHGPU_NODE_ETA: return 1;
      default: return 3;
   }
}

}  // namespace

extern "C" {

const char* rhref_last_error(void) { return g_err.c_str(); }

int rhref_create(const rhgpu_params* params,int32_t n_species,const rhgpu_species* sp,const int64_t*,int32_t,void** out) {
   if (g_active) return fail(RHGPU_ERR_STATE,"rhref: only one context at a time (reference state is static)");
   if (!params || !out || n_species < 1 || n_species > MAX_SPECIES) return fail(RHGPU_ERR_ARG,"rhref_create: bad arguments");
   RefCtx* c = new RefCtx();
   c->P = *params;
   const rhgpu_params& P = c->P;
   c->sim.dt = P.dt;
   c->sim.t = P.t_initial;
   c->sim.timestep = 0;
   c->sim.x_min = P.x_min; c->sim.y_min = P.y_min; c->sim.z_min = P.z_min;
   c->sim.x_max = P.x_min + P.nx*P.dx; c->sim.y_max = P.y_min + P.ny*P.dx; c->sim.z_max = P.z_min + P.nz*P.dx;
   c->sim.x_blocks = P.nx; c->sim.y_blocks = P.ny; c->sim.z_blocks = P.nz;
   int per[3] = {P.periodic[0],P.periodic[1],P.periodic[2]};
   c->sc.pargrid.build(P.nx,P.ny,P.nz,per);
   const size_t N = (size_t)P.nx*P.ny*P.nz;
   c->sc.blockCoordinates.resize(3*N);
   c->sc.blockSizes.resize(3*N);
   for (size_t b=0;b<N;++b) {
      const int i = (int)(b % P.nx), j = (int)((b/P.nx) % P.ny), k = (int)(b/((size_t)P.nx*P.ny));
      c->sc.blockCoordinates[3*b+0] = rh_block_origin(P.x_min,i,P.dx);
      c->sc.blockCoordinates[3*b+1] = rh_block_origin(P.y_min,j,P.dx);
      c->sc.blockCoordinates[3*b+2] = rh_block_origin(P.z_min,k,P.dx);
      for (int l=0;l<3;++l) c->sc.blockSizes[3*b+l] = P.dx;
   }
   pargrid::ParGrid& pg = c->sc.pargrid;
   Hybrid::dataFaceBID     = pg.addUserDataStatic<Real>(3);
   Hybrid::dataFaceJID     = pg.addUserDataStatic<Real>(3);
   Hybrid::dataCellRhoQiID = pg.addUserDataStatic<Real>(1);
   Hybrid::dataCellBID     = pg.addUserDataStatic<Real>(3);
   Hybrid::dataCellJID     = pg.addUserDataStatic<Real>(3);
   Hybrid::dataCellUeID    = pg.addUserDataStatic<Real>(3);
   Hybrid::dataCellJiID    = pg.addUserDataStatic<Real>(3);
   Hybrid::dataCellEpID    = pg.addUserDataStatic<Real>(3);
   Hybrid::dataNodeRhoQiID = pg.addUserDataStatic<Real>(1);
   Hybrid::dataNodeEID     = pg.addUserDataStatic<Real>(3);
   Hybrid::dataNodeBID     = pg.addUserDataStatic<Real>(3);
   Hybrid::dataNodeJID     = pg.addUserDataStatic<Real>(3);
   Hybrid::dataNodeUeID    = pg.addUserDataStatic<Real>(3);
   Hybrid::dataNodeJiID    = pg.addUserDataStatic<Real>(3);
   Hybrid::dataNodeEtaID   = pg.addUserDataStatic<Real>(1);
   Hybrid::dataInnerFlagFieldID    = pg.addUserDataStatic<bool>(1);
   Hybrid::dataInnerFlagNodeID     = pg.addUserDataStatic<bool>(1);
   Hybrid::dataInnerFlagParticleID = pg.addUserDataStatic<bool>(1);
   Hybrid::dataInnerFlagCellEpID   = pg.addUserDataStatic<bool>(1);
   Hybrid::dataCellAverageBID      = pg.addUserDataStatic<Real>(3);
#ifdef USE_GRID_CONSTRAINT_COUNTERS
   Hybrid::dataGridCounterCellMaxUeID    = pg.addUserDataStatic<Real>(1);
   Hybrid::dataGridCounterCellMaxViID    = pg.addUserDataStatic<Real>(1);
   Hybrid::dataGridCounterCellMinRhoQiID = pg.addUserDataStatic<Real>(1);
   Hybrid::dataGridCounterNodeMaxEID     = pg.addUserDataStatic<Real>(1);
   Hybrid::dataGridCounterNodeMaxVwID    = pg.addUserDataStatic<Real>(1);
#endif
   c->arrayIDs[RHGPU_FACE_B] = Hybrid::dataFaceBID;
   c->arrayIDs[RHGPU_CELL_B] = Hybrid::dataCellBID;
   c->arrayIDs[RHGPU_CELL_UE] = Hybrid::dataCellUeID;
   c->arrayIDs[RHGPU_CELL_EP] = Hybrid::dataCellEpID;
   c->arrayIDs[RHGPU_CELL_RHOQI] = Hybrid::dataCellRhoQiID;
   c->arrayIDs[RHGPU_CELL_JI] = Hybrid::dataCellJiID;
   c->arrayIDs[RHGPU_CELL_J] = Hybrid::dataCellJID;
   c->arrayIDs[RHGPU_NODE_RHOQI] = Hybrid::dataNodeRhoQiID;
   c->arrayIDs[RHGPU_NODE_JI] = Hybrid::dataNodeJiID;
   c->arrayIDs[RHGPU_NODE_J] = Hybrid::dataNodeJID;
   c->arrayIDs[RHGPU_NODE_UE] = Hybrid::dataNodeUeID;
   c->arrayIDs[RHGPU_NODE_B] = Hybrid::dataNodeBID;
   c->arrayIDs[RHGPU_NODE_E] = Hybrid::dataNodeEID;
   c->arrayIDs[RHGPU_NODE_ETA] = Hybrid::dataNodeEtaID;
   c->arrayIDs[RHGPU_CELL_AVERAGE_B] = Hybrid::dataCellAverageBID;
   c->dxBelow = std::nextafter(P.dx,0.0);

   c->nspecies = n_species;
   c->species.resize(n_species);
   c->plists.resize(MAX_SPECIES);
   c->counts.assign(n_species,std::vector<unsigned int>(N,0));
   for (int s=0;s<n_species;++s) {
      Species& S = c->species[s];
      S.name = "pop" + std::to_string(s+1);
      S.q = sp[s].q; S.m = sp[s].m; S.q_per_m = sp[s].q/sp[s].m;
      S.R2_obstacle = sp[s].R2_obstacle;
      S.popid = s+1;
      S.accumulate = sp[s].accumulate != 0;
      S.accelerate = sp[s].accelerate != 0;
      c->particleIDs.push_back(pg.addUserDataDynamic<PARTICLE>());
      c->plists[s].particleDataID = c->particleIDs[s];
   }
   setHybridStatics(*c);
   Accumulator* pool = accumulatorPool();
   for (int s=0;s<MAX_SPECIES;++s) {
      c->plists[s].species = &c->species[s < n_species ? s : 0];
      pool[s].initialize(c->sim,c->sc,c->cr,"",&c->plists[s]);
   }
   for (int s=0;s<n_species;++s) {
      c->bb[s].initialize(c->sim,c->sc,c->cr,"",&c->plists[s]);
      c->bc[s].initialize(c->sim,c->sc,c->cr,"",&c->plists[s]);
   }
   g_active = c;
   *out = c;
   return RHGPU_OK;
}

int rhref_destroy(void* h) {
   RefCtx* c = (RefCtx*)h;
   if (!c) return RHGPU_OK;
   if (g_active == c) g_active = nullptr;
   delete c;
   return RHGPU_OK;
}

int rhref_upload_array(void* h,int32_t id,const double* host) {
   RefCtx* c = (RefCtx*)h;
   if (id < 0 || id >= RHGPU_NUM_ARRAYS) return fail(RHGPU_ERR_ARG,"bad array id");
   const size_t n = (size_t)c->sc.pargrid.getNumberOfAllCells()*arrayDim(id);
   std::memcpy(c->sc.pargrid.getUserDataStatic<Real>(c->arrayIDs[id]),host,n*sizeof(Real));
   return RHGPU_OK;
}

int rhref_download_array(void* h,int32_t id,double* host) {
   RefCtx* c = (RefCtx*)h;
   if (id < 0 || id >= RHGPU_NUM_ARRAYS) return fail(RHGPU_ERR_ARG,"bad array id");
   const size_t n = (size_t)c->sc.pargrid.getNumberOfAllCells()*arrayDim(id);
   std::memcpy(host,c->sc.pargrid.getUserDataStatic<Real>(c->arrayIDs[id]),n*sizeof(Real));
   return RHGPU_OK;
}

int rhref_upload_cell_flags(void* h,const uint8_t* flags) {
   RefCtx* c = (RefCtx*)h;
   pargrid::ParGrid& pg = c->sc.pargrid;
   bool* f0 = pg.getUserDataStatic<bool>(Hybrid::dataInnerFlagFieldID);
   bool* f1 = pg.getUserDataStatic<bool>(Hybrid::dataInnerFlagNodeID);
   bool* f2 = pg.getUserDataStatic<bool>(Hybrid::dataInnerFlagParticleID);
   bool* f3 = pg.getUserDataStatic<bool>(Hybrid::dataInnerFlagCellEpID);
   for (size_t b=0;b<pg.getNumberOfAllCells();++b) {
      f0[b] = (flags[b] & RHGPU_FLAG_INNER_FIELD) != 0;
      f1[b] = (flags[b] & RHGPU_FLAG_INNER_NODE) != 0;
      f2[b] = (flags[b] & RHGPU_FLAG_INNER_PARTICLE) != 0;
      f3[b] = (flags[b] & RHGPU_FLAG_INNER_CELLEP) != 0;
   }
   return RHGPU_OK;
}

int rhref_upload_particles(void* h,int32_t s,const uint32_t* counts,const double* particles,int64_t n) {
   RefCtx* c = (RefCtx*)h;
   if (s < 0 || s >= c->nspecies) return fail(RHGPU_ERR_ARG,"bad species");
   pargrid::DataWrapper<PARTICLE> w = c->sc.pargrid.getUserDataDynamic<PARTICLE>(c->particleIDs[s]);
   const size_t N = c->sc.pargrid.getNumberOfAllCells();
   int64_t off = 0;
   for (size_t b=0;b<N;++b) {
      w.resize((pargrid::CellID)b,counts[b]);
      if (off + (int64_t)counts[b] > n) return fail(RHGPU_ERR_ARG,"counts exceed n_particles");
      if (counts[b]) std::memcpy(w.data()[b],particles + 7*off,(size_t)counts[b]*sizeof(PARTICLE));
      off += counts[b];
      c->counts[s][b] = counts[b];
   }
   if (off != n) return fail(RHGPU_ERR_ARG,"sum(counts) != n_particles");
   return RHGPU_OK;
}

int rhref_num_particles(void* h,int32_t s,int64_t* n) {
   RefCtx* c = (RefCtx*)h;
   int64_t t = 0;
   for (unsigned int x: c->counts[s]) t += x;
   *n = t;
   return RHGPU_OK;
}

int rhref_download_particles(void* h,int32_t s,uint32_t* counts,double* particles,int64_t cap,int64_t* n_out) {
   RefCtx* c = (RefCtx*)h;
   pargrid::DataWrapper<PARTICLE> w = c->sc.pargrid.getUserDataDynamic<PARTICLE>(c->particleIDs[s]);
   int64_t tot = 0;
   for (unsigned int x: c->counts[s]) tot += x;
   if (tot > cap) return fail(RHGPU_ERR_ARG,"capacity too small");
   int64_t off = 0;
   for (size_t b=0;b<c->counts[s].size();++b) {
      counts[b] = c->counts[s][b];
      if (counts[b]) std::memcpy(particles + 7*off,w.data()[b],(size_t)counts[b]*sizeof(PARTICLE));
      off += counts[b];
   }
   *n_out = tot;
   return RHGPU_OK;
}

int rhref_push(void* h) {
   RefCtx* c = (RefCtx*)h;
   Simulation& sim = c->sim;
   sim.timestep += 1;
   /* user.cpp:52-59 */
   if (Hybrid::initialFlowThroughPeriod < sim.t && Hybrid::useInitialFlowThrough == true) Hybrid::useInitialFlowThrough = false;
   setupGetFields(sim,c->sc);
   const std::vector<pargrid::CellID>& cells = c->sc.pargrid.getInnerCells(pargrid::DEFAULT_STENCIL);
   const Real* crd = getBlockCoordinateArray(sim,c->sc);
   for (int s=0;s<c->nspecies;++s) {
      for (pargrid::CellID b: cells) {
         if (c->counts[s][b] == 0) continue;
         c->bb[s].propagateCell(b,c->particleIDs[s],crd,c->counts[s][b]);
      }
      migrate(*c,s);
   }
   return RHGPU_OK;
}

int rhref_accumulate(void* h) {
   RefCtx* c = (RefCtx*)h;
   Accumulator* pool = accumulatorPool();
   for (int s=0;s<c->nspecies;++s) pool[s].clearAccumulationArrays();
   for (int s=0;s<c->nspecies;++s) pool[s].accumulateBoundaryCells(c->particleIDs[s],c->counts[s].data());
   for (int s=0;s<c->nspecies;++s) pool[s].accumulateInnerCells(c->particleIDs[s],c->counts[s].data());
   for (int s=0;s<MAX_SPECIES;++s) { pool[s].sendUpdates(); pool[s].wait(); }
   pool[MAX_SPECIES-1].addRemoteUpdates();
   return RHGPU_OK;
}

int rhref_apply_boundaries(void* h) {
   RefCtx* c = (RefCtx*)h;
   const std::vector<pargrid::CellID>& ext = c->sc.pargrid.getExteriorCells();
   for (int s=0;s<c->nspecies;++s) c->bc[s].apply(c->particleIDs[s],c->counts[s].data(),ext);
   return RHGPU_OK;
}

int rhref_propagate_fields(void* h) {
   RefCtx* c = (RefCtx*)h;
   std::vector<ParticleListBase*> lists;
   propagateB(c->sim,c->sc,lists);
   c->sim.t += c->sim.dt;
   return RHGPU_OK;
}

int rhref_step(void* h,int32_t nsteps) {
   for (int n=0;n<nsteps;++n) {
      rhref_push(h);
      rhref_accumulate(h);
      rhref_apply_boundaries(h);
      rhref_propagate_fields(h);
   }
   return RHGPU_OK;
}

int rhref_get_counters(void* h,double* out,int32_t n) {
   RefCtx* c = (RefCtx*)h;
   std::vector<double> v(RHGPU_NUM_FIELD_COUNTERS + RHGPU_CNT_PER_SPECIES*c->nspecies,0.0);
   v[RHGPU_CNT_FIELD_MIN_CELL_RHOQI] = Hybrid::logCounterFieldMinCellRhoQi;
   v[RHGPU_CNT_FIELD_MAX_CELL_UE] = Hybrid::logCounterFieldMaxCellUe;
   v[RHGPU_CNT_FIELD_MAX_NODE_UE] = Hybrid::logCounterFieldMaxNodeUe;
   v[RHGPU_CNT_FIELD_MAX_VW] = Hybrid::logCounterFieldMaxVw;
   v[RHGPU_CNT_FIELD_MAX_E] = Hybrid::logCounterFieldMaxE;
   v[RHGPU_CNT_FIELD_MIN_NODE_RHOQI] = Hybrid::logCounterFieldMinNodeRhoQi;
   v[RHGPU_CNT_GRID_AVERAGE_COUNTER] = Hybrid::gridTemporalAverageCounter;
   for (int s=0;s<c->nspecies;++s) {
      double* q = &v[RHGPU_NUM_FIELD_COUNTERS + RHGPU_CNT_PER_SPECIES*s];
      q[0] = Hybrid::logCounterParticleMaxVi[s];
      q[1] = Hybrid::logCounterParticleEscape[s];
      q[2] = Hybrid::logCounterParticleEscapeKineticEnergy[s];
      q[3] = Hybrid::logCounterParticleImpact[s];
      q[4] = Hybrid::logCounterParticleImpactKineticEnergy[s];
   }
   for (int i=0;i<n && i<(int)v.size();++i) out[i] = v[i];
   return RHGPU_OK;
}

/* the log files of logWriteParticleField: pop<NNN>_<name>.log and field.log in
 * cfg->directory, number format as src/user.cpp:2158-2187 sets it, no headers */
int rhref_log_open(void* h,const rhgpu_log_config* cfg) {
   RefCtx* c = (RefCtx*)h;
   if (!cfg || !cfg->directory || !cfg->species_names) return fail(RHGPU_ERR_ARG,"rhref_log_open: bad arguments");
   for (std::ofstream* o: Hybrid::logParticle) delete o;
   Hybrid::logParticle.clear();
   if (Hybrid::logField.is_open()) Hybrid::logField.close();
   const int prec = cfg->precision > 0 ? cfg->precision : 10;
   for (int s=0;s<c->nspecies;++s) {
      const std::string zero = s < 10 ? "00" : (s < 100 ? "0" : "");
      const std::string fn = std::string(cfg->directory) + "/pop" + zero + std::to_string(s+1) + "_" + cfg->species_names[s] + ".log";
      Hybrid::logParticle.push_back(new std::ofstream(fn.c_str(),std::ios_base::out));
      Hybrid::logParticle.back()->precision(prec);
      (*Hybrid::logParticle.back()) << std::scientific << std::showpos;
   }
   Hybrid::logField.open((std::string(cfg->directory) + "/field.log").c_str(),std::ios_base::out);
   Hybrid::logField.precision(prec);
   Hybrid::logField << std::scientific << std::showpos;
   Hybrid::includeInnerCellsInFieldLog = cfg->include_inner_cells != 0;
   Hybrid::maxBStopRun = cfg->max_B_stop_run;
   Hybrid::writeMainLogDiagnosticsAfterLogStep = false;
   Hybrid::logCounterTimeStart = c->sim.t;
   for (int s=0;s<MAX_SPECIES;++s) {
      Hybrid::logCounterParticleEscape[s] = 0; Hybrid::logCounterParticleImpact[s] = 0;
      Hybrid::logCounterParticleInject[s] = 0; Hybrid::logCounterParticleInjectMacroparticles[s] = 0;
      Hybrid::logCounterParticleEscapeKineticEnergy[s] = 0; Hybrid::logCounterParticleImpactKineticEnergy[s] = 0;
      Hybrid::logCounterParticleInjectKineticEnergy[s] = 0; Hybrid::logCounterParticleMaxVi[s] = 0;
   }
   Hybrid::logCounterFieldMaxCellUe = 0; Hybrid::logCounterFieldMaxNodeUe = 0; Hybrid::logCounterFieldMaxVw = 0;
   Hybrid::logCounterFieldMaxE = 0; Hybrid::logCounterFieldMinCellRhoQi = 0; Hybrid::logCounterFieldMinNodeRhoQi = 0;
   return RHGPU_OK;
}

int rhref_log_write(void* h,int32_t main_log,int32_t* stop_run,char* messages,int32_t cap) {
   RefCtx* c = (RefCtx*)h;
   if (Hybrid::logParticle.size() != (size_t)c->nspecies) return fail(RHGPU_ERR_STATE,"rhref_log_write: rhref_log_open first");
   /* the particle lists' sizes follow the per-cell counts the plugins keep */
   std::vector<ParticleListBase*> lists;
   for (int s=0;s<c->nspecies;++s) {
      pargrid::DataWrapper<PARTICLE> w = c->sc.pargrid.getUserDataDynamic<PARTICLE>(c->particleIDs[s]);
      for (size_t b=0;b<c->counts[s].size();++b) w.resize((pargrid::CellID)b,c->counts[s][b]);
      lists.push_back(&c->plists[s]);
   }
   Hybrid::writeMainLogDiagnosticsAfterLogStep = main_log != 0;
   const bool ok = diagnostics::logWriteParticleField(c->sim,c->sc,lists);
   for (std::ofstream* o: Hybrid::logParticle) o->flush();
   Hybrid::logField.flush();
   if (stop_run) *stop_run = ok ? 0 : 1;
   if (messages && cap > 0) messages[0] = 0;
   return RHGPU_OK;
}

int rhref_log_close(void*) {
   for (std::ofstream* o: Hybrid::logParticle) { o->close(); delete o; }
   Hybrid::logParticle.clear();
   if (Hybrid::logField.is_open()) Hybrid::logField.close();
   return RHGPU_OK;
}

/* output populations of the temporal averages: the reference's own
 * accumulateCell adds into their sums (particle_accumulator.cpp:148-150) */
int rhref_set_population_averages(void* h,int32_t n_groups,const int32_t* group) {
   RefCtx* c = (RefCtx*)h;
   pargrid::ParGrid& pg = c->sc.pargrid;
   Hybrid::outputPopVarId.assign(MAX_SPECIES,-1);
   Hybrid::outputPopVarIdVector.assign(n_groups,std::vector<unsigned int>());
   Hybrid::dataCellAverageDensityID.clear();
   Hybrid::dataCellAverageVelocityID.clear();
   for (int m=0;m<n_groups;++m) {
      Hybrid::dataCellAverageDensityID.push_back(pg.addUserDataStatic<Real>(1));
      Hybrid::dataCellAverageVelocityID.push_back(pg.addUserDataStatic<Real>(3));
   }
   for (int s=0;s<c->nspecies;++s) {
      if (group[s] < -1 || group[s] >= n_groups) return fail(RHGPU_ERR_ARG,"group index out of range");
      Hybrid::outputPopVarId[s] = group[s];
      if (group[s] >= 0) Hybrid::outputPopVarIdVector[group[s]].push_back(s);
   }
   Hybrid::N_outputPopVars = n_groups;
   return RHGPU_OK;
}

/* the output step's averages, restated from UserDataOP::writeData
 * (operator_userdata.cpp:155-223) over the reference's sums */
int rhref_output_averages(void* h,double* cellB,double* nOut,double* vOut) {
   RefCtx* c = (RefCtx*)h;
   pargrid::ParGrid& pg = c->sc.pargrid;
   const size_t N = pg.getNumberOfLocalCells();
   Real inv = 0.0;
   if (Hybrid::gridTemporalAverageCounter > 0) inv = 1.0/static_cast<Real>(Hybrid::gridTemporalAverageCounter);
   if (cellB) {
      Real* a = pg.getUserDataStatic<Real>(Hybrid::dataCellAverageBID);
      for (size_t n=0;n<N;++n) for (int l=0;l<3;++l) { cellB[3*n+l] = a[3*n+l]*inv; a[3*n+l] = 0.0; }
   }
   if (nOut || vOut) {
      for (unsigned int m=0;m<Hybrid::N_outputPopVars;++m) {
         Real* nA = pg.getUserDataStatic<Real>(Hybrid::dataCellAverageDensityID[m]);
         Real* vA = pg.getUserDataStatic<Real>(Hybrid::dataCellAverageVelocityID[m]);
         const Real q = c->species[Hybrid::outputPopVarIdVector[m][0]].q;
         for (size_t n=0;n<N;++n) {
            if (nOut) nOut[m*N + n] = nA[n]/(q*Hybrid::dV)*inv;
            for (int l=0;l<3;++l) {
               if (vOut) vOut[(m*N + n)*3 + l] = nA[n] > 0 ? vA[3*n+l]/nA[n] : 0.0;
               vA[3*n+l] = 0.0;
            }
            nA[n] = 0.0;
         }
      }
   }
   Hybrid::gridTemporalAverageCounter = 0;
   return RHGPU_OK;
}

#ifdef USE_GRID_CONSTRAINT_COUNTERS
/* the reference's per-cell constraint counters (built with
 * USE_GRID_CONSTRAINT_COUNTERS): zeroed here, read in the planes order of
 * rhgpu_download_grid_counters */
int rhref_set_grid_counters(void* h,int32_t) {
   RefCtx* c = (RefCtx*)h;
   pargrid::ParGrid& pg = c->sc.pargrid;
   const pargrid::DataID ids[5] = {Hybrid::dataGridCounterCellMaxUeID,Hybrid::dataGridCounterCellMaxViID,
                                   Hybrid::dataGridCounterCellMinRhoQiID,Hybrid::dataGridCounterNodeMaxEID,
                                   Hybrid::dataGridCounterNodeMaxVwID};
   for (int q=0;q<5;++q) {
      Real* a = pg.getUserDataStatic<Real>(ids[q]);
      for (size_t n=0;n<pg.getNumberOfAllCells();++n) a[n] = 0.0;
   }
   return RHGPU_OK;
}

int rhref_download_grid_counters(void* h,double* out) {
   RefCtx* c = (RefCtx*)h;
   pargrid::ParGrid& pg = c->sc.pargrid;
   const pargrid::DataID ids[5] = {Hybrid::dataGridCounterCellMaxUeID,Hybrid::dataGridCounterCellMaxViID,
                                   Hybrid::dataGridCounterCellMinRhoQiID,Hybrid::dataGridCounterNodeMaxEID,
                                   Hybrid::dataGridCounterNodeMaxVwID};
   const size_t N = pg.getNumberOfAllCells();
   for (int q=0;q<5;++q) std::memcpy(out + q*N,pg.getUserDataStatic<Real>(ids[q]),N*sizeof(Real));
   return RHGPU_OK;
}
#endif

/* The reference's own output operator, UserDataOP::writeData
 * (src/operator_userdata.cpp:55-312), run on the current state; the VLSV
 * stub of the shim keeps the arrays it writes. `params`: space-separated
 * output parameter names (Hybrid.output_parameters, user.cpp:2302-2343);
 * `group_names`: space-separated names of the output populations
 * (outputPopVarStr) of rhref_set_population_averages. The arrays are read
 * back with rhref_data_count / rhref_data_info / rhref_data_get. */
int rhref_write_data(void* h,const char* params,const char* group_names) {
   RefCtx* c = (RefCtx*)h;
   Hybrid::outputCellParams.clear();
   std::istringstream ps(params ? params : "");
   for (std::string w; ps >> w; ) Hybrid::outputCellParams[w] = true;
   Hybrid::outputPopVarStr.clear();
   std::istringstream gs(group_names ? group_names : "");
   for (std::string w; gs >> w; ) Hybrid::outputPopVarStr.push_back(w);
   if (Hybrid::outputPopVarStr.size() != Hybrid::N_outputPopVars)
      return fail(RHGPU_ERR_ARG,"rhref_write_data: one name per output population");
   std::vector<ParticleListBase*> lists;
   for (int s=0;s<c->nspecies;++s) {
      pargrid::DataWrapper<PARTICLE> w = c->sc.pargrid.getUserDataDynamic<PARTICLE>(c->particleIDs[s]);
      for (size_t b=0;b<c->counts[s].size();++b) w.resize((pargrid::CellID)b,c->counts[s][b]);
      lists.push_back(&c->plists[s]);
   }
   UserDataOP op;
   op.initialize(c->cr,c->sim,c->sc);
   c->sc.vlsv.arrays.clear();
   c->sc.vlsv.capture = true;
   const bool ok = op.writeData("SpatialGrid",lists);
   c->sc.vlsv.capture = false;
   return ok ? RHGPU_OK : fail(RHGPU_ERR_STATE,"rhref_write_data: writeData failed");
}

int rhref_data_count(void* h) { return (int)((RefCtx*)h)->sc.vlsv.arrays.size(); }

int rhref_data_info(void* h,int32_t i,char* name,int32_t cap,int64_t* arraySize,int64_t* vectorSize) {
   RefCtx* c = (RefCtx*)h;
   if (i < 0 || (size_t)i >= c->sc.vlsv.arrays.size() || cap < 1) return fail(RHGPU_ERR_ARG,"rhref_data_info: bad index");
   const VlsvArray& a = c->sc.vlsv.arrays[i];
   auto it = a.attribs.find("name");
   std::snprintf(name,cap,"%s",it == a.attribs.end() ? "" : it->second.c_str());
   *arraySize = (int64_t)a.arraySize;
   *vectorSize = (int64_t)a.vectorSize;
   return RHGPU_OK;
}

int rhref_data_get(void* h,int32_t i,double* out) {
   RefCtx* c = (RefCtx*)h;
   if (i < 0 || (size_t)i >= c->sc.vlsv.arrays.size()) return fail(RHGPU_ERR_ARG,"rhref_data_get: bad index");
   const VlsvArray& a = c->sc.vlsv.arrays[i];
   std::memcpy(out,a.data.data(),a.data.size()*sizeof(double));
   return RHGPU_OK;
}

int rhref_get_time(void* h,double* t,int64_t* ts) {
   RefCtx* c = (RefCtx*)h;
   *t = c->sim.t; *ts = c->sim.timestep;
   return RHGPU_OK;
}

}  // extern "C"

#ifdef RH_CORSAIR_ADAPTOR
/* The Corsair-side adaptor of the GPU library (rhybrid_b200/corsair/rhgpu_corsair.h)
 * driven on this driver's Corsair/ParGrid state: the plugins are made through
 * the object factories by the names a run's .cfg uses, initialized on the
 * particle lists, and called the way propagate() calls them (their per-cell
 * methods do nothing on the GPU); gpuPropagate runs each step, gpuDownload
 * brings the state back into the ParGrid containers, which rhref_download_*
 * then read. Built only into oracle/_ref/librhref_corsair.so (linked with
 * librhgpu.so). */
#include "object_factories.h"
#include "corsair/rhgpu_corsair.h"

extern "C" int rhcorsair_run(void* h, int32_t nsteps, int32_t path, int32_t device, char* err, int32_t err_cap) {
   RefCtx* c = (RefCtx*)h;
   if (!c || nsteps < 0) return fail(RHGPU_ERR_ARG, "rhcorsair_run: bad arguments");
   auto report = [&](const std::string& m) {
      if (err && err_cap > 0) { std::strncpy(err, m.c_str(), (size_t)err_cap - 1); err[err_cap - 1] = 0; }
      return fail(RHGPU_ERR_STATE, m);
   };
   ObjectFactories of;
   if (!rhgpu_corsair::registerObjectMakers<PARTICLE>(of)) return report("registerObjectMakers");
   std::vector<ParticleListBase*> lists;
   std::vector<ParticlePropagatorBase*> props;
   std::vector<ParticleAccumulatorBase*> accs;
   std::vector<ParticleBoundaryCondBase*> bcs;
   int rc = RHGPU_OK;
   for (int s = 0; s < c->nspecies; ++s) {
      lists.push_back(&c->plists[s]);
      props.push_back(of.particlePropagators.create("BorisBuneman"));
      accs.push_back(of.particleAccumulators.create("HybridAccumulator"));
      bcs.push_back(of.particleBoundaryConditions.create("HybridBoundaryCond"));
      if (!props.back() || !accs.back() || !bcs.back()) { rc = report("a plugin is not registered"); break; }
      props.back()->initialize(c->sim, c->sc, c->cr, "", &c->plists[s]);
      accs.back()->initialize(c->sim, c->sc, c->cr, "", &c->plists[s]);
      bcs.back()->initialize(c->sim, c->sc, c->cr, "", &c->plists[s]);
   }
   const int per[3] = {c->P.periodic[0], c->P.periodic[1], c->P.periodic[2]};
   if (!rc && !rhgpu_corsair::gpuSetup<PARTICLE>(c->sim, c->sc, lists, per, device, path)) rc = report(rhgpu_corsair::run().error);
   const std::vector<pargrid::CellID>& cells = c->sc.pargrid.getInnerCells(pargrid::DEFAULT_STENCIL);
   const Real* crd = getBlockCoordinateArray(c->sim, c->sc);
   for (int n = 0; n < nsteps && !rc; ++n) {
      c->sim.timestep += 1;
      for (int s = 0; s < c->nspecies; ++s) {
         pargrid::DataWrapper<PARTICLE> w = c->sc.pargrid.getUserDataDynamic<PARTICLE>(c->particleIDs[s]);
         for (pargrid::CellID b : cells)
            if (w.size()[b] > 0) props[s]->propagateCell(b, c->particleIDs[s], crd, (unsigned int)w.size()[b]);
         accs[s]->clearAccumulationArrays();
         accs[s]->accumulateBoundaryCells(c->particleIDs[s], c->counts[s].data());
         accs[s]->accumulateInnerCells(c->particleIDs[s], c->counts[s].data());
         accs[s]->addRemoteUpdates();
      }
      if (!rhgpu_corsair::gpuPropagate(c->sim, c->sc, lists)) rc = report(rhgpu_corsair::run().error);
      c->sim.t += c->sim.dt;
   }
   if (!rc && !rhgpu_corsair::gpuDownload<PARTICLE>(c->sim, c->sc, lists)) rc = report(rhgpu_corsair::run().error);
   if (!rc)
      for (int s = 0; s < c->nspecies; ++s) {
         pargrid::DataWrapper<PARTICLE> w = c->sc.pargrid.getUserDataDynamic<PARTICLE>(c->particleIDs[s]);
         for (size_t b = 0; b < c->counts[s].size(); ++b) c->counts[s][b] = (unsigned int)w.size()[b];
      }
   rhgpu_corsair::gpuFinalize();
   for (auto* p : props) delete p;
   for (auto* p : accs) delete p;
   for (auto* p : bcs) delete p;
   return rc;
}
#endif
