/* Oracle shim (test infrastructure only): Corsair ParticleListBase, reduced to
 * the species/injector accessors the RHybrid plugins call in initialize() and
 * the particle data ID the log reductions (diagnostics.h) ask for. */
#ifndef RHSHIM_PARTICLE_LIST_BASE_H
#define RHSHIM_PARTICLE_LIST_BASE_H
#include "simulationclasses.h"
class ParticleInjectorBase;
class ParticleListBase {
 public:
   virtual ~ParticleListBase() { }
   const void* getSpecies() const { return species; }
   ParticleInjectorBase* getInjector() const { return injector; }
   bool getParticles(pargrid::DataID& id) const { id = particleDataID; return particleDataID != pargrid::INVALID_DATAID; }
   pargrid::DataID particleDataID = pargrid::INVALID_DATAID;
   const void* species = nullptr;
   ParticleInjectorBase* injector = nullptr;
};
#endif
