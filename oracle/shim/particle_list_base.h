/* Oracle shim (test infrastructure only): Corsair ParticleListBase, reduced to
 * the species/injector accessors the RHybrid plugins call in initialize(). */
#ifndef RHSHIM_PARTICLE_LIST_BASE_H
#define RHSHIM_PARTICLE_LIST_BASE_H
#include "simulationclasses.h"
class ParticleInjectorBase;
class ParticleListBase {
 public:
   virtual ~ParticleListBase() { }
   const void* getSpecies() const { return species; }
   ParticleInjectorBase* getInjector() const { return injector; }
   const void* species = nullptr;
   ParticleInjectorBase* injector = nullptr;
};
#endif
