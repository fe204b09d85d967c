/* Oracle shim (test infrastructure only): Corsair's object factories,
 * reduced to registering a maker under a name and creating by that name. */
#ifndef RHSHIM_OBJECT_FACTORIES_H
#define RHSHIM_OBJECT_FACTORIES_H
#include <map>
#include <string>
#include "base_class_particle_accumulator.h"
#include "base_class_particle_boundary_condition.h"
#include "base_class_particle_propagator.h"
template <class BASE> class RhShimFactory {
 public:
   typedef BASE* (*Maker)();
   bool registerMaker(const std::string& name, Maker m) { return makers.emplace(name, m).second; }
   BASE* create(const std::string& name) const {
      const auto it = makers.find(name);
      return it == makers.end() ? nullptr : it->second();
   }
 private:
   std::map<std::string, Maker> makers;
};
struct ObjectFactories {
   RhShimFactory<ParticlePropagatorBase> particlePropagators;
   RhShimFactory<ParticleAccumulatorBase> particleAccumulators;
   RhShimFactory<ParticleBoundaryCondBase> particleBoundaryConditions;
};
#endif
