/* Oracle shim (test infrastructure only): common part of Corsair's plugin
 * base classes; initialize() records the Simulation and SimulationClasses. */
#ifndef RHSHIM_PLUGIN_BASE_H
#define RHSHIM_PLUGIN_BASE_H
#include <string>
#include "simulation.h"
#include "simulationclasses.h"
#include "configreader.h"
#include "particle_list_base.h"
class RhShimPluginBase {
 public:
   virtual ~RhShimPluginBase() { }
   virtual bool initialize(Simulation& s,SimulationClasses& sc,ConfigReader&,const std::string&,const ParticleListBase*) {
      sim = &s; simClasses = &sc; return true;
   }
 protected:
   Simulation* sim = nullptr;
   SimulationClasses* simClasses = nullptr;
};
#endif
