/* Oracle shim (test infrastructure only): Corsair DataOperator, reduced to
 * what UserDataOP (src/operator_userdata.{h,cpp}) uses: the initialize()
 * that keeps the simulation and its classes, getInitialized(), and the
 * writeData() hook it overrides. */
#ifndef RHSHIM_DATAOPERATOR_H
#define RHSHIM_DATAOPERATOR_H
#include <string>
#include <vector>
#include "configreader.h"
#include "simulation.h"
#include "simulationclasses.h"
#include "particle_list_base.h"
class DataOperator {
 public:
   DataOperator() { }
   virtual ~DataOperator() { }
   virtual bool finalize() { return true; }
   virtual std::string getName() const = 0;
   virtual bool initialize(ConfigReader&,Simulation& s,SimulationClasses& sc) {
      sim = &s; simClasses = &sc; initialized = true; return true;
   }
   virtual bool writeData(const std::string&,const std::vector<ParticleListBase*>&) = 0;
   bool getInitialized() const { return initialized; }
 protected:
   bool initialized = false;
   Simulation* sim = nullptr;
   SimulationClasses* simClasses = nullptr;
};
#endif
