/* Oracle shim (test infrastructure only): Corsair ParticleAccumulatorBase. */
#ifndef RHSHIM_BASE_CLASS_PARTICLE_ACCUMULATOR_H
#define RHSHIM_BASE_CLASS_PARTICLE_ACCUMULATOR_H
#include "plugin_base.h"
class ParticleAccumulatorBase: public RhShimPluginBase {
 public:
   virtual bool accumulateBoundaryCells(pargrid::DataID,const unsigned int*) = 0;
   virtual bool accumulateInnerCells(pargrid::DataID,const unsigned int*) = 0;
   virtual bool addRemoteUpdates() = 0;
   virtual bool clearAccumulationArrays() = 0;
   virtual bool sendUpdates() = 0;
   virtual bool wait() = 0;
};
#endif
