/* Oracle shim (test infrastructure only): Corsair ParticlePropagatorBase. */
#ifndef RHSHIM_BASE_CLASS_PARTICLE_PROPAGATOR_H
#define RHSHIM_BASE_CLASS_PARTICLE_PROPAGATOR_H
#include "plugin_base.h"
class ParticlePropagatorBase: public RhShimPluginBase {
 public:
   virtual bool propagateCell(pargrid::CellID,pargrid::DataID,const double* const,unsigned int) = 0;
};
#endif
