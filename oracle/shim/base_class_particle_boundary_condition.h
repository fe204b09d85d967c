/* Oracle shim (test infrastructure only): Corsair ParticleBoundaryCondBase. */
#ifndef RHSHIM_BASE_CLASS_PARTICLE_BOUNDARY_CONDITION_H
#define RHSHIM_BASE_CLASS_PARTICLE_BOUNDARY_CONDITION_H
#include "plugin_base.h"
class ParticleBoundaryCondBase: public RhShimPluginBase { };
#endif
