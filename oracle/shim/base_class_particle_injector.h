/* Oracle shim (test infrastructure only): Corsair ParticleInjectorBase
 * (declared so that particle_injector.h parses; no injector is built). */
#ifndef RHSHIM_BASE_CLASS_PARTICLE_INJECTOR_H
#define RHSHIM_BASE_CLASS_PARTICLE_INJECTOR_H
#include "plugin_base.h"
class ParticleInjectorBase: public RhShimPluginBase { };
#endif
