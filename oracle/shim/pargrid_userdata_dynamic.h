/* Oracle shim (test infrastructure only): DataWrapper lives in simulationclasses.h. */
#ifndef RHSHIM_PARGRID_USERDATA_DYNAMIC_H
#define RHSHIM_PARGRID_USERDATA_DYNAMIC_H
#include "simulationclasses.h"
#endif
