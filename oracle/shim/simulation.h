/* Oracle shim (test infrastructure only): the Corsair Simulation record, with
 * the members RHybrid's hot-path sources read. */
#ifndef RHSHIM_SIMULATION_H
#define RHSHIM_SIMULATION_H

#include "definitions.h"
#include "mpi.h"

struct Simulation {
   Real dt = 0;
   Real t = 0;
   unsigned int timestep = 0;
   bool atDataSaveStep = false;
   bool restarted = false;
   bool countPropagTime = false;
   int mpiRank = 0;
   int MASTER_RANK = 0;
   MPI_Comm comm = 0;
   Real x_min = 0, y_min = 0, z_min = 0, x_max = 0, y_max = 0, z_max = 0;
   int x_blocks = 0, y_blocks = 0, z_blocks = 0;
};

#endif
