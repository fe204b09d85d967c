/* Oracle shim (test infrastructure only): single-process MPI stubs for the
 * few MPI calls reachable from RHybrid's hot-path sources. Only rank 0 exists;
 * reductions copy input to output. */
#ifndef RHSHIM_MPI_H
#define RHSHIM_MPI_H

#include <cstdlib>
#include <cstring>
#include <chrono>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_INT 10
#define MPI_DOUBLE 11

template<typename T> inline MPI_Datatype MPI_Type() { return sizeof(T) == 8 ? MPI_DOUBLE : MPI_INT; }

inline int MPI_Abort(MPI_Comm,int code) { std::exit(code); return 0; }
inline int MPI_Type_contiguous(int,MPI_Datatype,MPI_Datatype* t) { *t = 0; return 0; }
inline int MPI_Reduce(const void* in,void* out,int n,MPI_Datatype t,MPI_Op,int,MPI_Comm) {
   std::memcpy(out,in,(size_t)n*(t == MPI_DOUBLE ? 8 : 4)); return 0;
}
inline int MPI_Allreduce(const void* in,void* out,int n,MPI_Datatype t,MPI_Op,MPI_Comm) {
   std::memcpy(out,in,(size_t)n*(t == MPI_DOUBLE ? 8 : 4)); return 0;
}
inline int MPI_Bcast(void*,int,MPI_Datatype,int,MPI_Comm) { return 0; }
inline double MPI_Wtime() {
   using namespace std::chrono;
   return duration<double>(steady_clock::now().time_since_epoch()).count();
}

#endif
