/* Oracle shim (test infrastructure only): a single-process stand-in for
 * Corsair's SimulationClasses and ParGrid, covering exactly the calls made by
 * RHybrid's hot-path sources (hybrid_propagator.cpp, particle_accumulator.cpp,
 * particle_propagator_boris_buneman.h, particle_boundary_cond_hybrid.h).
 *
 * Semantics restated here (Corsair/ParGrid are not vendored):
 *  - one process owns every cell; local ID == linear index i + nx*(j + ny*k);
 *  - neighbour type ID of offset (i,j,k) is (k+1)*9 + (j+1)*3 + (i+1);
 *    neighbour flag bit t is set when neighbour type t exists (itself
 *    included), so ALL_NEIGHBOURS_EXIST has 27 bits set;
 *  - non-periodic axes have no neighbour beyond the first/last cell; cells
 *    missing any neighbour are the exterior cells;
 *  - every local cell is an inner cell of every stencil, in increasing ID
 *    order; there are no boundary (remote-neighbour) cells;
 *  - halo exchanges are no-ops (there are no remote copies);
 *  - block::addValues3D adds the 27 entries of a 3x3x3 array into the 27
 *    neighbours of a cell, skipping neighbours that do not exist.
 */
#ifndef RHSHIM_SIMULATIONCLASSES_H
#define RHSHIM_SIMULATIONCLASSES_H

#include <cstdint>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>
#include <map>
#include <limits>
#include <memory>
#include <algorithm>
#include <climits>
#include <fstream>
#include <cmath>

#include "definitions.h"
#include "mpi.h"
#include "simulation.h"
#include "../../include/rhgpu.h"

namespace constants {
   const Real PERMEABILITY      = RHGPU_PERMEABILITY;
   const Real CHARGE_ELEMENTARY = RHGPU_CHARGE_ELEMENTARY;
   const Real MASS_PROTON       = RHGPU_MASS_PROTON;
   const Real BOLTZMANN         = RHGPU_BOLTZMANN;
   const Real GRAVITY           = RHGPU_GRAVITY;
   const Real EV_TO_KELVIN      = 11604.51812;
   const Real MASS_ELECTRON     = RHGPU_MASS_ELECTRON;
   const Real PERMITTIVITY      = RHGPU_PERMITTIVITY;
   const Real SPEED_LIGHT       = RHGPU_SPEED_OF_LIGHT;
}

namespace profile {
   inline bool start(const std::string&,int&) { return true; }
   inline bool stop() { return true; }
}

/* Logger: discards output unless RHSHIM_VERBOSE is set in the environment. */
class Logger {
 public:
   template<class T> Logger& operator<<(const T& x) { if (verbose()) std::cerr << x; return *this; }
   Logger& operator<<(std::ostream& (*f)(std::ostream&)) { if (verbose()) std::cerr << f; return *this; }
   Logger& operator<<(Logger& (*f)(Logger&)) { return f(*this); }
   static bool verbose() { static int v = -1; if (v < 0) v = std::getenv("RHSHIM_VERBOSE") ? 1 : 0; return v == 1; }
};
inline Logger& write(Logger& l) { if (Logger::verbose()) std::cerr << std::flush; return l; }

/* Corsair RNG stand-in: only referenced by magnetic-field profiles that the
 * oracle does not evaluate on the hot path. */
struct Random {
   uint64_t s = 6461674ull;
   Real uniform() { s = s*6364136223846793005ull + 1442695040888963407ull; return (Real)(s >> 11)*(1.0/9007199254740992.0); }
   Real uniformPM() { return 2.0*uniform() - 1.0; }
};

namespace pargrid {
   typedef uint32_t CellID;
   typedef unsigned int DataID;
   typedef unsigned int StencilID;
   typedef size_t ArraySizetype;
   const StencilID DEFAULT_STENCIL = 0;
   const StencilID INVALID_STENCILID = std::numeric_limits<StencilID>::max();
   const DataID INVALID_DATAID = std::numeric_limits<DataID>::max();
   const uint32_t ALL_NEIGHBOURS_EXIST = (1u << 27) - 1u;

   /* per-cell dynamic arrays (particle lists) */
   struct DynamicStore {
      size_t elemSize = 0;
      std::vector<std::vector<char> > cells;
      std::vector<char*> ptrs;
      std::vector<size_t> sizes;
   };

   template<class T> class DataWrapper {
    public:
      explicit DataWrapper(DynamicStore* s = nullptr): store(s) { }
      T** data() const { return reinterpret_cast<T**>(store->ptrs.data()); }
      const size_t* size() const { return store->sizes.data(); }
      size_t size(CellID b) const { return store->sizes[b]; }
      bool resize(CellID b,size_t n) {
         store->cells[b].resize(n*sizeof(T) + 16);
         store->ptrs[b] = store->cells[b].data();
         store->sizes[b] = n;
         return true;
      }
    private:
      DynamicStore* store;
   };

   class ParGrid {
    public:
      void build(int nx_,int ny_,int nz_,const int periodic_[3]) {
         nx = nx_; ny = ny_; nz = nz_;
         for (int a=0;a<3;++a) periodic[a] = periodic_[a];
         const size_t N = (size_t)nx*ny*nz;
         nbrIDs.assign(N*27,invalid());
         flags.assign(N,0);
         inner.clear(); exterior.clear(); globalIDs.resize(N);
         for (int k=0;k<nz;++k) for (int j=0;j<ny;++j) for (int i=0;i<nx;++i) {
            const CellID c = (CellID)(i + nx*(j + ny*k));
            globalIDs[c] = c;
            uint32_t f = 0;
            for (int dk=-1;dk<=1;++dk) for (int dj=-1;dj<=1;++dj) for (int di=-1;di<=1;++di) {
               int ii = i+di, jj = j+dj, kk = k+dk;
               if (!wrap(ii,nx,periodic[0]) || !wrap(jj,ny,periodic[1]) || !wrap(kk,nz,periodic[2])) continue;
               const unsigned t = calcNeighbourTypeID(di,dj,dk);
               nbrIDs[(size_t)c*27 + t] = (CellID)(ii + nx*(jj + ny*kk));
               f |= (1u << t);
            }
            flags[c] = f;
            inner.push_back(c);
            if (f != ALL_NEIGHBOURS_EXIST) exterior.push_back(c);
         }
      }
      static bool wrap(int& i,int n,int per) {
         if (i >= 0 && i < n) return true;
         if (!per) return false;
         i = (i + n) % n; return true;
      }
      unsigned int calcNeighbourTypeID(int i,int j,int k) const { return (unsigned)((k+1)*9 + (j+1)*3 + (i+1)); }
      CellID invalid() const { return std::numeric_limits<CellID>::max(); }
      uint32_t getNeighbourFlags(CellID b) const { return flags[b]; }
      const std::vector<uint32_t>& getNeighbourFlags() const { return flags; }
      const CellID* getCellNeighbourIDs(CellID b) const { return &nbrIDs[(size_t)b*27]; }
      const std::vector<CellID>& getInnerCells(StencilID) const { return inner; }
      const std::vector<CellID>& getBoundaryCells(StencilID) const { return boundary; }
      const std::vector<CellID>& getExteriorCells() const { return exterior; }
      CellID getNumberOfLocalCells() const { return (CellID)flags.size(); }
      int getRank() const { return 0; }
      CellID getNumberOfAllCells() const { return (CellID)flags.size(); }
      const std::vector<CellID>& getGlobalIDs() const { return globalIDs; }
      std::vector<double>& getCellWeights() { cellWeights.resize(flags.size()); return cellWeights; }
      bool startNeighbourExchange(StencilID,DataID) { return true; }
      bool wait(StencilID,DataID) { return true; }
      template<class T> bool getRemoteUpdates(StencilID,DataID,unsigned int*& offsets,T*& buffers) {
         offsets = nullptr; buffers = nullptr; return true;
      }

      /* static user data: elements values of type T per cell */
      template<class T> DataID addUserDataStatic(size_t elements) {
         StaticStore s; s.elemSize = sizeof(T); s.elements = elements;
         s.bytes.assign(flags.size()*elements*sizeof(T) + 64,0);
         statics.push_back(s);
         return (DataID)(statics.size()-1);
      }
      template<class T> T* getUserDataStatic(DataID id) {
         if (id >= statics.size()) return nullptr;
         return reinterpret_cast<T*>(statics[id].bytes.data());
      }
      char* getUserData(DataID id) { return id < statics.size() ? statics[id].bytes.data() : nullptr; }
      size_t getUserDataStaticElements(DataID id) const { return statics[id].elements; }

      /* dynamic user data (per-cell arrays of T) */
      template<class T> DataID addUserDataDynamic() {
         dynamics.emplace_back(new DynamicStore());
         DynamicStore& d = *dynamics.back();
         d.elemSize = sizeof(T);
         d.cells.assign(flags.size(),std::vector<char>(16));
         d.ptrs.resize(flags.size());
         d.sizes.assign(flags.size(),0);
         for (size_t b=0;b<flags.size();++b) d.ptrs[b] = d.cells[b].data();
         return (DataID)(dynamics.size()-1);
      }
      template<class T> DataWrapper<T> getUserDataDynamic(DataID id) { return DataWrapper<T>(dynamics[id].get()); }

      int nx = 0, ny = 0, nz = 0, periodic[3] = {0,0,0};
    private:
      struct StaticStore { size_t elemSize = 0, elements = 0; std::vector<char> bytes; };
      std::vector<CellID> nbrIDs;
      std::vector<uint32_t> flags;
      std::vector<CellID> inner, boundary, exterior, globalIDs;
      std::vector<double> cellWeights;
      std::vector<StaticStore> statics;
      std::vector<std::unique_ptr<DynamicStore> > dynamics;
   };
}

/* VLSV writer stand-in. open() fails, so the oracle never writes a VLSV
 * file (the reduced-state writer in diagnostics.h stops there). While
 * `capture` is on, writeArray() keeps each array in memory instead, as
 * doubles, with its tag, attributes and sizes: the arrays UserDataOP::writeData
 * hands to the writer, read back by the oracle driver. */
struct VlsvArray {
   std::string tag;
   std::map<std::string,std::string> attribs;
   uint64_t arraySize = 0,vectorSize = 0;
   std::vector<double> data;
};
struct VlsvWriterStub {
   bool capture = false;
   std::vector<VlsvArray> arrays;
   bool open(const std::string&,MPI_Comm,int) { return false; }
   template<class T> bool writeArray(const std::string& tag,const std::map<std::string,std::string>& attribs,
                                     uint64_t arraySize,uint64_t vectorSize,const T* d) {
      if (!capture) return false;
      VlsvArray a;
      a.tag = tag; a.attribs = attribs; a.arraySize = arraySize; a.vectorSize = vectorSize;
      a.data.resize(arraySize*vectorSize);
      for (size_t i=0;i<a.data.size();++i) a.data[i] = static_cast<double>(d[i]);
      arrays.push_back(a);
      return true;
   }
   bool close() { return false; }
   uint64_t getBytesWritten() const { return 0; }
};

struct SimulationClasses {
   pargrid::ParGrid pargrid;
   VlsvWriterStub vlsv;
   Logger logger;
   Random random;
   std::vector<Real> blockCoordinates; /* 3 per cell: minimum corner */
   std::vector<Real> blockSizes;       /* 3 per cell */
};

inline const Real* getBlockCoordinateArray(Simulation&,SimulationClasses& sc) { return sc.blockCoordinates.data(); }
inline void getBlockSize(SimulationClasses& sc,Simulation&,pargrid::CellID b,Real bs[3]) {
   for (int l=0;l<3;++l) bs[l] = sc.blockSizes[3*b+l];
}
inline void getBlockCellSize(SimulationClasses& sc,Simulation& s,pargrid::CellID b,Real bs[3]) { getBlockSize(sc,s,b,bs); }

namespace block {
   /* add the 3x3x3 (x vectorDim) array acc into the 27 neighbours of blockID */
   inline void addValues3D(SimulationClasses& sc,pargrid::CellID blockID,const Real* acc,Real* array,int vectorDim) {
      const pargrid::CellID* nbrs = sc.pargrid.getCellNeighbourIDs(blockID);
      for (int k=0;k<3;++k) for (int j=0;j<3;++j) for (int i=0;i<3;++i) {
         const pargrid::CellID nbr = nbrs[sc.pargrid.calcNeighbourTypeID(i-1,j-1,k-1)];
         if (nbr == sc.pargrid.invalid()) continue;
         for (int l=0;l<vectorDim;++l) array[(size_t)nbr*vectorDim + l] += acc[arrayIndex(i,j,k)*vectorDim + l];
      }
   }
}

#endif
