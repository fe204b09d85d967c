/* Oracle (test infrastructure only): a plain-C restatement of RHybrid's
 * per-timestep hot path, with the same C ABI as the GPU library
 * (include/rhgpu.h) under the prefix rho_. It is the checker for the GPU path
 * and the "port" CPU baseline; it is never part of the product path.
 *
 * It restates, with the reference's operation order (no FMA contraction,
 * same parenthesisation), the functions cited beside each routine below. It is
 * pinned bit for bit against the reference's own sources compiled through
 * oracle/shim (oracle/_ref/librhref.so) by tests/test_oracle_pin.py.
 *
 * Deposit order: RHO_DEPOSIT_REFERENCE reproduces accumulateCell +
 * block::addValues3D (particle_accumulator.cpp:44-156): per source cell a
 * sequential sum over its particles into a 3x3x3 array, then the 27 values
 * added into the neighbours, source cells in increasing index order.
 * RHO_DEPOSIT_GPU reproduces the summation order of the GPU deposit kernel
 * (rh_deposit_order_gpu below) so that the GPU result can be checked bit for
 * bit as well.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#include "oracle_common.h"
#include "../include/rhgpu.h"

#define RHO_MAX_SPECIES 8
#define RHO_DEPOSIT_REFERENCE 0
#define RHO_DEPOSIT_GPU 1

static __thread char g_err[256];
static int fail(int code,const char* msg) { snprintf(g_err,sizeof g_err,"%s",msg); return code; }

typedef struct {
   double* p;        /* 7 doubles per particle, grouped by cell */
   uint32_t* cnt;    /* particles per cell */
   int64_t* start;   /* N+1 offsets */
   int64_t n;
   int64_t cap;
   uint8_t* lx;      /* fast-path storage: dual x within the segment */
   int64_t capLx;
} PopStore;

typedef struct {
   rhgpu_params P;
   int ns;
   rhgpu_species sp[RHO_MAX_SPECIES];
   int nx,ny,nz;
   size_t N;
   int32_t* nbr;      /* 27 neighbour indices per cell, -1 if absent */
   uint32_t* nflags;  /* neighbour existence bits, as ParGrid's */
   uint8_t* cflags;   /* RHGPU_FLAG_* */
   int32_t* exterior; size_t nexterior;
   double* arr[RHGPU_NUM_ARRAYS];
   double* faceJ;
   PopStore pop[RHO_MAX_SPECIES];
   double t;
   int64_t timestep;
   int useIFT;
   double dxBelow;
   double cnt[RHGPU_NUM_FIELD_COUNTERS + RHGPU_CNT_PER_SPECIES*RHO_MAX_SPECIES];
   int depositOrder;   /* RHO_DEPOSIT_REFERENCE: cell storage; RHO_DEPOSIT_GPU: dual-cell storage */
   int nthreads;
   /* fast-path restatement (row-segment storage) */
   int nd[3];          /* dual cells per axis: n (periodic) or n+1 */
   size_t Nd;
   int nseg;           /* segments per dual row */
   size_t NS;          /* segments */
   double* RP;         /* row partial moments, 4 planes x rows x nx x 4 */
   double* RPB;        /* segment-boundary partials, 4 planes x rows x nseg x 4 */
   __int128* MM;       /* fixed-point moments of particles leaving their segment, 4 x N (exact sums) */
   int kR, kJ;         /* fixed-point exponents of charge and current */
} Ctx;

#define ALL_NBRS ((1u<<27)-1u)
#define TID(di,dj,dk) (((dk)+1)*9 + ((dj)+1)*3 + ((di)+1))
#define XPOS (1u<<TID(1,0,0))
#define XNEG (1u<<TID(-1,0,0))
#define YPOS (1u<<TID(0,1,0))
#define YNEG (1u<<TID(0,-1,0))
#define ZPOS (1u<<TID(0,0,1))
#define ZNEG (1u<<TID(0,0,-1))

static inline double sqr(double x) { return x*x; }
static int dualUpload(Ctx* c,int sidx,const uint32_t* counts,const double* parts,int64_t n);
static int dualDownload(Ctx* c,int sidx,uint32_t* counts,double* parts);
static void dualPushAll(Ctx* c);
static void dualGather(Ctx* c);
static inline int nb(const Ctx* c,size_t b,int di,int dj,int dk) { return c->nbr[b*27 + TID(di,dj,dk)]; }
static int arrayDim(int id) {
   return (id == RHGPU_CELL_RHOQI || id == RHGPU_NODE_RHOQI || id == RHGPU_NODE_ETA) ? 1 : 3;
}
/* + neighbours required (cell2Node, calcNodeJ, upwindNodeB, calcNodeE,
 * calcNodeUe, faceCurl: hybrid_propagator.cpp:1064-1067 etc.) */
static inline int plusOk(uint32_t f) { return (f & XPOS) && (f & YPOS) && (f & ZPOS); }

/* ------------------------------------------------------------------ */
/* parallel-for over cells with pthreads (cells are independent in the  */
/* field kernels restated below, so threads do not change results)     */
typedef void (*CellFn)(Ctx*,size_t);
typedef struct { Ctx* c; CellFn fn; size_t a,b; } Job;
static void* runJob(void* v) { Job* j = (Job*)v; for (size_t x=j->a;x<j->b;++x) j->fn(j->c,x); return NULL; }
static void forCells(Ctx* c,CellFn fn) {
   const int T = c->nthreads;
   if (T <= 1 || c->N < 4096) { for (size_t b=0;b<c->N;++b) fn(c,b); return; }
   pthread_t th[64]; Job jobs[64];
   for (int t=0;t<T;++t) {
      jobs[t].c = c; jobs[t].fn = fn; jobs[t].a = c->N*t/T; jobs[t].b = c->N*(t+1)/T;
      pthread_create(&th[t],NULL,runJob,&jobs[t]);
   }
   for (int t=0;t<T;++t) pthread_join(th[t],NULL);
}

/* ------------------------------------------------------------------ */
/* context                                                             */

int rho_create(const rhgpu_params* P,int32_t ns,const rhgpu_species* sp,const int64_t* cap,int32_t dev,void** out) {
   (void)cap; (void)dev;
   if (!P || !out || ns < 1 || ns > RHO_MAX_SPECIES) return fail(RHGPU_ERR_ARG,"rho_create: bad arguments");
   if (P->nx < 3 || P->ny < 3 || P->nz < 3) return fail(RHGPU_ERR_ARG,"rho_create: at least 3 cells per axis");
   Ctx* c = (Ctx*)calloc(1,sizeof(Ctx));
   c->P = *P; c->ns = ns;
   memcpy(c->sp,sp,sizeof(rhgpu_species)*ns);
   c->nx = P->nx; c->ny = P->ny; c->nz = P->nz;
   c->N = (size_t)c->nx*c->ny*c->nz;
   c->nbr = (int32_t*)malloc(sizeof(int32_t)*27*c->N);
   c->nflags = (uint32_t*)calloc(c->N,sizeof(uint32_t));
   c->cflags = (uint8_t*)calloc(c->N,1);
   c->exterior = (int32_t*)malloc(sizeof(int32_t)*c->N);
   for (int k=0;k<c->nz;++k) for (int j=0;j<c->ny;++j) for (int i=0;i<c->nx;++i) {
      const size_t b = (size_t)i + c->nx*((size_t)j + c->ny*(size_t)k);
      uint32_t f = 0;
      for (int dk=-1;dk<=1;++dk) for (int dj=-1;dj<=1;++dj) for (int di=-1;di<=1;++di) {
         int ii = i+di, jj = j+dj, kk = k+dk;
         int32_t id = -1;
         if (rh_wrap(&ii,c->nx,P->periodic[0]) && rh_wrap(&jj,c->ny,P->periodic[1]) && rh_wrap(&kk,c->nz,P->periodic[2])) {
            id = (int32_t)(ii + c->nx*(jj + c->ny*kk));
            f |= 1u << TID(di,dj,dk);
         }
         c->nbr[b*27 + TID(di,dj,dk)] = id;
      }
      c->nflags[b] = f;
      if (f != ALL_NBRS) c->exterior[c->nexterior++] = (int32_t)b;
   }
   for (int a=0;a<RHGPU_NUM_ARRAYS;++a) c->arr[a] = (double*)calloc(c->N*arrayDim(a),sizeof(double));
   c->faceJ = (double*)calloc(3*c->N,sizeof(double));
   for (int a=0;a<3;++a) c->nd[a] = (a==0 ? c->nx : a==1 ? c->ny : c->nz) + (P->periodic[a] ? 0 : 1);
   c->Nd = (size_t)c->nd[0]*c->nd[1]*c->nd[2];
   c->nseg = (c->nd[0] + RHGPU_FAST_SEGMENT - 1)/RHGPU_FAST_SEGMENT;
   c->NS = (size_t)c->nd[1]*c->nd[2]*c->nseg;
   for (int s=0;s<ns;++s) {
      c->pop[s].cnt = (uint32_t*)calloc(c->Nd,sizeof(uint32_t));
      c->pop[s].start = (int64_t*)calloc(c->Nd+1,sizeof(int64_t));
   }
   c->RP = (double*)calloc((size_t)16*c->nd[1]*c->nd[2]*c->nx,sizeof(double));
   c->RPB = (double*)calloc((size_t)16*c->nd[1]*c->nd[2]*c->nseg,sizeof(double));
   c->MM = (__int128*)calloc(4*c->N,sizeof(__int128));
   c->t = P->t_initial;
   c->timestep = 0;
   c->useIFT = P->use_initial_flow_through;
   c->dxBelow = nextafter(P->dx,0.0);
   c->depositOrder = RHO_DEPOSIT_REFERENCE;
   c->nthreads = 1;
   *out = c;
   return RHGPU_OK;
}

int rho_destroy(void* h) {
   Ctx* c = (Ctx*)h;
   if (!c) return 0;
   free(c->nbr); free(c->nflags); free(c->cflags); free(c->exterior); free(c->faceJ);
   free(c->RP); free(c->RPB); free(c->MM);
   for (int a=0;a<RHGPU_NUM_ARRAYS;++a) free(c->arr[a]);
   for (int s=0;s<c->ns;++s) { free(c->pop[s].p); free(c->pop[s].cnt); free(c->pop[s].start); free(c->pop[s].lx); }
   free(c);
   return 0;
}

const char* rho_last_error(void) { return g_err; }

/* 0: reference order (bitwise = reference), 1: GPU kernel order */
int rho_set_deposit_order(void* h,int32_t order) { ((Ctx*)h)->depositOrder = order; return 0; }
int rho_set_threads(void* h,int32_t n) { Ctx* c = (Ctx*)h; c->nthreads = n < 1 ? 1 : (n > 64 ? 64 : n); return 0; }

int rho_upload_array(void* h,int32_t id,const double* host) {
   Ctx* c = (Ctx*)h;
   if (id < 0 || id >= RHGPU_NUM_ARRAYS) return fail(RHGPU_ERR_ARG,"bad array id");
   memcpy(c->arr[id],host,sizeof(double)*c->N*arrayDim(id));
   return 0;
}
int rho_download_array(void* h,int32_t id,double* host) {
   Ctx* c = (Ctx*)h;
   if (id < 0 || id >= RHGPU_NUM_ARRAYS) return fail(RHGPU_ERR_ARG,"bad array id");
   memcpy(host,c->arr[id],sizeof(double)*c->N*arrayDim(id));
   return 0;
}
int rho_upload_cell_flags(void* h,const uint8_t* f) { Ctx* c = (Ctx*)h; memcpy(c->cflags,f,c->N); return 0; }

static void popReserve(PopStore* s,int64_t n) {
   if (n <= s->cap) return;
   s->cap = n + n/4 + 16;
   s->p = (double*)realloc(s->p,sizeof(double)*7*s->cap);
}
static void popStarts(Ctx* c,PopStore* s) {
   s->start[0] = 0;
   for (size_t b=0;b<c->N;++b) s->start[b+1] = s->start[b] + s->cnt[b];
   s->n = s->start[c->N];
}

int rho_upload_particles(void* h,int32_t sidx,const uint32_t* counts,const double* parts,int64_t n) {
   Ctx* c = (Ctx*)h;
   if (sidx < 0 || sidx >= c->ns) return fail(RHGPU_ERR_ARG,"bad species");
   PopStore* s = &c->pop[sidx];
   int64_t tot = 0;
   for (size_t b=0;b<c->N;++b) tot += counts[b];
   if (tot != n) return fail(RHGPU_ERR_ARG,"sum(counts) != n_particles");
   if (c->depositOrder == RHO_DEPOSIT_GPU) return dualUpload(c,sidx,counts,parts,n);
   popReserve(s,n);
   memcpy(s->cnt,counts,sizeof(uint32_t)*c->N);
   if (n) memcpy(s->p,parts,sizeof(double)*7*n);
   popStarts(c,s);
   return 0;
}
int rho_num_particles(void* h,int32_t sidx,int64_t* n) { *n = ((Ctx*)h)->pop[sidx].n; return 0; }
int rho_download_particles(void* h,int32_t sidx,uint32_t* counts,double* parts,int64_t cap,int64_t* nout) {
   Ctx* c = (Ctx*)h;
   PopStore* s = &c->pop[sidx];
   if (s->n > cap) return fail(RHGPU_ERR_ARG,"capacity too small");
   *nout = s->n;
   if (c->depositOrder == RHO_DEPOSIT_GPU) return dualDownload(c,sidx,counts,parts);
   memcpy(counts,s->cnt,sizeof(uint32_t)*c->N);
   if (s->n) memcpy(parts,s->p,sizeof(double)*7*s->n);
   *nout = s->n;
   return 0;
}

/* ------------------------------------------------------------------ */
/* push: BorisBuneman::propagate (particle_propagator_boris_buneman.h:64-194)
 * with getFields (hybrid_propagator.cpp:1879-1891): face2r (:1740-1778) for B,
 * cell2r (:1838-1858) for Ue and Ep. */

/* push of one particle st[7] (local coordinates in cell b); returns 1 if
 * the maximum ion speed clamp was applied */
static int pushParticle(Ctx* c,int sidx,size_t b,double* st) {
   const rhgpu_params* P = &c->P;
   const rhgpu_species* S = &c->sp[sidx];
   const int ci = (int)(b % c->nx), cj = (int)((b / c->nx) % c->ny), ck = (int)(b / ((size_t)c->nx*c->ny));
   const double xBlock = rh_block_origin(P->x_min,ci,P->dx);
   const double yBlock = rh_block_origin(P->y_min,cj,P->dx);
   const double zBlock = rh_block_origin(P->z_min,ck,P->dx);
   int accelerate = S->accelerate;
   if (c->nflags[b] != ALL_NBRS || c->useIFT) accelerate = 0;
   const double* faceB = c->arr[RHGPU_FACE_B];
   const double* cellUe = c->arr[RHGPU_CELL_UE];
   const double* cellEp = c->arr[RHGPU_CELL_EP];
   const double dt = P->dt, dx = P->dx;
   int clamped = 0;
   {
      if (accelerate) {
         double B[3],Ue[3],Ep[3] = {0,0,0},E[3];
         const double rGlobal[3] = {st[0]+xBlock,st[1]+yBlock,st[2]+zBlock};
         /* face2r: linear interpolation along each component's own axis */
         {
            const double x = st[0]/dx, y = st[1]/dx, z = st[2]/dx;
            int i = (int)floor(x), j = (int)floor(y), k = (int)floor(z);
            /* positions lie in [0,dx): i=j=k=0 (a quotient rounded up to 1
             * would index outside the reference's 3x3x3 array) */
            if (i != 0) i = 0;
            if (j != 0) j = 0;
            if (k != 0) k = 0;
            const double w111x = x - (double)(i+0), w111y = y - (double)(j+0), w111z = z - (double)(k+0);
            const double w011x = (double)(i+1) - x, w101y = (double)(j+1) - y, w110z = (double)(k+1) - z;
            B[0] = w111x*faceB[3*b+0] + w011x*faceB[3*nb(c,b,-1,0,0)+0];
            B[1] = w111y*faceB[3*b+1] + w101y*faceB[3*nb(c,b,0,-1,0)+1];
            B[2] = w111z*faceB[3*b+2] + w110z*faceB[3*nb(c,b,0,0,-1)+2];
         }
         for (int l=0;l<3;++l) Ue[l] = cellUe[3*b+l];
         if (P->use_electron_pressure) for (int l=0;l<3;++l) Ep[l] = cellEp[3*b+l];
         /* E = B x Ue = -Ue x B (boris.h:105-106) */
         E[0] = B[1]*Ue[2] - B[2]*Ue[1];
         E[1] = B[2]*Ue[0] - B[0]*Ue[2];
         E[2] = B[0]*Ue[1] - B[1]*Ue[0];
         if (P->use_electron_pressure) for (int l=0;l<3;++l) E[l] += Ep[l];
         /* Boris rotation (boris.h:111-135) */
         double tx,ty,tz,sx,sy,sz,dvx,dvy,dvz,vmx,vmy,vmz,v0x,v0y,v0z,vpx,vpy,vpz,qmideltT2,t2,b2;
         qmideltT2 = 0.5*S->q*dt/S->m;
         dvx = qmideltT2*E[0]; dvy = qmideltT2*E[1]; dvz = qmideltT2*E[2];
         tx = qmideltT2*B[0]; ty = qmideltT2*B[1]; tz = qmideltT2*B[2];
         t2 = tx*tx+ty*ty+tz*tz;
         b2 = 2./(1.+t2);
         sx = b2*tx; sy = b2*ty; sz = b2*tz;
         vmx = st[3]+dvx; vmy = st[4]+dvy; vmz = st[5]+dvz;
         v0x = vmx+vmy*tz-vmz*ty;
         v0y = vmy+vmz*tx-vmx*tz;
         v0z = vmz+vmx*ty-vmy*tx;
         vpx = vmx+v0y*sz-v0z*sy;
         vpy = vmy+v0z*sx-v0x*sz;
         vpz = vmz+v0x*sy-v0y*sx;
         st[3] = vpx+dvx; st[4] = vpy+dvy; st[5] = vpz+dvz;
         /* gravity (boris.h:137-145) */
         if (P->use_gravity) {
            const double rr = sqrt(sqr(rGlobal[0]) + sqr(rGlobal[1]) + sqr(rGlobal[2]));
            const double r3 = rr*rr*rr;
            if (r3 > 0) {
               const double sg = -P->GMdt/r3;
               st[3] += sg*rGlobal[0]; st[4] += sg*rGlobal[1]; st[5] += sg*rGlobal[2];
            }
         }
         /* maximum ion speed (boris.h:146-158) */
         const double v2 = sqr(st[3]) + sqr(st[4]) + sqr(st[5]);
         if (v2 > P->max_ion_speed2) {
            const double norm = sqrt(P->max_ion_speed2/v2);
            st[3] *= norm; st[4] *= norm; st[5] *= norm;
            clamped = 1;
         }
      }
      /* drift (boris.h:191-193) */
      st[0] += dt*st[3];
      st[1] += dt*st[4];
      st[2] += dt*st[5];
   }
   return clamped;
}

static void pushCell(Ctx* c,int sidx,size_t b) {
   PopStore* s = &c->pop[sidx];
   double* cntMaxVi = &c->cnt[RHGPU_NUM_FIELD_COUNTERS + RHGPU_CNT_PER_SPECIES*sidx + 0];
   for (int64_t p=s->start[b];p<s->start[b+1];++p) *cntMaxVi += pushParticle(c,sidx,b,s->p + 7*p);
}

/* canonical migration (oracle_common.h) */
static void migrate(Ctx* c,int sidx) {
   PopStore* s = &c->pop[sidx];
   const size_t N = c->N;
   const int64_t n = s->n;
   int64_t* key = (int64_t*)malloc(sizeof(int64_t)*(n > 0 ? n : 1));
   double* esc = &c->cnt[RHGPU_NUM_FIELD_COUNTERS + RHGPU_CNT_PER_SPECIES*sidx];
   for (size_t b=0;b<N;++b) {
      const int i = (int)(b % c->nx), j = (int)((b / c->nx) % c->ny), k = (int)(b / ((size_t)c->nx*c->ny));
      for (int64_t p=s->start[b];p<s->start[b+1];++p) {
         double* st = s->p + 7*p;
         int off[3];
         const int bad = rh_migrate_canonical(st,c->P.dx,c->dxBelow,off);
         int ti = i+off[0], tj = j+off[1], tk = k+off[2];
         const int inside = rh_wrap(&ti,c->nx,c->P.periodic[0]) && rh_wrap(&tj,c->ny,c->P.periodic[1]) && rh_wrap(&tk,c->nz,c->P.periodic[2]);
         if (bad || !inside) {
            esc[1] += st[6];
            esc[2] += st[6]*( sqr(st[3]) + sqr(st[4]) + sqr(st[5]) );
            key[p] = -1;
            continue;
         }
         const size_t d = (size_t)ti + c->nx*((size_t)tj + c->ny*(size_t)tk);
         key[p] = (int64_t)d*27 + rh_dir_rank(rh_dir_from_offset(-off[0],-off[1],-off[2]));
      }
   }
   int64_t* start = (int64_t*)calloc(N*27+1,sizeof(int64_t));
   for (int64_t p=0;p<n;++p) if (key[p] >= 0) start[key[p]+1]++;
   for (size_t q=0;q<N*27;++q) start[q+1] += start[q];
   double* np = (double*)malloc(sizeof(double)*7*(start[N*27] > 0 ? start[N*27] : 1));
   for (int64_t p=0;p<n;++p) if (key[p] >= 0) memcpy(np + 7*(start[key[p]]++),s->p + 7*p,7*sizeof(double));
   /* start[] now holds the end of each key; recover counts per cell */
   int64_t prev = 0;
   for (size_t b=0;b<N;++b) { const int64_t e = start[b*27+26]; s->cnt[b] = (uint32_t)(e - prev); prev = e; }
   free(s->p); s->p = np; s->cap = start[N*27] > 0 ? start[N*27] : 1;
   popStarts(c,s);
   free(start); free(key);
}

static int g_pushSpecies;
static void pushCellFn(Ctx* c,size_t b) { pushCell(c,g_pushSpecies,b); }

int rho_push(void* h) {
   Ctx* c = (Ctx*)h;
   c->timestep += 1;
   if (c->P.initial_flow_through_period < c->t && c->useIFT) c->useIFT = 0;
   if (c->depositOrder == RHO_DEPOSIT_GPU) { dualPushAll(c); return 0; }
   for (int s=0;s<c->ns;++s) {
      if (c->nthreads > 1) {
         /* the speed-clamp counter is summed per thread in pushCell; use
          * a serial pass when counting matters less than speed */
         g_pushSpecies = s; forCells(c,pushCellFn);
      } else {
         for (size_t b=0;b<c->N;++b) pushCell(c,s,b);
      }
      migrate(c,s);
   }
   return 0;
}

/* ------------------------------------------------------------------ */
/* deposit: Accumulator::accumulateCell (particle_accumulator.cpp:44-156)
 * with block::addValues3D, then addRemoteUpdates' finalize (:319-333). */

/* CIC weights and indices of one particle (particle_accumulator.cpp:68-110).
 * w8[0..7] in the order w000,w100,w010,w110,w001,w101,w011,w111 and the
 * index (0..26) of each in the 3x3x3 array. */
static inline void cicWeights(const double* st,double q,double dx,double w8[8],int ind[8]) {
   const double x = st[0], y = st[1], z = st[2];
   const double wq = st[6]*q;
   int i = (int)floor(x/dx), j = (int)floor(y/dx), k = (int)floor(z/dx);
   if (x < (i+0.5)*dx) { --i; }
   if (y < (j+0.5)*dx) { --j; }
   if (z < (k+0.5)*dx) { --k; }
   ++i; ++j; ++k;
   const double x0 = (i-1+0.5)*dx, y0 = (j-1+0.5)*dx, z0 = (k-1+0.5)*dx;
   const double w_x = (x-x0)/dx, w_y = (y-y0)/dx, w_z = (z-z0)/dx;
   w8[0] = (1-w_x)*(1-w_y)*(1-w_z) * wq;
   w8[1] =    w_x *(1-w_y)*(1-w_z) * wq;
   w8[2] = (1-w_x)*   w_y *(1-w_z) * wq;
   w8[3] =    w_x *   w_y *(1-w_z) * wq;
   w8[4] = (1-w_x)*(1-w_y)*   w_z  * wq;
   w8[5] =    w_x *(1-w_y)*   w_z  * wq;
   w8[6] = (1-w_x)*   w_y *   w_z  * wq;
   w8[7] =    w_x *  w_y  *   w_z  * wq;
   for (int o=0;o<8;++o) {
      const int a = i + (o&1), bb = j + ((o>>1)&1), cc = k + ((o>>2)&1);
      ind[o] = a + 3*(bb + 3*cc);
   }
}

/* per-cell 3x3x3 accumulation in particle order (reference order) */
static void accumulateCellRef(Ctx* c,int sidx,size_t b,double acc1[27],double acc2[81]) {
   PopStore* s = &c->pop[sidx];
   for (int e=0;e<27;++e) acc1[e] = 0.0;
   for (int e=0;e<81;++e) acc2[e] = 0.0;
   const double q = c->sp[sidx].q, dx = c->P.dx;
   for (int64_t p=s->start[b];p<s->start[b+1];++p) {
      const double* st = s->p + 7*p;
      double w8[8]; int ind[8];
      cicWeights(st,q,dx,w8,ind);
      for (int o=0;o<8;++o) acc1[ind[o]] += w8[o];
      for (int l=0;l<3;++l) for (int o=0;o<8;++o) acc2[ind[o]*3+l] += w8[o]*st[3+l];
   }
}

static void depositReference(Ctx* c,int sidx) {
   double* rho = c->arr[RHGPU_CELL_RHOQI];
   double* Ji = c->arr[RHGPU_CELL_JI];
   for (size_t b=0;b<c->N;++b) {
      if (c->pop[sidx].cnt[b] == 0) continue;   /* an empty cell adds zeros */
      double acc1[27],acc2[81];
      accumulateCellRef(c,sidx,b,acc1,acc2);
      for (int k=0;k<3;++k) for (int j=0;j<3;++j) for (int i=0;i<3;++i) {
         const int n = nb(c,b,i-1,j-1,k-1);
         if (n < 0) continue;
         const int e = i + 3*(j + 3*k);
         rho[n] += acc1[e];
         for (int l=0;l<3;++l) Ji[3*(size_t)n+l] += acc2[e*3+l];
      }
   }
}


int rho_accumulate(void* h) {
   Ctx* c = (Ctx*)h;
   if (c->depositOrder == RHO_DEPOSIT_GPU) { dualGather(c); return 0; }
   double* rho = c->arr[RHGPU_CELL_RHOQI];
   double* Ji = c->arr[RHGPU_CELL_JI];
   memset(rho,0,sizeof(double)*c->N);
   memset(Ji,0,sizeof(double)*3*c->N);
   for (int s=0;s<c->ns;++s) {
      if (!c->sp[s].accumulate) continue;
      depositReference(c,s);
   }
   const double dV = c->P.dx*c->P.dx*c->P.dx;
   for (size_t n=0;n<c->N;++n) {
      rho[n] /= dV;
      if (rho[n] < c->P.min_ion_charge_density) {
         rho[n] = c->P.min_ion_charge_density;
         c->cnt[RHGPU_CNT_FIELD_MIN_CELL_RHOQI] += 1;
      }
      for (int l=0;l<3;++l) Ji[3*n+l] /= dV;
   }
   return 0;
}

/* ------------------------------------------------------------------ */
/* particle boundary conditions (particle_boundary_cond_hybrid.h:112-185) */
int rho_apply_boundaries(void* h) {
   Ctx* c = (Ctx*)h;
   /* the fast path removes boundary particles inside its push (dualPushAll) */
   if (c->depositOrder == RHO_DEPOSIT_GPU) return 0;
   for (int sidx=0;sidx<c->ns;++sidx) {
      PopStore* s = &c->pop[sidx];
      double* q = &c->cnt[RHGPU_NUM_FIELD_COUNTERS + RHGPU_CNT_PER_SPECIES*sidx];
      /* exterior cells: remove all */
      for (size_t e=0;e<c->nexterior;++e) {
         const size_t b = (size_t)c->exterior[e];
         for (int64_t p=s->start[b];p<s->start[b+1];++p) {
            const double* st = s->p + 7*p;
            q[1] += st[6];
            q[2] += st[6]*( sqr(st[3]) + sqr(st[4]) + sqr(st[5]) );
         }
         s->cnt[b] = 0;
      }
      /* inner boundary: swap-remove particles with r^2 < R2_obstacle */
      const double R2 = c->sp[sidx].R2_obstacle;
      for (size_t b=0;b<c->N;++b) {
         if (!(c->cflags[b] & RHGPU_FLAG_INNER_PARTICLE)) continue;
         if (s->cnt[b] == 0) continue;
         const int i = (int)(b % c->nx), j = (int)((b / c->nx) % c->ny), k = (int)(b / ((size_t)c->nx*c->ny));
         const double xB = rh_block_origin(c->P.x_min,i,c->P.dx);
         const double yB = rh_block_origin(c->P.y_min,j,c->P.dx);
         const double zB = rh_block_origin(c->P.z_min,k,c->P.dx);
         double* base = s->p + 7*s->start[b];
         int cur = 0, end = (int)s->cnt[b] - 1;
         while (cur <= end) {
            double* st = base + 7*cur;
            const double xp = xB + st[0], yp = yB + st[1], zp = zB + st[2];
            const double r2 = sqr(xp) + sqr(yp) + sqr(zp);
            if (r2 < R2) {
               q[3] += st[6];
               q[4] += st[6]*( sqr(st[3]) + sqr(st[4]) + sqr(st[5]) );
               memcpy(st,base + 7*end,7*sizeof(double));
               --end;
               continue;
            }
            ++cur;
         }
         s->cnt[b] = (uint32_t)cur;
      }
      /* compact */
      int64_t w = 0;
      for (size_t b=0;b<c->N;++b) {
         const int64_t a = s->start[b];
         if (w != a && s->cnt[b]) memmove(s->p + 7*w,s->p + 7*a,sizeof(double)*7*s->cnt[b]);
         w += s->cnt[b];
      }
      popStarts(c,s);
   }
   return 0;
}

/* ------------------------------------------------------------------ */
/* Fast-path restatement (RHO_DEPOSIT_GPU): the order of operations of the
 * GPU's fused push-and-deposit kernel, so that its results can be checked bit
 * for bit. The arithmetic per particle and per cell is the reference's; only
 * the order in which the CIC contributions are summed, and the order of the
 * particles inside the storage, differ from RHO_DEPOSIT_REFERENCE.
 *
 * Dual cells: the 2x2x2 block of cells whose centres surround the particle:
 * base cell b = c + s - 1 per axis with s = 0 if x < 0.5 dx else 1 (the shift
 * of accumulateCell, :78-84). Dual index u = b + 1 on a non-periodic axis
 * (n+1 dual cells), b mod n on a periodic one. A dual row (uy, uz) is cut into
 * segments of RHGPU_FAST_SEGMENT dual cells along x, S = row*nseg + ux/SEG.
 * Particles are stored by segment, with their dual x within the segment.
 *
 * Step, per segment, species in order, particles in storage order: push
 * (pushParticle), drift, migrate (rh_migrate_canonical), then the CIC weights
 * of the new position. If the new dual cell lies in the same segment, the
 * particle's record (new dual cell, w8, v) joins the segment's record list;
 * otherwise its 8x4 contributions are added, as fixed point (value * 2^k
 * rounded to nearest, summed exactly), to the moments of the 8 destination
 * cells (MM). Per dual cell d of the segment and per (corner o, moment q):
 *    acc[d][o][q] = 0.0, then += w8[o] * f[q] over the records of d in list
 * order, with f = (1.0, vx, vy, vz).
 * A cell x of the row receives corner ox = 1 of its lower dual cell u_lo and
 * ox = 0 of its upper dual cell u_hi (non-periodic: u_lo = x, u_hi = x+1;
 * periodic: u_lo = x-1, u_hi = x): the row partial
 *    RP[(oy,oz)][row][x][q] = acc[u_lo][ox=1,oy,oz][q] + acc[u_hi][ox=0,oy,oz][q],
 * formed as RP = acc_lo (+ RPB = acc_hi) when u_hi starts another segment.
 * A cell's moment is RP(0,0) + RP(1,0) + RP(0,1) + RP(1,1) (rows of base
 * y-oy, z-oz) + MM*2^-k, then /dV and the minimum charge density clamp.
 * Particles that end in an exterior cell, or inside the obstacle of a flagged
 * cell, are deposited and then removed (the boundary conditions of the step);
 * particles leaving the box are removed before depositing.
 * New storage of a segment: its stayers in their previous order, then the
 * arrivals from other segments in order of (source segment, position in the
 * source segment).
 */
static inline int dualU(int b,int n,int per) { return per ? ((b % n) + n) % n : b + 1; }
static inline int dualB(int u,int per) { return per ? u : u - 1; }
static inline int halfS(double x,double dx) { return (x < (0+0.5)*dx) ? 0 : 1; }
#define SEG RHGPU_FAST_SEGMENT

/* cell of a particle of dual cell (ux,uy,uz) */
static size_t cellOfDual(const Ctx* c,int ux,int uy,int uz,const double* st) {
   const double dx = c->P.dx;
   int i = dualB(ux,c->P.periodic[0]) + 1 - halfS(st[0],dx);
   int j = dualB(uy,c->P.periodic[1]) + 1 - halfS(st[1],dx);
   int k = dualB(uz,c->P.periodic[2]) + 1 - halfS(st[2],dx);
   rh_wrap(&i,c->nx,1); rh_wrap(&j,c->ny,1); rh_wrap(&k,c->nz,1);
   return (size_t)i + c->nx*((size_t)j + c->ny*(size_t)k);
}

static void segStarts(Ctx* c,PopStore* s) {
   s->start[0] = 0;
   for (size_t d=0;d<c->NS;++d) s->start[d+1] = s->start[d] + s->cnt[d];
   s->n = s->start[c->NS];
}

/* stable counting sort of n records (7 doubles + dual x byte) by key[] in [0,nkeys) */
static void sortRecordsLx(const double* in,const uint8_t* inLx,const int64_t* key,int64_t n,int64_t nkeys,
                          double* out,uint8_t* outLx,uint32_t* cntOut) {
   int64_t* start = (int64_t*)calloc(nkeys+1,sizeof(int64_t));
   for (int64_t p=0;p<n;++p) start[key[p]+1]++;
   if (cntOut) for (int64_t q=0;q<nkeys;++q) cntOut[q] = (uint32_t)start[q+1];
   for (int64_t q=0;q<nkeys;++q) start[q+1] += start[q];
   for (int64_t p=0;p<n;++p) {
      const int64_t d = start[key[p]]++;
      memcpy(out + 7*d,in + 7*p,7*sizeof(double));
      if (outLx) outLx[d] = inLx ? inLx[p] : 0;
   }
   free(start);
}

static void popReserveLx(PopStore* s,int64_t n) {
   if (n <= s->capLx) return;
   popReserve(s,n);
   s->capLx = s->cap;
   s->lx = (uint8_t*)realloc(s->lx,s->capLx > 0 ? s->capLx : 1);
}

/* the fixed-point exponents: the largest possible contribution times 2^k
 * stays below 2^62 (charge: max |w q|; current: max |w q| times 2 dx/dt, the
 * largest velocity component of a particle that moved at most one cell) */
static void fixedPointExponents(Ctx* c) {
   double bR = 0.0;
   for (int s=0;s<c->ns;++s) {
      const PopStore* ps = &c->pop[s];
      double mw = 0.0;
      for (int64_t p=0;p<ps->n;++p) if (fabs(ps->p[7*p+6]) > mw) mw = fabs(ps->p[7*p+6]);
      const double b = mw*fabs(c->sp[s].q);
      if (b > bR) bR = b;
   }
   const double bJ = bR*(2.0*c->P.dx/c->P.dt);
   int e;
   frexp(bR > 0 ? bR : 1.0,&e); c->kR = 62 - e;
   frexp(bJ > 0 ? bJ : 1.0,&e); c->kJ = 62 - e;
}

static int dualUpload(Ctx* c,int sidx,const uint32_t* counts,const double* parts,int64_t n) {
   PopStore* s = &c->pop[sidx];
   int64_t* key = (int64_t*)malloc(sizeof(int64_t)*(n > 0 ? n : 1));
   uint8_t* lx = (uint8_t*)malloc(n > 0 ? n : 1);
   const double dx = c->P.dx;
   int64_t p = 0;
   for (size_t b=0;b<c->N;++b) {
      const int i = (int)(b % c->nx), j = (int)((b / c->nx) % c->ny), k = (int)(b / ((size_t)c->nx*c->ny));
      for (uint32_t t=0;t<counts[b];++t,++p) {
         const double* st = parts + 7*p;
         const int ux = dualU(i + halfS(st[0],dx) - 1,c->nx,c->P.periodic[0]);
         const int uy = dualU(j + halfS(st[1],dx) - 1,c->ny,c->P.periodic[1]);
         const int uz = dualU(k + halfS(st[2],dx) - 1,c->nz,c->P.periodic[2]);
         key[p] = ((int64_t)uy + (int64_t)c->nd[1]*uz)*c->nseg + ux/SEG;
         lx[p] = (uint8_t)(ux % SEG);
      }
   }
   popReserveLx(s,n);
   sortRecordsLx(parts,lx,key,n,(int64_t)c->NS,s->p,s->lx,s->cnt);
   segStarts(c,s);
   free(key); free(lx);
   fixedPointExponents(c);
   return 0;
}

static int dualDownload(Ctx* c,int sidx,uint32_t* counts,double* parts) {
   PopStore* s = &c->pop[sidx];
   int64_t* key = (int64_t*)malloc(sizeof(int64_t)*(s->n > 0 ? s->n : 1));
   for (size_t S=0;S<c->NS;++S) {
      const size_t row = S / c->nseg;
      const int u0 = (int)(S % c->nseg)*SEG;
      const int uy = (int)(row % c->nd[1]), uz = (int)(row / c->nd[1]);
      for (int64_t p=s->start[S];p<s->start[S+1];++p) key[p] = (int64_t)cellOfDual(c,u0 + s->lx[p],uy,uz,s->p + 7*p);
   }
   sortRecordsLx(s->p,NULL,key,s->n,(int64_t)c->N,parts,NULL,counts);
   free(key);
   return 0;
}

typedef struct { double st[7]; uint64_t key; int64_t dest; int lx; } OMover;
typedef struct { int d; double w8[8]; double f[4]; } ORecord;

static int cmpMover(const void* a,const void* b) {
   const uint64_t x = ((const OMover*)a)->key, y = ((const OMover*)b)->key;
   return x < y ? -1 : x > y;
}

static void dualPushAll(Ctx* c) {
   const rhgpu_params* P = &c->P;
   const double dx = P->dx;
   const int ndx = c->nd[0], nseg = c->nseg;
   const size_t nrows = (size_t)c->nd[1]*c->nd[2], NS = c->NS;
   memset(c->RP,0,sizeof(double)*16*nrows*c->nx);
   memset(c->RPB,0,sizeof(double)*16*nrows*nseg);
   memset(c->MM,0,sizeof(__int128)*4*c->N);
   const double scaleR = ldexp(1.0,c->kR), scaleJ = ldexp(1.0,c->kJ);
   /* per species: stayers (records + dual x) and their counts per segment, movers */
   double* sw[RHO_MAX_SPECIES]; uint8_t* slx[RHO_MAX_SPECIES]; uint32_t* scnt[RHO_MAX_SPECIES]; int64_t sn[RHO_MAX_SPECIES];
   OMover* mv[RHO_MAX_SPECIES]; int64_t mn[RHO_MAX_SPECIES];
   for (int s=0;s<c->ns;++s) {
      const int64_t n = c->pop[s].n > 0 ? c->pop[s].n : 1;
      sw[s] = (double*)malloc(sizeof(double)*7*n); slx[s] = (uint8_t*)malloc(n);
      scnt[s] = (uint32_t*)calloc(NS,sizeof(uint32_t)); sn[s] = 0;
      mv[s] = (OMover*)malloc(sizeof(OMover)*n); mn[s] = 0;
   }
   int64_t maxSeg = 1;
   for (size_t S=0;S<NS;++S) {
      int64_t t = 0;
      for (int s=0;s<c->ns;++s) t += c->pop[s].cnt[S];
      if (t > maxSeg) maxSeg = t;
   }
   ORecord* recs = (ORecord*)malloc(sizeof(ORecord)*maxSeg);
   double acc[SEG][32];
   for (size_t S=0;S<NS;++S) {
      const size_t row = S / nseg;
      const int gseg = (int)(S % nseg);
      const int uy = (int)(row % c->nd[1]), uz = (int)(row / c->nd[1]);
      const int u0 = gseg*SEG, u1 = u0 + SEG < ndx ? u0 + SEG : ndx;
      int64_t nrec = 0;
      for (int s=0;s<c->ns;++s) {
         const PopStore* ps = &c->pop[s];
         double* q5 = &c->cnt[RHGPU_NUM_FIELD_COUNTERS + RHGPU_CNT_PER_SPECIES*s];
         for (int64_t p=0;p<(int64_t)ps->cnt[S];++p) {
            double st[7];
            memcpy(st,ps->p + 7*(ps->start[S]+p),sizeof st);
            const size_t cb = cellOfDual(c,u0 + ps->lx[ps->start[S]+p],uy,uz,st);
            q5[0] += pushParticle(c,s,cb,st);
            const int ci = (int)(cb % c->nx), cj = (int)((cb / c->nx) % c->ny), ck = (int)(cb / ((size_t)c->nx*c->ny));
            int off[3];
            const int bad = rh_migrate_canonical(st,dx,c->dxBelow,off);
            int ti = ci+off[0], tj = cj+off[1], tk = ck+off[2];
            const int inside = rh_wrap(&ti,c->nx,P->periodic[0]) && rh_wrap(&tj,c->ny,P->periodic[1]) && rh_wrap(&tk,c->nz,P->periodic[2]);
            const double ke = st[6]*( sqr(st[3]) + sqr(st[4]) + sqr(st[5]) );
            if (bad || !inside) { q5[1] += st[6]; q5[2] += ke; continue; }
            const size_t cn = (size_t)ti + c->nx*((size_t)tj + c->ny*(size_t)tk);
            const int bx = ti + halfS(st[0],dx) - 1, by = tj + halfS(st[1],dx) - 1, bz = tk + halfS(st[2],dx) - 1;
            const int vx = dualU(bx,c->nx,P->periodic[0]), vy = dualU(by,c->ny,P->periodic[1]), vz = dualU(bz,c->nz,P->periodic[2]);
            const int inSeg = vy == uy && vz == uz && vx >= u0 && vx < u1;
            if (c->sp[s].accumulate) {
               double w8[8]; int ind[8];
               cicWeights(st,c->sp[s].q,dx,w8,ind);
               if (inSeg) {
                  ORecord* r = &recs[nrec++];
                  r->d = vx - u0;
                  memcpy(r->w8,w8,sizeof w8);
                  r->f[0] = 1.0; r->f[1] = st[3]; r->f[2] = st[4]; r->f[3] = st[5];
               } else {
                  for (int o=0;o<8;++o) {
                     int dxc = bx + (o&1), dyc = by + ((o>>1)&1), dzc = bz + ((o>>2)&1);
                     if (!rh_wrap(&dxc,c->nx,P->periodic[0]) || !rh_wrap(&dyc,c->ny,P->periodic[1]) || !rh_wrap(&dzc,c->nz,P->periodic[2])) continue;
                     const size_t dc = (size_t)dxc + c->nx*((size_t)dyc + c->ny*(size_t)dzc);
                     c->MM[dc] += (__int128)llrint(w8[o]*scaleR);
                     for (int l=0;l<3;++l) c->MM[(size_t)(1+l)*c->N + dc] += (__int128)llrint(w8[o]*st[3+l]*scaleJ);
                  }
               }
            }
            /* boundary conditions of the step (particle_boundary_cond_hybrid.h:112-185) */
            if (c->nflags[cn] != ALL_NBRS) { q5[1] += st[6]; q5[2] += ke; continue; }
            if (c->cflags[cn] & RHGPU_FLAG_INNER_PARTICLE) {
               const double xp = rh_block_origin(P->x_min,ti,dx) + st[0];
               const double yp = rh_block_origin(P->y_min,tj,dx) + st[1];
               const double zp = rh_block_origin(P->z_min,tk,dx) + st[2];
               if (sqr(xp) + sqr(yp) + sqr(zp) < c->sp[s].R2_obstacle) { q5[3] += st[6]; q5[4] += ke; continue; }
            }
            if (inSeg) {
               memcpy(sw[s] + 7*sn[s],st,sizeof st);
               slx[s][sn[s]] = (uint8_t)(vx - u0);
               sn[s]++;
               scnt[s][S]++;
            } else {
               OMover* m = &mv[s][mn[s]++];
               memcpy(m->st,st,sizeof st);
               m->key = ((uint64_t)S << 32) | (uint64_t)p;
               m->dest = ((int64_t)vy + (int64_t)c->nd[1]*vz)*nseg + vx/SEG;
               m->lx = vx % SEG;
            }
         }
      }
      /* the segment's sums, records of each dual cell in list order */
      for (int d=0;d<SEG;++d) for (int q=0;q<32;++q) acc[d][q] = 0.0;
      for (int64_t r=0;r<nrec;++r)
         for (int q=0;q<32;++q) acc[recs[r].d][q] += recs[r].w8[q >> 2]*recs[r].f[q & 3];
      /* row partials of the cells whose lower dual cell is in this segment */
      for (int dl=0;dl<u1-u0;++dl) {
         const int lo = u0 + dl;
         int x, hi;
         if (P->periodic[0]) {
            x = lo + 1 == c->nx ? 0 : lo + 1;
            hi = lo + 1 < u1 ? dl + 1 : (nseg == 1 ? 0 : -1);
         } else {
            x = lo;
            if (x >= c->nx) continue;
            hi = lo + 1 < u1 ? dl + 1 : -1;
         }
         for (int qq=0;qq<4;++qq) for (int m=0;m<4;++m) {
            double v = acc[dl][((1 + 2*qq) << 2) + m];
            if (hi >= 0) v = v + acc[hi][((2*qq) << 2) + m];
            c->RP[(((size_t)qq*nrows + row)*c->nx + x)*4 + m] = v;
         }
      }
      if (P->periodic[0] ? nseg > 1 : gseg >= 1)
         for (int qq=0;qq<4;++qq) for (int m=0;m<4;++m)
            c->RPB[(((size_t)qq*nrows + row)*nseg + gseg)*4 + m] = acc[0][((2*qq) << 2) + m];
   }
   free(recs);
   /* new storage: per segment its stayers, then its arrivals by key */
   for (int s=0;s<c->ns;++s) {
      PopStore* ps = &c->pop[s];
      qsort(mv[s],mn[s],sizeof(OMover),cmpMover);
      uint32_t* arr = (uint32_t*)calloc(NS,sizeof(uint32_t));
      for (int64_t m=0;m<mn[s];++m) arr[mv[s][m].dest]++;
      for (size_t S=0;S<NS;++S) ps->cnt[S] = scnt[s][S] + arr[S];
      popReserveLx(ps,sn[s] + mn[s]);
      segStarts(c,ps);
      int64_t* fill = (int64_t*)malloc(sizeof(int64_t)*(NS > 0 ? NS : 1));
      int64_t q = 0;
      for (size_t S=0;S<NS;++S) {
         memcpy(ps->p + 7*ps->start[S],sw[s] + 7*q,sizeof(double)*7*scnt[s][S]);
         memcpy(ps->lx + ps->start[S],slx[s] + q,scnt[s][S]);
         q += scnt[s][S];
         fill[S] = ps->start[S] + scnt[s][S];
      }
      for (int64_t m=0;m<mn[s];++m) {
         const OMover* M = &mv[s][m];
         const int64_t d = fill[M->dest]++;
         memcpy(ps->p + 7*d,M->st,sizeof M->st);
         ps->lx[d] = (uint8_t)M->lx;
      }
      free(fill); free(arr);
      free(sw[s]); free(slx[s]); free(scnt[s]); free(mv[s]);
   }
}

/* 128-bit fixed point to double: hi*2^(64-k) + lo*2^-k, each term rounded */
static double fixedToDouble(__int128 v,int k) {
   const int64_t hi = (int64_t)(v >> 64);
   const uint64_t lo = (uint64_t)v;
   return ldexp((double)hi,64 - k) + ldexp((double)lo,-k);
}

static void dualGather(Ctx* c) {
   const rhgpu_params* P = &c->P;
   double* rho = c->arr[RHGPU_CELL_RHOQI];
   double* Ji = c->arr[RHGPU_CELL_JI];
   const size_t nrows = (size_t)c->nd[1]*c->nd[2];
   const double dV = P->dx*P->dx*P->dx;
   for (int z=0;z<c->nz;++z) for (int y=0;y<c->ny;++y) for (int x=0;x<c->nx;++x) {
      const size_t n = (size_t)x + c->nx*((size_t)y + c->ny*(size_t)z);
      const int bnd = P->periodic[0] ? (c->nseg > 1 && x % SEG == 0) : ((x + 1) % SEG == 0);
      const int gb = P->periodic[0] ? x / SEG : (x + 1) / SEG;
      double v[4];
      for (int qq=0;qq<4;++qq) {
         const int uy = dualU(y - (qq & 1),c->ny,P->periodic[1]);
         const int uz = dualU(z - (qq >> 1),c->nz,P->periodic[2]);
         const size_t row = (size_t)uy + (size_t)c->nd[1]*uz;
         const double* rp = c->RP + (((size_t)qq*nrows + row)*c->nx + x)*4;
         const double* rb = c->RPB + (((size_t)qq*nrows + row)*c->nseg + gb)*4;
         for (int l=0;l<4;++l) {
            double r = rp[l];
            if (bnd) r = r + rb[l];
            v[l] = qq == 0 ? r : v[l] + r;
         }
      }
      v[0] += fixedToDouble(c->MM[n],c->kR);
      for (int l=0;l<3;++l) v[1+l] += fixedToDouble(c->MM[(size_t)(1+l)*c->N + n],c->kJ);
      double r = v[0]/dV;
      if (r < P->min_ion_charge_density) { r = P->min_ion_charge_density; c->cnt[RHGPU_CNT_FIELD_MIN_CELL_RHOQI] += 1; }
      rho[n] = r;
      for (int l=0;l<3;++l) Ji[3*n+l] = v[1+l]/dV;
   }
}

/* ------------------------------------------------------------------ */
/* field update: propagateB (hybrid_propagator.cpp:42-440)              */

#define A(id) (c->arr[id])

/* face2Cell (:1043-1056) */
static void face2CellFn(Ctx* c,size_t b) {
   if (c->nflags[b] != ALL_NBRS) return;
   const double* f = A(RHGPU_FACE_B); double* cb = A(RHGPU_CELL_B);
   cb[3*b+0] = 0.5*(f[3*b+0] + f[3*(size_t)nb(c,b,-1,0,0)+0]);
   cb[3*b+1] = 0.5*(f[3*b+1] + f[3*(size_t)nb(c,b,0,-1,0)+1]);
   cb[3*b+2] = 0.5*(f[3*b+2] + f[3*(size_t)nb(c,b,0,0,-1)+2]);
}

/* neumannCell (:443-655): exterior cells copy the inward neighbour; rules
 * applied in the reference's order on a snapshot taken per cell. */
static const int NEU_RULES[26][4] = {
   /* mask bits: 1=-x 2=+y 4=-y 8=+z 16=-z 32=+x ; then source offset */
   {1, +1,0,0},{2, 0,-1,0},{4, 0,+1,0},{8, 0,0,-1},{16, 0,0,+1},{32, -1,0,0},
   {1|4, +1,+1,0},{1|2, +1,-1,0},{32|4, -1,+1,0},{32|2, -1,-1,0},
   {1|16, +1,0,+1},{1|8, +1,0,-1},{32|16, -1,0,+1},{32|8, -1,0,-1},
   {4|16, 0,+1,+1},{4|8, 0,+1,-1},{2|16, 0,-1,+1},{2|8, 0,-1,-1},
   {1|4|16, +1,+1,+1},{1|4|8, +1,+1,-1},{1|2|16, +1,-1,+1},{1|2|8, +1,-1,-1},
   {32|4|16, -1,+1,+1},{32|4|8, -1,+1,-1},{32|2|16, -1,-1,+1},{32|2|8, -1,-1,-1}
};
static int missingMask(uint32_t f) {
   int m = 0;
   if (!(f & XNEG)) m |= 1;
   if (!(f & YPOS)) m |= 2;
   if (!(f & YNEG)) m |= 4;
   if (!(f & ZPOS)) m |= 8;
   if (!(f & ZNEG)) m |= 16;
   if (!(f & XPOS)) m |= 32;
   return m;
}
static void neumannCell(Ctx* c,double* d,int dim) {
   for (size_t e=0;e<c->nexterior;++e) {
      const size_t b = (size_t)c->exterior[e];
      const int m = missingMask(c->nflags[b]);
      double aa[27][3];
      for (int t=0;t<27;++t) {
         const int n = c->nbr[b*27+t];
         for (int l=0;l<dim;++l) aa[t][l] = n >= 0 ? d[(size_t)n*dim+l] : 0.0;
      }
      for (int r=0;r<26;++r) {
         if ((m & NEU_RULES[r][0]) != NEU_RULES[r][0]) continue;
         const int t = TID(NEU_RULES[r][1],NEU_RULES[r][2],NEU_RULES[r][3]);
         for (int l=0;l<dim;++l) d[b*dim+l] = aa[t][l];
      }
   }
}

/* neumannFace (:659-908): per rule, which components are copied from which
 * neighbour (the last rule of the reference, +x+y+z corner, copies none) */
typedef struct { int mask; int src[3][3]; int use[3]; } FaceRule;
static const FaceRule FACE_RULES[] = {
   {1,      {{0,0,0},{+1,0,0},{+1,0,0}},   {0,1,1}},
   {2,      {{0,-1,0},{0,0,0},{0,-1,0}},   {1,0,1}},
   {4,      {{0,+1,0},{0,0,0},{0,+1,0}},   {1,0,1}},
   {8,      {{0,0,-1},{0,0,-1},{0,0,0}},   {1,1,0}},
   {16,     {{0,0,+1},{0,0,+1},{0,0,0}},   {1,1,0}},
   {32,     {{0,0,0},{-1,0,0},{-1,0,0}},   {0,1,1}},
   {1|4,    {{0,+1,0},{+1,0,0},{+1,+1,0}}, {1,1,1}},
   {1|2,    {{0,-1,0},{0,0,0},{+1,-1,0}},  {1,0,1}},
   {32|4,   {{0,0,0},{-1,0,0},{-1,+1,0}},  {0,1,1}},
   {32|2,   {{0,0,0},{0,0,0},{-1,-1,0}},   {0,0,1}},
   {1|16,   {{0,0,+1},{+1,0,+1},{+1,0,0}}, {1,1,1}},
   {1|8,    {{0,0,-1},{+1,0,-1},{0,0,0}},  {1,1,0}},
   {32|16,  {{0,0,0},{-1,0,+1},{-1,0,0}},  {0,1,1}},
   {32|8,   {{0,0,0},{-1,0,-1},{0,0,0}},   {0,1,0}},
   {4|16,   {{0,+1,+1},{0,0,+1},{0,+1,0}}, {1,1,1}},
   {4|8,    {{0,+1,-1},{0,0,-1},{0,0,0}},  {1,1,0}},
   {2|16,   {{0,-1,+1},{0,0,0},{0,-1,0}},  {1,0,1}},
   {2|8,    {{0,-1,-1},{0,0,0},{0,0,0}},   {1,0,0}},
   {1|4|16, {{0,+1,+1},{+1,0,+1},{+1,+1,0}},{1,1,1}},
   {1|4|8,  {{0,+1,-1},{+1,0,-1},{0,0,0}}, {1,1,0}},
   {1|2|16, {{0,-1,+1},{0,0,0},{+1,-1,0}}, {1,0,1}},
   {1|2|8,  {{0,-1,-1},{0,0,0},{0,0,0}},   {1,0,0}},
   {32|4|16,{{0,0,0},{-1,0,+1},{-1,+1,0}}, {0,1,1}},
   {32|4|8, {{0,0,0},{-1,0,-1},{0,0,0}},   {0,1,0}},
   {32|2|16,{{0,0,0},{0,0,0},{-1,-1,0}},   {0,0,1}},
};
static void neumannFace(Ctx* c,double* d) {
   const int nr = (int)(sizeof(FACE_RULES)/sizeof(FACE_RULES[0]));
   for (size_t e=0;e<c->nexterior;++e) {
      const size_t b = (size_t)c->exterior[e];
      const int m = missingMask(c->nflags[b]);
      double aa[27][3];
      for (int t=0;t<27;++t) {
         const int n = c->nbr[b*27+t];
         for (int l=0;l<3;++l) aa[t][l] = n >= 0 ? d[(size_t)n*3+l] : 0.0;
      }
      for (int r=0;r<nr;++r) {
         if ((m & FACE_RULES[r].mask) != FACE_RULES[r].mask) continue;
         for (int l=0;l<3;++l) {
            if (!FACE_RULES[r].use[l]) continue;
            const int t = TID(FACE_RULES[r].src[l][0],FACE_RULES[r].src[l][1],FACE_RULES[r].src[l][2]);
            d[b*3+l] = aa[t][l];
         }
      }
   }
}

/* setIMFCell (:910-977), setIMFFace (:979-1040) */
static void setIMFCell(Ctx* c,double* cb) {
   const int order[6] = {32,1,2,4,8,16}; /* +x -x +y -y +z -z */
   for (size_t e=0;e<c->nexterior;++e) {
      const size_t b = (size_t)c->exterior[e];
      const int m = missingMask(c->nflags[b]);
      for (int w=0;w<6;++w) {
         if (!(m & order[w]) || !c->P.imf_boundary_cellB[w]) continue;
         for (int l=0;l<3;++l) cb[3*b+l] = c->P.imf_B[l];
      }
   }
}
static void setIMFFace(Ctx* c,double* fb) {
   const int order[6] = {32,1,2,4,8,16};
   for (size_t e=0;e<c->nexterior;++e) {
      const size_t b = (size_t)c->exterior[e];
      const int m = missingMask(c->nflags[b]);
      for (int w=0;w<6;++w) {
         if (!(m & order[w]) || !c->P.imf_boundary_faceB[w]) continue;
         const int axis = w/2; /* the face normal component is kept */
         for (int l=0;l<3;++l) if (l != axis) fb[3*b+l] = c->P.imf_B[l];
      }
   }
}

/* cell2Node (:1059-1089): node at the (+,+,+) corner = mean of 8 cells */
static void cell2Node(Ctx* c,const double* cd,double* nd,int dim) {
   for (size_t b=0;b<c->N;++b) {
      if (c->nflags[b] != ALL_NBRS && !plusOk(c->nflags[b])) continue;
      const size_t n000 = b, n001 = nb(c,b,0,0,1), n010 = nb(c,b,0,1,0), n100 = nb(c,b,1,0,0);
      const size_t n011 = nb(c,b,0,1,1), n110 = nb(c,b,1,1,0), n101 = nb(c,b,1,0,1), n111 = nb(c,b,1,1,1);
      for (int l=0;l<dim;++l) {
         nd[b*dim+l] = 0.125*(cd[n000*dim+l] + cd[n001*dim+l] + cd[n010*dim+l] + cd[n100*dim+l] +
                              cd[n011*dim+l] + cd[n110*dim+l] + cd[n101*dim+l] + cd[n111*dim+l]);
      }
   }
}

/* node2Cell (:1092-1112): cell = mean of its 8 corner nodes */
static void node2Cell(Ctx* c,const double* nd,double* cd) {
   for (size_t b=0;b<c->N;++b) {
      if (c->nflags[b] != ALL_NBRS) continue;
      const size_t a0 = b, a1 = nb(c,b,-1,0,0), a2 = nb(c,b,-1,-1,0), a3 = nb(c,b,0,-1,0);
      const size_t a4 = nb(c,b,0,0,-1), a5 = nb(c,b,0,-1,-1), a6 = nb(c,b,-1,0,-1), a7 = nb(c,b,-1,-1,-1);
      for (int l=0;l<3;++l) {
         cd[3*b+l] = 0.125*(nd[3*a0+l] + nd[3*a1+l] + nd[3*a2+l] + nd[3*a3+l] +
                            nd[3*a4+l] + nd[3*a5+l] + nd[3*a6+l] + nd[3*a7+l]);
      }
   }
}

/* calcNodeJ (:1449-1522), USE_EDGE_J */
static void calcNodeJFn(Ctx* c,size_t b) {
   if (c->nflags[b] != ALL_NBRS && !plusOk(c->nflags[b])) return;
   const double* f = A(RHGPU_FACE_B);
   const double* nB = A(RHGPU_NODE_B);
   const double* nR = A(RHGPU_NODE_RHOQI);
   double* nJ = A(RHGPU_NODE_J);
#define F(di,dj,dk,l) f[3*(size_t)nb(c,b,di,dj,dk)+(l)]
   const double edgeJx1 = - F(0,0,0,2) + F(0,0,0,1) + F(0,1,0,2) - F(0,0,1,1);
   const double edgeJx2 = - F(1,0,0,2) + F(1,0,0,1) + F(1,1,0,2) - F(1,0,1,1);
   const double edgeJy1 = + F(0,0,0,2) + F(0,0,1,0) - F(1,0,0,2) - F(0,0,0,0);
   const double edgeJy2 = + F(0,1,0,2) + F(0,1,1,0) - F(1,1,0,2) - F(0,1,0,0);
   const double edgeJz1 = - F(0,0,0,1) + F(0,0,0,0) + F(1,0,0,1) - F(0,1,0,0);
   const double edgeJz2 = - F(0,0,1,1) + F(0,0,1,0) + F(1,0,1,1) - F(0,1,1,0);
#undef F
   double d = 1.0;
   double vw = 0.0;
   const double ne = nR[b]/RHGPU_CHARGE_ELEMENTARY;
   const double Btot = sqrt( sqr(nB[3*b+0]) + sqr(nB[3*b+1]) + sqr(nB[3*b+2]) );
   if (ne > 0.0 && c->P.dx > 0.0) {
      vw = 2.0*Btot*M_PI/( RHGPU_PERMEABILITY*ne*RHGPU_CHARGE_ELEMENTARY*c->P.dx );
   }
   if (vw > c->P.max_whistler_speed && c->P.max_whistler_speed > 0.0) {
      d = vw/c->P.max_whistler_speed;
      c->cnt[RHGPU_CNT_FIELD_MAX_VW] += 1;
   }
   const double a = 0.5/(c->P.dx*RHGPU_PERMEABILITY*d);
   nJ[3*b+0] = (edgeJx1 + edgeJx2)*a;
   nJ[3*b+1] = (edgeJy1 + edgeJy2)*a;
   nJ[3*b+2] = (edgeJz1 + edgeJz2)*a;
}

/* calcCellUe (:1342-1387) */
static void calcCellUe(Ctx* c) {
   const double* J = A(RHGPU_CELL_J); const double* Ji = A(RHGPU_CELL_JI);
   const double* rho = A(RHGPU_CELL_RHOQI); double* Ue = A(RHGPU_CELL_UE);
   for (size_t b=0;b<c->N;++b) {
      if (c->nflags[b] != ALL_NBRS) continue;
      if (c->cflags[b] & RHGPU_FLAG_INNER_FIELD) {
         for (int l=0;l<3;++l) Ue[3*b+l] = c->P.field_obstacle_Ue[l];
         continue;
      }
      for (int l=0;l<3;++l) {
         if (fabs(rho[b]) > 0) {
            if (c->P.use_hall) Ue[3*b+l] = -(J[3*b+l] - Ji[3*b+l])/rho[b];
            else Ue[3*b+l] = Ji[3*b+l]/rho[b];
         } else Ue[3*b+l] = 0.0;
      }
      const double Ue2 = sqr(Ue[3*b+0]) + sqr(Ue[3*b+1]) + sqr(Ue[3*b+2]);
      if (Ue2 > c->P.max_electron_speed2) {
         const double norm = sqrt(c->P.max_electron_speed2/Ue2);
         Ue[3*b+0] *= norm; Ue[3*b+1] *= norm; Ue[3*b+2] *= norm;
         c->cnt[RHGPU_CNT_FIELD_MAX_CELL_UE] += 1;
      }
   }
}

/* calcNodeUe (:1524-1584), USE_NODE_UE */
static void calcNodeUe(Ctx* c) {
   double* rho = A(RHGPU_NODE_RHOQI); const double* Ji = A(RHGPU_NODE_JI);
   const double* J = A(RHGPU_NODE_J); double* Ue = A(RHGPU_NODE_UE);
   for (size_t b=0;b<c->N;++b) {
      if (c->nflags[b] != ALL_NBRS && !plusOk(c->nflags[b])) continue;
      if (c->cflags[b] & RHGPU_FLAG_INNER_NODE) {
         for (int l=0;l<3;++l) Ue[3*b+l] = c->P.field_obstacle_Ue[l];
         continue;
      }
      if (rho[b] < c->P.min_ion_charge_density) {
         rho[b] = c->P.min_ion_charge_density;
         c->cnt[RHGPU_CNT_FIELD_MIN_NODE_RHOQI] += 1;
      }
      for (int l=0;l<3;++l) {
         if (fabs(rho[b]) > 0) {
            if (c->P.use_hall) Ue[3*b+l] = -(J[3*b+l] - Ji[3*b+l])/rho[b];
            else Ue[3*b+l] = Ji[3*b+l]/rho[b];
         } else Ue[3*b+l] = 0.0;
      }
      const double Ue2 = sqr(Ue[3*b+0]) + sqr(Ue[3*b+1]) + sqr(Ue[3*b+2]);
      if (Ue2 > c->P.max_electron_speed2) {
         const double norm = sqrt(c->P.max_electron_speed2/Ue2);
         Ue[3*b+0] *= norm; Ue[3*b+1] *= norm; Ue[3*b+2] *= norm;
         c->cnt[RHGPU_CNT_FIELD_MAX_NODE_UE] += 1;
      }
   }
}

/* upwindNodeB (:1268-1339) */
static void upwindNodeBFn(Ctx* c,size_t b) {
   if (c->nflags[b] != ALL_NBRS && !plusOk(c->nflags[b])) return;
   const double* cB = A(RHGPU_CELL_B); const double* nUe = A(RHGPU_NODE_UE); double* nB = A(RHGPU_NODE_B);
   double xUpwind = -0.5, yUpwind = 0, zUpwind = 0;
   const double Ue = sqrt(sqr(nUe[3*b+0]) + sqr(nUe[3*b+1]) + sqr(nUe[3*b+2]));
   if (Ue > 0) {
      const double a = -0.5/Ue;
      xUpwind = nUe[3*b+0]*a; yUpwind = nUe[3*b+1]*a; zUpwind = nUe[3*b+2]*a;
   }
   /* cells around the node, offsets (X,Y,Z) in {0,1}; centroid at X-0.5 */
   const double w111 = 1/sqrt(sqr(-0.5-xUpwind) + sqr(-0.5-yUpwind) + sqr(-0.5-zUpwind));
   const double w112 = 1/sqrt(sqr(-0.5-xUpwind) + sqr(-0.5-yUpwind) + sqr(+0.5-zUpwind));
   const double w121 = 1/sqrt(sqr(-0.5-xUpwind) + sqr(+0.5-yUpwind) + sqr(-0.5-zUpwind));
   const double w211 = 1/sqrt(sqr(+0.5-xUpwind) + sqr(-0.5-yUpwind) + sqr(-0.5-zUpwind));
   const double w122 = 1/sqrt(sqr(-0.5-xUpwind) + sqr(+0.5-yUpwind) + sqr(+0.5-zUpwind));
   const double w221 = 1/sqrt(sqr(+0.5-xUpwind) + sqr(+0.5-yUpwind) + sqr(-0.5-zUpwind));
   const double w212 = 1/sqrt(sqr(+0.5-xUpwind) + sqr(-0.5-yUpwind) + sqr(+0.5-zUpwind));
   const double w222 = 1/sqrt(sqr(+0.5-xUpwind) + sqr(+0.5-yUpwind) + sqr(+0.5-zUpwind));
   const double wsum = w111+w112+w121+w211+w122+w221+w212+w222;
   if (wsum > 0) {
      const size_t c111 = b, c112 = nb(c,b,0,0,1), c121 = nb(c,b,0,1,0), c211 = nb(c,b,1,0,0);
      const size_t c122 = nb(c,b,0,1,1), c221 = nb(c,b,1,1,0), c212 = nb(c,b,1,0,1), c222 = nb(c,b,1,1,1);
      for (int l=0;l<3;++l) {
         nB[3*b+l] = (w111*cB[3*c111+l] + w112*cB[3*c112+l] + w121*cB[3*c121+l] + w211*cB[3*c211+l] +
                      w122*cB[3*c122+l] + w221*cB[3*c221+l] + w212*cB[3*c212+l] + w222*cB[3*c222+l])/wsum;
      }
   } else {
      nB[3*b+0] = nB[3*b+1] = nB[3*b+2] = 0.0;
   }
}

/* calcNodeE (:1392-1446) */
static void calcNodeE(Ctx* c) {
   const double* Ue = A(RHGPU_NODE_UE); const double* B = A(RHGPU_NODE_B);
   const double* eta = A(RHGPU_NODE_ETA); const double* J = A(RHGPU_NODE_J); double* E = A(RHGPU_NODE_E);
   for (size_t b=0;b<c->N;++b) {
      if (c->nflags[b] != ALL_NBRS && !plusOk(c->nflags[b])) continue;
      const size_t n3 = 3*b;
      E[n3+0] = -(Ue[n3+1]*B[n3+2] - Ue[n3+2]*B[n3+1]);
      E[n3+1] = -(Ue[n3+2]*B[n3+0] - Ue[n3+0]*B[n3+2]);
      E[n3+2] = -(Ue[n3+0]*B[n3+1] - Ue[n3+1]*B[n3+0]);
      E[n3+0] += eta[b]*J[n3+0];
      E[n3+1] += eta[b]*J[n3+1];
      E[n3+2] += eta[b]*J[n3+2];
      if (c->P.max_electric_field2 > 0) {
         const double E2 = sqr(E[n3+0]) + sqr(E[n3+1]) + sqr(E[n3+2]);
         if (E2 > c->P.max_electric_field2) {
            const double scaling = sqrt(c->P.max_electric_field2/E2);
            E[n3+0] *= scaling; E[n3+1] *= scaling; E[n3+2] *= scaling;
            c->cnt[RHGPU_CNT_FIELD_MAX_E] += 1;
         }
      }
   }
}

/* nodeAvg (:1115-1265): 27-point Gaussian. The reference's temp array is
 * initialised with only its first element set to numeric_limits::max()
 * (`new Real[n] {initVal}`), the rest to zero; neighbours that do not
 * exist therefore read 0, except the (-,-,-) corner x component, which reads
 * max() and is then excluded with renormalisation. Restated as is. */
static void nodeAvg(Ctx* c,const double* old,double* nd) {
   const double C1 = c->P.gaussian_coeffs[0], C2 = c->P.gaussian_coeffs[1];
   const double C3 = c->P.gaussian_coeffs[2], C4 = c->P.gaussian_coeffs[3];
   const double initVal = 1.7976931348623157e308;
   /* reference evaluation order of the 27 terms: (X,Y,Z) offsets + 1 */
   static const int ORD[27][3] = {
      {1,1,1},{1,1,0},{0,1,1},{1,2,1},{2,1,1},{1,0,1},{1,1,2},{0,1,0},{1,0,0},{1,2,0},{2,1,0},
      {0,0,1},{0,2,1},{2,2,1},{2,0,1},{0,1,2},{1,2,2},{2,1,2},{1,0,2},{0,0,2},{0,2,2},{2,0,2},
      {2,2,2},{0,0,0},{0,2,0},{2,0,0},{2,2,0}};
   for (size_t b=0;b<c->N;++b) {
      if (c->nflags[b] != ALL_NBRS && !plusOk(c->nflags[b])) continue;
      for (int l=0;l<3;++l) {
         double v[27], C[27];
         int zeroFound = 0;
         for (int q=0;q<27;++q) {
            const int X = ORD[q][0], Y = ORD[q][1], Z = ORD[q][2];
            const int n = nb(c,b,X-1,Y-1,Z-1);
            double val;
            if (n >= 0) val = old[3*(size_t)n+l];
            else val = (X == 0 && Y == 0 && Z == 0 && l == 0) ? initVal : 0.0;
            const int dist = (X != 1) + (Y != 1) + (Z != 1);
            double Cq = dist == 0 ? C1 : dist == 1 ? C2 : dist == 2 ? C3 : C4;
            if (val == initVal) { val = 0.0; Cq = 0.0; zeroFound = 1; }
            v[q] = val; C[q] = Cq;
         }
         if (zeroFound) {
            double Csum = C[0];
            for (int q=1;q<27;++q) Csum += C[q];
            if (Csum > 0.0) for (int q=0;q<27;++q) C[q] /= Csum;
         }
         double s = C[0]*v[0];
         for (int q=1;q<27;++q) s += C[q]*v[q];
         nd[3*b+l] = s;
      }
   }
}

/* faceCurl with doFaraday (:1587-1671) */
static void faradayFn(Ctx* c,size_t b) {
   int doX = 1, doY = 1, doZ = 1;
   const uint32_t f = c->nflags[b];
   if (f != ALL_NBRS) {
      if (!plusOk(f)) return;
      if (!(f & XNEG)) { doY = doZ = 0; }
      if (!(f & YNEG)) { doX = doZ = 0; }
      if (!(f & ZNEG)) { doX = doY = 0; }
   }
   const double* E = A(RHGPU_NODE_E); double* fb = A(RHGPU_FACE_B);
   const double dx = c->P.dx, dt = c->P.dt;
#define NE(di,dj,dk,l) E[3*(size_t)nb(c,b,di,dj,dk)+(l)]
   if (doX) {
      const double n5y = NE(0,-1,0,1), n5z = NE(0,-1,0,2), n6y = NE(0,-1,-1,1), n6z = NE(0,-1,-1,2);
      const double n7y = NE(0,0,-1,1), n7z = NE(0,0,-1,2), n8y = NE(0,0,0,1), n8z = NE(0,0,0,2);
      const double curlX = 0.5*(+n5z+n6z-n6y-n7y-n7z-n8z+n8y+n5y)/dx;
      fb[3*b+0] += dt*curlX;
   }
   if (doY) {
      const double n3x = NE(-1,0,-1,0), n3z = NE(-1,0,-1,2), n4x = NE(-1,0,0,0), n4z = NE(-1,0,0,2);
      const double n7x = NE(0,0,-1,0), n7z = NE(0,0,-1,2), n8x = NE(0,0,0,0), n8z = NE(0,0,0,2);
      const double curlY = 0.5*(-n4x-n8x+n8z+n7z+n7x+n3x-n3z-n4z)/dx;
      fb[3*b+1] += dt*curlY;
   }
   if (doZ) {
      const double n1x = NE(-1,-1,0,0), n1y = NE(-1,-1,0,1), n4x = NE(-1,0,0,0), n4y = NE(-1,0,0,1);
      const double n5x = NE(0,-1,0,0), n5y = NE(0,-1,0,1), n8x = NE(0,0,0,0), n8y = NE(0,0,0,1);
      const double curlZ = 0.5*(-n1x-n5x-n5y-n8y+n8x+n4x+n4y+n1y)/dx;
      fb[3*b+2] += dt*curlZ;
   }
#undef NE
}

/* calcCellEp (:1674-1737) */
static void calcCellEpFn(Ctx* c,size_t b) {
   if (c->nflags[b] != ALL_NBRS) return;
   const double* nr = A(RHGPU_NODE_RHOQI); const double* cr = A(RHGPU_CELL_RHOQI); double* Ep = A(RHGPU_CELL_EP);
   Ep[3*b+0] = 0.0; Ep[3*b+1] = 0.0; Ep[3*b+2] = 0.0;
   if (c->cflags[b] & RHGPU_FLAG_INNER_CELLEP) return;
#define R(di,dj,dk) nr[(size_t)nb(c,b,di,dj,dk)]
   const double xPos = 0.25*(R(0,0,0) + R(0,0,-1) + R(0,-1,-1) + R(0,-1,0));
   const double xNeg = 0.25*(R(-1,0,0) + R(-1,0,-1) + R(-1,-1,-1) + R(-1,-1,0));
   const double yPos = 0.25*(R(0,0,0) + R(0,0,-1) + R(-1,0,-1) + R(-1,0,0));
   const double yNeg = 0.25*(R(0,-1,0) + R(0,-1,-1) + R(-1,-1,-1) + R(-1,-1,0));
   const double zPos = 0.25*(R(0,0,0) + R(0,-1,0) + R(-1,-1,0) + R(-1,0,0));
   const double zNeg = 0.25*(R(0,0,-1) + R(0,-1,-1) + R(-1,-1,-1) + R(-1,0,-1));
#undef R
   const double dx = c->P.dx, C = c->P.electron_pressure_coeff;
   const double gx = (xPos - xNeg)/dx, gy = (yPos - yNeg)/dx, gz = (zPos - zNeg)/dx;
   if (!c->P.isothermal_electrons) {
      Ep[3*b+0] = -C*gx; Ep[3*b+1] = -C*gy; Ep[3*b+2] = -C*gz;
   } else if (fabs(cr[b]) > 0) {
      Ep[3*b+0] = -C*gx/cr[b]; Ep[3*b+1] = -C*gy/cr[b]; Ep[3*b+2] = -C*gz/cr[b];
   }
}

int rho_propagate_fields(void* h) {
   Ctx* c = (Ctx*)h;
   /* face -> cell B */
   forCells(c,face2CellFn);
   /* ghost cells */
   neumannCell(c,A(RHGPU_CELL_B),3);
   neumannCell(c,A(RHGPU_CELL_JI),3);
   neumannCell(c,A(RHGPU_CELL_RHOQI),1);
   setIMFCell(c,A(RHGPU_CELL_B));
   /* temporal average of cellB (WRITE_GRID_TEMPORAL_AVERAGES, :157-167) */
   {
      double* avg = A(RHGPU_CELL_AVERAGE_B); const double* cb = A(RHGPU_CELL_B);
      for (size_t i=0;i<3*c->N;++i) avg[i] += cb[i];
      c->cnt[RHGPU_CNT_GRID_AVERAGE_COUNTER] += 1;
   }
   /* cell -> node B, rho, Ji */
   cell2Node(c,A(RHGPU_CELL_B),A(RHGPU_NODE_B),3);
   cell2Node(c,A(RHGPU_CELL_RHOQI),A(RHGPU_NODE_RHOQI),1);
   cell2Node(c,A(RHGPU_CELL_JI),A(RHGPU_NODE_JI),3);
   /* nodeJ = avg edge curl(faceB)/mu0 */
   neumannFace(c,A(RHGPU_FACE_B));
   setIMFFace(c,A(RHGPU_FACE_B));
   {
      /* the whistler counter is summed in calcNodeJFn: serial pass */
      for (size_t b=0;b<c->N;++b) calcNodeJFn(c,b);
   }
   node2Cell(c,A(RHGPU_NODE_J),A(RHGPU_CELL_J));
   calcCellUe(c);
   neumannCell(c,A(RHGPU_CELL_UE),3);
   calcNodeUe(c);
   forCells(c,upwindNodeBFn);
   calcNodeE(c);
   for (int i=0;i<c->P.n_linear_smoothings_nodeE;++i) {
      node2Cell(c,A(RHGPU_NODE_E),A(RHGPU_CELL_J));
      neumannCell(c,A(RHGPU_CELL_J),3);
      cell2Node(c,A(RHGPU_CELL_J),A(RHGPU_NODE_E),3);
      memset(A(RHGPU_CELL_J),0,sizeof(double)*3*c->N);
   }
   if (c->P.use_gaussian_smoothing_nodeE) {
      double* old = (double*)malloc(sizeof(double)*3*c->N);
      memcpy(old,A(RHGPU_NODE_E),sizeof(double)*3*c->N);
      nodeAvg(c,old,A(RHGPU_NODE_E));
      free(old);
   }
   forCells(c,faradayFn);
   if (c->P.use_electron_pressure) forCells(c,calcCellEpFn);
   c->t += c->P.dt;
   return 0;
}

int rho_step(void* h,int32_t nsteps) {
   for (int n=0;n<nsteps;++n) {
      rho_push(h);
      rho_accumulate(h);
      rho_apply_boundaries(h);
      rho_propagate_fields(h);
   }
   return 0;
}

int rho_get_counters(void* h,double* out,int32_t n) {
   Ctx* c = (Ctx*)h;
   const int tot = RHGPU_NUM_FIELD_COUNTERS + RHGPU_CNT_PER_SPECIES*c->ns;
   for (int i=0;i<n && i<tot;++i) out[i] = c->cnt[i];
   return 0;
}

int rho_get_time(void* h,double* t,int64_t* ts) { Ctx* c = (Ctx*)h; *t = c->t; *ts = c->timestep; return 0; }
