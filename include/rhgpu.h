/* rhgpu.h - C ABI of the B200 (sm_100a) hybrid-PIC hot path for RHybrid.
 *
 * One time step of RHybrid's propagate() (src/user.cpp:49-158, order at
 * :118-134) runs on one GPU behind these entry points:
 *   1. Boris-Buneman ion push with the field gather at the particle
 *      (src/particle_propagator_boris_buneman.h:64-194, getFields
 *      src/hybrid_propagator.cpp:1879-1891): face-linear B, NGP Ue and Ep.
 *   2. Cell-to-cell migration of particles that left their cell (Corsair's
 *      particle list, not vendored): a coordinate that left [0,dx) shifts by
 *      exactly one cell (x+dx or x-dx; x+dx >= dx becomes the largest double
 *      below dx); a particle that moved more than one cell, or left a
 *      non-periodic box, is removed and counted as an escape.
 *   3. CIC charge and ion-current deposit (src/particle_accumulator.cpp:44-156)
 *      with the finalize step /dV and rho clamp (:319-333).
 *   4. Particle boundary conditions (src/particle_boundary_cond_hybrid.h:112-185).
 *   5. The staggered-grid field update propagateB (src/hybrid_propagator.cpp:42-440).
 *
 * Conventions shared with the reference:
 *   - cells are Corsair 1x1x1 blocks; the linear cell index is
 *     n = i + nx*(j + ny*k), x fastest;
 *   - vector grid arrays crossing this ABI are interleaved per cell
 *     (component l of cell n at [3*n+l]), exactly as ParGrid stores them;
 *   - a particle is 7 doubles {X,Y,Z,VX,VY,VZ,WEIGHT} with X,Y,Z local to
 *     its cell, in [0,dx) (src/particle_definition.h:29-38); particle arrays
 *     crossing this ABI are grouped by cell in linear cell order, with a
 *     per-cell count array (the flattened form of ParGrid's per-cell lists).
 *
 * All entry points return 0 on success or an RHGPU_ERR_* code; the text of
 * the last error of the calling thread is returned by rhgpu_last_error().
 * A context is used by one host thread at a time.
 */
#ifndef RHGPU_H
#define RHGPU_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Physical constants. Corsair's constants:: namespace is not vendored with
 * the reference; these are the CODATA 2018 values it is expected to hold
 * (used at src/hybrid_propagator.cpp:1505-1517, src/particle_species.cpp:67-94). */
#define RHGPU_PERMEABILITY       1.2566370614359173e-06
#define RHGPU_CHARGE_ELEMENTARY  1.602176634e-19
#define RHGPU_MASS_PROTON        1.67262192369e-27
#define RHGPU_BOLTZMANN          1.380649e-23
#define RHGPU_GRAVITY            6.67430e-11
/* used by the field log's scales and energies (src/diagnostics.h:375-395, 691-704) */
#define RHGPU_MASS_ELECTRON      9.1093837015e-31
#define RHGPU_PERMITTIVITY       8.8541878128e-12
#define RHGPU_SPEED_OF_LIGHT     299792458.0

/* status codes */
#define RHGPU_OK              0
#define RHGPU_ERR_ARG         1  /* bad argument */
#define RHGPU_ERR_CUDA        2  /* CUDA runtime error */
#define RHGPU_ERR_STATE       3  /* call out of order (e.g. step before upload) */
#define RHGPU_ERR_DEVICE      4  /* a kernel raised its device error word (see rhgpu_device_errors) */
#define RHGPU_ERR_NOMEM       5  /* device allocation failed */
#define RHGPU_ERR_CAPACITY    6  /* particle storage capacity exceeded */

/* device error word bits (rhgpu_device_errors) */
#define RHGPU_DEVERR_NAN_PARTICLE   1u  /* non-finite particle coordinate after the push */
#define RHGPU_DEVERR_FAST_PARTICLE  2u  /* particle moved more than one cell in a step */
#define RHGPU_DEVERR_CAPACITY       4u  /* particle buffer overflow during migration */
#define RHGPU_DEVERR_INJECT         8u  /* a particle source's rejection sampling ran out of tries */
#define RHGPU_DEVERR_DENOISER      16u  /* a denoiser convolution's wait on its tensor-core work ran out */

/* per-cell flag bits of the cell_flags array (user.cpp:1883-1941) */
#define RHGPU_FLAG_INNER_FIELD     1u  /* innerFlagField: cell centre inside R_fieldObstacle */
#define RHGPU_FLAG_INNER_NODE      2u  /* innerFlagNode: (+,+,+) node inside R_fieldObstacle */
#define RHGPU_FLAG_INNER_PARTICLE  4u  /* innerFlagParticle: cell may hold obstacle particles */
#define RHGPU_FLAG_INNER_CELLEP    8u  /* innerFlagCellEp: electron pressure field zeroed */

/* grid arrays addressable through rhgpu_download_array / rhgpu_upload_array
 * (names of the Hybrid:: DataIDs in src/hybrid.h:166-187) */
enum rhgpu_array_id {
   RHGPU_FACE_B = 0,      /* faceB,     3 per cell: component l lives on the +l face */
   RHGPU_CELL_B,          /* cellB,     3 */
   RHGPU_CELL_UE,         /* cellUe,    3 */
   RHGPU_CELL_EP,         /* cellEp,    3 */
   RHGPU_CELL_RHOQI,      /* cellRhoQi, 1 */
   RHGPU_CELL_JI,         /* cellJi,    3 */
   RHGPU_CELL_J,          /* cellJ,     3 */
   RHGPU_NODE_RHOQI,      /* nodeRhoQi, 1: node at the (+,+,+) corner of the cell */
   RHGPU_NODE_JI,         /* nodeJi,    3 */
   RHGPU_NODE_J,          /* nodeJ,     3 */
   RHGPU_NODE_UE,         /* nodeUe,    3 */
   RHGPU_NODE_B,          /* nodeB,     3 */
   RHGPU_NODE_E,          /* nodeE,     3 */
   RHGPU_NODE_ETA,        /* nodeEta,   1 */
   RHGPU_CELL_AVERAGE_B,  /* cellAverageB, 3 (WRITE_GRID_TEMPORAL_AVERAGES) */
   RHGPU_NUM_ARRAYS
};

/* counters (Hybrid::logCounter*, src/hybrid.h:313-327), rhgpu_get_counters order */
enum rhgpu_counter_id {
   RHGPU_CNT_FIELD_MIN_CELL_RHOQI = 0, /* logCounterFieldMinCellRhoQi  (particle_accumulator.cpp:329) */
   RHGPU_CNT_FIELD_MAX_CELL_UE,        /* logCounterFieldMaxCellUe     (hybrid_propagator.cpp:1384) */
   RHGPU_CNT_FIELD_MAX_NODE_UE,        /* logCounterFieldMaxNodeUe     (:1581) */
   RHGPU_CNT_FIELD_MAX_VW,             /* logCounterFieldMaxVw         (:1515) */
   RHGPU_CNT_FIELD_MAX_E,              /* logCounterFieldMaxE          (:1442) */
   RHGPU_CNT_FIELD_MIN_NODE_RHOQI,     /* logCounterFieldMinNodeRhoQi  (:1554) */
   RHGPU_CNT_GRID_AVERAGE_COUNTER,     /* gridTemporalAverageCounter   (:166) */
   RHGPU_NUM_FIELD_COUNTERS,
   /* then per species s, 5 values at RHGPU_NUM_FIELD_COUNTERS + 5*s + {0..4}:
    * logCounterParticleMaxVi, Escape (weight), EscapeKineticEnergy, Impact (weight),
    * ImpactKineticEnergy (boris.h:156, particle_boundary_cond_hybrid.h:120-121,148-149) */
   RHGPU_CNT_PER_SPECIES = 5
};

/* Simulation and Hybrid:: parameters the hot path reads. Derived values are
 * given already converted, as userLateInitialization leaves them
 * (src/user.cpp:356-1807): squared radii and speeds, SI resistivity table. */
typedef struct rhgpu_params {
   int32_t nx, ny, nz;            /* cells per axis, including exterior cells of non-periodic walls */
   int32_t periodic[3];           /* LogicallyCartesian x/y/z_periodic */
   double  x_min, y_min, z_min;   /* box minimum corner [m] */
   double  dx;                    /* cube cell side [m] (Hybrid::dx) */
   double  dt;                    /* time step [s] */
   double  t_initial;             /* simulation time at the first step [s] */
   int32_t use_hall;              /* Hybrid::useHallElectricField */
   int32_t use_electron_pressure; /* Hybrid::useElectronPressure */
   int32_t isothermal_electrons;  /* Hybrid::useIsothermalElectrons */
   int32_t use_gravity;           /* Hybrid::useGravity */
   int32_t use_initial_flow_through;       /* Hybrid::useInitialFlowThrough at start */
   int32_t n_linear_smoothings_nodeE;      /* Hybrid::N_linearSmoothingsNodeE */
   int32_t use_gaussian_smoothing_nodeE;   /* Hybrid::useGaussianSmoothingNodeE */
   int32_t reserved0;
   double  electron_pressure_coeff;        /* Hybrid::electronPressureCoeff */
   double  gaussian_coeffs[4];             /* Hybrid::gaussianSmoothingCoeffsNodeE */
   double  field_obstacle_Ue[3];           /* Hybrid::fieldObstacleUe */
   double  GMdt;                           /* Hybrid::GMdt */
   double  max_ion_speed2;                 /* Hybrid::maxIonSpeed2 */
   double  max_electron_speed2;            /* Hybrid::maxElectronSpeed2 */
   double  min_ion_charge_density;         /* Hybrid::minIonChargeDensity [C/m^3] */
   double  max_electric_field2;            /* Hybrid::maxElectricField2 (0: off) */
   double  max_whistler_speed;             /* Hybrid::maxWhistlerSpeed */
   double  initial_flow_through_period;    /* Hybrid::initialFlowThroughPeriod [s] */
   double  imf_B[3];                       /* Hybrid::IMFBx,IMFBy,IMFBz */
   int32_t imf_boundary_cellB[6];          /* Hybrid::IMFBoundaryCellB (+x -x +y -y +z -z) */
   int32_t imf_boundary_faceB[6];          /* Hybrid::IMFBoundaryFaceB */
} rhgpu_params;

/* One ion population (struct Species, src/particle_species.h:75-91). */
typedef struct rhgpu_species {
   double  q;            /* charge [C] */
   double  m;            /* mass [kg] */
   double  R2_obstacle;  /* squared particle obstacle radius [m^2] (negative: none) */
   int32_t accumulate;   /* deposit this population */
   int32_t accelerate;   /* push with the Lorentz force (else drift only) */
} rhgpu_species;

typedef struct rhgpu_ctx rhgpu_ctx;

/* Text of the last error raised on the calling thread ("" if none). */
const char* rhgpu_last_error(void);

/* Version string of the library build (architecture, build flags). */
const char* rhgpu_version(void);

/* Creates a context on the current CUDA device. Replaces the state that
 * userLateInitialization (src/user.cpp:356) sets up: grid arrays are
 * allocated and zeroed (src/user.cpp:1853-1868); particle storage holds up
 * to capacity[s] particles of species s. The device is cudaSetDevice'd to
 * `device` first. Every axis needs at least 3 cells (the reference also runs
 * periodic axes of 1 cell; RHGPU_ERR_ARG here) and 27 * cells below 2^31. */
int rhgpu_create(const rhgpu_params* params, int32_t n_species, const rhgpu_species* species,
                 const int64_t* capacity, int32_t device, rhgpu_ctx** out);

/* Frees all device memory of the context. */
int rhgpu_destroy(rhgpu_ctx* ctx);

/* Particle path of a context, chosen before the first particle upload:
 *  RHGPU_PATH_FAST  (default) fused push + deposit over particles binned by
 *                   row segments of RHGPU_FAST_SEGMENT CIC dual cells; the
 *                   per-particle and per-cell arithmetic is the reference's,
 *                   the CIC sums are formed in a fixed order of this library
 *                   (results deterministic, equal to the reference-order sums
 *                   to round-off); the segment length fixes that order;
 *  RHGPU_PATH_EXACT particles grouped by cell and deposited in the reference's
 *                   summation order: bitwise identical to the reference's CPU
 *                   results, at a lower speed;
 *  RHGPU_PATH_FP32  the precision form: particles stored as an int32 cell
 *                   index, FP32 offsets in the cell and FP32 velocities (one
 *                   macroparticle weight per species, checked at upload),
 *                   pushed and deposited in FP32 with FP32 accumulation; the
 *                   field update, the moments handed to it and the diagnostic
 *                   sums stay FP64. Its error against the FP64 paths is
 *                   measured, not bounded. */
#define RHGPU_PATH_FAST  0
#define RHGPU_PATH_EXACT 1
#define RHGPU_PATH_FP32  2
#define RHGPU_FAST_SEGMENT 32
int rhgpu_set_path(rhgpu_ctx* ctx, int32_t path);

/* Uploads one grid array (AoS, dim values per cell, nx*ny*nz cells). */
int rhgpu_upload_array(rhgpu_ctx* ctx, int32_t array_id, const double* host);

/* Downloads one grid array (AoS, dim values per cell). */
int rhgpu_download_array(rhgpu_ctx* ctx, int32_t array_id, double* host);

/* Uploads the per-cell flag bytes (RHGPU_FLAG_*). */
int rhgpu_upload_cell_flags(rhgpu_ctx* ctx, const uint8_t* host);

/* Replaces the particles of species s: counts[n] particles of cell n,
 * records grouped by cell in linear cell order (7 doubles each). */
int rhgpu_upload_particles(rhgpu_ctx* ctx, int32_t s, const uint32_t* counts,
                           const double* particles, int64_t n_particles);

/* Number of particles of species s currently stored. */
int rhgpu_num_particles(rhgpu_ctx* ctx, int32_t s, int64_t* n_out);

/* Downloads species s (layout as in rhgpu_upload_particles). `capacity` is the
 * size of `particles` in records; fails with RHGPU_ERR_ARG if too small. */
int rhgpu_download_particles(rhgpu_ctx* ctx, int32_t s, uint32_t* counts, double* particles,
                             int64_t capacity, int64_t* n_out);

/* FP32 form only (RHGPU_PATH_FP32; RHGPU_ERR_ARG otherwise): species s in the
 * form's own records, 6 floats per particle: the offsets in the cell in units
 * of dx, in [0, 1), then the velocity [m/s]; grouped by cell in linear cell
 * order with per-cell counts, as rhgpu_upload_particles; `weight` is the
 * species' one macroparticle weight. 24 bytes per particle cross the bus
 * instead of 56, for hosts that keep the FP32 form's particle lists
 * themselves. The reference has no counterpart: its particles are doubles. */
int rhgpu_upload_particles_f32(rhgpu_ctx* ctx, int32_t s, const uint32_t* counts,
                               const float* particles, int64_t n_particles, double weight);

/* The inverse of rhgpu_upload_particles_f32: species s as 6-float records
 * (capacity in records; RHGPU_ERR_ARG if too small) and its weight. */
int rhgpu_download_particles_f32(rhgpu_ctx* ctx, int32_t s, uint32_t* counts, float* particles,
                                 int64_t capacity, int64_t* n_out, double* weight_out);

/* Runs nsteps time steps of propagate() (src/user.cpp:118-134) on the
 * device: field gather + push, migration, deposit, particle boundary
 * conditions, propagateB. Host-resident nothing; returns after enqueueing and
 * checking the device error word once at the end. */
int rhgpu_step(rhgpu_ctx* ctx, int32_t nsteps);

/* The constituent calls, for a Corsair-style host that drives the plugins
 * one at a time (BorisBuneman::propagateCell, Accumulator::accumulate*,
 * ParticleBoundaryCondHybrid::apply, propagateB). rhgpu_step == the
 * sequence push -> accumulate -> boundary -> propagate_fields. */
int rhgpu_push(rhgpu_ctx* ctx);              /* all species: gather, push, drift, migrate */
int rhgpu_accumulate(rhgpu_ctx* ctx);        /* clear, deposit all species, finalize (/dV, clamp) */
int rhgpu_apply_boundaries(rhgpu_ctx* ctx);  /* exterior-cell and obstacle removal */
int rhgpu_propagate_fields(rhgpu_ctx* ctx);  /* propagateB */

/* rhgpu_accumulate for callers that cannot allocate device memory once the
 * run has started: a host that has handed the remaining GPU memory to its
 * own pool, or one that cannot afford the implicit device synchronisation a
 * cudaMalloc may cause. No counterpart in the reference (which has no device
 * memory); it computes exactly what rhgpu_accumulate computes on the exact
 * path, but keeps the deposit's per-cell scratch (108 doubles per cell) in a
 * fixed array in the library's static device memory instead of a buffer
 * allocated on first use, and allocates nothing at any call.
 * Limits: the context must use RHGPU_PATH_EXACT (else RHGPU_ERR_STATE) and
 * its grid must have at most RHGPU_NOALLOC_MAX_CELLS cells (else
 * RHGPU_ERR_ARG). The first call on a device looks up the scratch's device
 * address (cudaGetSymbolAddress) with that device current; make it before
 * any stream capture. The scratch is shared by every context on the device:
 * calls that overlap in time (other threads, other streams) race. */
#define RHGPU_NOALLOC_MAX_CELLS 16384
int rhgpu_accumulate_noalloc(rhgpu_ctx* ctx);

/* Synchronises and returns the accumulated device error word (RHGPU_DEVERR_*). */
int rhgpu_device_errors(rhgpu_ctx* ctx, uint32_t* word_out);

/* ---- learned denoiser of the moments (the learned form) -------------------
 * No counterpart in the reference. A 3-layer 3D convolutional network (3x3x3
 * kernels, 16 channels, leaky ReLU, residual) maps the (rho, Jx, Jy, Jz) moments of
 * a low particles-per-cell run to those of a high-ppc run. BF16 activations
 * and weights, FP32 accumulation on the tensor cores; forward, backward and
 * Adam training run on the GPU. Training pairs come from the method itself:
 * rhgpu_dn_add_pair deposits one in `factor` particles of a (high-ppc) fast
 * path context with weights times factor (the low-ppc input) next to the
 * deposit of all its particles (the target), both from its current state. rhgpu_set_denoiser applies it in
 * rhgpu_step between the deposit and the field update; the host switches it
 * off when its error against a high-ppc check run exceeds the threshold.
 * Parameters (FP32): per layer W[27][16 cin][16 cout] then b[16], tap
 * t = (dx+1) + 3(dy+1) + 9(dz+1); layer 0 reads cin < 4, layer 2 writes
 * cout < 4, the other entries are kept zero. Inputs are normalized by
 * rho_scale and j_scale (rhgpu_dn_set_scales). */
#define RHGPU_DN_PARAMS 20784
typedef struct rhgpu_dn rhgpu_dn;
int rhgpu_dn_create(int32_t nx, int32_t ny, int32_t nz, const int32_t* periodic, int32_t pair_capacity,
                    int32_t device, rhgpu_dn** out);
int rhgpu_dn_destroy(rhgpu_dn* dn);
int rhgpu_dn_set_params(rhgpu_dn* dn, const float* params, int64_t n);
int rhgpu_dn_get_params(rhgpu_dn* dn, float* params, int64_t n);
int rhgpu_dn_set_scales(rhgpu_dn* dn, double rho_scale, double j_scale);
/* velocity form (no counterpart in the reference; off by default): the network
 * sees rho / rho_scale and the bulk velocity (J / rho) / j_scale in place of
 * J / j_scale, in its training pairs and where it is applied, and hands back
 * J = rho' u' from its denoised density and velocity. j_scale is then a speed.
 * The deposit's rho and J carry the same particles' noise, which largely
 * cancels in J / rho; this form keeps that ratio as one quantity. */
int rhgpu_dn_set_velocity_form(rhgpu_dn* dn, int32_t enabled);
/* per cell (nx*ny*nz bytes, x fastest), nonzero: the cell's moments are left
 * as deposited where the network is applied (no counterpart in the
 * reference); NULL clears the mask. Training is unaffected. */
int rhgpu_dn_set_keep_mask(rhgpu_dn* dn, const uint8_t* keep);
/* host moments in the ABI layout (rho per cell, Ji interleaved) in and out;
 * rho_out is clamped at min_rho as the deposit's finalize does */
int rhgpu_dn_apply(rhgpu_dn* dn, const double* rho_in, const double* ji_in, double* rho_out, double* ji_out,
                   double min_rho);
/* mean squared error of the network on (in, target), normalized moments, and
 * its gradient (RHGPU_DN_PARAMS floats, zero where untrainable; may be NULL) */
int rhgpu_dn_loss_grad(rhgpu_dn* dn, const double* rho_in, const double* ji_in, const double* rho_target,
                       const double* ji_target, double* loss, float* grad);
int rhgpu_dn_add_pair(rhgpu_dn* dn, rhgpu_ctx* ctx, int32_t factor, int32_t offset);
/* Training pairs from crops of a larger grid, for a denoiser created with the
 * crop's dimensions (non-periodic): the context's moments are deposited as by
 * rhgpu_dn_add_pair (one in `factor` particles, weights times factor; and all
 * particles) on its whole grid, and each crop, corner origins[3q..3q+2] (cell
 * indices, inside the context's grid), is stored as one pair. The network is
 * convolutional: parameters trained on crops apply to the whole grid
 * (rhgpu_dn_get_params / rhgpu_dn_set_params). */
int rhgpu_dn_add_crops(rhgpu_dn* dn, rhgpu_ctx* ctx, int32_t factor, int32_t offset, int32_t ncrops,
                       const int32_t* origins);
/* leaves the voxels within `border` of a non-periodic face out of the training
 * loss (crops: their outer voxels see zeros instead of their neighbours;
 * three layers of 3x3x3 reach 3 voxels). Default 0. */
int rhgpu_dn_set_loss_border(rhgpu_dn* dn, int32_t border);
/* Adam steps, one random stored pair per step; mean loss over the steps */
int rhgpu_dn_train(rhgpu_dn* dn, int32_t iterations, float lr, double* mean_loss);
int rhgpu_set_denoiser(rhgpu_ctx* ctx, rhgpu_dn* dn, int32_t enabled);
/* relative L2 errors of stored pair `pair` against its target:
 * out4 = {raw rho, raw J, denoised rho, denoised J} */
int rhgpu_dn_pair_error(rhgpu_dn* dn, int32_t pair, double* out4);
/* pairs stored and the index of the newest */
int rhgpu_dn_num_pairs(rhgpu_dn* dn, int32_t* n_out, int32_t* newest);

/* Particle sources, the reference's injectors (src/particle_injector.cpp), on
 * the GPU: after the boundary conditions of every step (src/user.cpp:119-122)
 * each injection cell draws probRound(N) new macroparticles from a
 * counter-based stream (Philox-4x32-10 keyed by `seed`, the step and the
 * cell), so a run is reproducible and independent of thread order; they are
 * stored like particles arriving from another segment and deposit from the
 * next step on, as in the reference. Fast and FP32 paths only.
 *   RHGPU_INJECT_SOLARWIND (InjectorSolarWind, :517-730): `velocity` has one
 *     non-zero component U; the cells of the upstream outer wall that have
 *     both neighbours along the other axes get N = ppc |U| dt / dx per step
 *     at the wall face, the normal velocity from the flux of a drifting
 *     Maxwellian (sampleDerivGaussian) and Gaussian tangential velocities.
 *   RHGPU_INJECT_FLOW (InjectorFlow, :734-945): every cell of the walls in
 *     `inflow_walls` (bit 0 +x, 1 -x, 2 +y, 3 -y, 4 +z, 5 -z) gets N = ppc
 *     per step, uniform in the cell, velocity + Gaussian thermal velocity.
 *   RHGPU_INJECT_EXOSPHERE (InjectorExosphere, :1491-1840): a neutral
 *     density profile (`profile`, below; n0/H0/T0/k0 per component, r0) is
 *     averaged over each cell by Monte Carlo (1000 points, zero below the
 *     exobase) at set-up; with the ionization rate (or the total production
 *     rate) and the shadow factor (x < 0, y^2 + z^2 < shadow_radius^2) it
 *     gives each cell's expected macroparticles per step, the whole box
 *     N = macroparticles_per_cell_relative * upstream_macro_ratio per step,
 *     weight total_rate dt / N. New particles are uniform in the cell and
 *     above the exobase, with Gaussian velocities of the temperature.
 *   RHGPU_INJECT_IONOSPHERE (InjectorIonosphere, :947-1240): each cell's
 *     share of a spherical emission shell of `emission_radius` (1000 Monte
 *     Carlo points per cell projected on the shell) times the emission
 *     profile at the cell centre gives its expected macroparticles per step,
 *     N = macroparticles_per_cell_relative * upstream_macro_ratio per step in
 *     the box, weight total_production_rate dt / N. New particles are uniform
 *     in the cell with Gaussian velocities of the temperature, turned outward.
 *   RHGPU_INJECT_CHAPMAN_IONOSPHERE (InjectorChapmanIonosphere, :1242-1482):
 *     as the ionosphere, but each point is kept with the Chapman probability
 *     a exp(1 - h - exp(-h)), h = (r - R)/H - log(1/a), a the cos(SZA)-day /
 *     constant-night factor (noon_factor, night_factor), H the scale height
 *     k_B T / (m g_Mars) (150 K for the cells' shares, `temperature` for the
 *     new particles); cells with fewer than 10 of 1000 Monte Carlo points
 *     kept emit nothing.
 * Solar wind and flow: weight n dx^3 / ppc. Thermal speed sqrt(k_B T / m)
 * with the species' mass. n == 0 removes all sources. The call replaces the
 * whole source set; if any source is rejected, the previous set stays in force. */
#define RHGPU_INJECT_SOLARWIND 1
#define RHGPU_INJECT_FLOW      2
#define RHGPU_INJECT_EXOSPHERE 3
#define RHGPU_INJECT_IONOSPHERE 4
#define RHGPU_INJECT_CHAPMAN_IONOSPHERE 5
/* ionospheric emission profiles (InjectorIonosphere, particle_injector.cpp:1160-1210) */
#define RHGPU_IONO_COS_SZA_DAY_CONSTANT_NIGHT 1   /* ionoCosSzaDayConstantNight */
#define RHGPU_IONO_CONSTANT_DAY_CONSTANT_NIGHT 2  /* ionoConstantDayConstantNight */
#define RHGPU_IONO_CONSTANT 3                     /* ionoConstant */
#define RHGPU_IONO_POLAR_CAP 4                    /* ionoPolarCap */
/* neutral profiles (src/neutral_profiles.h) */
#define RHGPU_NEUTRAL_CHAMBERLAIN_H 1   /* sum n0 exp(-H0 (1/r0 - 1/r)) */
#define RHGPU_NEUTRAL_CHAMBERLAIN_T 2   /* sum n0 exp(-(G M m / k_B T0) (1/r0 - 1/r)) */
#define RHGPU_NEUTRAL_EXPONENTIAL   3   /* sum n0 exp(-(r - r0) / H0) */
#define RHGPU_NEUTRAL_POWER_LAW     4   /* sum n0 (r0 / r)^k0 */
/* planetary models (no parameters; the Sun on +x): */
#define RHGPU_NEUTRAL_VENUS_HYDROGEN 5  /* VenusHydrogen: thermal day/night + hot corona */
#define RHGPU_NEUTRAL_VENUS_OXYGEN   6  /* VenusOxygen: day/night Chamberlain-like */
#define RHGPU_NEUTRAL_MERCURY_SODIUM_EXNER20 7  /* MercurySodiumExner20: Exner et al. (2020) Na */
#define RHGPU_NEUTRAL_MAX_COMPONENTS 4
typedef struct rhgpu_injector {
   int32_t  species;                  /* population index */
   int32_t  type;                     /* RHGPU_INJECT_* */
   double   velocity[3];              /* bulk velocity [m/s] */
   double   density;                  /* number density [m^-3] */
   double   temperature;              /* [K] */
   double   macroparticles_per_cell;
   int32_t  inflow_walls;             /* flow: walls (bit mask above) */
   int32_t  reserved;
   uint64_t seed;
   /* exosphere */
   int32_t  profile;                  /* RHGPU_NEUTRAL_* */
   int32_t  n_components;             /* 1 .. RHGPU_NEUTRAL_MAX_COMPONENTS */
   double   r0;                       /* profile reference radius [m] */
   double   n0[4], H0[4], T0[4], k0[4];
   double   gm_object;                /* G M_object [m^3 s^-2] (Chamberlain T) */
   double   exobase_radius, shadow_radius;
   double   ionization_rate;          /* [1/s], or < 0: use total_production_rate */
   double   ionization_factor_shadow;
   double   total_production_rate;    /* [1/s], or < 0: use ionization_rate */
   double   macroparticles_per_cell_relative;
   double   upstream_macro_ratio;     /* Hybrid::upstreamMacroPleRatio (> 0) */
   /* ionosphere (also uses temperature, total_production_rate,
    * macroparticles_per_cell_relative, upstream_macro_ratio) */
   double   emission_radius;          /* radius of the emission shell [m] */
   double   noon_factor, night_factor;   /* `noon`, `night` (ionoPolarCap: tilt and cap half angle [deg]) */
   int32_t  iono_profile;             /* RHGPU_IONO_* */
   int32_t  reserved2;
} rhgpu_injector;
int rhgpu_set_injectors(rhgpu_ctx* ctx, int32_t n, const rhgpu_injector* injectors);
/* Replaces species s's particles by a uniform fill generated on the GPU, for
 * the fast path and the FP32 form (no host records: runs of 1e9 ions and more).
 * The reference's InjectorUniform::injectParticles (particle_injector.cpp:
 * 188-255): every cell whose centre lies in `region` (x_lo, x_hi, y_lo, y_hi,
 * z_lo, z_hi in metres; NULL: the whole box) draws probRound(ppc) macroparticles
 * (ppc = injector->macroparticles_per_cell), uniform in the central (1 - 1e-4)
 * of the cell, velocity injector->velocity + sqrt(k_B T / m) N(0,1) per
 * component, weight density dx^3 / ppc. Uses density, temperature, velocity,
 * macroparticles_per_cell and seed of the injector; particle k of cell c draws
 * from a Philox stream keyed by (seed, c, k), so the fill is reproducible. */
int rhgpu_fill_uniform(rhgpu_ctx* ctx, int32_t s, const rhgpu_injector* injector, const double* region);

/* expected macroparticles per step in every cell (N doubles, linear cell
 * order) of source `injector` (index into the last rhgpu_set_injectors
 * array). Filled for the rate-based sources: exosphere (cellExosphere,
 * particle_injector.cpp:1780-1792) and ionospheres (cellIonosphere,
 * :1205-1226). Zeros for the other types. These are the arrays the
 * reference's output step writes as prod_rate_exo<k> / prod_rate_iono<k>
 * (operator_userdata.cpp:123-154). Host memory only; no device work. */
int rhgpu_source_rates(rhgpu_ctx* ctx, int32_t injector, double* out);
/* injected per species: weight, macroparticles, weight * v^2
 * (logCounterParticleInject*, particle_injector.cpp:569-571); 3 * n_species doubles */
int rhgpu_get_injection_counters(rhgpu_ctx* ctx, double* out, int32_t n);

/* The neutral density [m^-3] of an exosphere source's profile (its profile,
 * n_components, r0, n0, H0, T0, k0, gm_object; `mass` is the ion mass the
 * Chamberlain T profile uses) at n points xyz (x, y, z interleaved, metres
 * from the planet's centre), evaluated on `device` as the source's set-up
 * does (getNeutralDensity, src/neutral_profiles.h:215-241). */
int rhgpu_neutral_density(const rhgpu_injector* profile, double mass, int64_t n, const double* xyz, double* out,
                          int32_t device);
/* Philox-4x32-10 of the particle sources, host side (for checks): out = philox(ctr, key) */
void rhgpu_philox4x32(const uint32_t* ctr, const uint32_t* key, uint32_t* out);

/* Counters: RHGPU_NUM_FIELD_COUNTERS + RHGPU_CNT_PER_SPECIES*n_species doubles. */
int rhgpu_get_counters(rhgpu_ctx* ctx, double* out, int32_t n);

/* Current simulation time and time-step number (Simulation::t, ::timestep). */
int rhgpu_get_time(rhgpu_ctx* ctx, double* t_out, int64_t* timestep_out);

/* Device-side FP64 reductions of the population and field logs
 * (logCalcParticle / logCalcField, diagnostics.h:187-404), n >= 8*n_species + 30:
 * out[8*s + 0..7] per species s: N macroparticles, sum w, sum w*vx, sum w*vy,
 *   sum w*vz, sum w*|v|, sum w*v^2, max |v|;
 * then 30 field values over the cells with all neighbours outside the inner
 * field boundary (the reference's default, includeInnerCellsInFieldLog = false;
 * rhgpu_log_open can include them):
 *   N cells, sum Bx, By, Bz, |B|, max |B|, sum |divB|, max |divB|, max |divB|/|B|,
 *   sum B^2 (cell B = mean of its two faces); sum Jix, Jiy, Jiz, |Ji|, max |Ji|;
 *   sum Epx, Epy, Epz, |Ep|, max |Ep|, sum Ep^2; sum nodeEx, Ey, Ez, |E|, max |E|,
 *   sum E^2; sum |Ue x B|^2; max |Ue|; sum cellRhoQi.
 * With n >= 8*n_species + 36, six more: the spatial, temporal and velocity
 * scales of the field log over the same cells (diagnostics.h:375-395): min and
 * max electron inertial length (from cellRhoQi > 0), min and max proton
 * inertial length and max Alfven speed (from the total ion mass density: every
 * species' w*m in the particle's cell, /dV, floored at
 * min_ion_charge_density*m_p/e), min ion Larmor period (from |B| > 0); where no
 * cell qualifies, the reference's starting values (DBL_MAX for minima,
 * -DBL_MAX for inertial-length maxima, 0 for the Alfven speed).
 * Sums are formed per block in a fixed tree and added on the host in block
 * order: deterministic, equal to the reference's sequential sums to round-off.
 * The mass density is the reference's sequential sum on the exact path and an
 * exact fixed-point sum on the fast and FP32 paths. */
int rhgpu_reduce_diagnostics(rhgpu_ctx* ctx, double* out, int32_t n);

/* Population and field log files (Hybrid.log_interval logging of
 * logWriteParticleField, src/diagnostics.h:405-818, with the files and headers
 * of src/user.cpp:2147-2231): pop001_<name>.log per species and field.log in
 * `directory`, numbers in scientific notation with a sign and `precision`
 * digits (Hybrid.log_precision, 10 by default). */
typedef struct rhgpu_log_config {
   const char* directory;
   const char* const* species_names;  /* n_species names (ParticleSpecies name) */
   int32_t precision;
   int32_t include_inner_cells;       /* Hybrid.includeInnerCellsInFieldLog */
   double max_B_stop_run;             /* Constraints.max_magnetic_field_stop_run [T] */
} rhgpu_log_config;

/* Opens (truncates) the log files, writes their headers, zeroes the log
 * counters and starts the rate interval at the current simulation time. */
int rhgpu_log_open(rhgpu_ctx* ctx, const rhgpu_log_config* cfg);

/* One log step (the caller's Hybrid.log_interval): appends one line to every
 * log file with the current state and the counter rates since the previous log
 * step, then zeroes the log counters (rhgpu_get_counters and
 * rhgpu_get_injection_counters read zero afterwards) as the reference does.
 * *stop_run is set to 1 when max |faceB| exceeds max_B_stop_run (the reference
 * stops the run), else 0. The reference's main-log text (warnings, the stop
 * message and, with main_log_diagnostics != 0, the diagnostics block) is
 * copied to `messages` (up to messages_cap bytes, NUL-terminated; may be NULL). */
int rhgpu_log_write(rhgpu_ctx* ctx, int32_t main_log_diagnostics, int32_t* stop_run, char* messages,
                    int32_t messages_cap);

/* Flushes and closes the log files (also done by rhgpu_destroy). */
int rhgpu_log_close(rhgpu_ctx* ctx);

/* Per-cell grid constraint counters (USE_GRID_CONSTRAINT_COUNTERS, off in the
 * reference's default build; hybrid_propagator.cpp:64-116, 1382, 1440, 1513,
 * 1579, boris.h:153-155, particle_accumulator.cpp:327): how many times each
 * cell or node hit a limit since the counters were switched on or last
 * zeroed. rhgpu_set_grid_counters(ctx, 1) allocates 40 bytes per cell and
 * zeroes them (a later call zeroes them again, as the reference does after a
 * save step); 0 frees them. rhgpu_download_grid_counters writes 5 planes of
 * N doubles: cellMaxUe (cell and node Ue limits, as the reference counts the
 * node one in the cell array), cellMaxVi (ion speed limit, the particle's
 * cell before it moves), cellMinRhoQi, nodeMaxE, nodeMaxVw. Every path. */
#define RHGPU_GRID_COUNTER_PLANES 5
int rhgpu_set_grid_counters(rhgpu_ctx* ctx, int32_t enable);
int rhgpu_download_grid_counters(rhgpu_ctx* ctx, double* out);

/* Temporal averages of the output populations (WRITE_GRID_TEMPORAL_AVERAGES,
 * on in the reference's default build). group_of_species[s] is the output
 * population of species s (Hybrid::outputPopVarId: species with the same
 * output string share one; -1: none), n_groups the number of output
 * populations. From the next step on, every accumulating species adds its CIC
 * charge and current sums to its population's sums
 * (particle_accumulator.cpp:148-150). Fast and exact paths; n_groups = 0
 * switches them off. Allocates 16 * (n_groups + 1) bytes per cell. */
int rhgpu_set_population_averages(rhgpu_ctx* ctx, int32_t n_groups, const int32_t* group_of_species);

/* The output step's averages (operator_userdata.cpp:155-223), each argument
 * NULL to skip it: cellB_average (3 per cell, interleaved) = cellAverageB /
 * count; per output population g, n_average[g*N + n] = charge sum /
 * (q dV) / count with q the charge of the population's first species, and
 * v_average[(g*N + n)*3 + l] = current sum / charge sum where the charge sum
 * is positive, else 0. The sums of what is returned restart from zero, and
 * the average counter always does (as the reference's writer). */
int rhgpu_output_averages(rhgpu_ctx* ctx, double* cellB_average, double* n_average, double* v_average);

/* The CUDA stream (cudaStream_t) the context enqueues on. */
void* rhgpu_stream(rhgpu_ctx* ctx);

/* Per-kernel CUDA-event timing of the last rhgpu_step call: fills names
 * (comma separated, up to name_cap bytes) and ms (total milliseconds per
 * kernel class, up to n entries); returns the number of classes in *n_out.
 * Timing is recorded only when enabled with rhgpu_set_timing(ctx, 1). */
int rhgpu_set_timing(rhgpu_ctx* ctx, int32_t enable);
int rhgpu_get_timing(rhgpu_ctx* ctx, char* names, int32_t name_cap, double* ms, int32_t n,
                     int32_t* n_out);

/* Number of kernel launches issued by the last rhgpu_step call. */
int rhgpu_last_launch_count(rhgpu_ctx* ctx, int64_t* out);

#ifdef __cplusplus
}
#endif

#endif
