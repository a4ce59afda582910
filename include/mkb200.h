/*
 * mkb200.h — C ABI of the B200 coupled lattice-Boltzmann / phase-field step.
 *
 * This is the drop-in boundary for MaterKit's solver path.  The reference
 * exposes a C++ class API from a Windows DLL (MaterKit/inc/MaterKit.h:28-35,
 * MK_API = __declspec(dllexport)); its lifecycle is
 *
 *   mkSpace(xml)                      MaterKit/inc/mkSpace.h:36
 *   solver(space), solver.reset(xml)  MaterKit/inc/mkFluidsLBM.h:35-38
 *   readParameters(loops,frames,xml)  MaterKit/inc/mkFunction.h:62
 *   solver.initialize(xml)            MaterKit/inc/mkFluidsMRT.h:39
 *   solver.initialize_geometry()      MaterKit/inc/mkFluidsMRT.h:40
 *   per loop: propagate()/relaxation*()/bdy*()   (MaterKit/MaterKit.cpp:204-237)
 *   write_vtkfile(loops), check_variables(...)   (MaterKit/inc/mkFluidsMRT.h:48,
 *                                                  MaterKit/inc/mkFluidsLBM.h:55)
 *
 * Every entry point here returns mk_status; no C++ exception crosses the ABI
 * (the reference throws mkIOError from MaterKit/xml/mkTINYXMLIO.hh:40).  All
 * arguments are plain pointers and sizes.  A handle owns its device memory and
 * one CUDA stream; it is thread-compatible (one host thread at a time).
 *
 * Field arrays exchanged through this header are dense, x fastest:
 *   index = x + nx * (y + ny * z).
 */
#ifndef MKB200_H
#define MKB200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define MKB200_ABI_VERSION 3

/* Status codes.  Replace the exception family of
 * MaterKit/inc/mkRunTimeDiagnostics.h:59-117 (mkIOError, mkMemoryError, ...). */
typedef enum mk_status {
  MK_OK = 0,
  MK_ERR_XML = 1,      /* unreadable XML or a tag with a malformed value */
  MK_ERR_ARG = 2,      /* invalid argument / unsupported combination      */
  MK_ERR_CUDA = 3,     /* CUDA runtime error (message in mk_last_error)   */
  MK_ERR_DIVERGED = 4, /* NaN/Inf or non-positive density detected        */
  MK_ERR_TIMEOUT = 5,  /* a bounded device wait gave up                   */
  MK_ERR_OOM = 6,      /* device or host allocation failed                */
  MK_ERR_IO = 7,       /* file could not be written / read                */
  MK_ERR_STATE = 8,    /* call not valid in the handle's current state    */
  MK_ERR_NODEVICE = 9  /* no CUDA device (the library has no CPU fallback) */
} mk_status;

/* Which solver path a case runs.  In the reference the driver picks this by
 * calling one run_* function (MaterKit/MaterKit.cpp:23-34). */
typedef enum mk_model {
  MK_MODEL_FLOW = 0,             /* single-phase flow, run_flow_Poiseuille (MaterKit.cpp:244-288) */
  MK_MODEL_MULTIPHASE = 1,       /* Allen-Cahn two-phase flow, run_flow_multiphase (:290-331)     */
  MK_MODEL_THERMAL_DENDRITE = 2, /* phase field + thermal ADE, run_thermal_dendrite (:743-788)    */
  MK_MODEL_SOLUTAL_DENDRITE = 3, /* phase field + solutal ADE, run_solutal_dendrite (:633-687)    */
  MK_MODEL_CONVECTION = 4,       /* flow + advected D3Q7 scalar with Boussinesq buoyancy and
                                    Dirichlet plates: Rayleigh-Benard (bdy_RBC, Thermal_NusseltRBC,
                                    mkThermalField.h:33-40, mkFluidsLBM.h:59-68)                  */
  MK_MODEL_FLOW_DENDRITE = 5,    /* thermal dendrite growing in a flow: porous bounce-back of the
                                    flow by the solid fraction, thermal lattice advected, inflow /
                                    outflow faces, run_flow_thermal_dendrite (MaterKit.cpp:467-527) */
  MK_MODEL_MULTIGRAIN = 6,       /* one conservative Allen-Cahn order parameter per seed (grain) on
                                    a D3Q19 lattice (the reference's D2Q9 on a one-cell periodic z) with
                                    a pairwise overlap penalty, aggregate phi = (N - 1) + sum phi_j,
                                    thermal ADE with latent heat: run_multiPhaseField
                                    (MaterKit.cpp:529-571), mkFluidsUser::propagate/relaxation
                                    (mkFluidsUser.cpp:68-299), mkMultiphaseField.h:24-60             */
  MK_MODEL_FLOW_SOLUTAL = 7      /* solutal dendrite growing in a flow: the flow lattice of
                                    MK_MODEL_FLOW_DENDRITE (porous bounce-back, inflow / outflow
                                    faces), the solutal phase field, the U-lattice advected by the
                                    flow with the solute inflow face: run_flow_solutal_dendrite
                                    (MaterKit.cpp:399-465; bdy_LBflowin, mkSolutalField.h:53)       */
} mk_model;

/* Population storage precision.  Collision arithmetic is FP64 for MK_PREC_FP64
 * and FP32 otherwise (FP32 divisions by densities, gradient norms and
 * capacities use the fast approximate division, about two ulp).  FP16/BF16
 * store the deviation from the rest state ("shifted storage"). */
typedef enum mk_precision {
  MK_PREC_FP64 = 0,
  MK_PREC_FP32 = 1,
  MK_PREC_FP16 = 2,
  MK_PREC_BF16 = 3
} mk_precision;

/* Collision operators of mkNode (MaterKit/inc/mkNode.h:74-87). */
typedef enum mk_collision {
  MK_COLL_BGK = 0,
  MK_COLL_TRT = 1,
  MK_COLL_MRT = 2
} mk_collision;

/* Velocity sets.  The reference's lattice class is MaterKit/inc/mkLattice.h:26-100. */
typedef enum mk_lattice {
  MK_D3Q7 = 7,
  MK_D3Q19 = 19,
  MK_D3Q27 = 27
} mk_lattice;

/* Boundary kind per axis. */
typedef enum mk_bc {
  MK_BC_PERIODIC = 0, /* periodic wrap, as mkFluidsLBM::neighbor (mkFluidsLBM.h:82)      */
  MK_BC_WALLS = 1,    /* cells 0 and n-1 are solid walls; half-way bounce-back          */
  MK_BC_CLOSED = 2    /* all cells fluid; the domain faces bounce back (zero flux)      */
} mk_bc;

/* Interfacial anisotropy a(n) of the phase field, n the crystal-frame normal
 * (mkPhaseField::anisotropy / _cbc / _hcp / _facet, mkPhaseField.h:61-64). */
typedef enum mk_anisotropy {
  MK_ANISO_CUBIC = 0, /* 1 - 3 e4 + 4 e4 sum n^4                                        */
  MK_ANISO_CBC = 1,   /* 1 + e4 (sum n^4 - 3/5) + e2 (3 sum n^4 + 66 nx^2 ny^2 nz^2 - 17/7) */
  MK_ANISO_HCP = 2,   /* 1 + e4 Re (nx + i ny)^6 + e2 (2 nz^2 - 1)                     */
  MK_ANISO_FACET = 3  /* 1 + e4 (sum sqrt(n^2 + e2^2) - sqrt(1 + e2^2) - 2 e2)          */
} mk_anisotropy;

/* Node flags, values of MaterKit/inc/mkGlobalDefs.h:140-145. */
#define MK_FLAG_FLUID 0
#define MK_FLAG_INTER 1
#define MK_FLAG_SOLID 2
#define MK_FLAG_WALLS 3

typedef enum mk_field {
  MK_FIELD_RHO = 0,      /* density                                          */
  MK_FIELD_UX = 1,       /* velocity x                                       */
  MK_FIELD_UY = 2,
  MK_FIELD_UZ = 3,
  MK_FIELD_T = 4,        /* dimensionless temperature u = (T - Tm)/(L/cp)    */
  MK_FIELD_C = 5,        /* solute: supersaturation U of the dilute alloy    */
  MK_FIELD_PHI = 6,      /* order parameter                                  */
  MK_FIELD_FLAG = 7,     /* node flag (as double)                            */
  MK_FIELD_PRESSURE = 8, /* normalised pressure p* (multiphase); the         *
                          * hydrodynamic pressure is rho p* / 3             */
  MK_FIELD_DPHI = 9,     /* phi(n) - phi(n-1), the latent-heat driver        */
  MK_FIELD_GRAIN = 10    /* grain id (seed index)                            */
} mk_field;

typedef enum mk_dtype {
  MK_DTYPE_F64 = 0,
  MK_DTYPE_F32 = 1
} mk_dtype;

#define MK_MAX_OBJECTS 64

/* Every resolved number of a case, in lattice units.  Filled from the
 * BoltzTechs XML tags the reference's cases use plus the optional <b200> block. */
typedef struct mk_params {
  int32_t model;      /* mk_model */
  int32_t lattice;    /* flow lattice (D3Q19/D3Q27); scalar lattices are D3Q7 */
  int32_t collision;  /* mk_collision of the flow lattice */
  int32_t precision;  /* mk_precision */
  int32_t nx, ny, nz; /* MeshXYZ */
  int32_t bc[3];      /* mk_bc per axis */
  int32_t max_loops;  /* output/numLoops */
  int32_t max_frames; /* output/numFrames */

  /* single-phase flow */
  double rho0;        /* initial density */
  double u0[3];       /* initial velocity */
  double tau;         /* BGK tau, TRT tau+, MRT shear tau */
  double magic;       /* TRT Lambda = (tau+ - 1/2)(tau- - 1/2) */
  double force[3];    /* body force density (flow) or gravity acceleration (multiphase) */

  /* two-phase Allen-Cahn flow */
  double rho_l, rho_g;   /* densities of phi = 1 and phi = 0 */
  double tau_l, tau_g;   /* flow relaxation times of the two fluids */
  double sigma;          /* surface tension */
  double width;          /* interface width W */
  double mobility;       /* Allen-Cahn mobility M */
  double contact_angle;  /* degrees, at solid walls */

  /* phase field (dendrites) */
  double eps4;        /* 4-fold anisotropy strength */
  double W0;          /* interface width */
  double tau0;        /* relaxation time of the phase field */
  double lambda;      /* coupling constant */
  double delta;       /* dimensionless undercooling (u0 = -delta) / supersaturation */
  double D;           /* thermal or solutal diffusivity (liquid) */
  double D_s;         /* solutal diffusivity in the solid */
  double k_part;      /* partition coefficient */
  double at_coef;     /* anti-trapping coefficient (1/(2 sqrt 2) for the standard current) */

  /* seeds (dendrites) or bubbles (multiphase) */
  int32_t n_objects;
  int32_t aniso;      /* mk_anisotropy of the phase field (dendrites) */
  double obj_center[MK_MAX_OBJECTS][3];
  double obj_angle[MK_MAX_OBJECTS][3];  /* degrees, rotate order ZYX */
  double obj_radius[MK_MAX_OBJECTS];
  uint64_t rng_seed;

  double eps2;        /* second anisotropy coefficient: cbc eps2, hcp eps_z, facet cusp width */

  /* plates and inlets (convection, flow) */
  int32_t wall_axis;    /* axis whose two faces are plates with a Dirichlet scalar / wall velocity; -1 none */
  int32_t inlet;        /* 1: velocity inlet at x = 0, pressure outlet at x = nx - 1 (flow) */
  double wall_value[2]; /* scalar (T or C) on the low / high plate */
  double wall_u[2][3];  /* velocity of the low / high plate (flow) */
  double beta;          /* Boussinesq expansion coefficient: F = -rho0 beta (s - s_ref) g, g = force */
  double s_ref;         /* reference value of the scalar in the buoyancy */

  /* multigrain: strength of the pairwise overlap penalty of grains 1..N-1
   * (grain 0 has none, mkFluidsUser.cpp:233-251); the mobility is `mobility`,
   * the interface width `W0` */
  double grain_kappa;
  /* multigrain: velocity in the equilibrium of grain 1 (the reference
   * relaxes grain 1 towards a moving equilibrium with u = (0.02, 0, 0),
   * mkFluidsUser.cpp:220-226, the default; every other grain is at rest) */
  double grain_u[3];
} mk_params;

/* Optional overrides at creation; a negative value keeps the XML/default. */
typedef struct mk_options {
  int32_t model;
  int32_t precision;
  int32_t collision;
  int32_t lattice;
  double magic;
  int32_t device;
  int32_t block_x;    /* launch shape override (0 = tuned default) */
  int32_t block_y;
} mk_options;

/* FP64 global sums (K6).  Replaces check_variables (mkFluidsLBM.h:55). */
typedef struct mk_diag {
  int64_t step;
  double mass;         /* sum of density over fluid cells          */
  double momentum[3];  /* sum of rho*u                             */
  double phi_sum;      /* sum of phi                               */
  double solid_frac;   /* fraction of fluid cells with phi > 0 (dendrite) or phi < 1/2 (multiphase gas) */
  double heat;         /* sum of T (+ latent part)                 */
  double solute;       /* sum of solute                            */
  double max_speed;    /* max |u|                                  */
  int32_t n_bad;       /* NaN/Inf/non-positive density cells       */
  int32_t _pad;
} mk_diag;

/* Interface tip of one seed: the distance from the seed's centre to the
 * outermost phi = iso crossing along +x, -x, +y, -y, +z, -z (phi sampled
 * bilinearly across the line through the centre, linearly along it; 0 when
 * the centre is outside, phi < iso), and its rate of change per loop since
 * the previous mk_tip_track call on the handle for the same seed and iso
 * (0 on the first call). */
typedef struct mk_tip {
  int64_t step;
  double length[6];
  double velocity[6];
} mk_tip;

typedef struct mk_handle mk_handle;

/* Library / ABI. */
int32_t mk_abi_version(void);
/* Select the CUDA device of handles created afterwards by this host thread. */
mk_status mk_set_device(int32_t device);
const char* mk_version_string(void);
/* Last error of a failed call that had no handle (e.g. mk_create_from_xml). */
const char* mk_last_global_error(void);

/* readParameters(maxLoops, maxFrame, xml) — MaterKit/inc/mkFunction.h:62.
 * Reads output/numLoops and output/numFrames. */
mk_status mk_read_parameters(const char* xml_path, int32_t* max_loops, int32_t* max_frames);

/* Resolve a case to its parameters without touching a GPU
 * (= mkSpace(xml) + reset + read_parameters, MaterKit/inc/mkFluidsLBM.h:37,42).
 * A <seed> whose <center> holds fewer than 3 * <number> values places the
 * seeds with a complete centre triple (n_objects = the count of full triples);
 * a short <radius> list repeats its last value, a short <angle> list gives 0. */
mk_status mk_case_params(const char* xml_path, const mk_options* opt, mk_params* out);

/* Host-side initial state of a case (= initialize + initialize_geometry,
 * MaterKit/inc/mkFluidsMRT.h:39-40).  Writes ncells doubles. */
mk_status mk_case_initial_field(const mk_params* p, int32_t field, double* out, size_t ncells);

/* Create a solver on the GPU from a BoltzTechs XML case.
 * = mkSpace(xml) + solver(space) + reset(xml) + initialize(xml) + initialize_geometry(). */
mk_status mk_create_from_xml(const char* xml_path, const mk_options* opt, mk_handle** out);
/* Same, from already-resolved parameters. */
mk_status mk_create(const mk_params* p, mk_handle** out);
mk_status mk_destroy(mk_handle* h);
const char* mk_last_error(const mk_handle* h);

mk_status mk_get_params(const mk_handle* h, mk_params* out);
int64_t mk_get_step(const mk_handle* h);

/* Advance n loops of the coupled step (propagate + relaxation of every field in
 * the reference's per-loop order).  Asynchronous on the handle's stream.  A
 * multiphase loop runs as a phi kernel plus a collision kernel, or as one
 * cooperative launch whose tiles exchange phi planes through flags with
 * bounded waits (mk_set_fused); the two forms give the same result. */
mk_status mk_advance(mk_handle* h, int64_t nsteps);
/* Capture the per-loop launches in a CUDA graph and replay it n times. */
mk_status mk_advance_graph(mk_handle* h, int64_t nsteps);
/* Wait for the handle's stream.  MK_ERR_TIMEOUT when a bounded device wait of
 * the fused multiphase loop ran out since the last check (the loops since
 * then are invalid; the handle stays usable). */
mk_status mk_sync(mk_handle* h);
/* Loop form of a multiphase case: 0 the phi kernel plus the collision kernel
 * (the default), 1 the fused one-launch loop (cases with an x extent that is a
 * multiple of 4 and at least 8 planes in z).  Both give bit-identical
 * results; the autotuner keeps the faster (the two-kernel loop on B200 for
 * the 256^3 bubble case).  MK_ERR_ARG when 1 is asked of a case that does not
 * admit the fused loop.  mk_get_fused reports the current form. */
mk_status mk_set_fused(mk_handle* h, int32_t fused);
int32_t mk_get_fused(const mk_handle* h);
/* Collision form of the two-kernel multiphase loop: 0 one thread per cell
 * loading its populations from global memory, 1 row-staged (whole x rows of
 * all 38 populations staged through shared memory by the bulk-copy engine,
 * several rows in flight per CTA; cases whose x rows hold at most 256 cells
 * and a multiple of 16 bytes).  Both give bit-identical results; the
 * autotuner keeps the faster.  MK_ERR_ARG when 1 is asked of a case that does
 * not admit it.  Also available on slab handles. */
mk_status mk_set_row_staging(mk_handle* h, int32_t on);
int32_t mk_get_row_staging(const mk_handle* h);

/* The launch configuration of a handle's loop: what mk_autotune chooses, or a
 * caller pins (a saved tuning reused for many runs of one case).  No
 * counterpart in the reference.  Every configuration gives the same result
 * (bit for bit with FP32, FP16 and BF16 storage). */
typedef struct mk_tuning {
  int32_t block_x, block_y;  /* block shape of the per-cell kernels (x a multiple of 32, at most 1024 threads) */
  int32_t minb;              /* occupancy variant of the dominant kernel: 1 or 2 resident 256-thread blocks;
                                multiphase also 3, 4, 5: registers capped at 112, 96, 80 */
  int32_t fused;             /* multiphase: the fused one-launch loop (mk_set_fused) */
  int32_t row_staged;        /* multiphase: the row-staged collision (mk_set_row_staging) */
  int32_t phi_tile;          /* multiphase: the collision stages each block's phi tile and its one-cell
                                halo into shared memory with one TMA tensor load (64 x 4 blocks; needs
                                nx a multiple of 4); at most one of fused, row_staged, phi_tile */
} mk_tuning;
mk_status mk_get_tuning(const mk_handle* h, mk_tuning* out);
/* MK_ERR_ARG for a shape or a form the case does not admit (nothing changed). */
mk_status mk_set_tuning(mk_handle* h, const mk_tuning* t);
/* Test hook of the failure detection, no counterpart in the reference.
 * kind 1: in the next loop of a fused multiphase case one tile publishes none
 * of its phi planes, so its neighbours' bounded waits run out (about a second)
 * and the next mk_sync / mk_diagnostics returns MK_ERR_TIMEOUT.  Nothing
 * faults or hangs.  MK_ERR_ARG for other kinds or cases without the fused loop. */
mk_status mk_inject_fault(mk_handle* h, int32_t kind);
/* The handle's cudaStream_t, for event timing by the caller. */
mk_status mk_get_stream(mk_handle* h, void** stream);

/* Copy a macroscopic field to host memory (synchronous). */
mk_status mk_get_field(mk_handle* h, int32_t field, int32_t dtype, void* host_dst, size_t bytes);
/* Multigrain: the order parameter of grain `grain` (phiVec[grain] of the
 * reference's node, mkFluidsUser.cpp:147-160), as mk_get_field. */
mk_status mk_get_grain_field(mk_handle* h, int32_t grain, int32_t dtype, void* host_dst, size_t bytes);
/* Replace the state by the equilibrium of host-provided macroscopic fields
 * (phi, and rho/u/T/C where the model has them).  Any pointer may be NULL to
 * keep the case's initial field.  Resets the step counter to 0. */
mk_status mk_set_state(mk_handle* h, const double* phi, const double* temp, const double* conc,
                       const double* rho, const double* ux, const double* uy, const double* uz);
/* Same from FP32 host buffers (pinned memory is used directly). */
mk_status mk_set_state_f32(mk_handle* h, const float* phi, const float* temp, const float* conc);

/* Legacy VTK RECTILINEAR_GRID writer in the reference's format
 * (MaterKit/src/mkFluidsUser.cpp:714-947); file <dir>/fluid_t<loops>.vtk. */
mk_status mk_write_vtk(mk_handle* h, int64_t loops, const char* dir);

/* Points of the phi = iso surface, in place of the ParaView contour of the
 * reference's post-processing (MaterKit/SaveContourBatch.py: Contour of
 * order_parameter at 0 on each fluid_t<loops>.vtk).  One point per grid edge
 * (no periodic wrap) whose end values straddle iso, placed by linear
 * interpolation in the VTK coordinates (cell index + 0.5): the vertices of a
 * marching-cubes contour.  Writes min(count, capacity) points: xyz gets 3
 * doubles per point, scalar (nullable) the temperature or solute of the
 * dendrite models interpolated the same way (0 for the others).  *count is
 * the total; capacity 0 only counts.  Order: by cell index, then axis.
 * MK_ERR_ARG for the models without an order parameter (flow, convection). */
mk_status mk_interface_points(mk_handle* h, double iso, double* xyz, double* scalar, int64_t capacity,
                              int64_t* count);

/* Tip lengths and velocities of seed `seed` (mk_tip); MK_ERR_ARG without an
 * order parameter or for a seed index out of range. */
mk_status mk_tip_track(mk_handle* h, int32_t seed, double iso, mk_tip* out);

/* FP64 conservation sums and the divergence watchdog. */
mk_status mk_diagnostics(mk_handle* h, mk_diag* out);

/* Nusselt number of a convection case (Thermal_NusseltRBC, mkFluidsLBM.h:67):
 * Nu = 1 + <u_a T> H / (kappa (T_low - T_high)), the volume average over the
 * fluid cells, a the plate axis, H the layer thickness between the half-way
 * plates, kappa the scalar diffusivity D.  FP64 reduction. */
mk_status mk_nusselt(mk_handle* h, double* nu);

/* Binary checkpoint: populations, phi, step and a parameter hash. */
mk_status mk_checkpoint(mk_handle* h, const char* path);
mk_status mk_restore(mk_handle* h, const char* path);

/* Timing of one kernel of the step (CUDA events on the handle's stream):
 * runs `launches` steps and returns the summed device time of the kernel
 * named `kernel` ("collide", "phi", ...), and the total step time. */
mk_status mk_profile_steps(mk_handle* h, int64_t nsteps, const char* kernel,
                           double* kernel_ms, double* step_ms, int64_t* kernel_launches);

/* Advance n loops bracketed by CUDA events on the handle's stream; returns the
 * device time in milliseconds (synchronises at the end). */
mk_status mk_time_advance(mk_handle* h, int64_t nsteps, int32_t use_graph, double* ms);

/* Launch-shape autotuner: times `trial_steps` loops of each candidate block
 * shape and occupancy variant of the step's kernels, and for a multiphase
 * case also the fused one-launch loop, the row-staged collision and the TMA
 * phi-tile collision, on a saved copy of the state (restored afterwards, so
 * the simulation is unchanged) and keeps the fastest.  Outputs may be NULL;
 * block_x = block_y = minb = 0 report that the fused loop won, minb = 0 with a
 * block shape that the row-staged or the phi-tile collision won (the shape is
 * the phi kernel's); mk_get_tuning gives the whole choice. */
mk_status mk_autotune(mk_handle* h, int32_t trial_steps, int32_t* block_x, int32_t* block_y, int32_t* minb,
                      double* ms_per_step);

/* Page-locked host buffers for end-to-end transfers (cudaHostAlloc). */
mk_status mk_host_alloc(size_t bytes, void** out);
mk_status mk_host_free(void* p);

/* ---- Gradients: discrete adjoint of the thermal dendrite loop -----------
 * L = sum over cells of (phi - target)^2, phi after `steps` loops from the
 * handle's current state.  Reverse mode over the loops the kernels run, with
 * state checkpoints every `checkpoint_every` loops (<= 0: 100) and each
 * segment recomputed forward.  Thermal dendrite cases, FP64 or FP32 storage;
 * the adjoint arithmetic is FP64.  The handle is left at the state after the
 * forward run (its step advanced by `steps`). */
typedef struct mk_loss {
  const double* target_phi; /* host, nx*ny*nz values, x fastest */
  int64_t steps;
  int64_t checkpoint_every;
} mk_loss;

typedef struct mk_grad {
  double loss;
  double d_eps4;   /* dL/d eps4 (the first anisotropy coefficient)                */
  double d_delta;  /* dL/d Delta: the initial u shifted uniformly by -Delta         */
  double d_tau_t;  /* dL/d tau_T, tau_T = 1/omega_T = 4 D + 1/2 (tau0 held fixed)   */
  int64_t forward_loops; /* loops run forward: the first pass plus the recomputation */
} mk_grad;

mk_status mk_backward(mk_handle* h, const mk_loss* loss, mk_grad* out);

/* ---- Ensembles: many dendrite domains advanced together ----------------
 * Batches unevenly sized domains (seed, anisotropy and undercooling sweeps of
 * run_solutal_dendrite / run_thermal_dendrite, MaterKit.cpp:633-687, 743-788)
 * into one packed cell index: every loop is two persistent launches over all
 * domains, and mk_ensemble_advance replays them as a CUDA graph.  All domains
 * share the model and the storage precision; each cell count must be a
 * multiple of 256. */
typedef struct mk_ensemble mk_ensemble;

/* Seeded generator of the solutal ensemble: n cubes with edges from
 * {48, 64, 80, 96, 128}, eps4 ~ U[0.02, 0.06], 1-6 seeds of radius U[4, 8]
 * with uniformly random orientations; k = 0.15, D_l = 0.1, D_s = 1e-4. */
mk_status mk_ensemble_case_params(uint64_t seed, int32_t n_domains, int32_t precision, mk_params* out);
mk_status mk_ensemble_create(const mk_params* params, int32_t n_domains, mk_ensemble** out);
mk_status mk_ensemble_destroy(mk_ensemble* e);
const char* mk_ensemble_last_error(const mk_ensemble* e);
mk_status mk_ensemble_advance(mk_ensemble* e, int64_t nsteps);
mk_status mk_ensemble_time_advance(mk_ensemble* e, int64_t nsteps, double* ms);
mk_status mk_ensemble_get_field(mk_ensemble* e, int32_t domain, int32_t field, int32_t dtype, void* host_dst,
                                size_t bytes);
/* Device time of one of the two launches of a loop ("phi" or "collide"),
 * summed over `nsteps` eager loops, and the total time of those loops. */
mk_status mk_ensemble_profile_steps(mk_ensemble* e, int64_t nsteps, const char* kernel, double* kernel_ms,
                                    double* step_ms);
/* Kernel launches issued so far (two per loop). */
int64_t mk_ensemble_launches(const mk_ensemble* e);
int64_t mk_ensemble_cells(const mk_ensemble* e);
int64_t mk_ensemble_step(const mk_ensemble* e);

/* Allocation-free FP64 statistics of a device-resident FP32 field.
 * No counterpart in the reference (its solver has no device code); it is the
 * diagnostics reduction for callers that may not call cudaMalloc, such as a
 * host code whose own pool owns the device memory.  Needs no handle.
 *   d_field: n floats in device memory; d_out: 5 doubles in device memory,
 *   {sum, sum of squares, min, max, count of non-finite values} (the first
 *   four over the finite values).  Asynchronous on `stream` (NULL = legacy
 *   default stream).
 * The block partials live in a fixed 80 KiB device array inside the library,
 * so n is limited to MK_NOALLOC_MAX_CELLS (larger n: MK_ERR_ARG, message in
 * mk_noalloc_last_error).  Every call on a device shares that array: calls
 * that overlap on the GPU race and must be serialised by the caller.  The
 * first call on a device looks up the array's address and should come before
 * any stream capture; the address is kept for the life of the process, so no
 * call may follow a cudaDeviceReset of that device.  Calls no allocating
 * routine. */
#define MK_NOALLOC_MAX_BLOCKS 2048
#define MK_NOALLOC_MAX_CELLS ((int64_t)MK_NOALLOC_MAX_BLOCKS * 256 * 64)
mk_status mk_field_stats_noalloc(const float* d_field, int64_t n, double* d_out, void* stream);
const char* mk_noalloc_last_error(void);

/* JSON-lines metrics log, no counterpart in the reference (its only record is
 * the write_document text file, MaterKit.cpp:126-184).  With a path set, every
 * mk_time_advance appends {"event": "time_advance", model, precision, step,
 * loops, ms, mlups, gbs (algorithmic bytes), launches_per_loop} and every
 * mk_diagnostics {"event": "diagnostics", model, step, mass, phi_sum,
 * mass_drift, phi_drift (relative to the handle's first diagnostics),
 * solid_frac, max_speed, n_bad}.  NULL stops the log.  Process-wide. */
mk_status mk_set_metrics_log(const char* path);

/* ---- A dendrite growing in a two-phase flow ------------------------------
 * run_flow_multiphase_dendrite (MaterKit/MaterKit.cpp:377-397) couples two
 * solver objects per loop: the dendrite's phase field, its thermal lattice
 * advected by the flow (update_velocity, mkThermalField.h:36), then the
 * multiphase flow with the dendrite's solid as geometry (update_geometry,
 * mkFluidsMultiphase.h:37).  Here the two objects are two handles of the same
 * grid on the same device, and a loop is
 *   mk_update_velocity(dendrite, flow); mk_advance(dendrite, 1);
 *   mk_update_geometry(flow, dendrite); mk_advance(flow, 1);
 * (the reference's bodies are in its closed DLL; these are the semantics
 * defined here). */

/* The multiphase flow's cells where the dendrite's phase field is positive
 * become solid (cumulative: a solid cell stays solid): a solid cell is not
 * updated, links into it bounce back (half-way), and the Allen-Cahn stencil
 * sees the wetting value there, as at a wall.  The change takes effect at the
 * flow's next even loop count, where the in-place streaming holds every
 * population in its own cell (the liquid of a cell that solidifies leaves the
 * flow).  The fused and row-staged forms are turned off for the flow.
 * MK_ERR_ARG unless flow is a multiphase and dendrite a thermal or solutal
 * dendrite handle of the same grid and device (no slab handles). */
mk_status mk_update_geometry(mk_handle* flow, mk_handle* dendrite);
/* The dendrite's scalar lattice is advected by the flow's current velocity
 * (its equilibrium w T (1 + 4 e.u), as in the flow + dendrite models); the
 * phase field is not.  Synchronous.  MK_ERR_ARG as for mk_update_geometry. */
mk_status mk_update_velocity(mk_handle* dendrite, mk_handle* flow);

/* ---- z-slab decomposition of one multiphase domain ----------------------
 * No counterpart in the reference: its solver runs one domain in one process,
 * its cell sweeps shared out by OpenMP (mkFluidsUser.cpp:70, 116, 147).  Here
 * one domain of the multiphase model is split into contiguous runs of z
 * planes, one per rank (one process per GPU, or several handles in one
 * process), and the ranks exchange plane-sized runs between the two kernels
 * of every loop.
 *
 * A slab handle holds its nz_own planes as the local planes 1 .. nz_own, plus
 * two ghost planes (local 0 below, nz_own + 1 above) that receive copies of
 * the neighbour slabs' boundary planes; its arrays have the layout of a
 * domain of nz_own + 2 planes (mk_get_params reports that nz), and
 * mk_get_field returns all nz_own + 2 planes.  Ghost cells are never updated.
 *
 * The in-place streaming (AA pattern) decides what crosses a slab face:
 *   MK_SLAB_FILL   before an odd loop: the 5 populations with e_z = -1 of the
 *                  top owned plane go up into the ghost 0 of the slab above,
 *                  the 5 with e_z = +1 of plane 1 go down into the top ghost
 *                  of the slab below (both lattices: 20 plane runs a slab);
 *   MK_SLAB_PHI    every loop, after the phi kernel: the top owned phi plane
 *                  up into ghost 0 above, plane 1 down into the top ghost
 *                  below (the gradient and Laplacian stencil of phi);
 *   MK_SLAB_RETURN after an odd loop, and once after mk_create_slab: the odd
 *                  loop (and the initial state) wrote the same 5 + 5 slots of
 *                  the ghost planes; they go back to the planes they belong
 *                  to (ghost 0 down to the top owned plane below, the top
 *                  ghost up to plane 1 above).  They land in the receiving
 *                  slab's halo buffer, and mk_slab_done merges them into the
 *                  owned plane on the handle's stream, except the slots whose
 *                  source cell across the face is not fluid (next to an x or
 *                  y wall or closed face, or a global wall plane): those the
 *                  cell wrote itself by bounce-back.
 * A loop is therefore [FILL if odd] RUN_PHI PHI RUN_COLLIDE [RETURN if odd];
 * mk_slab_next reports the next action and the run / done calls refuse any
 * other (MK_ERR_STATE).  Non-periodic global ends have no neighbour and
 * exchange nothing; a periodic z axis wraps (with one rank, onto itself).
 * Fused loops, graphs, the autotuner, checkpoints and the adjoint are not
 * available on slab handles (MK_ERR_STATE). */
enum {
  MK_SLAB_FILL = 0,
  MK_SLAB_PHI = 1,
  MK_SLAB_RETURN = 2,
  MK_SLAB_RUN_PHI = 3,
  MK_SLAB_RUN_COLLIDE = 4
};

/* One plane-sized run of a slab exchange: `count` elements at element
 * `offset` of an array of the slab (array 0: the pressure lattice g, whose
 * element offset is population * stride + plane * nx * ny; 1: the Allen-Cahn
 * lattice h, same; 2: phi, plane * nx * ny; 3: the halo buffer of a return
 * exchange, ((face * 2 + lattice) * 5 + k) * nx * ny for the k-th population
 * crossing the lower (face 0) or upper (face 1) face), sent to or received
 * from `peer`.
 * The two ends of one transfer carry the same `tag`; a rank's list is sorted
 * by (peer, tag), so two ranks that post their sends and receives in list
 * order match them pairwise. */
typedef struct mk_slab_xfer {
  int32_t peer;  /* the other rank (may be this rank, periodic z with one rank) */
  int32_t send;  /* 1: this rank sends the run, 0: it receives into the run    */
  int32_t tag;   /* 128 * (0 upward, 1 downward) + 32 * array + population    */
  int32_t array; /* 0 g, 1 h, 2 phi, 3 return halo                             */
  int64_t offset;
  int64_t count;
  int64_t bytes;
  void* ptr;     /* device address of the run (mk_slab_transfers); NULL from mk_slab_plan */
} mk_slab_xfer;

/* The planes rank `rank` of `nranks` owns of a domain of nz planes: the first
 * nz % nranks ranks own nz / nranks + 1, the others nz / nranks. */
mk_status mk_slab_split(int32_t nz, int32_t rank, int32_t nranks, int32_t* z0, int32_t* nz_own);
/* Host-only: the transfers of one exchange stage of rank `rank` for the global
 * case `global` (ptr NULL).  At most MK_SLAB_MAX_XFER entries (a slab with a
 * neighbour on both faces: 40 population runs, or 4 phi runs); `capacity`
 * below what the stage needs is MK_ERR_ARG with *count set to the need. */
#define MK_SLAB_MAX_XFER 40
mk_status mk_slab_plan(const mk_params* global, int32_t rank, int32_t nranks, int32_t stage, mk_slab_xfer* out,
                       int32_t capacity, int32_t* count);
/* Create the slab of rank `rank` of the multiphase case `global` on the current
 * device, from the global initial state (the same as mk_create's).  The first
 * action is MK_SLAB_RETURN. */
mk_status mk_create_slab(const mk_params* global, int32_t rank, int32_t nranks, mk_handle** out);
/* Slab geometry of a handle (MK_ERR_STATE for a whole-domain handle). */
mk_status mk_slab_info(const mk_handle* h, int32_t* rank, int32_t* nranks, int32_t* z0, int32_t* nz_own,
                       int32_t* nz_global);
/* Next action of the loop protocol (MK_SLAB_*), -1 for a whole-domain handle. */
int32_t mk_slab_next(const mk_handle* h);
/* mk_slab_plan of the handle's slab with device addresses filled in. */
mk_status mk_slab_transfers(const mk_handle* h, int32_t stage, mk_slab_xfer* out, int32_t capacity, int32_t* count);
/* The caller completed the exchange `stage` (every receive has landed and is
 * ordered before the handle's next launch: done on the handle's stream, or
 * synchronised).  For MK_SLAB_RETURN this launches the merge of the halo
 * buffer into the owned planes. */
mk_status mk_slab_done(mk_handle* h, int32_t stage);
/* Launch the next kernel: MK_SLAB_RUN_PHI or MK_SLAB_RUN_COLLIDE (the latter
 * completes the loop and advances mk_get_step). */
mk_status mk_slab_run(mk_handle* h, int32_t action);
/* In-process exchange among the n slabs of one decomposition (hs[r] is rank
 * r, all of the same case and stage): stream-ordered device copies (peer
 * copies across devices), then mk_slab_done on every handle. */
mk_status mk_slab_exchange_local(mk_handle* const* hs, int32_t n, int32_t stage);

/* Algorithmic bytes per cell per step of the handle's configuration. */
double mk_bytes_per_cell(const mk_handle* h);
/* Fluid cells the handle updates (a slab: its owned planes only). */
int64_t mk_fluid_cells(const mk_handle* h);
/* Number of kernel launches one step issues. */
int32_t mk_launches_per_step(const mk_handle* h);

#ifdef __cplusplus
}
#endif

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#endif /* MKB200_H */
