/*
 * dfdm.h -- C ABI of the B200 library for dopamine-fdm's single-phase fractional-step RK3 time step.
 *
 * The library replaces, on one GPU, the Fortran subroutines that make up one time step of the reference
 * solver (the RK3 driver, the momentum right-hand side, the AMD/Vreman eddy viscosity, the flat-wall
 * equilibrium wall model, the FFT x tridiagonal pressure Poisson solve with the velocity correction, and the
 * ghost fills). Every entry point is a plain C function with plain pointers and sizes, so a Fortran host can
 * bind it through ISO_C_BINDING (Bind(C, name="dfdm_...")).
 *
 * Array conventions (all host arrays): IEEE double, Fortran column-major order, in the reference's ghosted
 * one-rank shapes with nxg = nx+1, nyg = ny+1, nzg = nz+1 (nx, ny, nz = namelist face counts):
 *   U (nx ,nyg,nzg)   V (nxg,ny ,nzg)   W (nxg,nyg,nz )   P, nu_t (nxg,nyg,nzg)
 *   rhs_u (2:nx-1,2:nyg-1,2:nzg-1)  rhs_v (2:nxg-1,2:ny-1,2:nzg-1)  rhs_w (2:nxg-1,2:nyg-1,2:nz-1)
 *   rhs_p (2:nxg,2:nyg-1,2:nzg)
 * On the device the library keeps only the independent cells (periodic duplicates and ghosts are implied by
 * the boundary rules), in FP64 or in FP32 storage (DFDM_FP32_MIXED). Ghosts are regenerated on every copy
 * back to the host, exactly as apply_boundary_conditions / finish_pressure_ghosts would leave them.
 *
 * Every function returns a status code (DFDM_OK = 0); dfdm_last_error() gives the message of the last
 * failure on the calling thread. A context owns one CUDA stream and all of its device memory; contexts are not
 * thread-safe. Calls are synchronous unless their name ends in _async.
 */
#ifndef DFDM_H
#define DFDM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define DFDM_OK               0
#define DFDM_ERR_INVALID      1   /* invalid argument or grid */
#define DFDM_ERR_CUDA         2   /* CUDA runtime error (message in dfdm_last_error) */
#define DFDM_ERR_NOMEM        3   /* device allocation failed */
#define DFDM_ERR_UNSUPPORTED  4   /* configuration outside the single-phase path */
#define DFDM_ERR_NOT_FINITE   5   /* NaN/Inf or |U| > 1e8 found by the monitor guard */
#define DFDM_ERR_TIMEOUT      6   /* a bounded device wait gave up */

/* ---- storage precision ---- */
#define DFDM_FP64        0   /* plain FP64: every field and every kernel in double */
#define DFDM_FP32_MIXED  1   /* FP32 fields, stencils and FFTs; FP64 tridiagonal solves and reductions */

/* Grid of one case (one rank of the reference: x_global = x etc.).
 * Mirrors the &DOMAIN / &BOUNDARY_CONDITIONS namelists (src/input_output.f90:29-107) and the face arrays built
 * by generateGrid (src/genGridandIC.f90:14-265). Centres, ghost centres, dx/dz, weights, modified wavenumbers
 * and the Dyy operator are derived inside the library exactly as src/initialization.f90:243-644 does. */
typedef struct dfdm_grid {
    int nx, ny, nz;            /* face counts (namelist nx, ny, nz); nx and nz even */
    const double *x;           /* x(1:nx) face coordinates, uniform */
    const double *y;           /* y(1:ny) face coordinates, may be stretched */
    const double *z;           /* z(1:nz) face coordinates, uniform */
    int x_bc_type;             /* 0 periodic; 1 inflow/outflow (a context for dfdm_solve_poisson only, see below) */
    int y_bc_type;             /* 0 periodic, 1 walls */
    int z_bc_type;             /* 0 periodic; 1 walls (a context for dfdm_solve_poisson only: the duct or spanwise walls) */
    int bc_face_ylo, bc_face_yhi; /* 1 no-slip (the only value on this path) */
} dfdm_grid;

/* Physics and numerics of one case (&PHYSICS / &NUMERICS subset the step reads; defaults in
 * src/global.f90:305-312 and src/input_output.f90:109-127). Automatic values (-1) are resolved as
 * src/input_output.f90:938-940 (adv_wall_layers) and :967-970 (wm_filter_mode) do. */
typedef struct dfdm_params {
    double nu;                 /* kinematic viscosity */
    double dt;                 /* fixed time step (cfl_adaptive = 0) */
    double dPdx, dPdz;         /* imposed mean pressure gradients (flow_forcing_mode = 0) */
    int    sgs_model;          /* 0 DNS, 1 Vreman, 2 AMD */
    double Cs_vreman;          /* Vreman constant (0.17) */
    double C_amd;              /* AMD constant (1/3) */
    int    flat_wall_model_flag; /* 0 no-slip walls, 1 smooth Reichardt EQWM */
    int    advection_scheme;   /* 0 skew-symmetric blend, 1 divergence form, 2 skew-symmetric + upwind-biased
                                  dissipation (src/adv_hybrid.f90) */
    int    adv_wall_layers;    /* -1 automatic */
    int    wm_filter_mode;     /* -1 automatic, 0 raw, 1 temporal filter */
    double wm_filter_Tf_fac;   /* filter time-scale factor (1.0) */
    int    flow_forcing_mode;  /* 0 prescribed dPdx, 1 constant flux */
    double Ub_target;          /* bulk velocity target of the constant-flux forcing */
    int    precision;          /* DFDM_FP64 or DFDM_FP32_MIXED */
    int    adv_order;          /* advection_scheme = 2: order of the dissipation, 3 or 5 (default 3) */
    double adv_beta0;          /* advection_scheme = 2: its coefficient beta, >= 0 (default 0.05); with no immersed
                                  body beta = adv_beta0 everywhere (src/adv_hybrid.f90:22-74) */
} dfdm_params;

typedef struct dfdm_ctx dfdm_ctx;

/* Fill *p with the reference defaults (src/global.f90:305-312, src/input_output.f90:109-127). */
void dfdm_default_params(dfdm_params *p);

/* Text of the last failure on this thread ("" after success). */
const char *dfdm_last_error(void);

/* Library version string. */
const char *dfdm_version(void);

/* ---- lifetime: replaces initialize's device part (src/initialization.f90:37-862) ----
 * x_bc_type = 1 (inflow/outflow x; needs y walls, y_bc_type = 1, and nx - 1 <= 257) creates a context for the
 * DCT-IV pressure solve alone (src/projection.f90:124-130,334-343): dfdm_solve_poisson, the stream calls,
 * dfdm_synchronize, dfdm_launch_count and dfdm_destroy accept it, every other entry point returns
 * DFDM_ERR_UNSUPPORTED (the inflow/outflow step, boundary conditions and convective outflow are not built).
 * z_bc_type = 1 with y walls and periodic x (the 4-wall duct; nz - 1 <= 512) likewise creates a context for the
 * duct's pressure solve alone (src/projection.f90:172-217): the z-eigenmode transform of Dzz (diagonalised once here,
 * as the reference's dstev call at src/initialization.f90:579-608 does), one y-tridiagonal solve per (kx, z mode).
 * z_bc_type = 1 with periodic x and y (spanwise walls alone; nz - 1 <= 1024) creates a context for that pressure
 * solve (src/projection.f90:136-143,219-250): FFT in x and y, one z-tridiagonal solve per (kx, ky). The reference's
 * CPU build solves it; its GPU build rejects it. x_bc_type = 1 with z_bc_type = 1 and y walls (the duct with
 * inflow/outflow x, also the CPU build's) combines the DCT-IV x transform with the z eigenmodes; spanwise walls with
 * inflow/outflow x return DFDM_ERR_UNSUPPORTED. */
int dfdm_create(const dfdm_grid *grid, const dfdm_params *params, dfdm_ctx **out);
int dfdm_destroy(dfdm_ctx *ctx);
/* Bytes of device memory a context of this grid and precision would hold (serving admission). */
int dfdm_footprint_bytes(const dfdm_grid *grid, const dfdm_params *params, size_t *bytes);

/* Run the context's work on an externally owned CUDA stream (cudaStream_t passed as void*); NULL restores the
 * context's own stream. */
int dfdm_set_stream(dfdm_ctx *ctx, void *cuda_stream);
/* The stream the context's work runs on (its own, created non-blocking by dfdm_create, or the one set). */
int dfdm_get_stream(dfdm_ctx *ctx, void **cuda_stream);
int dfdm_synchronize(dfdm_ctx *ctx);   /* waits for the context's stream and its copy streams */

/* ---- state transfer: the reference's U, V, W, P, nu_t module arrays (src/global.f90:139,300) ----
 * set_state reads the interior (independent) cells; ghosts are implied. P may be NULL. */
int dfdm_set_state(dfdm_ctx *ctx, const double *U, const double *V, const double *W, const double *P);
int dfdm_get_state(dfdm_ctx *ctx, double *U, double *V, double *W, double *P);
/* The same transfers, enqueued without a host synchronisation: uploads run on a copy stream of their own, downloads
 * on another, the unpack/pack kernels on the context's stream in order with the steps.  A host loop of set_async,
 * step_async, get_async therefore overlaps one step's download with the next step's upload.  The host arrays must
 * stay untouched until dfdm_synchronize (pinned memory makes the copies asynchronous; pageable memory works but
 * copies synchronously).  The context's first FP32-mixed set_state fixes its base profile and is synchronous. */
int dfdm_set_state_async(dfdm_ctx *ctx, const double *U, const double *V, const double *W, const double *P);
int dfdm_get_state_async(dfdm_ctx *ctx, double *U, double *V, double *W, double *P);
int dfdm_get_nu_t(dfdm_ctx *ctx, double *nu_t);
int dfdm_set_nu_t(dfdm_ctx *ctx, const double *nu_t);
int dfdm_set_time(dfdm_ctx *ctx, double t);
int dfdm_get_time(dfdm_ctx *ctx, double *t);

/* ---- the step: compute_time_step_RK3 (src/time_integration.f90:120-713) ----
 * Advances nsteps full RK3 steps on the resident state and returns the new time in *t (may be NULL). */
int dfdm_compute_time_step_rk3(dfdm_ctx *ctx, int nsteps, double *t);
/* Same, enqueued on the context's stream without a host synchronisation. */
int dfdm_compute_time_step_rk3_async(dfdm_ctx *ctx, int nsteps);
/* Capture one full step in a CUDA graph on first use and replay it (same numerics as the plain call). */
int dfdm_enable_graphs(dfdm_ctx *ctx, int enable);

/* ---- unit entry points, one per reference subroutine, on the resident state ---- */
/* compute_sgs_model(U,V,W,nu_t) (src/sgs_model.f90:27-45, ghosts :538-609) */
int dfdm_compute_sgs_model(dfdm_ctx *ctx);
/* compute_rhs_u / _v / _w (src/equations.f90:25-257, :261-485, :489-721) on the resident U,V,W,nu_t and wall
 * stresses; results in the reference's rhs shapes. Any output pointer may be NULL. */
int dfdm_compute_rhs(dfdm_ctx *ctx, double *rhs_u, double *rhs_v, double *rhs_w);
/* update_wm_filter + compute_wall_model (src/wallmodel.f90:397-439, :197-233, :442-583); tau_x (nx,2,nzg) and
 * tau_z (nxg,2,nz) may be NULL. update_filter = 1 advances the temporal filter first (stage 1 of a step). */
int dfdm_compute_wall_model(dfdm_ctx *ctx, int update_filter, double *tau_x, double *tau_z);
/* apply_boundary_conditions (src/boundary_conditions.f90:186-260). On the device the ghost cells are implied by
 * the index rules, so this validates the context and returns; kept for drop-in completeness. */
int dfdm_apply_boundary_conditions(dfdm_ctx *ctx, int after_projection);
/* compute_projection_step (src/projection.f90:21-34): div, Poisson solve and velocity correction of the
 * resident velocity. save_p = 1 also stores P = phi/(dt*3/4) as the third RK stage does. */
int dfdm_compute_projection_step(dfdm_ctx *ctx, int save_p);
/* solve_poisson_equation's solve alone (src/projection.f90:100-382): rhs_p in, pseudo-pressure out, both in
 * the reference shape (2:nxg,2:nyg-1,2:nzg); the output ghost planes follow apply_periodic_xz_pressure.
 * On an inflow/outflow-x context (x_bc_type = 1) the x transform is the DCT-IV (FFTW REDFT11) of the nx - 1
 * cells 2:nxg-1 with kxx(i) = 2 (cos(pi (2i+1) / (2 (nx-1))) - 1) / dx^2 and no null-mode fix; the output's
 * plane i = nxg keeps the input, as the reference's array does, and the z plane nzg (unset by the reference's
 * apply_periodic_xz_pressure at one rank) keeps the input too.
 * On a 4-wall duct context (z_bc_type = 1) the z direction is solved in physical space through Dzz's eigenbasis; the
 * output's z plane nzg keeps the input (no z copy with a wall) apart from the x copy rhs_p(nxg-1) = rhs_p(2); with
 * spanwise walls (periodic y) the y copy rhs_p(:, nyg-1, :) = rhs_p(:, 2, :) covers that plane too. */
int dfdm_solve_poisson(dfdm_ctx *ctx, const double *rhs_p_in, double *phi_out);
/* No counterpart in the reference: dfdm_solve_poisson with no device allocation in the call.
 * dfdm_solve_poisson grows a per-context staging buffer with cudaMalloc on first use (and frees and regrows it,
 * which waits for the whole device, when a larger copy comes along). Hosts that pack many contexts onto one GPU
 * up to its memory limit, or that run other contexts' steps on concurrent streams, cannot take that: the
 * cudaMalloc may fail on a full device and the cudaFree stalls every stream. This variant stages rhs_p and phi
 * through one file-scope device array of DFDM_NOALLOC_MAX_POINTS doubles (16 MiB, reserved when the library is
 * loaded on a device) and otherwise runs the same kernels on the context's own buffers.
 *  - Sizes: (nxg-1)*(nyg-2)*(nzg-1) must not exceed DFDM_NOALLOC_MAX_POINTS, else DFDM_ERR_INVALID.
 *  - The first call on a device looks the array's address up on the current device; make that first call
 *    before any stream capture begins. The context's device must be current, as for every entry point.
 *  - Every call, from any context, shares the one array and leaves its contents behind; each call writes the
 *    part it reads before reading it. Calls whose GPU work overlaps (different streams, or different host
 *    threads) race on the array: serialise them. */
#define DFDM_NOALLOC_MAX_POINTS 2097152
int dfdm_solve_poisson_noalloc(dfdm_ctx *ctx, const double *rhs_p_in, double *phi_out);
/* ---- tuning (no counterpart in the reference) ----
 * The FP32 stage kernel (RHS + RK3 update) has three variants: 0 computes one cell per thread on 32 x 8 tiles,
 * 1 computes two x-neighbour cells per thread with the packed FP32x2 instructions on 64 x 8 tiles, 2 is variant 1
 * with its z-plane tiles brought in by the Tensor Memory Accelerator (3-D boxes completing on mbarriers, four planes
 * in flight); variant 2 needs walls in y and Nx a multiple of 4. dfdm_create times the eligible variants on the
 * context's grid and keeps the fastest; the choice is cached per device and grid shape for the process.
 * set_stage_variant forces 0, 1 or 2 (DFDM_ERR_UNSUPPORTED where not eligible), or re-times with -1 (FP64
 * contexts have variant 0 only); a change drops the context's captured step graph. get_stage_variant returns the
 * variant in use and the timings of variants 0 and 1, get_stage_timing that of any variant (ms per launch, -1
 * where not timed); any output pointer of get_stage_variant may be NULL. A bounded wait of variant 2 that gives up
 * makes the next synchronising call (dfdm_compute_time_step_rk3, dfdm_synchronize) return DFDM_ERR_TIMEOUT. */
int dfdm_set_stage_variant(dfdm_ctx *ctx, int variant);
int dfdm_get_stage_variant(dfdm_ctx *ctx, int *variant, double *ms_one, double *ms_pairs);
int dfdm_get_stage_timing(dfdm_ctx *ctx, int variant, double *ms);

/* ---- snapshots in the reference's restart format ----
 * output_data's staggered full snapshot (src/input_output.f90:1782-1880): a stream holding the mesh (int32 n and n
 * doubles for x, y, z and the centres xm, ym, zm) and then U, V, W, P and, with an SGS model, nu_t, each as int32 n1,
 * n2, n3 and the ghosted array in Fortran order. With the wall-model filter seeded (wm_filter_mode = 1),
 * write_wm_filter_state (:1990-2009) adds <path>.wmf with the six filter planes. The reference opens both files
 * without convert= (:1842, :1996), so they take its build's default byte order, which its CMakeLists.txt:210
 * sets to big-endian for every compiler (gfortran -fconvert=big-endian, Intel -convert big_endian, NVHPC
 * -Mbyteswapio). dfdm_write_snapshot therefore writes big-endian; dfdm_write_snapshot_ex takes the byte order
 * (DFDM_BIG_ENDIAN or DFDM_LITTLE_ENDIAN, the latter for a reference build without those flags). */
#define DFDM_LITTLE_ENDIAN 0
#define DFDM_BIG_ENDIAN    1
int dfdm_write_snapshot(dfdm_ctx *ctx, const char *path);
int dfdm_write_snapshot_ex(dfdm_ctx *ctx, const char *path, int byte_order);
/* write_box_snapshot (src/input_output.f90:1699-1767, field_box :1586-1598, fill_box_block :1623-1659): the
 * chunked or cell-centred box snapshot of the face box f1..f2 (1-based faces, f1 < f2 <= nx/ny/nz), which the reference
 * writes for chunked_snapshot and for snapshot_location = 1 (then over the whole domain, f1 = 1, f2 = n). Little-endian
 * stream: int32 -4242, location, step, nfields; float64 t; int32 f1(3), f2(3); per direction float64 faces
 * x(f1:f2) and centres xm(f1:f2-1); per field char name(8) (blank-padded U, V, W, P and, with an SGS model, nu_t),
 * int32 st(3), gl(3), gh(3); then each field's box gl:gh in Fortran order. location 0 keeps the velocities on their
 * faces (st = 1 in their own direction); location 1 averages them to the cell centres. step is the reference's
 * istep + nstep_init. Box snapshots cannot be read back as a restart. */
int dfdm_write_box_snapshot(dfdm_ctx *ctx, const char *path, const int32_t f1[3], const int32_t f2[3], int location,
                            int32_t step);
/* read_input_data (src/input_output.f90:1225-1341) with the pressure block of read_pressure_restart (:1972-1977)
 * and read_wm_filter_state (:2011-2031): loads U, V, W and P from a restart file of this grid (DFDM_ERR_INVALID
 * for a chunked/cell-centred snapshot, a short file, other face counts, other coordinates or a block of another
 * shape) and the filter planes from <path>.wmf when it exists; without it the filter re-seeds on the next step.
 * The byte order is taken from the file: big-endian when its first word read big-endian is nx, little-endian
 * when read little-endian it is (the reference reads only its build's order); the .wmf is read in the same order.
 * A first word of -4242 read little-endian marks a box snapshot, as the reference's probe (:1235) reads it. */
int dfdm_read_snapshot(dfdm_ctx *ctx, const char *path);
/* compute_bulk_velocity (src/monitor.f90:463-523), FP64 compensated sum. */
int dfdm_compute_bulk_velocity(dfdm_ctx *ctx, double *Ub);
/* check_divergence (src/projection.f90:607-639): max |div u| over the interior. */
int dfdm_check_divergence(dfdm_ctx *ctx, double *max_div);
/* compute_cfl (src/monitor.f90:304-424) for the single-phase path: dt * max over the centres of
 * |u_c|/dx + |v_c|/dy + |w_c|/dz (convective) and of (nu + nu_t) * 2 * (1/dx^2 + 1/dy^2 + 1/dz^2) (viscous). */
int dfdm_compute_cfl(dfdm_ctx *ctx, double *cfl_conv, double *cfl_visc);
/* Adaptive time step, cfl_adaptive = 1 of &TIME (src/global.f90:472-478): with enable != 0 every step starts, after
 * the SGS eddy viscosity, with select_dt (src/monitor.f90:429-444; src/time_integration.f90:146-160):
 * dt = max(dt_min, min(dt_max, dt * cfl_target / cfl * cfl_safety)) from cfl = max(cfl_conv, cfl_visc) of the
 * start-of-step velocity and the previous dt (the &NUMERICS dt before the first step).  dt and t stay on the device,
 * so steps and their graph replays need no host synchronisation; dfdm_get_dt / dfdm_get_time read them.
 * enable = 0 returns to the fixed dt.  Requires cfl_target, cfl_safety > 0 and 0 < dt_min <= dt_max. */
int dfdm_set_adaptive_dt(dfdm_ctx *ctx, int enable, double cfl_target, double cfl_safety, double dt_min, double dt_max);
/* Output landing of select_dt (nsave < 0, nsteps < 0; src/monitor.f90:436-458): with enable != 0 the coming steps
 * are shrunk by landing_dt so that t lands on t_land (a remainder below 2 dt in one step, one between dt and 2 dt in
 * two equal halves); dt returns to its value before the shrink after the step (src/time_integration.f90:711).
 * A target within 1e-10 of t counts as reached; the caller then sets the next one (a new target keeps the captured
 * step graph).  Works with the fixed and with the adaptive dt.  t_land must be finite.  It replaces every target set
 * through dfdm_set_landing_times (enable = 0 removes them all). */
int dfdm_set_landing_time(dfdm_ctx *ctx, int enable, double t_land);
/* All of select_dt's landing targets (src/monitor.f90:436-440), applied in turn in this order: tsave_next
 * (nsave < 0), chunk_tsave_next (chunked_snapshot with chunk_nsave < 0), slice_tnext (slice_freq < 0), line_tnext
 * (line_freq < 0), sim_end_time (nsteps < 0). t_land[q] for q < n, NaN for a slot without a target; 0 <= n <= 5, n = 0
 * removes every target. dfdm_set_landing_time(ctx, 1, t) is the single target {t}. */
int dfdm_set_landing_times(dfdm_ctx *ctx, int n, const double *t_land);
/* The reference's dt between steps: the fixed dt, or the adaptive dt of the last step before any landing shrink. */
int dfdm_get_dt(dfdm_ctx *ctx, double *dt);
/* The values output_monitor prints (src/monitor.f90:21-102), computed on the device. */
typedef struct dfdm_monitor {
    double t;          /* time */
    double dt;         /* the reference's dt between steps */
    double mean_u;     /* compute_bulk_velocity (meanU) */
    double max_u;      /* max |U| over the independent U faces (maxU) */
    double max_div;    /* check_divergence (max_divergence) */
    double cfl_conv;   /* compute_cfl of the current state, convective */
    double cfl_visc;   /* compute_cfl of the current state, viscous */
    double u_tau_lo;   /* wall_diag_sums (src/wallmodel.f90:700-723): mean u_tau of the lower wall over the reference's
                          (nx-2)*(nzg-2) columns (the periodic duplicate z-plane included); 0 without the y-wall model */
    double u_tau_hi;   /* the same for the upper wall */
    double nan_flag;   /* 1 when the guard of output_monitor trips (a NaN or Inf, or |u| > 1e8), else 0 */
} dfdm_monitor;
/* output_monitor: all of dfdm_monitor in one device pass and one copy.  Returns DFDM_ERR_NOT_FINITE, with *out filled,
 * when the guard trips (where the reference aborts the run).  The CFL numbers are those of the current state (the
 * reference prints those of the start of the step just taken). */
int dfdm_output_monitor(dfdm_ctx *ctx, dfdm_monitor *out);
/* Same, enqueued on the context's stream with no host synchronisation: *out (pinned host or device memory) is
 * written when the stream reaches it, after the steps enqueued before; check nan_flag there. */
int dfdm_output_monitor_async(dfdm_ctx *ctx, dfdm_monitor *out);
/* Kinetic energy 0.5*<u.u> (volume-weighted, compensated sum) -- diagnostic with no reference counterpart. */
int dfdm_kinetic_energy(dfdm_ctx *ctx, double *ke);
/* Monitor guard of output_monitor (src/monitor.f90:32-52): DFDM_ERR_NOT_FINITE if any velocity is NaN/Inf or
 * |U| > 1e8. */
int dfdm_check_finite(dfdm_ctx *ctx);
/* pad_field_dev (src/halo_pad.f90:185-194) builds copies of a field with extra x/z planes for wide stencils. Its
 * callers are the hybrid advection scheme (advection_scheme = 2), the immersed boundary and the particles. On one
 * GPU the hybrid scheme reads its +-3 x/z neighbours with periodic index wraps instead of padded copies
 * (k_adv_hybrid_faces), and the other two callers are not on the single-phase path, so no padded copy is ever
 * needed: this entry point returns DFDM_ERR_UNSUPPORTED. */
int dfdm_pad_field(dfdm_ctx *ctx, int field, int extra_planes, double *out);

/* ---- profiling hooks: launch one kernel family of one RK stage on the context's stream, no sync ----
 * which: 0 SGS, 1 stage (RHS + RK update), 2 div + forward x-FFT, 3 forward z-FFT, 4 y solve,
 *        5 inverse z-FFT, 6 inverse x-FFT, 7 velocity correction, 8 wall model, 9 constant-flux bulk sum + shift,
 *        10 CFL maxima, 11 the dissipative terms of advection_scheme = 2 */
int dfdm_launch_kernel_async(dfdm_ctx *ctx, int which, int rk_stage);
/* Fused corrections (on by default where they apply: the wall model only with its temporal filter, no hybrid
 * advection scheme; LES only with the eddy viscosity computed in the stage tiles, dfdm_set_sgs_in_tile).  The projections of RK stages 1
 * and 2 then run inside the next stage kernel's loader instead of as separate launches, and the step-start velocity
 * stays in place as the RK base state: two launches and 17 words per cell fewer per step, the same arithmetic.  No
 * counterpart in the reference; enable = 0 restores the separate corrections (DFDM_ERR_UNSUPPORTED for enable = 1
 * where they do not apply). */
int dfdm_set_fused_correction(dfdm_ctx *ctx, int enable);
int dfdm_get_fused_correction(dfdm_ctx *ctx, int *enabled);
/* LES (sgs_model > 0): with enable = 1 the stage kernels compute the eddy viscosity of compute_vreman
 * (src/sgs_model.f90:118-223) from their own shared-memory velocity tiles, on the tile and a one-cell halo, instead of
 * reading the field a separate full-grid pass wrote at the step start and after the stage-1 and stage-2 projections
 * (src/time_integration.f90:144,361,493), and the fused corrections come on with it (where they apply). The results
 * agree with the separate pass to rounding; from one state the field is the same bit for bit. The stage-3 kernel
 * stores its field, so dfdm_get_nu_t, the CFL numbers and snapshots after a step see the step's last nu_t as before;
 * the adaptive time step still runs the pass at the step start for its CFL. enable = 0 (the default: on the Re_tau 395
 * LES grid the separate pass measured faster, 0.254 against 0.326 ms per FP32 step) restores the pass and turns the
 * fused corrections off, since the pass reads the corrected velocity. With the wall model, both forms read the
 * first-cell gradient factor of the override from a per-wall-cell table that a small kernel fills from the same
 * velocity before each evaluation. DFDM_ERR_UNSUPPORTED without an SGS model. No counterpart in the reference. */
int dfdm_set_sgs_in_tile(dfdm_ctx *ctx, int enable);
int dfdm_get_sgs_in_tile(dfdm_ctx *ctx, int *enabled);
/* Algorithmic HBM bytes one launch of that kernel family moves (the roofline numerator). */
int dfdm_kernel_bytes(dfdm_ctx *ctx, int which, double *bytes);
/* Number of the library's own kernels enqueued by this context so far (graph replays included). */
int dfdm_launch_count(dfdm_ctx *ctx, long long *count);

/* ---- serving groups (no counterpart in the reference) ----
 * A host that serves many small cases on one GPU steps them one context at a time: per FP32 step a context enqueues
 * 19 to 22 kernels, and on a 32^3 to 64^3 grid each kernel fills a few SMs for a few microseconds, so the GPU idles
 * between launches however many streams run beside each other.  A group steps several contexts together.  Its
 * members fall into shape classes (stage-kernel form, Nx, Nz, periodic Ny); within a class every kernel family of the
 * step (stage kernel, div + forward x transform, z transforms, y solve or periodic-y transform, inverse x transform,
 * stage-3 correction, constant-flux sum and shift) is ONE launch for all the class's members, whose blocks find
 * their case in a job table and run the per-case kernel's code on it.  One group step is captured once as a CUDA
 * graph, each class (or each part of a class up to dfdm_group_set_branch_cells cells) on a branch of its own, so that
 * the branches' launches overlap.  A member's results do not depend on the other members: a case steps
 * bit-identically in a group of one and in any mix, on any stream.  Against k dfdm_compute_time_step_rk3 steps of
 * the same context they agree to FP32 rounding: the grouped kernels are a separate compilation of the per-case
 * kernels' source, whose scalar multiply-add contractions may differ.
 *  - Members: FP32-mixed contexts without SGS model, wall model or hybrid advection scheme, with the fused
 *    corrections on, a fixed time step (no adaptive step or landing target), two-level transform lengths
 *    (Nx/2, Nz and periodic Ny in {8,16,24,32,48,64,96,128,192,256}), Nx a multiple of 4, and a first step taken
 *    (dfdm_compute_time_step_rk3 after set_state; the group runs the steady step).  Else DFDM_ERR_UNSUPPORTED or
 *    DFDM_ERR_INVALID.  A context may belong to several groups; only one may step it at a time.
 *  - stream: where the group's work runs; NULL gives the group a non-blocking stream of its own (group_get_stream
 *    returns it; destroyed with the group).  group_step_async orders itself after the members' earlier work on
 *    their own streams and their later work after it, with events (no host wait), and advances each member's time
 *    by nsteps * dt.  group_synchronize waits for the group's stream.
 *  - Before its first step a group picks the tile shape of its grouped stage launches per branch: the z-chunk (the
 *    members' own chunking, the wave model's choice for the branch's tiles together, or one chunk per column) and
 *    whether one block runs per tile or resident blocks walk the tiles.  It times the candidates with stage-1
 *    launches (which write only F1 and u*, both rewritten by every step) and caches the choice per branch shape and
 *    member count.  Results do not depend on it.  dfdm_group_set_stage_tiles fixes it instead: kc > 0 planes per
 *    block (clipped to Nz), 0 each member's own; walk 1 for walking blocks; kc < 0 returns to the timed choice.
 *  - The members must outlive the group's enqueued steps; destroying the group does not wait for them (its graph is
 *    released when they are done) and leaves the members as they are. */
typedef struct dfdm_group dfdm_group;
int dfdm_group_create(dfdm_ctx *const *ctxs, int n, void *stream, dfdm_group **out);
int dfdm_group_step_async(dfdm_group *group, int nsteps);
int dfdm_group_synchronize(dfdm_group *group);
int dfdm_group_get_stream(dfdm_group *group, void **cuda_stream);
/* At most `cells` cells per graph branch (default 524288): a shape class with more splits into several branches of
 * consecutive members, which overlap on the device as the classes do (0: one branch per class).  Results do not
 * change.  The group's graph is recaptured at its next step. */
int dfdm_group_set_branch_cells(dfdm_group *group, long long cells);
int dfdm_group_set_stage_tiles(dfdm_group *group, int kc, int walk);
/* Number of the library's kernels the group has enqueued (graph replays included). */
int dfdm_group_launch_count(dfdm_group *group, long long *count);
int dfdm_group_destroy(dfdm_group *group);

#ifdef __cplusplus
}
#endif

#endif /* DFDM_H */
