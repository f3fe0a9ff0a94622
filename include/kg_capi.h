/*
 * kg_capi.h -- C ABI of the B200 method-of-lines solver for the Klein-Gordon
 * field on a Kerr-Schild / Schwarzschild background in (r, theta, phi).
 *
 * Every entry point is a plain C function over plain pointers and sizes.  Each
 * replaces one type-bound procedure of the reference's Fortran objects
 * (FlavioRosales/KG), cited beside it, so a Fortran host binds it through
 * iso_c_binding and keeps its evolve loop unchanged.  The MPI slab
 * decomposition of the reference is replaced by whole-grid residency on one
 * GPU: the solver owns every state array in device memory, the ghost-zone,
 * pole-parity and outer-boundary fills run on the device, and send_recv_xL/xR
 * have no counterpart.
 *
 * Conventions
 *   - Grid integers follow the reference namelist: Nx radial cells, Ny theta
 *     points (theta has Ny-1 cells plus pole ghosts), Nz phi points (period
 *     Nz-1, one duplicated point), g_pts ghosts (must be 2).
 *   - Host state arrays use the reference layout u(1:5, -g:Nx+g, -g:Ny+g, 0:Nz)
 *     of complex(8): a flat array of 2*5*(Nx+2g+1)*(Ny+2g+1)*(Nz+1) doubles,
 *     (re, im) pairs, variable index fastest.
 *   - Every function returns KG_OK (0) or a positive KG_E* code; the text of
 *     the last error of a handle is kg_last_error(h).  Nothing aborts the host.
 *   - A handle is used by one host thread at a time; all its device work is
 *     ordered on one CUDA stream (kg_get_stream).
 */
#ifndef KG_CAPI_H
#define KG_CAPI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum kg_status {
  KG_OK = 0,
  KG_EINVAL = 1,     /* bad argument or parameter combination */
  KG_ENOMEM = 2,     /* device or host allocation failed */
  KG_ECUDA = 3,      /* a CUDA call failed (message in kg_last_error) */
  KG_ESTATE = 4,     /* call not valid in the handle's current state */
  KG_ETIMEOUT = 5,   /* a bounded device wait ran out */
  KG_ENODEV = 6      /* no usable sm_100 device */
};

enum kg_metric { KG_KERR_SCHILD = 0, KG_SCHW_EF = 1 };
enum kg_bc_rmax { KG_OUTFLOW = 0, KG_INFLOW = 1 };

/* Mirrors the reference namelist &input (main/global_numbers.f90:76-90) and
 * the arguments of scalar_field_constructor (MoL/diagnostic_lib.f90:40-42). */
typedef struct kg_params {
  int Nx, Ny, Nz, g_pts;
  double xmin, xmax, tmin, tmax, CFL;
  double a, M_bh, m;          /* spin, black-hole mass, field mass */
  int metric;                 /* enum kg_metric */
  int bc_rmax;                /* enum kg_bc_rmax */
  int n_det;                  /* detectors, >= 2 */
  int l_max;                  /* Y_lm order of the detector projection */
  double dt_override;         /* > 0 replaces the reference dt rule */
  double save_;               /* diagnostic cadence in time units (namelist save_) */
} kg_params;

typedef struct kg_solver kg_solver;

/* --- lifetime ---------------------------------------------------------- */

/* scalar_field_constructor (MoL/diagnostic_lib.f90:40-151) together with
 * mesh_refinement_boundary/create (MoL/mesh_refinement_lib.f90:100-147),
 * geometry_load_metric/inverse (MoL/geometry.f90:92-352) and the dt rule
 * (MoL/diagnostic_lib.f90:101-107).  Allocates all device state, builds the
 * metric tables and detector list, zeroes the state.  device < 0: current. */
int kg_create(const kg_params *p, int device, kg_solver **out);
/* no reference counterpart (the reference never deallocates) */
int kg_destroy(kg_solver *h);
/* text of the handle's last error; with h = NULL, of the calling thread's
 * last handle-less call */
const char *kg_last_error(const kg_solver *h);
/* scalars: dx, dy, dz, dt, t, xmin, xmax, Nt, r_max (9 doubles) */
int kg_get_scalars(const kg_solver *h, double *out9);
int kg_set_time(kg_solver *h, double t);
int kg_set_dt(kg_solver *h, double dt);
/* the CUDA stream (cudaStream_t) the handle orders its work on */
void *kg_get_stream(const kg_solver *h);
/* bytes of device memory held by the handle */
size_t kg_device_bytes(const kg_solver *h);
/* wait until the handle's queued device work has finished (the steppers and
 * diagnostics enqueue and return; the reference's calls were synchronous) */
int kg_synchronize(kg_solver *h);

/* --- state exchange (the Fortran host's MoL%u, MoL%u_stage, ...) -------- */

/* which: 0 = u, 1 = u_stage, 2 = u_stage_2, 3 = u_p.  Host arrays in the
 * Fortran layout above; the device keeps r-fastest planes per variable. */
int kg_set_state(kg_solver *h, int which, const double *host_u);
int kg_get_state(kg_solver *h, int which, double *host_u);
/* same, from / to a device buffer in the Fortran layout */
int kg_set_state_device(kg_solver *h, int which, const double *dev_u);
int kg_get_state_device(kg_solver *h, int which, double *dev_u);

/* --- time steppers (MoL/lines_method_lib.f90) ---------------------------- */

/* pirk2 (:271-332), nsteps consecutive calls.  For nsteps >= 2 the steps run
 * as replays of a CUDA graph of two steps, captured on first use */
int kg_pirk2(kg_solver *h, int nsteps);
/* pirk3 (:334-408) */
int kg_pirk3(kg_solver *h, int nsteps);
/* rk3 (:211-269) with rhs(1) = the type-bound rhs_* set applied to u */
int kg_rk3(kg_solver *h, int nsteps);
/* rk4 (:411-474) with the same rhs */
int kg_rk4(kg_solver *h, int nsteps);
/* Precision of kg_rk4 on this handle: 0 = FP64 throughout (the reference's
 * arithmetic, default); 1 = mixed: the stencil RHS in FP32 on FP32 stage states,
 * u^n and the update u^n + (k1 + 2k2 + 2k3 + k4)/6 in FP64, FP64 RHS on the
 * excision planes and next to the poles.  The other steppers stay FP64. */
int kg_set_precision(kg_solver *h, int mode);
int kg_get_precision(const kg_solver *h);
/* Method of kg_rk4: 0 = the reference's second-order scheme (default);
 * 1 = configured: fourth-order centred differences (the stencil of
 * first_derivative_x_4, tools/finite_differences.f90:124-154, with its one-sided
 * r closures), sixth-order Kreiss-Oliger dissipation of strength ko_eps, a
 * Sommerfeld condition on the outermost r plane and parity-correct pole ghosts
 * (psi_2 negated).  Kerr_Schild form, FP64, kg_rk4 only (other steppers return
 * KG_EINVAL while it is set). */
int kg_set_scheme(kg_solver *h, int scheme, double ko_eps);
int kg_get_scheme(const kg_solver *h);
/* the configured method's ghost fills applied to u (after a kg_set_state of
 * initial data that does not already satisfy them) */
int kg_fill_ghosts_cfg(kg_solver *h);
/* turn graph replay of multi-step calls on (default) or off */
int kg_set_graphs(kg_solver *h, int on);

/* --- RHS and boundaries (parity hooks) ----------------------------------- */

/* rhs_phi/psi1/psi2/psi3/pi (:671-753) evaluated on host vars (Fortran layout);
 * bit v of var_mask selects rhs variable v; unselected outputs are left as
 * passed in rhs_inout. */
int kg_rhs(kg_solver *h, const double *host_vars, double *host_rhs_inout, unsigned var_mask);
/* boundary_xL, xR, yL, yR, zL, zR (:507-597) on u, bits 0..5 in that order,
 * applied in that order; xR 'inflow' copies from u_p. */
int kg_boundary(kg_solver *h, unsigned face_mask);
/* send_recv_xL / send_recv_xR (:475-505): single domain, nothing to exchange */
int kg_send_recv(kg_solver *h);

/* --- geometry ------------------------------------------------------------- */

/* 2-D (r, theta) tables, each (Ny+2g+1) x (Nx+2g+1) doubles, r fastest, in the
 * order alpha, beta^r, d_r beta^r, sqrt(gamma), gamma^rr, gamma^rphi,
 * gamma^thth, gamma^phph (MoL/geometry.f90:273-352; phi-independent). */
int kg_get_metric(kg_solver *h, double *host_tables8);
/* replace the tables above (a host that built its own geometry) */
int kg_set_metric(kg_solver *h, const double *host_tables8);
/* validate_inverse_metric (MoL/geometry.f90:409-492): error counts of the
 * 4-metric and 3-metric identities at tolerance 1e-10 over the whole grid */
int kg_validate_inverse_metric(kg_solver *h, int *errors_4d, int *errors_3d);

/* --- diagnostics (MoL/diagnostic_lib.f90) --------------------------------- */

/* density (:277-289): rho from the current u, kept on the device */
int kg_density(kg_solver *h);
/* download rho ((Nz+1) x (Ny+2g+1) x (Nx+2g+1) doubles, r fastest) */
int kg_get_density(kg_solver *h, double *host_rho);
/* Mass_scalar = integrate(rho*sqrtg) (:214, tools/integral.f90:646-674) */
int kg_mass_scalar(kg_solver *h, double *out);
/* currents_ADM + currents_detectors (:219-229, :252-274): momentum(3, n_det),
 * component fastest; detectors outside the grid are left as passed */
int kg_currents_detectors(kg_solver *h, double *host_momentum);
/* proyector_detectors (:231-250): alm(l, m, d) complex, l fastest then m
 * (-l_max..l_max) then detector; detectors outside the grid are left as passed */
int kg_proyector_detectors(kg_solver *h, double *host_alm);
/* diagnostic(index) (:185-217): density is not recomputed (as in the
 * reference); every `save` steps currents and a_lm are refreshed on device. */
int kg_diagnostic(kg_solver *h, int index, double *mass_out);
/* replace the detector radii (the reference places them at MoL/diagnostic_lib.f90:124-134);
 * each radius is located on the vertex grid the same way (main/global_numbers.f90:152-164) */
int kg_set_detectors(kg_solver *h, int n, const double *radii);
/* check_point / read_from_check_point (MoL/lines_method_lib.f90:599-667), as a
 * complete binary file: a 128-byte header (magic "KGB2CKPT", version, grid
 * integers, metric, outer BC, scheme, precision, t, dt, ...), then u and, when
 * the handle has them, u_stage and u_stage_2, each complex(8)
 * u(1:5,-g:Nx+g,-g:Ny+g,0:Nz).  The stage arrays carry the previous step's Pi
 * that PIRK stage 1 reads, so loading into a handle of the same grid resumes
 * bit for bit (the reference's text checkpoint keeps u and t only, and its
 * reader deletes the file before opening it).  Load returns KG_EINVAL, with the
 * handle unchanged, when the file's grid, metric, outer BC, field mass, xmin,
 * xmax, scheme (and Kreiss-Oliger eps) or precision mode differ from the
 * handle's, or when the file is truncated; stage arrays the file lacks are
 * reset to a fresh handle's (zero, Pi slot 4). */
int kg_save_checkpoint(kg_solver *h, const char *path);
int kg_load_checkpoint(kg_solver *h, const char *path);
/* detector radii and vertex indices (1-based) */
int kg_get_detectors(kg_solver *h, double *r_det, int *index_det);
/* proyector_detectors applied at every vertex shell r(1..Nx) (tools/FFT_sph.f90:247-279
 * at all radii): alm(l, m, shell) complex, l fastest, m = -L..L, then shell.
 * precision 0: FP64 reduction per (l, m, shell); 1: the contraction as one GEMM
 * on the tensor cores (tcgen05), operands split into BF16 head + tail, three
 * passes hi.hi + hi.lo + lo.hi accumulated in FP32. */
int kg_project_all_shells(kg_solver *h, int L, int precision, double *host_alm);
/* generate_full_bessel_basis (tools/FFT_sph.f90:13-95): k_values(0:L, Nk) and the
 * normalised j_basis(0:L, Nk, Nx) on the vertex radii, Fortran order (l fastest);
 * either output may be NULL.  k_ln = (n-th zero of j_l) / r_max. */
int kg_bessel_basis(kg_solver *h, int L, int Nk, double *k_values, double *j_basis);
/* SphFT_discrete_radial (tools/FFT_sph.f90:213-244): ft(1:Nk, 0:L, -L:L) complex,
 * n fastest, = trapezium over the shells of flm(r) j_basis(l,n,r) r^2, with flm
 * the all-shell projection of phi (precision as kg_project_all_shells). */
int kg_sph_ft_radial(kg_solver *h, int L, int Nk, int precision, double *host_ft);
/* sph_harmonics (tools/FFT_sph.f90:282-336) on the vertex grid:
 * Ylm(l, m, j, k) complex, l fastest, m = -L..L, theta then phi */
int kg_sph_harmonics(kg_solver *h, int L, double *host_ylm);

/* --- instrumentation (no reference counterpart; the reference times its
 * evolve loop with MPI_Wtime, main/evolve.f90:7, main/save_gnuplot.f90:158) */

/* when on, every kernel launch of the handle is bracketed by CUDA events on
 * the handle's stream and its duration is accumulated per kernel kind */
int kg_profile_enable(kg_solver *h, int on);
/* accumulated milliseconds and launch counts per kernel kind (arrays of
 * kg_profile_kinds() entries); clears the accumulators */
int kg_profile_read(kg_solver *h, double *ms, long long *launches);
int kg_profile_kinds(void);
const char *kg_profile_kind_name(int kind);
/* total kernel launches issued by the handle since creation */
long long kg_launch_count(const kg_solver *h);
/* stage-kernel form: 3 (default) = marching kernels fed by a TMA shared-memory
 * ring, with PIRK stage 1 (pirk2 :278-289) fused into one kernel; 2 = the same
 * with PIRK stage 1 as two launches; 1 = 2.5-D marching kernels with register
 * prefetch; 0 = one thread per
 * point with cached neighbour loads.  All give bit-identical results, except
 * that forms 1-3 divide by sqrt(gamma) through a reciprocal product that can be
 * one unit off IEEE division for dividends below about 2^-1000 in magnitude
 * (form 0 divides outright).  The configured method
 * (kg_set_scheme) takes 0 for one thread per point and any other value for
 * its tiled form, which gives the same bits. */
int kg_set_kernel_variant(kg_solver *h, int variant);
/* theta rows of the TMA tiles of the RK4 stages (FP64 forms 2, 3 and the mixed
 * form): 8 (default; 32 x 8 tiles, 2 CTAs per SM) or 4 (32 x 4 tiles, 3 CTAs per
 * SM, twice the tiles per grid).  The same bits either way.  No reference
 * counterpart. */
int kg_set_tile_rows(kg_solver *h, int rows);
/* No reference counterpart (the reference stops on errors).  Exercises the
 * failure path every TMA-fed kernel takes when a bounded wait runs out, without
 * a fault: one warp waits, at most `polls` (1..2^20) polls, on an mbarrier phase
 * that nothing completes, sets the handle's device error flag and returns.  The
 * call returns KG_ETIMEOUT with the message of a stage launch whose copies never
 * landed, then clears the flag, so the handle and its context stay usable.  (A
 * flag already set by an earlier launch is reported and left set.) */
int kg_check_wait_timeout(kg_solver *h, long long polls);
int kg_get_tile_rows(const kg_solver *h);

/* --- batched engine ------------------------------------------------------------ */
/* No reference counterpart (the reference runs one solve per MPI job): many
 * independent solves, each a kg_solver handle with its own grid, field mass and
 * state, advanced together by RK4.  Each stage is ONE persistent launch over the
 * ragged work list of all members' tiles (TMA-fed kernels), followed by one
 * batched ghost fill; a whole step is captured once into a CUDA graph and
 * replayed.  Members keep their own handles for state exchange and diagnostics
 * (which wait for the batch).  All members share one metric kind. */
typedef struct kg_batch kg_batch;
int kg_batch_create(int device, kg_batch **out);
int kg_batch_destroy(kg_batch *b);
const char *kg_batch_last_error(const kg_batch *b);
int kg_batch_add(kg_batch *b, kg_solver *h);
int kg_batch_remove(kg_batch *b, kg_solver *h);
int kg_batch_size(const kg_batch *b);
/* rk4 (MoL/lines_method_lib.f90:411-474) for every member, nsteps times */
int kg_batch_rk4(kg_batch *b, int nsteps);
int kg_batch_synchronize(kg_batch *b);
/* launch shape: phi planes per work item and persistent CTAs (the tuner's knobs) */
int kg_batch_set_tuning(kg_batch *b, int kchunk, int blocks);
/* 0 = FP64 RK4 for every member (default), 1 = mixed precision as kg_set_precision */
int kg_batch_set_precision(kg_batch *b, int mode);
/* proyector_detectors (MoL/diagnostic_lib.f90:231-250) for every member at once,
 * ordered behind the batch's steps, one synchronisation: host_alm receives each
 * member's a_lm(0:L, -L:L, n_det) block (as kg_proyector_detectors writes it) in
 * member order. */
int kg_batch_proyector_detectors(kg_batch *b, double *host_alm);
/* complex values kg_batch_proyector_detectors writes (sum over members) */
long long kg_batch_alm_count(const kg_batch *b);
int kg_batch_get_tuning(const kg_batch *b, int *kchunk, int *blocks);
/* how kg_batch_rk4 runs the members: dispatch 0 = one persistent launch per RK4
 * stage over all members (default); 1 = each member's own single-solve kernels
 * on its own stream, all members concurrently, forked from and joined back into
 * the batch stream (the same bits as kg_rk4 on each member alone).  variant: in
 * dispatch 1 the members' stage-kernel form (kg_set_kernel_variant), -1 to keep
 * each member's own; the mixed form takes -1, 2 or 3.  The tuner's third and
 * fourth knobs. */
int kg_batch_set_dispatch(kg_batch *b, int dispatch, int variant);
int kg_batch_get_dispatch(const kg_batch *b, int *dispatch, int *variant);
/* theta rows of the TMA tiles (8 or 4, as kg_set_tile_rows): the persistent
 * launch's work items, and in dispatch 1 every member's RK4 stage kernels.  The
 * tuner's fifth knob. */
int kg_batch_set_tile_rows(kg_batch *b, int rows);
int kg_batch_get_tile_rows(const kg_batch *b, int *rows);
long long kg_batch_launch_count(const kg_batch *b);
void *kg_batch_get_stream(const kg_batch *b);

/* --- Berger-Oliger refinement ------------------------------------------------ */

/* A hierarchy of radially nested 2:1 levels (the reference's
 * mesh_refinement_memory/boundary/create, MoL/mesh_refinement_lib.f90:76-179,
 * build one uniform level; the nesting is new).  Level 0 is kg_create(base);
 * level l = 1..nlevels-1 covers [xmin, ~r_fine[l-1]] with dx_0 / 2^l and takes
 * dt_0 / 2^l steps, same theta/phi grid.  Per coarse RK4 step each finer level
 * steps twice per parent step; after every stage its 4 outermost planes take
 * the parent's values (cubic in r, linear in time between the parent's states
 * at its step's start and end); after its two steps it is injected onto the
 * parent except for its last 8 planes.  Levels are ordinary solver handles
 * (kg_hier_level) for state access and diagnostics; they belong to the
 * hierarchy (kg_hier_destroy frees them). */
typedef struct kg_hier kg_hier;
int kg_hier_create(const kg_params *base, int nlevels, const double *r_fine, int device, kg_hier **out);
int kg_hier_destroy(kg_hier *H);
const char *kg_hier_last_error(const kg_hier *H);
int kg_hier_levels(const kg_hier *H);
kg_solver *kg_hier_level(kg_hier *H, int level);
int kg_hier_rk4(kg_hier *H, int coarse_steps);
/* the same hierarchy stepped by SSP-RK3 (rk3, MoL/lines_method_lib.f90:211-269);
 * the stage inputs stand at t, t+dt and t+dt/2 for the buffer-plane times */
int kg_hier_rk3(kg_hier *H, int coarse_steps);
/* the same hierarchy stepped by PIRK2 / PIRK3 (pirk2, MoL/lines_method_lib.f90:271-332;
 * pirk3, :334-408).  u_stage stands at t+dt and u_stage_2 (PIRK3) at t+dt/2, so
 * their buffer planes take the parent's state at those times, Pi included; the
 * stale-Pi slot that stage 1 reads then holds, on the buffer planes, the
 * parent's Pi at the step's start. */
int kg_hier_pirk2(kg_hier *H, int coarse_steps);
int kg_hier_pirk3(kg_hier *H, int coarse_steps);
int kg_hier_synchronize(kg_hier *H);

/* --- allocation-free diagnostic --------------------------------------------- */

/* Mass_scalar = integrate(rho*sqrtg) without allocating anything.  No
 * counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc -- a host whose device memory belongs to its own pool or a fixed
 * budget already given to live solves, or one that must not take the
 * device-wide synchronisation of cudaMalloc / cudaFree inside its time loop.  The caller passes everything in its own device memory: rho as
 * (Nz+1) x (Ny+2g+1) x (Nx+2g+1) doubles (r fastest, ghosts included, g = 2),
 * sqrtg as (Ny+2g+1) x (Nx+2g+1), and one double for the result; the work is
 * enqueued on `stream` (a cudaStream_t, NULL for the default stream) and the
 * call returns without waiting.  Intermediate sums live in a static device
 * array of 2^19 doubles (4 MiB, held by every GPU that loads the library
 * until exit): a grid needing more than (Nx+1)*(Ny+1) + Nx+1 <= 2^19 is
 * rejected with KG_EINVAL, text in kg_last_error(NULL).  Calls share that
 * array, so calls that overlap on the GPU race.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress, with that device
 * current) and must come before any stream capture. */
int kg_integrate_mass_noalloc(const double *rho_dev, const double *sqrtg_dev, int Nx, int Ny, int Nz,
                              double dx, double dy, double dz, double *out_dev, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* KG_CAPI_H */
