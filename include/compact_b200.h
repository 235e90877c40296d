/*
 * compact_b200.h -- C ABI of compact_schemes_b200, a B200 (sm_100a)
 * implementation of the compact-scheme hot path of EnricoDeg/compact_schemes.
 *
 * Conventions
 *  - Fields are structure-of-arrays in device memory, q[v*lmx + idx] with
 *    idx = i + lxi*(j + let*k) (x fastest), exactly the reference layout
 *    (src/cuda/kernels/physics.hpp:55-100).  All pointers passed to compute
 *    entry points are device pointers unless the name says _host.
 *  - Every entry point returns an int status (CS_OK = 0, negative on error)
 *    instead of the reference's print-and-exit (src/cuda/check.hpp:36-41);
 *    cs_last_error() gives a message.
 *  - `stream` is a cudaStream_t passed as void*; 0 = legacy default stream.
 *    No entry point synchronizes the host unless documented.
 *  - The whole domain is one rank: the reference's MPI halo exchange
 *    (numerics_base::mpigo, src/numerics_base.hpp:119-180) becomes a local
 *    copy for faces whose neighbour is the block itself (periodic).
 *
 * Each declaration cites the reference interface it replaces (file:line,
 * relative to the reference project root).
 */
#ifndef COMPACT_B200_H
#define COMPACT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CS_OK 0
#define CS_ERR_INVALID (-1)     /* bad argument (dims, pointer, axis, size) */
#define CS_ERR_CUDA (-2)        /* CUDA runtime error */
#define CS_ERR_UNSUPPORTED (-3) /* line too long/short for the kernels */
#define CS_ERR_ALLOC (-4)       /* device allocation failed */
#define CS_ERR_STATE (-5)       /* call order (e.g. deriv before deriv_setup) */
#define CS_ERR_TIMEOUT (-6)     /* a bounded device-side wait ran out; that call's results are invalid */

/* Boundary codes, src/common/parameters.hpp:46-52. */
#define CS_BC_NON_REFLECTIVE 10
#define CS_BC_WALL_INVISCID 20
#define CS_BC_WALL_VISCOUS 25
#define CS_BC_INTER_CURV 30
#define CS_BC_INTER_STRAIGHT 35
#define CS_BC_INTER_SUBDOMAINS 40
#define CS_BC_PERIODIC 45

/* Halo source for interface (ndf = 1) faces of a derivative. */
#define CS_HALO_RECV 0 /* read the numerics object's recv buffer (reference data flow) */
#define CS_HALO_SELF 1 /* single-rank periodic: sums taken in-kernel from the line's far end */

/* t_dcomp, src/common/data_types.hpp:33-39 (point counts). */
typedef struct {
    int lmx;
    int lxi;
    int let;
    int lze;
} cs_dcomp;

const char *cs_last_error(void);
int cs_version(void);

/* ---------------------------------------------------------------------------
 * numerics: compact derivative / filter line solves
 * ------------------------------------------------------------------------- */
typedef struct cs_numerics cs_numerics;

/* numerics_base<T>(t_dcomp, int nbc[2][3]) (src/numerics_base.hpp:43-93):
 * allocates drva/send/recv scratch per axis and derives ndf per face. */
int cs_numerics_create(cs_numerics **out, cs_dcomp d, const int nbc[2][3]);
/* ~numerics_base (src/numerics_base.hpp:96-112). */
int cs_numerics_destroy(cs_numerics *nm);
/* numerics_base::deriv_setup (src/numerics_base.hpp:182-297): interface
 * weights pbco/pbci (copied to the device) and the line-solver tables. */
int cs_deriv_setup(cs_numerics *nm);
/* The same weights computed on the host without a numerics object (no device
 * needed), bit-identical to the reference's deriv_setup. */
int cs_interface_coeffs(double pbco[16], double pbci[16]);
/* Host copies of pbco/pbci (16 each). */
int cs_get_coeffs(const cs_numerics *nm, double pbco[16], double pbci[16]);
/* ndf[face][axis] as in numerics_base::ndf (src/numerics_base.hpp:73-93). */
int cs_get_ndf(const cs_numerics *nm, int ndf[2][3]);
/* Device scratch owned by the object (numerics_base::drva_buffer,
 * send_buffer, recv_buffer, src/numerics_base.hpp:389-395):
 * drva [2][5][F], send/recv [5][2][2][F] for the given axis (F = face size). */
int cs_get_buffers(cs_numerics *nm, int axis, double **drva, double **send, double **recv);

/* numerics_pc::deriv1d / deriv2d (src/numerics_pc.hpp:74-168): compact first
 * derivative along `axis` in index space of in[comp*lmx + .] into
 * out[slot*lmx + .] (deriv1d: comp = slot = 0; deriv2d: slot = axis).
 * nstart/nend: ndf of face 0 / 1.  Line-end values go to drva[axis] at
 * variable `var`.  halo: CS_HALO_RECV or CS_HALO_SELF.  FP64. */
int cs_deriv(cs_numerics *nm, int axis, const double *in, double *out, int nstart, int nend,
             cs_dcomp d, unsigned var, unsigned comp, unsigned slot, int halo, void *stream);
/* The derivative of cs_deriv (FP64, deriv1d semantics: in and out are single
 * fields) for callers that cannot let a library allocate device memory, e.g.
 * applications that give all device memory to their own pool at start-up or
 * that must not have cudaMalloc/cudaFree synchronize the device mid-loop.
 * No counterpart in the reference.  It needs no numerics object and calls no
 * allocation routine: its line-solver tables live in a file-scope device
 * array of 64000 bytes (lines of at most 1024 points; longer lines return
 * CS_ERR_UNSUPPORTED) that every GPU loading the library holds until exit.
 * Interface faces (nstart/nend = 1) use the single-rank periodic closure; no
 * line-end values are stored.  The first call on a device looks the array's
 * address up (cudaGetSymbolAddress) and should come before any stream
 * capture.  With CUDA's lazy module loading (the default), that first call,
 * and the first call for each chunk length (lines up to 64, 128, 256, 512,
 * 1024 points), may also load the kernel's module, which can allocate and
 * synchronize inside the CUDA runtime: make a warm-up call with each line
 * length before the loop that must not allocate (or set
 * CUDA_MODULE_LOADING=EAGER).  All calls share the array and each rewrites
 * it: calls that may overlap on the GPU (different streams, no ordering)
 * race; calls on one stream are ordered. */
int cs_deriv_noalloc(int axis, const double *in, double *out, int nstart, int nend, cs_dcomp d,
                     void *stream);
/* Same for numerics_pc<float>: FP32 data and arithmetic. */
int cs_deriv_f32(cs_numerics *nm, int axis, const float *in, float *out, int nstart, int nend,
                 cs_dcomp d, unsigned var, unsigned comp, unsigned slot, int halo, void *stream);

/* numerics_pc::fill_buffers<m0,m1> (src/numerics_pc.hpp:231-287) with
 * gpu_buffer::fill / fill_gpu_buffer_kernel (src/cuda/kernels/numerics_pc.hpp:42-122):
 * pbco-weighted interface sums of variables [var_lo, var_hi) of the
 * [5][3][lmx] field block `in` into the send buffers.  nrt as the reference. */
int cs_fill_buffers(cs_numerics *nm, const double *in, int var_lo, int var_hi, int nrt,
                    cs_dcomp d, void *stream);
/* Single-rank numerics_base::mpigo (src/numerics_base.hpp:119-180): for every
 * axis whose two faces are interface faces (ndf = 1) the block is its own
 * neighbour; recv of face 0 <- send of face 1 and vice versa, variable var. */
int cs_halo_exchange_self(cs_numerics *nm, unsigned var, void *stream);

/* Compact filter along `axis` (no reference implementation: the sixth-order
 * tridiagonal filter of Gaitonde & Visbal, AIAA J. 38 (2000)).  ndf faces of the
 * axis both 1: cyclic; both 0: reduced-order boundary closure. */
int cs_filter(cs_numerics *nm, int axis, const double *in, double *out, double alpha_f,
              cs_dcomp d, void *stream);

/* Introspection of the line-solver tables (tests, autotuner): fills meta =
 * {n, lt, p, last_len, cyclic, pcr64, pcr32} (pcr*: PCR steps the FP64 / FP32
 * solves run) and, if tables != NULL, the 6*lt*32 + 13*64 + lt*32 doubles
 * fwd1,fwd2,bwd1,bwd2,rca,rcc,k1,k2,invb (FP64 depth),cycz,{s1,s2}.
 * scheme 0 = derivative (nstart/nend), 1 = filter (alpha_f). */
int cs_line_tables(int n, int scheme, int nstart, int nend, double alpha_f, int meta[7],
                   double *tables, size_t tables_len);

/* ---------------------------------------------------------------------------
 * physics: the reference-shaped (unfused) path with per-point metric arrays
 * ------------------------------------------------------------------------- */
typedef struct cs_physics cs_physics;

/* physics<EnableViscous, T>(t_dcomp) (src/physics_pc.hpp:62-72,
 * src/physics_base.hpp:45-89): owns buffer / buffer_deriv [5][3][lmx],
 * stress tensor [6][lmx] (xx, yy, zz, xy, yz, zx) and heat flux [3][lmx]. */
int cs_physics_create(cs_physics **out, cs_dcomp d, int viscous);
int cs_physics_destroy(cs_physics *ph);
/* physics_base::umf (src/physics_base.hpp:155). */
int cs_physics_set_umf(cs_physics *ph, const double umf[3]);
/* Device pointers of the object's buffers (any may be NULL). */
int cs_physics_buffers(cs_physics *ph, double **buffer, double **buffer_deriv, double **tau,
                       double **heat);
/* calc_fluxes_pre_compute (src/cuda/physics.hpp:41-62): the 15 contravariant
 * fluxes into buffer, de[4] <- qa[4] + p.  de[1..3] hold u, v, w. */
int cs_calc_fluxes_pre(cs_physics *ph, const double *qa, const double *p, double *de,
                       const double *xim, const double *etm, const double *zem, void *stream);
/* physics::calc_fluxes (src/physics_pc.hpp:83-149): pre-compute, interface
 * sums and single-rank halo exchange, 15 compact derivatives,
 * de[m] = sum_a d/dxi_a F[m][a].  Uses the numerics object's scratch. */
int cs_calc_fluxes(cs_physics *ph, cs_numerics *nm, const double *qa, const double *p, double *de,
                   const double *xim, const double *etm, const double *zem, cs_dcomp d,
                   void *stream);
/* physics::calc_viscous_shear_stress (src/physics_pc.hpp:151-227): gradients
 * of de[1..4] = (u, v, w, T) by compact derivatives, chain rule through the
 * metrics, stress tensor and energy flux into the object's buffers; like the
 * reference it leaves de[0] = ssk and de[4] = 2/3 div u. */
int cs_calc_viscous_shear_stress(cs_physics *ph, cs_numerics *nm, double *de, const double *ssk,
                                 const double *xim, const double *etm, const double *zem,
                                 const double *yaco, cs_dcomp d, void *stream);
/* physics::calc_time_step (src/physics_pc.hpp:229-256): the CFL and viscous
 * maxima on the device, dte = min(cfl / max1, 0.5 / max2) on the host
 * (synchronizes the stream). */
int cs_calc_time_step(cs_physics *ph, const double *xim, const double *etm, const double *zem,
                      const double *de, const double *yaco, const double *ssk, double cfl,
                      double *dte, size_t size, void *stream);
/* Primitive recovery for the slot the reference driver leaves empty
 * (driver/canard.cu:142-143): de0 = 1/rho, de1..3 = u, v, w,
 * de4 = gamma p / rho (T in CANARD units, rho_inf = c_inf = 1), p. */
int cs_thermo(const double *q, double *de, double *p, size_t n, void *stream);
/* Metrics and Jacobian of a curvilinear grid, the arrays the flux kernels
 * read (xim, etm, zem = J^-1 grad(xi_a), yaco = J;
 * src/cuda/kernels/physics.hpp:42-193), which the reference's grid class does
 * not generate (grid::generate, src/grid.hpp:89-213, makes coordinates only).
 * Cross-product form with the compact derivative of nm (its closures):
 * xim = r_eta x r_zeta, etm = r_zeta x r_xi, zem = r_xi x r_eta,
 * yaco = 1 / (r_xi . xim).  xyz: [3][lmx] device coordinates; period[a][c]
 * (nullable): the jump of coordinate c across axis a, used on axes whose ndf
 * is 1 (r_a = D(c - i_a period/n_a) + period/n_a).  Outputs are device
 * arrays [3][lmx] (xim, etm, zem) and [lmx] (yaco).  Needs cs_deriv_setup;
 * overwrites nm's drva variable 0; allocates 10 lmx doubles for the call
 * (stream-ordered) and synchronizes the stream.  CS_ERR_INVALID on a cell of
 * zero volume. */
int cs_grid_metrics(cs_numerics *nm, const double *xyz, const double period[3][3], double *xim,
                    double *etm, double *zem, double *yaco, void *stream);

/* Wall boundary state update, wall_condition_update (src/gcbc.hpp:188-228):
 * on every face coded CS_BC_WALL_INVISCID or CS_BC_WALL_VISCOUS, at the face
 * points with npex == 0 (npex: [lmx] int mask), inviscid: the isentropic total
 * energy rho^gamma / (gamma (gamma-1)) + |m|^2 / (2 rho); viscous: m = -rho umf
 * and the isothermal energy rho / (gamma (gamma-1)) + |m|^2 / (2 rho).  The
 * face plane is index ip * (n - 1) along the axis. */
int cs_wall_condition_update(double *q, const int *npex, const double umf[3], cs_dcomp d, const int nbc[2][3],
                             void *stream);
/* The update physics_base::movef leaves empty (src/physics_base.hpp:147-150):
 * qout = qn - dtk * yaco * de (dtk = dt / (4 - k) for stage k). */
int cs_rk_update(const double *qn, const double *de, const double *yaco, double dtk, double *qout,
                 size_t n, void *stream);
/* gcbc_go (src/gcbc.hpp:86-186) with the reference's parameters, every face
 * code of a single-rank block: non-reflective, inviscid / viscous wall and
 * curvilinear-interface (GCIC) faces.  drva[a] ([2][5][F], the last
 * derivatives' line-end values of axis a, e.g. a numerics object's drva
 * buffers) is turned into characteristic form in place (gcbc_setup_kernel,
 * src/cuda/kernels/gcbc.hpp:251-342: from drva on non-reflective faces, from
 * the full J de elsewhere); for curvilinear-interface faces drvb[a] face ip
 * receives drva[a] face 1-ip (the block is its own neighbour; the MPI
 * exchange of src/gcbc.hpp:132-157, mcd unused); then de += sbcc * xtr2q *
 * (cha - drva) on the first 4 planes of every such face (update kernels,
 * :344-695).  cm[a]: [2][3][F] unit face normals; umf / dudtmf: frame
 * velocity / acceleration; dtwi: 1/dt, the wall's relaxation rate.  Faces
 * coded periodic or interface are skipped.  Reference defects fixed: the
 * xtq2r typos, the accumulating output index, the plane of face 1 (dim-1),
 * the thread part of the face index, and the wall update's missing
 * subtraction of drva. */
int cs_gcbc_apply(double *const drva[3], double *const cm[3], double *const drvb[3], const double *qa, double *de,
                  const double *p, const double *yaco, const double *sbcc, const double umf[3],
                  const double dudtmf[3], cs_dcomp d, double dtwi, const int nbc[2][3], const int mcd[2][3],
                  void *stream);
/* gcbc_go (src/gcbc.hpp:86-186) for non-reflective faces: characteristic
 * projection of the numerics object's drva, incoming acoustic waves removed,
 * de += sbcc * correction on the first 4 planes.  Faces coded periodic or
 * interface are skipped; wall and curvilinear-interface codes return
 * CS_ERR_UNSUPPORTED.  cm[axis]: [2][3][F] face normals. */
int cs_gcbc_go(cs_numerics *nm, double *const cm[3], const double *qa, double *de, const double *p,
               const double *yaco, const double *sbcc, const double umf[3], cs_dcomp d,
               const int nbc[2][3], void *stream);

/* ---------------------------------------------------------------------------
 * solver: fused RHS + RK stage on a uniform Cartesian grid
 *
 * Replaces, for one block held as a single rank, the per-stage sequence of
 * the reference driver (driver/canard.cu:132-224): calc_time_step
 * (src/physics_pc.hpp:229-256), calc_viscous_shear_stress (:151-227),
 * calc_fluxes (:83-149), gcbc_go for non-reflective faces
 * (src/gcbc.hpp:86-186) and the conserved-variable update that movef leaves
 * empty (src/physics_base.hpp:147-150):
 *     q^(k) = q^n - dt/(4-k) * J * de(q^(k-1)),  k = 0..3.
 * Metrics are those of the uniform grid: xim = (dy dz, 0, 0),
 * etm = (0, dx dz, 0), zem = (0, 0, dx dy), yaco = 1/(dx dy dz).
 * ------------------------------------------------------------------------- */
typedef struct cs_solver cs_solver;

#define CS_PREC_FP64 0  /* plain FP64 */
#define CS_PREC_MIXED 1 /* FP32 fluxes and line solves (FP64 right-hand sides, refinement
                           as cfg.refine), FP64 state, RK accumulation and thermodynamics */
#define CS_PREC_MIXED_F32 2 /* as CS_PREC_MIXED, with FP32 arithmetic in the interior: fluxes
                               evaluated in FP32, interior right-hand sides in FP32 (closure
                               rows in FP64) and per-row solver factors as constants, on every
                               axis whose lines have uniform chunk factors (interface or periodic
                               closure, length a multiple of the chunk); cfg.refine adds the
                               FP64-residual sweep of the FP32 right-hand side; other axes run
                               as CS_PREC_MIXED */

#define CS_REFINE_NONE 0 /* mixed: no refinement sweep */
#define CS_REFINE_ALL 1  /* mixed: a refinement sweep after every FP32 line solve */
#define CS_REFINE_FLUX 2 /* mixed: refinement in the flux passes only; the gradients feed the
                            state only through the viscous terms */

#define CS_SCHED_AUTO 0     /* the measured-faster schedule: one-phase on B200 */
#define CS_SCHED_ONEPHASE 1 /* each CTA loads a tile, solves it, stores it (tile[][] applies) */
#define CS_SCHED_PIPELINE 2 /* persistent CTAs: memory warps store tile k-1 and stage tile k+1
                               while solver warps solve tile k; error where the tiles do not fit */
#define CS_FILTER_NONE 0  /* no filter in the time step */
#define CS_FILTER_STEP 1  /* the compact filter along x, y, z on the state after every RK step */
#define CS_FILTER_STAGE 2 /* the same after every RK stage (FP64 only) */

#define CS_SCHED_TMA 3      /* gradient passes: persistent CTAs whose pencils of the state are
                               staged into shared memory by TMA two tiles ahead (FP64: lines of
                               up to 512 points, even row lengths; mixed: the FP32 shadow of every
                               gradient pass but a step's first, lines of up to 512 points, row
                               lengths and points a multiple of 4; else one-phase); flux passes
                               one-phase */

typedef struct {
    int lxi, let, lze;  /* points per axis */
    int nbc[2][3];      /* boundary code per face / axis (both faces of an axis periodic or both physical) */
    int viscous;        /* physics<EnableViscous, T> */
    double mu;          /* ssk: dynamic viscosity (constant) */
    double umf[3];      /* physics_base::umf, moving-frame velocity */
    double dx, dy, dz;  /* grid spacing */
    double cfl;         /* CFL number when the time step is computed */
    int gcbc;           /* apply non-reflective GCBC on x faces coded CS_BC_NON_REFLECTIVE */
    int use_graph;      /* cs_solver_step replays a captured CUDA graph of the step */
    int tile[2][3];     /* lines per tile of the [gradient|flux] pass along each axis:
                           8, or 16 for y/z; 0 = default (16 for the z flux pass, else 8);
                           tiles that do not fit shared memory fall back to 8; the mixed
                           form uses 8 for y */
    int precision;      /* CS_PREC_FP64 or CS_PREC_MIXED */
    int refine;         /* mixed: CS_REFINE_ALL one FP64-residual refinement sweep per line
                           solve, CS_REFINE_NONE none, CS_REFINE_FLUX in the flux passes only */
    int schedule;       /* CS_SCHED_*: how a pass overlaps its line solves with its HBM traffic */
    int filter;         /* CS_FILTER_*: the compact filter of cs_filter applied to the conserved
                           state inside the time step (all five fields, x then y then z) */
    double alpha_f;     /* filter parameter, -0.5 < alpha_f <= 0.5 (cs_filter's) */
} cs_solver_config;

int cs_solver_create(cs_solver **out, const cs_solver_config *cfg);
int cs_solver_destroy(cs_solver *s);
/* RHS de[m] = sum_a d/dxi_a F[m][a] of state q (physics::calc_viscous_shear_stress
 * then physics::calc_fluxes, src/physics_pc.hpp:83-227), into rhs [5][lmx]. */
int cs_solver_rhs(cs_solver *s, const double *q, double *rhs, void *stream);
/* One RK stage k (0..3) with a given dt: qout = qn - dt/(4-k) J de(qin). */
int cs_solver_stage(cs_solver *s, int k, const double *qn, const double *qin, double *qout,
                    double dt, void *stream);
/* One full RK step in place on the device state q [5][lmx]; dt <= 0 computes
 * dt from q^n with the CFL formula of calc_time_step.  No host sync. */
int cs_solver_step(cs_solver *s, double *q, double dt, void *stream);
/* Same with host buffers: copies q_in_host [5][lmx] to a solver-owned device
 * state, steps, copies the result to q_out_host and synchronizes the stream
 * (pinned host memory makes the copies asynchronous DMA). */
int cs_solver_step_host(cs_solver *s, const double *q_in_host, double *q_out_host, double dt,
                        void *stream);
/* dt used by the last step (synchronizing device-to-host copy). */
int cs_solver_last_dt(cs_solver *s, double *dt);
/* Device address of that dt (for stream-ordered readers). */
int cs_solver_dt_device(cs_solver *s, double **dt_dev);
/* Per-pass device timing of the eager step path (a graph step is not
 * profiled): between begin and end every pass is bracketed by CUDA events on
 * its stream; end synchronizes and returns the summed milliseconds and launch
 * counts per pass kind: 0-2 gradient x/y/z, 3-5 flux x/y/z (z carries the RK
 * update), 6 GCBC, 7 filter (one launch per axis). */
#define CS_PASS_KINDS 8
/* Autotuner: times `reps` eager steps of every feasible pass schedule (one-
 * phase with 8- or 16-line tiles, pipelined) on a scratch copy of q (q is not
 * modified) and keeps the fastest per pass; choice[kind][axis] (may be NULL)
 * receives 8 or 16 (one-phase tile lines), 0 (pipelined) or 1 (TMA-staged,
 * gradient passes) for the gradient (kind 0) and flux (kind 1) passes.
 * Synchronizes. */
int cs_solver_autotune(cs_solver *s, const double *q, int reps, int choice[2][3], void *stream);
/* The schedule each pass runs now, coded as cs_solver_autotune's choice. */
int cs_solver_schedule(const cs_solver *s, int choice[2][3]);
/* Per-point metrics for the fused solver: device arrays xim, etm, zem
 * ([3][lmx], J^-1 grad(xi_a)) and yaco ([lmx], J), as cs_grid_metrics
 * writes them, read by every later step, stage and RHS call instead of the
 * uniform grid of dx, dy, dz (the arrays must outlive that use; all four null
 * returns to the uniform grid).  FP64 only; the passes run the one-phase
 * kernels (CS_ERR_UNSUPPORTED for CS_PREC_MIXED or pipelined passes; the
 * autotuner then picks among the one-phase tiles).  With GCBC the face normal
 * and J are those of each face point. */
int cs_solver_set_metrics(cs_solver *s, const double *xim, const double *etm, const double *zem,
                          const double *yaco);
int cs_solver_profile_begin(cs_solver *s);
int cs_solver_profile_end(cs_solver *s, double ms[CS_PASS_KINDS], int launches[CS_PASS_KINDS]);
/* Taylor-Green initial state on a periodic [0,2pi)^3 grid in CANARD units
 * (no reference implementation: physics::init is empty, src/physics_pc.hpp:78-81). */
int cs_tgv_init(double *q, int lxi, int let, int lze, double mach, double noise_amp,
                uint64_t seed, void *stream);

/* ---------------------------------------------------------------------------
 * Batched ensemble: independent boxes of uneven sizes advanced together.
 * No reference counterpart (the reference advances one block per rank,
 * driver/canard.cu:132-224); each box is a cs_solver_config (FP64, uniform
 * grid, no GCBC; every axis 8..256 points).  One persistent launch per RK
 * stage pulls tiles of lines of all boxes from a device work queue ordered so
 * that each box's gradient, x-, y- and z-flux phases follow the phase they
 * depend on; a step (4 stages) replays one captured CUDA graph.  Per box the
 * arithmetic is that of cs_solver_step with a CFL time step: a box whose axes
 * all have more than 64 points gives bit for bit the result of its own
 * cs_solver; lines of up to 64 points are solved in 4-point chunks (two
 * fields per half-warp) where cs_solver uses 2-point chunks, which agrees
 * with it to rounding (1e-12 relative per field).
 * The state of all boxes is one packed device array: box b's q [5][lmx_b]
 * starts at cs_ensemble_box_offset(b).  At most 96 boxes per ensemble; the
 * stage kernel reads the box table from constant memory that every ensemble
 * of a device shares, so ensembles on one device step one at a time (steps
 * issued on one stream, or synchronized between streams).
 * ------------------------------------------------------------------------- */
typedef struct cs_ensemble cs_ensemble;

typedef struct {
    int window;      /* queue lag: phase p of the box of size rank r is queued at slot r + p * window
                        (0 = number of boxes: every box's gradients first, then x fluxes, ...) */
    int tile;        /* lines per work item: 4 or 8 */
    int ctas_per_sm; /* resident CTAs per SM of the persistent grid; 0 = as many as fit */
    int chunk;       /* tiles per work item taken from the queue: 1..64 */
} cs_ensemble_tuning;

int cs_ensemble_create(cs_ensemble **out, int nbox, const cs_solver_config *boxes);
int cs_ensemble_destroy(cs_ensemble *e);
/* Length in doubles of the packed state, and the offset of box b in it. */
int cs_ensemble_state_size(const cs_ensemble *e, int64_t *n_doubles);
int cs_ensemble_box_offset(const cs_ensemble *e, int box, int64_t *offset);
/* One RK step of every box, in place on the packed device state q; dt per box
 * from the CFL formula of calc_time_step on that box.  No host sync. */
int cs_ensemble_step(cs_ensemble *e, double *q, void *stream);
/* dt of every box in the last step (synchronizes); CS_ERR_TIMEOUT if a
 * dependency wait of the work queue ran out since the previous check. */
int cs_ensemble_last_dt(cs_ensemble *e, double *dt_host);
int cs_ensemble_set_tuning(cs_ensemble *e, const cs_ensemble_tuning *t);
/* Failure-detection hook of the stage kernel's dependency wait: a wait gives
 * up after poll_limit polls of about 100 ns (default 2e7), records the work
 * item in the error word, skips the item and lets the launch finish, and
 * cs_ensemble_last_dt returns CS_ERR_TIMEOUT (the step's state is then
 * invalid).  extra > 0 makes every wait need `extra` more finished items than
 * the queue can produce, so every dependent item times out: a test of that
 * path that faults nothing.  (default_polls, 0) restores the default. */
#define CS_ENSEMBLE_DEFAULT_POLLS 20000000LL
int cs_ensemble_set_wait(cs_ensemble *e, long long poll_limit, int extra);
int cs_ensemble_get_tuning(const cs_ensemble *e, cs_ensemble_tuning *t);
/* Autotuner: times `reps` steps of every candidate tuning (tile width x tiles
 * per work item x queue lag) on a scratch copy of q (q is not modified),
 * keeps the fastest and returns it with its milliseconds per step.
 * Synchronizes. */
int cs_ensemble_autotune(cs_ensemble *e, const double *q, int reps, cs_ensemble_tuning *best, double *best_ms,
                         void *stream);

/* ---------------------------------------------------------------------------
 * Tangent-linear and adjoint of the RHS and of the RK step (no reference
 * counterpart).  For a cs_solver_config (FP64, lines of at most 512 points;
 * with gcbc set, the non-reflective x-face correction is linearized too),
 * with dt held fixed:
 *   R'(q) dq    = sum_a D_a [dF_a/dq dq + dF_a/dG dG],   dG_b = D_b (dphi/dq dq)
 *   R'(q)^T l   = dF/dq^T mu + dphi/dq^T sum_b D_b^T (dF/dG^T mu)_b,   mu_a = D_a^T l
 * where D_a = A^-1 B is the compact derivative along axis a (its transpose is
 * a solve with A^T followed by B^T), F_a the flux of calc_fluxes_pre_compute
 * (src/cuda/kernels/physics.hpp:42-193) and phi = (u, v, w, T).
 * All arrays are device [nf][lmx] fields unless named _host.
 * ------------------------------------------------------------------------- */
typedef struct cs_adjoint cs_adjoint;

int cs_adjoint_create(cs_adjoint **out, const cs_solver_config *cfg);
int cs_adjoint_destroy(cs_adjoint *a);
/* out[f] (= or +=) D_axis in[f] (transpose = 0) or D_axis^T in[f], f < nfields. */
int cs_adjoint_deriv(cs_adjoint *a, int axis, int transpose, const double *in, double *out, int nfields,
                     int accumulate, void *stream);
/* out[f] (= or +=) F_axis in[f] or F_axis^T in[f] for the compact filter of
 * cs_filter (same alpha_f, the configuration's boundary codes). */
int cs_adjoint_filter(cs_adjoint *a, int axis, int transpose, double alpha_f, const double *in, double *out,
                      int nfields, int accumulate, void *stream);
int cs_rhs_jvp(cs_adjoint *a, const double *q, const double *dq, double *dR, void *stream);
int cs_rhs_vjp(cs_adjoint *a, const double *q, const double *lam, double *out, void *stream);
/* Stage states of one step with time step dt: stages[0] = q^n (copied unless
 * stages[0] == qn), stages[k] = q^(k-1) for k = 1..3; q_next = q^(n+1) (may be null). */
int cs_adjoint_stages(cs_adjoint *a, const double *qn, double dt, double *const stages[4], double *q_next,
                      void *stream);
/* Tangent / adjoint of one RK step about the stage states of cs_adjoint_stages. */
int cs_step_jvp(cs_adjoint *a, const double *const stages[4], double dt, const double *dq_n, double *dq_next,
                void *stream);
int cs_step_vjp(cs_adjoint *a, const double *const stages[4], double dt, const double *lam_next, double *lam_n,
                void *stream);
/* J = 1/2 sum (m.m)/rho dx dy dz (synchronizes when J_host is set) and dJ/dq (may be null). */
int cs_kinetic_energy(cs_adjoint *a, const double *q, double *J_host, double *dJdq, void *stream);
/* dJ/dq0 of J = kinetic energy after nsteps steps with time steps dt_host[s]:
 * forward sweep keeping a checkpoint every `every` steps, then a reverse sweep
 * that recomputes each segment's stage states from its checkpoint and applies
 * cs_step_vjp step by step.  Synchronizes.  The sweep buffer
 * (cs_adjoint_gradient_bytes) stays allocated for later calls until
 * cs_adjoint_destroy. */
int cs_adjoint_gradient(cs_adjoint *a, const double *q0, int nsteps, const double *dt_host, int every,
                        double *grad_q0, double *J_host, void *stream);
/* Device bytes cs_adjoint_gradient allocates for its sweeps (checkpoints,
 * running state, one segment's stage states, two adjoint states). */
int cs_adjoint_gradient_bytes(const cs_adjoint *a, int nsteps, int every, size_t *bytes);
/* Host-side pointwise linearizations (no device memory): the flux F_axis(q, G)
 * with G[b*4 + c] = d(phi_c)/d(xi_b), metrics M (row-major 3x3), Jacobian J,
 * viscosity mu, frame velocity umf; and the primitives phi(q). */
int cs_point_flux(int axis, int viscous, const double q[5], const double G[12], const double M[9], double J,
                  double mu, const double umf[3], double F[5]);
int cs_point_flux_jvp(int axis, int viscous, const double q[5], const double G[12], const double dq[5],
                      const double dG[12], const double M[9], double J, double mu, const double umf[3], double dF[5]);
int cs_point_flux_vjp(int axis, int viscous, const double q[5], const double G[12], const double Fbar[5],
                      const double M[9], double J, double mu, const double umf[3], double qbar[5], double Gbar[12]);
int cs_point_prim(const double q[5], double phi[4]);
int cs_point_prim_jvp(const double q[5], const double dq[5], double dphi[4]);
int cs_point_prim_vjp(const double q[5], const double phibar[4], double qbar[5]);

/* Headless VTK output (io::go_vtk, src/IO.hpp:108-159): legacy binary
 * STRUCTURED_GRID of lxi*let*lze points; data = [nvars][points] host floats,
 * variables 0..2 the point coordinates, variables 3.. named by names[v-3]. */
int cs_vtk_write(const char *path, int lxi, int let, int lze, const float *data, int nvars,
                 const char *const *names);

#ifdef __cplusplus
}
#endif
#endif
