/*
 * oracle.h -- FP64 CPU restatement of the EnricoDeg/compact_schemes hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path in
 * compact_schemes_b200; it is loaded by tests/, by __graft_entry__.smoke() and
 * by bench.py's cpu_baseline / reference arm, never by the product path.
 *
 * Every function names the reference file:line it restates (paths relative to
 * the reference project root).  Field layout is the reference's SoA layout:
 * q[v*lmx + idx], idx = i + lxi*(j + let*k), x fastest
 * (src/cuda/kernels/physics.hpp:55-100).
 *
 * Parity pins: or_deriv_setup is checked against the reference's own
 * numerics_base::deriv_setup compiled from its sources (oracle/Makefile, target ref);
 * or_fluxes_pre and or_time_step against the reference's CPU twins in
 * tests/test_physics_serial.cu:41-163 and tests/test_physics.cu:57-117
 * compiled the same way; or_deriv against the known-answer linear-field test
 * of tests/test_numerics_serial.cu:60-131.  RK update, thermodynamic recovery,
 * Taylor-Green initial state, GCBC (reference defects fixed) and the compact
 * filter have no working reference implementation: their parity is unpinned.
 */
#ifndef COMPACT_ORACLE_H
#define COMPACT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Metrics: either per-point arrays (xim/etm/zem: [3][lmx], yaco: [lmx]) or,
 * when an array pointer is NULL, the constant in c_* is used everywhere. */
typedef struct {
    const double *xim, *etm, *zem, *yaco;
    double c_xim[3], c_etm[3], c_zem[3], c_yaco;
} or_metrics;

/* numerics_base::deriv_setup (src/numerics_base.hpp:182-297). */
void or_deriv_setup(double pbco[16], double pbci[16]);

/* Interface sums of one face (fill_gpu_buffer_kernel,
 * src/cuda/kernels/numerics_pc.hpp:42-122): send[0..F) = sum pbco[i] f[istart+inc*i],
 * send[F..2F) = sum pbco[8+i] f[...], istart = face*(N-1), inc = 1-2*face. */
void or_fill_buffer(const double *in, double *send, int lxi, int let, int lze,
                    int axis, int face, const double *pbco);

/* Compact first derivative along `axis` in index space (build_system +
 * solve, src/cuda/kernels/numerics_device_pc.hpp:176-351), solved by Thomas.
 * nstart/nend = ndf of face 0 / face 1 (0: physical closure, 1: interface).
 * recv: per-variable receive buffer [4F] laid out as the reference uses it
 * (rows 0, 1, N-1, N-2); NULL means single-rank periodic self-exchange.
 * drva (nullable): [2][5][F]; rows 0 and N-1 stored at variable slot `var`.
 * Returns 0 or a negative error code. */
int or_deriv(const double *in, double *out, int lxi, int let, int lze, int axis,
             int nstart, int nend, const double *recv, double *drva, int var,
             const double *pbco, const double *pbci);

/* Same on a single line of N points (stride 1), for unit tests. */
int or_deriv_line(const double *f, double *x, int n, int nstart, int nend,
                  const double recv4[4], const double *pbco, const double *pbci);

/* Compact filter along `axis` (no reference implementation; see oracle.cpp). */
int or_filter(const double *in, double *out, int lxi, int let, int lze, int axis,
              int nstart, int nend, double alpha_f);
int or_filter_line(const double *f, double *x, int n, int nstart, int nend, double alpha_f);

/* calc_fluxes_pre_compute_kernel<Visc> (src/cuda/kernels/physics.hpp:42-193).
 * buffer: [5][3][n]; tau: [6][n] (xx,yy,zz,xy,yz,zx) and heat: [3][n], both
 * NULL for the inviscid form.  Writes de[4*n+i] = qa[4] + p as the reference. */
void or_fluxes_pre(double *buffer, const double *qa, const double *p, double *de,
                   const double *xim, const double *etm, const double *zem,
                   const double *tau, const double *heat, const double umf[3], int64_t n);

/* calc_time_step (src/physics_pc.hpp:229-256, kernel src/cuda/kernels/physics.hpp:335-427). */
double or_time_step(const double *xim, const double *etm, const double *zem,
                    const double *de, const double *yaco, const double *ssk,
                    const double umf[3], double cfl, int64_t n);
/* Same two maxima with constant metrics and constant ssk (mu). */
double or_time_step_m(const double *de, or_metrics m, double mu, const double umf[3],
                      double cfl, int64_t n);

/* Primitive recovery into the reference's de slots: de0 = 1/rho,
 * de1..3 = u,v,w, de4 = gamma*p/rho (c^2, the CANARD temperature), p. */
void or_thermo(const double *q, double *de, double *p, int64_t n);

/* Intended calc_viscous_shear_stress (src/physics_pc.hpp:151-227 with the
 * chain rule applied to the derivatives): de1..4 = u,v,w,T in, tau [6][n],
 * heat [3][n] out.  ndf[face][axis]. */
int or_viscous(const double *de, double mu, or_metrics m, int lxi, int let, int lze,
               const int ndf[2][3], const double *pbco, const double *pbci,
               double *tau, double *heat);

/* Full RHS de[m] = sum_a d/dxi_a F[m][a] from the conserved state q
 * (physics::calc_viscous_shear_stress then physics::calc_fluxes).
 * drva_x (nullable) receives the x-axis line-end derivatives [2][5][F]. */
int or_rhs(const double *q, double *rhs, double mu, or_metrics m, const double umf[3],
           int lxi, int let, int lze, const int ndf[2][3], int viscous, double *drva_x);

/* Same, also returning scale5[m] = max over points of sum_a |d_a F[m][a]|,
 * the magnitude of the terms the RHS sums (the scale of its rounding error). */
int or_rhs_scaled(const double *q, double *rhs, double mu, or_metrics m, const double umf[3],
                  int lxi, int let, int lze, const int ndf[2][3], int viscous, double *drva_x,
                  double *scale5);

/* GCBC non-reflective correction of rhs on the x faces
 * (gcbc_go / gcbc_setup_kernel / gcbc_update_non_reflective_kernel,
 * src/gcbc.hpp:86-186, src/cuda/kernels/gcbc.hpp:251-454) with the reference
 * defects fixed.  cm: [2][3][F] face normals, sbcc: [lmx]. */
/* Wall boundary state update (wall_condition_update, src/gcbc.hpp:188-228;
 * wall_inviscid_kernel / wall_viscous_kernel, src/cuda/kernels/gcbc.hpp:160-249)
 * on every face coded BC_WALL_INVISCID (20) or BC_WALL_VISCOUS (25): at the
 * face's points with npex == 0, inviscid: rho E = rho^gamma / (gamma (gamma-1))
 * + |m|^2 / (2 rho); viscous: m = -rho umf, rho E = rho / (gamma (gamma-1)) +
 * |m|^2 / (2 rho) with the updated m.  Face plane ip * (n - 1). */
int or_wall_update(double *q, const int *npex, const double umf[3], int lxi, int let, int lze,
                   const int nbc[6]);
int or_gcbc_x(double *rhs, const double *drva_x, const double *cm, const double *q,
              const double *yaco, const double *sbcc, double c_yaco, const double umf[3],
              int lxi, int let, int lze, const int nbc[2][3]);

/* One explicit RK step of nkrk=4 stages, q <- q^{n+1}; stage k uses
 * q^(k) = q^n - dt/(4-k) * J * rhs(q^(k-1)).  dt <= 0: computed from q^n by
 * the CFL formula with `cfl`.  gcbc != 0 applies or_gcbc_x each stage.
 * Returns the dt used (negative on error). */
double or_rk_step(double *q, double mu, or_metrics m, const double umf[3], int lxi, int let,
                  int lze, const int nbc[2][3], int viscous, double dt, double cfl, int gcbc);

/* One stage k of that step: qout = qn - dt/(4-k) * J * rhs(qin). */
double or_rk_stage(const double *qn, const double *qin, double *qout, int k, double dt, double mu,
                   or_metrics m, const double umf[3], int lxi, int let, int lze, const int nbc[2][3],
                   int viscous);

/* Metrics (xim, etm, zem: [3][n]) and Jacobian (yaco: [n]) of the grid with
 * coordinates xyz ([3][n]), cross-product form with compact derivatives;
 * period[a][c]: jump of coordinate c across axis a (axes with ndf = 1).
 * Returns 0, -1 on a bad size, -2 on a zero cell volume. */
int or_grid_metrics(const double *xyz, const double period[3][3], int lxi, int let, int lze,
                    const int ndf[2][3], double *xim, double *etm, double *zem, double *yaco);

/* gcbc_go (src/gcbc.hpp:86-186) on all faces of a single-rank block:
 * non-reflective (10), inviscid / viscous wall (20 / 25) and curvilinear
 * interface (30) faces; drva[a] ([2][5][F], in: line-end derivatives, out:
 * characteristic form), cm[a] ([2][3][F] unit normals), drvb[a] ([2][5][F],
 * out: the neighbour's characteristic values, here face 1-ip of the block
 * itself); de [5][n] updated on kMbci planes per face with weights sbcc [n].
 * Returns 0, -1 on a missing buffer. */
int or_gcbc_go(double *drva[3], const double *cm[3], double *drvb[3], const double *qa, double *de,
               const double *p, const double *yaco, const double *sbcc, const double umf[3],
               const double dudtmf[3], int lxi, int let, int lze, double dtwi, const int nbc[2][3]);

/* Taylor-Green initial state on a periodic [0,2pi)^3 grid (CANARD units:
 * rho0 = 1, c_inf = 1, p0 = 1/gamma), density noise amp*U(-1,1) from the
 * counter-based generator or_noise. */
void or_tgv_init(double *q, int lxi, int let, int lze, double mach, double noise_amp,
                 uint64_t seed);
double or_noise(uint64_t seed, uint64_t index);

/* The derivative-and-filter test field on the non-periodic unit cube
 * (x = i/(lxi-1), ...): f = sum_m A_m sin(2 pi (kx x + ky y + kz z) + phi_m)
 * over nmodes modes drawn from std::mt19937_64(seed), per mode in the order
 * A, kx, ky, kz, phi, each from u = (top 53 bits of one draw) * 2^-53:
 * A = 0.1 + 0.9 u, k = 1 + floor(8 u), phi = 2 pi u.  modes: [nmodes][5]
 * (A, kx, ky, kz, phi), may be NULL; f: [lxi*let*lze], may be NULL. */
void or_fourier_field(int lxi, int let, int lze, uint64_t seed, int nmodes, double *modes, double *f);

/* Solve every line bottom-up instead of top-down (same mathematics, other
 * rounding): the oracle against itself in this mode measures the FP64 noise
 * floor of a quantity. */
void or_set_reversed_solves(int on);

int or_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
