// fused_kernels.cuh -- device code of the fused RHS / RK-stage passes and
// their launch templates (instantiated per axis in fused_axis{0,1,2}.cu).
#pragma once

#include <cuda.h>

#include <cmath>

#include "context.h"
#include "tile.cuh"

// Tuning knobs (compile-time; defaults chosen by measurement on B200):
// points per thread loaded together in the load phase of the gradient / flux
// passes, points per thread in the store phase, minimum resident CTAs
// (register cap) and the number of fields solved together by one warp.
#ifndef CSB_GRAD_UNROLL
#define CSB_GRAD_UNROLL 2
#endif
#ifndef CSB_FLUX_UNROLL
#define CSB_FLUX_UNROLL 2
#endif
#ifndef CSB_STORE_UNROLL
#define CSB_STORE_UNROLL 2
#endif
#ifndef CSB_GRAD_MINB
#define CSB_GRAD_MINB 2
#endif
#ifndef CSB_FLUX_MINB
#define CSB_FLUX_MINB 2
#endif
#ifndef CSB_SOLVE_GROUP
#define CSB_SOLVE_GROUP 2
#endif
#ifndef CSB_GRAD_SOLVE_GROUP
#define CSB_GRAD_SOLVE_GROUP CSB_SOLVE_GROUP
#endif
#ifndef CSB_RMW_CHUNK
#define CSB_RMW_CHUNK 4     // points per chunk when only R is read back
#endif
#ifndef CSB_RMW_CHUNK_RK
#define CSB_RMW_CHUNK_RK 2  // points per chunk when R and q^n are read (RK pass)
#endif

namespace csb {

// L2 prefetch of one box of a tensor map (cp.async.bulk.prefetch.tensor: a
// hint with nothing to wait for; the map covers this GPU's memory only).
__device__ __forceinline__ void tma_prefetch_3d(const CUtensorMap *map, int c0, int c1, int c2) {
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(c0), "r"(c1), "r"(c2)
                 : "memory");
}
__device__ __forceinline__ void tma_prefetch_4d(const CUtensorMap *map, int c0, int c1, int c2, int c3) {
    asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(c0), "r"(c1), "r"(c2), "r"(c3)
                 : "memory");
}

// Geometry of the L2 prefetch of a flux pass's read-modify-write inputs: the
// tile's lines of the RHS accumulator R and, in the RK modes, of q^n, as boxes
// of TL lines by boxlen points along the line by five fields.
struct FluxPrefetch {
    int on;      // 0: no prefetch (the maps are not valid)
    int nbox;    // boxes along the line (1 or 2)
    int boxlen;  // points per box along the line
    int lxi;     // points per x row (y tiles)
};

// Issue the prefetch boxes of the tile starting at line line0 (one thread).
template <int AXIS>
__device__ __forceinline__ void prefetch_tile(const CUtensorMap *map, const FluxPrefetch &pf, int64_t line0) {
    for (int b = 0; b < pf.nbox; ++b) {
        if (AXIS == 0) tma_prefetch_3d(map, b * pf.boxlen, (int)line0, 0);
        else if (AXIS == 1) tma_prefetch_4d(map, (int)(line0 % pf.lxi), b * pf.boxlen, (int)(line0 / pf.lxi), 0);
        else tma_prefetch_3d(map, (int)line0, b * pf.boxlen, 0);
    }
}

struct Phys {
    double M[3][3];  // metric rows xim, etm, zem (J^-1 grad xi_a)
    double J;        // yaco
    double mu;       // ssk (dynamic viscosity, constant)
    double umf[3];   // moving-frame velocity
    double rr1;      // sum of squared metric entries
};

// Per-point metrics of a curvilinear grid (xim, etm, zem: [3][lmx], yaco:
// [lmx]; the arrays calc_fluxes_pre_compute_kernel reads,
// src/cuda/kernels/physics.hpp:42-193).  Kernels compiled with FM = true read
// them; the others use the constants of Phys.
struct FieldMet {
    const double *xim = nullptr, *etm = nullptr, *zem = nullptr, *yaco = nullptr;
};

// Metric rows and Jacobian at one point.
struct PointMet {
    double M[3][3];
    double J;
};
template <bool FM>
__device__ __forceinline__ PointMet point_met(const Phys &ph, const FieldMet &fm, int64_t lmx, int64_t gi) {
    PointMet m;
    if (FM) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            m.M[0][k] = __ldg(fm.xim + k * lmx + gi);
            m.M[1][k] = __ldg(fm.etm + k * lmx + gi);
            m.M[2][k] = __ldg(fm.zem + k * lmx + gi);
        }
        m.J = __ldg(fm.yaco + gi);
    } else {
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
            for (int k = 0; k < 3; ++k) m.M[b][k] = ph.M[b][k];
        m.J = ph.J;
    }
    return m;
}

struct RkParams {
    double div;        // nkrk - k: stage coefficient dt / (nkrk - k)
    double dt_fixed;   // > 0: use it; else CFL dt from dtacc
    double cfl;
    const unsigned long long *dtacc;  // two maxima as bit patterns of non-negative doubles
    double *dt_out;
};

// CG: the maxima were reduced earlier in the same launch by other CTAs, so
// they are read from L2 (ld.global.cg) rather than through a possibly stale L1.
template <bool CG = false>
__device__ __forceinline__ double rk_dt(const RkParams &rk) {
    if (rk.dt_fixed > 0.0) return rk.dt_fixed;
    const double m1 = __longlong_as_double((long long)(CG ? __ldcg(rk.dtacc) : rk.dtacc[0]));
    const double m2 = __longlong_as_double((long long)(CG ? __ldcg(rk.dtacc + 1) : rk.dtacc[1]));
    const double a = rk.cfl / m1, b = 0.5 / m2;
    return a < b ? a : b;
}

// Primitive variables from the conserved state (CANARD units: T stored as
// c^2 = gamma p / rho).
struct Prim {
    double rho, ri, u, v, w, p, T;
};
__device__ __forceinline__ Prim primitives(double q0, double q1, double q2, double q3, double q4) {
    Prim s;
    s.rho = q0;
    s.ri = 1.0 / q0;
    s.u = xmul(q1, s.ri);
    s.v = xmul(q2, s.ri);
    s.w = xmul(q3, s.ri);
    s.p = xmul(kGamm1, q4 - xmul(0.5, xmul(q1, s.u) + xmul(q2, s.v) + xmul(q3, s.w)));
    s.T = xmul(xmul(kGam, s.p), s.ri);
    return s;
}

template <int LT, int TL>
__device__ __forceinline__ double *field_line(double *sm, int field, int line) {
    return sm + (field * TL + line) * LineLayout<LT>::kSlot;
}

// Solve fields c0 .. c0+G-1 (those below NF) of this warp's line held in
// shared memory and overwrite them with the result, in one warp_solve call
// (their table loads and shuffles are interleaved).  ROWS: the single-rank
// periodic closure rows of the group are formed on 8 lanes per line
// (group_closure_rows) instead of serially by the owner lanes; bit-identical
// either way.
template <int LT, int TL, int NF, int G, bool ROWS>
__device__ __forceinline__ void solve_field_group(double *sm, int w, int lane, const DevTables<double> &tab,
                                                  int nstart, int nend, const Coeffs &cf, int c0);

// solve_field_group for an even G on a line of at most 16 chunks whose solve
// needs at most 5 PCR steps: each half-warp solves G/2 of the fields (lanes
// 16 s + c hold chunk c of fields c0 + s G/2 + g), so every shuffle and table
// factor of the solve serves two fields at once.  The closure rows are formed
// as in solve_field_group (8 lanes per field line) and the arithmetic of each
// row is the same: bit-identical to it.
template <int LT, int TL, int NF, int G>
__device__ __forceinline__ void solve_field_group_halves(double *sm, int w, int lane, const DevTables<double> &tab,
                                                         int nstart, int nend, const Coeffs &cf, int c0) {
    constexpr int H = G / 2;
    const int s = lane >> 4, c = lane & 15;
    double *lines[G];
#pragma unroll
    for (int g = 0; g < G; ++g) lines[g] = field_line<LT, TL>(sm, c0 + g < NF ? c0 + g : c0, w);
    const bool sums = nstart != 0 || nend != 0;
    const double rows = sums ? group_closure_rows<LT, double, double, G>(lines, NF - c0, tab.n, lane, cf) : 0.0;
    double d[H][LT];
#pragma unroll
    for (int g = 0; g < H; ++g) {
        const int gg = s * H + g;
        double own2[2];
        if (sums) {
            const int src = 8 * gg + (c == 0 ? 0 : 4);
            own2[0] = __shfl_sync(0xffffffffu, rows, src);
            own2[1] = __shfl_sync(0xffffffffu, rows, src + 1);
        }
        const double *line = field_line<LT, TL>(sm, c0 + gg < NF ? c0 + gg : c0, w);
        if (c0 + gg < NF) deriv_rhs<LT, double, double>(line, tab.n, c, nstart, nend, nullptr, cf, d[g],
                                                        sums ? own2 : nullptr);
        else {
#pragma unroll
            for (int t = 0; t < LT; ++t) d[g][t] = 0.0;
        }
    }
    warp_solve<LT, H, double, 16>(tab, d, c);
    __syncwarp();
#pragma unroll
    for (int g = 0; g < H; ++g) {
        const int gg = s * H + g;
        if (c0 + gg >= NF) continue;
        double *line = field_line<LT, TL>(sm, c0 + gg, w);
#pragma unroll
        for (int t = 0; t < LT; ++t)
            if (c * LT + t < tab.n) line[LineLayout<LT>::pos_ct(c, t)] = d[g][t];
    }
}

template <int LT, int TL, int NF, int G, bool ROWS>
__device__ __forceinline__ void solve_field_group(double *sm, int w, int lane, const DevTables<double> &tab,
                                                  int nstart, int nend, const Coeffs &cf, int c0) {
    if constexpr (ROWS && G % 2 == 0) {
        if (tab.p <= 16 && tab.pcr <= 5) {
            solve_field_group_halves<LT, TL, NF, G>(sm, w, lane, tab, nstart, nend, cf, c0);
            return;
        }
    }
    double d[G][LT];
    double *lines[G];
#pragma unroll
    for (int g = 0; g < G; ++g) lines[g] = field_line<LT, TL>(sm, c0 + g < NF ? c0 + g : c0, w);
    const bool sums = ROWS && (nstart != 0 || nend != 0);
    const double rows = sums ? group_closure_rows<LT, double, double, G>(lines, NF - c0, tab.n, lane, cf) : 0.0;
#pragma unroll
    for (int g = 0; g < G; ++g) {
        double own2[2];
        if (sums) take_closure_rows(rows, g, lane, own2);
        if (c0 + g < NF) deriv_rhs<LT, double, double>(lines[g], tab.n, lane, nstart, nend, nullptr, cf, d[g],
                                                       sums ? own2 : nullptr);
        else {
#pragma unroll
            for (int t = 0; t < LT; ++t) d[g][t] = 0.0;
        }
    }
    warp_solve<LT, G, double>(tab, d, lane);
    __syncwarp();
#pragma unroll
    for (int g = 0; g < G; ++g) {
        if (c0 + g >= NF) continue;
        double *line = field_line<LT, TL>(sm, c0 + g, w);
#pragma unroll
        for (int t = 0; t < LT; ++t)
            if (lane * LT + t < tab.n) line[LineLayout<LT>::pos_ct(lane, t)] = d[g][t];
    }
}

// Solve the derivative of NF fields of this warp's line, G fields per
// warp_solve call (solve_field_group).  With ROWS a last group of fewer than
// G fields is solved as a group of its own size; without, it is padded with
// zero right-hand sides (measured: the one-phase FP64 passes keep the serial
// closure form and the padded group).
template <int LT, int TL, int NF, int G = CSB_SOLVE_GROUP, bool ROWS = false>
__device__ __forceinline__ void solve_fields(double *sm, int w, int lane, const DevTables<double> &tab,
                                             int nstart, int nend, const Coeffs &cf) {
    constexpr int REM = ROWS ? NF % G : 0;
    constexpr int NFULL = NF - REM;
#pragma unroll 1
    for (int c0 = 0; c0 < NFULL; c0 += G) solve_field_group<LT, TL, NF, G, ROWS>(sm, w, lane, tab, nstart, nend, cf, c0);
    if constexpr (REM > 0) solve_field_group<LT, TL, NF, REM, ROWS>(sm, w, lane, tab, nstart, nend, cf, NFULL);
}

// One tile of the gradient pass: lines line0 .. line0+TL-1 (TL * 32 threads;
// sm holds 4 * TL line slots).  SG: fields per warp solve (0: the pass
// default); ROWS: periodic closure rows formed lane-parallel (solve_fields).
template <int LT, int AXIS, int TL, bool DTRED, bool FM = false, int SG = 0, bool ROWS = false>
__device__ __forceinline__ void grad_tile(double *sm, int64_t line0, const double *__restrict__ q,
                                          double *__restrict__ g, const DevTables<double> &tab, int lxi, int let,
                                          int64_t lmx, int64_t F, int nstart, int nend, const Coeffs &cf,
                                          const Phys &ph, unsigned long long *__restrict__ dtacc,
                                          const FieldMet &fm = FieldMet{}) {
    using L = LineLayout<LT>;
    const int n = tab.n;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double m1 = 0.0, m2 = 0.0;
    tile_for_each<AXIS, TL, CSB_GRAD_UNROLL>(line0, F, n, lxi, let, [&](int l, int j, int64_t gi) {
        const Prim s = primitives(__ldg(q + gi), __ldg(q + lmx + gi), __ldg(q + 2 * lmx + gi),
                                  __ldg(q + 3 * lmx + gi), __ldg(q + 4 * lmx + gi));
        const int pj = L::pos(j);
        field_line<LT, TL>(sm, 0, l)[pj] = s.u;
        field_line<LT, TL>(sm, 1, l)[pj] = s.v;
        field_line<LT, TL>(sm, 2, l)[pj] = s.w;
        field_line<LT, TL>(sm, 3, l)[pj] = s.T;
        if (DTRED) {
            // calc_time_step_kernel (src/cuda/kernels/physics.hpp:335-427)
            const double uu = s.u + ph.umf[0], vv = s.v + ph.umf[1], ww = s.w + ph.umf[2];
            const PointMet pm = point_met<FM>(ph, fm, lmx, gi);
            double rr1 = ph.rr1;
            if (FM) {
                rr1 = 0.0;
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int c = 0; c < 3; ++c) rr1 += xmul(pm.M[a][c], pm.M[a][c]);
            }
            double rr2 = 0.0;
#pragma unroll
            for (int a = 0; a < 3; ++a)
                rr2 += fabs(xmul(pm.M[a][0], uu) + xmul(pm.M[a][1], vv) + xmul(pm.M[a][2], ww));
            const double ssi = fabs(pm.J);
            const double v1 = xmul(sqrt(xmul(s.T, rr1)) + rr2, ssi);
            const double v2 = s.ri * ph.mu * rr1 * ssi * ssi;
            m1 = fmax(m1, v1);
            m2 = fmax(m2, v2);
        }
    });
    tile_sync<AXIS, TL>();
    const int64_t fidx = line0 + w;
    if (fidx < F)
        solve_fields<LT, TL, 4, (SG > 0 ? SG : (LT >= 16 ? 1 : CSB_GRAD_SOLVE_GROUP)), ROWS>(sm, w, lane, tab, nstart,
                                                                                         nend, cf);
    tile_sync<AXIS, TL>();
    tile_for_each<AXIS, TL, CSB_STORE_UNROLL>(line0, F, n, lxi, let, [&](int l, int j, int64_t gi) {
        const int pj = L::pos(j);
#pragma unroll
        for (int c = 0; c < 4; ++c) g[c * lmx + gi] = field_line<LT, TL>(sm, c, l)[pj];
    });
    if (DTRED) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
            m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
        }
        if (lane == 0) {
            atomicMax(dtacc, (unsigned long long)__double_as_longlong(m1));
            atomicMax(dtacc + 1, (unsigned long long)__double_as_longlong(m2));
        }
    }
}

// ----------------------------------------------------------------------------
// gradient pass: G[AXIS][c] = d/dxi_AXIS of (u, v, w, T)
// ----------------------------------------------------------------------------
template <int LT, int AXIS, int TL, bool DTRED, bool FM = false>
__global__ void __launch_bounds__(TL * 32, TL == 8 ? CSB_GRAD_MINB : 1)
k_grad(const double *__restrict__ q, double *__restrict__ g, DevTables<double> tab, int lxi, int let,
       int64_t lmx, int64_t F, int nstart, int nend, Coeffs cf, Phys ph,
       unsigned long long *__restrict__ dtacc, FieldMet fm) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    grad_tile<LT, AXIS, TL, DTRED, FM>(reinterpret_cast<double *>(smem_raw), (int64_t)blockIdx.x * TL, q, g, tab,
                                       lxi, let, lmx, F, nstart, nend, cf, ph, dtacc, fm);
}

// ----------------------------------------------------------------------------
// flux pass
// ----------------------------------------------------------------------------
enum FluxMode { kWrite = 0, kAccum = 1, kAccumRk = 2, kWriteRk = 3 };

// Flux components F[m][AXIS] at one point from the state and the gradients
// (calc_fluxes_pre_compute_kernel<Visc>, src/cuda/kernels/physics.hpp:42-193,
// with tau / heat flux of calc_viscous_shear_stress_final_kernel, :285-333),
// from the point's values: state q0..q4, gradients gr[12] (G[b][c] at
// 4 b + c) and metrics pm.  DIAG: the metric matrix is diagonal (the uniform
// Cartesian grid, M[b][k] = 0 for b != k), and the products with its zero
// entries are left out: each sum then adds the same nonzero terms in the same
// order, so the result equals the full evaluation's (up to the sign of an
// exactly zero value).
template <int AXIS, bool VISC, bool DIAG = false>
__device__ __forceinline__ void flux_values(double q0, double q1, double q2, double q3, double q4,
                                            const double (&gr)[12], const PointMet &pm, const Phys &ph,
                                            double (&fl)[5]) {
    const Prim s = primitives(q0, q1, q2, q3, q4);
    const double *Ma = pm.M[AXIS];
    const double vel[3] = {s.u, s.v, s.w};
    double ss;
    if (DIAG) ss = xmul(Ma[AXIS], vel[AXIS] + ph.umf[AXIS]);
    else ss = xmul(Ma[0], s.u + ph.umf[0]) + xmul(Ma[1], s.v + ph.umf[1]) + xmul(Ma[2], s.w + ph.umf[2]);
    fl[0] = xmul(q0, ss);
    if (DIAG) {
        fl[1] = xmul(q1, ss);
        fl[2] = xmul(q2, ss);
        fl[3] = xmul(q3, ss);
        fl[1 + AXIS] += xmul(Ma[AXIS], s.p);
        fl[4] = xmul(q4 + s.p, ss) - xmul(s.p, xmul(ph.umf[AXIS], Ma[AXIS]));
    } else {
        fl[1] = xmul(q1, ss) + xmul(Ma[0], s.p);
        fl[2] = xmul(q2, ss) + xmul(Ma[1], s.p);
        fl[3] = xmul(q3, ss) + xmul(Ma[2], s.p);
        fl[4] = xmul(q4 + s.p, ss) -
                xmul(s.p, xmul(ph.umf[0], Ma[0]) + xmul(ph.umf[1], Ma[1]) + xmul(ph.umf[2], Ma[2]));
    }
    if (VISC) {
        // physical gradients without the J factor: dc/dx_k = sum_b M[b][k] G[b][c]
        double dx[4][3];
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int k = 0; k < 3; ++k)
                dx[c][k] = DIAG ? xmul(pm.M[k][k], gr[4 * k + c])
                                : xmul(pm.M[0][k], gr[c]) + xmul(pm.M[1][k], gr[4 + c]) + xmul(pm.M[2][k], gr[8 + c]);
        const double muj = xmul(ph.mu, pm.J);
        const double kap = xmul(kGamm1Prndtli, muj);
        const double div = xmul(2.0 / 3.0, dx[0][0] + dx[1][1] + dx[2][2]);
        const double txx = xmul(muj, xmul(2.0, dx[0][0]) - div);
        const double tyy = xmul(muj, xmul(2.0, dx[1][1]) - div);
        const double tzz = xmul(muj, xmul(2.0, dx[2][2]) - div);
        const double txy = xmul(muj, dx[1][0] + dx[0][1]);
        const double tyz = xmul(muj, dx[2][1] + dx[1][2]);
        const double tzx = xmul(muj, dx[0][2] + dx[2][0]);
        // rows of the stress tensor: t[k] = (tau_kx, tau_ky, tau_kz)
        const double t[3][3] = {{txx, txy, tzx}, {txy, tyy, tyz}, {tzx, tyz, tzz}};
        if (DIAG) {
            // only the AXIS column of tau and the AXIS component of h are needed
            const double hA = xmul(kap, dx[3][AXIS]) + xmul(s.u, t[0][AXIS]) + xmul(s.v, t[1][AXIS]) +
                              xmul(s.w, t[2][AXIS]);
            fl[1] -= xmul(Ma[AXIS], t[0][AXIS]);
            fl[2] -= xmul(Ma[AXIS], t[1][AXIS]);
            fl[3] -= xmul(Ma[AXIS], t[2][AXIS]);
            fl[4] -= xmul(Ma[AXIS], hA);
        } else {
            const double hx = xmul(kap, dx[3][0]) + xmul(s.u, txx) + xmul(s.v, txy) + xmul(s.w, tzx);
            const double hy = xmul(kap, dx[3][1]) + xmul(s.u, txy) + xmul(s.v, tyy) + xmul(s.w, tyz);
            const double hz = xmul(kap, dx[3][2]) + xmul(s.u, tzx) + xmul(s.v, tyz) + xmul(s.w, tzz);
            fl[1] -= xmul(Ma[0], txx) + xmul(Ma[1], txy) + xmul(Ma[2], tzx);
            fl[2] -= xmul(Ma[0], txy) + xmul(Ma[1], tyy) + xmul(Ma[2], tyz);
            fl[3] -= xmul(Ma[0], tzx) + xmul(Ma[1], tyz) + xmul(Ma[2], tzz);
            fl[4] -= xmul(Ma[0], hx) + xmul(Ma[1], hy) + xmul(Ma[2], hz);
        }
    }
}

// The same loading the point's values from HBM.  CG: the gradients were
// written earlier in the same launch by other CTAs (ensemble launch) and are
// read from L2 (ld.global.cg).
template <int AXIS, bool VISC, bool CG = false, bool FM = false>
__device__ __forceinline__ void point_flux(const double *__restrict__ q, const double *__restrict__ g,
                                           int64_t lmx, int64_t gi, const Phys &ph, double (&fl)[5],
                                           const FieldMet &fm = FieldMet{}) {
    const double q0 = __ldg(q + gi), q1 = __ldg(q + lmx + gi), q2 = __ldg(q + 2 * lmx + gi);
    const double q3 = __ldg(q + 3 * lmx + gi), q4 = __ldg(q + 4 * lmx + gi);
    double gr[12];
    if (VISC) {
#pragma unroll
        for (int k = 0; k < 12; ++k) gr[k] = CG ? __ldcg(g + k * lmx + gi) : __ldg(g + k * lmx + gi);
    }
    const PointMet pm = point_met<FM>(ph, fm, lmx, gi);
    // the uniform grid of Phys is Cartesian: its metric matrix is diagonal
    flux_values<AXIS, VISC, !FM>(q0, q1, q2, q3, q4, gr, pm, ph, fl);
}

// One tile of the flux pass (TL * 32 threads; sm holds 5 * TL line slots).
// CG: the RHS accumulator, gradients and CFL maxima come from other CTAs of
// the same launch (ensemble) and are read from L2.  SG, ROWS: as grad_tile.
template <int LT, int AXIS, int TL, int MODE, bool VISC, bool CG = false,
          int P = MODE == kAccum ? (LT >= 16 ? 2 : CSB_RMW_CHUNK) : (LT >= 16 ? 1 : CSB_RMW_CHUNK_RK),
          bool FM = false, int SG = 0, bool ROWS = false>
__device__ __forceinline__ void flux_tile(double *sm, int64_t line0, const double *__restrict__ q,
                                          const double *__restrict__ g, double *__restrict__ rhs,
                                          const double *__restrict__ qn, double *__restrict__ qout,
                                          double *__restrict__ drva, const DevTables<double> &tab, int lxi, int let,
                                          int64_t lmx, int64_t F, int nstart, int nend, const Coeffs &cf,
                                          const Phys &ph, const RkParams &rk, const FieldMet &fm = FieldMet{}) {
    using L = LineLayout<LT>;
    const int n = tab.n;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // per-point metrics add 10 loads per point: one point per thread in flight
    tile_for_each<AXIS, TL, FM ? 1 : CSB_FLUX_UNROLL>(line0, F, n, lxi, let, [&](int l, int j, int64_t gi) {
        double fl[5];
        point_flux<AXIS, VISC, CG, FM>(q, g, lmx, gi, ph, fl, fm);
        const int pj = L::pos(j);
#pragma unroll
        for (int m = 0; m < 5; ++m) field_line<LT, TL>(sm, m, l)[pj] = fl[m];
    });
    tile_sync<AXIS, TL>();
    const int64_t fidx = line0 + w;
    if (fidx < F) {
        solve_fields<LT, TL, 5, (SG > 0 ? SG : (LT >= 16 ? 1 : CSB_SOLVE_GROUP)), ROWS>(sm, w, lane, tab, nstart, nend,
                                                                                    cf);
        if (drva) {
            // line-end derivatives for the characteristic boundary closure
            // (drva of deriv_kernel_2d, src/cuda/kernels/numerics_pc.hpp:237-248)
            __syncwarp();
            if (lane < 10) {
                const int m = lane % 5, face = lane / 5;
                drva[(int64_t)(face * 5 + m) * F + fidx] = field_line<LT, TL>(sm, m, w)[L::pos(face ? n - 1 : 0)];
            }
        }
    }
    tile_sync<AXIS, TL>();
    double dtk = 0.0, dtd = 0.0;
    if (MODE >= kAccumRk) {
        const double dt = rk_dt<CG>(rk);
        dtd = dt / rk.div;
        dtk = xmul(dtd, ph.J);
        if (rk.dt_out && line0 == 0 && threadIdx.x == 0) *rk.dt_out = dt;
    }
    if (MODE == kWrite) {
        tile_for_each<AXIS, TL, CSB_STORE_UNROLL>(line0, F, n, lxi, let, [&](int l, int j, int64_t gi) {
            const int pj = L::pos(j);
#pragma unroll
            for (int m = 0; m < 5; ++m) rhs[m * lmx + gi] = field_line<LT, TL>(sm, m, l)[pj];
        });
    } else {
        // read-modify-write: all loads of a chunk of P points first
        double rv[P][5], qv[P][5], jv[P];
        tile_for_each_chunked<AXIS, TL, P>(
            line0, F, n, lxi, let,
            [&](int p, int l, int j, int64_t gi) {
                if (FM && MODE >= kAccumRk) jv[p] = xmul(dtd, __ldg(fm.yaco + gi));
#pragma unroll
                for (int m = 0; m < 5; ++m) {
                    rv[p][m] = MODE == kWriteRk ? 0.0 : (CG ? __ldcg(rhs + m * lmx + gi) : rhs[m * lmx + gi]);
                    if (MODE >= kAccumRk) qv[p][m] = qn[m * lmx + gi];
                }
            },
            [&](int p, int l, int j, int64_t gi) {
                const int pj = L::pos(j);
#pragma unroll
                for (int m = 0; m < 5; ++m) {
                    const double dfv = field_line<LT, TL>(sm, m, l)[pj];
                    if (MODE == kAccum) {
                        rhs[m * lmx + gi] = rv[p][m] + dfv;
                    } else {
                        const double r = MODE == kAccumRk ? rv[p][m] + dfv : dfv;
                        qout[m * lmx + gi] = qv[p][m] - xmul(FM ? jv[p] : dtk, r);
                    }
                }
            });
    }
}

template <int LT, int AXIS, int TL, int MODE, bool VISC, bool FM = false>
__global__ void __launch_bounds__(TL * 32, TL == 8 ? CSB_FLUX_MINB : 1)
k_flux(const double *__restrict__ q, const double *__restrict__ g, double *__restrict__ rhs,
       const double *__restrict__ qn, double *__restrict__ qout, double *__restrict__ drva,
       DevTables<double> tab, int lxi, int let, int64_t lmx, int64_t F, int nstart, int nend,
       Coeffs cf, Phys ph, RkParams rk, FieldMet fm) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int P = MODE == kAccum ? (LT >= 16 ? 2 : CSB_RMW_CHUNK) : (LT >= 16 ? 1 : CSB_RMW_CHUNK_RK);
    flux_tile<LT, AXIS, TL, MODE, VISC, false, P, FM>(reinterpret_cast<double *>(smem_raw), (int64_t)blockIdx.x * TL,
                                                      q, g, rhs, qn, qout, drva, tab, lxi, let, lmx, F, nstart, nend,
                                                      cf, ph, rk, fm);
}


// Derivative closure of a boundary code: 0 physical, 1 interface / periodic, -1 unknown.
int bc_ndf(int code);
// Metrics, Jacobian and viscosity of the uniform grid of a solver configuration.
void uniform_phys(const cs_solver_config &cfg, Phys &ph);

// Everything one pass needs, independent of the solver object.
struct PassArgs {
    int64_t lmx;
    int lxi, let;
    int64_t F;
    int nstart, nend;
    int tl;        // lines per tile (8 or 16) of the one-phase kernels
    int pl;        // nonzero: run the producer/consumer (pipelined) kernels
    int nsm;       // multiprocessors of the device (persistent grid)
    int viscous;
    const DeviceTables *tab;
    Coeffs cf;
    Phys ph;
    FieldMet fm;   // per-point metrics (xim null: the constants of ph)
    double *grad;  // [3][4][lmx]
    double *rhs;   // [5][lmx]
    unsigned long long *dtacc;
};

// Tile width of the pipelined passes for chunk length LT and element type T:
// 8 lines for lines of up to 256 (FP64) / 512 (FP32) points, else 4, so that
// two staging buffers fit in shared memory side by side.
template <int LT, typename T>
constexpr int pl_tile() {
    return (sizeof(T) == 8 ? LT <= 8 : LT <= 16) ? 8 : 4;
}
inline int pl_tile_for(int lt, bool fp32) { return (fp32 ? lt <= 16 : lt <= 8) ? 8 : 4; }

template <typename KernelT>
inline int set_smem(KernelT kern, size_t bytes) {
    if (bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute");
    }
    return CS_OK;
}

// Host side (tma_grad.cu): tensor maps over nf consecutive fields, boxes of
// tl lines by boxlen points along `axis` by nf fields.
int tma_field_map(int axis, const cs_dcomp &d, int tl, int boxlen, int nf, const double *base, CUtensorMap &map);
int tma_field_map32(int axis, const cs_dcomp &d, int tl, int boxlen, int nf, const float *base, CUtensorMap &map);
inline int tma_field_map_t(int axis, const cs_dcomp &d, int tl, int boxlen, int nf, const double *base,
                           CUtensorMap &map) {
    return tma_field_map(axis, d, tl, boxlen, nf, base, map);
}
inline int tma_field_map_t(int axis, const cs_dcomp &d, int tl, int boxlen, int nf, const float *base,
                           CUtensorMap &map) {
    return tma_field_map32(axis, d, tl, boxlen, nf, base, map);
}

// Prefetch geometry and tensor maps of a flux pass with the RK update (none
// for the other modes; none where the rows or field blocks are not 16-byte
// multiples, or the lines are longer than two boxes).  RT: element type of
// the RHS accumulator R.  The mixed form's RK pass uses it; in the FP64 RK
// pass, whose R and q^n are 80 B/pt, it measured slower at 256^3
// (flux z + RK 0.849 -> 0.891 ms) and is not used.
template <int AXIS, int TL, int MODE, typename RT>
FluxPrefetch flux_prefetch(const PassArgs &b, const RT *rhs, const double *qn, CUtensorMap &mr, CUtensorMap &mq) {
    FluxPrefetch pf{};
    if (MODE < kAccumRk) return pf;
    const int lze = (int)(b.lmx / ((int64_t)b.lxi * b.let));
    const cs_dcomp d{(int)b.lmx, b.lxi, b.let, lze};
    const int n = AXIS == 0 ? b.lxi : (AXIS == 1 ? b.let : lze);
    if (n > 512 || b.lmx % 4 || (AXIS < 2 ? b.lxi % 4 : ((int64_t)b.lxi * b.let) % 4)) return pf;
    if (reinterpret_cast<uintptr_t>(rhs) % 16 || reinterpret_cast<uintptr_t>(qn) % 16) return pf;
    pf.nbox = n > 256 ? 2 : 1;
    // box starts along the line (the innermost coordinate for x lines) on
    // 16-byte boundaries; boxes that reach past the line read nothing
    pf.boxlen = ((n + pf.nbox - 1) / pf.nbox + 3) / 4 * 4;
    pf.lxi = b.lxi;
    if (MODE != kWriteRk && tma_field_map_t(AXIS, d, TL, pf.boxlen, 5, rhs, mr)) return FluxPrefetch{};
    if (tma_field_map_t(AXIS, d, TL, pf.boxlen, 5, qn, mq)) return FluxPrefetch{};
    pf.on = 1;
    return pf;
}

template <int LT, int AXIS, int TL>
int launch_grad_t(const PassArgs &a, const double *q, bool dtred, cudaStream_t st) {
    const size_t smem = (size_t)4 * TL * LineLayout<LT>::kSlot * sizeof(double);
    auto kern = dtred ? k_grad<LT, AXIS, TL, true> : k_grad<LT, AXIS, TL, false>;
    if (dtred && a.fm.xim) kern = k_grad<LT, AXIS, TL, true, true>;
    if (int rc = set_smem(kern, smem)) return rc;
    const unsigned blocks = (unsigned)((a.F + TL - 1) / TL);
    kern<<<blocks, TL * 32, smem, st>>>(q, a.grad + (int64_t)AXIS * 4 * a.lmx, a.tab->t64, a.lxi, a.let,
                                        a.lmx, a.F, a.nstart, a.nend, a.cf, a.ph, a.dtacc, a.fm);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

template <int LT, int AXIS, int TL, int MODE>
int launch_flux_t(const PassArgs &a, const double *q, const double *qn, double *qout, double *drva,
                  const RkParams &rk, cudaStream_t st) {
    const size_t smem = (size_t)5 * TL * LineLayout<LT>::kSlot * sizeof(double);
    auto kern = a.viscous ? k_flux<LT, AXIS, TL, MODE, true> : k_flux<LT, AXIS, TL, MODE, false>;
    if (a.fm.xim) kern = a.viscous ? k_flux<LT, AXIS, TL, MODE, true, true> : k_flux<LT, AXIS, TL, MODE, false, true>;
    if (int rc = set_smem(kern, smem)) return rc;
    const unsigned blocks = (unsigned)((a.F + TL - 1) / TL);
    kern<<<blocks, TL * 32, smem, st>>>(q, a.grad, a.rhs, qn, qout, drva, a.tab->t64, a.lxi, a.let, a.lmx,
                                        a.F, a.nstart, a.nend, a.cf, a.ph, rk, a.fm);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

template <int AXIS, int TL>
int launch_grad_tl(const PassArgs &a, const double *q, bool dtred, cudaStream_t st) {
    switch (a.tab->lt) {
        case 2: return launch_grad_t<2, AXIS, TL>(a, q, dtred, st);
        case 4: return launch_grad_t<4, AXIS, TL>(a, q, dtred, st);
        case 8: return launch_grad_t<8, AXIS, TL>(a, q, dtred, st);
        case 16: return launch_grad_t<16, AXIS, TL>(a, q, dtred, st);
    }
    return set_error(CS_ERR_UNSUPPORTED, "chunk length");
}

template <int AXIS, int TL, int MODE>
int launch_flux_tm(const PassArgs &a, const double *q, const double *qn, double *qout, double *drva,
                   const RkParams &rk, cudaStream_t st) {
    switch (a.tab->lt) {
        case 2: return launch_flux_t<2, AXIS, TL, MODE>(a, q, qn, qout, drva, rk, st);
        case 4: return launch_flux_t<4, AXIS, TL, MODE>(a, q, qn, qout, drva, rk, st);
        case 8: return launch_flux_t<8, AXIS, TL, MODE>(a, q, qn, qout, drva, rk, st);
        case 16: return launch_flux_t<16, AXIS, TL, MODE>(a, q, qn, qout, drva, rk, st);
    }
    return set_error(CS_ERR_UNSUPPORTED, "chunk length");
}

template <int AXIS, int TL>
int launch_flux_tl(const PassArgs &a, int mode, const double *q, const double *qn, double *qout,
                   double *drva, const RkParams &rk, cudaStream_t st) {
    switch (mode) {
        case kWrite: return launch_flux_tm<AXIS, TL, kWrite>(a, q, qn, qout, drva, rk, st);
        case kAccum: return launch_flux_tm<AXIS, TL, kAccum>(a, q, qn, qout, drva, rk, st);
        case kAccumRk: return launch_flux_tm<AXIS, TL, kAccumRk>(a, q, qn, qout, drva, rk, st);
        default: return launch_flux_tm<AXIS, TL, kWriteRk>(a, q, qn, qout, drva, rk, st);
    }
}

// The compact filter along `axis` applied in place to the five conserved
// fields of q [5][lmx] (filter_pass.cu; kFilter tables of that axis).
int filter_state(double *q, int axis, const DeviceTables &t, const cs_dcomp &d, double af, cudaStream_t st);

// Geometry of the TMA copies of one gradient-pass tile (tma_grad.cuh).
struct TmaGeom {
    int nbox;     // copies along the line (1 or 2)
    int boxlen;   // points per copy along the line
    int ntiles;   // tiles of the pass
    int tiles_x;  // y axis: tiles per x row; unused otherwise
    unsigned tile_bytes;  // bytes of one staged tile (all copies, OOB fill included)
};
// Copy geometry of a TMA gradient pass along `axis`; false when that form
// does not apply (lines longer than 512 points, row strides that are not
// multiples of 16 bytes, or more shared memory than smem_max).
bool tma_grad_geometry(int axis, const cs_dcomp &d, int lt, int smem_max, TmaGeom &g, size_t &smem_bytes);
// The same for the mixed form's gradient passes: the four FP32 shadow fields
// (u, v, w, T - T0) in tiles of 8 lines (4 for lines of 257-512 points).
bool tma_grad_mx_geometry(int axis, const cs_dcomp &d, int lt, int smem_max, TmaGeom &g, size_t &smem_bytes);
// TMA-staged gradient pass along AXIS (tma_grad_axis{0,1,2}.cu); err receives
// a nonzero code if a staging copy did not complete in time.
template <int AXIS>
int launch_grad_tma(const PassArgs &a, const cs_dcomp &d, const double *q, bool dtred, int *err,
                    cudaStream_t st);

// Per-axis entry points (fused_axis{0,1,2}.cu); they run the pipelined
// kernels (pipeline_axis{0,1,2}.cu) when PassArgs::pl is set.
template <int AXIS>
int launch_grad_pl(const PassArgs &a, const double *q, bool dtred, cudaStream_t st);
template <int AXIS>
int launch_flux_pl(const PassArgs &a, int mode, const double *q, const double *qn, double *qout,
                   double *drva, const RkParams &rk, cudaStream_t st);
template <int AXIS>
int launch_grad(const PassArgs &a, const double *q, bool dtred, cudaStream_t st);
template <int AXIS>
int launch_flux(const PassArgs &a, int mode, const double *q, const double *qn, double *qout,
                double *drva, const RkParams &rk, cudaStream_t st);

}  // namespace csb
