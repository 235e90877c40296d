// fused_mixed.cuh -- mixed-precision form of the fused RK-stage passes.
//
// FP64 master state q and FP64 RK accumulation; what the line solves consume
// is FP32:
//   * an FP32 "deviation shadow" of the stage state, (rho - rho0, u, v, w,
//     T - T0) with the free-stream rho0 = 1, T0 = gamma p0 / rho0 = 1 (CANARD
//     units).  It is formed from q in FP64 (pressure and temperature
//     recovered from total energy in FP64, where low-Mach cancellation needs
//     it), so FP32 keeps its relative precision on the small deviations;
//   * FP32 gradients of (u, v, w, T - T0) and an FP32 RHS accumulator R;
//   * fluxes evaluated in FP64 from the shadow and rounded once to FP32 when
//     staged.  They use the pressure deviation: with constant metrics the
//     derivative of the constant part M*p0 is zero, so dropping it leaves the
//     RHS unchanged while the FP32 derivative of a pressure-dominated flux
//     keeps its precision;
//   * line solves in FP32 on right-hand sides formed in FP64 (closure rows
//     included), optionally followed by one iterative-refinement sweep whose
//     residual r - A x is formed in FP64 (cfg.refine: none, all passes, or
//     the flux passes only).  The state error against the FP64 path is set by
//     the FP32 shadow, gradients and RHS accumulator, not by the solves: it is
//     the same with and without the sweep.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "fused_kernels.cuh"

namespace csb {

constexpr double kRho0 = 1.0;
constexpr double kP0 = 1.0 / kGam;
constexpr double kT0 = kGam * kP0 / kRho0;  // = 1

template <int LT, int TL>
__device__ __forceinline__ float *field_line32(float *sm, int field, int line) {
    return sm + (field * TL + line) * LineLayout<LT>::kSlot;
}

// Tridiagonal row coefficients of the derivative system (deriv_rows).
__device__ __forceinline__ void deriv_row(int j, int n, int nstart, int nend, double &a, double &c) {
    a = kAlpha;
    c = kAlpha;
    if (j == 0) { a = 0.0; c = nstart ? kAlpha : kAlpha01; }
    else if (j == 1) { a = nstart ? kAlpha : kAlpha10; c = a; }
    if (j == n - 1) { a = nend ? kAlpha : kAlpha01; c = 0.0; }
    else if (j == n - 2) { a = nend ? kAlpha : kAlpha10; c = a; }
}

// FP32 solve of the derivative of G FP32 lines in shared memory (lines[g],
// g < nf valid) with right-hand sides formed in FP64 and, if refine, one
// FP64-residual refinement; the results overwrite the lines.  The G fields
// share each warp_solve (table loads, shuffle latency) and the row
// coefficients of the residual.  MAYREF = false compiles the sweep out (the
// kernels without refinement then need fewer registers).
template <int LT, int G, bool MAYREF = true>
__device__ __forceinline__ void solve_lines_mx(float *const (&lines)[G], int nf, int lane,
                                               const DevTables<float> &tab, int nstart, int nend,
                                               const Coeffs &cf, int refine) {
    const int n = tab.n;
    const int len = lane_len(lane, LT, tab.p, tab.last_len);
    // right-hand sides formed in FP64 (their differences cancel), rounded once
    float r32[G][LT], x[G][LT];
    // single-rank periodic closures: the group's closure sums on 8 lanes per line
    const bool sums = nstart != 0 || nend != 0;
    const double rows = sums ? group_closure_rows<LT, double, float, G>(lines, nf, n, lane, cf) : 0.0;
#pragma unroll
    for (int g = 0; g < G; ++g) {
        double own2[2];
        if (sums) take_closure_rows(rows, g, lane, own2);
        if (g < nf) {
            double r64[LT];
            deriv_rhs<LT, double, float>(lines[g], n, lane, nstart, nend, nullptr, cf, r64, sums ? own2 : nullptr);
#pragma unroll
            for (int t = 0; t < LT; ++t) x[g][t] = r32[g][t] = (float)r64[t];
        } else {
#pragma unroll
            for (int t = 0; t < LT; ++t) x[g][t] = r32[g][t] = 0.0f;
        }
    }
    warp_solve<LT, G, float>(tab, x, lane);
    if (MAYREF && refine) {
        float xm0[G], xp0[G];
#pragma unroll
        for (int g = 0; g < G; ++g) {
            xm0[g] = __shfl_up_sync(0xffffffffu, x[g][LT - 1], 1);
            xp0[g] = __shfl_down_sync(0xffffffffu, x[g][0], 1);
        }
#pragma unroll
        for (int t = 0; t < LT; ++t) {
            const int j = lane * LT + t;
            double ra, rc;
            deriv_row(j, n, nstart, nend, ra, rc);
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const double xm = t > 0 ? (double)x[g][t > 0 ? t - 1 : 0] : (double)xm0[g];
                double xp = (double)xp0[g];
#pragma unroll
                for (int u = 0; u + 1 < LT; ++u)
                    if (u == t && t + 1 < len) xp = (double)x[g][u + 1];
                const double res = (double)r32[g][t] - (ra * xm + (double)x[g][t] + rc * xp);
                r32[g][t] = j < n ? (float)res : 0.0f;  // the residual replaces the right-hand side
            }
        }
        warp_solve<LT, G, float>(tab, r32, lane);
#pragma unroll
        for (int g = 0; g < G; ++g)
#pragma unroll
            for (int t = 0; t < LT; ++t) x[g][t] += r32[g][t];
    }
    __syncwarp();
#pragma unroll
    for (int g = 0; g < G; ++g) {
        if (g >= nf) continue;
#pragma unroll
        for (int t = 0; t < LT; ++t)
            if (lane * LT + t < n) lines[g][LineLayout<LT>::pos_ct(lane, t)] = x[g][t];
    }
}

template <int LT>
__device__ __forceinline__ void solve_line_mx(float *line, int lane, const DevTables<float> &tab, int nstart,
                                              int nend, const Coeffs &cf, int refine) {
    float *const lines[1] = {line};
    solve_lines_mx<LT, 1>(lines, 1, lane, tab, nstart, nend, cf, refine);
}

#ifndef CSB_MX_SOLVE_GROUP
#define CSB_MX_SOLVE_GROUP 2
#endif
// fields per warp solve of the ChunkFactors form (four: the flux passes solve
// five fields as 4 + 1; measured against 2 + 2 + 1 at 256^3, flux z + RK
// 0.720 -> 0.690 ms, the mixed step 7.47 -> 7.36 ms)
#ifndef CSB_CF_SOLVE_GROUP
#define CSB_CF_SOLVE_GROUP 4
#endif
// resident 256-thread CTAs per SM asked of the compiler (register cap) for
// the mixed one-phase flux passes with ChunkFactors and no refinement sweep
// (with the sweep they would spill; measured at 256^3: three
// CTAs per SM cut the x / y flux passes from 0.31 / 0.50 to 0.25 / 0.41 ms),
// and points per thread loaded together in their load phase
#ifndef CSB_MX_FLUX_MINB
#define CSB_MX_FLUX_MINB 3
#endif
#ifndef CSB_MX_FLUX_UNROLL
#define CSB_MX_FLUX_UNROLL CSB_FLUX_UNROLL
#endif

// FP32 solve of G lines with ChunkFactors (interface closure on both ends,
// full chunks): interior right-hand sides in FP32, the four closure rows of
// each line in FP64 (group_closure_rows), per-row factors from the kernel
// parameters.  REF adds one refinement sweep: the residual r - A x of the
// FP32 right-hand side r and solution x is formed in FP64 (rows
// alpha x[j-1] + x[j] + alpha x[j+1], with no coupling outside the line),
// rounded once, solved in FP32 and added to x.  The results overwrite the
// lines.
template <int LT, int G, bool REF = false>
__device__ __forceinline__ void solve_lines_cf(float *const (&lines)[G], int nf, int lane,
                                               const DevTables<float> &tab, const ChunkFactors<LT> &U,
                                               const Coeffs &cf) {
    const int p = tab.p;
    const double rows = group_closure_rows<LT, double, float, G>(lines, nf, tab.n, lane, cf);
    float x[G][LT];
#pragma unroll
    for (int g = 0; g < G; ++g) {
        double own2[2];
        take_closure_rows(rows, g, lane, own2);
        if (g < nf) deriv_rhs_cf<LT>(lines[g], p, lane, own2, x[g]);
        else {
#pragma unroll
            for (int t = 0; t < LT; ++t) x[g][t] = 0.0f;
        }
    }
    if (REF) {
        float r[G][LT];
#pragma unroll
        for (int g = 0; g < G; ++g)
#pragma unroll
            for (int t = 0; t < LT; ++t) r[g][t] = x[g][t];
        warp_solve_cf<LT, G>(U, tab, x, lane);
        const bool first = lane == 0, last = lane == p - 1, live = lane < p;
#pragma unroll
        for (int g = 0; g < G; ++g) {
            const double xm0 = (double)__shfl_up_sync(0xffffffffu, x[g][LT - 1], 1);
            const double xp0 = (double)__shfl_down_sync(0xffffffffu, x[g][0], 1);
            double xm = first ? 0.0 : xm0, xc = (double)x[g][0];
#pragma unroll
            for (int t = 0; t < LT; ++t) {
                const double xp = t + 1 < LT ? (double)x[g][t + 1] : (last ? 0.0 : xp0);
                const double res = (double)r[g][t] - fma(kAlpha, xm + xp, xc);
                r[g][t] = live ? (float)res : 0.0f;
                xm = xc;
                xc = xp;
            }
        }
        warp_solve_cf<LT, G>(U, tab, r, lane);
#pragma unroll
        for (int g = 0; g < G; ++g)
#pragma unroll
            for (int t = 0; t < LT; ++t) x[g][t] += r[g][t];
    } else {
        warp_solve_cf<LT, G>(U, tab, x, lane);
    }
    __syncwarp();
#pragma unroll
    for (int g = 0; g < G; ++g) {
        if (g >= nf) continue;
        if (lane < p) {
#pragma unroll
            for (int t = 0; t < LT; ++t) lines[g][LineLayout<LT>::pos_ct(lane, t)] = x[g][t];
        }
    }
}

// The NF fields of this warp's line of the tile, CSB_MX_SOLVE_GROUP at a time
// (one at a time for lines of more than 256 points when the refinement sweep
// is compiled in: registers).
// CF: the lines have ChunkFactors (solve_lines_cf, with the sweep if REF).
template <int LT, int TL, int NF, bool REF, bool CF = false>
__device__ __forceinline__ void solve_fields_mx(float *sm, int w, int lane, const DevTables<float> &tab,
                                                int nstart, int nend, const Coeffs &cf,
                                                const ChunkFactors<LT> &U) {
    if (CF) {
        // full groups of G fields, then the NF % G remaining fields as one
        // smaller group (no solve of a padding field)
        constexpr int G = REF && LT >= 16 ? 1 : CSB_CF_SOLVE_GROUP;
        constexpr int NFULL = NF / G * G, REM = NF - NFULL;
#pragma unroll 1
        for (int c = 0; c < NFULL; c += G) {
            float *lines[G];
#pragma unroll
            for (int g = 0; g < G; ++g) lines[g] = field_line32<LT, TL>(sm, c + g, w);
            solve_lines_cf<LT, G, REF>(lines, G, lane, tab, U, cf);
        }
        if constexpr (REM > 0) {
            float *lines[REM];
#pragma unroll
            for (int g = 0; g < REM; ++g) lines[g] = field_line32<LT, TL>(sm, NFULL + g, w);
            solve_lines_cf<LT, REM, REF>(lines, REM, lane, tab, U, cf);
        }
        return;
    }
    constexpr int G = (LT >= 16 && REF) ? 1 : CSB_MX_SOLVE_GROUP;
#pragma unroll 1
    for (int c = 0; c < NF; c += G) {
        float *lines[G];
#pragma unroll
        for (int g = 0; g < G; ++g) lines[g] = field_line32<LT, TL>(sm, c + g < NF ? c + g : c, w);
        solve_lines_mx<LT, G, REF>(lines, NF - c, lane, tab, nstart, nend, cf, REF ? 1 : 0);
    }
}

// FP32 shadow values of one point from the FP64 state (thermo in FP64).
__device__ __forceinline__ void shadow_from_q(double q0, double q1, double q2, double q3, double q4,
                                              float (&sh)[5], Prim &s) {
    s = primitives(q0, q1, q2, q3, q4);
    sh[0] = (float)(q0 - kRho0);
    sh[1] = (float)s.u;
    sh[2] = (float)s.v;
    sh[3] = (float)s.w;
    sh[4] = (float)(s.T - kT0);
}

// p - p0 from the shadow deviations, in FP64: with p = rho T / gamma and
// gamma p0 = rho0 T0 = 1, p - p0 = (drho + dT + drho dT) / gamma.
__device__ __forceinline__ double pres_dev(double dr, double dT) { return (dr + dT + dr * dT) * (1.0 / kGam); }

// ----------------------------------------------------------------------------
// gradient pass (FIRST: reads the FP64 state, writes the shadow, reduces CFL)
// ----------------------------------------------------------------------------
template <int LT, int AXIS, int TL, bool FIRST, bool REF, bool CF = false>
__global__ void __launch_bounds__(TL * 32, TL == 8 ? 2 : 1)
k_grad_mx(const double *__restrict__ q, float *__restrict__ sh, float *__restrict__ g,
          DevTables<float> tab, int lxi, int let, int64_t lmx, int64_t F, int nstart, int nend, Coeffs cf,
          Phys ph, unsigned long long *__restrict__ dtacc, ChunkFactors<LT> U) {
    using L = LineLayout<LT>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *sm = reinterpret_cast<float *>(smem_raw);
    const int n = tab.n;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t line0 = (int64_t)blockIdx.x * TL;
    double m1 = 0.0, m2 = 0.0;
    tile_for_each<AXIS, TL, CSB_GRAD_UNROLL>(line0, F, n, lxi, let, [&](int l, int j, int64_t gi) {
        float u, v, wv, tp;
        if (FIRST) {
            float s5[5];
            Prim s;
            shadow_from_q(__ldg(q + gi), __ldg(q + lmx + gi), __ldg(q + 2 * lmx + gi), __ldg(q + 3 * lmx + gi),
                          __ldg(q + 4 * lmx + gi), s5, s);
#pragma unroll
            for (int k = 0; k < 5; ++k) sh[k * lmx + gi] = s5[k];
            u = s5[1];
            v = s5[2];
            wv = s5[3];
            tp = s5[4];
            const double uu = s.u + ph.umf[0], vv = s.v + ph.umf[1], ww = s.w + ph.umf[2];
            double rr2 = 0.0;
#pragma unroll
            for (int a = 0; a < 3; ++a)
                rr2 += fabs(xmul(ph.M[a][0], uu) + xmul(ph.M[a][1], vv) + xmul(ph.M[a][2], ww));
            const double ssi = fabs(ph.J);
            m1 = fmax(m1, xmul(sqrt(xmul(s.T, ph.rr1)) + rr2, ssi));
            m2 = fmax(m2, s.ri * ph.mu * ph.rr1 * ssi * ssi);
        } else {
            const float dt = __ldg(sh + 4 * lmx + gi);
            u = __ldg(sh + lmx + gi);
            v = __ldg(sh + 2 * lmx + gi);
            wv = __ldg(sh + 3 * lmx + gi);
            tp = dt;
        }
        const int pj = L::pos(j);
        field_line32<LT, TL>(sm, 0, l)[pj] = u;
        field_line32<LT, TL>(sm, 1, l)[pj] = v;
        field_line32<LT, TL>(sm, 2, l)[pj] = wv;
        field_line32<LT, TL>(sm, 3, l)[pj] = tp;
    });
    tile_sync<AXIS, TL>();
    if (line0 + w < F) solve_fields_mx<LT, TL, 4, REF, CF>(sm, w, lane, tab, nstart, nend, cf, U);
    tile_sync<AXIS, TL>();
    tile_for_each<AXIS, TL, CSB_STORE_UNROLL>(line0, F, n, lxi, let, [&](int l, int j, int64_t gi) {
        const int pj = L::pos(j);
#pragma unroll
        for (int c = 0; c < 4; ++c) g[c * lmx + gi] = field_line32<LT, TL>(sm, c, l)[pj];
    });
    if (FIRST) {
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

// Flux components F[m][AXIS], evaluated in FP64 from the FP32 shadow and FP32
// gradients (the inputs are exact in FP64, so only the final rounding to FP32
// when staging adds error).
template <int AXIS, bool VISC>
__device__ __forceinline__ void point_flux_mx(const float *__restrict__ sh, const float *__restrict__ g,
                                              int64_t lmx, int64_t gi, const Phys &ph, float (&flo)[5]) {
    const double dr = __ldg(sh + gi), u = __ldg(sh + lmx + gi), v = __ldg(sh + 2 * lmx + gi);
    const double wv = __ldg(sh + 3 * lmx + gi), dp = pres_dev(dr, __ldg(sh + 4 * lmx + gi));
    double gr[12];
    if (VISC) {
#pragma unroll
        for (int k = 0; k < 12; ++k) gr[k] = (double)__ldg(g + k * lmx + gi);
    }
    const double rho = kRho0 + dr;
    // the mixed form runs on the uniform Cartesian grid: the metric matrix is
    // diagonal, so only the AXIS entries of the sums below are nonzero
    const double mA = ph.M[AXIS][AXIS];
    const double vel[3] = {u, v, wv};
    const double ss = mA * (vel[AXIS] + ph.umf[AXIS]);
    // rho*H = gamma/(gamma-1) p + rho |u|^2 / 2 with p = p0 + dp
    const double rH = kGam * kHamm1 * (kP0 + dp) + 0.5 * rho * (u * u + v * v + wv * wv);
    double fl[5];
    fl[0] = rho * ss;
    fl[1] = rho * u * ss;
    fl[2] = rho * v * ss;
    fl[3] = rho * wv * ss;
    fl[1 + AXIS] += mA * dp;
    fl[4] = rH * ss - dp * (ph.umf[AXIS] * mA);
    if (VISC) {
        double dx[4][3];
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int k = 0; k < 3; ++k) dx[c][k] = ph.M[k][k] * gr[4 * k + c];
        const double muj = ph.mu * ph.J;
        const double kap = kGamm1Prndtli * muj;
        const double div = 2.0 / 3.0 * (dx[0][0] + dx[1][1] + dx[2][2]);
        const double txx = muj * (2.0 * dx[0][0] - div), tyy = muj * (2.0 * dx[1][1] - div);
        const double tzz = muj * (2.0 * dx[2][2] - div);
        const double txy = muj * (dx[1][0] + dx[0][1]), tyz = muj * (dx[2][1] + dx[1][2]);
        const double tzx = muj * (dx[0][2] + dx[2][0]);
        // rows of the stress tensor: t[k] = (tau_kx, tau_ky, tau_kz); only column AXIS is needed
        const double t[3][3] = {{txx, txy, tzx}, {txy, tyy, tyz}, {tzx, tyz, tzz}};
        const double hA = kap * dx[3][AXIS] + u * t[0][AXIS] + v * t[1][AXIS] + wv * t[2][AXIS];
        fl[1] -= mA * t[0][AXIS];
        fl[2] -= mA * t[1][AXIS];
        fl[3] -= mA * t[2][AXIS];
        fl[4] -= mA * hA;
    }
#pragma unroll
    for (int m = 0; m < 5; ++m) flo[m] = (float)fl[m];
}

// Uniform-grid constants of the flux in FP32.
struct PhysF {
    float mA[3];   // diagonal metric entries M[k][k]
    float umf[3];  // moving-frame velocity
    float muj;     // mu J
    float kap;     // heat conduction coefficient mu J / ((gamma - 1) Pr)
};
__device__ __forceinline__ PhysF phys_f32(const Phys &ph) {
    PhysF f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        f.mA[k] = (float)ph.M[k][k];
        f.umf[k] = (float)ph.umf[k];
    }
    f.muj = (float)(ph.mu * ph.J);
    f.kap = (float)(kGamm1Prndtli * ph.mu * ph.J);
    return f;
}

// point_flux_mx evaluated in FP32 (the flux arithmetic of the mixed form on
// lines with ChunkFactors), divided by the pass's metric entry
// mA = M[AXIS][AXIS]: every term of F[m][AXIS] on the uniform grid carries
// exactly one factor mA and the compact derivative is linear, so the pass
// multiplies the derivative by mA instead.  Leaving the factor out, and
// forming each value with fused multiply-adds around its largest term, keeps
// the FP32 rounding of the flux values (which the derivative amplifies by
// about 1 / h) near one rounding per value, as when they are evaluated in
// FP64 and rounded once.  The pressure enters as its deviation
// p - p0 = (drho + dT + drho dT) / gamma.
template <int AXIS, bool VISC>
__device__ __forceinline__ void point_flux_f32(const float *__restrict__ sh, const float *__restrict__ g,
                                               int64_t lmx, int64_t gi, const PhysF &pf, float (&fl)[5]) {
    const float dr = __ldg(sh + gi), u = __ldg(sh + lmx + gi), v = __ldg(sh + 2 * lmx + gi);
    const float wv = __ldg(sh + 3 * lmx + gi), dT = __ldg(sh + 4 * lmx + gi);
    float gr[12];
    if (VISC) {
#pragma unroll
        for (int k = 0; k < 12; ++k) gr[k] = __ldg(g + k * lmx + gi);
    }
    constexpr float gami = (float)(1.0 / kGam), hamm1 = (float)kHamm1, cp0 = (float)(kGam * kHamm1 * kP0);
    const float dpg = fmaf(dr, dT, dr + dT);  // gamma (p - p0)
    const float dp = dpg * gami;
    const float vel[3] = {u, v, wv};
    const float sp = vel[AXIS] + pf.umf[AXIS];  // contravariant velocity / mA
    const float rsp = fmaf(dr, sp, sp);         // rho * sp
    fl[0] = rsp;
    fl[1] = rsp * u;
    fl[2] = rsp * v;
    fl[3] = rsp * wv;
    fl[1 + AXIS] = fmaf(rsp, vel[AXIS], dp);
    // rho H = gamma p / (gamma - 1) + rho |u|^2 / 2 = cp0 + dpg / (gamma - 1) + rho |u|^2 / 2
    const float q2 = fmaf(u, u, fmaf(v, v, wv * wv));
    const float rest = fmaf(0.5f * (1.0f + dr), q2, hamm1 * dpg);
    fl[4] = fmaf(cp0, sp, rest * sp) - dp * pf.umf[AXIS];
    if (VISC) {
        float dx[4][3];
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int k = 0; k < 3; ++k) dx[c][k] = pf.mA[k] * gr[4 * k + c];
        const float div = (2.0f / 3.0f) * (dx[0][0] + dx[1][1] + dx[2][2]);
        float t[3];  // column AXIS of the stress tensor
#pragma unroll
        for (int k = 0; k < 3; ++k)
            t[k] = k == AXIS ? pf.muj * (2.0f * dx[k][k] - div) : pf.muj * (dx[k][AXIS] + dx[AXIS][k]);
        const float hA = fmaf(pf.kap, dx[3][AXIS], fmaf(u, t[0], fmaf(v, t[1], wv * t[2])));
        fl[1] -= t[0];
        fl[2] -= t[1];
        fl[3] -= t[2];
        fl[4] -= hA;
    }
}

template <int LT, int AXIS, int TL, int MODE, bool VISC, bool SHADOW_OUT, bool REF, bool CF = false>
__global__ void __launch_bounds__(TL * 32, TL == 8 ? (CF && !REF ? CSB_MX_FLUX_MINB : 2) : 1)
k_flux_mx(const float *__restrict__ sh, const float *__restrict__ g, float *__restrict__ rhs,
          const double *__restrict__ qn, double *__restrict__ qout, float *__restrict__ sh_out,
          double *__restrict__ drva, DevTables<float> tab, int lxi, int let, int64_t lmx, int64_t F,
          int nstart, int nend, Coeffs cf, Phys ph, RkParams rk, ChunkFactors<LT> U,
          const __grid_constant__ CUtensorMap pf_r, const __grid_constant__ CUtensorMap pf_q, FluxPrefetch pfg) {
    using L = LineLayout<LT>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *sm = reinterpret_cast<float *>(smem_raw);
    const int n = tab.n;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t line0 = (int64_t)blockIdx.x * TL;
    const PhysF pf = phys_f32(ph);
    tile_for_each<AXIS, TL, CSB_MX_FLUX_UNROLL>(line0, F, n, lxi, let, [&](int l, int j, int64_t gi) {
        float fl[5];
        if (CF) point_flux_f32<AXIS, VISC>(sh, g, lmx, gi, pf, fl);
        else point_flux_mx<AXIS, VISC>(sh, g, lmx, gi, ph, fl);
        const int pj = L::pos(j);
#pragma unroll
        for (int m = 0; m < 5; ++m) field_line32<LT, TL>(sm, m, l)[pj] = fl[m];
    });
    // the RK store phase's R and q^n of this tile, fetched into L2 while the
    // tile is solved (measured at 256^3: flux z + RK 0.689 -> 0.639 ms; issued
    // before the load phase it competed with it and was slower, and the
    // R-only prefetch of the accumulate pass did not pay)
    if (MODE >= kAccumRk && pfg.on && threadIdx.x == 0) {
        if (MODE != kWriteRk) prefetch_tile<AXIS>(&pf_r, pfg, line0);
        prefetch_tile<AXIS>(&pf_q, pfg, line0);
    }
    tile_sync<AXIS, TL>();
    const int64_t fidx = line0 + w;
    if (fidx < F) {
        solve_fields_mx<LT, TL, 5, REF, CF>(sm, w, lane, tab, nstart, nend, cf, U);
        if (drva) {
            __syncwarp();
            if (lane < 10) {
                const int m = lane % 5, face = lane / 5;
                const double dv = (double)field_line32<LT, TL>(sm, m, w)[L::pos(face ? n - 1 : 0)];
                drva[(int64_t)(face * 5 + m) * F + fidx] = CF ? ph.M[AXIS][AXIS] * dv : dv;
            }
        }
    }
    tile_sync<AXIS, TL>();
    double dtk = 0.0;
    if (MODE >= kAccumRk) {
        const double dt = rk_dt(rk);
        dtk = xmul(dt / rk.div, ph.J);
        if (rk.dt_out && blockIdx.x == 0 && threadIdx.x == 0) *rk.dt_out = dt;
    }
    // CF kernels solved F / mA (point_flux_f32): the derivative is scaled here
    const float mA32 = pf.mA[AXIS];
    const double mA64 = ph.M[AXIS][AXIS];
    if (MODE == kWrite) {
        tile_for_each<AXIS, TL, CSB_STORE_UNROLL>(line0, F, n, lxi, let, [&](int l, int j, int64_t gi) {
            const int pj = L::pos(j);
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                const float dv = field_line32<LT, TL>(sm, m, l)[pj];
                rhs[m * lmx + gi] = CF ? mA32 * dv : dv;
            }
        });
    } else {
        constexpr int P = MODE == kAccum ? (LT >= 16 ? 2 : CSB_RMW_CHUNK) : (LT >= 16 ? 1 : CSB_RMW_CHUNK_RK);
        float rv[P][5];
        double qv[P][5];
        tile_for_each_chunked<AXIS, TL, P>(
            line0, F, n, lxi, let,
            [&](int p, int l, int j, int64_t gi) {
#pragma unroll
                for (int m = 0; m < 5; ++m) {
                    rv[p][m] = MODE == kWriteRk ? 0.0f : rhs[m * lmx + gi];
                    if (MODE >= kAccumRk) qv[p][m] = qn[m * lmx + gi];
                }
            },
            [&](int p, int l, int j, int64_t gi) {
                const int pj = L::pos(j);
                if (MODE == kAccum) {
#pragma unroll
                    for (int m = 0; m < 5; ++m) {
                        const float dv = field_line32<LT, TL>(sm, m, l)[pj];
                        rhs[m * lmx + gi] = CF ? fmaf(mA32, dv, rv[p][m]) : rv[p][m] + dv;
                    }
                } else {
                    double qo[5];
#pragma unroll
                    for (int m = 0; m < 5; ++m) {
                        const double dv = (double)field_line32<LT, TL>(sm, m, l)[pj];
                        const double r = CF ? fma(mA64, dv, (double)rv[p][m]) : (double)rv[p][m] + dv;
                        qo[m] = qv[p][m] - xmul(dtk, r);
                        qout[m * lmx + gi] = qo[m];
                    }
                    if (SHADOW_OUT) {
                        float s5[5];
                        Prim s;
                        shadow_from_q(qo[0], qo[1], qo[2], qo[3], qo[4], s5, s);
#pragma unroll
                        for (int m = 0; m < 5; ++m) sh_out[m * lmx + gi] = s5[m];
                    }
                }
            });
    }
}

struct MixedArgs {
    PassArgs base;
    float *shadow;  // [5][lmx]
    float *grad;    // [3][4][lmx]
    float *rhs;     // [5][lmx]
    int refine;
    int fp32;       // FP32 interior arithmetic where the line has ChunkFactors
};

// The pass runs the ChunkFactors kernels: FP32 interior arithmetic asked for,
// the interface closure on both ends (deriv_rhs_cf forms those closure rows)
// and the line's tables uniform (the refinement sweep, if on, is theirs).
// Uniform tables alone do not imply the interface closure: with 2-row chunks
// the physical closure's rows only enter the reduced system.
inline bool use_cf(const MixedArgs &a) {
    return a.fp32 && a.base.nstart && a.base.nend && a.base.tab->uniform;
}

template <int LT>
ChunkFactors<LT> chunk_factors_of(const DeviceTables &dt) {
    ChunkFactors<LT> U{};
    if (!dt.uniform || dt.lt != LT) return U;
    for (int t = 0; t < LT; ++t) {
        U.f1[t] = dt.cfu[t];
        U.f2[t] = dt.cfu[LT + t];
        U.b1[t] = dt.cfu[2 * LT + t];
        U.b2[t] = dt.cfu[3 * LT + t];
        U.nra[t] = dt.cfu[4 * LT + t];
        U.nrc[t] = dt.cfu[5 * LT + t];
    }
    return U;
}

template <int LT, int AXIS, int TL>
int launch_grad_mx_t(const MixedArgs &a, const double *q, bool first, cudaStream_t st) {
    const size_t smem = (size_t)4 * TL * LineLayout<LT>::kSlot * sizeof(float);
    const bool cfp = use_cf(a);
    auto kern = first ? (a.refine ? (cfp ? k_grad_mx<LT, AXIS, TL, true, true, true> : k_grad_mx<LT, AXIS, TL, true, true>)
                                  : (cfp ? k_grad_mx<LT, AXIS, TL, true, false, true> : k_grad_mx<LT, AXIS, TL, true, false>))
                      : (a.refine ? (cfp ? k_grad_mx<LT, AXIS, TL, false, true, true> : k_grad_mx<LT, AXIS, TL, false, true>)
                                  : (cfp ? k_grad_mx<LT, AXIS, TL, false, false, true>
                                         : k_grad_mx<LT, AXIS, TL, false, false>));
    if (int rc = set_smem(kern, smem)) return rc;
    const PassArgs &b = a.base;
    const unsigned blocks = (unsigned)((b.F + TL - 1) / TL);
    kern<<<blocks, TL * 32, smem, st>>>(q, a.shadow, a.grad + (int64_t)AXIS * 4 * b.lmx, b.tab->t32, b.lxi,
                                        b.let, b.lmx, b.F, b.nstart, b.nend, b.cf, b.ph, b.dtacc,
                                        chunk_factors_of<LT>(*b.tab));
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

template <int LT, int AXIS, int TL, int MODE>
int launch_flux_mx_t(const MixedArgs &a, const double *qn, double *qout, bool shadow_out, double *drva,
                     const RkParams &rk, cudaStream_t st) {
    const size_t smem = (size_t)5 * TL * LineLayout<LT>::kSlot * sizeof(float);
    const PassArgs &b = a.base;
    // the shadow is written only by the RK modes
    constexpr bool kRk = MODE >= kAccumRk;
    auto pick = [&](auto ref, auto cfv) {
        constexpr bool R = decltype(ref)::value;
        constexpr bool C = decltype(cfv)::value;
        return b.viscous ? (shadow_out && kRk ? k_flux_mx<LT, AXIS, TL, MODE, true, kRk, R, C>
                                              : k_flux_mx<LT, AXIS, TL, MODE, true, false, R, C>)
                         : (shadow_out && kRk ? k_flux_mx<LT, AXIS, TL, MODE, false, kRk, R, C>
                                              : k_flux_mx<LT, AXIS, TL, MODE, false, false, R, C>);
    };
    const bool cfp = use_cf(a);
    auto kern = a.refine ? (cfp ? pick(std::true_type{}, std::true_type{}) : pick(std::true_type{}, std::false_type{}))
                         : (cfp ? pick(std::false_type{}, std::true_type{}) : pick(std::false_type{}, std::false_type{}));
    if (int rc = set_smem(kern, smem)) return rc;
    const unsigned blocks = (unsigned)((b.F + TL - 1) / TL);
    CUtensorMap mr{}, mq{};
    const FluxPrefetch pfg = flux_prefetch<AXIS, TL, MODE>(b, a.rhs, qn, mr, mq);
    kern<<<blocks, TL * 32, smem, st>>>(a.shadow, a.grad, a.rhs, qn, qout, a.shadow, drva, b.tab->t32, b.lxi,
                                        b.let, b.lmx, b.F, b.nstart, b.nend, b.cf, b.ph, rk,
                                        chunk_factors_of<LT>(*b.tab), mr, mq, pfg);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

template <int AXIS, int TL>
int launch_grad_mx_tl(const MixedArgs &a, const double *q, bool first, cudaStream_t st) {
    switch (a.base.tab->lt) {
        case 2: return launch_grad_mx_t<2, AXIS, TL>(a, q, first, st);
        case 4: return launch_grad_mx_t<4, AXIS, TL>(a, q, first, st);
        case 8: return launch_grad_mx_t<8, AXIS, TL>(a, q, first, st);
        case 16: return launch_grad_mx_t<16, AXIS, TL>(a, q, first, st);
    }
    return set_error(CS_ERR_UNSUPPORTED, "chunk length");
}

template <int AXIS, int TL, int MODE>
int launch_flux_mx_tm(const MixedArgs &a, const double *qn, double *qout, bool shadow_out, double *drva,
                      const RkParams &rk, cudaStream_t st) {
    switch (a.base.tab->lt) {
        case 2: return launch_flux_mx_t<2, AXIS, TL, MODE>(a, qn, qout, shadow_out, drva, rk, st);
        case 4: return launch_flux_mx_t<4, AXIS, TL, MODE>(a, qn, qout, shadow_out, drva, rk, st);
        case 8: return launch_flux_mx_t<8, AXIS, TL, MODE>(a, qn, qout, shadow_out, drva, rk, st);
        case 16: return launch_flux_mx_t<16, AXIS, TL, MODE>(a, qn, qout, shadow_out, drva, rk, st);
    }
    return set_error(CS_ERR_UNSUPPORTED, "chunk length");
}

template <int AXIS, int TL>
int launch_flux_mx_tl(const MixedArgs &a, int mode, const double *qn, double *qout, bool shadow_out,
                      double *drva, const RkParams &rk, cudaStream_t st) {
    switch (mode) {
        case kWrite: return launch_flux_mx_tm<AXIS, TL, kWrite>(a, qn, qout, shadow_out, drva, rk, st);
        case kAccum: return launch_flux_mx_tm<AXIS, TL, kAccum>(a, qn, qout, shadow_out, drva, rk, st);
        case kAccumRk: return launch_flux_mx_tm<AXIS, TL, kAccumRk>(a, qn, qout, shadow_out, drva, rk, st);
        default: return launch_flux_mx_tm<AXIS, TL, kWriteRk>(a, qn, qout, shadow_out, drva, rk, st);
    }
}

// Per-axis entry points (fused_mixed_axis{0,1,2}.cu); they run the pipelined
// kernels (pipeline_mixed_axis{0,1,2}.cu) when PassArgs::pl is set.
template <int AXIS>
int launch_grad_mx_pl(const MixedArgs &m, const double *q, bool first, cudaStream_t st);
template <int AXIS>
int launch_flux_mx_pl(const MixedArgs &m, int mode, const double *qn, double *qout, bool shadow_out,
                      double *drva, const RkParams &rk, cudaStream_t st);
template <int AXIS>
int launch_grad_mx(const MixedArgs &a, const double *q, bool first, cudaStream_t st);
// TMA-staged gradient pass of the mixed form (not the first of a step: it
// reads the FP32 shadow), tma_grad_mx_axis{0,1,2}.cu; err receives a nonzero
// code if a staging copy did not complete in time.
template <int AXIS>
int launch_grad_mx_tma(const MixedArgs &m, const cs_dcomp &d, int *err, cudaStream_t st);
template <int AXIS>
int launch_flux_mx(const MixedArgs &a, int mode, const double *qn, double *qout, bool shadow_out,
                   double *drva, const RkParams &rk, cudaStream_t st);

}  // namespace csb
