// adjoint_point.cuh -- tangent (forward-mode) and adjoint (reverse-mode)
// linearizations of the pointwise parts of the RHS:
//   * the primitives phi(q) = (u, v, w, T) that the gradient passes
//     differentiate (T = gamma p / rho, CANARD units);
//   * the flux F_a(q, G) of calc_fluxes_pre_compute_kernel<Visc> with the
//     viscous stress and heat flux of calc_viscous_shear_stress
//     (src/cuda/kernels/physics.hpp:42-193, :285-333), G[b*4 + c] being the
//     derivative along xi_b of primitive c.
// Plain FP64 arithmetic (the linearizations are not required to be
// bit-identical to anything); host and device so that the library can expose
// them to host-side checks.
#pragma once

#include "cs_common.h"

namespace csb {

struct PointPhys {
    double M[3][3];
    double J, mu, umf[3];
};

#define CSB_HD __host__ __device__ __forceinline__

// ---------------------------------------------------------------- primitives
CSB_HD void prim_eval(const double q[5], double phi[4]) {
    const double ri = 1.0 / q[0];
    const double u = q[1] * ri, v = q[2] * ri, w = q[3] * ri;
    const double p = kGamm1 * (q[4] - 0.5 * (q[1] * u + q[2] * v + q[3] * w));
    phi[0] = u;
    phi[1] = v;
    phi[2] = w;
    phi[3] = kGam * p * ri;
}

// d phi = (d phi / d q) dq
CSB_HD void prim_tan(const double q[5], const double dq[5], double dphi[4]) {
    const double ri = 1.0 / q[0];
    const double u = q[1] * ri, v = q[2] * ri, w = q[3] * ri;
    const double p = kGamm1 * (q[4] - 0.5 * (q[1] * u + q[2] * v + q[3] * w));
    const double dri = -ri * ri * dq[0];
    const double du = dq[1] * ri + q[1] * dri, dv = dq[2] * ri + q[2] * dri, dw = dq[3] * ri + q[3] * dri;
    // p = (g-1)(E - 0.5 (m.m) ri)
    const double mm = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    const double dmm = 2.0 * (q[1] * dq[1] + q[2] * dq[2] + q[3] * dq[3]);
    const double dp = kGamm1 * (dq[4] - 0.5 * (dmm * ri + mm * dri));
    dphi[0] = du;
    dphi[1] = dv;
    dphi[2] = dw;
    dphi[3] = kGam * (dp * ri + p * dri);
}

// qbar += (d phi / d q)^T phibar
CSB_HD void prim_adj(const double q[5], const double pb[4], double qbar[5]) {
    const double ri = 1.0 / q[0];
    const double u = q[1] * ri, v = q[2] * ri, w = q[3] * ri;
    const double p = kGamm1 * (q[4] - 0.5 * (q[1] * u + q[2] * v + q[3] * w));
    const double mm = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    // T = g p ri
    const double pbar = kGam * ri * pb[3];
    double ribar = kGam * p * pb[3];
    // u = q1 ri, ...
    qbar[1] += ri * pb[0];
    qbar[2] += ri * pb[1];
    qbar[3] += ri * pb[2];
    ribar += q[1] * pb[0] + q[2] * pb[1] + q[3] * pb[2];
    // p = (g-1)(q4 - 0.5 mm ri)
    qbar[4] += kGamm1 * pbar;
    const double mmbar = -0.5 * kGamm1 * ri * pbar;
    ribar += -0.5 * kGamm1 * mm * pbar;
    qbar[1] += 2.0 * q[1] * mmbar;
    qbar[2] += 2.0 * q[2] * mmbar;
    qbar[3] += 2.0 * q[3] * mmbar;
    // ri = 1 / q0
    qbar[0] += -ri * ri * ribar;
}

// ---------------------------------------------------------------------- flux
// Forward evaluation in the same structure as the linearizations below.
template <bool VISC>
CSB_HD void flux_eval(int a, const double q[5], const double G[12], const PointPhys &ph, double F[5]) {
    const double ri = 1.0 / q[0];
    const double u = q[1] * ri, v = q[2] * ri, w = q[3] * ri;
    const double p = kGamm1 * (q[4] - 0.5 * (q[1] * u + q[2] * v + q[3] * w));
    const double *Ma = ph.M[a];
    const double ss = Ma[0] * (u + ph.umf[0]) + Ma[1] * (v + ph.umf[1]) + Ma[2] * (w + ph.umf[2]);
    const double mu_dot = ph.umf[0] * Ma[0] + ph.umf[1] * Ma[1] + ph.umf[2] * Ma[2];
    F[0] = q[0] * ss;
    F[1] = q[1] * ss + Ma[0] * p;
    F[2] = q[2] * ss + Ma[1] * p;
    F[3] = q[3] * ss + Ma[2] * p;
    F[4] = (q[4] + p) * ss - p * mu_dot;
    if (VISC) {
        double dx[4][3];
        for (int c = 0; c < 4; ++c)
            for (int k = 0; k < 3; ++k)
                dx[c][k] = ph.M[0][k] * G[c] + ph.M[1][k] * G[4 + c] + ph.M[2][k] * G[8 + c];
        const double muj = ph.mu * ph.J, kap = kGamm1Prndtli * muj;
        const double div = 2.0 / 3.0 * (dx[0][0] + dx[1][1] + dx[2][2]);
        const double t[3][3] = {{muj * (2.0 * dx[0][0] - div), muj * (dx[1][0] + dx[0][1]), muj * (dx[0][2] + dx[2][0])},
                                {muj * (dx[1][0] + dx[0][1]), muj * (2.0 * dx[1][1] - div), muj * (dx[2][1] + dx[1][2])},
                                {muj * (dx[0][2] + dx[2][0]), muj * (dx[2][1] + dx[1][2]), muj * (2.0 * dx[2][2] - div)}};
        const double uu[3] = {u, v, w};
        for (int i = 0; i < 3; ++i) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += Ma[k] * t[i][k];
            F[1 + i] -= s;
        }
        for (int k = 0; k < 3; ++k) {
            const double h = kap * dx[3][k] + uu[0] * t[0][k] + uu[1] * t[1][k] + uu[2] * t[2][k];
            F[4] -= Ma[k] * h;
        }
    }
}

// dF = (dF/dq) dq + (dF/dG) dG
template <bool VISC>
CSB_HD void flux_tan(int a, const double q[5], const double G[12], const double dq[5], const double dG[12],
                     const PointPhys &ph, double dF[5]) {
    const double ri = 1.0 / q[0];
    const double u = q[1] * ri, v = q[2] * ri, w = q[3] * ri;
    const double p = kGamm1 * (q[4] - 0.5 * (q[1] * u + q[2] * v + q[3] * w));
    const double dri = -ri * ri * dq[0];
    const double du = dq[1] * ri + q[1] * dri, dv = dq[2] * ri + q[2] * dri, dw = dq[3] * ri + q[3] * dri;
    const double mm = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    const double dmm = 2.0 * (q[1] * dq[1] + q[2] * dq[2] + q[3] * dq[3]);
    const double dp = kGamm1 * (dq[4] - 0.5 * (dmm * ri + mm * dri));
    const double *Ma = ph.M[a];
    const double ss = Ma[0] * (u + ph.umf[0]) + Ma[1] * (v + ph.umf[1]) + Ma[2] * (w + ph.umf[2]);
    const double dss = Ma[0] * du + Ma[1] * dv + Ma[2] * dw;
    const double mu_dot = ph.umf[0] * Ma[0] + ph.umf[1] * Ma[1] + ph.umf[2] * Ma[2];
    dF[0] = dq[0] * ss + q[0] * dss;
    dF[1] = dq[1] * ss + q[1] * dss + Ma[0] * dp;
    dF[2] = dq[2] * ss + q[2] * dss + Ma[1] * dp;
    dF[3] = dq[3] * ss + q[3] * dss + Ma[2] * dp;
    dF[4] = (dq[4] + dp) * ss + (q[4] + p) * dss - dp * mu_dot;
    if (VISC) {
        double dx[4][3], ddx[4][3];
        for (int c = 0; c < 4; ++c)
            for (int k = 0; k < 3; ++k) {
                dx[c][k] = ph.M[0][k] * G[c] + ph.M[1][k] * G[4 + c] + ph.M[2][k] * G[8 + c];
                ddx[c][k] = ph.M[0][k] * dG[c] + ph.M[1][k] * dG[4 + c] + ph.M[2][k] * dG[8 + c];
            }
        const double muj = ph.mu * ph.J, kap = kGamm1Prndtli * muj;
        double t[3][3], dt[3][3];
        const double div = 2.0 / 3.0 * (dx[0][0] + dx[1][1] + dx[2][2]);
        const double ddiv = 2.0 / 3.0 * (ddx[0][0] + ddx[1][1] + ddx[2][2]);
        for (int i = 0; i < 3; ++i)
            for (int k = 0; k < 3; ++k) {
                t[i][k] = muj * (dx[i][k] + dx[k][i]) - (i == k ? muj * div : 0.0);
                dt[i][k] = muj * (ddx[i][k] + ddx[k][i]) - (i == k ? muj * ddiv : 0.0);
            }
        const double uu[3] = {u, v, w}, duu[3] = {du, dv, dw};
        for (int i = 0; i < 3; ++i) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += Ma[k] * dt[i][k];
            dF[1 + i] -= s;
        }
        for (int k = 0; k < 3; ++k) {
            double dh = kap * ddx[3][k];
            for (int i = 0; i < 3; ++i) dh += duu[i] * t[i][k] + uu[i] * dt[i][k];
            dF[4] -= Ma[k] * dh;
        }
    }
}

// qbar += (dF/dq)^T Fb,  Gbar += (dF/dG)^T Fb
template <bool VISC>
CSB_HD void flux_adj(int a, const double q[5], const double G[12], const double Fb[5], const PointPhys &ph,
                     double qbar[5], double Gbar[12]) {
    const double ri = 1.0 / q[0];
    const double u = q[1] * ri, v = q[2] * ri, w = q[3] * ri;
    const double mm = q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
    const double p = kGamm1 * (q[4] - 0.5 * (q[1] * u + q[2] * v + q[3] * w));
    const double *Ma = ph.M[a];
    const double ss = Ma[0] * (u + ph.umf[0]) + Ma[1] * (v + ph.umf[1]) + Ma[2] * (w + ph.umf[2]);
    const double mu_dot = ph.umf[0] * Ma[0] + ph.umf[1] * Ma[1] + ph.umf[2] * Ma[2];
    double ub[3] = {0.0, 0.0, 0.0};
    if (VISC) {
        double dx[4][3];
        for (int c = 0; c < 4; ++c)
            for (int k = 0; k < 3; ++k)
                dx[c][k] = ph.M[0][k] * G[c] + ph.M[1][k] * G[4 + c] + ph.M[2][k] * G[8 + c];
        const double muj = ph.mu * ph.J, kap = kGamm1Prndtli * muj;
        const double div = 2.0 / 3.0 * (dx[0][0] + dx[1][1] + dx[2][2]);
        double t[3][3];
        for (int i = 0; i < 3; ++i)
            for (int k = 0; k < 3; ++k) t[i][k] = muj * (dx[i][k] + dx[k][i]) - (i == k ? muj * div : 0.0);
        const double uu[3] = {u, v, w};
        // F4 -= sum_k Ma[k] h_k,  h_k = kap dx[3][k] + sum_i u_i t[i][k]
        // F(1+i) -= sum_k Ma[k] t[i][k]
        double tb[3][3], dxb[4][3];
        for (int c = 0; c < 4; ++c)
            for (int k = 0; k < 3; ++k) dxb[c][k] = 0.0;
        for (int k = 0; k < 3; ++k) {
            const double hb = -Ma[k] * Fb[4];
            dxb[3][k] += kap * hb;
            for (int i = 0; i < 3; ++i) {
                ub[i] += t[i][k] * hb;
                tb[i][k] = uu[i] * hb - Ma[k] * Fb[1 + i];
            }
        }
        // t[i][k] = muj (dx[i][k] + dx[k][i]) - [i==k] muj div
        double divb = 0.0;
        for (int i = 0; i < 3; ++i)
            for (int k = 0; k < 3; ++k) {
                dxb[i][k] += muj * tb[i][k];
                dxb[k][i] += muj * tb[i][k];
                if (i == k) divb -= muj * tb[i][k];
            }
        for (int i = 0; i < 3; ++i) dxb[i][i] += 2.0 / 3.0 * divb;
        // dx[c][k] = sum_b M[b][k] G[b*4 + c]
        for (int b = 0; b < 3; ++b)
            for (int c = 0; c < 4; ++c) {
                double s = 0.0;
                for (int k = 0; k < 3; ++k) s += ph.M[b][k] * dxb[c][k];
                Gbar[b * 4 + c] += s;
            }
    }
    // inviscid part
    // F0 = q0 ss; F(1+i) = q(1+i) ss + Ma[i] p; F4 = (q4 + p) ss - p mu_dot
    double ssb = q[0] * Fb[0] + q[1] * Fb[1] + q[2] * Fb[2] + q[3] * Fb[3] + (q[4] + p) * Fb[4];
    const double pb = Ma[0] * Fb[1] + Ma[1] * Fb[2] + Ma[2] * Fb[3] + (ss - mu_dot) * Fb[4];
    qbar[0] += ss * Fb[0];
    qbar[1] += ss * Fb[1];
    qbar[2] += ss * Fb[2];
    qbar[3] += ss * Fb[3];
    qbar[4] += ss * Fb[4];
    // ss = sum_k Ma[k] (u_k + umf_k)
    ub[0] += Ma[0] * ssb;
    ub[1] += Ma[1] * ssb;
    ub[2] += Ma[2] * ssb;
    // p = (g-1)(q4 - 0.5 mm ri)
    qbar[4] += kGamm1 * pb;
    const double mmb = -0.5 * kGamm1 * ri * pb;
    double rib = -0.5 * kGamm1 * mm * pb;
    qbar[1] += 2.0 * q[1] * mmb;
    qbar[2] += 2.0 * q[2] * mmb;
    qbar[3] += 2.0 * q[3] * mmb;
    // u_i = q(1+i) ri
    for (int i = 0; i < 3; ++i) {
        qbar[1 + i] += ri * ub[i];
        rib += q[1 + i] * ub[i];
    }
    qbar[0] += -ri * ri * rib;
}

#undef CSB_HD

}  // namespace csb

namespace csb {

// Forward-mode dual number (value, one directional derivative) for the
// face-local GCBC linearization.
struct Dual {
    double v, d;
};
__host__ __device__ __forceinline__ Dual dual(double v, double d = 0.0) { return Dual{v, d}; }
__host__ __device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__host__ __device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__host__ __device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__host__ __device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__host__ __device__ __forceinline__ Dual operator*(double s, Dual a) { return {s * a.v, s * a.d}; }
__host__ __device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    const double iv = 1.0 / b.v;
    return {a.v * iv, (a.d - a.v * iv * b.d) * iv};
}
__host__ __device__ __forceinline__ Dual dsqrt(Dual a) {
    const double s = sqrt(a.v);
    return {s, 0.5 * a.d / s};
}

// Non-reflective GCBC correction of the RHS at one x-face point (the
// arithmetic of k_gcbc_x: characteristic amplitudes of the two acoustic waves
// from r = d/dxi F_x at the point, incoming ones removed, mapped back to
// conservative variables, scaled by 1/J), on dual numbers.  The wave
// selection is taken from the values.
__host__ __device__ __forceinline__ void gcbc_point(const Dual q[5], const Dual r[5], const double c[3],
                                                    const PointPhys &ph, int ip, Dual out[5]) {
    const Dual rho = q[0], rhoi = dual(1.0) / rho;
    const Dual ve[3] = {q[1] * rhoi, q[2] * rhoi, q[3] * rhoi};
    const Dual hv2 = 0.5 * (ve[0] * ve[0] + ve[1] * ve[1] + ve[2] * ve[2]);
    const Dual pp = kGamm1 * (q[4] - rho * hv2);
    const Dual ao = dsqrt(kGam * (rhoi * pp)), aoi = dual(1.0) / ao;
    const Dual vn = c[0] * ve[0] + c[1] * ve[1] + c[2] * ve[2];
    const double vs = c[0] * ph.umf[0] + c[1] * ph.umf[1] + c[2] * ph.umf[2];
    Dual dr[5];
    for (int v = 0; v < 5; ++v) dr[v] = ph.J * r[v];
    const Dual ho = kGamm1 * (aoi * aoi), bo = dual(1.0) - ho * hv2, co = aoi * vn;
    const Dual dm[3] = {c[0] * aoi, c[1] * aoi, c[2] * aoi};
    const Dual rv[3] = {ho * ve[0], ho * ve[1], ho * ve[2]};
    const Dual cha3 = (dual(1.0) - bo - co) * dr[0] + (dm[0] - rv[0]) * dr[1] + (dm[1] - rv[1]) * dr[2] +
                      (dm[2] - rv[2]) * dr[3] + ho * dr[4];
    const Dual cha4 = (dual(1.0) - bo + co) * dr[0] + (-dm[0] - rv[0]) * dr[1] + (-dm[1] - rv[1]) * dr[2] +
                      (-dm[2] - rv[2]) * dr[3] + ho * dr[4];
    const double ra0 = 1.0 - 2.0 * ip;
    const Dual d3 = ra0 * (vn.v + vs + ao.v) > 0 ? -cha3 : dual(0.0);
    const Dual d4 = ra0 * (vn.v + vs - ao.v) > 0 ? -cha4 : dual(0.0);
    const Dual bo2 = hv2 + kHamm1 * (ao * ao), co2 = ao * vn;
    const Dual em[3] = {c[0] * ao, c[1] * ao, c[2] * ao};
    const double sb = 1.0 / ph.J;
    out[0] = sb * (0.5 * d3 + 0.5 * d4);
    for (int k = 0; k < 3; ++k) {
        const Dual s3 = 0.5 * (ve[k] + em[k]);
        out[1 + k] = sb * (s3 * d3 + (s3 - em[k]) * d4);
    }
    const Dual s3 = 0.5 * (bo2 + co2);
    out[4] = sb * (s3 * d3 + (s3 - co2) * d4);
}

// Unit normal of the x faces from the metric row grad(xi).
__host__ __device__ __forceinline__ void xface_normal(const PointPhys &ph, double c[3]) {
    const double nrm = sqrt(ph.M[0][0] * ph.M[0][0] + ph.M[0][1] * ph.M[0][1] + ph.M[0][2] * ph.M[0][2]);
    c[0] = ph.M[0][0] / nrm;
    c[1] = ph.M[0][1] / nrm;
    c[2] = ph.M[0][2] / nrm;
}

}  // namespace csb
