// physics.cu -- the reference-shaped (unfused) physics path over the C ABI:
// physics::calc_fluxes, physics::calc_viscous_shear_stress,
// physics::calc_time_step (src/physics_pc.hpp:83-256) and gcbc_go
// (src/gcbc.hpp:86-186) with per-point metric arrays, for drop-in callers
// that hold the reference's buffers.  Line solves go through cs_deriv with
// the numerics object's interface buffers (fill_buffers -> single-rank halo
// exchange -> deriv2d), exactly the reference's data flow.  The fused solver
// (fused.cu) is the fast path; this file is the compatibility path.
#include <cmath>
#include <cstring>

#include "context.h"
#include "line_solver.cuh"

struct cs_physics {
    cs_dcomp d{};
    int viscous = 1;
    double umf[3] = {0.0, 0.0, 0.0};
    double *buffer = nullptr;        // [5][3][lmx] fluxes (calc_fluxes) / u,v,w,T (viscous)
    double *buffer_deriv = nullptr;  // [5][3][lmx]
    double *tau = nullptr;           // [6][lmx] xx, yy, zz, xy, yz, zx
    double *heat = nullptr;          // [3][lmx]
    double *ss = nullptr;            // [3][lmx] temperature gradient
    double *dt_acc = nullptr;        // [2]
};

namespace csb {

// calc_fluxes_pre_compute_kernel<Visc> (src/cuda/kernels/physics.hpp:42-193),
// operation order of the reference twin (tests/test_physics_serial.cu:41-163).
template <bool VISC>
__global__ void k_fluxes_pre(double *__restrict__ buf, const double *__restrict__ qa,
                             const double *__restrict__ p, double *__restrict__ de,
                             const double *__restrict__ xim, const double *__restrict__ etm,
                             const double *__restrict__ zem, const double *__restrict__ tau,
                             const double *__restrict__ heat, double u0, double u1, double u2, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double M[3][3] = {{xim[i], xim[n + i], xim[2 * n + i]},
                            {etm[i], etm[n + i], etm[2 * n + i]},
                            {zem[i], zem[n + i], zem[2 * n + i]}};
    const double rr0 = de[n + i] + u0, rr1 = de[2 * n + i] + u1, rr2 = de[3 * n + i] + u2;
    double ss[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) ss[a] = xmul(M[a][0], rr0) + xmul(M[a][1], rr1) + xmul(M[a][2], rr2);
    const double pp = p[i];
    double t[6] = {0, 0, 0, 0, 0, 0}, h[3] = {0, 0, 0};
    if (VISC) {
#pragma unroll
        for (int c = 0; c < 6; ++c) t[c] = tau[c * n + i];
#pragma unroll
        for (int c = 0; c < 3; ++c) h[c] = heat[c * n + i];
    }
    const double tr[3][3] = {{t[0], t[3], t[5]}, {t[3], t[1], t[4]}, {t[5], t[4], t[2]}};
#pragma unroll
    for (int a = 0; a < 3; ++a) buf[a * n + i] = xmul(qa[i], ss[a]);
#pragma unroll
    for (int m = 1; m <= 3; ++m)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double v = xmul(qa[m * n + i], ss[a]) + xmul(M[a][m - 1], pp);
            if (VISC) v -= xmul(M[a][0], tr[m - 1][0]) + xmul(M[a][1], tr[m - 1][1]) + xmul(M[a][2], tr[m - 1][2]);
            buf[(m * 3 + a) * n + i] = v;
        }
    const double h0 = qa[4 * n + i] + pp;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        double v = xmul(h0, ss[a]) - xmul(pp, xmul(u0, M[a][0]) + xmul(u1, M[a][1]) + xmul(u2, M[a][2]));
        if (VISC) v -= xmul(M[a][0], h[0]) + xmul(M[a][1], h[1]) + xmul(M[a][2], h[2]);
        buf[(12 + a) * n + i] = v;
    }
    de[4 * n + i] = h0;
}

// calc_fluxes_post_compute_kernel<m> (src/cuda/kernels/physics.hpp:195-209), all m.
__global__ void k_fluxes_post(double *__restrict__ de, const double *__restrict__ bd, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int m = 0; m < 5; ++m) de[m * n + i] = bd[(m * 3) * n + i] + bd[(m * 3 + 1) * n + i] + bd[(m * 3 + 2) * n + i];
}

// calc_viscous_shear_stress_init_kernel (physics.hpp:211-225).
__global__ void k_visc_init(double *__restrict__ buf, const double *__restrict__ de, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int m = 1; m < 5; ++m) buf[(m * 3) * n + i] = de[m * n + i];
}

// calc_viscous_shear_stress_post_compute_kernel<m> (physics.hpp:228-283),
// applied to the derivatives (the reference passes the underived buffer).
__global__ void k_visc_post(double *__restrict__ tau, double *__restrict__ heat, double *__restrict__ ss,
                            const double *__restrict__ bd, const double *__restrict__ xim,
                            const double *__restrict__ etm, const double *__restrict__ zem, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double *out[5][3] = {{nullptr, nullptr, nullptr},
                         {tau, heat + 2 * n, tau + 5 * n},
                         {tau + 3 * n, tau + 1 * n, heat},
                         {heat + 1 * n, tau + 4 * n, tau + 2 * n},
                         {ss, ss + n, ss + 2 * n}};
#pragma unroll
    for (int m = 1; m < 5; ++m) {
        const double g0 = bd[(m * 3) * n + i], g1 = bd[(m * 3 + 1) * n + i], g2 = bd[(m * 3 + 2) * n + i];
#pragma unroll
        for (int k = 0; k < 3; ++k)
            out[m][k][i] = xmul(xim[k * n + i], g0) + xmul(etm[k * n + i], g1) + xmul(zem[k * n + i], g2);
    }
}

// calc_viscous_shear_stress_final_kernel (physics.hpp:285-333), including its
// side effects on de (de0 <- ssk, de4 <- 2/3 div).
__global__ void k_visc_final(double *__restrict__ de, double *__restrict__ tau, double *__restrict__ heat,
                             const double *__restrict__ ss, const double *__restrict__ ssk,
                             const double *__restrict__ yaco, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double muj = xmul(ssk[i], yaco[i]);
    const double kap = xmul(kGamm1Prndtli, muj);
    const double ux = tau[i], vy = tau[n + i], wz = tau[2 * n + i];
    const double vx = tau[3 * n + i], wy = tau[4 * n + i], uz = tau[5 * n + i];
    const double vz = heat[i], wx = heat[n + i], uy = heat[2 * n + i];
    const double div = xmul(2.0 / 3.0, ux + vy + wz);
    const double txx = xmul(muj, xmul(2.0, ux) - div), tyy = xmul(muj, xmul(2.0, vy) - div);
    const double tzz = xmul(muj, xmul(2.0, wz) - div);
    const double txy = xmul(muj, vx + uy), tyz = xmul(muj, wy + vz), tzx = xmul(muj, uz + wx);
    const double u = de[n + i], v = de[2 * n + i], w = de[3 * n + i];
    tau[i] = txx; tau[n + i] = tyy; tau[2 * n + i] = tzz;
    tau[3 * n + i] = txy; tau[4 * n + i] = tyz; tau[5 * n + i] = tzx;
    heat[i] = xmul(kap, ss[i]) + xmul(u, txx) + xmul(v, txy) + xmul(w, tzx);
    heat[n + i] = xmul(kap, ss[n + i]) + xmul(u, txy) + xmul(v, tyy) + xmul(w, tyz);
    heat[2 * n + i] = xmul(kap, ss[2 * n + i]) + xmul(u, tzx) + xmul(v, tyz) + xmul(w, tzz);
    de[i] = ssk[i];
    de[4 * n + i] = div;
}

// calc_time_step_kernel (physics.hpp:335-427): two maxima, reduced with a
// warp shuffle and an integer atomic max on the non-negative bit patterns.
__global__ void k_time_step(const double *__restrict__ xim, const double *__restrict__ etm,
                            const double *__restrict__ zem, const double *__restrict__ de,
                            const double *__restrict__ yaco, const double *__restrict__ ssk,
                            double u0, double u1, double u2, unsigned long long *__restrict__ acc, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double m1 = 0.0, m2 = 0.0;
    if (i < n) {
        double M[3][3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            M[0][c] = xim[c * n + i];
            M[1][c] = etm[c * n + i];
            M[2][c] = zem[c * n + i];
        }
        double rr1 = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int c = 0; c < 3; ++c) rr1 += xmul(M[a][c], M[a][c]);
        double rr2 = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a)
            rr2 += fabs(xmul(M[a][0], de[n + i] + u0) + xmul(M[a][1], de[2 * n + i] + u1) +
                        xmul(M[a][2], de[3 * n + i] + u2));
        const double ssi = fabs(yaco[i]);
        m1 = xmul(sqrt(xmul(de[4 * n + i], rr1)) + rr2, ssi);
        m2 = de[i] * ssk[i] * rr1 * ssi * ssi;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
        m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(acc, (unsigned long long)__double_as_longlong(m1));
        atomicMax(acc + 1, (unsigned long long)__double_as_longlong(m2));
    }
}

// GCBC on any face with per-point arrays: gcbc_setup_kernel (flag = 1 for
// non-reflective) + gcbc_update_non_reflective_kernel
// (src/cuda/kernels/gcbc.hpp:251-454; defects fixed as in the oracle).
template <int AXIS>
__global__ void k_gcbc_face(double *__restrict__ de, const double *__restrict__ drva,
                            const double *__restrict__ cm, const double *__restrict__ qa,
                            const double *__restrict__ p, const double *__restrict__ yaco,
                            const double *__restrict__ sbcc, double u0, double u1, double u2, int lxi,
                            int let, int lze, int ip) {
    const int64_t n = (int64_t)lxi * let * lze;
    const int64_t F = AXIS == 0 ? (int64_t)let * lze : (AXIS == 1 ? (int64_t)lxi * lze : (int64_t)lxi * let);
    const int64_t fi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (fi >= F) return;
    int64_t base, stride;
    int dim;
    if (AXIS == 0) { base = fi * lxi; stride = 1; dim = lxi; }
    else if (AXIS == 1) { base = (fi / lxi) * (int64_t)lxi * let + fi % lxi; stride = lxi; dim = let; }
    else { base = fi; stride = (int64_t)lxi * let; dim = lze; }
    const int64_t idx = base + (int64_t)(ip ? dim - 1 : 0) * stride;
    const double c[3] = {cm[(ip * 3 + 0) * F + fi], cm[(ip * 3 + 1) * F + fi], cm[(ip * 3 + 2) * F + fi]};
    const double rho = qa[idx], rhoi = 1.0 / rho;
    const double ve[3] = {xmul(qa[n + idx], rhoi), xmul(qa[2 * n + idx], rhoi), xmul(qa[3 * n + idx], rhoi)};
    const double hv2 = xmul(0.5, xmul(ve[0], ve[0]) + xmul(ve[1], ve[1]) + xmul(ve[2], ve[2]));
    const double pp = p[idx];
    const double ao = sqrt(xmul(xmul(kGam, rhoi), pp)), aoi = 1.0 / ao;
    const double vn = xmul(c[0], ve[0]) + xmul(c[1], ve[1]) + xmul(c[2], ve[2]);
    const double vs = xmul(c[0], u0) + xmul(c[1], u1) + xmul(c[2], u2);
    double dr[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) dr[v] = xmul(yaco[idx], drva[(int64_t)(ip * 5 + v) * F + fi]);
    const double ho = xmul(xmul(kGamm1, aoi), aoi), bo = 1.0 - xmul(ho, hv2), co = xmul(aoi, vn);
    const double dm[3] = {xmul(aoi, c[0]), xmul(aoi, c[1]), xmul(aoi, c[2])};
    const double rv[3] = {xmul(ho, ve[0]), xmul(ho, ve[1]), xmul(ho, ve[2])};
    const double cha3 = xmul(1.0 - bo - co, dr[0]) + xmul(dm[0] - rv[0], dr[1]) + xmul(dm[1] - rv[1], dr[2]) +
                        xmul(dm[2] - rv[2], dr[3]) + xmul(ho, dr[4]);
    const double cha4 = xmul(1.0 - bo + co, dr[0]) + xmul(-dm[0] - rv[0], dr[1]) + xmul(-dm[1] - rv[1], dr[2]) +
                        xmul(-dm[2] - rv[2], dr[3]) + xmul(ho, dr[4]);
    const double ra0 = 1.0 - 2.0 * ip;
    const double d3 = ra0 * (vn + vs + ao) > 0 ? -cha3 : 0.0;
    const double d4 = ra0 * (vn + vs - ao) > 0 ? -cha4 : 0.0;
    const double bo2 = hv2 + xmul(xmul(kHamm1, ao), ao), co2 = xmul(ao, vn);
    const double em[3] = {xmul(ao, c[0]), xmul(ao, c[1]), xmul(ao, c[2])};
    double dq[5];
    dq[0] = xmul(0.5, d3) + xmul(0.5, d4);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double s3 = xmul(0.5, ve[k] + em[k]);
        dq[1 + k] = xmul(s3, d3) + xmul(s3 - em[k], d4);
    }
    {
        const double s3 = xmul(0.5, bo2 + co2);
        dq[4] = xmul(s3, d3) + xmul(s3 - co2, d4);
    }
    const int iq = 1 - 2 * ip;
    for (int ii = 0; ii < kMbci && ii < dim; ++ii) {
        const int64_t o = idx + (int64_t)ii * iq * stride;
#pragma unroll
        for (int v = 0; v < 5; ++v) de[v * n + o] += xmul(sbcc[o], dq[v]);
    }
}

// Characteristic state of one face point (gcbc_vgpr::eleme,
// src/cuda/kernels/gcbc.hpp:43-57) and the two transformation matrices
// (xtr2q :59-107, xtq2r :109-150 with its typos fixed: dm[2] = aoi c[2],
// xt[0][4] = -ho c[0], xt[4][0] = 1 - bo + co), in the oracle's operation order.
struct GcPt {
    double c[3], ve[3], hv2, ao, aoi, vn, vs;
};
__device__ __forceinline__ GcPt gc_eleme(const double c[3], double rho, double m0, double m1, double m2, double pp,
                                         double u0, double u1, double u2) {
    GcPt g;
    const double rhoi = 1.0 / rho;
#pragma unroll
    for (int k = 0; k < 3; ++k) g.c[k] = c[k];
    g.ao = sqrt(xmul(xmul(kGam, rhoi), pp));
    g.aoi = 1.0 / g.ao;
    g.ve[0] = xmul(rhoi, m0);
    g.ve[1] = xmul(rhoi, m1);
    g.ve[2] = xmul(rhoi, m2);
    g.hv2 = xmul(0.5, xmul(g.ve[0], g.ve[0]) + xmul(g.ve[1], g.ve[1]) + xmul(g.ve[2], g.ve[2]));
    g.vn = xmul(c[0], g.ve[0]) + xmul(c[1], g.ve[1]) + xmul(c[2], g.ve[2]);
    g.vs = xmul(c[0], u0) + xmul(c[1], u1) + xmul(c[2], u2);
    return g;
}
__device__ __forceinline__ void gc_xtq2r(const GcPt &g, double L[5][5]) {
    const double *c = g.c, *ve = g.ve;
    const double ho = xmul(xmul(kGamm1, g.aoi), g.aoi), bo = 1.0 - xmul(ho, g.hv2), co = xmul(g.aoi, g.vn);
    const double dm[3] = {xmul(g.aoi, c[0]), xmul(g.aoi, c[1]), xmul(g.aoi, c[2])};
    const double rv[3] = {xmul(ho, ve[0]), xmul(ho, ve[1]), xmul(ho, ve[2])};
    L[0][0] = xmul(bo, c[0]) + xmul(dm[1], ve[2]) - xmul(dm[2], ve[1]);
    L[0][1] = xmul(c[0], rv[0]);
    L[0][2] = xmul(c[0], rv[1]) + dm[2];
    L[0][3] = xmul(c[0], rv[2]) - dm[1];
    L[0][4] = xmul(-ho, c[0]);
    L[1][0] = xmul(bo, c[1]) + xmul(dm[2], ve[0]) - xmul(dm[0], ve[2]);
    L[1][1] = xmul(c[1], rv[0]) - dm[2];
    L[1][2] = xmul(c[1], rv[1]);
    L[1][3] = xmul(c[1], rv[2]) + dm[0];
    L[1][4] = xmul(-ho, c[1]);
    L[2][0] = xmul(bo, c[2]) + xmul(dm[0], ve[1]) - xmul(dm[1], ve[0]);
    L[2][1] = xmul(c[2], rv[0]) + dm[1];
    L[2][2] = xmul(c[2], rv[1]) - dm[0];
    L[2][3] = xmul(c[2], rv[2]);
    L[2][4] = xmul(-ho, c[2]);
    L[3][0] = 1.0 - bo - co;
    L[3][1] = dm[0] - rv[0];
    L[3][2] = dm[1] - rv[1];
    L[3][3] = dm[2] - rv[2];
    L[3][4] = ho;
    L[4][0] = 1.0 - bo + co;
    L[4][1] = -dm[0] - rv[0];
    L[4][2] = -dm[1] - rv[1];
    L[4][3] = -dm[2] - rv[2];
    L[4][4] = ho;
}
__device__ __forceinline__ void gc_xtr2q(const GcPt &g, double S[5][5]) {
    const double *c = g.c, *ve = g.ve;
    const double bo = g.hv2 + xmul(xmul(kHamm1, g.ao), g.ao), co = xmul(g.ao, g.vn);
    const double dm[3] = {xmul(g.ao, c[0]), xmul(g.ao, c[1]), xmul(g.ao, c[2])};
    S[0][0] = c[0];
    S[0][1] = c[1];
    S[0][2] = c[2];
    S[0][3] = 0.5;
    S[0][4] = 0.5;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int k1 = (k + 1) % 3, k2 = (k + 2) % 3;
        // row 1 + k: c[j] ve[k] plus the rotation part +-dm[k1], +-dm[k2]
        S[1 + k][k] = xmul(c[k], ve[k]);
        S[1 + k][3] = xmul(0.5, ve[k] + dm[k]);
        S[1 + k][4] = xmul(0.5, ve[k] + dm[k]) - dm[k];
        S[1 + k][k1] = xmul(c[k1], ve[k]) - dm[k2];
        S[1 + k][k2] = xmul(c[k2], ve[k]) + dm[k1];
    }
    S[4][0] = xmul(g.hv2, c[0]) + xmul(dm[2], ve[1]) - xmul(dm[1], ve[2]);
    S[4][1] = xmul(g.hv2, c[1]) + xmul(dm[0], ve[2]) - xmul(dm[2], ve[0]);
    S[4][2] = xmul(g.hv2, c[2]) + xmul(dm[1], ve[0]) - xmul(dm[0], ve[1]);
    S[4][3] = xmul(0.5, bo + co);
    S[4][4] = xmul(0.5, bo + co) - co;
}
__device__ __forceinline__ void gc_matvec(const double A[5][5], const double *x, double *y) {
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < 5; ++k) v += xmul(A[r][k], x[k]);
        y[r] = v;
    }
}

// Face point fi of face ip along AXIS (the derivative's drva face index) and
// the stride into the block.
template <int AXIS>
__device__ __forceinline__ int64_t gc_point(int64_t fi, int ip, int lxi, int let, int lze, int64_t &stride,
                                            int &dim) {
    int64_t base;
    if (AXIS == 0) { base = fi * lxi; stride = 1; dim = lxi; }
    else if (AXIS == 1) { base = (fi / lxi) * (int64_t)lxi * let + fi % lxi; stride = lxi; dim = let; }
    else { base = fi; stride = (int64_t)lxi * let; dim = lze; }
    return base + (int64_t)(ip ? dim - 1 : 0) * stride;
}

// gcbc_setup_kernel (src/cuda/kernels/gcbc.hpp:251-342): drva of face ip in
// place into characteristic form, from drva (flag, non-reflective faces) or
// from the full right-hand side de (walls, curvilinear interfaces), times J.
template <int AXIS>
__global__ void k_gc_setup(double *__restrict__ drva, const double *__restrict__ cm, const double *__restrict__ qa,
                           const double *__restrict__ de, const double *__restrict__ p,
                           const double *__restrict__ yaco, double u0, double u1, double u2, int ip, int flag,
                           int lxi, int let, int lze) {
    const int64_t n = (int64_t)lxi * let * lze;
    const int64_t F = AXIS == 0 ? (int64_t)let * lze : (AXIS == 1 ? (int64_t)lxi * lze : (int64_t)lxi * let);
    const int64_t fi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (fi >= F) return;
    int64_t stride;
    int dim;
    const int64_t idx = gc_point<AXIS>(fi, ip, lxi, let, lze, stride, dim);
    const double c[3] = {cm[(ip * 3 + 0) * F + fi], cm[(ip * 3 + 1) * F + fi], cm[(ip * 3 + 2) * F + fi]};
    const GcPt g = gc_eleme(c, qa[idx], qa[n + idx], qa[2 * n + idx], qa[3 * n + idx], p[idx], u0, u1, u2);
    double L[5][5], src[5], cha[5];
    gc_xtq2r(g, L);
#pragma unroll
    for (int v = 0; v < 5; ++v) src[v] = xmul(yaco[idx], flag ? drva[(ip * 5 + v) * F + fi] : de[v * n + idx]);
    gc_matvec(L, src, cha);
#pragma unroll
    for (int v = 0; v < 5; ++v) drva[(ip * 5 + v) * F + fi] = cha[v];
}

// The update kernels (src/cuda/kernels/gcbc.hpp:344-695) for one face:
// kind 0 non-reflective (incoming acoustic waves zeroed), 1 wall (incoming
// acoustic wave reflected from the outgoing one with the frame acceleration
// and the normal velocity relaxed at rate dtwi), 2 curvilinear interface
// (incoming waves from the neighbour's drvb).  de += sbcc xtr2q (cha - drva)
// on kMbci planes; the wall update subtracts drva like the other two (the
// reference's wall kernel adds xtr2q cha, the whole right-hand side).
template <int AXIS>
__global__ void k_gc_update(int kind, const double *__restrict__ drva, const double *__restrict__ drvb,
                            const double *__restrict__ cm, const double *__restrict__ qa, double *__restrict__ de,
                            const double *__restrict__ p, const double *__restrict__ sbcc, double u0, double u1,
                            double u2, double a0, double a1, double a2, double dtwi, int ip, int lxi, int let,
                            int lze) {
    const int64_t n = (int64_t)lxi * let * lze;
    const int64_t F = AXIS == 0 ? (int64_t)let * lze : (AXIS == 1 ? (int64_t)lxi * lze : (int64_t)lxi * let);
    const int64_t fi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (fi >= F) return;
    int64_t stride;
    int dim;
    const int64_t idx = gc_point<AXIS>(fi, ip, lxi, let, lze, stride, dim);
    const double c[3] = {cm[(ip * 3 + 0) * F + fi], cm[(ip * 3 + 1) * F + fi], cm[(ip * 3 + 2) * F + fi]};
    const double rho = qa[idx];
    const GcPt g = gc_eleme(c, rho, qa[n + idx], qa[2 * n + idx], qa[3 * n + idx], p[idx], u0, u1, u2);
    double dr[5], cha[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) cha[v] = dr[v] = drva[(ip * 5 + v) * F + fi];
    const double ra0 = 1.0 - 2.0 * ip;
    if (kind == 0) {
        if (ra0 * (g.vn + g.vs + g.ao) > 0) cha[3] = 0.0;
        if (ra0 * (g.vn + g.vs - g.ao) > 0) cha[4] = 0.0;
    } else if (kind == 2) {
        double dh[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) dh[v] = drvb[(ip * 5 + v) * F + fi];
        if (ra0 * (g.vn + g.vs) > 0) { cha[0] = dh[0]; cha[1] = dh[1]; cha[2] = dh[2]; }
        if (ra0 * (g.vn + g.vs + g.ao) > 0) cha[3] = dh[3];
        if (ra0 * (g.vn + g.vs - g.ao) > 0) cha[4] = dh[4];
    } else {
        const double acc = xmul(c[0], a0) + xmul(c[1], a1) + xmul(c[2], a2);
        const double w = xmul(xmul(xmul(2.0, ra0), g.aoi), rho);
        if (ip == 0) cha[3] = cha[4] + xmul(w, acc + xmul(dtwi, g.vn + g.vs));
        else cha[4] = cha[3] + xmul(w, acc + xmul(dtwi, g.vn + g.vs));
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) cha[v] -= dr[v];
    double S[5][5], dq[5];
    gc_xtr2q(g, S);
    gc_matvec(S, cha, dq);
    const int iq = 1 - 2 * ip;
    for (int ii = 0; ii < kMbci && ii < dim; ++ii) {
        const int64_t o = idx + (int64_t)ii * iq * stride;
#pragma unroll
        for (int v = 0; v < 5; ++v) de[v * n + o] += xmul(sbcc[o], dq[v]);
    }
}

// Primitive recovery into the reference's de slots (the empty slot of the
// driver, driver/canard.cu:142-143): de0 = 1/rho, de1..3 = u, v, w,
// de4 = gamma p / rho (c^2, the CANARD temperature), p.
__global__ void k_thermo(const double *__restrict__ q, double *__restrict__ de, double *__restrict__ p,
                         int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double q1 = q[n + i], q2 = q[2 * n + i], q3 = q[3 * n + i];
    const double ri = 1.0 / q[i];
    const double u = xmul(q1, ri), v = xmul(q2, ri), w = xmul(q3, ri);
    const double pp = xmul(kGamm1, q[4 * n + i] - xmul(0.5, xmul(q1, u) + xmul(q2, v) + xmul(q3, w)));
    de[i] = ri;
    de[n + i] = u;
    de[2 * n + i] = v;
    de[3 * n + i] = w;
    de[4 * n + i] = xmul(xmul(kGam, pp), ri);
    p[i] = pp;
}

// Conserved-variable update that physics_base::movef leaves empty
// (src/physics_base.hpp:147-150): q = q^n - dtk * J * de.
__global__ void k_rk_update(const double *__restrict__ qn, const double *__restrict__ de,
                            const double *__restrict__ yaco, double dtk, double *__restrict__ qout, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double s = xmul(dtk, yaco[i]);
#pragma unroll
    for (int v = 0; v < 5; ++v) qout[v * n + i] = qn[v * n + i] - xmul(s, de[v * n + i]);
}

static int check_physics(const cs_physics *ph, const cs_numerics *nm, const cs_dcomp &d) {
    if (!ph) return set_error(CS_ERR_INVALID, "null physics object");
    if (d.lmx != ph->d.lmx || d.lxi != ph->d.lxi || d.let != ph->d.let || d.lze != ph->d.lze)
        return set_error(CS_ERR_INVALID, "dims differ from the physics object");
    if (nm) {
        int ndf[2][3];
        if (cs_get_ndf(nm, ndf)) return CS_ERR_INVALID;
    }
    return CS_OK;
}

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace csb

using namespace csb;

// Wall boundary state update at one face plane (wall_inviscid_kernel /
// wall_viscous_kernel, src/cuda/kernels/gcbc.hpp:160-249): points with
// npex == 0 get, inviscid, rho E = rho^gamma / (gamma (gamma-1)) + |m|^2 / (2 rho)
// (isentropic pressure, momentum kept); viscous, m = -rho umf and
// rho E = rho / (gamma (gamma-1)) + |m|^2 / (2 rho) with the updated m
// (isothermal wall, T = 1).  plane = ip * (n - 1).
__global__ void k_wall_face(double *__restrict__ q, const int *__restrict__ npex, double u0, double u1, double u2,
                            int lxi, int let, int64_t lmx, int axis, int plane, int viscous, int64_t nf) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nf) return;
    int64_t idx;
    if (axis == 0) idx = plane + (int64_t)lxi * t;                                   // t = j + let k
    else if (axis == 1) idx = t % lxi + (int64_t)lxi * (plane + (int64_t)let * (t / lxi));  // t = i + lxi k
    else idx = t + (int64_t)lxi * let * plane;                                       // t = i + lxi j
    if (npex[idx] != 0) return;
    const double hamhamm1 = (1.0 / kGam) * kHamm1;
    const double rho = q[idx];
    if (viscous) {
        q[lmx + idx] = -rho * u0;
        q[2 * lmx + idx] = -rho * u1;
        q[3 * lmx + idx] = -rho * u2;
    }
    const double m1 = q[lmx + idx], m2 = q[2 * lmx + idx], m3 = q[3 * lmx + idx];
    const double ke = 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / rho;
    q[4 * lmx + idx] = (viscous ? hamhamm1 * rho : hamhamm1 * pow(rho, kGam)) + ke;
}

extern "C" {

int cs_physics_create(cs_physics **out, cs_dcomp d, int viscous) {
    if (!out) return set_error(CS_ERR_INVALID, "null argument");
    *out = nullptr;
    if (d.lxi < 1 || d.let < 1 || d.lze < 1 || (int64_t)d.lxi * d.let * d.lze != (int64_t)d.lmx)
        return set_error(CS_ERR_INVALID, "inconsistent t_dcomp");
    auto *ph = new cs_physics();
    ph->d = d;
    ph->viscous = viscous ? 1 : 0;
    const int64_t n = d.lmx;
    bool ok = cudaMalloc(&ph->buffer, 15 * n * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&ph->buffer_deriv, 15 * n * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&ph->tau, 6 * n * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&ph->heat, 3 * n * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&ph->ss, 3 * n * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&ph->dt_acc, 2 * sizeof(double)) == cudaSuccess;
    if (!ok) {
        cs_physics_destroy(ph);
        return set_error(CS_ERR_ALLOC, "physics buffers allocation failed");
    }
    cudaMemset(ph->buffer, 0, 15 * n * sizeof(double));
    cudaMemset(ph->buffer_deriv, 0, 15 * n * sizeof(double));
    cudaMemset(ph->tau, 0, 6 * n * sizeof(double));
    cudaMemset(ph->heat, 0, 3 * n * sizeof(double));
    *out = ph;
    return CS_OK;
}

int cs_physics_destroy(cs_physics *ph) {
    if (!ph) return CS_OK;
    for (void *p : {(void *)ph->buffer, (void *)ph->buffer_deriv, (void *)ph->tau, (void *)ph->heat,
                    (void *)ph->ss, (void *)ph->dt_acc})
        if (p) cudaFree(p);
    delete ph;
    return CS_OK;
}

int cs_physics_set_umf(cs_physics *ph, const double umf[3]) {
    if (!ph || !umf) return set_error(CS_ERR_INVALID, "null argument");
    std::memcpy(ph->umf, umf, sizeof ph->umf);
    return CS_OK;
}

int cs_physics_buffers(cs_physics *ph, double **buffer, double **buffer_deriv, double **tau,
                       double **heat) {
    if (!ph) return set_error(CS_ERR_INVALID, "null argument");
    if (buffer) *buffer = ph->buffer;
    if (buffer_deriv) *buffer_deriv = ph->buffer_deriv;
    if (tau) *tau = ph->tau;
    if (heat) *heat = ph->heat;
    return CS_OK;
}

int cs_calc_fluxes_pre(cs_physics *ph, const double *qa, const double *p, double *de, const double *xim,
                       const double *etm, const double *zem, void *stream) {
    if (!ph || !qa || !p || !de || !xim || !etm || !zem) return set_error(CS_ERR_INVALID, "null argument");
    const int64_t n = ph->d.lmx;
    cudaStream_t st = (cudaStream_t)stream;
    if (ph->viscous)
        k_fluxes_pre<true><<<blocks_for(n, 256), 256, 0, st>>>(ph->buffer, qa, p, de, xim, etm, zem, ph->tau,
                                                              ph->heat, ph->umf[0], ph->umf[1], ph->umf[2], n);
    else
        k_fluxes_pre<false><<<blocks_for(n, 256), 256, 0, st>>>(ph->buffer, qa, p, de, xim, etm, zem, nullptr,
                                                               nullptr, ph->umf[0], ph->umf[1], ph->umf[2], n);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

int cs_calc_fluxes(cs_physics *ph, cs_numerics *nm, const double *qa, const double *p, double *de,
                   const double *xim, const double *etm, const double *zem, cs_dcomp d, void *stream) {
    if (int rc = check_physics(ph, nm, d)) return rc;
    if (!nm) return set_error(CS_ERR_INVALID, "null numerics object");
    if (int rc = cs_calc_fluxes_pre(ph, qa, p, de, xim, etm, zem, stream)) return rc;
    int ndf[2][3];
    cs_get_ndf(nm, ndf);
    if (int rc = cs_fill_buffers(nm, ph->buffer, 0, 5, 0, d, stream)) return rc;
    const int64_t n = d.lmx;
    for (unsigned m = 0; m < 5; ++m) {
        if (int rc = cs_halo_exchange_self(nm, m, stream)) return rc;
        for (int a = 0; a < 3; ++a) {
            if ((a == 0 ? d.lxi : (a == 1 ? d.let : d.lze)) == 1) {
                CSB_CUDA(cudaMemsetAsync(ph->buffer_deriv + (m * 3 + a) * n, 0, n * sizeof(double),
                                         (cudaStream_t)stream));
                continue;
            }
            if (int rc = cs_deriv(nm, a, ph->buffer + m * 3 * n, ph->buffer_deriv + m * 3 * n, ndf[0][a],
                                  ndf[1][a], d, m, a, a, CS_HALO_RECV, stream))
                return rc;
        }
    }
    k_fluxes_post<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(de, ph->buffer_deriv, n);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

int cs_calc_viscous_shear_stress(cs_physics *ph, cs_numerics *nm, double *de, const double *ssk,
                                 const double *xim, const double *etm, const double *zem,
                                 const double *yaco, cs_dcomp d, void *stream) {
    if (int rc = check_physics(ph, nm, d)) return rc;
    if (!nm || !de || !ssk || !xim || !etm || !zem || !yaco) return set_error(CS_ERR_INVALID, "null argument");
    const int64_t n = d.lmx;
    cudaStream_t st = (cudaStream_t)stream;
    k_visc_init<<<blocks_for(n, 256), 256, 0, st>>>(ph->buffer, de, n);
    CSB_CUDA(cudaGetLastError());
    int ndf[2][3];
    cs_get_ndf(nm, ndf);
    if (int rc = cs_fill_buffers(nm, ph->buffer, 1, 5, 1, d, stream)) return rc;
    for (unsigned m = 1; m < 5; ++m) {
        if (int rc = cs_halo_exchange_self(nm, m, stream)) return rc;
        for (int a = 0; a < 3; ++a) {
            if ((a == 0 ? d.lxi : (a == 1 ? d.let : d.lze)) == 1) {
                CSB_CUDA(cudaMemsetAsync(ph->buffer_deriv + (m * 3 + a) * n, 0, n * sizeof(double), st));
                continue;
            }
            if (int rc = cs_deriv(nm, a, ph->buffer + m * 3 * n, ph->buffer_deriv + m * 3 * n, ndf[0][a],
                                  ndf[1][a], d, m, 0, a, CS_HALO_RECV, stream))
                return rc;
        }
    }
    k_visc_post<<<blocks_for(n, 256), 256, 0, st>>>(ph->tau, ph->heat, ph->ss, ph->buffer_deriv, xim, etm, zem, n);
    k_visc_final<<<blocks_for(n, 256), 256, 0, st>>>(de, ph->tau, ph->heat, ph->ss, ssk, yaco, n);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

int cs_calc_time_step(cs_physics *ph, const double *xim, const double *etm, const double *zem,
                      const double *de, const double *yaco, const double *ssk, double cfl, double *dte,
                      size_t size, void *stream) {
    if (!ph || !xim || !etm || !zem || !de || !yaco || !ssk || !dte) return set_error(CS_ERR_INVALID, "null argument");
    if ((int64_t)size != ph->d.lmx) return set_error(CS_ERR_INVALID, "size %zu != lmx", size);
    cudaStream_t st = (cudaStream_t)stream;
    CSB_CUDA(cudaMemsetAsync(ph->dt_acc, 0, 2 * sizeof(double), st));
    k_time_step<<<blocks_for((int64_t)size, 256), 256, 0, st>>>(xim, etm, zem, de, yaco, ssk, ph->umf[0],
                                                               ph->umf[1], ph->umf[2],
                                                               (unsigned long long *)ph->dt_acc, (int64_t)size);
    CSB_CUDA(cudaGetLastError());
    double h[2];
    CSB_CUDA(cudaMemcpyAsync(h, ph->dt_acc, sizeof h, cudaMemcpyDeviceToHost, st));
    CSB_CUDA(cudaStreamSynchronize(st));
    const double a = cfl / h[0], b = 0.5 / h[1];
    *dte = a < b ? a : b;
    return CS_OK;
}

int cs_wall_condition_update(double *q, const int *npex, const double umf[3], cs_dcomp d, const int nbc[2][3],
                             void *stream) {
    if (!q || !npex || !umf || !nbc) return set_error(CS_ERR_INVALID, "null argument");
    if (d.lxi < 1 || d.let < 1 || d.lze < 1 || d.lmx != d.lxi * d.let * d.lze) return set_error(CS_ERR_INVALID, "dims");
    const int dims[3] = {d.lxi, d.let, d.lze};
    for (int a = 0; a < 3; ++a)
        for (int ip = 0; ip < 2; ++ip) {
            const int code = nbc[ip][a];
            if (code != CS_BC_WALL_INVISCID && code != CS_BC_WALL_VISCOUS) continue;
            const int64_t nf = (int64_t)d.lmx / dims[a];
            k_wall_face<<<blocks_for(nf, 256), 256, 0, (cudaStream_t)stream>>>(
                q, npex, umf[0], umf[1], umf[2], d.lxi, d.let, d.lmx, a, ip * (dims[a] - 1),
                code == CS_BC_WALL_VISCOUS ? 1 : 0, nf);
            CSB_CUDA(cudaGetLastError());
        }
    return CS_OK;
}

int cs_thermo(const double *q, double *de, double *p, size_t n, void *stream) {
    if (!q || !de || !p || n == 0) return set_error(CS_ERR_INVALID, "bad argument");
    k_thermo<<<blocks_for((int64_t)n, 256), 256, 0, (cudaStream_t)stream>>>(q, de, p, (int64_t)n);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

int cs_rk_update(const double *qn, const double *de, const double *yaco, double dtk, double *qout,
                 size_t n, void *stream) {
    if (!qn || !de || !yaco || !qout || n == 0) return set_error(CS_ERR_INVALID, "bad argument");
    k_rk_update<<<blocks_for((int64_t)n, 256), 256, 0, (cudaStream_t)stream>>>(qn, de, yaco, dtk, qout, (int64_t)n);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

int cs_gcbc_go(cs_numerics *nm, double *const cm[3], const double *qa, double *de, const double *p,
               const double *yaco, const double *sbcc, const double umf[3], cs_dcomp d, const int nbc[2][3],
               void *stream) {
    if (!nm || !cm || !qa || !de || !p || !yaco || !sbcc || !umf || !nbc) return set_error(CS_ERR_INVALID, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    for (int a = 0; a < 3; ++a) {
        const int dim = a == 0 ? d.lxi : (a == 1 ? d.let : d.lze);
        const int64_t F = a == 0 ? (int64_t)d.let * d.lze : (a == 1 ? (int64_t)d.lxi * d.lze : (int64_t)d.lxi * d.let);
        double *drva = nullptr;
        cs_get_buffers(nm, a, &drva, nullptr, nullptr);
        for (int ip = 0; ip < 2; ++ip) {
            const int np = nbc[ip][a];
            if (np == CS_BC_PERIODIC || np == CS_BC_INTER_STRAIGHT || np == CS_BC_INTER_SUBDOMAINS) continue;
            if (np != CS_BC_NON_REFLECTIVE)
                return set_error(CS_ERR_UNSUPPORTED, "cs_gcbc_go: boundary code %d (walls / curvilinear interfaces) "
                                 "needs drvb, dudtmf and dtwi: use cs_gcbc_apply", np);
            if (dim < 2) return set_error(CS_ERR_INVALID, "gcbc on a degenerate axis");
            if (!cm[a]) return set_error(CS_ERR_INVALID, "cm[%d] is null", a);
            const unsigned b = blocks_for(F, 128);
            if (a == 0) k_gcbc_face<0><<<b, 128, 0, st>>>(de, drva, cm[a], qa, p, yaco, sbcc, umf[0], umf[1], umf[2], d.lxi, d.let, d.lze, ip);
            else if (a == 1) k_gcbc_face<1><<<b, 128, 0, st>>>(de, drva, cm[a], qa, p, yaco, sbcc, umf[0], umf[1], umf[2], d.lxi, d.let, d.lze, ip);
            else k_gcbc_face<2><<<b, 128, 0, st>>>(de, drva, cm[a], qa, p, yaco, sbcc, umf[0], umf[1], umf[2], d.lxi, d.let, d.lze, ip);
            CSB_CUDA(cudaGetLastError());
        }
    }
    return CS_OK;
}

static bool gc_active(int np) {
    return np == CS_BC_NON_REFLECTIVE || np == CS_BC_WALL_INVISCID || np == CS_BC_WALL_VISCOUS ||
           np == CS_BC_INTER_CURV;
}

int cs_gcbc_apply(double *const drva[3], double *const cm[3], double *const drvb[3], const double *qa, double *de,
                  const double *p, const double *yaco, const double *sbcc, const double umf[3],
                  const double dudtmf[3], cs_dcomp d, double dtwi, const int nbc[2][3], const int mcd[2][3],
                  void *stream) {
    (void)mcd;  // single rank: every curvilinear interface pairs with the block's own opposite face
    if (!drva || !cm || !drvb || !qa || !de || !p || !yaco || !sbcc || !umf || !dudtmf || !nbc)
        return set_error(CS_ERR_INVALID, "null argument");
    if (d.lxi < 1 || d.let < 1 || d.lze < 1 || (int64_t)d.lxi * d.let * d.lze != (int64_t)d.lmx)
        return set_error(CS_ERR_INVALID, "inconsistent t_dcomp");
    cudaStream_t st = (cudaStream_t)stream;
    const int dims[3] = {d.lxi, d.let, d.lze};
    int64_t F[3] = {(int64_t)d.let * d.lze, (int64_t)d.lxi * d.lze, (int64_t)d.lxi * d.let};
    for (int a = 0; a < 3; ++a)
        for (int ip = 0; ip < 2; ++ip) {
            const int np = nbc[ip][a];
            if (!gc_active(np)) continue;
            if (dims[a] < 2) return set_error(CS_ERR_INVALID, "gcbc on a degenerate axis %d", a);
            if (!drva[a] || !cm[a]) return set_error(CS_ERR_INVALID, "drva[%d] / cm[%d] is null", a, a);
            if (np == CS_BC_INTER_CURV && !drvb[a]) return set_error(CS_ERR_INVALID, "drvb[%d] is null", a);
        }
    // 1. characteristic form of drva (gcbc_setup_kernel)
    for (int a = 0; a < 3; ++a)
        for (int ip = 0; ip < 2; ++ip) {
            const int np = nbc[ip][a];
            if (!gc_active(np)) continue;
            const int flag = np == CS_BC_NON_REFLECTIVE;
            const unsigned b = blocks_for(F[a], 128);
            if (a == 0) k_gc_setup<0><<<b, 128, 0, st>>>(drva[a], cm[a], qa, de, p, yaco, umf[0], umf[1], umf[2], ip, flag, d.lxi, d.let, d.lze);
            else if (a == 1) k_gc_setup<1><<<b, 128, 0, st>>>(drva[a], cm[a], qa, de, p, yaco, umf[0], umf[1], umf[2], ip, flag, d.lxi, d.let, d.lze);
            else k_gc_setup<2><<<b, 128, 0, st>>>(drva[a], cm[a], qa, de, p, yaco, umf[0], umf[1], umf[2], ip, flag, d.lxi, d.let, d.lze);
            CSB_CUDA(cudaGetLastError());
        }
    // 2. GCIC exchange (src/gcbc.hpp:132-157): the neighbour across face ip
    //    is the block itself, adjacent through its face 1 - ip
    for (int a = 0; a < 3; ++a)
        for (int ip = 0; ip < 2; ++ip)
            if (nbc[ip][a] == CS_BC_INTER_CURV)
                CSB_CUDA(cudaMemcpyAsync(drvb[a] + (int64_t)ip * 5 * F[a], drva[a] + (int64_t)(1 - ip) * 5 * F[a],
                                         5 * F[a] * sizeof(double), cudaMemcpyDeviceToDevice, st));
    // 3. update kernels
    for (int a = 0; a < 3; ++a)
        for (int ip = 0; ip < 2; ++ip) {
            const int np = nbc[ip][a];
            if (!gc_active(np)) continue;
            const int kind = np == CS_BC_NON_REFLECTIVE ? 0 : (np == CS_BC_INTER_CURV ? 2 : 1);
            const unsigned b = blocks_for(F[a], 128);
            const double *db = drvb[a];
            if (a == 0) k_gc_update<0><<<b, 128, 0, st>>>(kind, drva[a], db, cm[a], qa, de, p, sbcc, umf[0], umf[1], umf[2], dudtmf[0], dudtmf[1], dudtmf[2], dtwi, ip, d.lxi, d.let, d.lze);
            else if (a == 1) k_gc_update<1><<<b, 128, 0, st>>>(kind, drva[a], db, cm[a], qa, de, p, sbcc, umf[0], umf[1], umf[2], dudtmf[0], dudtmf[1], dudtmf[2], dtwi, ip, d.lxi, d.let, d.lze);
            else k_gc_update<2><<<b, 128, 0, st>>>(kind, drva[a], db, cm[a], qa, de, p, sbcc, umf[0], umf[1], umf[2], dudtmf[0], dudtmf[1], dudtmf[2], dtwi, ip, d.lxi, d.let, d.lze);
            CSB_CUDA(cudaGetLastError());
        }
    return CS_OK;
}

}  // extern "C"
