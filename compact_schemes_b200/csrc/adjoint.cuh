// adjoint.cuh -- device kernels of the tangent and adjoint RHS.
//
// The compact derivative along a line is D = A^-1 B (A tridiagonal, B the
// explicit stencil with its closure rows: deriv_rhs).  Tangents apply D;
// adjoints apply D^T = B^T A^-T: a solve with the transposed tridiagonal
// matrix (its own precomputed tables, scheme kDerivT) followed by the
// transposed stencil, whose closure columns are gathered from the four
// boundary rows (physical rows, or the interface rows with their pbci / pbco
// weights, numerics_device_pc.hpp:176-293).
#pragma once

#include "adjoint_point.cuh"
#include "fused_kernels.cuh"

namespace csb {

// Column j of the closure rows 0, 1, n-2, n-1 of B.
__device__ __forceinline__ double brow0(int j, int n, int nstart, const Coeffs &cf) {
    if (nstart) return (j < kLmd ? cf.pbci[j] : 0.0) + (n - 1 - j < kLmd ? cf.pbco[n - 1 - j] : 0.0);
    return j == 0 ? kAb00 : (j == 1 ? kAb01 : (j == 2 ? kAb02 : 0.0));
}
__device__ __forceinline__ double brow1(int j, int n, int nstart, const Coeffs &cf) {
    if (nstart)
        return (j < kLmd ? cf.pbci[kLmd + j] : 0.0) + (n - 1 - j < kLmd ? cf.pbco[kLmd + n - 1 - j] : 0.0);
    return j == 0 ? -kAb10 : (j == 2 ? kAb10 : 0.0);
}
__device__ __forceinline__ double browm1(int j, int n, int nend, const Coeffs &cf) {
    if (nend) return -((n - 1 - j < kLmd ? cf.pbci[n - 1 - j] : 0.0) + (j < kLmd ? cf.pbco[j] : 0.0));
    return j == n - 1 ? -kAb00 : (j == n - 2 ? -kAb01 : (j == n - 3 ? -kAb02 : 0.0));
}
__device__ __forceinline__ double browm2(int j, int n, int nend, const Coeffs &cf) {
    if (nend)
        return -((n - 1 - j < kLmd ? cf.pbci[kLmd + n - 1 - j] : 0.0) + (j < kLmd ? cf.pbco[kLmd + j] : 0.0));
    return j == n - 3 ? -kAb10 : (j == n - 1 ? kAb10 : 0.0);
}

// o = B^T z for this lane's rows (z: a line in shared memory).
template <int LT>
__device__ __forceinline__ void stencil_t(const double *z, int n, int lane, int nstart, int nend, const Coeffs &cf,
                                          double (&o)[LT]) {
    using L = LineLayout<LT>;
    const double z0 = z[L::pos(0)], z1 = z[L::pos(1)], zm2 = z[L::pos(n - 2)], zm1 = z[L::pos(n - 1)];
#pragma unroll
    for (int t = 0; t < LT; ++t) {
        const int j = lane * LT + t;
        double s = 0.0;
        if (j < n) {
            // interior rows i in [2, n-3]: B[i][i+-1] = +-a, B[i][i+-2] = +-b
            if (j - 1 >= 2 && j - 1 <= n - 3) s += kAa * z[L::pos(j - 1)];
            if (j + 1 >= 2 && j + 1 <= n - 3) s -= kAa * z[L::pos(j + 1)];
            if (j - 2 >= 2 && j - 2 <= n - 3) s += kBb * z[L::pos(j - 2)];
            if (j + 2 >= 2 && j + 2 <= n - 3) s -= kBb * z[L::pos(j + 2)];
            if (j < kLmd || j >= n - kLmd)
                s += z0 * brow0(j, n, nstart, cf) + z1 * brow1(j, n, nstart, cf) + zm2 * browm2(j, n, nend, cf) +
                     zm1 * browm1(j, n, nend, cf);
        }
        o[t] = s;
    }
}

// o = B_f^T z for the compact filter's right-hand side (filter_rhs): rows
// i = j-3 .. j+3 contribute their coefficient at offset j - i; without
// wrap-around, rows at distance 0, 1, 2 from an end use the identity, second-
// and fourth-order stencils.
template <int LT>
__device__ __forceinline__ void filter_stencil_t(const double *z, int n, int lane, bool cyclic, double af,
                                                 double (&o)[LT]) {
    using L = LineLayout<LT>;
    const double a60 = (11.0 + 10.0 * af) / 16.0, a61 = (15.0 + 34.0 * af) / 32.0;
    const double a62 = (-3.0 + 6.0 * af) / 16.0, a63 = (1.0 - 2.0 * af) / 32.0;
    const double a40 = (5.0 + 6.0 * af) / 8.0, a41 = (1.0 + 2.0 * af) / 2.0, a42 = (-1.0 + 2.0 * af) / 8.0;
    const double a20 = (1.0 + 2.0 * af) / 2.0;
#pragma unroll
    for (int t = 0; t < LT; ++t) {
        const int j = lane * LT + t;
        double s = 0.0;
        if (j < n) {
#pragma unroll
            for (int d = -3; d <= 3; ++d) {
                int i = j + d;
                if (cyclic) i = i < 0 ? i + n : (i >= n ? i - n : i);
                else if (i < 0 || i >= n) continue;
                const int o = d < 0 ? -d : d;  // |j - i|
                const int dist = cyclic ? 3 : (i < n - 1 - i ? i : n - 1 - i);
                double c;
                if (dist >= 3) c = o == 0 ? a60 : (o == 1 ? 0.5 * a61 : (o == 2 ? 0.5 * a62 : 0.5 * a63));
                else if (dist == 2) c = o == 0 ? a40 : (o == 1 ? 0.5 * a41 : (o == 2 ? 0.5 * a42 : 0.0));
                else if (dist == 1) c = o == 0 ? a20 : (o == 1 ? 0.5 * a20 : 0.0);
                else c = o == 0 ? 1.0 : 0.0;
                s += c * z[L::pos(i)];
            }
        }
        o[t] = s;
    }
}

// out[f] (=|+=) scale * D (or D^T) in[f] along AXIS, field f = blockIdx.y, or
// the compact filter (FILTER) and its transpose; one warp per line, 8 lines
// per CTA.
template <int LT, int AXIS, bool TRANS, bool FILTER = false>
__global__ void __launch_bounds__(256) k_lines(const double *__restrict__ in, int64_t in_fs,
                                               double *__restrict__ out, int64_t out_fs, int accum, double scale,
                                               DevTables<double> tab, int lxi, int let, int64_t F, int nstart,
                                               int nend, Coeffs cf, double af = 0.0) {
    constexpr int TL = 8;
    using L = LineLayout<LT>;
    __shared__ double sm[TL * L::kSlot];
    const int n = tab.n;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t line0 = (int64_t)blockIdx.x * TL;
    const double *src = in + blockIdx.y * in_fs;
    double *dst = out + blockIdx.y * out_fs;
    tile_for_each<AXIS, TL>(line0, F, n, lxi, let,
                            [&](int l, int j, int64_t gi) { sm[l * L::kSlot + L::pos(j)] = src[gi]; });
    tile_sync<AXIS, TL>();
    if (line0 + w < F) {
        double *line = sm + w * L::kSlot;
        double d[1][LT];
        if (!TRANS) {
            if (FILTER) filter_rhs<LT, double, double>(line, n, lane, tab.cyclic != 0, af, d[0]);
            else deriv_rhs<LT, double, double>(line, n, lane, nstart, nend, nullptr, cf, d[0]);
            warp_solve<LT, 1, double>(tab, d, lane);
        } else {
#pragma unroll
            for (int t = 0; t < LT; ++t) d[0][t] = lane * LT + t < n ? line[L::pos_ct(lane, t)] : 0.0;
            warp_solve<LT, 1, double>(tab, d, lane);
            __syncwarp();
#pragma unroll
            for (int t = 0; t < LT; ++t)
                if (lane * LT + t < n) line[L::pos_ct(lane, t)] = d[0][t];
            __syncwarp();
            if (FILTER) filter_stencil_t<LT>(line, n, lane, tab.cyclic != 0, af, d[0]);
            else stencil_t<LT>(line, n, lane, nstart, nend, cf, d[0]);
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < LT; ++t)
            if (lane * LT + t < n) line[L::pos_ct(lane, t)] = d[0][t];
    }
    tile_sync<AXIS, TL>();
    tile_for_each<AXIS, TL>(line0, F, n, lxi, let, [&](int l, int j, int64_t gi) {
        const double v = scale * sm[l * L::kSlot + L::pos(j)];
        dst[gi] = accum ? dst[gi] + v : v;
    });
}

// --------------------------------------------------------------- pointwise
struct AdjPoint {
    PointPhys ph;
    int64_t lmx;
    int viscous;
};

#define CSB_GRID_STRIDE(i, n) for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); \
                                   i += (int64_t)gridDim.x * blockDim.x)

// dphi = (dphi/dq) dq
__global__ void k_prim_tan(const double *__restrict__ q, const double *__restrict__ dq, double *__restrict__ dphi,
                           int64_t lmx) {
    CSB_GRID_STRIDE(i, lmx) {
        double qq[5], d[5], o[4];
        for (int m = 0; m < 5; ++m) { qq[m] = q[m * lmx + i]; d[m] = dq[m * lmx + i]; }
        prim_tan(qq, d, o);
        for (int c = 0; c < 4; ++c) dphi[c * lmx + i] = o[c];
    }
}

// dF[a][m] = (dF_a/dq) dq + (dF_a/dG) dG for every active axis a
template <bool VISC>
__global__ void k_flux_tan(const double *__restrict__ q, const double *__restrict__ G, const double *__restrict__ dq,
                           const double *__restrict__ dG, double *__restrict__ dF, AdjPoint ap, int amask) {
    const int64_t lmx = ap.lmx;
    CSB_GRID_STRIDE(i, lmx) {
        double qq[5], d[5], g[12], dg[12], o[5];
        for (int m = 0; m < 5; ++m) { qq[m] = q[m * lmx + i]; d[m] = dq[m * lmx + i]; }
        for (int k = 0; k < 12; ++k) {
            g[k] = VISC ? G[k * lmx + i] : 0.0;
            dg[k] = VISC ? dG[k * lmx + i] : 0.0;
        }
        for (int a = 0; a < 3; ++a) {
            if (!(amask >> a & 1)) continue;
            flux_tan<VISC>(a, qq, g, d, dg, ap.ph, o);
            for (int m = 0; m < 5; ++m) dF[(a * 5 + m) * lmx + i] = o[m];
        }
    }
}

// qbar = sum_a (dF_a/dq)^T mu_a,  Gbar = sum_a (dF_a/dG)^T mu_a
template <bool VISC>
__global__ void k_flux_adj(const double *__restrict__ q, const double *__restrict__ G, const double *__restrict__ mu,
                           double *__restrict__ qbar, double *__restrict__ Gbar, AdjPoint ap, int amask) {
    const int64_t lmx = ap.lmx;
    CSB_GRID_STRIDE(i, lmx) {
        double qq[5], g[12], qb[5] = {0, 0, 0, 0, 0}, gb[12], fb[5];
        for (int m = 0; m < 5; ++m) qq[m] = q[m * lmx + i];
        for (int k = 0; k < 12; ++k) {
            g[k] = VISC ? G[k * lmx + i] : 0.0;
            gb[k] = 0.0;
        }
        for (int a = 0; a < 3; ++a) {
            if (!(amask >> a & 1)) continue;
            for (int m = 0; m < 5; ++m) fb[m] = mu[(a * 5 + m) * lmx + i];
            flux_adj<VISC>(a, qq, g, fb, ap.ph, qb, gb);
        }
        for (int m = 0; m < 5; ++m) qbar[m * lmx + i] = qb[m];
        if (VISC)
            for (int k = 0; k < 12; ++k) Gbar[k * lmx + i] = gb[k];
    }
}

// w = scale * (qbar + (dphi/dq)^T phibar); out = w (if set); acc_out =
// (acc_in if set, else acc_out) + w (if acc_out is set).
__global__ void k_prim_adj(const double *__restrict__ q, const double *__restrict__ qbar,
                           const double *__restrict__ phibar, double *__restrict__ out, double scale, int64_t lmx,
                           int have_phibar, const double *__restrict__ acc_in, double *__restrict__ acc_out) {
    CSB_GRID_STRIDE(i, lmx) {
        double qq[5], qb[5], pb[4];
        for (int m = 0; m < 5; ++m) { qq[m] = q[m * lmx + i]; qb[m] = qbar[m * lmx + i]; }
        if (have_phibar) {
            for (int c = 0; c < 4; ++c) pb[c] = phibar[c * lmx + i];
            prim_adj(qq, pb, qb);
        }
        for (int m = 0; m < 5; ++m) {
            const double w = scale * qb[m];
            if (out) out[m * lmx + i] = w;
            if (acc_out) acc_out[m * lmx + i] = (acc_in ? acc_in[m * lmx + i] : acc_out[m * lmx + i]) + w;
        }
    }
}

// z = x + a * y  (n values)
__global__ void k_xpay(const double *__restrict__ x, double a, const double *__restrict__ y, double *__restrict__ z,
                       int64_t n) {
    CSB_GRID_STRIDE(i, n) z[i] = x[i] + a * y[i];
}

// Kinetic energy 0.5 * sum (m.m)/rho * dV (block partial sums) and its
// gradient with respect to q.
__global__ void k_kinetic(const double *__restrict__ q, int64_t lmx, double dv, double *__restrict__ partial,
                          double *__restrict__ seed) {
    __shared__ double red[256];
    double acc = 0.0;
    CSB_GRID_STRIDE(i, lmx) {
        const double r = q[i], m1 = q[lmx + i], m2 = q[2 * lmx + i], m3 = q[3 * lmx + i];
        const double mm = m1 * m1 + m2 * m2 + m3 * m3, ri = 1.0 / r;
        acc += 0.5 * mm * ri * dv;
        if (seed) {
            seed[i] = -0.5 * mm * ri * ri * dv;
            seed[lmx + i] = m1 * ri * dv;
            seed[2 * lmx + i] = m2 * ri * dv;
            seed[3 * lmx + i] = m3 * ri * dv;
            seed[4 * lmx + i] = 0.0;
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

}  // namespace csb

namespace csb {

// F_x(q, G) at every point (the forward x flux; its x derivative at the
// faces is what the GCBC correction reads).
template <bool VISC>
__global__ void k_flux_x_eval(const double *__restrict__ q, const double *__restrict__ G, double *__restrict__ Fx,
                              AdjPoint ap) {
    const int64_t lmx = ap.lmx;
    CSB_GRID_STRIDE(i, lmx) {
        double qq[5], g[12], o[5];
        for (int m = 0; m < 5; ++m) qq[m] = q[m * lmx + i];
        for (int k = 0; k < 12; ++k) g[k] = VISC ? G[k * lmx + i] : 0.0;
        flux_eval<VISC>(0, qq, g, ap.ph, o);
        for (int m = 0; m < 5; ++m) Fx[m * lmx + i] = o[m];
    }
}

// face[(ip*5 + v)*F + fi] = src[v][point fi of face ip] (x faces)
__global__ void k_xface_extract(const double *__restrict__ src, double *__restrict__ face, int lxi, int64_t lmx,
                                int64_t F) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * F) return;
    const int ip = (int)(t / F);
    const int64_t fi = t % F, idx = fi * lxi + (ip ? lxi - 1 : 0);
    for (int v = 0; v < 5; ++v) face[(int64_t)(ip * 5 + v) * F + fi] = src[v * lmx + idx];
}

// Tangent of the GCBC correction at the non-reflective x faces:
// dR[face point] += d g(q, r)[dq, dr].
__global__ void k_gcbc_tan(const double *__restrict__ q, const double *__restrict__ rf,
                           const double *__restrict__ dq, const double *__restrict__ drf, double *__restrict__ dR,
                           int lxi, int64_t lmx, int64_t F, int face_mask, PointPhys ph) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * F) return;
    const int ip = (int)(t / F);
    if (!((face_mask >> ip) & 1)) return;
    const int64_t fi = t % F, idx = fi * lxi + (ip ? lxi - 1 : 0);
    double c[3];
    xface_normal(ph, c);
    Dual qd[5], rd[5], o[5];
    for (int v = 0; v < 5; ++v) {
        qd[v] = dual(q[v * lmx + idx], dq[v * lmx + idx]);
        rd[v] = dual(rf[(int64_t)(ip * 5 + v) * F + fi], drf[(int64_t)(ip * 5 + v) * F + fi]);
    }
    gcbc_point(qd, rd, c, ph, ip, o);
    for (int v = 0; v < 5; ++v) dR[v * lmx + idx] += o[v].d;
}

// Adjoint of the GCBC correction: with the 5 x 10 Jacobian of g(q, r) at a
// face point (ten dual evaluations), lam_x[face point] = lam + dg/dr^T lam
// (the adjoint of the x-derivative term there) and qbf[face] = dg/dq^T lam.
__global__ void k_gcbc_adj(const double *__restrict__ q, const double *__restrict__ rf,
                           const double *__restrict__ lam, double *__restrict__ lam_x, double *__restrict__ qbf,
                           int lxi, int64_t lmx, int64_t F, int face_mask, PointPhys ph) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * F) return;
    const int ip = (int)(t / F);
    if (!((face_mask >> ip) & 1)) return;
    const int64_t fi = t % F, idx = fi * lxi + (ip ? lxi - 1 : 0);
    double c[3];
    xface_normal(ph, c);
    double qv[5], rv[5], lv[5];
    for (int v = 0; v < 5; ++v) {
        qv[v] = q[v * lmx + idx];
        rv[v] = rf[(int64_t)(ip * 5 + v) * F + fi];
        lv[v] = lam[v * lmx + idx];
    }
    for (int k = 0; k < 10; ++k) {
        Dual qd[5], rd[5], o[5];
        for (int v = 0; v < 5; ++v) {
            qd[v] = dual(qv[v], k == v ? 1.0 : 0.0);
            rd[v] = dual(rv[v], k == 5 + v ? 1.0 : 0.0);
        }
        gcbc_point(qd, rd, c, ph, ip, o);
        double s = 0.0;
        for (int v = 0; v < 5; ++v) s += o[v].d * lv[v];
        if (k < 5) qbf[(int64_t)(ip * 5 + k) * F + fi] = s;
        else lam_x[(k - 5) * lmx + idx] = lv[k - 5] + s;
    }
}

// qbar[face point] += qbf[face] on the faces of face_mask
__global__ void k_xface_add(const double *__restrict__ qbf, double *__restrict__ qbar, int lxi, int64_t lmx,
                            int64_t F, int face_mask) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * F) return;
    const int ip = (int)(t / F);
    if (!((face_mask >> ip) & 1)) return;
    const int64_t fi = t % F, idx = fi * lxi + (ip ? lxi - 1 : 0);
    for (int v = 0; v < 5; ++v) qbar[v * lmx + idx] += qbf[(int64_t)(ip * 5 + v) * F + fi];
}

}  // namespace csb
