/*
 * oracle.cpp -- FP64 CPU restatement of the EnricoDeg/compact_schemes hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never the product.
 * Straightforward scalar/OpenMP loops that follow the reference's algorithm
 * step by step; each function cites the reference file:line it restates
 * (paths relative to the reference project root).  Tridiagonal systems are
 * solved with the Thomas algorithm in FP64 (the reference uses PCR; both are
 * exact up to rounding).
 */
#include "oracle.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Scheme constants, src/common/parameters.hpp:35-43.
constexpr double kAlpha = 1.0 / 3.0;
constexpr double kAlpha01 = 2.0;
constexpr double kAlpha10 = 1.0 / 4.0;
constexpr double kA = 7.0 / 9.0;
constexpr double kB = 1.0 / 36.0;
constexpr double kAb00 = -5.0 / 2.0;
constexpr double kAb01 = 2.0;
constexpr double kAb02 = 1.0 / 2.0;
constexpr double kAb10 = 3.0 / 4.0;
constexpr int kLmd = 8;
constexpr int kMbci = 4;
// Gas constants, src/common/parameters.hpp:61-67.
constexpr double kGam = 1.4;
constexpr double kGamm1 = kGam - 1.0;
constexpr double kHamm1 = 1.0 / kGamm1;
constexpr double kPrndtl = 0.71;
constexpr double kGamm1Prndtli = 1.0 / (kGamm1 * kPrndtl);
constexpr int kBcNonReflective = 10;

struct Dims {
    int lxi, let, lze;
    int64_t lmx() const { return (int64_t)lxi * let * lze; }
};

// Line geometry per axis; face index convention of deriv_kernel_1d_impl
// (src/cuda/kernels/numerics_device_pc.hpp:308-315 with transforms.hpp).
struct LineMap {
    int n;        // points on the line
    int64_t F;    // number of lines (face size)
    int64_t stride;
    Dims d;
    int axis;
    int64_t base(int64_t fidx) const {
        if (axis == 0) return fidx * d.lxi;                       // fidx = k*let + j
        if (axis == 1) {                                          // fidx = k*lxi + i
            int64_t k = fidx / d.lxi, i = fidx % d.lxi;
            return k * (int64_t)d.lxi * d.let + i;
        }
        return fidx;                                              // fidx = j*lxi + i
    }
};

LineMap line_map(Dims d, int axis) {
    LineMap m;
    m.d = d;
    m.axis = axis;
    if (axis == 0) { m.n = d.lxi; m.F = (int64_t)d.let * d.lze; m.stride = 1; }
    else if (axis == 1) { m.n = d.let; m.F = (int64_t)d.lxi * d.lze; m.stride = d.lxi; }
    else { m.n = d.lze; m.F = (int64_t)d.lxi * d.let; m.stride = (int64_t)d.lxi * d.let; }
    return m;
}

void thomas(int n, const double *a, const double *b, const double *c, const double *r, double *x) {
    std::vector<double> cp(n), dp(n);
    cp[0] = c[0] / b[0];
    dp[0] = r[0] / b[0];
    for (int i = 1; i < n; ++i) {
        double m = b[i] - a[i] * cp[i - 1];
        cp[i] = c[i] / m;
        dp[i] = (r[i] - a[i] * dp[i - 1]) / m;
    }
    x[n - 1] = dp[n - 1];
    for (int i = n - 2; i >= 0; --i) x[i] = dp[i] - cp[i] * x[i + 1];
}

// When set, every derivative/filter line is solved bottom-up (Thomas on the
// index-reversed system): exact-arithmetic identical, different rounding.
// Tests use it to measure the FP64 noise floor of the scheme itself.
int g_reversed = 0;

void thomas_dir(int n, const double *a, const double *b, const double *c, const double *r, double *x) {
    if (!g_reversed) { thomas(n, a, b, c, r, x); return; }
    std::vector<double> ra(n), rb(n), rc(n), rr(n), rx(n);
    for (int i = 0; i < n; ++i) {
        ra[i] = c[n - 1 - i]; rb[i] = b[n - 1 - i]; rc[i] = a[n - 1 - i]; rr[i] = r[n - 1 - i];
    }
    thomas(n, ra.data(), rb.data(), rc.data(), rr.data(), rx.data());
    for (int i = 0; i < n; ++i) x[i] = rx[n - 1 - i];
}

// Cyclic tridiagonal (a[0] couples x[n-1], c[n-1] couples x[0]) by the
// Sherman-Morrison correction of a non-cyclic system.
void thomas_cyclic(int n, const double *a, const double *b, const double *c, const double *r, double *x) {
    std::vector<double> bb(b, b + n), u(n, 0.0), z(n);
    double gamma = -b[0];
    bb[0] = b[0] - gamma;
    bb[n - 1] = b[n - 1] - a[0] * c[n - 1] / gamma;
    std::vector<double> aa(a, a + n), cc(c, c + n);
    aa[0] = 0.0;
    cc[n - 1] = 0.0;
    thomas(n, aa.data(), bb.data(), cc.data(), r, x);
    u[0] = gamma;
    u[n - 1] = c[n - 1];
    thomas(n, aa.data(), bb.data(), cc.data(), u.data(), z.data());
    double fact = (x[0] + a[0] * x[n - 1] / gamma) / (1.0 + z[0] + a[0] * z[n - 1] / gamma);
    for (int i = 0; i < n; ++i) x[i] -= fact * z[i];
}

// Matrix inverse by the steps of numerics_base::mtrxi / maxloc
// (src/numerics_base.hpp:300-386): Gauss-Jordan elimination on the flattened
// array rx[col + row*n], with the pivot column chosen by the largest |entry|
// of row i among columns i .. n-2, columns swapped and a permutation kept.
// The steps are kept identical (same operations in the same order) because
// the interface weights it produces feed sums with strong cancellation, so
// they must match the reference's to the last bit.
void invert_like_reference(int n, const double *m, double *inv) {
    std::vector<double> rx(m, m + n * n), temp(n);
    std::vector<int> ipvt(n);
    for (int i = 0; i < n; ++i) ipvt[i] = i;
    for (int i = 0; i < n; ++i) {
        const int loc = i * n + i, len = n - i - 1;
        int imax = 0;
        double dmax = std::fabs(rx[loc]);
        for (int k = 1; k < len; ++k)
            if (std::fabs(rx[loc + k]) > dmax) { dmax = std::fabs(rx[loc + k]); imax = k; }
        const int mk = i + imax;
        if (mk != i) {
            std::swap(ipvt[mk], ipvt[i]);
            for (int l = 0; l < n; ++l) std::swap(rx[mk + l * n], rx[i + l * n]);
        }
        const double ra0 = 1.0 / rx[i + i * n];
        for (int k = 0; k < n; ++k) temp[k] = rx[k + i * n];
        for (int k = 0; k < n; ++k) {
            const double ra1 = ra0 * rx[i + k * n];
            for (int l = 0; l < n; ++l) rx[l + k * n] = rx[l + k * n] - ra1 * temp[l];
            rx[i + k * n] = ra1;
        }
        for (int k = 0; k < n; ++k) rx[k + i * n] = -ra0 * temp[k];
        rx[i + i * n] = ra0;
    }
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) inv[i + ipvt[j] * n] = rx[i + j * n];
}

// Rows of the compact derivative system for one line, restating
// build_system (src/cuda/kernels/numerics_device_pc.hpp:176-293).
void build_deriv_rows(const double *f, int n, int nstart, int nend, const double recv4[4],
                      const double *pbci, double *a, double *b, double *c, double *r) {
    for (int i = 2; i < n - 2; ++i) {
        r[i] = kA * (f[i + 1] - f[i - 1]) + kB * (f[i + 2] - f[i - 2]);
        a[i] = kAlpha; b[i] = 1.0; c[i] = kAlpha;
    }
    if (nstart == 0) {
        r[0] = kAb00 * f[0] + kAb01 * f[1] + kAb02 * f[2];
        a[0] = 0.0; b[0] = 1.0; c[0] = kAlpha01;
        r[1] = kAb10 * (f[2] - f[0]);
        a[1] = kAlpha10; b[1] = 1.0; c[1] = kAlpha10;
    } else {
        double s0 = 0.0, s1 = 0.0;
        for (int i = 0; i < kLmd; ++i) s0 += pbci[i] * f[i];
        for (int i = 0; i < kLmd; ++i) s1 += pbci[kLmd + i] * f[i];
        r[0] = s0 + recv4[0];
        a[0] = 0.0; b[0] = 1.0; c[0] = kAlpha;
        r[1] = s1 + recv4[1];
        a[1] = kAlpha; b[1] = 1.0; c[1] = kAlpha;
    }
    if (nend == 0) {
        r[n - 1] = -(kAb00 * f[n - 1] + kAb01 * f[n - 2] + kAb02 * f[n - 3]);
        a[n - 1] = kAlpha01; b[n - 1] = 1.0; c[n - 1] = 0.0;
        r[n - 2] = -kAb10 * (f[n - 3] - f[n - 1]);
        a[n - 2] = kAlpha10; b[n - 2] = 1.0; c[n - 2] = kAlpha10;
    } else {
        double s0 = 0.0, s1 = 0.0;
        for (int i = 0; i < kLmd; ++i) s0 += pbci[i] * f[n - 1 - i];
        s0 += recv4[2];
        for (int i = 0; i < kLmd; ++i) s1 += pbci[kLmd + i] * f[n - 1 - i];
        s1 += recv4[3];
        r[n - 1] = -s0;
        a[n - 1] = kAlpha; b[n - 1] = 1.0; c[n - 1] = 0.0;
        r[n - 2] = -s1;
        a[n - 2] = kAlpha; b[n - 2] = 1.0; c[n - 2] = kAlpha;
    }
}

double g_pbco[16], g_pbci[16];
bool g_coeff_ready = false;

void ensure_coeffs() {
    if (!g_coeff_ready) {
        or_deriv_setup(g_pbco, g_pbci);
        g_coeff_ready = true;
    }
}

inline double metric(const double *arr, const double *c3, int comp, int64_t n, int64_t i) {
    return arr ? arr[comp * n + i] : c3[comp];
}
inline double jac(const or_metrics &m, int64_t i) { return m.yaco ? m.yaco[i] : m.c_yaco; }

}  // namespace

extern "C" {

void or_set_reversed_solves(int on) { g_reversed = on ? 1 : 0; }

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// numerics_base::deriv_setup (src/numerics_base.hpp:182-297): a 16-point
// two-block Pade system P f' = Q f; R = P~ P^-1 Q where P~ drops the coupling
// across the block interface; rows 8 and 9 of R give the sender (pbco,
// reversed order) and receiver (pbci) interface weights.
void or_deriv_setup(double pbco[16], double pbci[16]) {
    const int n = 2 * kLmd;
    std::vector<double> Q(n * n, 0.0), P(n * n, 0.0), Pi(n * n), T(n * n), R(n * n);
    auto q = [&](int i, int j) -> double & { return Q[i * n + j]; };
    auto p = [&](int i, int j) -> double & { return P[i * n + j]; };
    q(0, 0) = kAb00; q(0, 1) = kAb01; q(0, 2) = kAb02;
    q(1, 0) = -kAb10; q(1, 2) = kAb10;
    q(n - 1, n - 1) = -kAb02; q(n - 1, n - 2) = -kAb01; q(n - 1, n - 3) = -kAb00;
    q(n - 2, n - 1) = kAb10; q(n - 2, n - 3) = -kAb10;
    for (int i = 2; i < n - 2; ++i) {
        q(i, i - 1) = -kA; q(i, i + 1) = kA; q(i, i - 2) = -kB; q(i, i + 2) = kB;
    }
    p(0, 0) = 1.0; p(0, 1) = kAlpha01;
    p(n - 1, n - 1) = 1.0; p(n - 1, n - 2) = kAlpha01;
    p(1, 0) = kAlpha10; p(1, 1) = 1.0; p(1, 2) = kAlpha10;
    p(n - 2, n - 1) = kAlpha10; p(n - 2, n - 2) = 1.0; p(n - 2, n - 3) = kAlpha10;
    for (int i = 2; i < n - 2; ++i) { p(i, i) = 1.0; p(i, i - 1) = kAlpha; p(i, i + 1) = kAlpha; }
    invert_like_reference(n, P.data(), Pi.data());
    int i = n / 2 - 2;
    p(i, i + 2) = 0.0; p(i + 1, i + 2) = 0.0; p(i + 1, i + 3) = 0.0;
    i = n / 2 + 1;
    p(i, i - 2) = 0.0; p(i - 1, i - 2) = 0.0; p(i - 1, i - 3) = 0.0;
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            double s = 0.0;
            for (int k = 0; k < n; ++k) s += Pi[r * n + k] * Q[k * n + c];
            T[r * n + c] = s;
        }
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            double s = 0.0;
            for (int k = 0; k < n; ++k) s += P[r * n + k] * T[k * n + c];
            R[r * n + c] = s;
        }
    for (int k = 0; k < kLmd; ++k) {
        pbco[kLmd - 1 - k] = R[(n / 2) * n + k];
        pbci[k] = R[(n / 2) * n + kLmd + k];
        pbco[2 * kLmd - 1 - k] = R[(n / 2 + 1) * n + k];
        pbci[kLmd + k] = R[(n / 2 + 1) * n + kLmd + k];
    }
}

void or_fill_buffer(const double *in, double *send, int lxi, int let, int lze, int axis,
                    int face, const double *pbco) {
    LineMap lm = line_map(Dims{lxi, let, lze}, axis);
    const int istart = face * (lm.n - 1), inc = 1 - 2 * face;
#pragma omp parallel for
    for (int64_t fi = 0; fi < lm.F; ++fi) {
        int64_t b = lm.base(fi);
        double v0 = 0.0, v1 = 0.0;
        for (int i = 0; i < kLmd; ++i) v0 += pbco[i] * in[b + (istart + inc * i) * lm.stride];
        for (int i = 0; i < kLmd; ++i) v1 += pbco[kLmd + i] * in[b + (istart + inc * i) * lm.stride];
        send[fi] = v0;
        send[lm.F + fi] = v1;
    }
}

int or_deriv_line(const double *f, double *x, int n, int nstart, int nend, const double recv4[4],
                  const double *pbco, const double *pbci) {
    if (n < 5 || ((nstart || nend) && n < kLmd)) return -1;
    double self[4];
    if ((nstart || nend) && !recv4) {
        // Single-rank periodic: face 0 receives what face 1 sends and vice
        // versa (tag pairing of src/numerics_base.hpp:161-176).
        double s[4] = {0, 0, 0, 0};
        for (int i = 0; i < kLmd; ++i) s[0] += pbco[i] * f[n - 1 - i];
        for (int i = 0; i < kLmd; ++i) s[1] += pbco[kLmd + i] * f[n - 1 - i];
        for (int i = 0; i < kLmd; ++i) s[2] += pbco[i] * f[i];
        for (int i = 0; i < kLmd; ++i) s[3] += pbco[kLmd + i] * f[i];
        std::memcpy(self, s, sizeof s);
        recv4 = self;
    }
    std::vector<double> a(n), b(n), c(n), r(n);
    build_deriv_rows(f, n, nstart, nend, recv4, pbci, a.data(), b.data(), c.data(), r.data());
    thomas_dir(n, a.data(), b.data(), c.data(), r.data(), x);
    return 0;
}

int or_deriv(const double *in, double *out, int lxi, int let, int lze, int axis, int nstart,
             int nend, const double *recv, double *drva, int var, const double *pbco,
             const double *pbci) {
    LineMap lm = line_map(Dims{lxi, let, lze}, axis);
    const int n = lm.n;
    if (n < 5 || ((nstart || nend) && n < kLmd) || axis < 0 || axis > 2) return -1;
    int err = 0;
#pragma omp parallel
    {
        std::vector<double> f(n), x(n);
#pragma omp for
        for (int64_t fi = 0; fi < lm.F; ++fi) {
            int64_t b = lm.base(fi);
            for (int j = 0; j < n; ++j) f[j] = in[b + j * lm.stride];
            double r4[4];
            const double *rp = nullptr;
            if (recv) {
                r4[0] = recv[fi]; r4[1] = recv[lm.F + fi];
                r4[2] = recv[2 * lm.F + fi]; r4[3] = recv[3 * lm.F + fi];
                rp = r4;
            }
            if (or_deriv_line(f.data(), x.data(), n, nstart, nend, rp, pbco, pbci)) err = -1;
            for (int j = 0; j < n; ++j) out[b + j * lm.stride] = x[j];
            if (drva) {
                drva[(int64_t)var * lm.F + fi] = x[0];
                drva[5 * lm.F + (int64_t)var * lm.F + fi] = x[n - 1];
            }
        }
    }
    return err;
}

// Compact filter.  The reference has none; this is the sixth-order
// tridiagonal Pade filter of Gaitonde & Visbal (AIAA J. 38(11), 2000;
// Visbal & Gaitonde, J. Comput. Phys. 181, 2002):
//   af*g[i-1] + g[i] + af*g[i+1] = sum_n a_n/2 (f[i+n] + f[i-n])
// interior a0=(11+10af)/16, a1=(15+34af)/32, a2=(-3+6af)/16, a3=(1-2af)/32.
// Non-periodic ends: boundary point unfiltered, second point second order
// (a0=a1=(1+2af)/2), third point fourth order (a0=(5+6af)/8,
// a1=(1+2af)/2, a2=(-1+2af)/8).  Both faces periodic: cyclic sixth order.
int or_filter_line(const double *f, double *x, int n, int nstart, int nend, double af) {
    const bool cyclic = nstart && nend;
    if (n < 7 || (nstart != nend)) return -1;
    const double a6[4] = {(11 + 10 * af) / 16, (15 + 34 * af) / 32, (-3 + 6 * af) / 16,
                          (1 - 2 * af) / 32};
    const double a4[3] = {(5 + 6 * af) / 8, (1 + 2 * af) / 2, (-1 + 2 * af) / 8};
    const double a2[2] = {(1 + 2 * af) / 2, (1 + 2 * af) / 2};
    std::vector<double> a(n), b(n, 1.0), c(n), r(n);
    auto at = [&](int i) { return cyclic ? f[((i % n) + n) % n] : f[i]; };
    for (int i = 0; i < n; ++i) {
        int dist = cyclic ? 99 : std::min(i, n - 1 - i);
        if (dist == 0) {
            a[i] = 0; c[i] = 0; r[i] = f[i];
        } else if (dist == 1) {
            a[i] = af; c[i] = af;
            r[i] = a2[0] * at(i) + (0.5 * a2[1]) * (at(i + 1) + at(i - 1));
        } else if (dist == 2) {
            a[i] = af; c[i] = af;
            r[i] = a4[0] * at(i) + (0.5 * a4[1]) * (at(i + 1) + at(i - 1)) +
                   (0.5 * a4[2]) * (at(i + 2) + at(i - 2));
        } else {
            a[i] = af; c[i] = af;
            r[i] = a6[0] * at(i) + (0.5 * a6[1]) * (at(i + 1) + at(i - 1)) +
                   (0.5 * a6[2]) * (at(i + 2) + at(i - 2)) + (0.5 * a6[3]) * (at(i + 3) + at(i - 3));
        }
    }
    if (cyclic) thomas_cyclic(n, a.data(), b.data(), c.data(), r.data(), x);
    else thomas(n, a.data(), b.data(), c.data(), r.data(), x);
    return 0;
}

int or_filter(const double *in, double *out, int lxi, int let, int lze, int axis, int nstart,
              int nend, double af) {
    LineMap lm = line_map(Dims{lxi, let, lze}, axis);
    const int n = lm.n;
    if (n < 7 || nstart != nend) return -1;
    int err = 0;
#pragma omp parallel
    {
        std::vector<double> f(n), x(n);
#pragma omp for
        for (int64_t fi = 0; fi < lm.F; ++fi) {
            int64_t b = lm.base(fi);
            for (int j = 0; j < n; ++j) f[j] = in[b + j * lm.stride];
            if (or_filter_line(f.data(), x.data(), n, nstart, nend, af)) err = -1;
            for (int j = 0; j < n; ++j) out[b + j * lm.stride] = x[j];
        }
    }
    return err;
}

// calc_fluxes_pre_compute_kernel<Visc> (src/cuda/kernels/physics.hpp:42-193).
void or_fluxes_pre(double *buffer, const double *qa, const double *p, double *de,
                   const double *xim, const double *etm, const double *zem, const double *tau,
                   const double *heat, const double umf[3], int64_t n) {
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        const double M[3][3] = {{xim[i], xim[n + i], xim[2 * n + i]},
                                {etm[i], etm[n + i], etm[2 * n + i]},
                                {zem[i], zem[n + i], zem[2 * n + i]}};
        const double rr[3] = {de[n + i] + umf[0], de[2 * n + i] + umf[1], de[3 * n + i] + umf[2]};
        double ss[3];
        for (int a = 0; a < 3; ++a) ss[a] = M[a][0] * rr[0] + M[a][1] * rr[1] + M[a][2] * rr[2];
        const double pp = p[i];
        double t[6] = {0, 0, 0, 0, 0, 0}, h[3] = {0, 0, 0};
        if (tau)
            for (int c = 0; c < 6; ++c) t[c] = tau[c * n + i];
        if (heat)
            for (int c = 0; c < 3; ++c) h[c] = heat[c * n + i];
        // stress rows: x-momentum uses (xx, xy, zx), y (xy, yy, yz), z (zx, yz, zz)
        const double tr[3][3] = {{t[0], t[3], t[5]}, {t[3], t[1], t[4]}, {t[5], t[4], t[2]}};
        for (int a = 0; a < 3; ++a) buffer[(0 * 3 + a) * n + i] = qa[i] * ss[a];
        for (int m = 1; m <= 3; ++m)
            for (int a = 0; a < 3; ++a) {
                double v = qa[m * n + i] * ss[a] + M[a][m - 1] * pp;
                if (tau) v -= M[a][0] * tr[m - 1][0] + M[a][1] * tr[m - 1][1] + M[a][2] * tr[m - 1][2];
                buffer[(m * 3 + a) * n + i] = v;
            }
        const double h0 = qa[4 * n + i] + pp;
        for (int a = 0; a < 3; ++a) {
            double v = h0 * ss[a] - pp * (umf[0] * M[a][0] + umf[1] * M[a][1] + umf[2] * M[a][2]);
            if (heat) v -= M[a][0] * h[0] + M[a][1] * h[1] + M[a][2] * h[2];
            buffer[(4 * 3 + a) * n + i] = v;
        }
        de[4 * n + i] = h0;
    }
}

static void time_step_maxima(const double *xim, const double *etm, const double *zem,
                             const double *de, const or_metrics *mm, const double *yaco,
                             const double *ssk, double mu, const double umf[3], int64_t n,
                             double *m1, double *m2) {
    double r1 = 0.0, r2 = 0.0;
    bool first = true;
    (void)first;
#pragma omp parallel for reduction(max : r1, r2)
    for (int64_t i = 0; i < n; ++i) {
        double M[3][3];
        for (int c = 0; c < 3; ++c) {
            M[0][c] = xim ? xim[c * n + i] : mm->c_xim[c];
            M[1][c] = etm ? etm[c * n + i] : mm->c_etm[c];
            M[2][c] = zem ? zem[c * n + i] : mm->c_zem[c];
        }
        double rr1 = 0.0;
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 3; ++c) rr1 += M[a][c] * M[a][c];
        double rr2 = 0.0;
        for (int a = 0; a < 3; ++a)
            rr2 += std::fabs(M[a][0] * (de[n + i] + umf[0]) + M[a][1] * (de[2 * n + i] + umf[1]) +
                             M[a][2] * (de[3 * n + i] + umf[2]));
        double ssi = std::fabs(yaco ? yaco[i] : mm->c_yaco);
        double v1 = (std::sqrt(de[4 * n + i] * rr1) + rr2) * ssi;
        double v2 = de[i] * (ssk ? ssk[i] : mu) * rr1 * ssi * ssi;
        r1 = v1 > r1 ? v1 : r1;
        r2 = v2 > r2 ? v2 : r2;
    }
    *m1 = r1;
    *m2 = r2;
}

// calc_time_step (src/physics_pc.hpp:229-256; CPU twin tests/test_physics.cu:57-117):
// dt = min(cfl / max((sqrt(c^2 |grad xi|^2) + sum|M_a.(u+umf)|)|J|), 0.5 / max(de0 mu |grad xi|^2 J^2)).
double or_time_step(const double *xim, const double *etm, const double *zem, const double *de,
                    const double *yaco, const double *ssk, const double umf[3], double cfl,
                    int64_t n) {
    double m1, m2;
    time_step_maxima(xim, etm, zem, de, nullptr, yaco, ssk, 0.0, umf, n, &m1, &m2);
    double a = cfl / m1, b = 0.5 / m2;
    return a < b ? a : b;
}

double or_time_step_m(const double *de, or_metrics m, double mu, const double umf[3], double cfl,
                      int64_t n) {
    double m1, m2;
    time_step_maxima(m.xim, m.etm, m.zem, de, &m, m.yaco, nullptr, mu, umf, n, &m1, &m2);
    double a = cfl / m1, b = 0.5 / m2;
    return a < b ? a : b;
}

// Primitive recovery (the slot at driver/canard.cu:142-143; CANARD units
// rho_inf = 1, c_inf = 1, p_inf = 1/gamma, so T is stored as c^2 = gamma p / rho,
// consistent with the sqrt(de4*...) sound speed of src/cuda/kernels/physics.hpp:404).
void or_thermo(const double *q, double *de, double *p, int64_t n) {
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        double rhoi = 1.0 / q[i];
        double u = q[n + i] * rhoi, v = q[2 * n + i] * rhoi, w = q[3 * n + i] * rhoi;
        double pp = kGamm1 * (q[4 * n + i] - 0.5 * (q[n + i] * u + q[2 * n + i] * v + q[3 * n + i] * w));
        de[i] = rhoi;
        de[n + i] = u;
        de[2 * n + i] = v;
        de[3 * n + i] = w;
        de[4 * n + i] = kGam * pp * rhoi;
        p[i] = pp;
    }
}

// Intended calc_viscous_shear_stress (src/physics_pc.hpp:151-227 and kernels
// src/cuda/kernels/physics.hpp:211-333), with two reference defects fixed:
// the chain rule uses the derivatives (the reference passes the underived
// buffer) and each axis uses its own ndf (the reference swaps axes 0 and 2).
int or_viscous(const double *de, double mu, or_metrics m, int lxi, int let, int lze,
               const int ndf[2][3], const double *pbco, const double *pbci, double *tau,
               double *heat) {
    const int64_t n = (int64_t)lxi * let * lze;
    std::vector<double> g(3 * n), ss(3 * n);
    // slot targets of calc_viscous_shear_stress_post_compute_kernel<m> (physics.hpp:239-263)
    double *out[5][3] = {{nullptr, nullptr, nullptr},
                         {tau + 0 * n, heat + 2 * n, tau + 5 * n},   // u: xx, heat.zz, zx
                         {tau + 3 * n, tau + 1 * n, heat + 0 * n},   // v: xy, yy, heat.xx
                         {heat + 1 * n, tau + 4 * n, tau + 2 * n},   // w: heat.yy, yz, zz
                         {ss.data(), ss.data() + n, ss.data() + 2 * n}};  // T
    for (int v = 1; v < 5; ++v) {
        for (int a = 0; a < 3; ++a) {
            int rc = or_deriv(de + v * n, g.data() + a * n, lxi, let, lze, a, ndf[0][a], ndf[1][a],
                              nullptr, nullptr, 0, pbco, pbci);
            if (rc) return rc;
        }
#pragma omp parallel for
        for (int64_t i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k)
                out[v][k][i] = metric(m.xim, m.c_xim, k, n, i) * g[i] +
                               metric(m.etm, m.c_etm, k, n, i) * g[n + i] +
                               metric(m.zem, m.c_zem, k, n, i) * g[2 * n + i];
    }
    // calc_viscous_shear_stress_final_kernel (physics.hpp:285-333)
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        double muj = mu * jac(m, i);
        double kap = kGamm1Prndtli * muj;
        double ux = tau[0 * n + i], vy = tau[1 * n + i], wz = tau[2 * n + i];
        double vx = tau[3 * n + i], wy = tau[4 * n + i], uz = tau[5 * n + i];
        double vz = heat[0 * n + i], wx = heat[1 * n + i], uy = heat[2 * n + i];
        double div = 2.0 / 3.0 * (ux + vy + wz);
        double txx = muj * (2.0 * ux - div), tyy = muj * (2.0 * vy - div), tzz = muj * (2.0 * wz - div);
        double txy = muj * (vx + uy), tyz = muj * (wy + vz), tzx = muj * (uz + wx);
        double u = de[n + i], v = de[2 * n + i], w = de[3 * n + i];
        tau[0 * n + i] = txx; tau[1 * n + i] = tyy; tau[2 * n + i] = tzz;
        tau[3 * n + i] = txy; tau[4 * n + i] = tyz; tau[5 * n + i] = tzx;
        heat[0 * n + i] = kap * ss[i] + u * txx + v * txy + w * tzx;
        heat[1 * n + i] = kap * ss[n + i] + u * txy + v * tyy + w * tyz;
        heat[2 * n + i] = kap * ss[2 * n + i] + u * tzx + v * tyz + w * tzz;
    }
    return 0;
}

// physics::calc_viscous_shear_stress + physics::calc_fluxes
// (src/physics_pc.hpp:83-227): de[m] = sum_a d_a F[m][a].
int or_rhs(const double *q, double *rhs, double mu, or_metrics m, const double umf[3], int lxi,
           int let, int lze, const int ndf[2][3], int viscous, double *drva_x) {
    return or_rhs_scaled(q, rhs, mu, m, umf, lxi, let, lze, ndf, viscous, drva_x, nullptr);
}

int or_rhs_scaled(const double *q, double *rhs, double mu, or_metrics m, const double umf[3],
                  int lxi, int let, int lze, const int ndf[2][3], int viscous, double *drva_x,
                  double *scale5) {
    ensure_coeffs();
    const int64_t n = (int64_t)lxi * let * lze;
    std::vector<double> de(5 * n), p(n), tau, heat;
    or_thermo(q, de.data(), p.data(), n);
    if (viscous) {
        tau.resize(6 * n);
        heat.resize(3 * n);
        int rc = or_viscous(de.data(), mu, m, lxi, let, lze, ndf, g_pbco, g_pbci, tau.data(), heat.data());
        if (rc) return rc;
    }
    std::vector<double> xim(3 * n), etm(3 * n), zem(3 * n);
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            xim[c * n + i] = metric(m.xim, m.c_xim, c, n, i);
            etm[c * n + i] = metric(m.etm, m.c_etm, c, n, i);
            zem[c * n + i] = metric(m.zem, m.c_zem, c, n, i);
        }
    std::vector<double> buf(15 * n), d(n), absum(scale5 ? n : 0);
    or_fluxes_pre(buf.data(), q, p.data(), de.data(), xim.data(), etm.data(), zem.data(),
                  viscous ? tau.data() : nullptr, viscous ? heat.data() : nullptr, umf, n);
    for (int v = 0; v < 5; ++v) {
        for (int a = 0; a < 3; ++a) {
            int rc = or_deriv(buf.data() + (v * 3 + a) * n, d.data(), lxi, let, lze, a, ndf[0][a],
                              ndf[1][a], nullptr, a == 0 ? drva_x : nullptr, v, g_pbco, g_pbci);
            if (rc) return rc;
            // calc_fluxes_post_compute_kernel<m> (physics.hpp:195-209)
            double *r = rhs + v * n;
            if (a == 0) {
#pragma omp parallel for
                for (int64_t i = 0; i < n; ++i) r[i] = d[i];
            } else {
#pragma omp parallel for
                for (int64_t i = 0; i < n; ++i) r[i] += d[i];
            }
            if (scale5) {
                double *s = absum.data();
                if (a == 0) {
#pragma omp parallel for
                    for (int64_t i = 0; i < n; ++i) s[i] = std::fabs(d[i]);
                } else {
#pragma omp parallel for
                    for (int64_t i = 0; i < n; ++i) s[i] += std::fabs(d[i]);
                }
            }
        }
        if (scale5) {
            double mx = 0.0;
#pragma omp parallel for reduction(max : mx)
            for (int64_t i = 0; i < n; ++i) mx = absum[i] > mx ? absum[i] : mx;
            scale5[v] = mx;
        }
    }
    return 0;
}

// GCBC non-reflective on the x faces: gcbc_setup_kernel (flag = 1) then
// gcbc_update_non_reflective_kernel (src/cuda/kernels/gcbc.hpp:251-454) with
// the characteristic matrices of gcbc_vgpr (:38-158).  Defects fixed here:
// xtq2r dm[2] = aoi*cm[2], xt[0][4] = -ho*cm[0], xt[4][0] = 1-bo+co (so that
// xtq2r is the inverse of xtr2q); de updated at (plane, variable) instead of
// the accumulating out_idx; face 1 at plane dim-1 (not dim); face_idx
// includes the thread index.
int or_gcbc_x(double *rhs, const double *drva_x, const double *cm, const double *q,
              const double *yaco, const double *sbcc, double c_yaco, const double umf[3],
              int lxi, int let, int lze, const int nbc[2][3]) {
    const int64_t n = (int64_t)lxi * let * lze;
    const int64_t F = (int64_t)let * lze;
    for (int ip = 0; ip < 2; ++ip) {
        if (nbc[ip][0] != kBcNonReflective) continue;
#pragma omp parallel for
        for (int64_t fi = 0; fi < F; ++fi) {
            const int64_t idx = fi * lxi + (ip ? lxi - 1 : 0);
            const double c[3] = {cm[(ip * 3 + 0) * F + fi], cm[(ip * 3 + 1) * F + fi],
                                 cm[(ip * 3 + 2) * F + fi]};
            const double rho = q[idx];
            const double rhoi = 1.0 / rho;
            const double ve[3] = {q[n + idx] * rhoi, q[2 * n + idx] * rhoi, q[3 * n + idx] * rhoi};
            const double hv2 = 0.5 * (ve[0] * ve[0] + ve[1] * ve[1] + ve[2] * ve[2]);
            const double pp = kGamm1 * (q[4 * n + idx] - rho * hv2);
            const double ao = std::sqrt(kGam * rhoi * pp), aoi = 1.0 / ao;
            const double vn = c[0] * ve[0] + c[1] * ve[1] + c[2] * ve[2];
            const double vs = c[0] * umf[0] + c[1] * umf[1] + c[2] * umf[2];
            // xtq2r (conservative -> characteristic)
            double L[5][5];
            {
                double ho = kGamm1 * aoi * aoi, bo = 1.0 - ho * hv2, co = aoi * vn;
                double dm[3] = {aoi * c[0], aoi * c[1], aoi * c[2]};
                double rv[3] = {ho * ve[0], ho * ve[1], ho * ve[2]};
                double t[5][5] = {
                    {bo * c[0] + dm[1] * ve[2] - dm[2] * ve[1], c[0] * rv[0], c[0] * rv[1] + dm[2], c[0] * rv[2] - dm[1], -ho * c[0]},
                    {bo * c[1] + dm[2] * ve[0] - dm[0] * ve[2], c[1] * rv[0] - dm[2], c[1] * rv[1], c[1] * rv[2] + dm[0], -ho * c[1]},
                    {bo * c[2] + dm[0] * ve[1] - dm[1] * ve[0], c[2] * rv[0] + dm[1], c[2] * rv[1] - dm[0], c[2] * rv[2], -ho * c[2]},
                    {1.0 - bo - co, dm[0] - rv[0], dm[1] - rv[1], dm[2] - rv[2], ho},
                    {1.0 - bo + co, -dm[0] - rv[0], -dm[1] - rv[1], -dm[2] - rv[2], ho}};
                std::memcpy(L, t, sizeof t);
            }
            double J = yaco ? yaco[idx] : c_yaco;
            double cha[5], dr[5];
            for (int v = 0; v < 5; ++v) dr[v] = J * drva_x[ip * 5 * F + v * F + fi];
            for (int r = 0; r < 5; ++r) {
                double s = 0.0;
                for (int k = 0; k < 5; ++k) s += L[r][k] * dr[k];
                cha[r] = s;
            }
            // zero the incoming acoustic characteristics
            double del[5] = {0, 0, 0, 0, 0};
            const double ra0 = 1.0 - 2.0 * ip;
            if (ra0 * (vn + vs + ao) > 0) del[3] = -cha[3];
            if (ra0 * (vn + vs - ao) > 0) del[4] = -cha[4];
            // xtr2q (characteristic -> conservative)
            double S[5][5];
            {
                double bo = hv2 + kHamm1 * ao * ao, co = ao * vn;
                double dm[3] = {ao * c[0], ao * c[1], ao * c[2]};
                double t[5][5] = {
                    {c[0], c[1], c[2], 0.5, 0.5},
                    {c[0] * ve[0], c[1] * ve[0] - dm[2], c[2] * ve[0] + dm[1], 0.5 * (ve[0] + dm[0]), 0.5 * (ve[0] + dm[0]) - dm[0]},
                    {c[0] * ve[1] + dm[2], c[1] * ve[1], c[2] * ve[1] - dm[0], 0.5 * (ve[1] + dm[1]), 0.5 * (ve[1] + dm[1]) - dm[1]},
                    {c[0] * ve[2] - dm[1], c[1] * ve[2] + dm[0], c[2] * ve[2], 0.5 * (ve[2] + dm[2]), 0.5 * (ve[2] + dm[2]) - dm[2]},
                    {hv2 * c[0] + dm[2] * ve[1] - dm[1] * ve[2], hv2 * c[1] + dm[0] * ve[2] - dm[2] * ve[0],
                     hv2 * c[2] + dm[1] * ve[0] - dm[0] * ve[1], 0.5 * (bo + co), 0.5 * (bo + co) - co}};
                std::memcpy(S, t, sizeof t);
            }
            double dq[5];
            for (int r = 0; r < 5; ++r) {
                double s = 0.0;
                for (int k = 0; k < 5; ++k) s += S[r][k] * del[k];
                dq[r] = s;
            }
            const int iq = 1 - 2 * ip;
            for (int ii = 0; ii < kMbci; ++ii) {
                int64_t o = idx + (int64_t)ii * iq;
                for (int v = 0; v < 5; ++v) rhs[v * n + o] += sbcc[o] * dq[v];
            }
        }
    }
    return 0;
}

// Characteristic state of one face point (gcbc_vgpr::eleme,
// src/cuda/kernels/gcbc.hpp:43-57): face normal c, density, momenta, pressure.
struct GcPt {
    double c[3], ve[3], hv2, ao, aoi, vn, vs;
};
static GcPt gc_eleme(const double c[3], double rho, const double m[3], double pp, const double umf[3]) {
    GcPt g;
    const double rhoi = 1.0 / rho;
    for (int k = 0; k < 3; ++k) g.c[k] = c[k];
    g.ao = std::sqrt(kGam * rhoi * pp);
    g.aoi = 1.0 / g.ao;
    g.ve[0] = rhoi * m[0];
    g.ve[1] = rhoi * m[1];
    g.ve[2] = rhoi * m[2];
    g.hv2 = 0.5 * (g.ve[0] * g.ve[0] + g.ve[1] * g.ve[1] + g.ve[2] * g.ve[2]);
    g.vn = c[0] * g.ve[0] + c[1] * g.ve[1] + c[2] * g.ve[2];
    g.vs = c[0] * umf[0] + c[1] * umf[1] + c[2] * umf[2];
    return g;
}
// xtq2r (conservative -> characteristic, :109-150) with its three typos fixed.
static void gc_xtq2r(const GcPt &g, double L[5][5]) {
    const double *c = g.c, *ve = g.ve;
    const double ho = kGamm1 * g.aoi * g.aoi, bo = 1.0 - ho * g.hv2, co = g.aoi * g.vn;
    const double dm[3] = {g.aoi * c[0], g.aoi * c[1], g.aoi * c[2]};
    const double rv[3] = {ho * ve[0], ho * ve[1], ho * ve[2]};
    const double t[5][5] = {
        {bo * c[0] + dm[1] * ve[2] - dm[2] * ve[1], c[0] * rv[0], c[0] * rv[1] + dm[2], c[0] * rv[2] - dm[1], -ho * c[0]},
        {bo * c[1] + dm[2] * ve[0] - dm[0] * ve[2], c[1] * rv[0] - dm[2], c[1] * rv[1], c[1] * rv[2] + dm[0], -ho * c[1]},
        {bo * c[2] + dm[0] * ve[1] - dm[1] * ve[0], c[2] * rv[0] + dm[1], c[2] * rv[1] - dm[0], c[2] * rv[2], -ho * c[2]},
        {1.0 - bo - co, dm[0] - rv[0], dm[1] - rv[1], dm[2] - rv[2], ho},
        {1.0 - bo + co, -dm[0] - rv[0], -dm[1] - rv[1], -dm[2] - rv[2], ho}};
    std::memcpy(L, t, sizeof t);
}
// xtr2q (characteristic -> conservative, :59-107).
static void gc_xtr2q(const GcPt &g, double S[5][5]) {
    const double *c = g.c, *ve = g.ve;
    const double bo = g.hv2 + kHamm1 * g.ao * g.ao, co = g.ao * g.vn;
    const double dm[3] = {g.ao * c[0], g.ao * c[1], g.ao * c[2]};
    const double t[5][5] = {
        {c[0], c[1], c[2], 0.5, 0.5},
        {c[0] * ve[0], c[1] * ve[0] - dm[2], c[2] * ve[0] + dm[1], 0.5 * (ve[0] + dm[0]), 0.5 * (ve[0] + dm[0]) - dm[0]},
        {c[0] * ve[1] + dm[2], c[1] * ve[1], c[2] * ve[1] - dm[0], 0.5 * (ve[1] + dm[1]), 0.5 * (ve[1] + dm[1]) - dm[1]},
        {c[0] * ve[2] - dm[1], c[1] * ve[2] + dm[0], c[2] * ve[2], 0.5 * (ve[2] + dm[2]), 0.5 * (ve[2] + dm[2]) - dm[2]},
        {g.hv2 * c[0] + dm[2] * ve[1] - dm[1] * ve[2], g.hv2 * c[1] + dm[0] * ve[2] - dm[2] * ve[0],
         g.hv2 * c[2] + dm[1] * ve[0] - dm[0] * ve[1], 0.5 * (bo + co), 0.5 * (bo + co) - co}};
    std::memcpy(S, t, sizeof t);
}
static void gc_matvec(const double A[5][5], const double *x, double *y) {
    for (int r = 0; r < 5; ++r) {
        double v = 0.0;
        for (int k = 0; k < 5; ++k) v += A[r][k] * x[k];
        y[r] = v;
    }
}

// Point `fi` of face ip of axis a: linear index of its face point and the
// stride into the block (face index convention of the derivative's drva).
static int64_t gc_face_point(int a, int ip, int64_t fi, int lxi, int let, int lze, int64_t &stride) {
    int64_t base;
    int dim;
    if (a == 0) { base = fi * lxi; stride = 1; dim = lxi; }
    else if (a == 1) { base = (fi / lxi) * (int64_t)lxi * let + fi % lxi; stride = lxi; dim = let; }
    else { base = fi; stride = (int64_t)lxi * let; dim = lze; }
    return base + (int64_t)(ip ? dim - 1 : 0) * stride;
}

// gcbc_go (src/gcbc.hpp:86-186) on every face, single rank: gcbc_setup_kernel
// (src/cuda/kernels/gcbc.hpp:251-342) turns drva of non-reflective, wall and
// curvilinear-interface faces into characteristic form in place (from drva,
// flag 1, on non-reflective faces; from the full right-hand side J de, flag 0,
// on the others); the GCIC exchange copies drva of face 1-ip into drvb of
// face ip for curvilinear-interface faces (the block is its own neighbour,
// as mpi exchange::trigger pairs them, src/gcbc.hpp:132-157); then the
// update kernels (:344-695) add sbcc * xtr2q * (cha - drva) to de on mbci
// planes.  Defects fixed as in or_gcbc_x, and the wall update subtracts drva
// from cha as the other two do (gcbc_update_wall_kernel adds xtr2q * cha,
// the whole characteristic right-hand side, :531-545).
int or_gcbc_go(double *drva[3], const double *cm[3], double *drvb[3], const double *qa, double *de,
               const double *p, const double *yaco, const double *sbcc, const double umf[3],
               const double dudtmf[3], int lxi, int let, int lze, double dtwi, const int nbc[2][3]) {
    const int64_t n = (int64_t)lxi * let * lze;
    const int dims[3] = {lxi, let, lze};
    auto active = [](int np) {
        return np == kBcNonReflective || np == 20 || np == 25 || np == 30;
    };
    for (int a = 0; a < 3; ++a) {
        const int64_t F = a == 0 ? (int64_t)let * lze : (a == 1 ? (int64_t)lxi * lze : (int64_t)lxi * let);
        for (int ip = 0; ip < 2; ++ip) {
            const int np = nbc[ip][a];
            if (!active(np)) continue;
            if (dims[a] < 2 || !drva[a] || !cm[a]) return -1;
            const bool flag = np == kBcNonReflective;
            for (int64_t fi = 0; fi < F; ++fi) {
                int64_t stride;
                const int64_t idx = gc_face_point(a, ip, fi, lxi, let, lze, stride);
                const double c[3] = {cm[a][(ip * 3 + 0) * F + fi], cm[a][(ip * 3 + 1) * F + fi],
                                     cm[a][(ip * 3 + 2) * F + fi]};
                const double m[3] = {qa[n + idx], qa[2 * n + idx], qa[3 * n + idx]};
                const GcPt g = gc_eleme(c, qa[idx], m, p[idx], umf);
                double L[5][5], src[5], cha[5];
                gc_xtq2r(g, L);
                for (int v = 0; v < 5; ++v)
                    src[v] = yaco[idx] * (flag ? drva[a][(ip * 5 + v) * F + fi] : de[v * n + idx]);
                gc_matvec(L, src, cha);
                for (int v = 0; v < 5; ++v) drva[a][(ip * 5 + v) * F + fi] = cha[v];
            }
        }
    }
    for (int a = 0; a < 3; ++a) {
        const int64_t F = a == 0 ? (int64_t)let * lze : (a == 1 ? (int64_t)lxi * lze : (int64_t)lxi * let);
        for (int ip = 0; ip < 2; ++ip)
            if (nbc[ip][a] == 30) {
                if (!drvb[a]) return -1;
                std::memcpy(drvb[a] + (int64_t)ip * 5 * F, drva[a] + (int64_t)(1 - ip) * 5 * F, 5 * F * sizeof(double));
            }
    }
    for (int a = 0; a < 3; ++a) {
        const int64_t F = a == 0 ? (int64_t)let * lze : (a == 1 ? (int64_t)lxi * lze : (int64_t)lxi * let);
        for (int ip = 0; ip < 2; ++ip) {
            const int np = nbc[ip][a];
            if (!active(np)) continue;
            const double ra0 = 1.0 - 2.0 * ip;
            for (int64_t fi = 0; fi < F; ++fi) {
                int64_t stride;
                const int64_t idx = gc_face_point(a, ip, fi, lxi, let, lze, stride);
                const double c[3] = {cm[a][(ip * 3 + 0) * F + fi], cm[a][(ip * 3 + 1) * F + fi],
                                     cm[a][(ip * 3 + 2) * F + fi]};
                const double m[3] = {qa[n + idx], qa[2 * n + idx], qa[3 * n + idx]};
                const GcPt g = gc_eleme(c, qa[idx], m, p[idx], umf);
                double dr[5], cha[5], dq[5], S[5][5];
                for (int v = 0; v < 5; ++v) cha[v] = dr[v] = drva[a][(ip * 5 + v) * F + fi];
                if (np == kBcNonReflective) {
                    if (ra0 * (g.vn + g.vs + g.ao) > 0) cha[3] = 0.0;
                    if (ra0 * (g.vn + g.vs - g.ao) > 0) cha[4] = 0.0;
                } else if (np == 30) {
                    double dh[5];
                    for (int v = 0; v < 5; ++v) dh[v] = drvb[a][(ip * 5 + v) * F + fi];
                    if (ra0 * (g.vn + g.vs) > 0) { cha[0] = dh[0]; cha[1] = dh[1]; cha[2] = dh[2]; }
                    if (ra0 * (g.vn + g.vs + g.ao) > 0) cha[3] = dh[3];
                    if (ra0 * (g.vn + g.vs - g.ao) > 0) cha[4] = dh[4];
                } else {
                    const double acc = c[0] * dudtmf[0] + c[1] * dudtmf[1] + c[2] * dudtmf[2];
                    cha[3 + ip] = cha[4 - ip] + 2.0 * ra0 * g.aoi * qa[idx] * (acc + dtwi * (g.vn + g.vs));
                }
                for (int v = 0; v < 5; ++v) cha[v] -= dr[v];
                gc_xtr2q(g, S);
                gc_matvec(S, cha, dq);
                const int iq = 1 - 2 * ip;
                for (int ii = 0; ii < kMbci && ii < dims[a]; ++ii) {
                    const int64_t o = idx + (int64_t)ii * iq * stride;
                    for (int v = 0; v < 5; ++v) de[v * n + o] += sbcc[o] * dq[v];
                }
            }
        }
    }
    return 0;
}

// One step of the driver's RK loop (driver/canard.cu:132-224), with the
// update the reference leaves empty (movef, src/physics_base.hpp:147-150):
// four stages q^(k) = q^n - dt/(nkrk-k) * J * rhs(q^(k-1)), k = 0..3
// (the 1-based dt/(nkrk-nk+1) of the driver, see driver/canard.cu:199).
double or_rk_step(double *q, double mu, or_metrics m, const double umf[3], int lxi, int let,
                  int lze, const int nbc[2][3], int viscous, double dt, double cfl, int gcbc) {
    ensure_coeffs();
    const int64_t n = (int64_t)lxi * let * lze;
    int ndf[2][3];
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 3; ++a) ndf[f][a] = nbc[f][a] >= 35 ? 1 : 0;
    if (dt <= 0.0) {
        std::vector<double> de(5 * n), p(n);
        or_thermo(q, de.data(), p.data(), n);
        dt = or_time_step_m(de.data(), m, mu, umf, cfl, n);
    }
    std::vector<double> qn(q, q + 5 * n), rhs(5 * n), qk(q, q + 5 * n);
    std::vector<double> drva, cm, sbcc;
    const int64_t F = (int64_t)let * lze;
    if (gcbc) {
        drva.assign(10 * F, 0.0);
        cm.assign(6 * F, 0.0);
        for (int64_t i = 0; i < F; ++i) { cm[i] = 1.0; cm[3 * F + i] = 1.0; }
        if (m.xim) {
            // curvilinear: the face normal is grad(xi) / |grad(xi)| at the face point
            for (int ip = 0; ip < 2; ++ip)
                for (int64_t fi = 0; fi < F; ++fi) {
                    const int64_t idx = fi * lxi + (ip ? lxi - 1 : 0);
                    const double x0 = m.xim[idx], x1 = m.xim[n + idx], x2 = m.xim[2 * n + idx];
                    const double nrm = std::sqrt(x0 * x0 + x1 * x1 + x2 * x2);
                    cm[(ip * 3 + 0) * F + fi] = x0 / nrm;
                    cm[(ip * 3 + 1) * F + fi] = x1 / nrm;
                    cm[(ip * 3 + 2) * F + fi] = x2 / nrm;
                }
        }
        sbcc.assign(n, 0.0);
        for (int64_t fi = 0; fi < F; ++fi) {
            int64_t i0 = fi * lxi, i1 = fi * lxi + lxi - 1;
            sbcc[i0] = 1.0 / (m.yaco ? m.yaco[i0] : m.c_yaco);
            sbcc[i1] = 1.0 / (m.yaco ? m.yaco[i1] : m.c_yaco);
        }
    }
    for (int k = 0; k < 4; ++k) {
        int rc = or_rhs(qk.data(), rhs.data(), mu, m, umf, lxi, let, lze, ndf, viscous,
                        gcbc ? drva.data() : nullptr);
        if (rc) return -1.0;
        if (gcbc)
            or_gcbc_x(rhs.data(), drva.data(), cm.data(), qk.data(), m.yaco, sbcc.data(), m.c_yaco,
                      umf, lxi, let, lze, nbc);
        const double dtk = dt / (4 - k);
#pragma omp parallel for
        for (int64_t i = 0; i < n; ++i) {
            double J = jac(m, i);
            for (int v = 0; v < 5; ++v) qk[v * n + i] = qn[v * n + i] - dtk * J * rhs[v * n + i];
        }
    }
    std::memcpy(q, qk.data(), sizeof(double) * 5 * n);
    return dt;
}

double or_rk_stage(const double *qn, const double *qin, double *qout, int k, double dt, double mu,
                   or_metrics m, const double umf[3], int lxi, int let, int lze, const int nbc[2][3],
                   int viscous) {
    ensure_coeffs();
    const int64_t n = (int64_t)lxi * let * lze;
    int ndf[2][3];
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 3; ++a) ndf[f][a] = nbc[f][a] >= 35 ? 1 : 0;
    std::vector<double> rhs(5 * n);
    if (or_rhs(qin, rhs.data(), mu, m, umf, lxi, let, lze, ndf, viscous, nullptr)) return -1.0;
    const double dtk = dt / (4 - k);
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) {
        const double J = jac(m, i);
        for (int v = 0; v < 5; ++v) qout[v * n + i] = qn[v * n + i] - dtk * J * rhs[v * n + i];
    }
    return dt;
}

// Metrics and Jacobian of a curvilinear grid.  The reference's grid class only
// generates coordinates (grid::generate, src/grid.hpp:89-213); the metric
// arrays its physics kernels read (xim, etm, zem = J^-1 grad xi_a, yaco = J,
// src/cuda/kernels/physics.hpp:42-193) have no generator there.  This is the
// cross-product form with index-space compact derivatives r_a = d r / d xi_a:
//   xim = r_eta x r_zeta,  etm = r_zeta x r_xi,  zem = r_xi x r_eta,
//   yaco = 1 / (r_xi . xim).
// On an axis with interface closures the coordinate c is split into a
// periodic part and a ramp, c = c~ + i_a * s, s = period[a][c] / n_a, and
// r_a = D c~ + s.
int or_grid_metrics(const double *xyz, const double period[3][3], int lxi, int let, int lze,
                    const int ndf[2][3], double *xim, double *etm, double *zem, double *yaco) {
    ensure_coeffs();
    const int64_t n = (int64_t)lxi * let * lze;
    const int dims[3] = {lxi, let, lze};
    std::vector<double> d(9 * n), tmp(n);
    for (int a = 0; a < 3; ++a) {
        const bool ramp = ndf[0][a] || ndf[1][a];
        for (int c = 0; c < 3; ++c) {
            const double sl = ramp ? period[a][c] / dims[a] : 0.0;
            const double *src = xyz + c * n;
#pragma omp parallel for
            for (int64_t i = 0; i < n; ++i) {
                const int64_t ia = a == 0 ? i % lxi : (a == 1 ? (i / lxi) % let : i / ((int64_t)lxi * let));
                tmp[i] = src[i] - (double)ia * sl;
            }
            double *dc = d.data() + (a * 3 + c) * n;
            int rc = or_deriv(tmp.data(), dc, lxi, let, lze, a, ndf[0][a], ndf[1][a], nullptr, nullptr, 0,
                              g_pbco, g_pbci);
            if (rc) return rc;
#pragma omp parallel for
            for (int64_t i = 0; i < n; ++i) dc[i] += sl;
        }
    }
    int err = 0;
#pragma omp parallel for reduction(|: err)
    for (int64_t i = 0; i < n; ++i) {
        double r[3][3];
        for (int a = 0; a < 3; ++a)
            for (int c = 0; c < 3; ++c) r[a][c] = d[(a * 3 + c) * n + i];
        double *out[3] = {xim, etm, zem};
        for (int a = 0; a < 3; ++a) {
            const double *p = r[(a + 1) % 3], *q = r[(a + 2) % 3];
            out[a][i] = p[1] * q[2] - p[2] * q[1];
            out[a][n + i] = p[2] * q[0] - p[0] * q[2];
            out[a][2 * n + i] = p[0] * q[1] - p[1] * q[0];
        }
        const double vol = r[0][0] * xim[i] + r[0][1] * xim[n + i] + r[0][2] * xim[2 * n + i];
        if (!(vol != 0.0)) err = 1;
        yaco[i] = 1.0 / vol;
    }
    return err ? -2 : 0;
}

// splitmix64 of (seed, index) mapped to [-1, 1): a counter-based generator
// that a GPU thread, numpy and this file all evaluate identically.
double or_noise(uint64_t seed, uint64_t index) {
    uint64_t z = seed * 0x9E3779B97F4A7C15ull + index + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

void or_fourier_field(int lxi, int let, int lze, uint64_t seed, int nmodes, double *modes, double *f) {
    const double two_pi = 6.283185307179586476925286766559;
    std::mt19937_64 g(seed);
    auto u = [&g]() { return (double)(g() >> 11) * (1.0 / 9007199254740992.0); };
    std::vector<double> m((size_t)nmodes * 5);
    for (int k = 0; k < nmodes; ++k) {
        double *r = &m[(size_t)k * 5];
        r[0] = 0.1 + 0.9 * u();
        for (int a = 1; a <= 3; ++a) r[a] = 1.0 + std::floor(8.0 * u());
        r[4] = two_pi * u();
    }
    if (modes) std::memcpy(modes, m.data(), m.size() * sizeof(double));
    if (!f) return;
    const int64_t n = (int64_t)lxi * let * lze;
    const double hx = 1.0 / (lxi - 1), hy = 1.0 / (let - 1), hz = 1.0 / (lze - 1);
#pragma omp parallel for
    for (int64_t idx = 0; idx < n; ++idx) {
        const int64_t i = idx % lxi, j = (idx / lxi) % let, k = idx / ((int64_t)lxi * let);
        const double x = i * hx, y = j * hy, z = k * hz;
        double s = 0.0;
        for (int q = 0; q < nmodes; ++q) {
            const double *r = &m[(size_t)q * 5];
            s += r[0] * std::sin(two_pi * (r[1] * x + r[2] * y + r[3] * z) + r[4]);
        }
        f[idx] = s;
    }
}

void or_tgv_init(double *q, int lxi, int let, int lze, double mach, double amp, uint64_t seed) {
    const int64_t n = (int64_t)lxi * let * lze;
    const double two_pi = 6.283185307179586476925286766559;
    const double hx = two_pi / lxi, hy = two_pi / let, hz = two_pi / lze;
    const double u0 = mach, p0 = 1.0 / kGam;
#pragma omp parallel for
    for (int64_t idx = 0; idx < n; ++idx) {
        int64_t i = idx % lxi, j = (idx / lxi) % let, k = idx / ((int64_t)lxi * let);
        double x = i * hx, y = j * hy, z = k * hz;
        double u = u0 * std::sin(x) * std::cos(y) * std::cos(z);
        double v = -u0 * std::cos(x) * std::sin(y) * std::cos(z);
        double w = 0.0;
        double p = p0 + u0 * u0 / 16.0 * (std::cos(2 * x) + std::cos(2 * y)) * (std::cos(2 * z) + 2.0);
        double rho = 1.0 + amp * or_noise(seed, (uint64_t)idx);
        q[idx] = rho;
        q[n + idx] = rho * u;
        q[2 * n + idx] = rho * v;
        q[3 * n + idx] = rho * w;
        q[4 * n + idx] = p * kHamm1 + 0.5 * rho * (u * u + v * v + w * w);
    }
}

// Wall boundary state update: wall_condition_update (src/gcbc.hpp:188-228)
// with wall_inviscid_kernel / wall_viscous_kernel (src/cuda/kernels/gcbc.hpp:160-249).
// Deviations: the face plane is ip * (n - 1) (the reference's ip * n is one
// past the end), and the viscous energy uses the updated momentum.
int or_wall_update(double *q, const int *npex, const double umf[3], int lxi, int let, int lze,
                   const int nbc[6]) {
    const int64_t n = (int64_t)lxi * let * lze;
    const int dims[3] = {lxi, let, lze};
    const double hamhamm1 = (1.0 / kGam) * kHamm1;
    for (int a = 0; a < 3; ++a)
        for (int ip = 0; ip < 2; ++ip) {
            const int code = nbc[ip * 3 + a];
            if (code != 20 && code != 25) continue;
            const int plane = ip * (dims[a] - 1);
            for (int k = 0; k < lze; ++k)
                for (int j = 0; j < let; ++j)
                    for (int i = 0; i < lxi; ++i) {
                        const int c[3] = {i, j, k};
                        if (c[a] != plane) continue;
                        const int64_t idx = i + (int64_t)lxi * (j + (int64_t)let * k);
                        if (npex[idx] != 0) continue;
                        const double rho = q[idx];
                        if (code == 20) {
                            const double m2 = q[n + idx] * q[n + idx] + q[2 * n + idx] * q[2 * n + idx] +
                                              q[3 * n + idx] * q[3 * n + idx];
                            q[4 * n + idx] = hamhamm1 * std::pow(rho, kGam) + 0.5 * m2 / rho;
                        } else {
                            for (int d = 0; d < 3; ++d) q[(1 + d) * n + idx] = -rho * umf[d];
                            const double m2 = q[n + idx] * q[n + idx] + q[2 * n + idx] * q[2 * n + idx] +
                                              q[3 * n + idx] * q[3 * n + idx];
                            q[4 * n + idx] = hamhamm1 * rho + 0.5 * m2 / rho;
                        }
                    }
        }
    return 0;
}

}  // extern "C"
