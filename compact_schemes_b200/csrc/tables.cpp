// tables.cpp -- host-side setup of the compact_schemes_b200 line solver.
//
// Every line of a given length and boundary type shares one tridiagonal
// matrix, so everything in the partitioned solve that depends only on the
// matrix is computed here once, in FP64, and uploaded: the per-lane local
// elimination factors, the coefficients of the 64-row reduced system's PCR
// sweeps and, for cyclic systems, the Sherman-Morrison correction vector.
// The device then only transforms right-hand sides.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "cs_common.h"

namespace csb {

// Interface closure weights (numerics_base::deriv_setup,
// src/numerics_base.hpp:182-297).  Two coupled 8-point blocks form a 16-row
// Pade system P f' = Q f; R = P~ P^-1 Q, where P~ is P without the rows'
// coupling across the block interface.  Rows 8 and 9 of R hold the weights
// a block applies to its neighbour's points (pbco, nearest point first) and
// to its own points (pbci).
//
// P^-1 is formed with the same Gauss-Jordan steps, in the same order, as
// numerics_base::mtrxi (src/numerics_base.hpp:324-386), and the products in
// the order of matmul_square (:388-398).  The weights multiply field values
// in sums that cancel the field's mean, so for fields with a large mean (the
// pressure part of a momentum flux) any last-bit difference in a weight is
// amplified a few hundred times; reproducing the reference's operation order
// makes the weights bit-identical to the reference's.
static void invert_gauss_jordan(int n, const double *m, double *inv) {
    std::vector<double> rx(m, m + n * n), temp(n);
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int i = 0; i < n; ++i) {
        // pivot column: largest |rx| in row i over columns i .. n-2
        const int row0 = i * n + i, count = n - i - 1;
        int best = 0;
        double big = std::fabs(rx[row0]);
        for (int k = 1; k < count; ++k) {
            const double v = std::fabs(rx[row0 + k]);
            if (v > big) { big = v; best = k; }
        }
        const int col = i + best;
        if (col != i) {
            std::swap(perm[col], perm[i]);
            for (int r = 0; r < n; ++r) std::swap(rx[col + r * n], rx[i + r * n]);
        }
        const double piv_inv = 1.0 / rx[i + i * n];
        for (int k = 0; k < n; ++k) temp[k] = rx[k + i * n];
        for (int r = 0; r < n; ++r) {
            const double f = piv_inv * rx[i + r * n];
            for (int k = 0; k < n; ++k) rx[k + r * n] = rx[k + r * n] - f * temp[k];
            rx[i + r * n] = f;
        }
        for (int k = 0; k < n; ++k) rx[k + i * n] = -piv_inv * temp[k];
        rx[i + i * n] = piv_inv;
    }
    for (int r = 0; r < n; ++r)
        for (int k = 0; k < n; ++k) inv[k + perm[r] * n] = rx[k + r * n];
}

void compute_interface_coeffs(Coeffs &cf) {
    const int n = 2 * kLmd;
    std::vector<double> P(n * n, 0.0), Q(n * n, 0.0), Pi(n * n), T(n * n);
    auto p = [&](int r, int c) -> double & { return P[r * n + c]; };
    auto q = [&](int r, int c) -> double & { return Q[r * n + c]; };
    p(0, 0) = 1.0; p(0, 1) = kAlpha01;
    p(1, 0) = kAlpha10; p(1, 1) = 1.0; p(1, 2) = kAlpha10;
    p(n - 1, n - 1) = 1.0; p(n - 1, n - 2) = kAlpha01;
    p(n - 2, n - 1) = kAlpha10; p(n - 2, n - 2) = 1.0; p(n - 2, n - 3) = kAlpha10;
    q(0, 0) = kAb00; q(0, 1) = kAb01; q(0, 2) = kAb02;
    q(1, 0) = -kAb10; q(1, 2) = kAb10;
    q(n - 1, n - 1) = -kAb02; q(n - 1, n - 2) = -kAb01; q(n - 1, n - 3) = -kAb00;
    q(n - 2, n - 1) = kAb10; q(n - 2, n - 3) = -kAb10;
    for (int i = 2; i < n - 2; ++i) {
        p(i, i - 1) = kAlpha; p(i, i) = 1.0; p(i, i + 1) = kAlpha;
        q(i, i - 2) = -kBb; q(i, i - 1) = -kAa; q(i, i + 1) = kAa; q(i, i + 2) = kBb;
    }
    invert_gauss_jordan(n, P.data(), Pi.data());
    // P~: drop the interface coupling of rows 6..9
    p(6, 8) = 0.0; p(7, 8) = 0.0; p(7, 9) = 0.0;
    p(9, 7) = 0.0; p(8, 7) = 0.0; p(8, 6) = 0.0;
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) {
            double acc = 0.0;
            for (int k = 0; k < n; ++k) acc += Pi[r * n + k] * Q[k * n + c];
            T[r * n + c] = acc;
        }
    for (int row = 8; row <= 9; ++row)
        for (int c = 0; c < n; ++c) {
            double acc = 0.0;
            for (int k = 0; k < n; ++k) acc += P[row * n + k] * T[k * n + c];
            if (c < kLmd) cf.pbco[(row - 8) * kLmd + kLmd - 1 - c] = acc;
            else cf.pbci[(row - 8) * kLmd + c - kLmd] = acc;
        }
}

#ifndef CSB_MIN_CHUNK
#define CSB_MIN_CHUNK 2
#endif

int chunk_length(int n, int min_lt) {
    int lt = min_lt > CSB_MIN_CHUNK ? min_lt : CSB_MIN_CHUNK;
    while (lt < 32 && (n + lt - 1) / lt > 32) lt *= 2;
    return lt;
}

void deriv_rows(int n, int nstart, int nend, double *a, double *b, double *c) {
    for (int i = 0; i < n; ++i) { a[i] = kAlpha; b[i] = 1.0; c[i] = kAlpha; }
    a[0] = 0.0;
    c[n - 1] = 0.0;
    if (nstart == 0) {
        c[0] = kAlpha01;
        a[1] = kAlpha10; c[1] = kAlpha10;
    }
    if (nend == 0) {
        a[n - 1] = kAlpha01;
        a[n - 2] = kAlpha10; c[n - 2] = kAlpha10;
    }
}

void filter_rows(int n, bool cyclic, double af, double *a, double *b, double *c) {
    for (int i = 0; i < n; ++i) { a[i] = af; b[i] = 1.0; c[i] = af; }
    if (!cyclic) {
        a[0] = 0.0; c[0] = 0.0;
        a[n - 1] = 0.0; c[n - 1] = 0.0;
    }
}

static void thomas(int n, const double *a, const double *b, const double *c, const double *r,
                   double *x) {
    std::vector<double> cp(n), dp(n);
    cp[0] = c[0] / b[0];
    dp[0] = r[0] / b[0];
    for (int i = 1; i < n; ++i) {
        const double m = b[i] - a[i] * cp[i - 1];
        cp[i] = c[i] / m;
        dp[i] = (r[i] - a[i] * dp[i - 1]) / m;
    }
    x[n - 1] = dp[n - 1];
    for (int i = n - 2; i >= 0; --i) x[i] = dp[i] - cp[i] * x[i + 1];
}

bool build_tables(int n, const double *a_in, const double *b_in, const double *c_in, bool cyclic,
                  HostTables &T, int min_lt) {
    if (n < 5 || n > kMaxLine) return false;
    std::vector<double> a(a_in, a_in + n), b(b_in, b_in + n), c(c_in, c_in + n);
    T = HostTables();
    T.n = n;
    T.cyclic = cyclic;
    if (cyclic) {
        // Sherman-Morrison: A = A' + u v^T with u = (g, 0..0, c[n-1]),
        // v = (1, 0..0, a[0]/g), g = -b[0]; solve A' then correct.
        const double g = -b[0], top = a[0], bottom = c[n - 1];
        b[0] -= g;
        b[n - 1] -= bottom * top / g;
        a[0] = 0.0;
        c[n - 1] = 0.0;
        std::vector<double> u(n, 0.0), z(n);
        u[0] = g;
        u[n - 1] = bottom;
        thomas(n, a.data(), b.data(), c.data(), u.data(), z.data());
        T.cyc_s2 = top / g;
        T.cyc_s1 = 1.0 / (1.0 + z[0] + T.cyc_s2 * z[n - 1]);
        T.cycz = z;  // reshaped below
    }
    const int lt = chunk_length(n, min_lt);
    const int p = (n + lt - 1) / lt;
    T.lt = lt;
    T.p = p;
    T.last_len = n - (p - 1) * lt;
    const int W = 32;
    auto zeros = [&](std::vector<double> &v, double fill = 0.0) { v.assign((size_t)lt * W, fill); };
    zeros(T.fwd1); zeros(T.fwd2); zeros(T.bwd1, 1.0); zeros(T.bwd2); zeros(T.rca); zeros(T.rcc);
    std::vector<double> cz;
    if (cyclic) {
        cz.assign((size_t)lt * W, 0.0);
        for (int j = 0; j < n; ++j) cz[(j % lt) * W + j / lt] = T.cycz[j];
        T.cycz = cz;
    }
    // reduced tridiagonal system, rows r = 2*lane + k
    double ra[64], rb[64], rc[64];
    for (int r = 0; r < 64; ++r) { ra[r] = 0.0; rb[r] = 1.0; rc[r] = 0.0; }
    for (int lane = 0; lane < p; ++lane) {
        const int s = lane * lt;
        const int len = lane < p - 1 ? lt : T.last_len;
        std::vector<double> A(lt, 0.0), C(lt, 0.0);
        auto at = [&](int t) { return (size_t)t * W + lane; };
        for (int t = 0; t < len; ++t) {
            const int j = s + t;
            if (t < 2) {
                T.fwd1[at(t)] = 1.0 / b[j];
                T.fwd2[at(t)] = 0.0;
                A[t] = a[j] / b[j];
                C[t] = c[j] / b[j];
            } else {
                const double r = 1.0 / (b[j] - a[j] * C[t - 1]);
                T.fwd1[at(t)] = r;
                T.fwd2[at(t)] = -r * a[j];
                A[t] = -r * a[j] * A[t - 1];
                C[t] = r * c[j];
            }
        }
        if (len >= 3) {
            for (int t = len - 3; t >= 1; --t) {
                T.bwd1[at(t)] = 1.0;
                T.bwd2[at(t)] = -C[t];
                A[t] = A[t] - C[t] * A[t + 1];
                C[t] = -C[t] * C[t + 1];
            }
            const double r = 1.0 / (1.0 - C[0] * A[1]);
            T.bwd1[at(0)] = r;
            T.bwd2[at(0)] = -r * C[0];
            A[0] = r * A[0];
            C[0] = -r * C[0] * C[1];
        }
        for (int t = 1; t + 1 < len; ++t) {
            T.rca[at(t)] = A[t];
            T.rcc[at(t)] = C[t];
        }
        // first row of the chunk couples (lane-1, last) and (lane, last)
        ra[2 * lane] = A[0];
        rc[2 * lane] = len >= 2 ? C[0] : 0.0;
        if (len >= 2) {
            // last row couples (lane, first) and (lane+1, first)
            ra[2 * lane + 1] = A[len - 1];
            rc[2 * lane + 1] = C[len - 1];
        }
    }
    // PCR on the 64-row reduced system; strides 1, 2, ..., 32.  The depth is
    // the first step count after which every remaining coupling relative to
    // its diagonal is below kPcrTol64 (kPcrTol32): dropping them then changes
    // the solution by less than the arithmetic's own rounding.
    constexpr double kPcrTol64 = 1e-20, kPcrTol32 = 1e-12;
    T.k1.assign(kPcrSteps * 2 * W, 0.0);
    T.k2.assign(kPcrSteps * 2 * W, 0.0);
    T.invb.assign(2 * W, 1.0);
    T.invb32.assign(2 * W, 1.0);
    T.pcr64 = T.pcr32 = kPcrSteps;
    bool have64 = false, have32 = false;
    auto record = [&](int steps) {
        double res = 0.0;
        for (int r = 0; r < 64; ++r) res = std::max(res, (std::fabs(ra[r]) + std::fabs(rc[r])) / std::fabs(rb[r]));
        if (steps == kPcrSteps) res = 0.0;  // the full depth is exact
        if (!have32 && res <= kPcrTol32) {
            have32 = true;
            T.pcr32 = steps;
            for (int r = 0; r < 64; ++r) T.invb32[(size_t)(r & 1) * W + (r >> 1)] = 1.0 / rb[r];
        }
        if (!have64 && res <= kPcrTol64) {
            have64 = true;
            T.pcr64 = steps;
            for (int r = 0; r < 64; ++r) T.invb[(size_t)(r & 1) * W + (r >> 1)] = 1.0 / rb[r];
        }
    };
    for (int st = 0; st < kPcrSteps; ++st) {
        const int sg = 1 << st;
        double na[64], nb[64], nc[64];
        for (int r = 0; r < 64; ++r) {
            const double k1 = r - sg >= 0 ? ra[r] / rb[r - sg] : 0.0;
            const double k2 = r + sg < 64 ? rc[r] / rb[r + sg] : 0.0;
            nb[r] = rb[r] - (r - sg >= 0 ? rc[r - sg] * k1 : 0.0) - (r + sg < 64 ? ra[r + sg] * k2 : 0.0);
            na[r] = r - sg >= 0 ? -ra[r - sg] * k1 : 0.0;
            nc[r] = r + sg < 64 ? -rc[r + sg] * k2 : 0.0;
            T.k1[(size_t)(st * 2 + (r & 1)) * W + (r >> 1)] = k1;
            T.k2[(size_t)(st * 2 + (r & 1)) * W + (r >> 1)] = k2;
        }
        std::memcpy(ra, na, sizeof ra);
        std::memcpy(rb, nb, sizeof rb);
        std::memcpy(rc, nc, sizeof rc);
        // the first step is always run (it couples each lane's two rows)
        if (st >= 1) record(st + 1);
    }
    return true;
}

}  // namespace csb
