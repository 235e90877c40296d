// line_solver.cuh -- device side of the compact_schemes_b200 line solver.
//
// One warp solves one line of n <= 1024 points.  Lane c owns the contiguous
// chunk of rows [c*LT, c*LT + len) in registers.  The solve is the
// partitioned ("modified Thomas" + PCR) algorithm:
//   1. each lane eliminates inside its chunk (forward then backward sweep),
//      leaving its first and last rows coupled only to the neighbouring
//      chunks' end rows;
//   2. the 64-row reduced system (2 rows per lane) is solved by six
//      parallel-cyclic-reduction steps over warp shuffles;
//   3. each lane back-substitutes its interior rows.
// Because every line of one configuration shares its matrix, all elimination
// factors are precomputed on the host (tables.cpp); the device work per row
// is a handful of FMAs on the right-hand side only.
#pragma once

#include <cuda_runtime.h>

#include "cs_common.h"

namespace csb {

// Round-to-nearest products that the compiler may not contract into FMAs:
// the pointwise arithmetic (fluxes, primitives, stencil right-hand sides) is
// written with them in the operation order of a plain C++ evaluation, so its
// results are bit-identical to the FP64 oracle built without contraction.
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }

template <typename CT>
struct DevTables {
    const CT *fwd1, *fwd2, *bwd1, *bwd2, *rca, *rcc, *k1, *k2, *invb, *cycz;
    CT cyc_s1, cyc_s2;
    int n, p, last_len, cyclic;
    int pcr;  // PCR steps run on the reduced system (2..6)
    // every lane's per-row factors (fwd1 .. rcc) equal interior_chunk<LT>'s:
    // warp_solve then takes them as compile-time constants
    int interior;
};

// Shared-memory layout of one line: element j = c*LT + t lives at
// t*32 + ((c + (32/LT)*t) & 31).  Lane c reading its element t touches 32
// consecutive words (conflict free); 32 threads writing consecutive j also
// spread over all banks.
template <int LT>
struct LineLayout {
    static constexpr int kRot = 32 / LT;
    static constexpr int kSlot = 32 * LT + 1;  // odd stride between lines of a tile
    __device__ __forceinline__ static int pos(int j) {
        const int c = j / LT, t = j % LT;
        return t * 32 + ((c + kRot * t) & 31);
    }
    __device__ __forceinline__ static int pos_ct(int c, int t) { return t * 32 + ((c + kRot * t) & 31); }
};

__device__ __forceinline__ int lane_len(int lane, int lt, int p, int last_len) {
    return lane < p - 1 ? lt : (lane == p - 1 ? last_len : 0);
}

// Per-row factors of one full chunk of LT rows of the constant interior rows
// (alpha, 1, alpha) of the compact derivative, computed at compile time with
// the operations and operation order of build_tables (tables.cpp), so that
// they equal the tables of any line whose every chunk is such a chunk (the
// interface / periodic closure with n a multiple of LT; the host checks the
// equality before it sets DevTables::interior).
template <int LT>
struct InteriorChunk {
    double fwd1[LT], fwd2[LT], bwd1[LT], bwd2[LT], rca[LT], rcc[LT];
};
template <int LT>
__host__ __device__ constexpr InteriorChunk<LT> interior_chunk() {
    InteriorChunk<LT> k{};
    double A[LT] = {}, C[LT] = {};
    const double a = kAlpha, b = 1.0, c = kAlpha;
    for (int t = 0; t < LT; ++t) {
        k.bwd1[t] = 1.0;
        if (t < 2) {
            k.fwd1[t] = 1.0 / b;
            k.fwd2[t] = 0.0;
            A[t] = a / b;
            C[t] = c / b;
        } else {
            const double r = 1.0 / (b - a * C[t - 1]);
            k.fwd1[t] = r;
            k.fwd2[t] = -r * a;
            A[t] = -r * a * A[t - 1];
            C[t] = r * c;
        }
    }
    if (LT >= 3) {
        for (int t = LT - 3; t >= 1; --t) {
            k.bwd1[t] = 1.0;
            k.bwd2[t] = -C[t];
            A[t] = A[t] - C[t] * A[t + 1];
            C[t] = -C[t] * C[t + 1];
        }
        const double r = 1.0 / (1.0 - C[0] * A[1]);
        k.bwd1[0] = r;
        k.bwd2[0] = -r * C[0];
        A[0] = r * A[0];
        C[0] = -r * C[0] * C[1];
    }
    for (int t = 1; t + 1 < LT; ++t) {
        k.rca[t] = A[t];
        k.rcc[t] = C[t];
    }
    return k;
}

template <int LT, int NV, typename CT, int W = 32>
__device__ __forceinline__ void warp_solve_interior(const DevTables<CT> &T, CT (&d)[NV][LT], int lane);

// Solve NV right-hand sides held as d[v][t] by the lanes of one warp; the
// solution overwrites d.  All 32 lanes must call it (warp shuffles).  W < 32:
// every W lanes solve a line of their own (lines with p <= W chunks and at
// most log2(W) + 1 PCR steps), `lane` is the lane within its W-lane segment.
template <int LT, int NV, typename CT, int W = 32>
__device__ __forceinline__ void warp_solve(const DevTables<CT> &T, CT (&d)[NV][LT], int lane) {
    if (LT >= 2 && T.interior) {
        warp_solve_interior<LT, NV, CT, W>(T, d, lane);
        return;
    }
    const int len = lane_len(lane, LT, T.p, T.last_len);
#pragma unroll
    for (int t = 0; t < LT; ++t) {
        const CT f1 = T.fwd1[t * 32 + lane];
        if (t == 0) {
#pragma unroll
            for (int v = 0; v < NV; ++v) d[v][0] = f1 * d[v][0];
        } else {
            const CT f2 = T.fwd2[t * 32 + lane];
#pragma unroll
            for (int v = 0; v < NV; ++v) d[v][t] = f1 * d[v][t] + f2 * d[v][t - 1];
        }
    }
#pragma unroll
    for (int t = LT - 2; t >= 0; --t) {
        const CT b1 = T.bwd1[t * 32 + lane], b2 = T.bwd2[t * 32 + lane];
#pragma unroll
        for (int v = 0; v < NV; ++v) d[v][t] = b1 * d[v][t] + b2 * d[v][t + 1];
    }
    CT y0[NV], y1[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        y0[v] = d[v][0];
        y1[v] = CT(0);
#pragma unroll
        for (int t = 1; t < LT; ++t)
            if (t == len - 1) y1[v] = d[v][t];
    }
    {
        const CT ka = T.k1[lane], kb = T.k2[lane], kc = T.k1[32 + lane], kd = T.k2[32 + lane];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const CT up1 = __shfl_up_sync(0xffffffffu, y1[v], 1, W);
            const CT dn0 = __shfl_down_sync(0xffffffffu, y0[v], 1, W);
            const CT n0 = y0[v] - ka * up1 - kb * y1[v];
            const CT n1 = y1[v] - kc * y0[v] - kd * dn0;
            y0[v] = n0;
            y1[v] = n1;
        }
    }
#pragma unroll
    for (int s = 1; s < kPcrSteps; ++s) {
        if (s >= T.pcr) break;
        const int dl = 1 << (s - 1);
        const CT ka = T.k1[s * 64 + lane], kb = T.k2[s * 64 + lane];
        const CT kc = T.k1[s * 64 + 32 + lane], kd = T.k2[s * 64 + 32 + lane];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const CT u0 = __shfl_up_sync(0xffffffffu, y0[v], dl, W);
            const CT d0 = __shfl_down_sync(0xffffffffu, y0[v], dl, W);
            const CT u1 = __shfl_up_sync(0xffffffffu, y1[v], dl, W);
            const CT d1 = __shfl_down_sync(0xffffffffu, y1[v], dl, W);
            y0[v] = y0[v] - ka * u0 - kb * d0;
            y1[v] = y1[v] - kc * u1 - kd * d1;
        }
    }
    const CT ib0 = T.invb[lane], ib1 = T.invb[32 + lane];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const CT X0 = y0[v] * ib0, X1 = y1[v] * ib1;
#pragma unroll
        for (int t = 0; t < LT; ++t) {
            CT x = d[v][t] - T.rca[t * 32 + lane] * X0 - T.rcc[t * 32 + lane] * X1;
            if (t == 0) x = X0;
            if (t != 0 && t == len - 1) x = X1;
            d[v][t] = x;
        }
        if (T.cyclic) {
            const CT last = len >= 2 ? X1 : X0;
            const CT ya = __shfl_sync(0xffffffffu, X0, 0, W);
            const CT yb = __shfl_sync(0xffffffffu, last, T.p - 1, W);
            const CT beta = (ya + T.cyc_s2 * yb) * T.cyc_s1;
#pragma unroll
            for (int t = 0; t < LT; ++t) d[v][t] -= beta * T.cycz[t * 32 + lane];
        }
    }
}

// Per-row factors of a line whose lanes all share them: every chunk is full
// (n a multiple of LT) and the matrix rows that shape a chunk's elimination
// are the constant interior rows, as for the compact derivative with the
// interface (single-rank periodic) closure on both ends.  Only the reduced
// system then differs between lanes.  The factors travel by value in the
// kernel's parameters, so the solve reads them as constants instead of
// loading six per-lane table entries per row.  nra / nrc are the negated
// spike coefficients (rca / rcc of the tables).
template <int LT, typename CT = float>
struct ChunkFactors {
    CT f1[LT], f2[LT], b1[LT], b2[LT], nra[LT], nrc[LT];
};

__device__ __forceinline__ float cf_fma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double cf_fma(double a, double b, double c) { return fma(a, b, c); }

// warp_solve for lines with ChunkFactors (all chunks full, no cyclic
// correction): NV right-hand sides held as d[v][t], FP32 or FP64.  The
// structure of the tables fixes fwd2 = 0 for rows 0 and 1 of a chunk, bwd1 = 1
// and bwd2 = 0 for row LT - 2, and bwd1 = 1 for rows 1 .. LT - 3; those
// products are left out.  All 32 lanes must call it.
template <int LT, int NV, typename CT, int W = 32>
__device__ __forceinline__ void warp_solve_cf(const ChunkFactors<LT, CT> &U, const DevTables<CT> &T,
                                              CT (&d)[NV][LT], int lane) {
    static_assert(LT >= 2, "chunk");
#pragma unroll
    for (int t = 0; t < LT; ++t)
#pragma unroll
        for (int v = 0; v < NV; ++v)
            d[v][t] = t < 2 ? U.f1[t] * d[v][t] : cf_fma(U.f2[t], d[v][t - 1], U.f1[t] * d[v][t]);
#pragma unroll
    for (int t = LT - 3; t >= 0; --t)
#pragma unroll
        for (int v = 0; v < NV; ++v)
            d[v][t] = t == 0 ? cf_fma(U.b2[0], d[v][1], U.b1[0] * d[v][0]) : cf_fma(U.b2[t], d[v][t + 1], d[v][t]);
    CT y0[NV], y1[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        y0[v] = d[v][0];
        y1[v] = d[v][LT - 1];
    }
    {
        const CT ka = T.k1[lane], kb = T.k2[lane], kc = T.k1[32 + lane], kd = T.k2[32 + lane];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const CT up1 = __shfl_up_sync(0xffffffffu, y1[v], 1, W);
            const CT dn0 = __shfl_down_sync(0xffffffffu, y0[v], 1, W);
            const CT n0 = y0[v] - ka * up1 - kb * y1[v];
            const CT n1 = y1[v] - kc * y0[v] - kd * dn0;
            y0[v] = n0;
            y1[v] = n1;
        }
    }
#pragma unroll
    for (int s = 1; s < kPcrSteps; ++s) {
        if (s >= T.pcr) break;
        const int dl = 1 << (s - 1);
        const CT ka = T.k1[s * 64 + lane], kb = T.k2[s * 64 + lane];
        const CT kc = T.k1[s * 64 + 32 + lane], kd = T.k2[s * 64 + 32 + lane];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const CT u0 = __shfl_up_sync(0xffffffffu, y0[v], dl, W);
            const CT d0 = __shfl_down_sync(0xffffffffu, y0[v], dl, W);
            const CT u1 = __shfl_up_sync(0xffffffffu, y1[v], dl, W);
            const CT d1 = __shfl_down_sync(0xffffffffu, y1[v], dl, W);
            y0[v] = y0[v] - ka * u0 - kb * d0;
            y1[v] = y1[v] - kc * u1 - kd * d1;
        }
    }
    const CT ib0 = T.invb[lane], ib1 = T.invb[32 + lane];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const CT X0 = y0[v] * ib0, X1 = y1[v] * ib1;
        d[v][0] = X0;
#pragma unroll
        for (int t = 1; t + 1 < LT; ++t) d[v][t] = cf_fma(U.nrc[t], X1, cf_fma(U.nra[t], X0, d[v][t]));
        d[v][LT - 1] = X1;
    }
}

// warp_solve for tables flagged `interior`: the per-row factors are the
// compile-time interior_chunk<LT> values.
template <int LT, int NV, typename CT, int W>
__device__ __forceinline__ void warp_solve_interior(const DevTables<CT> &T, CT (&d)[NV][LT], int lane) {
    if constexpr (LT >= 2) {
        constexpr InteriorChunk<LT> K = interior_chunk<LT>();
        ChunkFactors<LT, CT> U{};
#pragma unroll
        for (int t = 0; t < LT; ++t) {
            U.f1[t] = (CT)K.fwd1[t];
            U.f2[t] = (CT)K.fwd2[t];
            U.b1[t] = (CT)K.bwd1[t];
            U.b2[t] = (CT)K.bwd2[t];
            U.nra[t] = (CT)(-K.rca[t]);
            U.nrc[t] = (CT)(-K.rcc[t]);
        }
        warp_solve_cf<LT, NV, CT, W>(U, T, d, lane);
    }
}

// Right-hand side of the compact derivative in FP32 for a line with
// ChunkFactors (p = n / LT full chunks, interface closure on both ends):
// interior rows aa (f[j+1] - f[j-1]) + bb (f[j+2] - f[j-2]), differences
// first; rows 0, 1 (lane 0) and n-1, n-2 (lane p-1) are the closure rows
// `own2` formed in FP64 by group_closure_rows / take_closure_rows.  Lanes
// >= p hold no rows.  `f` is the line in LineLayout<LT> order.
template <int LT>
__device__ __forceinline__ void deriv_rhs_cf(const float *f, int p, int lane, const double (&own2)[2],
                                             float (&d)[LT]) {
    using L = LineLayout<LT>;
    float w[LT + 4];
#pragma unroll
    for (int k = 0; k < LT + 4; ++k) {
        const int t = (k + LT - 2) % LT;
        const int dc = k < 2 ? -1 : (k >= LT + 2 ? 1 : 0);
        w[k] = f[L::pos_ct(lane + dc, t)];
    }
    constexpr float aa = (float)kAa, bb = (float)kBb;
#pragma unroll
    for (int t = 0; t < LT; ++t) d[t] = fmaf(bb, w[t + 4] - w[t], aa * (w[t + 3] - w[t + 1]));
    if (lane == 0) {
        d[0] = (float)own2[0];
        d[1] = (float)own2[1];
    }
    if (lane == p - 1) {
        d[LT - 1] = (float)(-own2[0]);
        d[LT - 2] = (float)(-own2[1]);
    }
    if (lane >= p) {
#pragma unroll
        for (int t = 0; t < LT; ++t) d[t] = 0.0f;
    }
}

// Select d[t] for a runtime t without dynamic register indexing.
template <int LT, typename CT>
__device__ __forceinline__ void set_at(CT (&d)[LT], int t, CT val) {
#pragma unroll
    for (int k = 0; k < LT; ++k)
        if (k == t) d[k] = val;
}
template <int LT, typename CT>
__device__ __forceinline__ CT get_at(const CT (&d)[LT], int t) {
    CT r = CT(0);
#pragma unroll
    for (int k = 0; k < LT; ++k)
        if (k == t) r = d[k];
    return r;
}

// One of the eight interface-closure sums of a line held in LineLayout<LT>
// order in shared memory (single-rank periodic closure), summed in index
// order k = 0..7 like the serial evaluation in deriv_rhs:
//   d = 0 / 1: sum_k pbci[k] f[k] / pbci[8+k] f[k]           (rows 0 / 1, own end)
//   d = 2 / 3: sum_k pbco[k] f[n-1-k] / pbco[8+k] f[n-1-k]   (rows 0 / 1, far end)
//   d = 4 / 5: sum_k pbci[k] f[n-1-k] / pbci[8+k] f[n-1-k]   (rows n-1 / n-2, own end)
//   d = 6 / 7: sum_k pbco[k] f[k] / pbco[8+k] f[k]           (rows n-1 / n-2, far end)
template <int LT, typename CT, typename FT>
__device__ __forceinline__ CT interface_sum(const FT *f, int n, int d, const Coeffs &cf) {
    using L = LineLayout<LT>;
    const bool bci = d < 2 || d == 4 || d == 5;
    const bool asc = d < 2 || d >= 6;
    const bool second = (d & 1) != 0;
    CT s = CT(0);
#pragma unroll
    for (int k = 0; k < kLmd; ++k) {
        const double c = bci ? (second ? cf.pbci[kLmd + k] : cf.pbci[k]) : (second ? cf.pbco[kLmd + k] : cf.pbco[k]);
        s += xmul(CT(c), CT(f[L::pos(asc ? k : n - 1 - k)]));
    }
    return s;
}

// The closure rows of the single-rank periodic closure for a group of up to
// four lines (lines[g], g < ng) solved together by one warp: lane 8g + d forms
// interface_sum d of line g, so all 8 ng sums are formed at once instead of
// one after another on the two owner lanes, then lanes 8g + {0, 1, 4, 5} add
// the own-end and far-end sums of rows 0, 1, n-1, n-2 (the operations of the
// serial evaluation, so the rows are bit-identical to it).  All 32 lanes must
// call it.
template <int LT, typename CT, typename FT, int G>
__device__ __forceinline__ CT group_closure_rows(FT *const (&lines)[G], int ng, int n, int lane, const Coeffs &cf) {
    static_assert(G <= 4, "eight lanes per line");
    const int g = lane >> 3;
    const FT *f = lines[0];
#pragma unroll
    for (int k = 1; k < G; ++k)
        if (g == k) f = lines[k];
    const CT dv = g < ng && g < G ? interface_sum<LT, CT, FT>(f, n, lane & 7, cf) : CT(0);
    return dv + __shfl_down_sync(0xffffffffu, dv, 2);
}
// Rows of line g from group_closure_rows: lane 0 takes rows 0 and 1, every
// other lane rows n-1 and n-2 (the owners of those rows are never lane 0 for
// lines of 8 or more points).  All 32 lanes must call it.
template <typename CT>
__device__ __forceinline__ void take_closure_rows(CT x, int g, int lane, CT (&own2)[2]) {
    const int src = 8 * g + (lane == 0 ? 0 : 4);
    own2[0] = __shfl_sync(0xffffffffu, x, src);
    own2[1] = __shfl_sync(0xffffffffu, x, src + 1);
}

// Right-hand side of the compact derivative for the rows of this lane,
// restating build_system (src/cuda/kernels/numerics_device_pc.hpp:176-293):
// interior aa*(f[j+1]-f[j-1]) + bb*(f[j+2]-f[j-2]); physical closure rows
// (ndf = 0) or interface closure rows (ndf = 1: 8-point pbci sums plus the
// received pbco sums; `recv4` = {row0, row1, row n-1, row n-2} received
// values, or the line's own far-end sums for single-rank periodic; `own2`,
// when given for that case, holds the line's closure rows already summed by
// group_closure_rows / take_closure_rows).
// `f` is the line in LineLayout<LT> order in shared memory.
template <int LT, typename CT, typename FT>
__device__ __forceinline__ void deriv_rhs(const FT *f, int n, int lane, int nstart, int nend,
                                          const CT *recv4_or_null, const Coeffs &cf,
                                          CT (&d)[LT], const CT *own2 = nullptr) {
    using L = LineLayout<LT>;
    const int j0 = lane * LT;
    // points j0-2 .. j0+LT+1: the last two of the previous lane's chunk, this
    // lane's chunk and the first two of the next lane's (compile-time slots,
    // no clamping).  Outside 0..n-1 the slot positions wrap inside the line's
    // slot and hold unused values: only rows 0, 1, n-2, n-1 reach there, and
    // the owner lanes rebuild those rows below.
    CT w[LT + 4];
#pragma unroll
    for (int k = 0; k < LT + 4; ++k) {
        const int t = (k + LT - 2) % LT;
        const int dc = k < 2 ? -1 : (k >= LT + 2 ? 1 : 0);
        w[k] = CT(f[L::pos_ct(lane + dc, t)]);
    }
#pragma unroll
    for (int t = 0; t < LT; ++t)
        d[t] = (j0 + t < n) ? xmul(CT(kAa), w[t + 3] - w[t + 1]) + xmul(CT(kBb), w[t + 4] - w[t]) : CT(0);

    const bool own_lo = lane == 0;
    const int own_hi1 = (n - 1) / LT, own_hi2 = (n - 2) / LT;
    if (own_lo || lane == own_hi1 || lane == own_hi2) {
        // the few boundary rows are rebuilt from scratch by their owner lanes
        if (own_lo) {
            const CT f0 = CT(f[L::pos(0)]), f1 = CT(f[L::pos(1)]), f2 = CT(f[L::pos(2)]);
            if (nstart == 0) {
                d[0] = xmul(CT(kAb00), f0) + xmul(CT(kAb01), f1) + xmul(CT(kAb02), f2);
                d[1] = xmul(CT(kAb10), f2 - f0);
            } else if (own2 && !recv4_or_null) {
                d[0] = own2[0];
                d[1] = own2[1];
            } else {
                CT r0, r1;
                if (recv4_or_null) {
                    r0 = recv4_or_null[0];
                    r1 = recv4_or_null[1];
                } else {
                    r0 = CT(0);
                    r1 = CT(0);
#pragma unroll
                    for (int k = 0; k < kLmd; ++k) r0 += xmul(CT(cf.pbco[k]), CT(f[L::pos(n - 1 - k)]));
#pragma unroll
                    for (int k = 0; k < kLmd; ++k) r1 += xmul(CT(cf.pbco[kLmd + k]), CT(f[L::pos(n - 1 - k)]));
                }
                CT s0 = CT(0), s1 = CT(0);
#pragma unroll
                for (int k = 0; k < kLmd; ++k) s0 += xmul(CT(cf.pbci[k]), CT(f[L::pos(k)]));
#pragma unroll
                for (int k = 0; k < kLmd; ++k) s1 += xmul(CT(cf.pbci[kLmd + k]), CT(f[L::pos(k)]));
                d[0] = s0 + r0;
                d[1] = s1 + r1;
            }
        }
        if (lane == own_hi1 || lane == own_hi2) {
            const CT g0 = CT(f[L::pos(n - 1)]), g1 = CT(f[L::pos(n - 2)]), g2 = CT(f[L::pos(n - 3)]);
            CT e1, e2;  // rows n-1 and n-2
            if (nend == 0) {
                e1 = -(xmul(CT(kAb00), g0) + xmul(CT(kAb01), g1) + xmul(CT(kAb02), g2));
                e2 = xmul(-CT(kAb10), g2 - g0);
            } else if (own2 && !recv4_or_null) {
                e1 = -own2[0];
                e2 = -own2[1];
            } else {
                CT r2, r3;
                if (recv4_or_null) {
                    r2 = recv4_or_null[2];
                    r3 = recv4_or_null[3];
                } else {
                    r2 = CT(0);
                    r3 = CT(0);
#pragma unroll
                    for (int k = 0; k < kLmd; ++k) r2 += xmul(CT(cf.pbco[k]), CT(f[L::pos(k)]));
#pragma unroll
                    for (int k = 0; k < kLmd; ++k) r3 += xmul(CT(cf.pbco[kLmd + k]), CT(f[L::pos(k)]));
                }
                CT s0 = CT(0), s1 = CT(0);
#pragma unroll
                for (int k = 0; k < kLmd; ++k) s0 += xmul(CT(cf.pbci[k]), CT(f[L::pos(n - 1 - k)]));
                s0 += r2;
#pragma unroll
                for (int k = 0; k < kLmd; ++k) s1 += xmul(CT(cf.pbci[kLmd + k]), CT(f[L::pos(n - 1 - k)]));
                s1 += r3;
                e1 = -s0;
                e2 = -s1;
            }
            if (lane == own_hi1) set_at<LT, CT>(d, (n - 1) - lane * LT, e1);
            if (lane == own_hi2) set_at<LT, CT>(d, (n - 2) - lane * LT, e2);
        }
    }
}

// Right-hand side of the sixth-order tridiagonal filter (Gaitonde & Visbal):
//   sum_m a_m/2 (f[j+m] + f[j-m]); near non-periodic ends the boundary point
// is copied and points 1 / 2 use the second / fourth order centred formulas.
// cyclic: indices wrap.
template <int LT, typename CT, typename FT>
__device__ __forceinline__ void filter_rhs(const FT *f, int n, int lane, bool cyclic, CT af,
                                           CT (&d)[LT]) {
    using L = LineLayout<LT>;
    const CT a60 = (CT(11) + xmul(CT(10), af)) / CT(16), a61 = (CT(15) + xmul(CT(34), af)) / CT(32);
    const CT a62 = (CT(-3) + xmul(CT(6), af)) / CT(16), a63 = (CT(1) - xmul(CT(2), af)) / CT(32);
    const CT a40 = (CT(5) + xmul(CT(6), af)) / CT(8), a41 = (CT(1) + xmul(CT(2), af)) / CT(2);
    const CT a42 = (CT(-1) + xmul(CT(2), af)) / CT(8);
    const CT a20 = (CT(1) + xmul(CT(2), af)) / CT(2);
    const CT h61 = xmul(CT(0.5), a61), h62 = xmul(CT(0.5), a62), h63 = xmul(CT(0.5), a63);
    const CT h41 = xmul(CT(0.5), a41), h42 = xmul(CT(0.5), a42), h21 = xmul(CT(0.5), a20);
    const int j0 = lane * LT;
    CT w[LT + 6];
#pragma unroll
    for (int k = 0; k < LT + 6; ++k) {
        int j = j0 + k - 3;
        if (cyclic) j = j < 0 ? j + n : (j >= n ? j - n : j);
        else j = j < 0 ? 0 : (j > n - 1 ? n - 1 : j);
        w[k] = CT(f[L::pos(j)]);
    }
#pragma unroll
    for (int t = 0; t < LT; ++t) {
        const int j = j0 + t;
        const CT c0 = w[t + 3];
        const CT s1 = w[t + 4] + w[t + 2], s2 = w[t + 5] + w[t + 1], s3 = w[t + 6] + w[t];
        CT r = xmul(a60, c0) + xmul(h61, s1) + xmul(h62, s2) + xmul(h63, s3);
        if (!cyclic) {
            const int dist = j < n - 1 - j ? j : n - 1 - j;
            if (dist == 0) r = c0;
            else if (dist == 1) r = xmul(a20, c0) + xmul(h21, s1);
            else if (dist == 2) r = xmul(a40, c0) + xmul(h41, s1) + xmul(h42, s2);
        }
        d[t] = j < n ? r : CT(0);
    }
}

}  // namespace csb
