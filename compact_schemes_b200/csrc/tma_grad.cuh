// tma_grad.cuh -- gradient pass with pencils staged into shared memory by TMA.
//
// Persistent CTAs walk the tiles t_k = blockIdx.x + k * gridDim.x of a
// gradient pass: two 256-thread CTAs per SM for lines of up to 256 points,
// one 512-thread CTA for lines of 257-512 points.  A tile is TL = 4 lines of
// the state q along AXIS; one thread issues it as tensor copies
// (cp.async.bulk.tensor, no multicast) of all five conserved fields into one
// of two staging buffers, completing on that buffer's mbarrier, two tiles
// ahead of the tile being solved.  The y and z pencils are boxes of TL
// consecutive x (or x-y) positions by the whole line, so the strided lines
// arrive as dense rows; the x pencils are TL consecutive rows.  Per tile:
//   1. wait for the staging buffer (bounded);
//   2. every thread reads its points of the staged q, forms the primitives
//      (u, v, w, T) and writes them into the line-solver layout (the staged
//      rows are read along the tile's x, the transposition into lines happens
//      here), and reduces the CFL maxima when asked;
//   3. one thread refills the staging buffer with tile k + 2;
//   4. each warp solves two fields (one for 512-point lines) of one line in
//      place;
//   5. the four derivatives go to HBM with coalesced stores.
// The HBM reads of two tiles are in flight while a tile is formed, solved
// and stored, with no per-element address arithmetic on the load side, and
// with two CTAs per SM one CTA's solve overlaps the other's stores.  The
// arithmetic is that of k_grad (same primitives, same right-hand sides, same
// warp solves and field grouping): results are bit-identical to it.
//
// Lines of up to 256 points are one box; up to 512 points, two boxes along
// the line (a TMA box dimension holds at most 256 elements).  Boxes that
// reach past the end of the array read zeros (TMA out-of-bounds fill); those
// lines are never stored and their CFL terms are skipped.
#pragma once

#include <cuda.h>

#include "pipeline.cuh"

namespace csb {

// iterations of a bounded mbarrier wait (each try_wait suspends for a
// hardware-chosen time; with the backoff below the limit is well over 1 s)
constexpr unsigned kTmaWaitLimit = 1u << 22;
constexpr int kErrTmaTimeout = 0x7101;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase `parity` of a barrier; false when it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity) {
    for (unsigned it = 0; it < kTmaWaitLimit; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it > 8) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
        : "memory");
}

// Tiles of the TMA gradient pass: 4 lines.  Lines of up to 256 points run
// 256-thread CTAs, two per SM (each 113 KB of shared memory), so that one CTA
// solves while the other stages and stores; lines of 257-512 points run one
// 512-thread CTA per SM.
constexpr int kTmaTile = 4;
template <int LT>
constexpr int tma_threads() {
    return LT <= 8 ? 256 : 512;
}

// Issue the copies of tile t into the staging buffer dst (one thread).
template <int AXIS, int TL>
__device__ __forceinline__ void tma_issue_tile(double *dst, const CUtensorMap *map, int t, const TmaGeom &g,
                                               uint64_t *bar) {
    mbar_arrive_expect_tx(bar, g.tile_bytes);
    for (int b = 0; b < g.nbox; ++b) {
        double *d = dst + b * 5 * TL * g.boxlen;
        if (AXIS == 0) tma_load_3d(d, map, b * g.boxlen, t * TL, 0, bar);
        else if (AXIS == 1) tma_load_4d(d, map, (t % g.tiles_x) * TL, b * g.boxlen, t / g.tiles_x, 0, bar);
        else tma_load_3d(d, map, t * TL, b * g.boxlen, 0, bar);
    }
}

// Linear index of point j of tile line l, and whether the line exists.
template <int AXIS, int TL>
__device__ __forceinline__ bool tma_line(int t, int l, const TmaGeom &g, int lxi, int let, int64_t F,
                                         int64_t &base, int64_t &stride) {
    if (AXIS == 0) {
        const int64_t fidx = (int64_t)t * TL + l;
        base = fidx * lxi;
        stride = 1;
        return fidx < F;
    }
    if (AXIS == 1) {
        const int i = (t % g.tiles_x) * TL + l, k = t / g.tiles_x;
        base = i + (int64_t)lxi * let * k;
        stride = lxi;
        return i < lxi;
    }
    const int64_t fidx = (int64_t)t * TL + l;
    base = fidx;
    stride = (int64_t)lxi * let;
    return fidx < F;
}

template <int LT, int AXIS, bool DTRED>
__global__ void __launch_bounds__(tma_threads<LT>(), LT <= 8 ? 2 : 1)
k_grad_tma(const __grid_constant__ CUtensorMap qmap, double *__restrict__ g, DevTables<double> tab, TmaGeom geo,
           int lxi, int let, int64_t lmx, int64_t F, int nstart, int nend, Coeffs cf, Phys ph,
           unsigned long long *__restrict__ dtacc, int *__restrict__ err) {
    constexpr int TL = kTmaTile;
    constexpr int NT = tma_threads<LT>();
    constexpr int FPW = 4 * TL / (NT / 32);  // fields per warp solve
    using L = LineLayout<LT>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int stage_elems = geo.nbox * 5 * TL * geo.boxlen;
    // staging boxes start on 128-byte boundaries (the launch adds the slack)
    double *stage0 = reinterpret_cast<double *>(smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u));
    double *solve = stage0 + 2 * stage_elems;
    uint64_t *bars = reinterpret_cast<uint64_t *>(solve + 4 * TL * L::kSlot);
    const int n = tab.n;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    const int G = gridDim.x;
    const int K = geo.ntiles > (int)blockIdx.x ? (geo.ntiles - 1 - (int)blockIdx.x) / G + 1 : 0;
    if (tid == 0)
        for (int k = 0; k < 2 && k < K; ++k)
            tma_issue_tile<AXIS, TL>(stage0 + k * stage_elems, &qmap, blockIdx.x + k * G, geo, &bars[k]);
    double m1 = 0.0, m2 = 0.0;
    for (int k = 0; k < K; ++k) {
        const int t = blockIdx.x + k * G, b = k & 1;
        double *stg = stage0 + b * stage_elems;
        const bool ok = mbar_wait_bounded(&bars[b], (unsigned)(k >> 1) & 1u);
        if (__syncthreads_or(!ok)) {
            // a copy never completed: record it, let the other buffer's copy
            // (if any) land within the same limit, and leave
            if (tid == 0) {
                atomicExch(err, kErrTmaTimeout);
                if (k + 1 < K) (void)mbar_wait_bounded(&bars[b ^ 1], (unsigned)((k + 1) >> 1) & 1u);
            }
            return;
        }
        // this thread's line of the tile (fixed per thread) and where it lives
        // in HBM and in the staging buffer
        const int ml = AXIS == 0 ? w % TL : tid % TL;
        const int mj0 = AXIS == 0 ? (w / TL) * 32 + lane : tid / TL;
        constexpr int MDJ = AXIS == 0 ? 32 * (NT / 32 / TL) : NT / TL;
        int64_t mbase, mstride;
        const bool mvalid = tma_line<AXIS, TL>(t, ml, geo, lxi, let, F, mbase, mstride);
        const int fstride = AXIS == 0 ? TL * geo.boxlen : geo.boxlen * TL;  // between staged fields
        const int box_elems = 5 * TL * geo.boxlen;
        // primitives into the line layout
        if (mvalid) {
            for (int j = mj0; j < n; j += MDJ) {
                const int bx = j >= geo.boxlen ? 1 : 0, jj = j - bx * geo.boxlen;
                const int o = bx * box_elems + (AXIS == 0 ? ml * geo.boxlen + jj : jj * TL + ml);
                const Prim s = primitives(stg[o], stg[o + fstride], stg[o + 2 * fstride], stg[o + 3 * fstride],
                                          stg[o + 4 * fstride]);
                const int pj = L::pos(j);
                field_line<LT, TL>(solve, 0, ml)[pj] = s.u;
                field_line<LT, TL>(solve, 1, ml)[pj] = s.v;
                field_line<LT, TL>(solve, 2, ml)[pj] = s.w;
                field_line<LT, TL>(solve, 3, ml)[pj] = s.T;
                if (DTRED) {
                    // calc_time_step_kernel (src/cuda/kernels/physics.hpp:335-427), uniform metrics
                    const double uu = s.u + ph.umf[0], vv = s.v + ph.umf[1], ww = s.w + ph.umf[2];
                    double rr2 = 0.0;
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        rr2 += fabs(xmul(ph.M[a][0], uu) + xmul(ph.M[a][1], vv) + xmul(ph.M[a][2], ww));
                    const double ssi = fabs(ph.J);
                    const double v1 = xmul(sqrt(xmul(s.T, ph.rr1)) + rr2, ssi);
                    const double v2 = s.ri * ph.mu * ph.rr1 * ssi * ssi;
                    m1 = fmax(m1, v1);
                    m2 = fmax(m2, v2);
                }
            }
        }
        __syncthreads();
        if (tid == 0 && k + 2 < K) tma_issue_tile<AXIS, TL>(stg, &qmap, t + 2 * G, geo, &bars[b]);
        {
            int64_t base, stride;
            const int l = w % TL;
            if (tma_line<AXIS, TL>(t, l, geo, lxi, let, F, base, stride))
                solve_group<LT, TL, FPW, true>(solve, l, (w / TL) * FPW, 4, lane, tab, nstart, nend, cf);
        }
        __syncthreads();
        if (mvalid) {
            for (int j = mj0; j < n; j += MDJ) {
                const int64_t gi = mbase + j * mstride;
                const int pj = L::pos(j);
#pragma unroll
                for (int c = 0; c < 4; ++c) g[c * lmx + gi] = field_line<LT, TL>(solve, c, ml)[pj];
            }
        }
        __syncthreads();
    }
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

// Host side (tma_grad.cu).
// Encode the tensor map of q [5][lmx] for a gradient pass along `axis`.
int tma_grad_map(int axis, const cs_dcomp &d, const TmaGeom &g, const double *q, CUtensorMap &map);
// Tensor map over nf consecutive fields [nf][lmx] starting at base, boxes of
// tl lines by boxlen points along `axis` by nf fields.
// (tma_field_map / tma_field_map32: declared in fused_mixed.cuh)

template <int LT, int AXIS>
int launch_grad_tma_t(const PassArgs &a, const cs_dcomp &d, const double *q, bool dtred, int *err,
                      cudaStream_t st) {
    TmaGeom geo;
    size_t smem = 0;
    if (!tma_grad_geometry(AXIS, d, LT, 1 << 30, geo, smem))
        return set_error(CS_ERR_UNSUPPORTED, "TMA gradient pass: unsupported geometry");
    CUtensorMap map;
    if (int rc = tma_grad_map(AXIS, d, geo, q, map)) return rc;
    auto kern = dtred ? k_grad_tma<LT, AXIS, true> : k_grad_tma<LT, AXIS, false>;
    if (int rc = set_smem(kern, smem)) return rc;
    int per = 0;
    CSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, tma_threads<LT>(), smem));
    if (per < 1) return set_error(CS_ERR_UNSUPPORTED, "TMA gradient pass: a CTA does not fit an SM");
    const int blocks = geo.ntiles < a.nsm * per ? geo.ntiles : a.nsm * per;
    kern<<<blocks, tma_threads<LT>(), smem, st>>>(map, a.grad + (int64_t)AXIS * 4 * a.lmx, a.tab->t64, geo, a.lxi, a.let,
                                            a.lmx, a.F, a.nstart, a.nend, a.cf, a.ph, a.dtacc, err);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

template <int AXIS>
int launch_grad_tma_impl(const PassArgs &a, const cs_dcomp &d, const double *q, bool dtred, int *err, cudaStream_t st) {
    switch (a.tab->lt) {
        case 2: return launch_grad_tma_t<2, AXIS>(a, d, q, dtred, err, st);
        case 4: return launch_grad_tma_t<4, AXIS>(a, d, q, dtred, err, st);
        case 8: return launch_grad_tma_t<8, AXIS>(a, d, q, dtred, err, st);
        case 16: return launch_grad_tma_t<16, AXIS>(a, d, q, dtred, err, st);
    }
    return set_error(CS_ERR_UNSUPPORTED, "chunk length");
}

}  // namespace csb
