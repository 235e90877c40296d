// tma_grad_mx.cuh -- gradient pass of the mixed-precision form with its
// pencils staged into shared memory by TMA.
//
// The mixed form's gradient passes (all but the first of a step, which forms
// the FP32 shadow from the FP64 state) read the four FP32 shadow fields
// (u, v, w, T - T0) and write their four FP32 derivatives along AXIS: 32 bytes
// per point, so the pass is bound by how many of its loads are in flight.
// Persistent CTAs of 256 threads (two per SM) walk the tiles
// t_k = blockIdx.x + k * gridDim.x; one thread issues a tile as tensor copies
// (cp.async.bulk.tensor, no multicast) of the four fields into one of two
// staging buffers, two tiles ahead of the tile being solved, completing on
// that buffer's mbarrier.  A tile is TL = 8 lines (4 for lines of 257-512
// points).  Per tile:
//   1. wait for the staging buffer (bounded);
//   2. every thread copies its points of the staged fields into the
//      line-solver layout (the y and z pencils arrive as rows of TL
//      consecutive x positions, so the transposition into lines happens here);
//   3. one thread refills the staging buffer with tile k + 2;
//   4. each warp solves its fields of one line in place: the FP32 interior
//      form with per-row constants (solve_lines_cf) where the line has
//      ChunkFactors, else the table form (solve_lines_mx); either with the
//      refinement sweep when it is on;
//   5. the four derivatives go to HBM with coalesced stores.
// The arithmetic is that of k_grad_mx with the same solve: results are
// bit-identical to it.  Boxes that reach past the end of the array read zeros
// (TMA out-of-bounds fill); those lines are never stored.
#pragma once

#include "tma_grad.cuh"

namespace csb {

constexpr int kErrTmaMxTimeout = 0x7102;

// fields per warp solve of the ChunkFactors form without the sweep (all four
// fields of a line in one solve: 256^3 gradient y / z passes 0.195 / 0.202 ->
// 0.164 / 0.160 ms against two solves of two fields)
#ifndef CSB_TMA_MX_GROUP
#define CSB_TMA_MX_GROUP 4
#endif

template <int LT>
constexpr int tma_mx_tile() {
    return LT <= 8 ? 8 : 4;
}

// MODE: 0 table solve, 1 table solve with the refinement sweep, 2 ChunkFactors,
// 3 ChunkFactors with the refinement sweep.
template <int LT, int AXIS, int MODE>
__global__ void __launch_bounds__(256, 2)
k_grad_mx_tma(const __grid_constant__ CUtensorMap smap, float *__restrict__ g, DevTables<float> tab, TmaGeom geo,
              int lxi, int let, int64_t lmx, int64_t F, int nstart, int nend, Coeffs cf, ChunkFactors<LT> U,
              int *__restrict__ err) {
    constexpr int TL = tma_mx_tile<LT>();
    constexpr int NT = 256;
    constexpr int FPW = 4 * TL / (NT / 32);  // fields per warp: 4 (TL 8) or 2 (TL 4)
    constexpr int G = (MODE == 1 || MODE == 3) && LT >= 16 ? 1 : (MODE == 2 && FPW % CSB_TMA_MX_GROUP == 0 ? CSB_TMA_MX_GROUP : 2);
    using L = LineLayout<LT>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int stage_elems = geo.nbox * 4 * TL * geo.boxlen;
    // staging boxes start on 128-byte boundaries (the launch adds the slack)
    float *stage0 = reinterpret_cast<float *>(smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u));
    float *solve = stage0 + 2 * stage_elems;
    uint64_t *bars = reinterpret_cast<uint64_t *>(
        reinterpret_cast<uintptr_t>(solve + 4 * TL * L::kSlot + 1) & ~uintptr_t(7));
    const int n = tab.n;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    const int Gd = gridDim.x;
    const int K = geo.ntiles > (int)blockIdx.x ? (geo.ntiles - 1 - (int)blockIdx.x) / Gd + 1 : 0;
    if (tid == 0)
        for (int k = 0; k < 2 && k < K; ++k) {
            const int t = blockIdx.x + k * Gd;
            float *dst = stage0 + k * stage_elems;
            mbar_arrive_expect_tx(&bars[k], geo.tile_bytes);
            for (int b = 0; b < geo.nbox; ++b) {
                float *d = dst + b * 4 * TL * geo.boxlen;
                if (AXIS == 0) tma_load_3d(d, &smap, b * geo.boxlen, t * TL, 0, &bars[k]);
                else if (AXIS == 1) tma_load_4d(d, &smap, (t % geo.tiles_x) * TL, b * geo.boxlen, t / geo.tiles_x, 0, &bars[k]);
                else tma_load_3d(d, &smap, t * TL, b * geo.boxlen, 0, &bars[k]);
            }
        }
    // this thread's line of the tile (fixed per thread) and its first point
    const int ml = AXIS == 0 ? w % TL : tid % TL;
    const int mj0 = AXIS == 0 ? (w / TL) * 32 + lane : tid / TL;
    constexpr int MDJ = AXIS == 0 ? 32 * (NT / 32 / TL) : NT / TL;
    const int fstride = TL * geo.boxlen;  // between staged fields
    const int box_elems = 4 * TL * geo.boxlen;
    for (int k = 0; k < K; ++k) {
        const int t = blockIdx.x + k * Gd, b = k & 1;
        float *stg = stage0 + b * stage_elems;
        const bool ok = mbar_wait_bounded(&bars[b], (unsigned)(k >> 1) & 1u);
        if (__syncthreads_or(!ok)) {
            // a copy never completed: record it, let the other buffer's copy
            // (if any) land within the same limit, and leave
            if (tid == 0) {
                atomicExch(err, kErrTmaMxTimeout);
                if (k + 1 < K) (void)mbar_wait_bounded(&bars[b ^ 1], (unsigned)((k + 1) >> 1) & 1u);
            }
            return;
        }
        int64_t mbase, mstride;
        const bool mvalid = tma_line<AXIS, TL>(t, ml, geo, lxi, let, F, mbase, mstride);
        if (mvalid) {
            for (int j = mj0; j < n; j += MDJ) {
                const int bx = j >= geo.boxlen ? 1 : 0, jj = j - bx * geo.boxlen;
                const int o = bx * box_elems + (AXIS == 0 ? ml * geo.boxlen + jj : jj * TL + ml);
                const int pj = L::pos(j);
#pragma unroll
                for (int c = 0; c < 4; ++c) field_line32<LT, TL>(solve, c, ml)[pj] = stg[o + c * fstride];
            }
        }
        __syncthreads();
        if (tid == 0 && k + 2 < K) {
            const int tn = t + 2 * Gd;
            mbar_arrive_expect_tx(&bars[b], geo.tile_bytes);
            for (int bb = 0; bb < geo.nbox; ++bb) {
                float *d = stg + bb * box_elems;
                if (AXIS == 0) tma_load_3d(d, &smap, bb * geo.boxlen, tn * TL, 0, &bars[b]);
                else if (AXIS == 1)
                    tma_load_4d(d, &smap, (tn % geo.tiles_x) * TL, bb * geo.boxlen, tn / geo.tiles_x, 0, &bars[b]);
                else tma_load_3d(d, &smap, tn * TL, bb * geo.boxlen, 0, &bars[b]);
            }
        }
        {
            int64_t base, stride;
            const int l = w % TL, c0 = (w / TL) * FPW;
            if (tma_line<AXIS, TL>(t, l, geo, lxi, let, F, base, stride)) {
#pragma unroll 1
                for (int c = c0; c < c0 + FPW; c += G) {
                    float *lines[G];
#pragma unroll
                    for (int gg = 0; gg < G; ++gg) lines[gg] = field_line32<LT, TL>(solve, c + gg, l);
                    if (MODE >= 2) solve_lines_cf<LT, G, MODE == 3>(lines, G, lane, tab, U, cf);
                    else solve_lines_mx<LT, G, MODE == 1>(lines, G, lane, tab, nstart, nend, cf, MODE == 1 ? 1 : 0);
                }
            }
        }
        __syncthreads();
        if (mvalid) {
            for (int j = mj0; j < n; j += MDJ) {
                const int64_t gi = mbase + j * mstride;
                const int pj = L::pos(j);
#pragma unroll
                for (int c = 0; c < 4; ++c) g[c * lmx + gi] = field_line32<LT, TL>(solve, c, ml)[pj];
            }
        }
        __syncthreads();
    }
}


template <int LT, int AXIS>
int launch_grad_mx_tma_t(const MixedArgs &a, const cs_dcomp &d, int *err, cudaStream_t st) {
    const PassArgs &b = a.base;
    TmaGeom geo;
    size_t smem = 0;
    if (!tma_grad_mx_geometry(AXIS, d, LT, 1 << 30, geo, smem))
        return set_error(CS_ERR_UNSUPPORTED, "mixed TMA gradient pass: unsupported geometry");
    CUtensorMap map;
    if (int rc = tma_field_map32(AXIS, d, tma_mx_tile<LT>(), geo.boxlen, 4, a.shadow + b.lmx, map)) return rc;
    auto kern = use_cf(a) ? (a.refine ? k_grad_mx_tma<LT, AXIS, 3> : k_grad_mx_tma<LT, AXIS, 2>)
                          : (a.refine ? k_grad_mx_tma<LT, AXIS, 1> : k_grad_mx_tma<LT, AXIS, 0>);
    if (int rc = set_smem(kern, smem)) return rc;
    int per = 0;
    CSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 256, smem));
    if (per < 1) return set_error(CS_ERR_UNSUPPORTED, "mixed TMA gradient pass: a CTA does not fit an SM");
    const int blocks = geo.ntiles < b.nsm * per ? geo.ntiles : b.nsm * per;
    kern<<<blocks, 256, smem, st>>>(map, a.grad + (int64_t)AXIS * 4 * b.lmx, b.tab->t32, geo, b.lxi, b.let, b.lmx,
                                    b.F, b.nstart, b.nend, b.cf, chunk_factors_of<LT>(*b.tab), err);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

template <int AXIS>
int launch_grad_mx_tma_impl(const MixedArgs &a, const cs_dcomp &d, int *err, cudaStream_t st) {
    switch (a.base.tab->lt) {
        case 2: return launch_grad_mx_tma_t<2, AXIS>(a, d, err, st);
        case 4: return launch_grad_mx_tma_t<4, AXIS>(a, d, err, st);
        case 8: return launch_grad_mx_tma_t<8, AXIS>(a, d, err, st);
        case 16: return launch_grad_mx_tma_t<16, AXIS>(a, d, err, st);
    }
    return set_error(CS_ERR_UNSUPPORTED, "chunk length");
}

}  // namespace csb
