// tile.cuh -- mapping of a CTA's threads onto a tile of lines.
//
// A tile is TL lines along AXIS (TL * 32 threads).  For x (AXIS 0) lines are contiguous
// in memory and warp w owns line w of the tile (256-byte coalesced rows, no
// cross-warp synchronization).  For y and z, the tile's lines are TL
// consecutive x (or x-y) positions, so a row of the tile is TL consecutive
// doubles; thread t covers line t % TL and rows t / TL + 32 k.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace csb {

// Default tile of the single-field kernels (numerics.cu); the fused passes
// take the tile width TL as a template parameter (TL * 32 threads).
constexpr int kTileLines = 8;
constexpr int kThreads = 256;

// First point of line `fidx` (face index convention of the reference,
// src/cuda/kernels/transforms.hpp: axis 0 k*let+j, axis 1 k*lxi+i, axis 2 j*lxi+i).
template <int AXIS>
__device__ __forceinline__ int64_t line_base(int64_t fidx, int lxi, int let) {
    if (AXIS == 0) return fidx * lxi;
    if (AXIS == 1) return (fidx / lxi) * (int64_t)lxi * let + fidx % lxi;
    return fidx;
}

template <int AXIS>
__device__ __forceinline__ int64_t line_stride(int lxi, int let) {
    return AXIS == 0 ? 1 : (AXIS == 1 ? (int64_t)lxi : (int64_t)lxi * let);
}

// Row order of the y/z tiles: 0 = the CTA's threads cover 32 consecutive
// rows at a time; 1 = each group of TL threads walks its own block of rows,
// so one CTA's concurrent accesses span the whole line; 2 = as 1, with the
// starting row rotated per CTA so that CTAs sharing a plane do not read the
// same rows at the same time.
#ifndef CSB_ROW_ORDER
#define CSB_ROW_ORDER 0
#endif

// Calls fn(l, j, gidx) for every point (line l of the tile, position j) this
// thread owns; gidx is the point's linear index.
template <int AXIS, int TL, int UNROLL = 1, typename Fn>
__device__ __forceinline__ void tile_for_each(int64_t line0, int64_t F, int n, int lxi, int let, Fn &&fn) {
    const int tid = threadIdx.x;
    if (AXIS == 0) {
        const int w = tid >> 5, lane = tid & 31;
        const int64_t fidx = line0 + w;
        if (fidx < F) {
            const int64_t base = fidx * n;
#pragma unroll UNROLL
            for (int j = lane; j < n; j += 32) fn(w, j, base + j);
        }
    } else {
        const int l = tid % TL;
        const int64_t fidx = line0 + l;
        if (fidx < F) {
            const int64_t base = line_base<AXIS>(fidx, lxi, let), s = line_stride<AXIS>(lxi, let);
            if (CSB_ROW_ORDER == 0) {
#pragma unroll UNROLL
                for (int j = tid / TL; j < n; j += 32) fn(l, j, base + j * s);
            } else {
                const int rows = (n + 31) / 32, g = tid / TL;
                const int rot = CSB_ROW_ORDER == 2 ? (int)((blockIdx.x * 7u) % (unsigned)rows) : 0;
#pragma unroll UNROLL
                for (int t = 0; t < rows; ++t) {
                    int tt = t + rot;
                    tt = tt >= rows ? tt - rows : tt;
                    const int j = g * rows + tt;
                    if (j < n) fn(l, j, base + j * s);
                }
            }
        }
    }
}

// Same traversal in chunks of P points per thread: load(p, l, j, gidx) runs
// for all points of a chunk before store(p, l, j, gidx) runs for any, so the
// global loads of a read-modify-write are all in flight together even when
// they go through the pointer that is stored to.
template <int AXIS, int TL, int P, typename FnLoad, typename FnStore>
__device__ __forceinline__ void tile_for_each_chunked(int64_t line0, int64_t F, int n, int lxi, int let,
                                                      FnLoad &&load, FnStore &&store) {
    const int tid = threadIdx.x;
    int l, j0, dj;
    int64_t base, s;
    if (AXIS == 0) {
        l = tid >> 5;
        j0 = tid & 31;
        dj = 32;
        base = (line0 + l) * n;
        s = 1;
    } else {
        l = tid % TL;
        j0 = tid / TL;
        dj = 32;
        base = line_base<AXIS>(line0 + l, lxi, let);
        s = line_stride<AXIS>(lxi, let);
    }
    if (line0 + l >= F) return;
    for (int jc = j0; jc < n; jc += P * dj) {
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const int j = jc + p * dj;
            if (j < n) load(p, l, j, base + j * s);
        }
#pragma unroll
        for (int p = 0; p < P; ++p) {
            const int j = jc + p * dj;
            if (j < n) store(p, l, j, base + j * s);
        }
    }
}

template <int AXIS, int TL = kTileLines>
__device__ __forceinline__ void tile_sync() {
    if (AXIS == 0) __syncwarp();
    else __syncthreads();
}

}  // namespace csb

namespace csb {

// Role-relative traversal for the two-role (pipelined) passes: NT threads of one
// role (rtid = 0..NT-1) cover a tile of TL lines.  x: TPL = max(32, NT / TL)
// consecutive threads per line (warp w handles lines w, w + NT/32, ... when
// TPL is 32); y/z: thread t covers line t % TL, rows t / TL + (NT / TL) k.
template <int AXIS, int TL, int NT, int UNROLL = 1, typename Fn>
__device__ __forceinline__ void tile_for_each_r(int rtid, int64_t line0, int64_t F, int n, int lxi, int let,
                                                Fn &&fn) {
    if (AXIS == 0) {
        constexpr int TPL = NT / TL >= 32 ? NT / TL : 32;
        for (int l = rtid / TPL; l < TL; l += NT / TPL) {
            const int64_t fidx = line0 + l;
            if (fidx >= F) break;
            const int64_t base = fidx * n;
#pragma unroll UNROLL
            for (int j = rtid % TPL; j < n; j += TPL) fn(l, j, base + j);
        }
    } else {
        const int l = rtid % TL;
        const int64_t fidx = line0 + l;
        if (fidx < F) {
            const int64_t base = line_base<AXIS>(fidx, lxi, let), s = line_stride<AXIS>(lxi, let);
#pragma unroll UNROLL
            for (int j = rtid / TL; j < n; j += NT / TL) fn(l, j, base + j * s);
        }
    }
}

// Chunked read-modify-write form of tile_for_each_r (see tile_for_each_chunked).
template <int AXIS, int TL, int NT, int P, typename FnLoad, typename FnStore>
__device__ __forceinline__ void tile_for_each_r_chunked(int rtid, int64_t line0, int64_t F, int n, int lxi,
                                                        int let, FnLoad &&load, FnStore &&store) {
    constexpr int TPL = AXIS == 0 ? (NT / TL >= 32 ? NT / TL : 32) : NT / TL;
    const int lfirst = AXIS == 0 ? rtid / TPL : rtid % TL;
    const int lstep = AXIS == 0 ? NT / TPL : TL;
    const int j0 = AXIS == 0 ? rtid % TPL : rtid / TL;
    const int64_t s = line_stride<AXIS>(lxi, let);
    for (int l = lfirst; l < TL; l += lstep) {
        const int64_t fidx = line0 + l;
        if (fidx >= F) break;
        const int64_t base = line_base<AXIS>(fidx, lxi, let);
        for (int jc = j0; jc < n; jc += P * TPL) {
#pragma unroll
            for (int p = 0; p < P; ++p) {
                const int j = jc + p * TPL;
                if (j < n) load(p, l, j, base + j * s);
            }
#pragma unroll
            for (int p = 0; p < P; ++p) {
                const int j = jc + p * TPL;
                if (j < n) store(p, l, j, base + j * s);
            }
        }
    }
}

// Named CTA barriers for the two-role (pipelined) passes (barrier 0 is
// __syncthreads).  bar.sync waits until `count` threads have arrived;
// bar.arrive counts the caller without waiting.
__device__ __forceinline__ void named_bar_sync(int id, int count) {
    __syncwarp();
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}
__device__ __forceinline__ void named_bar_arrive(int id, int count) {
    __syncwarp();
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(count) : "memory");
}
constexpr int kBarFull0 = 1;  // + buffer: tile staged, ready to solve

}  // namespace csb
