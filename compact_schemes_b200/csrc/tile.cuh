// tile.cuh -- mapping of a CTA's threads onto a tile of lines.
//
// A tile is kTileLines lines along AXIS.  For x (AXIS 0) lines are contiguous
// in memory and warp w owns line w of the tile (256-byte coalesced rows, no
// cross-warp synchronization).  For y and z, the tile's lines are 8
// consecutive x (or x-y) positions, so a row of the tile is 8 consecutive
// doubles; thread t covers line t % 8 and rows t / 8 + 32 k.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace csb {

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

// Calls fn(l, j, gidx) for every point (line l of the tile, position j) this
// thread owns; gidx is the point's linear index.
template <int AXIS, int UNROLL = 1, typename Fn>
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
        const int l = tid % kTileLines;
        const int64_t fidx = line0 + l;
        if (fidx < F) {
            const int64_t base = line_base<AXIS>(fidx, lxi, let), s = line_stride<AXIS>(lxi, let);
#pragma unroll UNROLL
            for (int j = tid / kTileLines; j < n; j += kThreads / kTileLines) fn(l, j, base + j * s);
        }
    }
}

template <int AXIS>
__device__ __forceinline__ void tile_sync() {
    if (AXIS == 0) __syncwarp();
    else __syncthreads();
}

}  // namespace csb
