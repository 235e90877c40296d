// ensemble.cuh -- persistent work-queue kernel of the batched ensemble.
//
// Many independent boxes advance one RK stage in a single launch.  The work
// is a list of items, each one tile of TL lines of one pass of one box,
// grouped in segments (box, pass kind) and numbered in an order in which every
// item comes after the items it depends on:
//   phase 0  gradient passes x, y, z   (read the stage state)
//   phase 1  flux pass x               (needs all of phase 0 of the box)
//   phase 2  flux pass y               (needs all of phase 1: it accumulates R)
//   phase 3  flux pass z + RK update   (needs all of phase 2)
// A CTA takes the next item number from a device counter, waits until the
// box's previous phase has completed (a per-box counter of finished items),
// runs the tile with the same device functions as the per-box passes
// (grad_tile / flux_tile), and counts the item as finished.  Items are handed
// out in order, so an item only ever waits for items already taken by running
// CTAs: the queue cannot deadlock, whatever the grid size.  Each wait is
// bounded; when it runs out the kernel records the item in an error word and
// skips the item instead of hanging.
//
// Data that other CTAs produce within the launch (gradients, the RHS
// accumulator, the CFL maxima) is read through L2 (ld.global.cg), since an
// SM's L1 is not kept coherent with other SMs' stores.
#pragma once

#include "fused_kernels.cuh"

namespace csb {

constexpr int kEnsMaxLt = 8;        // lines of up to 256 points
constexpr int kEnsPhases = 4;
// bounded wait for a dependency: polls x sleep of about 2 s in all
constexpr long long kEnsWaitPolls = 20000000;

// Kinds of work items: 0-2 gradient pass along axis k, 3-5 flux pass along axis k - 3.
struct EnsBox {
    DevTables<double> tab[3];
    Phys ph;
    double cfl;
    int64_t lmx, F[3];
    int64_t qoff, goff, roff;  // element offsets of the box in the packed state / gradients / RHS
    int lxi, let, lze;
    int lt[3];
    int nstart[3], nend[3];
};

struct EnsSeg {
    int start;       // first item number
    int ntiles;      // tiles of the pass; item k of the segment covers tiles [k * chunk, (k + 1) * chunk)
    int box;         // index into the box array
    int kind;        // pass kind
    int wait_count;  // finished items of the previous phase this segment waits for (0: none)
    int phase;
};

constexpr int kEnsSmemStarts = 4096;  // segment starts searched in shared memory up to this many segments

struct EnsArgs {
    const EnsSeg *segs;
    int nseg;
    int nitems;
    const EnsBox *boxes;
    int *queue;      // next item number
    int *done;       // [nbox][kEnsPhases] finished items
    int *err;        // 0, or 1 + the item whose dependency wait ran out
    long long poll_limit;  // polls of a dependency wait before it gives up
    int wait_bias;   // finished items a wait needs beyond its count (0; > 0 only to test the timeout)
    double *q;       // packed state q^n (updated in place by the last stage)
    double *q1;      // packed intermediate stage state
    double *grad;    // packed gradients [12][lmx] per box
    double *rhs;     // packed RHS accumulator [5][lmx] per box
    unsigned long long *dtacc;  // [nbox][2] CFL maxima
    double *dt;      // [nbox] dt of the step
    Coeffs cf;
    const Coeffs *cf_dev;  // device copy of cf (source of the constant copy)
    int stage;       // 0..3
    int chunk;       // tiles per work item
    int tile_doubles;  // shared memory of the tile buffer (the segment starts follow it)
};

// The box descriptors of the launch live in constant memory (one copy per
// translation unit, refreshed from the ensemble's device table before every
// stage launch): the compiler may then reload a parameter instead of keeping
// it in a register, since constant memory cannot change during the launch.
constexpr int kEnsMaxBoxes = 96;
static __constant__ EnsBox c_ens_boxes[kEnsMaxBoxes];
static __constant__ Coeffs c_ens_cf;

// Points per read-modify-write chunk in the ensemble's flux items (fewer than
// the per-box passes: the items have fewer registers to spare; measured on
// the 64-box set, one point beats two or four).
#ifndef CSB_ENS_RMW
#define CSB_ENS_RMW 1
#endif
#ifndef CSB_ENS_RMW_RK
#define CSB_ENS_RMW_RK 1
#endif
constexpr int kEnsRmwChunk = CSB_ENS_RMW, kEnsRmwChunkRk = CSB_ENS_RMW_RK;

// Line solves of the work items: fields per warp solve for lines of up to 128
// points (LT <= 4), and whether the periodic closure rows are formed
// lane-parallel (8 lanes per field line) instead of by the two owner lanes.
// Short lines make the serial closure sums a large share of the solve, which
// runs on one lane while the other 31 wait.
#ifndef CSB_ENS_SG
#define CSB_ENS_SG 4
#endif
#ifndef CSB_ENS_ROWS
#define CSB_ENS_ROWS 1
#endif
template <int LT>
constexpr int ens_solve_group() {
    return LT <= 4 ? CSB_ENS_SG : 2;
}

// One work item of pass KIND for chunk length LT, inlined into the stage
// kernel (with the box parameters in constant memory the combined body spills
// little; separate functions measured slower by their call overhead).
template <int TL, bool VISC, int LT, int KIND>
__device__ __forceinline__ void ens_item(const EnsArgs &a, int b, int64_t line0, double *sm) {
    const EnsBox &bx = c_ens_boxes[b];
    const int stage = a.stage;
    const double *qin = (stage == 0 ? a.q : a.q1) + bx.qoff;
    double *g = a.grad + bx.goff;
    constexpr int AX = KIND % 3;
    const Phys &ph = bx.ph;
    const DevTables<double> &tab = bx.tab[AX];
    if (KIND < 3) {
        constexpr int SG = ens_solve_group<LT>();
        constexpr bool ROWS = CSB_ENS_ROWS != 0;
        if (KIND == 0 && stage == 0)
            grad_tile<LT, 0, TL, true, false, SG, ROWS>(sm, line0, qin, g, tab, bx.lxi, bx.let, bx.lmx, bx.F[0],
                                                        bx.nstart[0], bx.nend[0], c_ens_cf, ph, a.dtacc + 2 * b);
        else
            grad_tile<LT, AX, TL, false, false, SG, ROWS>(sm, line0, qin, g + 4 * AX * bx.lmx, tab, bx.lxi, bx.let,
                                                          bx.lmx, bx.F[AX], bx.nstart[AX], bx.nend[AX], c_ens_cf, ph,
                                                          nullptr);
        return;
    }
    double *rhs = a.rhs + bx.roff;
    RkParams rk{};
    if (KIND == 5) {
        rk.div = 4 - stage;
        rk.dt_fixed = 0.0;
        rk.cfl = bx.cfl;
        rk.dtacc = a.dtacc + 2 * b;
        rk.dt_out = stage == 0 ? a.dt + b : nullptr;
    }
    const double *qn = a.q + bx.qoff;
    double *qout = (stage == 3 ? a.q : a.q1) + bx.qoff;
    constexpr int MODE = KIND == 3 ? kWrite : (KIND == 4 ? kAccum : kAccumRk);
    constexpr int P = MODE == kAccum ? kEnsRmwChunk : kEnsRmwChunkRk;
    flux_tile<LT, AX, TL, MODE, VISC, true, P, false, ens_solve_group<LT>(), CSB_ENS_ROWS != 0>(
        sm, line0, qin, g, rhs, qn, qout, nullptr, tab, bx.lxi, bx.let, bx.lmx, bx.F[AX], bx.nstart[AX], bx.nend[AX],
        c_ens_cf, ph, rk);
}

template <int TL, bool VISC, int LT>
__device__ __forceinline__ void ens_run_lt(const EnsArgs &a, int b, int kind, int64_t line0, double *sm) {
    switch (kind) {
        case 0: ens_item<TL, VISC, LT, 0>(a, b, line0, sm); break;
        case 1: ens_item<TL, VISC, LT, 1>(a, b, line0, sm); break;
        case 2: ens_item<TL, VISC, LT, 2>(a, b, line0, sm); break;
        case 3: ens_item<TL, VISC, LT, 3>(a, b, line0, sm); break;
        case 4: ens_item<TL, VISC, LT, 4>(a, b, line0, sm); break;
        default: ens_item<TL, VISC, LT, 5>(a, b, line0, sm); break;
    }
}

template <int TL, bool VISC>
__device__ __forceinline__ void ens_run_item(const EnsArgs &a, int b, int kind, int64_t line0, double *sm) {
    const int lt = c_ens_boxes[b].lt[kind % 3];
    if (lt == 2) ens_run_lt<TL, VISC, 2>(a, b, kind, line0, sm);
    else if (lt == 4) ens_run_lt<TL, VISC, 4>(a, b, kind, line0, sm);
    else ens_run_lt<TL, VISC, 8>(a, b, kind, line0, sm);
}

__device__ __forceinline__ int ens_load_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <int TL, bool VISC>
__global__ void __launch_bounds__(TL * 32, TL == 8 ? 2 : 4) k_ensemble_stage(const __grid_constant__ EnsArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sm = reinterpret_cast<double *>(smem_raw);
    int *s_starts = reinterpret_cast<int *>(sm + a.tile_doubles);
    const bool starts_in_smem = a.nseg <= kEnsSmemStarts;
    if (starts_in_smem)
        for (int i = threadIdx.x; i < a.nseg; i += blockDim.x) s_starts[i] = a.segs[i].start;
    __shared__ int s_next, s_seg, s_ok;
    if (threadIdx.x == 0) s_next = atomicAdd(a.queue, 1);
    for (;;) {
        __syncthreads();  // s_next is visible, the previous item is complete
        const int it = s_next;
        if (it >= a.nitems) break;
        if (threadIdx.x == 0) {
            int lo = 0, hi = a.nseg - 1;  // last segment with start <= it
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if ((starts_in_smem ? s_starts[mid] : a.segs[mid].start) <= it) lo = mid;
                else hi = mid - 1;
            }
            int ok = 1;
            const EnsSeg sg = a.segs[lo];
            if (sg.wait_count > 0) {
                const int *dp = a.done + sg.box * kEnsPhases + sg.phase - 1;
                long long polls = 0;
                while (ens_load_acquire(dp) < sg.wait_count + a.wait_bias) {
                    if (++polls > a.poll_limit) { ok = 0; break; }
                    __nanosleep(100);
                }
                if (!ok) atomicCAS(a.err, 0, 1 + it);
            }
            s_seg = lo;
            s_ok = ok;
        }
        __syncthreads();  // every thread has read s_next; the segment is decoded
        // claim the next item now: the atomic's latency overlaps this item's work
        if (threadIdx.x == 0) s_next = atomicAdd(a.queue, 1);
        const EnsSeg sg = a.segs[s_seg];
        if (s_ok) {
            const int t0 = (it - sg.start) * a.chunk;
            const int t1 = min(t0 + a.chunk, sg.ntiles);
            for (int t = t0; t < t1; ++t) {
                if (t > t0) __syncthreads();  // the tile buffer is reused
                ens_run_item<TL, VISC>(a, sg.box, sg.kind, (int64_t)t * TL, sm);
            }
        }
        __syncthreads();  // the item's stores are issued by every thread
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(a.done + sg.box * kEnsPhases + sg.phase, 1);
        }
    }
}

}  // namespace csb

namespace csb {

// Launch one stage of the ensemble with TL-line work items: ctas_per_sm
// resident CTAs per SM (0: as many as fit), at most one CTA per item.
template <int TL>
int ens_launch_t(const EnsArgs &a, bool visc, int ctas_per_sm, int nsm, size_t smem, cudaStream_t st, int nbox) {
    // this translation unit's constant copy of the box table (stream-ordered)
    CSB_CUDA(cudaMemcpyToSymbolAsync(c_ens_boxes, a.boxes, (size_t)nbox * sizeof(EnsBox), 0,
                                     cudaMemcpyDeviceToDevice, st));
    CSB_CUDA(cudaMemcpyToSymbolAsync(c_ens_cf, a.cf_dev, sizeof(Coeffs), 0, cudaMemcpyDeviceToDevice, st));
    auto kern = visc ? k_ensemble_stage<TL, true> : k_ensemble_stage<TL, false>;
    if (int rc = set_smem(kern, smem)) return rc;
    int nb = 0;
    CSB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, TL * 32, smem));
    if (nb < 1) return set_error(CS_ERR_UNSUPPORTED, "ensemble: a %d-line tile does not fit an SM", TL);
    const int per = ctas_per_sm > 0 && ctas_per_sm < nb ? ctas_per_sm : nb;
    int64_t grid = (int64_t)(nsm > 0 ? nsm : 1) * per;
    if (grid > a.nitems) grid = a.nitems;
    if (grid < 1) return CS_OK;
    kern<<<(unsigned)grid, TL * 32, smem, st>>>(a);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

// ensemble_tl4.cu / ensemble_tl8.cu
int ens_launch_tl4(const EnsArgs &a, bool visc, int ctas_per_sm, int nsm, size_t smem, cudaStream_t st, int nbox);
int ens_launch_tl8(const EnsArgs &a, bool visc, int ctas_per_sm, int nsm, size_t smem, cudaStream_t st, int nbox);

}  // namespace csb
