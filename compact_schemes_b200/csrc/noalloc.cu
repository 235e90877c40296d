// noalloc.cu -- a compact derivative entry point that allocates no device memory.
//
// cs_deriv keeps the line-solver tables of every line configuration in device
// memory that the library allocates with cudaMalloc on first use.  Some
// callers cannot allow that: applications that hand all device memory to
// their own pool allocator at start-up, or that must not let a library
// allocate (cudaMalloc and cudaFree can synchronize the whole device) in the
// middle of a time-critical loop.  cs_deriv_noalloc computes the same
// derivative with its tables held in one file-scope device array that exists
// from module load until process exit on every GPU that loads the library.
#include <cstring>
#include <mutex>
#include <vector>

#include "context.h"
#include "tile.cuh"

namespace csb {

// Capacity of the table array: 6 per-lane tables of LT x 32 entries, the
// 832-entry reduced-system block and the cyclic vector (unused by the
// derivative), for the largest chunk LT = 32, i.e. lines of up to 1024 points.
constexpr int kNoAllocMaxLine = kMaxLine;
constexpr size_t kNoAllocTableDoubles = (size_t)7 * 32 * 32 + 832;  // 8000 doubles, 64000 bytes

static __device__ __align__(256) double g_noalloc_tables[kNoAllocTableDoubles];

// Device address of g_noalloc_tables, looked up once per device.
constexpr int kMaxDevices = 64;
static double *g_noalloc_addr[kMaxDevices] = {};
static std::mutex g_noalloc_mu;

static int noalloc_tables_address(double **out) {
    int dev = 0;
    CSB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return set_error(CS_ERR_UNSUPPORTED, "device ordinal %d", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_tables);
        if (e != cudaSuccess) return check_cuda(e, "cudaGetSymbolAddress(g_noalloc_tables)");
        g_noalloc_addr[dev] = static_cast<double *>(p);
    }
    *out = g_noalloc_addr[dev];
    return CS_OK;
}

// Same tile / warp-solve structure as k_deriv (numerics.cu), without the
// interface receive buffer and the line-end output: interface faces take the
// single-rank periodic sums from the line's far end.
template <int LT, int AXIS>
__global__ void __launch_bounds__(kThreads)
k_deriv_noalloc(const double *__restrict__ in, double *__restrict__ out, DevTables<double> tab, int lxi,
                int let, int nstart, int nend, int64_t F, Coeffs cf) {
    using L = LineLayout<LT>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sm = reinterpret_cast<double *>(smem_raw);
    const int n = tab.n;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const int64_t line0 = (int64_t)blockIdx.x * kTileLines;
    // stage
    if (AXIS == 0) {
        const int64_t fidx = line0 + w;
        if (fidx < F)
            for (int j = lane; j < n; j += 32) sm[w * L::kSlot + L::pos(j)] = in[fidx * n + j];
        __syncwarp();
    } else {
        const int l = tid % kTileLines;
        const int64_t fidx = line0 + l;
        if (fidx < F) {
            const int64_t base = line_base<AXIS>(fidx, lxi, let), s = line_stride<AXIS>(lxi, let);
            for (int j = tid / kTileLines; j < n; j += kThreads / kTileLines)
                sm[l * L::kSlot + L::pos(j)] = in[base + j * s];
        }
        __syncthreads();
    }
    // solve
    const int64_t fidx = line0 + w;
    if (fidx < F) {
        double d[1][LT];
        double *line = sm + w * L::kSlot;
        deriv_rhs<LT, double, double>(line, n, lane, nstart, nend, nullptr, cf, d[0]);
        warp_solve<LT, 1, double>(tab, d, lane);
        __syncwarp();
#pragma unroll
        for (int t = 0; t < LT; ++t)
            if (lane * LT + t < n) line[L::pos_ct(lane, t)] = d[0][t];
    }
    // store
    if (AXIS == 0) {
        __syncwarp();
        if (fidx < F)
            for (int j = lane; j < n; j += 32) out[fidx * n + j] = sm[w * L::kSlot + L::pos(j)];
    } else {
        __syncthreads();
        const int l = tid % kTileLines;
        const int64_t f2 = line0 + l;
        if (f2 < F) {
            const int64_t base = line_base<AXIS>(f2, lxi, let), s = line_stride<AXIS>(lxi, let);
            for (int j = tid / kTileLines; j < n; j += kThreads / kTileLines)
                out[base + j * s] = sm[l * L::kSlot + L::pos(j)];
        }
    }
}

template <int LT, int AXIS>
static int launch_noalloc_lt(const double *in, double *out, const DevTables<double> &tab, const cs_dcomp &d,
                             int nstart, int nend, int64_t F, const Coeffs &cf, cudaStream_t st) {
    const size_t smem = (size_t)kTileLines * LineLayout<LT>::kSlot * sizeof(double);
    auto kern = k_deriv_noalloc<LT, AXIS>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute");
    }
    const int64_t blocks = (F + kTileLines - 1) / kTileLines;
    kern<<<(unsigned)blocks, kThreads, smem, st>>>(in, out, tab, d.lxi, d.let, nstart, nend, F, cf);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

template <int AXIS>
static int launch_noalloc(int lt, const double *in, double *out, const DevTables<double> &tab,
                          const cs_dcomp &d, int nstart, int nend, int64_t F, const Coeffs &cf,
                          cudaStream_t st) {
    switch (lt) {
        case 2: return launch_noalloc_lt<2, AXIS>(in, out, tab, d, nstart, nend, F, cf, st);
        case 4: return launch_noalloc_lt<4, AXIS>(in, out, tab, d, nstart, nend, F, cf, st);
        case 8: return launch_noalloc_lt<8, AXIS>(in, out, tab, d, nstart, nend, F, cf, st);
        case 16: return launch_noalloc_lt<16, AXIS>(in, out, tab, d, nstart, nend, F, cf, st);
        case 32: return launch_noalloc_lt<32, AXIS>(in, out, tab, d, nstart, nend, F, cf, st);
    }
    return set_error(CS_ERR_UNSUPPORTED, "chunk length %d", lt);
}

}  // namespace csb

using namespace csb;

extern "C" int cs_deriv_noalloc(int axis, const double *in, double *out, int nstart, int nend, cs_dcomp d,
                                void *stream) {
    if (!in || !out) return set_error(CS_ERR_INVALID, "null argument");
    if (d.lxi < 1 || d.let < 1 || d.lze < 1 || (int64_t)d.lxi * d.let * d.lze != (int64_t)d.lmx)
        return set_error(CS_ERR_INVALID, "inconsistent t_dcomp {%d,%d,%d,%d}", d.lmx, d.lxi, d.let, d.lze);
    if (axis < 0 || axis > 2) return set_error(CS_ERR_INVALID, "axis %d", axis);
    const int n = axis == 0 ? d.lxi : (axis == 1 ? d.let : d.lze);
    if (n > kNoAllocMaxLine)
        return set_error(CS_ERR_UNSUPPORTED,
                         "cs_deriv_noalloc: line length %d exceeds the %d-point maximum of its preallocated "
                         "%zu-byte table array", n, kNoAllocMaxLine, kNoAllocTableDoubles * sizeof(double));
    if (n < 5 || ((nstart || nend) && n < kLmd))
        return set_error(CS_ERR_UNSUPPORTED, "line length %d too short for the closure", n);
    std::vector<double> a(n), b(n), c(n);
    deriv_rows(n, nstart, nend, a.data(), b.data(), c.data());
    HostTables h;
    if (!build_tables(n, a.data(), b.data(), c.data(), false, h))
        return set_error(CS_ERR_UNSUPPORTED, "line length %d", n);
    // pack: fwd1, fwd2, bwd1, bwd2, rca, rcc (lt x 32 each), k1, k2 (384 each), invb (64)
    std::vector<double> packed;
    for (auto *v : {&h.fwd1, &h.fwd2, &h.bwd1, &h.bwd2, &h.rca, &h.rcc, &h.k1, &h.k2, &h.invb})
        packed.insert(packed.end(), v->begin(), v->end());
    if (packed.size() > kNoAllocTableDoubles)
        return set_error(CS_ERR_UNSUPPORTED, "cs_deriv_noalloc: %zu table entries exceed the capacity %zu",
                         packed.size(), kNoAllocTableDoubles);
    double *base = nullptr;
    if (int rc = noalloc_tables_address(&base)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // The whole used region is rewritten by every call; nothing needs zeroing.
    CSB_CUDA(cudaMemcpyAsync(base, packed.data(), packed.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    DevTables<double> tab{};
    const size_t tl = (size_t)h.lt * 32;
    tab.fwd1 = base;
    tab.fwd2 = base + tl;
    tab.bwd1 = base + 2 * tl;
    tab.bwd2 = base + 3 * tl;
    tab.rca = base + 4 * tl;
    tab.rcc = base + 5 * tl;
    tab.k1 = base + 6 * tl;
    tab.k2 = base + 6 * tl + 384;
    tab.invb = base + 6 * tl + 768;
    tab.cycz = nullptr;
    tab.n = h.n;
    tab.p = h.p;
    tab.last_len = h.last_len;
    tab.cyclic = 0;
    tab.pcr = h.pcr64;
    Coeffs cf;
    compute_interface_coeffs(cf);
    const int64_t F = axis == 0 ? (int64_t)d.let * d.lze : (axis == 1 ? (int64_t)d.lxi * d.lze : (int64_t)d.lxi * d.let);
    switch (axis) {
        case 0: return launch_noalloc<0>(h.lt, in, out, tab, d, nstart, nend, F, cf, st);
        case 1: return launch_noalloc<1>(h.lt, in, out, tab, d, nstart, nend, F, cf, st);
        default: return launch_noalloc<2>(h.lt, in, out, tab, d, nstart, nend, F, cf, st);
    }
}
