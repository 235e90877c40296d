// numerics.cu -- compact derivative / filter line solves and the numerics_*
// C-ABI (replaces src/numerics_base.hpp, src/numerics_pc.hpp,
// src/numerics_rtc.hpp and src/cuda/kernels/numerics_*.hpp of the reference).
//
// Kernel shape: a CTA of 8 warps stages a tile of 8 lines in shared memory
// (LineLayout order), each warp solves one line with the partitioned
// warp-shuffle solver, and the tile is written back.  x lines are
// contiguous, so each warp stages its own line with 256-byte coalesced
// accesses; y and z lines are staged cooperatively as rows of 8 consecutive
// lines (64-byte segments per row, full 32-byte sectors).
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "context.h"
#include "tile.cuh"

namespace csb {

static thread_local char g_err[512] = "";

int set_error(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

int check_cuda(cudaError_t e, const char *what) {
    return set_error(CS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

TableCache::~TableCache() {
    for (auto &kv : map_) {
        if (kv.second->d64) cudaFree(kv.second->d64);
        if (kv.second->d32) cudaFree(kv.second->d32);
        delete kv.second;
    }
}

// Whether every lane's per-row factors equal the compile-time interior_chunk
// values (exact comparison): the line's chunks are all full and hold only the
// constant interior rows.
template <int LT>
static bool interior_match(const HostTables &h) {
    constexpr InteriorChunk<LT> K = interior_chunk<LT>();
    const std::vector<double> *tabs[6] = {&h.fwd1, &h.fwd2, &h.bwd1, &h.bwd2, &h.rca, &h.rcc};
    const double *ref[6] = {K.fwd1, K.fwd2, K.bwd1, K.bwd2, K.rca, K.rcc};
    for (int k = 0; k < 6; ++k)
        for (int t = 0; t < LT; ++t)
            for (int lane = 0; lane < h.p; ++lane)
                if ((*tabs[k])[(size_t)t * 32 + lane] != ref[k][t]) return false;
    return true;
}
static bool interior_tables(const HostTables &h) {
    if (h.cyclic || h.n != h.p * h.lt || h.p < 2) return false;
    switch (h.lt) {
        case 2: return interior_match<2>(h);
        case 4: return interior_match<4>(h);
        case 8: return interior_match<8>(h);
        case 16: return interior_match<16>(h);
        case 32: return interior_match<32>(h);
    }
    return false;
}

template <typename CT>
static void bind(DevTables<CT> &t, CT *base, const HostTables &h) {
    const size_t tl = (size_t)h.lt * 32;
    t.fwd1 = base;
    t.fwd2 = base + tl;
    t.bwd1 = base + 2 * tl;
    t.bwd2 = base + 3 * tl;
    t.rca = base + 4 * tl;
    t.rcc = base + 5 * tl;
    t.k1 = base + 6 * tl;
    t.k2 = base + 6 * tl + 384;
    t.invb = base + 6 * tl + 768;
    t.cycz = base + 6 * tl + 832;
    t.cyc_s1 = (CT)h.cyc_s1;
    t.cyc_s2 = (CT)h.cyc_s2;
    t.n = h.n;
    t.p = h.p;
    t.last_len = h.last_len;
    t.cyclic = h.cyclic ? 1 : 0;
    t.pcr = sizeof(CT) == 4 ? h.pcr32 : h.pcr64;
    t.interior = interior_tables(h) ? 1 : 0;
}

// Device layout of the tables; fp32 selects the inverse diagonals of the
// FP32 PCR depth.
static std::vector<double> pack(const HostTables &h, bool fp32 = false) {
    std::vector<double> v;
    for (auto *a : {&h.fwd1, &h.fwd2, &h.bwd1, &h.bwd2, &h.rca, &h.rcc, &h.k1, &h.k2, fp32 ? &h.invb32 : &h.invb})
        v.insert(v.end(), a->begin(), a->end());
    if (h.cyclic) v.insert(v.end(), h.cycz.begin(), h.cycz.end());
    else v.insert(v.end(), (size_t)h.lt * 32, 0.0);
    return v;
}

// Whether all lanes of a table set share lane 0's per-row chunk factors
// (every chunk full, no cyclic correction), and those factors in FP32.  The
// comparison is exact, so a line qualifies only when its tables say so.
static void chunk_factors(const HostTables &h, bool &uniform, float *cfu) {
    uniform = !h.cyclic && h.lt <= 32 && h.n == h.p * h.lt && h.p >= 2;
    const std::vector<double> *tabs[6] = {&h.fwd1, &h.fwd2, &h.bwd1, &h.bwd2, &h.rca, &h.rcc};
    for (int k = 0; k < 6 && uniform; ++k)
        for (int t = 0; t < h.lt && uniform; ++t)
            for (int lane = 1; lane < h.p; ++lane)
                if ((*tabs[k])[(size_t)t * 32 + lane] != (*tabs[k])[(size_t)t * 32]) {
                    uniform = false;
                    break;
                }
    if (!uniform) return;
    for (int k = 0; k < 6; ++k)
        for (int t = 0; t < h.lt; ++t) {
            const double v = (*tabs[k])[(size_t)t * 32];
            cfu[k * h.lt + t] = (float)(k >= 4 ? -v : v);
        }
}

static bool host_tables_for(int n, int scheme, int nstart, int nend, double af, HostTables &h, int min_lt = 2) {
    std::vector<double> a(n), b(n), c(n);
    bool cyclic = false;
    if (scheme == kDeriv) {
        deriv_rows(n, nstart, nend, a.data(), b.data(), c.data());
    } else if (scheme == kDerivT) {
        std::vector<double> a0(n), c0(n);
        deriv_rows(n, nstart, nend, a0.data(), b.data(), c0.data());
        for (int i = 0; i < n; ++i) {
            a[i] = i > 0 ? c0[i - 1] : 0.0;
            c[i] = i < n - 1 ? a0[i + 1] : 0.0;
        }
    } else {
        cyclic = nstart && nend;
        filter_rows(n, cyclic, af, a.data(), b.data(), c.data());
        if (scheme == kFilterT && !cyclic) {  // the cyclic filter matrix is symmetric
            std::vector<double> a0(a), c0(c);
            for (int i = 0; i < n; ++i) {
                a[i] = i > 0 ? c0[i - 1] : 0.0;
                c[i] = i < n - 1 ? a0[i + 1] : 0.0;
            }
        }
    }
    return build_tables(n, a.data(), b.data(), c.data(), cyclic, h, min_lt);
}

const DeviceTables *TableCache::get(int n, int scheme, int nstart, int nend, double af, int min_lt) {
    uint64_t bits = 0;
    if (scheme == kFilter || scheme == kFilterT) std::memcpy(&bits, &af, sizeof bits);
    TableKey key{n, scheme, nstart ? 1 : 0, nend ? 1 : 0, bits, min_lt};
    std::lock_guard<std::mutex> lk(mu_);
    auto it = map_.find(key);
    if (it != map_.end()) return it->second;
    auto *dt = new DeviceTables();
    if (!host_tables_for(n, scheme, nstart, nend, af, dt->host, min_lt)) {
        delete dt;
        set_error(CS_ERR_UNSUPPORTED, "line length %d outside [5, %d]", n, kMaxLine);
        return nullptr;
    }
    std::vector<double> v = pack(dt->host);
    const std::vector<double> v32 = pack(dt->host, true);
    std::vector<float> vf(v32.begin(), v32.end());
    if (cudaMalloc(&dt->d64, v.size() * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&dt->d32, vf.size() * sizeof(float)) != cudaSuccess ||
        cudaMemcpy(dt->d64, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(dt->d32, vf.data(), vf.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        if (dt->d64) cudaFree(dt->d64);
        if (dt->d32) cudaFree(dt->d32);
        delete dt;
        set_error(CS_ERR_ALLOC, "line-solver table upload failed");
        return nullptr;
    }
    bind(dt->t64, dt->d64, dt->host);
    bind(dt->t32, dt->d32, dt->host);
    dt->lt = dt->host.lt;
    chunk_factors(dt->host, dt->uniform, dt->cfu);
    map_[key] = dt;
    return dt;
}

// ----------------------------------------------------------------------------
// kernels
// ----------------------------------------------------------------------------
// Stage the tile's lines into shared memory.
template <int LT, int AXIS, typename T>
__device__ __forceinline__ void load_tile(const T *__restrict__ in, T *sm, int64_t line0, int64_t F,
                                          int n, int lxi, int let) {
    using L = LineLayout<LT>;
    const int tid = threadIdx.x;
    if (AXIS == 0) {
        const int w = tid >> 5, lane = tid & 31;
        const int64_t fidx = line0 + w;
        if (fidx < F) {
            const T *src = in + fidx * n;
            for (int j = lane; j < n; j += 32) sm[w * L::kSlot + L::pos(j)] = src[j];
        }
    } else {
        const int l = tid % kTileLines;
        const int64_t fidx = line0 + l;
        if (fidx < F) {
            const int64_t base = line_base<AXIS>(fidx, lxi, let), s = line_stride<AXIS>(lxi, let);
            for (int j = tid / kTileLines; j < n; j += kThreads / kTileLines)
                sm[l * L::kSlot + L::pos(j)] = in[base + j * s];
        }
    }
}

template <int LT, int AXIS, typename T>
__device__ __forceinline__ void store_tile(T *__restrict__ out, const T *sm, int64_t line0, int64_t F,
                                           int n, int lxi, int let) {
    using L = LineLayout<LT>;
    const int tid = threadIdx.x;
    if (AXIS == 0) {
        const int w = tid >> 5, lane = tid & 31;
        const int64_t fidx = line0 + w;
        if (fidx < F) {
            T *dst = out + fidx * n;
            for (int j = lane; j < n; j += 32) dst[j] = sm[w * L::kSlot + L::pos(j)];
        }
    } else {
        const int l = tid % kTileLines;
        const int64_t fidx = line0 + l;
        if (fidx < F) {
            const int64_t base = line_base<AXIS>(fidx, lxi, let), s = line_stride<AXIS>(lxi, let);
            for (int j = tid / kTileLines; j < n; j += kThreads / kTileLines)
                out[base + j * s] = sm[l * L::kSlot + L::pos(j)];
        }
    }
}

template <int LT, typename T>
__device__ __forceinline__ void store_line_regs(T *line, const T (&d)[LT], int lane, int n) {
    using L = LineLayout<LT>;
#pragma unroll
    for (int t = 0; t < LT; ++t)
        if (lane * LT + t < n) line[L::pos_ct(lane, t)] = d[t];
}

// Compact first derivative of one field along AXIS (deriv_kernel_1d/2d,
// src/cuda/kernels/numerics_pc.hpp:124-249).
template <int LT, int AXIS, typename T>
__global__ void __launch_bounds__(kThreads)
k_deriv(const T *__restrict__ in, T *__restrict__ out, DevTables<T> tab, int lxi, int let,
        int nstart, int nend, const T *__restrict__ recv, T *__restrict__ drva, int64_t F, Coeffs cf) {
    using L = LineLayout<LT>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *sm = reinterpret_cast<T *>(smem_raw);
    const int n = tab.n;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t line0 = (int64_t)blockIdx.x * kTileLines;
    load_tile<LT, AXIS>(in, sm, line0, F, n, lxi, let);
    if (AXIS == 0) __syncwarp();
    else __syncthreads();
    const int64_t fidx = line0 + w;
    if (fidx < F) {
        T d[1][LT];
        T r4[4];
        const T *rp = nullptr;
        if (recv && (nstart || nend)) {
#pragma unroll
            for (int k = 0; k < 4; ++k) r4[k] = recv[k * F + fidx];
            rp = r4;
        }
        T *line = sm + w * L::kSlot;
        deriv_rhs<LT, T, T>(line, n, lane, nstart, nend, rp, cf, d[0]);
        warp_solve<LT, 1, T>(tab, d, lane);
        if (drva) {
            if (lane == 0) drva[fidx] = d[0][0];
            if (lane == (n - 1) / LT) drva[5 * F + fidx] = get_at<LT, T>(d[0], (n - 1) - lane * LT);
        }
        __syncwarp();
        store_line_regs<LT, T>(line, d[0], lane, n);
    }
    if (AXIS == 0) __syncwarp();
    else __syncthreads();
    store_tile<LT, AXIS>(out, sm, line0, F, n, lxi, let);
}

// Same derivative with two lines per warp: a CTA of kThreads threads holds
// kPairLines lines, warp w solves lines 2w and 2w+1 in one warp_solve (their
// table loads and shuffle latencies are shared), and the y/z tiles cover 16
// consecutive x positions (128-byte rows).  Used for chunks of up to 8 rows.
constexpr int kPairLines = 16;
#ifndef CSB_PAIR_MINB
#define CSB_PAIR_MINB 3
#endif

template <int LT, int AXIS, typename T, bool STORE>
__device__ __forceinline__ void pair_tile_io(const T *__restrict__ in, T *__restrict__ out, T *sm, int64_t line0,
                                             int64_t F, int n, int lxi, int let) {
    using L = LineLayout<LT>;
    const int tid = threadIdx.x;
    if (AXIS == 0) {
        const int w = tid >> 5, lane = tid & 31;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int l = 2 * w + h;
            const int64_t fidx = line0 + l;
            if (fidx >= F) continue;
            for (int j = lane; j < n; j += 32) {
                if (STORE) out[fidx * n + j] = sm[l * L::kSlot + L::pos(j)];
                else sm[l * L::kSlot + L::pos(j)] = in[fidx * n + j];
            }
        }
    } else {
        const int l = tid % kPairLines;
        const int64_t fidx = line0 + l;
        if (fidx < F) {
            const int64_t base = line_base<AXIS>(fidx, lxi, let), s = line_stride<AXIS>(lxi, let);
            for (int j = tid / kPairLines; j < n; j += kThreads / kPairLines) {
                if (STORE) out[base + j * s] = sm[l * L::kSlot + L::pos(j)];
                else sm[l * L::kSlot + L::pos(j)] = in[base + j * s];
            }
        }
    }
}

template <int LT, int AXIS, typename T>
__global__ void __launch_bounds__(kThreads, CSB_PAIR_MINB)
k_deriv_pair(const T *__restrict__ in, T *__restrict__ out, DevTables<T> tab, int lxi, int let, int nstart,
             int nend, const T *__restrict__ recv, T *__restrict__ drva, int64_t F, Coeffs cf) {
    using L = LineLayout<LT>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *sm = reinterpret_cast<T *>(smem_raw);
    const int n = tab.n;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t line0 = (int64_t)blockIdx.x * kPairLines;
    pair_tile_io<LT, AXIS, T, false>(in, nullptr, sm, line0, F, n, lxi, let);
    if (AXIS == 0) __syncwarp();
    else __syncthreads();
    const int64_t fidx0 = line0 + 2 * w;
    if (fidx0 < F) {
        T d[2][LT];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t fidx = fidx0 + h;
            if (fidx < F) {
                T r4[4];
                const T *rp = nullptr;
                if (recv && (nstart || nend)) {
#pragma unroll
                    for (int k = 0; k < 4; ++k) r4[k] = recv[k * F + fidx];
                    rp = r4;
                }
                deriv_rhs<LT, T, T>(sm + (2 * w + h) * L::kSlot, n, lane, nstart, nend, rp, cf, d[h]);
            } else {
#pragma unroll
                for (int t = 0; t < LT; ++t) d[h][t] = T(0);
            }
        }
        warp_solve<LT, 2, T>(tab, d, lane);
        __syncwarp();
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t fidx = fidx0 + h;
            if (fidx >= F) continue;
            if (drva) {
                if (lane == 0) drva[fidx] = d[h][0];
                if (lane == (n - 1) / LT) drva[5 * F + fidx] = get_at<LT, T>(d[h], (n - 1) - lane * LT);
            }
            store_line_regs<LT, T>(sm + (2 * w + h) * L::kSlot, d[h], lane, n);
        }
    }
    if (AXIS == 0) __syncwarp();
    else __syncthreads();
    pair_tile_io<LT, AXIS, T, true>(nullptr, out, sm, line0, F, n, lxi, let);
}

// Compact filter of one field along AXIS.
template <int LT, int AXIS>
__global__ void __launch_bounds__(kThreads)
k_filter(const double *__restrict__ in, double *__restrict__ out, DevTables<double> tab, int lxi,
         int let, double af, int64_t F) {
    using L = LineLayout<LT>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sm = reinterpret_cast<double *>(smem_raw);
    const int n = tab.n;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t line0 = (int64_t)blockIdx.x * kTileLines;
    load_tile<LT, AXIS>(in, sm, line0, F, n, lxi, let);
    if (AXIS == 0) __syncwarp();
    else __syncthreads();
    const int64_t fidx = line0 + w;
    if (fidx < F) {
        double d[1][LT];
        double *line = sm + w * L::kSlot;
        filter_rhs<LT, double, double>(line, n, lane, tab.cyclic != 0, af, d[0]);
        warp_solve<LT, 1, double>(tab, d, lane);
        __syncwarp();
        store_line_regs<LT, double>(line, d[0], lane, n);
    }
    if (AXIS == 0) __syncwarp();
    else __syncthreads();
    store_tile<LT, AXIS>(out, sm, line0, F, n, lxi, let);
}

// Interface sums of one face (fill_gpu_buffer_kernel,
// src/cuda/kernels/numerics_pc.hpp:42-122).
template <int AXIS>
__global__ void k_fill(const double *__restrict__ in, double *__restrict__ send, int lxi, int let,
                       int n, int face, int64_t F, Coeffs cf) {
    const int64_t fidx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (fidx >= F) return;
    const int64_t base = line_base<AXIS>(fidx, lxi, let), s = line_stride<AXIS>(lxi, let);
    const int istart = face * (n - 1), inc = 1 - 2 * face;
    double v0 = 0.0, v1 = 0.0;
#pragma unroll
    for (int i = 0; i < kLmd; ++i) {
        const double f = in[base + (int64_t)(istart + inc * i) * s];
        v0 += cf.pbco[i] * f;
        v1 += cf.pbco[kLmd + i] * f;
    }
    send[fidx] = v0;
    send[F + fidx] = v1;
}

// ----------------------------------------------------------------------------
// launch helpers
// ----------------------------------------------------------------------------
inline int64_t face_size(const cs_dcomp &d, int axis) {
    return axis == 0 ? (int64_t)d.let * d.lze : (axis == 1 ? (int64_t)d.lxi * d.lze : (int64_t)d.lxi * d.let);
}
inline int line_len(const cs_dcomp &d, int axis) { return axis == 0 ? d.lxi : (axis == 1 ? d.let : d.lze); }

template <typename KernelT>
static int prep_smem(KernelT kern, size_t bytes) {
    if (bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute");
    }
    return CS_OK;
}

template <int LT, int AXIS, typename T>
static int launch_deriv_lt(const T *in, T *out, const DevTables<T> &tab, const cs_dcomp &d,
                           int nstart, int nend, const T *recv, T *drva, const Coeffs &cf,
                           cudaStream_t st) {
    const int64_t F = face_size(d, AXIS);
    if constexpr (LT <= 8) {
        const size_t smem = (size_t)kPairLines * LineLayout<LT>::kSlot * sizeof(T);
        auto kern = k_deriv_pair<LT, AXIS, T>;
        if (int rc = prep_smem(kern, smem)) return rc;
        const int64_t blocks = (F + kPairLines - 1) / kPairLines;
        kern<<<(unsigned)blocks, kThreads, smem, st>>>(in, out, tab, d.lxi, d.let, nstart, nend, recv, drva, F,
                                                      cf);
        CSB_CUDA(cudaGetLastError());
        return CS_OK;
    }
    const size_t smem = (size_t)kTileLines * LineLayout<LT>::kSlot * sizeof(T);
    auto kern = k_deriv<LT, AXIS, T>;
    int rc = prep_smem(kern, smem);
    if (rc) return rc;
    const int64_t blocks = (F + kTileLines - 1) / kTileLines;
    kern<<<(unsigned)blocks, kThreads, smem, st>>>(in, out, tab, d.lxi, d.let, nstart, nend, recv,
                                                  drva, F, cf);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

template <int AXIS, typename T>
static int launch_deriv_axis(int lt, const T *in, T *out, const DevTables<T> &tab, const cs_dcomp &d,
                             int nstart, int nend, const T *recv, T *drva, const Coeffs &cf,
                             cudaStream_t st) {
    switch (lt) {
        case 2: return launch_deriv_lt<2, AXIS, T>(in, out, tab, d, nstart, nend, recv, drva, cf, st);
        case 4: return launch_deriv_lt<4, AXIS, T>(in, out, tab, d, nstart, nend, recv, drva, cf, st);
        case 8: return launch_deriv_lt<8, AXIS, T>(in, out, tab, d, nstart, nend, recv, drva, cf, st);
        case 16: return launch_deriv_lt<16, AXIS, T>(in, out, tab, d, nstart, nend, recv, drva, cf, st);
        case 32: return launch_deriv_lt<32, AXIS, T>(in, out, tab, d, nstart, nend, recv, drva, cf, st);
    }
    return set_error(CS_ERR_UNSUPPORTED, "chunk length %d", lt);
}

template <int LT, int AXIS>
static int launch_filter_lt(const double *in, double *out, const DevTables<double> &tab,
                            const cs_dcomp &d, double af, cudaStream_t st) {
    const int64_t F = face_size(d, AXIS);
    const size_t smem = (size_t)kTileLines * LineLayout<LT>::kSlot * sizeof(double);
    auto kern = k_filter<LT, AXIS>;
    int rc = prep_smem(kern, smem);
    if (rc) return rc;
    const int64_t blocks = (F + kTileLines - 1) / kTileLines;
    kern<<<(unsigned)blocks, kThreads, smem, st>>>(in, out, tab, d.lxi, d.let, af, F);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

template <int AXIS>
static int launch_filter_axis(int lt, const double *in, double *out, const DevTables<double> &tab,
                              const cs_dcomp &d, double af, cudaStream_t st) {
    switch (lt) {
        case 2: return launch_filter_lt<2, AXIS>(in, out, tab, d, af, st);
        case 4: return launch_filter_lt<4, AXIS>(in, out, tab, d, af, st);
        case 8: return launch_filter_lt<8, AXIS>(in, out, tab, d, af, st);
        case 16: return launch_filter_lt<16, AXIS>(in, out, tab, d, af, st);
        case 32: return launch_filter_lt<32, AXIS>(in, out, tab, d, af, st);
    }
    return set_error(CS_ERR_UNSUPPORTED, "chunk length %d", lt);
}

static int check_dims(const cs_dcomp &d) {
    if (d.lxi < 1 || d.let < 1 || d.lze < 1 || (int64_t)d.lxi * d.let * d.lze != (int64_t)d.lmx)
        return set_error(CS_ERR_INVALID, "inconsistent t_dcomp {%d,%d,%d,%d}", d.lmx, d.lxi, d.let, d.lze);
    return CS_OK;
}

static bool same_dims(const cs_dcomp &a, const cs_dcomp &b) {
    return a.lmx == b.lmx && a.lxi == b.lxi && a.let == b.let && a.lze == b.lze;
}

template <typename T>
const DevTables<T> &pick_tables(const DeviceTables &dt);
template <>
const DevTables<double> &pick_tables<double>(const DeviceTables &dt) { return dt.t64; }
template <>
const DevTables<float> &pick_tables<float>(const DeviceTables &dt) { return dt.t32; }

template <typename T>
static int deriv_impl(cs_numerics *nm, int axis, const T *in, T *out, int nstart, int nend,
                      cs_dcomp d, unsigned var, unsigned comp, unsigned slot, int halo,
                      void *stream) {
    if (!nm || !in || !out) return set_error(CS_ERR_INVALID, "null argument");
    if (!nm->setup_done) return set_error(CS_ERR_STATE, "cs_deriv before cs_deriv_setup");
    if (int rc = check_dims(d)) return rc;
    if (!same_dims(d, nm->d)) return set_error(CS_ERR_INVALID, "dims differ from the numerics object");
    if (axis < 0 || axis > 2 || var >= 5 || comp > 14 || slot > 14)
        return set_error(CS_ERR_INVALID, "axis %d var %u comp %u slot %u", axis, var, comp, slot);
    const int n = line_len(d, axis);
    if ((nstart || nend) && n < kLmd) return set_error(CS_ERR_UNSUPPORTED, "interface closure needs n >= 8");
    const DeviceTables *dt = nm->tables.get(n, kDeriv, nstart, nend, 0.0);
    if (!dt) return CS_ERR_UNSUPPORTED;
    const int64_t F = face_size(d, axis);
    const T *recv = nullptr;
    T *drva = nullptr;
    if (sizeof(T) == sizeof(double)) {
        if (halo == CS_HALO_RECV) recv = reinterpret_cast<const T *>(nm->recv[axis] + (int64_t)var * 4 * F);
        drva = reinterpret_cast<T *>(nm->drva[axis] + (int64_t)var * F);
    } else if (halo == CS_HALO_RECV && (nstart || nend)) {
        return set_error(CS_ERR_UNSUPPORTED, "FP32 derivative supports CS_HALO_SELF only");
    }
    const T *src = in + (int64_t)comp * d.lmx;
    T *dst = out + (int64_t)slot * d.lmx;
    cudaStream_t st = (cudaStream_t)stream;
    const DevTables<T> &tab = pick_tables<T>(*dt);
    switch (axis) {
        case 0: return launch_deriv_axis<0, T>(dt->lt, src, dst, tab, d, nstart, nend, recv, drva, nm->cf, st);
        case 1: return launch_deriv_axis<1, T>(dt->lt, src, dst, tab, d, nstart, nend, recv, drva, nm->cf, st);
        default: return launch_deriv_axis<2, T>(dt->lt, src, dst, tab, d, nstart, nend, recv, drva, nm->cf, st);
    }
}

}  // namespace csb

using namespace csb;

extern "C" {

const char *cs_last_error(void) { return csb::g_err; }
int cs_version(void) { return 1; }

int cs_numerics_create(cs_numerics **out, cs_dcomp d, const int nbc[2][3]) {
    if (!out || !nbc) return set_error(CS_ERR_INVALID, "null argument");
    *out = nullptr;
    if (int rc = check_dims(d)) return rc;
    auto *nm = new cs_numerics();
    nm->d = d;
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 3; ++a) {
            const int b = nbc[f][a];
            nm->nbc[f][a] = b;
            if (b == CS_BC_NON_REFLECTIVE || b == CS_BC_WALL_INVISCID || b == CS_BC_WALL_VISCOUS ||
                b == CS_BC_INTER_CURV) nm->ndf[f][a] = 0;
            else if (b == CS_BC_INTER_STRAIGHT || b == CS_BC_INTER_SUBDOMAINS || b == CS_BC_PERIODIC)
                nm->ndf[f][a] = 1;
            else {
                delete nm;
                return set_error(CS_ERR_INVALID, "unknown boundary code %d", b);
            }
        }
    for (int a = 0; a < 3; ++a) {
        const int64_t F = face_size(d, a);
        if (cudaMalloc(&nm->drva[a], 2 * 5 * F * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&nm->send[a], 4 * 5 * F * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&nm->recv[a], 4 * 5 * F * sizeof(double)) != cudaSuccess) {
            cs_numerics_destroy(nm);
            return set_error(CS_ERR_ALLOC, "numerics scratch allocation failed");
        }
        cudaMemset(nm->drva[a], 0, 2 * 5 * F * sizeof(double));
        cudaMemset(nm->send[a], 0, 4 * 5 * F * sizeof(double));
        cudaMemset(nm->recv[a], 0, 4 * 5 * F * sizeof(double));
    }
    *out = nm;
    return CS_OK;
}

int cs_numerics_destroy(cs_numerics *nm) {
    if (!nm) return CS_OK;
    for (int a = 0; a < 3; ++a) {
        if (nm->drva[a]) cudaFree(nm->drva[a]);
        if (nm->send[a]) cudaFree(nm->send[a]);
        if (nm->recv[a]) cudaFree(nm->recv[a]);
    }
    delete nm;
    return CS_OK;
}

int cs_deriv_setup(cs_numerics *nm) {
    if (!nm) return set_error(CS_ERR_INVALID, "null argument");
    compute_interface_coeffs(nm->cf);
    for (int a = 0; a < 3; ++a) {
        const int n = line_len(nm->d, a);
        if (n < 5) continue;  // degenerate axis: derivative along it is rejected at call time
        if (!nm->tables.get(n, kDeriv, nm->ndf[0][a], nm->ndf[1][a], 0.0)) return CS_ERR_UNSUPPORTED;
    }
    nm->setup_done = true;
    return CS_OK;
}

int cs_interface_coeffs(double pbco[16], double pbci[16]) {
    if (!pbco || !pbci) return set_error(CS_ERR_INVALID, "null argument");
    Coeffs cf;
    compute_interface_coeffs(cf);
    std::memcpy(pbco, cf.pbco, sizeof cf.pbco);
    std::memcpy(pbci, cf.pbci, sizeof cf.pbci);
    return CS_OK;
}

int cs_get_coeffs(const cs_numerics *nm, double pbco[16], double pbci[16]) {
    if (!nm || !pbco || !pbci) return set_error(CS_ERR_INVALID, "null argument");
    if (!nm->setup_done) return set_error(CS_ERR_STATE, "cs_get_coeffs before cs_deriv_setup");
    std::memcpy(pbco, nm->cf.pbco, sizeof nm->cf.pbco);
    std::memcpy(pbci, nm->cf.pbci, sizeof nm->cf.pbci);
    return CS_OK;
}

int cs_get_ndf(const cs_numerics *nm, int ndf[2][3]) {
    if (!nm || !ndf) return set_error(CS_ERR_INVALID, "null argument");
    std::memcpy(ndf, nm->ndf, sizeof nm->ndf);
    return CS_OK;
}

int cs_get_buffers(cs_numerics *nm, int axis, double **drva, double **send, double **recv) {
    if (!nm || axis < 0 || axis > 2) return set_error(CS_ERR_INVALID, "bad argument");
    if (drva) *drva = nm->drva[axis];
    if (send) *send = nm->send[axis];
    if (recv) *recv = nm->recv[axis];
    return CS_OK;
}

int cs_deriv(cs_numerics *nm, int axis, const double *in, double *out, int nstart, int nend,
             cs_dcomp d, unsigned var, unsigned comp, unsigned slot, int halo, void *stream) {
    return deriv_impl<double>(nm, axis, in, out, nstart, nend, d, var, comp, slot, halo, stream);
}

int cs_deriv_f32(cs_numerics *nm, int axis, const float *in, float *out, int nstart, int nend,
                 cs_dcomp d, unsigned var, unsigned comp, unsigned slot, int halo, void *stream) {
    return deriv_impl<float>(nm, axis, in, out, nstart, nend, d, var, comp, slot, halo, stream);
}

int cs_fill_buffers(cs_numerics *nm, const double *in, int var_lo, int var_hi, int nrt, cs_dcomp d,
                    void *stream) {
    if (!nm || !in) return set_error(CS_ERR_INVALID, "null argument");
    if (!nm->setup_done) return set_error(CS_ERR_STATE, "cs_fill_buffers before cs_deriv_setup");
    if (int rc = check_dims(d)) return rc;
    if (var_lo < 0 || var_hi > 5 || var_lo > var_hi) return set_error(CS_ERR_INVALID, "variable range");
    cudaStream_t st = (cudaStream_t)stream;
    for (int m = var_lo; m < var_hi; ++m)
        for (int nn = 0; nn < 3; ++nn) {
            const int nzk = (1 - nrt) * nn;
            const int64_t F = face_size(d, nn);
            const int n = line_len(d, nn);
            const double *src = in + ((int64_t)nzk + (int64_t)m * 3) * d.lmx;
            for (int ip = 0; ip < 2; ++ip) {
                if (nm->ndf[ip][nn] != 1) continue;
                if (n < kLmd) return set_error(CS_ERR_UNSUPPORTED, "interface face needs n >= 8");
                double *snd = nm->send[nn] + (int64_t)m * 4 * F + (int64_t)ip * 2 * F;
                const unsigned blocks = (unsigned)((F + 255) / 256);
                if (nn == 0) k_fill<0><<<blocks, 256, 0, st>>>(src, snd, d.lxi, d.let, n, ip, F, nm->cf);
                else if (nn == 1) k_fill<1><<<blocks, 256, 0, st>>>(src, snd, d.lxi, d.let, n, ip, F, nm->cf);
                else k_fill<2><<<blocks, 256, 0, st>>>(src, snd, d.lxi, d.let, n, ip, F, nm->cf);
                CSB_CUDA(cudaGetLastError());
            }
        }
    return CS_OK;
}

int cs_halo_exchange_self(cs_numerics *nm, unsigned var, void *stream) {
    if (!nm || var >= 5) return set_error(CS_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    for (int nn = 0; nn < 3; ++nn) {
        if (nm->ndf[0][nn] != nm->ndf[1][nn])
            return set_error(CS_ERR_UNSUPPORTED,
                             "axis %d has one interface face: a single rank has no neighbour for it", nn);
        if (nm->ndf[0][nn] != 1) continue;
        const int64_t F = face_size(nm->d, nn);
        double *snd = nm->send[nn] + (int64_t)var * 4 * F;
        double *rcv = nm->recv[nn] + (int64_t)var * 4 * F;
        // face 0 receives face 1's sums, face 1 receives face 0's
        // (tag pairing of src/numerics_base.hpp:161-176).
        CSB_CUDA(cudaMemcpyAsync(rcv, snd + 2 * F, 2 * F * sizeof(double), cudaMemcpyDeviceToDevice, st));
        CSB_CUDA(cudaMemcpyAsync(rcv + 2 * F, snd, 2 * F * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    return CS_OK;
}

int cs_filter(cs_numerics *nm, int axis, const double *in, double *out, double alpha_f, cs_dcomp d,
              void *stream) {
    if (!nm || !in || !out) return set_error(CS_ERR_INVALID, "null argument");
    if (int rc = check_dims(d)) return rc;
    if (!same_dims(d, nm->d)) return set_error(CS_ERR_INVALID, "dims differ from the numerics object");
    if (axis < 0 || axis > 2) return set_error(CS_ERR_INVALID, "axis %d", axis);
    if (nm->ndf[0][axis] != nm->ndf[1][axis])
        return set_error(CS_ERR_UNSUPPORTED, "filter needs both faces periodic or both physical");
    if (!(alpha_f > -0.5 && alpha_f <= 0.5)) return set_error(CS_ERR_INVALID, "alpha_f %g", alpha_f);
    const int n = line_len(d, axis);
    if (n < 7) return set_error(CS_ERR_UNSUPPORTED, "filter needs n >= 7");
    const DeviceTables *dt = nm->tables.get(n, kFilter, nm->ndf[0][axis], nm->ndf[1][axis], alpha_f);
    if (!dt) return CS_ERR_UNSUPPORTED;
    cudaStream_t st = (cudaStream_t)stream;
    switch (axis) {
        case 0: return launch_filter_axis<0>(dt->lt, in, out, dt->t64, d, alpha_f, st);
        case 1: return launch_filter_axis<1>(dt->lt, in, out, dt->t64, d, alpha_f, st);
        default: return launch_filter_axis<2>(dt->lt, in, out, dt->t64, d, alpha_f, st);
    }
}

int cs_line_tables(int n, int scheme, int nstart, int nend, double alpha_f, int meta[7],
                   double *tables, size_t tables_len) {
    if (!meta) return set_error(CS_ERR_INVALID, "null meta");
    HostTables h;
    if (!host_tables_for(n, scheme, nstart, nend, alpha_f, h))
        return set_error(CS_ERR_UNSUPPORTED, "line length %d", n);
    meta[0] = h.n; meta[1] = h.lt; meta[2] = h.p; meta[3] = h.last_len; meta[4] = h.cyclic;
    meta[5] = h.pcr64; meta[6] = h.pcr32;
    if (tables) {
        std::vector<double> v = pack(h);
        v.push_back(h.cyc_s1);
        v.push_back(h.cyc_s2);
        if (tables_len < v.size()) return set_error(CS_ERR_INVALID, "tables buffer too small (%zu)", v.size());
        std::memcpy(tables, v.data(), v.size() * sizeof(double));
    }
    return CS_OK;
}

}  // extern "C"
