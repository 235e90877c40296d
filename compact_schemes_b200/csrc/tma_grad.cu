// tma_grad.cu -- host side of the TMA-staged gradient pass: copy geometry and
// the tensor map of the state (cuTensorMapEncodeTiled through the runtime's
// driver entry point, so the library needs no link against libcuda).
#include <cudaTypedefs.h>

#include <mutex>

#include "tma_grad.cuh"

namespace csb {

bool tma_grad_geometry(int axis, const cs_dcomp &d, int lt, int smem_max, TmaGeom &g, size_t &smem_bytes) {
    const int n = axis == 0 ? d.lxi : (axis == 1 ? d.let : d.lze);
    if (n > 512 || lt > 16) return false;
    const int tl = kTmaTile;
    // row strides of the tensor maps are multiples of 16 bytes
    if (axis < 2 ? (d.lxi % 2) : (((int64_t)d.lxi * d.let) % 2)) return false;
    g.nbox = n > 256 ? 2 : 1;
    const int per = (n + g.nbox - 1) / g.nbox;
    g.boxlen = (per + 3) / 4 * 4;  // boxes of 5 x 4 x boxlen doubles: 128-byte aligned in shared memory
    if (g.boxlen > 256) return false;
    const int64_t F = axis == 0 ? (int64_t)d.let * d.lze : (axis == 1 ? (int64_t)d.lxi * d.lze : (int64_t)d.lxi * d.let);
    g.tiles_x = (d.lxi + tl - 1) / tl;
    const int64_t nt = axis == 1 ? (int64_t)g.tiles_x * d.lze : (F + tl - 1) / tl;
    if (nt > (1 << 30)) return false;
    g.ntiles = (int)nt;
    const size_t stage = (size_t)g.nbox * 5 * tl * g.boxlen * sizeof(double);
    g.tile_bytes = (unsigned)stage;
    const size_t slot = (size_t)32 * lt + 1;
    // two staging buffers, the line-solver layout of 4 fields, two mbarriers,
    // and up to 128 bytes to align the staging buffers
    smem_bytes = 2 * stage + (size_t)4 * tl * slot * sizeof(double) + 2 * sizeof(uint64_t) + 128;
    return smem_bytes <= (size_t)smem_max;
}

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Tensor map over nf consecutive fields of E-byte elements (FP64 or FP32).
static int field_map(int axis, const cs_dcomp &d, int tl, int boxlen, int nf, const void *base, cuuint64_t E,
                     CUtensorMap &map) {
    auto fn = encode_fn();
    if (!fn) return set_error(CS_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    if (reinterpret_cast<uintptr_t>(base) % 16) return set_error(CS_ERR_INVALID, "TMA pass: field block not 16-byte aligned");
    const cuuint64_t lmx = (cuuint64_t)d.lmx;
    cuuint64_t dims[4], strides[3];
    cuuint32_t box[4], estr[4] = {1, 1, 1, 1};
    cuuint32_t rank;
    if (axis == 0) {
        rank = 3;
        dims[0] = d.lxi; dims[1] = (cuuint64_t)d.let * d.lze; dims[2] = nf;
        strides[0] = d.lxi * E; strides[1] = lmx * E;
        box[0] = boxlen; box[1] = tl; box[2] = nf;
    } else if (axis == 1) {
        rank = 4;
        dims[0] = d.lxi; dims[1] = d.let; dims[2] = d.lze; dims[3] = nf;
        strides[0] = d.lxi * E; strides[1] = (cuuint64_t)d.lxi * d.let * E; strides[2] = lmx * E;
        box[0] = tl; box[1] = boxlen; box[2] = 1; box[3] = nf;
    } else {
        rank = 3;
        dims[0] = (cuuint64_t)d.lxi * d.let; dims[1] = d.lze; dims[2] = nf;
        strides[0] = (cuuint64_t)d.lxi * d.let * E; strides[1] = lmx * E;
        box[0] = tl; box[1] = boxlen; box[2] = nf;
    }
    CUresult r = fn(&map, E == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank,
                    const_cast<void *>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(CS_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return CS_OK;
}

int tma_field_map(int axis, const cs_dcomp &d, int tl, int boxlen, int nf, const double *base, CUtensorMap &map) {
    return field_map(axis, d, tl, boxlen, nf, base, sizeof(double), map);
}

int tma_field_map32(int axis, const cs_dcomp &d, int tl, int boxlen, int nf, const float *base, CUtensorMap &map) {
    return field_map(axis, d, tl, boxlen, nf, base, sizeof(float), map);
}

bool tma_grad_mx_geometry(int axis, const cs_dcomp &d, int lt, int smem_max, TmaGeom &g, size_t &smem_bytes) {
    const int n = axis == 0 ? d.lxi : (axis == 1 ? d.let : d.lze);
    if (n > 512 || lt > 16) return false;
    const int tl = lt <= 8 ? 8 : 4;
    // FP32 rows: strides and the field offset (the map starts at field 1 of
    // the shadow) are multiples of 16 bytes
    if (d.lmx % 4 || (axis < 2 ? (d.lxi % 4) : (((int64_t)d.lxi * d.let) % 4))) return false;
    g.nbox = n > 256 ? 2 : 1;
    const int per = (n + g.nbox - 1) / g.nbox;
    g.boxlen = (per + 3) / 4 * 4;
    if (g.boxlen > 256) return false;
    const int64_t F = axis == 0 ? (int64_t)d.let * d.lze : (axis == 1 ? (int64_t)d.lxi * d.lze : (int64_t)d.lxi * d.let);
    g.tiles_x = (d.lxi + tl - 1) / tl;
    const int64_t nt = axis == 1 ? (int64_t)g.tiles_x * d.lze : (F + tl - 1) / tl;
    if (nt > (1 << 30)) return false;
    g.ntiles = (int)nt;
    const size_t stage = (size_t)g.nbox * 4 * tl * g.boxlen * sizeof(float);
    g.tile_bytes = (unsigned)stage;
    const size_t slot = (size_t)32 * lt + 1;
    smem_bytes = 2 * stage + (size_t)4 * tl * slot * sizeof(float) + 2 * sizeof(uint64_t) + 128;
    return smem_bytes <= (size_t)smem_max;
}

int tma_grad_map(int axis, const cs_dcomp &d, const TmaGeom &g, const double *q, CUtensorMap &map) {
    return tma_field_map(axis, d, kTmaTile, g.boxlen, 5, q, map);
}

}  // namespace csb
