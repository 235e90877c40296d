// context.h -- host-side objects behind the opaque C-ABI handles.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <tuple>

#include "cs_common.h"
#include "line_solver.cuh"

namespace csb {

int set_error(int code, const char *fmt, ...);
int check_cuda(cudaError_t e, const char *what);

#define CSB_CUDA(call)                                      \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) return check_cuda(e_, #call); \
    } while (0)

// Device copy of the tables of one line configuration, in FP64 and FP32.
struct DeviceTables {
    HostTables host;
    double *d64 = nullptr;
    float *d32 = nullptr;
    DevTables<double> t64{};
    DevTables<float> t32{};
    int lt = 0;
    // every lane's chunk shares lane 0's per-row factors (full chunks, the
    // constant interior rows only: ChunkFactors); cfu holds them in FP32 as
    // [f1, f2, b1, b2, -rca, -rcc][lt]
    bool uniform = false;
    float cfu[6 * 32] = {};
};

// key: n, scheme, nstart, nend, alpha_f bits
using TableKey = std::tuple<int, int, int, int, uint64_t, int>;

// Cache of device tables (one per device/line configuration).
class TableCache {
public:
    ~TableCache();
    // Returns nullptr and sets the error on failure.  min_lt: shortest chunk
    // of the tables (build_tables).
    const DeviceTables *get(int n, int scheme, int nstart, int nend, double alpha_f, int min_lt = 2);

private:
    std::mutex mu_;
    std::map<TableKey, DeviceTables *> map_;
};

}  // namespace csb

struct cs_numerics {
    cs_dcomp d{};
    int nbc[2][3]{};
    int ndf[2][3]{};
    csb::Coeffs cf{};
    bool setup_done = false;
    double *drva[3] = {nullptr, nullptr, nullptr};
    double *send[3] = {nullptr, nullptr, nullptr};
    double *recv[3] = {nullptr, nullptr, nullptr};
    csb::TableCache tables;
};
