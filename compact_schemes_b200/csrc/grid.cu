// grid.cu -- metrics and Jacobian of a curvilinear grid.
//
// The reference's grid class generates coordinates only (grid::generate,
// src/grid.hpp:89-213); the metric arrays its physics kernels read
// (xim, etm, zem = J^-1 grad(xi_a), yaco = J; calc_fluxes_pre_compute_kernel,
// src/cuda/kernels/physics.hpp:42-193) have no generator there.  This file
// fills them with the same compact derivative as the flow solver, in the
// cross-product form
//   xim = r_eta x r_zeta,  etm = r_zeta x r_xi,  zem = r_xi x r_eta,
//   yaco = 1 / (r_xi . xim),
// r_a = d(x, y, z)/d xi_a in index space.  On an axis with interface
// closures (periodic) each coordinate is a periodic part plus a ramp,
// c = c~ + i_a * s with s = period[a][c] / n_a, and r_a = D c~ + s.
#include <cuda_runtime.h>

#include "context.h"
#include "line_solver.cuh"

namespace csb {

// tmp = c - i_a * s: the periodic part of one coordinate along axis a.
__global__ void k_grid_ramp(const double *__restrict__ c, double *__restrict__ tmp, int lxi, int let,
                            int64_t lmx, int axis, double s) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= lmx) return;
    const int64_t ia = axis == 0 ? i % lxi : (axis == 1 ? (i / lxi) % let : i / ((int64_t)lxi * let));
    tmp[i] = c[i] - xmul((double)ia, s);
}

// d: [3 axes][3 coordinates][lmx] derivatives of the periodic parts;
// sl: the ramp slopes in the same order.
struct Slopes {
    double s[9];
};

__global__ void k_grid_metrics(const double *__restrict__ d, Slopes sl, double *__restrict__ xim,
                               double *__restrict__ etm, double *__restrict__ zem, double *__restrict__ yaco,
                               int64_t lmx, int *__restrict__ bad) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= lmx) return;
    double r[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int c = 0; c < 3; ++c) r[a][c] = d[(int64_t)(a * 3 + c) * lmx + i] + sl.s[a * 3 + c];
    double *out[3] = {xim, etm, zem};
    double x0 = 0.0, x1 = 0.0, x2 = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double *p = r[(a + 1) % 3], *q = r[(a + 2) % 3];
        const double m0 = xmul(p[1], q[2]) - xmul(p[2], q[1]);
        const double m1 = xmul(p[2], q[0]) - xmul(p[0], q[2]);
        const double m2 = xmul(p[0], q[1]) - xmul(p[1], q[0]);
        out[a][i] = m0;
        out[a][lmx + i] = m1;
        out[a][2 * lmx + i] = m2;
        if (a == 0) { x0 = m0; x1 = m1; x2 = m2; }
    }
    const double vol = xmul(r[0][0], x0) + xmul(r[0][1], x1) + xmul(r[0][2], x2);
    if (!(vol != 0.0)) atomicOr(bad, 1);
    yaco[i] = 1.0 / vol;
}

// CS_OK, or the CUDA error recorded as the library's last error.
static int cuda_status(cudaError_t e, const char *what) { return e == cudaSuccess ? CS_OK : check_cuda(e, what); }

}  // namespace csb

using namespace csb;

extern "C" int cs_grid_metrics(cs_numerics *nm, const double *xyz, const double period[3][3], double *xim,
                               double *etm, double *zem, double *yaco, void *stream) {
    if (!nm || !xyz || !xim || !etm || !zem || !yaco) return set_error(CS_ERR_INVALID, "null argument");
    if (!nm->setup_done) return set_error(CS_ERR_STATE, "cs_grid_metrics before cs_deriv_setup");
    const cs_dcomp d = nm->d;
    const int dims[3] = {d.lxi, d.let, d.lze};
    for (int a = 0; a < 3; ++a)
        if (dims[a] < 5) return set_error(CS_ERR_UNSUPPORTED, "metrics need every axis of >= 5 points");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t lmx = d.lmx;
    double *scratch = nullptr;
    int *bad = nullptr;
    if (cudaMallocAsync(&scratch, (size_t)10 * lmx * sizeof(double), st) != cudaSuccess ||
        cudaMallocAsync(&bad, sizeof(int), st) != cudaSuccess) {
        if (scratch) cudaFreeAsync(scratch, st);
        return set_error(CS_ERR_ALLOC, "grid metrics scratch allocation failed");
    }
    double *tmp = scratch + 9 * lmx;
    Slopes sl{};
    const unsigned blocks = (unsigned)((lmx + 255) / 256);
    int rc = cuda_status(cudaMemsetAsync(bad, 0, sizeof(int), st), "cudaMemsetAsync");
    for (int a = 0; a < 3 && rc == CS_OK; ++a) {
        const int nstart = nm->ndf[0][a], nend = nm->ndf[1][a];
        const bool ramp = nstart || nend;
        for (int c = 0; c < 3 && rc == CS_OK; ++c) {
            const double s = ramp && period ? period[a][c] / dims[a] : 0.0;
            sl.s[a * 3 + c] = s;
            k_grid_ramp<<<blocks, 256, 0, st>>>(xyz + c * lmx, tmp, d.lxi, d.let, lmx, a, s);
            rc = cuda_status(cudaGetLastError(), "k_grid_ramp");
            if (rc == CS_OK)
                rc = cs_deriv(nm, a, tmp, scratch + (int64_t)(a * 3 + c) * lmx, nstart, nend, d, 0, 0, 0,
                              CS_HALO_SELF, stream);
        }
    }
    int hbad = 0;
    if (rc == CS_OK) {
        k_grid_metrics<<<blocks, 256, 0, st>>>(scratch, sl, xim, etm, zem, yaco, lmx, bad);
        rc = cuda_status(cudaGetLastError(), "k_grid_metrics");
    }
    if (rc == CS_OK) rc = cuda_status(cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st),
                                     "cudaMemcpyAsync");
    cudaFreeAsync(scratch, st);
    cudaFreeAsync(bad, st);
    if (rc == CS_OK) rc = cuda_status(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    if (rc == CS_OK && hbad) rc = set_error(CS_ERR_INVALID, "grid has a cell of zero volume");
    return rc;
}
