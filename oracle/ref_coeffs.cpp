/* Pin for the oracle's coefficient setup: runs the reference's own
 * numerics_base<double>::deriv_setup (src/numerics_base.hpp:182-297),
 * compiled from its sources by oracle/Makefile (target `ref`), on the host.
 * CUDA allocation/copy calls of that header are served from host memory. */
#include <cstdlib>
#include <cstring>
#include <cuda_runtime.h>

extern "C" {
cudaError_t cudaMalloc(void **p, size_t n) { *p = std::malloc(n); return cudaSuccess; }
cudaError_t cudaFree(void *p) { std::free(p); return cudaSuccess; }
cudaError_t cudaMemcpy(void *d, const void *s, size_t n, cudaMemcpyKind) { std::memcpy(d, s, n); return cudaSuccess; }
const char *cudaGetErrorString(cudaError_t) { return "host stand-in"; }
}

#include "host/functional.hpp"
#include "numerics_base.hpp"

extern "C" void ref_deriv_setup(double pbco[16], double pbci[16]) {
    t_dcomp d{8 * 8 * 8, 8, 8, 8};
    int nbc[2][3];
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 3; ++a) nbc[f][a] = BC_PERIODIC;
    numerics_base<double> nb(d, nbc);
    nb.deriv_setup();
    std::memcpy(pbco, nb.pbco, 16 * sizeof(double));
    std::memcpy(pbci, nb.pbci, 16 * sizeof(double));
}
