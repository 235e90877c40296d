// tma_grad_axis1.cu -- TMA-staged gradient pass along axis 1 (one
// translation unit per axis keeps the build parallel).
#include "tma_grad.cuh"

namespace csb {

template <>
int launch_grad_tma<1>(const PassArgs &a, const cs_dcomp &d, const double *q, bool dtred, int *err,
                        cudaStream_t st) {
    return launch_grad_tma_impl<1>(a, d, q, dtred, err, st);
}

}  // namespace csb
