// tma_grad_axis2.cu -- TMA-staged gradient pass along axis 2 (one
// translation unit per axis keeps the build parallel).
#include "tma_grad.cuh"

namespace csb {

template <>
int launch_grad_tma<2>(const PassArgs &a, const cs_dcomp &d, const double *q, bool dtred, int *err,
                        cudaStream_t st) {
    return launch_grad_tma_impl<2>(a, d, q, dtred, err, st);
}

}  // namespace csb
