// tma_grad_axis0.cu -- TMA-staged gradient pass along axis 0 (one
// translation unit per axis keeps the build parallel).
#include "tma_grad.cuh"

namespace csb {

template <>
int launch_grad_tma<0>(const PassArgs &a, const cs_dcomp &d, const double *q, bool dtred, int *err,
                        cudaStream_t st) {
    return launch_grad_tma_impl<0>(a, d, q, dtred, err, st);
}

}  // namespace csb
