// tma_grad_mx_axis0.cu -- TMA-staged gradient pass of the mixed form along
// axis 0 (one translation unit per axis keeps the build parallel).
#include "tma_grad_mx.cuh"

namespace csb {

template <>
int launch_grad_mx_tma<0>(const MixedArgs &m, const cs_dcomp &d, int *err, cudaStream_t st) {
    return launch_grad_mx_tma_impl<0>(m, d, err, st);
}

}  // namespace csb
