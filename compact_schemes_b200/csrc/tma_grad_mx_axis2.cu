// tma_grad_mx_axis2.cu -- TMA-staged gradient pass of the mixed form along
// axis 2 (one translation unit per axis keeps the build parallel).
#include "tma_grad_mx.cuh"

namespace csb {

template <>
int launch_grad_mx_tma<2>(const MixedArgs &m, const cs_dcomp &d, int *err, cudaStream_t st) {
    return launch_grad_mx_tma_impl<2>(m, d, err, st);
}

}  // namespace csb
