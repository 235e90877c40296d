// tma_grad_mx_axis1.cu -- TMA-staged gradient pass of the mixed form along
// axis 1 (one translation unit per axis keeps the build parallel).
#include "tma_grad_mx.cuh"

namespace csb {

template <>
int launch_grad_mx_tma<1>(const MixedArgs &m, const cs_dcomp &d, int *err, cudaStream_t st) {
    return launch_grad_mx_tma_impl<1>(m, d, err, st);
}

}  // namespace csb
