// pipeline_mixed_axis0.cu -- mixed-precision producer/consumer passes along axis 0.
#include "pipeline.cuh"

namespace csb {

template <>
int launch_grad_mx_pl<0>(const MixedArgs &m, const double *q, bool first, cudaStream_t st) {
    return launch_grad_mx_pl_impl<0>(m, q, first, st);
}

template <>
int launch_flux_mx_pl<0>(const MixedArgs &m, int mode, const double *qn, double *qout, bool shadow_out,
                          double *drva, const RkParams &rk, cudaStream_t st) {
    return launch_flux_mx_pl_impl<0>(m, mode, qn, qout, shadow_out, drva, rk, st);
}

}  // namespace csb
