// pipeline_axis1.cu -- FP64 producer/consumer passes along axis 1.
#include "pipeline.cuh"

namespace csb {

template <>
int launch_grad_pl<1>(const PassArgs &a, const double *q, bool dtred, cudaStream_t st) {
    return launch_grad_pl_impl<1>(a, q, dtred, st);
}

template <>
int launch_flux_pl<1>(const PassArgs &a, int mode, const double *q, const double *qn, double *qout,
                       double *drva, const RkParams &rk, cudaStream_t st) {
    return launch_flux_pl_impl<1>(a, mode, q, qn, qout, drva, rk, st);
}

}  // namespace csb
