// fused_axis0.cu -- instantiation of the fused passes along axis 0 (one
// translation unit per axis keeps the build parallel).
#include "fused_kernels.cuh"

namespace csb {

template <>
int launch_grad<0>(const PassArgs &a, const double *q, bool dtred, cudaStream_t st) {
    if (a.pl) return launch_grad_pl<0>(a, q, dtred, st);
    return launch_grad_tl<0, 8>(a, q, dtred, st);
}

template <>
int launch_flux<0>(const PassArgs &a, int mode, const double *q, const double *qn, double *qout,
                   double *drva, const RkParams &rk, cudaStream_t st) {
    if (a.pl) return launch_flux_pl<0>(a, mode, q, qn, qout, drva, rk, st);
    return launch_flux_tl<0, 8>(a, mode, q, qn, qout, drva, rk, st);
}

}  // namespace csb
