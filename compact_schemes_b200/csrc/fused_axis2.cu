// fused_axis2.cu -- instantiation of the fused passes along axis 2 (one
// translation unit per axis keeps the build parallel).
#include "fused_kernels.cuh"

namespace csb {

template <>
int launch_grad<2>(const PassArgs &a, const double *q, bool dtred, cudaStream_t st) {
    if (a.pl) return launch_grad_pl<2>(a, q, dtred, st);
    if (a.tl == 16) return launch_grad_tl<2, 16>(a, q, dtred, st);
    return launch_grad_tl<2, 8>(a, q, dtred, st);
}

template <>
int launch_flux<2>(const PassArgs &a, int mode, const double *q, const double *qn, double *qout,
                   double *drva, const RkParams &rk, cudaStream_t st) {
    if (a.pl) return launch_flux_pl<2>(a, mode, q, qn, qout, drva, rk, st);
    if (a.tl == 16) return launch_flux_tl<2, 16>(a, mode, q, qn, qout, drva, rk, st);
    return launch_flux_tl<2, 8>(a, mode, q, qn, qout, drva, rk, st);
}

}  // namespace csb
