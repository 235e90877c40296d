// fused_mixed_axis1.cu -- instantiation of the mixed-precision passes along
// axis 1 (tiles of 8 lines; 8 or 16 along z).
#include "fused_mixed.cuh"

namespace csb {

template <>
int launch_grad_mx<1>(const MixedArgs &a, const double *q, bool first, cudaStream_t st) {
    if (a.base.pl) return launch_grad_mx_pl<1>(a, q, first, st);
    return launch_grad_mx_tl<1, 8>(a, q, first, st);
}

template <>
int launch_flux_mx<1>(const MixedArgs &a, int mode, const double *qn, double *qout, bool shadow_out,
                      double *drva, const RkParams &rk, cudaStream_t st) {
    if (a.base.pl) return launch_flux_mx_pl<1>(a, mode, qn, qout, shadow_out, drva, rk, st);
    return launch_flux_mx_tl<1, 8>(a, mode, qn, qout, shadow_out, drva, rk, st);
}

}  // namespace csb
