// ensemble_tl4.cu -- the ensemble's persistent stage kernel with 4-line work items.
#include "ensemble.cuh"

namespace csb {

int ens_launch_tl4(const EnsArgs &a, bool visc, int ctas_per_sm, int nsm, size_t smem, cudaStream_t st, int nbox) {
    return ens_launch_t<4>(a, visc, ctas_per_sm, nsm, smem, st, nbox);
}

}  // namespace csb
