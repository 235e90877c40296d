// ensemble_tl8.cu -- the ensemble's persistent stage kernel with 8-line work items.
#include "ensemble.cuh"

namespace csb {

int ens_launch_tl8(const EnsArgs &a, bool visc, int ctas_per_sm, int nsm, size_t smem, cudaStream_t st, int nbox) {
    return ens_launch_t<8>(a, visc, ctas_per_sm, nsm, smem, st, nbox);
}

}  // namespace csb
