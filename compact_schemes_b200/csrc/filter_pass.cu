// filter_pass.cu -- the compact filter applied to the solver's conserved
// state inside the time step: one pass per axis filters all five fields of a
// tile of full lines in place (stage the lines in shared memory, solve the
// sixth-order tridiagonal filter for each field, store back), 80 bytes per
// point per pass.  The filter is the one of cs_filter (filter_rhs and the
// kFilter line tables: cyclic on periodic axes, reduced-order closures on
// physical faces); the reference names the filter but has no code for it
// (README.md:5-8).
#include "fused_kernels.cuh"

namespace csb {

template <int LT, int AXIS, int TL>
__global__ void __launch_bounds__(TL * 32, TL == 8 ? 2 : 1)
k_filter_state(double *__restrict__ q, DevTables<double> tab, int lxi, int let, int64_t lmx, int64_t F,
               double af) {
    using L = LineLayout<LT>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sm = reinterpret_cast<double *>(smem_raw);
    const int n = tab.n;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t line0 = (int64_t)blockIdx.x * TL;
    tile_for_each<AXIS, TL, 2>(line0, F, n, lxi, let, [&](int l, int j, int64_t gi) {
        const int pj = L::pos(j);
#pragma unroll
        for (int m = 0; m < 5; ++m) field_line<LT, TL>(sm, m, l)[pj] = q[m * lmx + gi];
    });
    tile_sync<AXIS, TL>();
    if (line0 + w < F) {
        constexpr int G = LT >= 16 ? 1 : 2;
#pragma unroll 1
        for (int c0 = 0; c0 < 5; c0 += G) {
            double d[G][LT];
#pragma unroll
            for (int g = 0; g < G; ++g) {
                if (c0 + g < 5) filter_rhs<LT, double, double>(field_line<LT, TL>(sm, c0 + g, w), n, lane,
                                                               tab.cyclic != 0, af, d[g]);
                else {
#pragma unroll
                    for (int t = 0; t < LT; ++t) d[g][t] = 0.0;
                }
            }
            warp_solve<LT, G, double>(tab, d, lane);
            __syncwarp();
#pragma unroll
            for (int g = 0; g < G; ++g) {
                if (c0 + g >= 5) continue;
                double *ln = field_line<LT, TL>(sm, c0 + g, w);
#pragma unroll
                for (int t = 0; t < LT; ++t)
                    if (lane * LT + t < n) ln[L::pos_ct(lane, t)] = d[g][t];
            }
        }
    }
    tile_sync<AXIS, TL>();
    tile_for_each<AXIS, TL, 2>(line0, F, n, lxi, let, [&](int l, int j, int64_t gi) {
        const int pj = L::pos(j);
#pragma unroll
        for (int m = 0; m < 5; ++m) q[m * lmx + gi] = field_line<LT, TL>(sm, m, l)[pj];
    });
}

template <int LT, int AXIS>
static int launch_filter_state_t(double *q, const DeviceTables &t, const cs_dcomp &d, int64_t F, double af,
                                 cudaStream_t st) {
    constexpr int TL = 8;
    const size_t smem = (size_t)5 * TL * LineLayout<LT>::kSlot * sizeof(double);
    auto kern = k_filter_state<LT, AXIS, TL>;
    if (int rc = set_smem(kern, smem)) return rc;
    kern<<<(unsigned)((F + TL - 1) / TL), TL * 32, smem, st>>>(q, t.t64, d.lxi, d.let, d.lmx, F, af);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

template <int AXIS>
static int launch_filter_state_axis(double *q, const DeviceTables &t, const cs_dcomp &d, int64_t F, double af,
                                    cudaStream_t st) {
    switch (t.lt) {
        case 2: return launch_filter_state_t<2, AXIS>(q, t, d, F, af, st);
        case 4: return launch_filter_state_t<4, AXIS>(q, t, d, F, af, st);
        case 8: return launch_filter_state_t<8, AXIS>(q, t, d, F, af, st);
        case 16: return launch_filter_state_t<16, AXIS>(q, t, d, F, af, st);
    }
    return set_error(CS_ERR_UNSUPPORTED, "filter: chunk length %d", t.lt);
}

int filter_state(double *q, int axis, const DeviceTables &t, const cs_dcomp &d, double af, cudaStream_t st) {
    const int64_t F = axis == 0 ? (int64_t)d.let * d.lze : (axis == 1 ? (int64_t)d.lxi * d.lze
                                                                       : (int64_t)d.lxi * d.let);
    if (axis == 0) return launch_filter_state_axis<0>(q, t, d, F, af, st);
    if (axis == 1) return launch_filter_state_axis<1>(q, t, d, F, af, st);
    return launch_filter_state_axis<2>(q, t, d, F, af, st);
}

}  // namespace csb
