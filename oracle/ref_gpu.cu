/* C entry points that launch the reference's own precompiled ("pc") CUDA
 * kernels, compiled for sm_100a from the reference sources by
 * oracle/Makefile (target `ref`).  Test infrastructure: GPU-side parity pins
 * and the reference kernel timings.  Launch shapes follow
 * numerics_pc::deriv2d (src/numerics_pc.hpp:121-168),
 * gpu_buffer::fill (src/cuda/numerics_pc.hpp:39-80) and
 * calc_fluxes_pre_compute (src/cuda/physics.hpp:41-62). */
#include <cstdint>
#include "host/functional.hpp"
#include "cuda/kernels/numerics_pc.hpp"
#include "cuda/kernels/physics.hpp"

extern "C" int ref_gpu_deriv2d(int axis, double *in, double *out, double *recv, double *pbci,
                               double *drva, int nstart, int nend, int lxi, int let, int lze,
                               unsigned var, unsigned comp, void *stream) {
    t_dcomp d{lxi * let * lze, lxi, let, lze};
    cudaStream_t s = (cudaStream_t)stream;
    if (axis == 0) {
        deriv_kernel_2d<0, double><<<dim3(let, lze), lxi, 5 * lxi * sizeof(double), s>>>(
            in, out, recv, pbci, drva, nstart, nend, d, var, comp);
    } else if (axis == 1) {
        deriv_kernel_2d<1, double><<<dim3(lxi, lze), let, 5 * let * sizeof(double), s>>>(
            in, out, recv, pbci, drva, nstart, nend, d, var, comp);
    } else {
        deriv_kernel_2d<2, double><<<dim3(lxi, let), lze, 5 * lze * sizeof(double), s>>>(
            in, out, recv, pbci, drva, nstart, nend, d, var, comp);
    }
    return (int)cudaGetLastError();
}

extern "C" int ref_gpu_fill_buffer(int axis, double *in, double *send, double *pbco, int lxi,
                                   int let, int lze, int istart, int inc, int offset, void *stream) {
    t_dcomp d{lxi * let * lze, lxi, let, lze};
    cudaStream_t s = (cudaStream_t)stream;
    if (axis == 0) fill_gpu_buffer_kernel<0, double><<<lze, let, 0, s>>>(in, send, pbco, d, istart, inc, offset);
    else if (axis == 1) fill_gpu_buffer_kernel<1, double><<<lze, lxi, 0, s>>>(in, send, pbco, d, istart, inc, offset);
    else fill_gpu_buffer_kernel<2, double><<<let, lxi, 0, s>>>(in, send, pbco, d, istart, inc, offset);
    return (int)cudaGetLastError();
}

/* tau6/heat3: device arrays [6][n], [3][n]; the reference kernel wants
 * device-resident structs of pointers, built here in `structs` (device
 * memory of at least 9 pointers supplied by the caller). */
extern "C" int ref_gpu_fluxes_pre(double *buffer, double *qa, double *p, double *de, double *xim,
                                  double *etm, double *zem, double *tau6, double *heat3,
                                  double umfx, double umfy, double umfz, unsigned n, void *structs,
                                  void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    t_stress_tensor<double> st{tau6, tau6 + n, tau6 + 2 * (size_t)n, tau6 + 3 * (size_t)n,
                               tau6 + 4 * (size_t)n, tau6 + 5 * (size_t)n};
    t_heat_fluxes<double> hf{heat3, heat3 + n, heat3 + 2 * (size_t)n};
    auto *dst = (t_stress_tensor<double> *)structs;
    auto *dhf = (t_heat_fluxes<double> *)((char *)structs + sizeof(st));
    cudaMemcpyAsync(dst, &st, sizeof st, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dhf, &hf, sizeof hf, cudaMemcpyHostToDevice, s);
    t_point<double> umf{umfx, umfy, umfz};
    calc_fluxes_pre_compute_kernel<true, double><<<(n + 255) / 256, 256, 0, s>>>(
        buffer, qa, p, de, xim, etm, zem, dst, dhf, umf, n);
    cudaStreamSynchronize(s);
    return (int)cudaGetLastError();
}

/* Timing of the reference's flux pre-compute kernel: the stress / heat-flux
 * pointer structs are uploaded once, then `reps` launches on `stream` are
 * bracketed by CUDA events; *ms = average milliseconds per launch. */
extern "C" int ref_gpu_fluxes_pre_time(double *buffer, double *qa, double *p, double *de, double *xim,
                                       double *etm, double *zem, double *tau6, double *heat3, double umfx,
                                       double umfy, double umfz, unsigned n, void *structs, int reps,
                                       void *stream, float *ms) {
    cudaStream_t s = (cudaStream_t)stream;
    t_stress_tensor<double> st{tau6, tau6 + n, tau6 + 2 * (size_t)n, tau6 + 3 * (size_t)n,
                               tau6 + 4 * (size_t)n, tau6 + 5 * (size_t)n};
    t_heat_fluxes<double> hf{heat3, heat3 + n, heat3 + 2 * (size_t)n};
    auto *dst = (t_stress_tensor<double> *)structs;
    auto *dhf = (t_heat_fluxes<double> *)((char *)structs + sizeof(st));
    cudaMemcpyAsync(dst, &st, sizeof st, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dhf, &hf, sizeof hf, cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
    t_point<double> umf{umfx, umfy, umfz};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps; ++r)
        calc_fluxes_pre_compute_kernel<true, double><<<(n + 255) / 256, 256, 0, s>>>(
            buffer, qa, p, de, xim, etm, zem, dst, dhf, umf, n);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    *ms /= reps;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return (int)cudaGetLastError();
}
