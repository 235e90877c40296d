/* C entry points to the reference's CPU twins, compiled from the reference
 * test sources by oracle/Makefile (target `ref`):
 *   calc_fluxes_pre_compute_cpu  tests/test_physics_serial.cu:41-163
 *   calc_time_step_cpu           tests/test_physics.cu:57-117
 * Both are float-typed in the reference.  The two test files define the
 * same non-inline helpers, so each twin goes into its own library. */
#include "common/data_types.hpp"

#ifdef TWIN_FLUX
void calc_fluxes_pre_compute_cpu(float *buffer, float *qa, float *pressure, float *de, float *xim,
                                 float *etm, float *zem, t_stress_tensor<float> *stress_tensor,
                                 t_heat_fluxes<float> *heat_fluxes, t_point<float> umf,
                                 unsigned int size);
#endif
#ifdef TWIN_DT
float calc_time_step_cpu(float *xim, float *etm, float *zem, float *de, float *yaco, float *ssk,
                         t_point<float> umf, float cfl, unsigned int size);
#endif

#ifdef TWIN_FLUX
extern "C" void ref_fluxes_pre_cpu(float *buffer, float *qa, float *p, float *de, float *xim,
                                   float *etm, float *zem, float *tau6, float *heat3,
                                   const float umf[3], unsigned n) {
    t_stress_tensor<float> st{tau6, tau6 + n, tau6 + 2 * n, tau6 + 3 * n, tau6 + 4 * n, tau6 + 5 * n};
    t_heat_fluxes<float> hf{heat3, heat3 + n, heat3 + 2 * n};
    t_point<float> u{umf[0], umf[1], umf[2]};
    calc_fluxes_pre_compute_cpu(buffer, qa, p, de, xim, etm, zem, &st, &hf, u, n);
}
#endif

#ifdef TWIN_DT
extern "C" float ref_time_step_cpu(float *xim, float *etm, float *zem, float *de, float *yaco,
                                   float *ssk, const float umf[3], float cfl, unsigned n) {
    t_point<float> u{umf[0], umf[1], umf[2]};
    return calc_time_step_cpu(xim, etm, zem, de, yaco, ssk, u, cfl, n);
}
#endif
