// compact_schemes/physics_pc.hpp -- drop-in physics<EnableViscous, Type>
// (src/physics_pc.hpp, src/physics_base.hpp) over libcompact_b200, FP64.
// calc_viscous_shear_stress computes the chain rule on the derivatives and
// uses each axis' own face flags (the reference passes the underived buffer
// and swaps the flags of axes 0 and 2).
#pragma once

#include "numerics_pc.hpp"

template <typename Type>
struct t_stress_tensor {
    Type *xx, *yy, *zz, *xy, *yz, *zx;
};
template <typename Type>
struct t_heat_fluxes {
    Type *xx, *yy, *zz;
};

template <bool EnableViscous, typename Type>
struct physics {
    // The reference driver instantiates physics<true, float>; this drop-in path
    // computes the fluxes, stresses, time step and RHS in FP64 only: the
    // hot path's parity bar is FP64 (1e-12 against the host path), and the
    // library's FP32 arithmetic lives in the fused mixed-precision step
    // (CS_PREC_MIXED) and in numerics_pc<float>::deriv1d/deriv2d.
    static_assert(std::is_same<Type, double>::value,
                  "physics<Visc, Type>: the drop-in physics path is FP64 (use double; FP32 runs in the fused "
                  "solver's CS_PREC_MIXED form and numerics_pc<float> derivatives)");

    explicit physics(t_dcomp dcomp_info) : d(dcomp_info) {
        compact_b200::check(cs_physics_create(&handle, compact_b200::to_c(d), EnableViscous ? 1 : 0),
                            "physics");
        double *tau, *heat;
        compact_b200::check(cs_physics_buffers(handle, &buffer, &buffer_deriv, &tau, &heat),
                            "cs_physics_buffers");
        const size_t n = (size_t)d.lmx;
        stress_tensor = {tau, tau + n, tau + 2 * n, tau + 3 * n, tau + 4 * n, tau + 5 * n};
        heat_fluxes = {heat, heat + n, heat + 2 * n};
    }
    ~physics() { cs_physics_destroy(handle); }
    physics(const physics &) = delete;
    physics &operator=(const physics &) = delete;

    void init() {}  // empty in the reference (src/physics_pc.hpp:78-81)

    // physics::calc_fluxes (src/physics_pc.hpp:83-149).
    void calc_fluxes(Type *qa, Type *pressure, Type *de, Type *xim, Type *etm, Type *zem,
                     t_dcomp dcomp_info, int mcd[2][3], numerics_pc<Type> *numerics_instance,
                     cudaStream_t *streams) {
        (void)mcd;
        sync_umf();
        cudaStream_t st = streams ? streams[0] : nullptr;
        compact_b200::check(cs_calc_fluxes(handle, numerics_instance->handle, qa, pressure, de, xim, etm,
                                           zem, compact_b200::to_c(dcomp_info), st),
                            "calc_fluxes");
        cudaStreamSynchronize(st);
    }

    // physics::calc_viscous_shear_stress (src/physics_pc.hpp:151-227).
    void calc_viscous_shear_stress(Type *de, Type *ssk, Type *xim, Type *etm, Type *zem, Type *yaco,
                                   t_dcomp dcomp_info, int mcd[2][3],
                                   numerics_pc<Type> *numerics_instance, cudaStream_t *streams) {
        (void)mcd;
        cudaStream_t st = streams ? streams[0] : nullptr;
        compact_b200::check(cs_calc_viscous_shear_stress(handle, numerics_instance->handle, de, ssk, xim,
                                                         etm, zem, yaco, compact_b200::to_c(dcomp_info), st),
                            "calc_viscous_shear_stress");
        cudaStreamSynchronize(st);
    }

    // physics::calc_time_step (src/physics_pc.hpp:229-256).
    void calc_time_step(Type *xim, Type *etm, Type *zem, Type *de, Type *yaco, Type *ssk, Type cfl,
                        Type *dte, unsigned int size) {
        sync_umf();
        compact_b200::check(cs_calc_time_step(handle, xim, etm, zem, de, yaco, ssk, cfl, dte, size, nullptr),
                            "calc_time_step");
    }

    // Empty in the reference (src/physics_base.hpp:147-150); the conserved
    // update is cs_rk_update / compact_b200::rk_update below.
    void movef(Type, Type, Type) {}

    cs_physics *handle = nullptr;
    t_dcomp d;
    Type *buffer = nullptr;
    Type *buffer_deriv = nullptr;
    t_stress_tensor<Type> stress_tensor;  // host struct of device pointers
    t_heat_fluxes<Type> heat_fluxes;
    t_point<Type> umf{0, 0, 0};
    t_point<Type> dudtmf{0, 0, 0};

private:
    void sync_umf() {
        const double u[3] = {umf.x, umf.y, umf.z};
        compact_b200::check(cs_physics_set_umf(handle, u), "umf");
    }
};

template <bool EnableViscous, typename Type>
using physics_rtc = physics<EnableViscous, Type>;

namespace compact_b200 {
// q <- q^n - dtk * J * de, the update physics_base::movef leaves empty.
inline void rk_update(const double *qn, const double *de, const double *yaco, double dtk, double *qout,
                      size_t lmx, cudaStream_t st = nullptr) {
    check(cs_rk_update(qn, de, yaco, dtk, qout, lmx, st), "rk_update");
}
// Primitive recovery (the empty slot of driver/canard.cu:142-143).
inline void thermo(const double *q, double *de, double *p, size_t lmx, cudaStream_t st = nullptr) {
    check(cs_thermo(q, de, p, lmx, st), "thermo");
}
}  // namespace compact_b200
