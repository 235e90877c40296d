"""ctypes signatures of include/compact_b200.h."""
import ctypes

vp = ctypes.c_void_p
i32 = ctypes.c_int
u32 = ctypes.c_uint
f64 = ctypes.c_double
sz = ctypes.c_size_t


def declare(L):
    from . import Dcomp
    pp = ctypes.POINTER(ctypes.c_void_p)
    L.cs_last_error.restype = ctypes.c_char_p
    L.cs_version.restype = i32
    L.cs_numerics_create.argtypes = [pp, Dcomp, vp]
    L.cs_numerics_destroy.argtypes = [vp]
    L.cs_deriv_setup.argtypes = [vp]
    L.cs_get_coeffs.argtypes = [vp, vp, vp]
    L.cs_interface_coeffs.argtypes = [vp, vp]
    L.cs_get_ndf.argtypes = [vp, vp]
    L.cs_get_buffers.argtypes = [vp, i32, pp, pp, pp]
    L.cs_deriv.argtypes = [vp, i32, vp, vp, i32, i32, Dcomp, u32, u32, u32, i32, vp]
    L.cs_deriv_noalloc.argtypes = [i32, vp, vp, i32, i32, Dcomp, vp]
    L.cs_deriv_noalloc.restype = i32
    L.cs_deriv_f32.argtypes = [vp, i32, vp, vp, i32, i32, Dcomp, u32, u32, u32, i32, vp]
    L.cs_fill_buffers.argtypes = [vp, vp, i32, i32, i32, Dcomp, vp]
    L.cs_halo_exchange_self.argtypes = [vp, u32, vp]
    L.cs_filter.argtypes = [vp, i32, vp, vp, f64, Dcomp, vp]
    L.cs_line_tables.argtypes = [i32, i32, i32, i32, f64, vp, vp, sz]
    L.cs_physics_create.argtypes = [pp, Dcomp, i32]
    L.cs_physics_destroy.argtypes = [vp]
    L.cs_physics_set_umf.argtypes = [vp, vp]
    L.cs_physics_buffers.argtypes = [vp, pp, pp, pp, pp]
    L.cs_calc_fluxes_pre.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp]
    L.cs_calc_fluxes.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, Dcomp, vp]
    L.cs_calc_viscous_shear_stress.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, Dcomp, vp]
    L.cs_calc_time_step.argtypes = [vp, vp, vp, vp, vp, vp, vp, f64, ctypes.POINTER(f64), sz, vp]
    L.cs_gcbc_go.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, Dcomp, vp, vp]
    L.cs_gcbc_apply.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, Dcomp, ctypes.c_double, vp, vp, vp]
    L.cs_gcbc_apply.restype = i32
    L.cs_thermo.argtypes = [vp, vp, vp, sz, vp]
    L.cs_wall_condition_update.argtypes = [vp, vp, ctypes.POINTER(f64), Dcomp, vp, vp]
    L.cs_wall_condition_update.restype = i32
    L.cs_rk_update.argtypes = [vp, vp, vp, f64, vp, sz, vp]
    for name in ("cs_physics_create", "cs_physics_destroy", "cs_physics_set_umf", "cs_physics_buffers",
                 "cs_calc_fluxes_pre", "cs_calc_fluxes", "cs_calc_viscous_shear_stress",
                 "cs_calc_time_step", "cs_gcbc_go", "cs_thermo", "cs_rk_update"):
        getattr(L, name).restype = i32
    from .solver import SolverConfig
    L.cs_solver_create.argtypes = [pp, ctypes.POINTER(SolverConfig)]
    L.cs_solver_destroy.argtypes = [vp]
    L.cs_solver_rhs.argtypes = [vp, vp, vp, vp]
    L.cs_solver_stage.argtypes = [vp, i32, vp, vp, vp, f64, vp]
    L.cs_solver_step.argtypes = [vp, vp, f64, vp]
    L.cs_solver_step_host.argtypes = [vp, vp, vp, f64, vp]
    L.cs_solver_last_dt.argtypes = [vp, ctypes.POINTER(f64)]
    L.cs_solver_dt_device.argtypes = [vp, pp]
    L.cs_tgv_init.argtypes = [vp, i32, i32, i32, f64, f64, ctypes.c_uint64, vp]
    from .ensemble import EnsembleTuning
    pt = ctypes.POINTER(EnsembleTuning)
    i64p = ctypes.POINTER(ctypes.c_int64)
    L.cs_ensemble_create.argtypes = [pp, i32, ctypes.POINTER(SolverConfig)]
    L.cs_ensemble_destroy.argtypes = [vp]
    L.cs_ensemble_state_size.argtypes = [vp, i64p]
    L.cs_ensemble_box_offset.argtypes = [vp, i32, i64p]
    L.cs_ensemble_step.argtypes = [vp, vp, vp]
    L.cs_ensemble_last_dt.argtypes = [vp, ctypes.POINTER(f64)]
    L.cs_ensemble_set_tuning.argtypes = [vp, pt]
    L.cs_ensemble_set_wait.argtypes = [vp, ctypes.c_longlong, i32]
    L.cs_ensemble_set_wait.restype = i32
    L.cs_ensemble_get_tuning.argtypes = [vp, pt]
    L.cs_ensemble_autotune.argtypes = [vp, vp, i32, pt, ctypes.POINTER(f64), vp]
    for name in ("cs_ensemble_create", "cs_ensemble_destroy", "cs_ensemble_state_size", "cs_ensemble_box_offset",
                 "cs_ensemble_step", "cs_ensemble_last_dt", "cs_ensemble_set_tuning", "cs_ensemble_get_tuning",
                 "cs_ensemble_autotune"):
        getattr(L, name).restype = i32
    dp = ctypes.POINTER(f64)
    L.cs_adjoint_create.argtypes = [pp, ctypes.POINTER(SolverConfig)]
    L.cs_adjoint_destroy.argtypes = [vp]
    L.cs_adjoint_deriv.argtypes = [vp, i32, i32, vp, vp, i32, i32, vp]
    L.cs_adjoint_filter.argtypes = [vp, i32, i32, f64, vp, vp, i32, i32, vp]
    L.cs_adjoint_filter.restype = i32
    L.cs_rhs_jvp.argtypes = [vp, vp, vp, vp, vp]
    L.cs_rhs_vjp.argtypes = [vp, vp, vp, vp, vp]
    L.cs_adjoint_stages.argtypes = [vp, vp, f64, pp, vp, vp]
    L.cs_step_jvp.argtypes = [vp, pp, f64, vp, vp, vp]
    L.cs_step_vjp.argtypes = [vp, pp, f64, vp, vp, vp]
    L.cs_kinetic_energy.argtypes = [vp, vp, dp, vp, vp]
    L.cs_adjoint_gradient.argtypes = [vp, vp, i32, dp, i32, vp, dp, vp]
    L.cs_adjoint_gradient_bytes.argtypes = [vp, i32, i32, ctypes.POINTER(sz)]
    L.cs_adjoint_gradient_bytes.restype = i32
    L.cs_point_flux.argtypes = [i32, i32, dp, dp, dp, f64, f64, dp, dp]
    L.cs_point_flux_jvp.argtypes = [i32, i32, dp, dp, dp, dp, dp, f64, f64, dp, dp]
    L.cs_point_flux_vjp.argtypes = [i32, i32, dp, dp, dp, dp, f64, f64, dp, dp, dp]
    L.cs_point_prim.argtypes = [dp, dp]
    L.cs_point_prim_jvp.argtypes = [dp, dp, dp]
    L.cs_point_prim_vjp.argtypes = [dp, dp, dp]
    for name in ("cs_adjoint_create", "cs_adjoint_destroy", "cs_adjoint_deriv", "cs_rhs_jvp", "cs_rhs_vjp",
                 "cs_adjoint_stages", "cs_step_jvp", "cs_step_vjp", "cs_kinetic_energy", "cs_adjoint_gradient",
                 "cs_point_flux", "cs_point_flux_jvp", "cs_point_flux_vjp", "cs_point_prim", "cs_point_prim_jvp",
                 "cs_point_prim_vjp"):
        getattr(L, name).restype = i32
    L.cs_solver_autotune.argtypes = [vp, vp, i32, ctypes.POINTER(ctypes.c_int * 3 * 2), vp]
    L.cs_solver_autotune.restype = i32
    L.cs_solver_schedule.argtypes = [vp, ctypes.POINTER(ctypes.c_int * 3 * 2)]
    L.cs_solver_schedule.restype = i32
    L.cs_solver_set_metrics.argtypes = [vp, vp, vp, vp, vp]
    L.cs_solver_set_metrics.restype = i32
    L.cs_grid_metrics.argtypes = [vp, vp, ctypes.POINTER(f64 * 3 * 3), vp, vp, vp, vp, vp]
    L.cs_grid_metrics.restype = i32
    L.cs_vtk_write.argtypes = [ctypes.c_char_p, i32, i32, i32, vp, i32, ctypes.POINTER(ctypes.c_char_p)]
    L.cs_vtk_write.restype = i32
    L.cs_solver_profile_begin.argtypes = [vp]
    L.cs_solver_profile_end.argtypes = [vp, vp, vp]
    for name in ("cs_solver_create", "cs_solver_destroy", "cs_solver_rhs", "cs_solver_stage",
                 "cs_solver_step", "cs_solver_step_host", "cs_solver_last_dt", "cs_solver_dt_device", "cs_tgv_init",
                 "cs_solver_profile_begin", "cs_solver_profile_end",
                 "cs_numerics_create", "cs_numerics_destroy", "cs_deriv_setup", "cs_get_coeffs",
                 "cs_interface_coeffs",
                 "cs_get_ndf", "cs_get_buffers", "cs_deriv", "cs_deriv_f32", "cs_fill_buffers",
                 "cs_halo_exchange_self", "cs_filter", "cs_line_tables"):
        getattr(L, name).restype = i32
