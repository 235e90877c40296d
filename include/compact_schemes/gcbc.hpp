// compact_schemes/gcbc.hpp -- drop-in gcbc<Type, TypeIndex>, gcbc_go and
// wall_condition_update (src/gcbc.hpp) over libcompact_b200, FP64.
#pragma once

#include "numerics_pc.hpp"

template <typename Type, typename TypeIndex>
struct gcbc {
    explicit gcbc(t_dcomp d) {
        const size_t n = (size_t)d.lmx;
        cudaMalloc(&npex, n * sizeof(TypeIndex));
        const size_t f[3] = {(size_t)d.let * d.lze, (size_t)d.lxi * d.lze, (size_t)d.lxi * d.let};
        for (int a = 0; a < 3; ++a) cudaMalloc(&drvb[a], 2 * NumberOfVariables * f[a] * sizeof(Type));
        cudaMalloc(&sbcc, n * sizeof(Type));
        cudaMemset(sbcc, 0, n * sizeof(Type));
        drvb0 = drvb[0];
        drvb1 = drvb[1];
        drvb2 = drvb[2];
    }
    ~gcbc() {
        cudaFree(npex);
        for (int a = 0; a < 3; ++a) cudaFree(drvb[a]);
        cudaFree(sbcc);
    }
    void init() {}
    TypeIndex *npex = nullptr;
    Type *drvb0, *drvb1, *drvb2;
    Type *drvb[3];
    Type *sbcc = nullptr;
};

// gcbc_go (src/gcbc.hpp:86-186) with the reference's parameter list: every
// face code (non-reflective, inviscid / viscous wall, curvilinear interface)
// of a single-rank block; drva_buffer is turned into characteristic form in
// place as the reference does, drvb_buffer receives the GCIC exchange (the
// block is its own neighbour; mcd is not needed).  FP64.
template <typename Type>
void gcbc_go(Type *drva_buffer[3], Type *cm_buffer[3], Type *drvb_buffer[3], Type *qa, Type *de, Type *pressure,
             Type *yaco, Type *sbcc, t_point<Type> umf, t_point<Type> dudtmf, t_dcomp dcomp_info, Type dtwi,
             int nbc[2][3], int mcd[2][3], cudaStream_t stream = nullptr) {
    static_assert(std::is_same<Type, double>::value,
                  "gcbc_go: FP64 (the drop-in physics path computes in double, see physics<Visc, Type>)");
    const double u[3] = {umf.x, umf.y, umf.z};
    const double a[3] = {dudtmf.x, dudtmf.y, dudtmf.z};
    compact_b200::check(cs_gcbc_apply(drva_buffer, cm_buffer, drvb_buffer, qa, de, pressure, yaco, sbcc, u, a,
                                      compact_b200::to_c(dcomp_info), dtwi, nbc, mcd, stream),
                        "gcbc_go");
}

// gcbc_go for non-reflective faces with drva taken from the numerics object
// that computed the last flux derivatives (the library's own shorthand; faces
// coded periodic / interface are skipped).
template <typename Type>
void gcbc_go(numerics_pc<Type> *numerics_instance, Type *cm_buffer[3], Type *qa, Type *de,
             Type *pressure, Type *yaco, Type *sbcc, t_point<Type> umf, t_dcomp dcomp_info,
             int nbc[2][3], cudaStream_t stream = nullptr) {
    const double u[3] = {umf.x, umf.y, umf.z};
    compact_b200::check(cs_gcbc_go(numerics_instance->handle, cm_buffer, qa, de, pressure, yaco, sbcc, u,
                                   compact_b200::to_c(dcomp_info), nbc, stream),
                        "gcbc_go");
}

// wall_condition_update (src/gcbc.hpp:188-228): the wall state at faces coded
// BC_WALL_INVISCID / BC_WALL_VISCOUS, points where npex == 0.  FP64 and an
// int mask, as the reference instantiates it.
template <typename Type, typename TypeIndex>
void wall_condition_update(Type *qa, TypeIndex *npex, t_point<Type> umf, t_dcomp dcomp_info, int nbc[2][3],
                           cudaStream_t stream = nullptr) {
    static_assert(sizeof(Type) == sizeof(double) && sizeof(TypeIndex) == sizeof(int),
                  "wall_condition_update: double state and int mask");
    const double u[3] = {umf.x, umf.y, umf.z};
    compact_b200::check(cs_wall_condition_update(reinterpret_cast<double *>(qa), reinterpret_cast<const int *>(npex),
                                                 u, compact_b200::to_c(dcomp_info), nbc, stream),
                        "wall_condition_update");
}
