// compact_schemes/gcbc.hpp -- drop-in gcbc<Type, TypeIndex> and gcbc_go
// (src/gcbc.hpp) over libcompact_b200, FP64, non-reflective faces.
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

// gcbc_go (src/gcbc.hpp:86-186).  drva comes from the numerics object that
// computed the last flux derivatives; faces coded periodic / interface are
// skipped; wall and curvilinear-interface faces are not in this build.
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
