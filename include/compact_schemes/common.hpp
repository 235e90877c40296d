// compact_schemes/common.hpp -- drop-in types and constants for code written
// against EnricoDeg/compact_schemes (src/common/data_types.hpp,
// src/common/parameters.hpp), backed by libcompact_b200 (compact_b200.h).
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

#include "../compact_b200.h"

// t_dcomp (src/common/data_types.hpp:33-39): layout-compatible with cs_dcomp.
struct t_dcomp {
    int lmx;
    int lxi;
    int let;
    int lze;
};
static_assert(sizeof(t_dcomp) == sizeof(cs_dcomp), "t_dcomp layout");

template <typename Type>
struct t_point {
    Type x;
    Type y;
    Type z;
};

// Scheme and gas constants (src/common/parameters.hpp:35-74).
static constexpr unsigned int lmd = 8;
static constexpr unsigned int mbci = 4;
static constexpr unsigned int NumberOfVariables = 5;
static constexpr unsigned int NumberOfSpatialDims = 3;
static constexpr unsigned int NumberOfFaces = 2;
static constexpr int BC_NON_REFLECTIVE = CS_BC_NON_REFLECTIVE;
static constexpr int BC_WALL_INVISCID = CS_BC_WALL_INVISCID;
static constexpr int BC_WALL_VISCOUS = CS_BC_WALL_VISCOUS;
static constexpr int BC_INTER_CURV = CS_BC_INTER_CURV;
static constexpr int BC_INTER_STRAIGHT = CS_BC_INTER_STRAIGHT;
static constexpr int BC_INTER_SUBDOMAINS = CS_BC_INTER_SUBDOMAINS;
static constexpr int BC_PERIODIC = CS_BC_PERIODIC;
static constexpr int nrall = 0;
static constexpr int nkrk = 4;

namespace compact_b200 {

inline cs_dcomp to_c(const t_dcomp &d) { return cs_dcomp{d.lmx, d.lxi, d.let, d.lze}; }

// The reference prints and exits on any CUDA error (src/cuda/check.hpp:36-41);
// the drop-in classes keep that behaviour on top of the status codes.
inline void check(int rc, const char *what) {
    if (rc != CS_OK) {
        std::fprintf(stderr, "compact_b200: %s failed (%d): %s\n", what, rc, cs_last_error());
        std::exit(EXIT_FAILURE);
    }
}

}  // namespace compact_b200
