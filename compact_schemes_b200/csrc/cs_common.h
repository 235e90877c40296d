// cs_common.h -- shared host/device definitions of the compact_schemes_b200
// library: scheme constants, line geometry and the precomputed tables of the
// partitioned tridiagonal line solver.
#pragma once

#include <cstdint>
#include <vector>

#include "../../include/compact_b200.h"

namespace csb {

// Compact scheme constants (reference src/common/parameters.hpp:35-43): sixth
// order interior Pade first derivative and its third/fourth order closures.
constexpr double kAlpha = 1.0 / 3.0;
constexpr double kAlpha01 = 2.0;
constexpr double kAlpha10 = 1.0 / 4.0;
constexpr double kAa = 7.0 / 9.0;
constexpr double kBb = 1.0 / 36.0;
constexpr double kAb00 = -5.0 / 2.0;
constexpr double kAb01 = 2.0;
constexpr double kAb02 = 1.0 / 2.0;
constexpr double kAb10 = 3.0 / 4.0;
constexpr int kLmd = 8;    // interface stencil width
constexpr int kMbci = 4;   // GCBC planes
// Gas constants (src/common/parameters.hpp:61-67).
constexpr double kGam = 1.4;
constexpr double kGamm1 = kGam - 1.0;
constexpr double kHamm1 = 1.0 / kGamm1;
constexpr double kPrndtl = 0.71;
constexpr double kGamm1Prndtli = 1.0 / (kGamm1 * kPrndtl);

// Maximum line length: 32 lanes x 32 points per lane.
constexpr int kMaxLine = 1024;
// Reduced system of the partitioned solve: 2 rows per lane, 64 rows,
// six PCR steps (strides 1..32).
constexpr int kPcrSteps = 6;

// kDerivT / kFilterT: the transposed left-hand-side matrices A^T (adjoint
// line solves).
enum Scheme { kDeriv = 0, kFilter = 1, kDerivT = 2, kFilterT = 3 };

// Interface closure weights of the quasi-disjoint compact scheme
// (numerics_base::deriv_setup, src/numerics_base.hpp:182-297).
struct Coeffs {
    double pbco[16];
    double pbci[16];
};
void compute_interface_coeffs(Coeffs &c);

// Host copy of the solver tables of one line configuration.  Device arrays
// are laid out [t][lane] (t < LT) so that lane `c` reading element `t` is a
// coalesced / bank-conflict-free access.
struct HostTables {
    int n = 0, lt = 0, p = 0, last_len = 0;
    bool cyclic = false;
    double cyc_s1 = 0.0, cyc_s2 = 0.0;
    // per (t, lane)
    std::vector<double> fwd1, fwd2, bwd1, bwd2, rca, rcc, cycz;
    // reduced system: [step][row-in-lane][lane] and [row-in-lane][lane]
    std::vector<double> k1, k2, invb;
    // PCR depth: the reduced system's couplings decay geometrically, so after
    // pcr64 (pcr32) steps the remaining ones are below FP64 (FP32) resolution;
    // invb / invb32 are the inverse diagonals after that many steps
    int pcr64 = 6, pcr32 = 6;
    std::vector<double> invb32;
};

// Choose the per-lane chunk length (power of two) for a line of n points.
int chunk_length(int n, int min_lt = 2);
// Build tables for the tridiagonal matrix rows a (sub), b (diag), c (super)
// of a line of n points.  cyclic: a[0] couples x[n-1] and c[n-1] couples x[0].
// min_lt: shortest chunk (a power of two >= 2); the chunk doubles from there
// until the line fits 32 lanes.
bool build_tables(int n, const double *a, const double *b, const double *c, bool cyclic,
                  HostTables &out, int min_lt = 2);
// Matrix rows of the compact derivative (build_system,
// src/cuda/kernels/numerics_device_pc.hpp:176-293) for face flags nstart/nend.
void deriv_rows(int n, int nstart, int nend, double *a, double *b, double *c);
// Matrix rows of the compact filter (see filter_rhs in line_solver.cuh).
void filter_rows(int n, bool cyclic, double alpha_f, double *a, double *b, double *c);

}  // namespace csb
