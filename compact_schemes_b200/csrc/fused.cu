// fused.cu -- the fused RHS / RK-stage pipeline of compact_schemes_b200.
//
// One RK stage of the compressible Navier-Stokes RHS of the reference
// (physics::calc_viscous_shear_stress + physics::calc_fluxes,
// src/physics_pc.hpp:83-227, followed by the RK update that
// physics_base::movef leaves empty, src/physics_base.hpp:147-150) runs as six
// line-solve passes over the state, each staging a tile of full lines in
// shared memory:
//   grad pass a (a = x, y, z): q -> u, v, w, T on the fly -> 4 compact
//       derivatives along a -> G[a] (4 fields).  The first pass of a step
//       also reduces the two CFL maxima of calc_time_step.
//   flux pass a: q, G -> tau, heat flux, flux F[m][a] (m = 0..4) on the fly
//       -> 5 compact derivatives along a -> R (= for x, += for y) or, for the
//       last axis, q_out = q^n - dt/(4-k) * J * (R + dF)  (RK update fused).
// Metrics are those of a uniform Cartesian grid (constants, not read) unless
// cs_solver_set_metrics gave per-point arrays; the FP64 one-phase kernels
// then read them (FM instantiations, 8-line tiles).
#include <cmath>
#include <cstring>
#include <vector>

#include "fused_mixed.cuh"

namespace csb {

// ----------------------------------------------------------------------------
// GCBC, non-reflective, x faces (gcbc_setup_kernel + gcbc_update_non_reflective_kernel,
// src/cuda/kernels/gcbc.hpp:251-454, reference defects fixed: see oracle/oracle.cpp)
// ----------------------------------------------------------------------------
// With per-point metrics (xim_f, yaco_f non-null) the face normal and J are
// those of the face point and the closure weight is sbcc = 1 / J there.
template <typename RT>
__global__ void k_gcbc_x(RT *__restrict__ rhs, const double *__restrict__ drva,
                         const double *__restrict__ q, int lxi, int64_t lmx, int64_t F, int face_mask,
                         Phys ph, double sb0, double sb1, double sb2, double sb3,
                         const double *__restrict__ xim_f = nullptr, const double *__restrict__ yaco_f = nullptr) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 2 * F) return;
    const int ip = (int)(t / F);
    const int64_t fi = t % F;
    if (!((face_mask >> ip) & 1)) return;
    const int64_t idx = fi * lxi + (ip ? lxi - 1 : 0);
    if (xim_f) {
#pragma unroll
        for (int k = 0; k < 3; ++k) ph.M[0][k] = xim_f[k * lmx + idx];
        ph.J = yaco_f[idx];
        sb0 = 1.0 / ph.J;
        sb1 = sb2 = sb3 = 0.0;
    }
    // face normal: grad(xi) / |grad(xi)| (exactly (+-1, 0, 0) on a Cartesian grid)
    double c[3];
    if (ph.M[0][1] == 0.0 && ph.M[0][2] == 0.0) {
        c[0] = ph.M[0][0] > 0.0 ? 1.0 : -1.0; c[1] = 0.0; c[2] = 0.0;
    } else {
        const double nrm = sqrt(xmul(ph.M[0][0], ph.M[0][0]) + xmul(ph.M[0][1], ph.M[0][1]) +
                                xmul(ph.M[0][2], ph.M[0][2]));
        c[0] = ph.M[0][0] / nrm; c[1] = ph.M[0][1] / nrm; c[2] = ph.M[0][2] / nrm;
    }
    const double rho = q[idx], rhoi = 1.0 / rho;
    const double ve[3] = {xmul(q[lmx + idx], rhoi), xmul(q[2 * lmx + idx], rhoi), xmul(q[3 * lmx + idx], rhoi)};
    const double hv2 = xmul(0.5, xmul(ve[0], ve[0]) + xmul(ve[1], ve[1]) + xmul(ve[2], ve[2]));
    const double pp = xmul(kGamm1, q[4 * lmx + idx] - xmul(rho, hv2));
    const double ao = sqrt(xmul(xmul(kGam, rhoi), pp)), aoi = 1.0 / ao;
    const double vn = xmul(c[0], ve[0]) + xmul(c[1], ve[1]) + xmul(c[2], ve[2]);
    const double vs = xmul(c[0], ph.umf[0]) + xmul(c[1], ph.umf[1]) + xmul(c[2], ph.umf[2]);
    double dr[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) dr[v] = xmul(ph.J, drva[(int64_t)(ip * 5 + v) * F + fi]);
    // characteristic amplitudes of the two acoustic waves (rows 3, 4 of xtq2r)
    const double ho = xmul(xmul(kGamm1, aoi), aoi), bo = 1.0 - xmul(ho, hv2), co = xmul(aoi, vn);
    const double dm[3] = {xmul(aoi, c[0]), xmul(aoi, c[1]), xmul(aoi, c[2])};
    const double rv[3] = {xmul(ho, ve[0]), xmul(ho, ve[1]), xmul(ho, ve[2])};
    const double cha3 = xmul(1.0 - bo - co, dr[0]) + xmul(dm[0] - rv[0], dr[1]) + xmul(dm[1] - rv[1], dr[2]) +
                        xmul(dm[2] - rv[2], dr[3]) + xmul(ho, dr[4]);
    const double cha4 = xmul(1.0 - bo + co, dr[0]) + xmul(-dm[0] - rv[0], dr[1]) + xmul(-dm[1] - rv[1], dr[2]) +
                        xmul(-dm[2] - rv[2], dr[3]) + xmul(ho, dr[4]);
    const double ra0 = 1.0 - 2.0 * ip;
    const double d3 = ra0 * (vn + vs + ao) > 0 ? -cha3 : 0.0;
    const double d4 = ra0 * (vn + vs - ao) > 0 ? -cha4 : 0.0;
    // back to conservative variables: columns 3, 4 of xtr2q
    const double bo2 = hv2 + xmul(xmul(kHamm1, ao), ao), co2 = xmul(ao, vn);
    const double em[3] = {xmul(ao, c[0]), xmul(ao, c[1]), xmul(ao, c[2])};
    double dq[5];
    dq[0] = xmul(0.5, d3) + xmul(0.5, d4);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double s3 = xmul(0.5, ve[k] + em[k]);
        dq[1 + k] = xmul(s3, d3) + xmul(s3 - em[k], d4);
    }
    {
        const double s3 = xmul(0.5, bo2 + co2);
        dq[4] = xmul(s3, d3) + xmul(s3 - co2, d4);
    }
    const double sb[4] = {sb0, sb1, sb2, sb3};
    const int iq = 1 - 2 * ip;
#pragma unroll
    for (int ii = 0; ii < kMbci; ++ii) {
        if (sb[ii] == 0.0) continue;
        const int64_t o = idx + (int64_t)ii * iq;
#pragma unroll
        for (int v = 0; v < 5; ++v) rhs[v * lmx + o] = (RT)((double)rhs[v * lmx + o] + xmul(sb[ii], dq[v]));
    }
}

// Taylor-Green initial state (see oracle or_tgv_init for the definition).
__device__ __forceinline__ double noise01(uint64_t seed, uint64_t index) {
    uint64_t z = seed * 0x9E3779B97F4A7C15ull + index + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

__global__ void k_tgv(double *__restrict__ q, int lxi, int let, int64_t lmx, double mach, double amp,
                      uint64_t seed, double hx, double hy, double hz) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= lmx) return;
    const int64_t i = idx % lxi, j = (idx / lxi) % let, k = idx / ((int64_t)lxi * let);
    const double x = i * hx, y = j * hy, z = k * hz;
    const double u = mach * sin(x) * cos(y) * cos(z);
    const double v = -mach * cos(x) * sin(y) * cos(z);
    const double w = 0.0;
    const double p = 1.0 / kGam + mach * mach / 16.0 * (cos(2 * x) + cos(2 * y)) * (cos(2 * z) + 2.0);
    const double rho = 1.0 + amp * noise01(seed, (uint64_t)idx);
    q[idx] = rho;
    q[lmx + idx] = rho * u;
    q[2 * lmx + idx] = rho * v;
    q[3 * lmx + idx] = rho * w;
    q[4 * lmx + idx] = p * kHamm1 + 0.5 * rho * (u * u + v * v + w * w);
}

}  // namespace csb

using namespace csb;

struct cs_solver {
    cs_solver_config cfg{};
    cs_dcomp d{};
    int ndf[2][3]{};
    Coeffs cf{};
    Phys ph{};
    FieldMet fm{};  // per-point metrics (cs_solver_set_metrics), else null
    TableCache tables;
    const DeviceTables *tab[3] = {nullptr, nullptr, nullptr};
    int active[3] = {0, 0, 0};
    double *q1 = nullptr, *grad = nullptr, *rhs = nullptr, *drva = nullptr;
    double *qhost_dev = nullptr;  // device state for cs_solver_step_host
    // mixed precision: FP32 deviation shadow, gradients and RHS
    bool mixed = false;
    float *sh32 = nullptr, *grad32 = nullptr, *rhs32 = nullptr;
    unsigned long long *dtacc = nullptr;
    double *dt_dev = nullptr;
    int64_t F[3] = {0, 0, 0};
    int tile[2][3] = {{8, 8, 8}, {8, 8, 16}};  // lines per tile: [gradient|flux][axis]
    int pl[2][3] = {{0, 0, 0}, {0, 0, 0}};     // pipelined kernels per [gradient|flux][axis]
    int can[2][3] = {{0, 0, 0}, {0, 0, 0}};    // feasible schedules: 1 tile 8, 2 tile 16, 4 pipelined,
                                               // 8 TMA-staged (gradient passes)
    int tma[3] = {0, 0, 0};                    // gradient pass along each axis stages its pencils by TMA
    int *err = nullptr;                        // device word: nonzero if a TMA staging copy timed out
    const DeviceTables *ftab[3] = {nullptr, nullptr, nullptr};  // filter tables (cfg.filter)
    int nsm = 0;
    // optional per-pass event timing (eager path only)
    bool profiling = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof;
    std::vector<cudaEvent_t> event_pool;
    // captured step graph
    cudaGraphExec_t graph = nullptr;
    const double *graph_q = nullptr;
    double graph_dt = 0.0;
    cudaStream_t graph_stream = nullptr;
};

namespace csb {

// Pass kinds reported by cs_solver_profile_end.
enum PassKind { kPassGradX = 0, kPassGradY, kPassGradZ, kPassFluxX, kPassFluxY, kPassFluxZ, kPassGcbc,
                kPassFilter, kPassKinds };
static_assert(kPassKinds == CS_PASS_KINDS, "pass kinds");

static cudaEvent_t take_event(cs_solver *s) {
    if (!s->event_pool.empty()) {
        cudaEvent_t e = s->event_pool.back();
        s->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// RAII bracket: records a start/stop event pair around one pass when profiling.
struct PassTimer {
    cs_solver *s;
    cudaStream_t st;
    int kind;
    cudaEvent_t a = nullptr, b = nullptr;
    PassTimer(cs_solver *s_, cudaStream_t st_, int kind_) : s(s_), st(st_), kind(kind_) {
        if (s->profiling) {
            a = take_event(s);
            b = take_event(s);
            cudaEventRecord(a, st);
        }
    }
    ~PassTimer() {
        if (s->profiling) {
            cudaEventRecord(b, st);
            s->prof.push_back({kind, {a, b}});
        }
    }
};

int bc_ndf(int code) {
    if (code == CS_BC_NON_REFLECTIVE || code == CS_BC_WALL_INVISCID || code == CS_BC_WALL_VISCOUS ||
        code == CS_BC_INTER_CURV) return 0;
    if (code == CS_BC_INTER_STRAIGHT || code == CS_BC_INTER_SUBDOMAINS || code == CS_BC_PERIODIC) return 1;
    return -1;
}

void uniform_phys(const cs_solver_config &cfg, Phys &ph) {
    const double hx = cfg.dx, hy = cfg.dy, hz = cfg.dz;
    std::memset(&ph, 0, sizeof ph);
    ph.M[0][0] = hy * hz;
    ph.M[1][1] = hx * hz;
    ph.M[2][2] = hx * hy;
    ph.J = 1.0 / (hx * hy * hz);
    ph.mu = cfg.mu;
    for (int c = 0; c < 3; ++c) ph.umf[c] = cfg.umf[c];
    ph.rr1 = ph.M[0][0] * ph.M[0][0] + ph.M[1][1] * ph.M[1][1] + ph.M[2][2] * ph.M[2][2];
}

static int64_t fsize(const cs_dcomp &d, int a) {
    return a == 0 ? (int64_t)d.let * d.lze : (a == 1 ? (int64_t)d.lxi * d.lze : (int64_t)d.lxi * d.let);
}
static int llen(const cs_dcomp &d, int a) { return a == 0 ? d.lxi : (a == 1 ? d.let : d.lze); }

static PassArgs pass_args(cs_solver *s, int a, int kind) {
    PassArgs p;
    p.lmx = s->d.lmx;
    p.lxi = s->d.lxi;
    p.let = s->d.let;
    p.F = s->F[a];
    p.nstart = s->ndf[0][a];
    p.nend = s->ndf[1][a];
    p.tl = s->tile[kind][a];
    p.pl = s->pl[kind][a];
    p.nsm = s->nsm;
    p.viscous = s->cfg.viscous;
    p.tab = s->tab[a];
    p.cf = s->cf;
    p.ph = s->ph;
    p.fm = s->fm;
    p.grad = s->grad;
    p.rhs = s->rhs;
    p.dtacc = s->dtacc;
    return p;
}

static int grad_pass(cs_solver *s, int a, const double *q, bool dtred, cudaStream_t st) {
    PassTimer pt(s, st, kPassGradX + a);
    const PassArgs p = pass_args(s, a, 0);
    // the TMA form reads the uniform-grid constants and needs a 16-byte aligned state
    if (s->tma[a] && !(dtred && s->fm.xim) && reinterpret_cast<uintptr_t>(q) % 16 == 0) {
        if (a == 0) return launch_grad_tma<0>(p, s->d, q, dtred, s->err, st);
        if (a == 1) return launch_grad_tma<1>(p, s->d, q, dtred, s->err, st);
        return launch_grad_tma<2>(p, s->d, q, dtred, s->err, st);
    }
    if (a == 0) return launch_grad<0>(p, q, dtred, st);
    if (a == 1) return launch_grad<1>(p, q, dtred, st);
    return launch_grad<2>(p, q, dtred, st);
}

static int flux_pass(cs_solver *s, int a, int mode, const double *q, const double *qn, double *qout,
                     double *drva, const RkParams &rk, cudaStream_t st) {
    PassTimer pt(s, st, kPassFluxX + a);
    const PassArgs p = pass_args(s, a, 1);
    if (a == 0) return launch_flux<0>(p, mode, q, qn, qout, drva, rk, st);
    if (a == 1) return launch_flux<1>(p, mode, q, qn, qout, drva, rk, st);
    return launch_flux<2>(p, mode, q, qn, qout, drva, rk, st);
}

static MixedArgs mixed_args(cs_solver *s, int a, int kind) {
    MixedArgs m;
    m.base = pass_args(s, a, kind);
    m.shadow = s->sh32;
    m.grad = s->grad32;
    m.rhs = s->rhs32;
    // CS_REFINE_FLUX: the gradient passes skip the refinement sweep (their
    // FP32 solve error only reaches the state through the viscous terms)
    m.refine = s->cfg.refine == CS_REFINE_FLUX ? (kind == 1) : s->cfg.refine;
    m.fp32 = s->cfg.precision == CS_PREC_MIXED_F32;
    return m;
}

static int grad_pass_mx(cs_solver *s, int a, const double *q, bool first, cudaStream_t st) {
    PassTimer pt(s, st, kPassGradX + a);
    const MixedArgs m = mixed_args(s, a, 0);
    // the TMA form reads the FP32 shadow, which the first pass of a step writes
    if (s->tma[a] && !first) {
        if (a == 0) return launch_grad_mx_tma<0>(m, s->d, s->err, st);
        if (a == 1) return launch_grad_mx_tma<1>(m, s->d, s->err, st);
        return launch_grad_mx_tma<2>(m, s->d, s->err, st);
    }
    if (a == 0) return launch_grad_mx<0>(m, q, first, st);
    if (a == 1) return launch_grad_mx<1>(m, q, first, st);
    return launch_grad_mx<2>(m, q, first, st);
}

static int flux_pass_mx(cs_solver *s, int a, int mode, const double *qn, double *qout, bool shadow_out,
                        double *drva, const RkParams &rk, cudaStream_t st) {
    PassTimer pt(s, st, kPassFluxX + a);
    const MixedArgs m = mixed_args(s, a, 1);
    if (a == 0) return launch_flux_mx<0>(m, mode, qn, qout, shadow_out, drva, rk, st);
    if (a == 1) return launch_flux_mx<1>(m, mode, qn, qout, shadow_out, drva, rk, st);
    return launch_flux_mx<2>(m, mode, qn, qout, shadow_out, drva, rk, st);
}

static bool gcbc_on(const cs_solver *s) {
    return s->cfg.gcbc && s->active[0] &&
           (s->cfg.nbc[0][0] == CS_BC_NON_REFLECTIVE || s->cfg.nbc[1][0] == CS_BC_NON_REFLECTIVE);
}

// RHS of one state (rk == nullptr) or one full RK stage.
static int run_stage(cs_solver *s, const double *qin, const double *qn, double *qout, double *rhs_out,
                     const RkParams *rk, bool dtred, cudaStream_t st) {
    int axes[3], na = 0;
    for (int a = 0; a < 3; ++a)
        if (s->active[a]) axes[na++] = a;
    if (s->cfg.viscous)
        for (int i = 0; i < na; ++i)
            if (int rc = grad_pass(s, axes[i], qin, dtred && i == 0, st)) return rc;
    if (dtred && !s->cfg.viscous) {
        // inviscid: the CFL maxima come from a gradient-free reduction; reuse
        // the x gradient pass into scratch (its output is unused)
        if (int rc = grad_pass(s, axes[0], qin, true, st)) return rc;
    }
    double *saved_rhs = s->rhs;
    if (rhs_out) s->rhs = rhs_out;
    RkParams none{};
    for (int i = 0; i < na; ++i) {
        const int a = axes[i];
        int mode;
        if (!rk) mode = i == 0 ? kWrite : kAccum;
        else if (na == 1) mode = kWriteRk;
        else mode = i == 0 ? kWrite : (i == na - 1 ? kAccumRk : kAccum);
        double *drva = (a == 0 && gcbc_on(s)) ? s->drva : nullptr;
        int rc = flux_pass(s, a, mode, qin, qn, qout, drva, rk ? *rk : none, st);
        if (rc) { s->rhs = saved_rhs; return rc; }
        if (drva && (mode == kWrite || mode == kAccum) && !(rk && na == 1)) {
            PassTimer pt(s, st, kPassGcbc);
            const int64_t F = s->F[0];
            int mask = (s->cfg.nbc[0][0] == CS_BC_NON_REFLECTIVE ? 1 : 0) |
                       (s->cfg.nbc[1][0] == CS_BC_NON_REFLECTIVE ? 2 : 0);
            k_gcbc_x<double><<<(unsigned)((2 * F + 127) / 128), 128, 0, st>>>(s->rhs, s->drva, qin, s->d.lxi,
                                                                    s->d.lmx, F, mask, s->ph,
                                                                    1.0 / s->ph.J, 0.0, 0.0, 0.0,
                                                                    s->fm.xim, s->fm.yaco);
            if (cudaGetLastError() != cudaSuccess) { s->rhs = saved_rhs; return set_error(CS_ERR_CUDA, "gcbc launch"); }
        }
    }
    s->rhs = saved_rhs;
    return CS_OK;
}

// Mixed-precision stage.  The shadow of qin must be current unless
// first_pass (stage 0), where the first gradient pass builds it from the FP64
// state (and reduces the CFL maxima).
static int run_stage_mx(cs_solver *s, const double *qin, const double *qn, double *qout, bool rhs_only,
                        const RkParams *rk, bool first_pass, bool shadow_out, cudaStream_t st) {
    int axes[3], na = 0;
    for (int a = 0; a < 3; ++a)
        if (s->active[a]) axes[na++] = a;
    for (int i = 0; i < na; ++i)
        if (s->cfg.viscous || (i == 0 && first_pass))
            if (int rc = grad_pass_mx(s, axes[i], qin, first_pass && i == 0, st)) return rc;
    RkParams none{};
    for (int i = 0; i < na; ++i) {
        const int a = axes[i];
        int mode;
        if (rhs_only) mode = i == 0 ? kWrite : kAccum;
        else if (na == 1) mode = kWriteRk;
        else mode = i == 0 ? kWrite : (i == na - 1 ? kAccumRk : kAccum);
        double *drva = (a == 0 && gcbc_on(s)) ? s->drva : nullptr;
        if (int rc = flux_pass_mx(s, a, mode, qn, qout, shadow_out, drva, rk ? *rk : none, st)) return rc;
        if (drva && (mode == kWrite || mode == kAccum)) {
            PassTimer pt(s, st, kPassGcbc);
            const int64_t F = s->F[0];
            const int mask = (s->cfg.nbc[0][0] == CS_BC_NON_REFLECTIVE ? 1 : 0) |
                             (s->cfg.nbc[1][0] == CS_BC_NON_REFLECTIVE ? 2 : 0);
            k_gcbc_x<float><<<(unsigned)((2 * F + 127) / 128), 128, 0, st>>>(s->rhs32, s->drva, qin, s->d.lxi,
                                                                           s->d.lmx, F, mask, s->ph,
                                                                           1.0 / s->ph.J, 0.0, 0.0, 0.0);
            CSB_CUDA(cudaGetLastError());
        }
    }
    return CS_OK;
}

// The compact filter over every active axis, in place on the state q.
static int filter_pass(cs_solver *s, double *q, cudaStream_t st) {
    for (int a = 0; a < 3; ++a) {
        if (!s->active[a]) continue;
        PassTimer pt(s, st, kPassFilter);
        if (int rc = filter_state(q, a, *s->ftab[a], s->d, s->cfg.alpha_f, st)) return rc;
    }
    return CS_OK;
}

static int run_step(cs_solver *s, double *q, double dt, cudaStream_t st) {
    const bool cfl = !(dt > 0.0);
    if (cfl) CSB_CUDA(cudaMemsetAsync(s->dtacc, 0, 2 * sizeof(unsigned long long), st));
    for (int k = 0; k < 4; ++k) {
        RkParams rk{};
        rk.div = 4 - k;
        rk.dt_fixed = cfl ? 0.0 : dt;
        rk.cfl = s->cfg.cfl;
        rk.dtacc = s->dtacc;
        rk.dt_out = k == 0 ? s->dt_dev : nullptr;
        const double *qin = k == 0 ? q : s->q1;
        double *qout = k == 3 ? q : s->q1;
        if (s->mixed) {
            if (int rc = run_stage_mx(s, qin, q, qout, false, &rk, k == 0, k < 3, st)) return rc;
            if (k == 3 && s->cfg.filter == CS_FILTER_STEP)
                if (int rc = filter_pass(s, q, st)) return rc;
            continue;
        }
        if (int rc = run_stage(s, qin, q, qout, nullptr, &rk, cfl && k == 0, st)) return rc;
        if (s->cfg.filter == CS_FILTER_STAGE)
            if (int rc = filter_pass(s, qout, st)) return rc;
    }
    if (s->cfg.filter == CS_FILTER_STEP)
        if (int rc = filter_pass(s, q, st)) return rc;
    return CS_OK;
}

}  // namespace csb

extern "C" {

int cs_solver_create(cs_solver **out, const cs_solver_config *cfg) {
    if (!out || !cfg) return set_error(CS_ERR_INVALID, "null argument");
    *out = nullptr;
    if (cfg->lxi < 1 || cfg->let < 1 || cfg->lze < 1) return set_error(CS_ERR_INVALID, "dims");
    if (!(cfg->dx > 0 && cfg->dy > 0 && cfg->dz > 0)) return set_error(CS_ERR_INVALID, "grid spacing");
    auto *s = new cs_solver();
    s->cfg = *cfg;
    s->d = cs_dcomp{cfg->lxi * cfg->let * cfg->lze, cfg->lxi, cfg->let, cfg->lze};
    for (int f = 0; f < 2; ++f)
        for (int a = 0; a < 3; ++a) {
            s->ndf[f][a] = bc_ndf(cfg->nbc[f][a]);
            if (s->ndf[f][a] < 0) { delete s; return set_error(CS_ERR_INVALID, "boundary code %d", cfg->nbc[f][a]); }
        }
    for (int a = 0; a < 3; ++a) {
        const int n = llen(s->d, a);
        s->F[a] = fsize(s->d, a);
        if (n == 1) continue;  // degenerate axis: no derivative along it
        if (s->ndf[0][a] != s->ndf[1][a]) {
            delete s;
            return set_error(CS_ERR_UNSUPPORTED, "axis %d: a single rank needs both faces periodic or both physical", a);
        }
        if (n < 5 || (s->ndf[0][a] && n < kLmd)) { delete s; return set_error(CS_ERR_UNSUPPORTED, "axis %d too short", a); }
        s->tab[a] = s->tables.get(n, kDeriv, s->ndf[0][a], s->ndf[1][a], 0.0);
        if (!s->tab[a]) { delete s; return CS_ERR_UNSUPPORTED; }
        if (s->tab[a]->lt > 16) {
            delete s;
            return set_error(CS_ERR_UNSUPPORTED, "axis %d: the fused passes take lines of at most 512 points", a);
        }
        s->active[a] = 1;
    }
    if (cfg->precision != CS_PREC_FP64 && cfg->precision != CS_PREC_MIXED && cfg->precision != CS_PREC_MIXED_F32) {
        delete s;
        return set_error(CS_ERR_INVALID, "precision %d", cfg->precision);
    }
    if (cfg->refine < CS_REFINE_NONE || cfg->refine > CS_REFINE_FLUX) {
        delete s;
        return set_error(CS_ERR_INVALID, "refine %d", cfg->refine);
    }
    if (cfg->filter < CS_FILTER_NONE || cfg->filter > CS_FILTER_STAGE) {
        delete s;
        return set_error(CS_ERR_INVALID, "filter %d", cfg->filter);
    }
    if (cfg->filter != CS_FILTER_NONE) {
        if (!(cfg->alpha_f > -0.5 && cfg->alpha_f <= 0.5)) {
            delete s;
            return set_error(CS_ERR_INVALID, "alpha_f %g: the filter needs -0.5 < alpha_f <= 0.5", cfg->alpha_f);
        }
        if (cfg->filter == CS_FILTER_STAGE && cfg->precision != CS_PREC_FP64) {
            delete s;
            return set_error(CS_ERR_UNSUPPORTED, "the mixed form filters after every step only");
        }
        for (int a = 0; a < 3; ++a) {
            if (!s->active[a]) continue;
            if (llen(s->d, a) < 7) { delete s; return set_error(CS_ERR_UNSUPPORTED, "axis %d: the filter needs 7 points", a); }
            s->ftab[a] = s->tables.get(llen(s->d, a), kFilter, s->ndf[0][a], s->ndf[1][a], cfg->alpha_f);
            if (!s->ftab[a] || s->ftab[a]->lt > 16) {
                delete s;
                return set_error(CS_ERR_UNSUPPORTED, "axis %d: no filter tables for this line", a);
            }
        }
    }
    if (cfg->schedule < CS_SCHED_AUTO || cfg->schedule > CS_SCHED_TMA) {
        delete s;
        return set_error(CS_ERR_INVALID, "schedule %d", cfg->schedule);
    }
    int smem_max = 0, dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        smem_max = 227 * 1024;
    const size_t elem = cfg->precision != CS_PREC_FP64 ? sizeof(float) : sizeof(double);
    for (int k = 0; k < 2; ++k)
        for (int a = 0; a < 3; ++a) {
            const int t = cfg->tile[k][a];
            if (t != 0 && t != 8 && !(t == 16 && a > 0)) {
                delete s;
                return set_error(CS_ERR_INVALID, "tile[%d][%d] = %d: 8, or 16 for y/z, or 0", k, a, t);
            }
            if (t) s->tile[k][a] = t;
            // the mixed form compiles 16-line tiles for the z axis only
            if (cfg->precision != CS_PREC_FP64 && a == 1) s->tile[k][a] = 8;
            if (!s->active[a]) continue;
            // a tile holds 4 (gradient) or 5 (flux) staged fields of full lines
            const size_t slot = (size_t)32 * s->tab[a]->lt + 1;
            auto bytes = [&](int tl) { return (size_t)(k == 0 ? 4 : 5) * tl * slot * elem; };
            if (bytes(s->tile[k][a]) > (size_t)smem_max) {
                if (t) {
                    delete s;
                    return set_error(CS_ERR_UNSUPPORTED, "tile[%d][%d] = %d needs %zu bytes of shared memory", k, a,
                                     t, bytes(t));
                }
                s->tile[k][a] = 8;
            }
            // producer/consumer form: two staging buffers of pl_tile_for() lines
            const bool pl_fits = 2 * bytes(pl_tile_for(s->tab[a]->lt, elem == 4)) <= (size_t)smem_max;
            if (cfg->schedule == CS_SCHED_PIPELINE && !pl_fits) {
                delete s;
                return set_error(CS_ERR_UNSUPPORTED, "axis %d: the pipelined %s passes need %zu bytes of shared "
                                 "memory", a, elem == 8 ? "FP64" : "mixed",
                                 2 * bytes(pl_tile_for(s->tab[a]->lt, elem == 4)));
            }
            s->pl[k][a] = cfg->schedule == CS_SCHED_PIPELINE && pl_fits;
            s->can[k][a] = (bytes(8) <= (size_t)smem_max ? 1 : 0) |
                           (a > 0 && !(elem == 4 && a == 1) && bytes(16) <= (size_t)smem_max ? 2 : 0) |
                           (pl_fits ? 4 : 0);
            if (k == 0) {
                TmaGeom g;
                size_t tb = 0;
                if (cfg->precision == CS_PREC_FP64 ? tma_grad_geometry(a, s->d, s->tab[a]->lt, smem_max, g, tb)
                                                   : tma_grad_mx_geometry(a, s->d, s->tab[a]->lt, smem_max, g, tb))
                    s->can[0][a] |= 8;
                s->tma[a] = cfg->schedule == CS_SCHED_TMA && (s->can[0][a] & 8);
            }
            if (!s->pl[k][a] && !(k == 0 && s->tma[a]) && bytes(s->tile[k][a]) > (size_t)smem_max) {
                delete s;
                return set_error(CS_ERR_UNSUPPORTED,
                                 "axis %d: lines of %d points do not fit the fused %s passes (%zu bytes of shared "
                                 "memory per 8-line tile)", a, llen(s->d, a), elem == 8 ? "FP64" : "mixed", bytes(8));
            }
        }
    if (cudaDeviceGetAttribute(&s->nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) s->nsm = 1;
    compute_interface_coeffs(s->cf);
    uniform_phys(*cfg, s->ph);
    const int64_t lmx = s->d.lmx;
    bool ok = cudaMalloc(&s->q1, 5 * lmx * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&s->grad, 12 * lmx * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&s->rhs, 5 * lmx * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&s->drva, 10 * s->F[0] * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&s->dtacc, 2 * sizeof(unsigned long long)) == cudaSuccess &&
              cudaMalloc(&s->dt_dev, sizeof(double)) == cudaSuccess &&
              cudaMalloc(&s->err, sizeof(int)) == cudaSuccess;
    if (!ok) {
        cs_solver_destroy(s);
        return set_error(CS_ERR_ALLOC, "solver scratch allocation failed");
    }
    cudaMemset(s->grad, 0, 12 * lmx * sizeof(double));
    if (cfg->precision != CS_PREC_FP64) {
        s->mixed = true;
        const bool okm = cudaMalloc(&s->sh32, 5 * lmx * sizeof(float)) == cudaSuccess &&
                         cudaMalloc(&s->grad32, 12 * lmx * sizeof(float)) == cudaSuccess &&
                         cudaMalloc(&s->rhs32, 5 * lmx * sizeof(float)) == cudaSuccess;
        if (!okm) {
            cs_solver_destroy(s);
            return set_error(CS_ERR_ALLOC, "mixed-precision scratch allocation failed");
        }
        cudaMemset(s->grad32, 0, 12 * lmx * sizeof(float));
    }
    cudaMemset(s->dtacc, 0, 2 * sizeof(unsigned long long));
    cudaMemset(s->dt_dev, 0, sizeof(double));
    cudaMemset(s->err, 0, sizeof(int));
    *out = s;
    return CS_OK;
}

int cs_solver_profile_begin(cs_solver *s) {
    if (!s) return set_error(CS_ERR_INVALID, "null argument");
    for (auto &p : s->prof) {
        s->event_pool.push_back(p.second.first);
        s->event_pool.push_back(p.second.second);
    }
    s->prof.clear();
    s->profiling = true;
    return CS_OK;
}

int cs_solver_profile_end(cs_solver *s, double ms[CS_PASS_KINDS], int launches[CS_PASS_KINDS]) {
    if (!s || !ms || !launches) return set_error(CS_ERR_INVALID, "null argument");
    s->profiling = false;
    for (int k = 0; k < kPassKinds; ++k) { ms[k] = 0.0; launches[k] = 0; }
    for (auto &p : s->prof) {
        CSB_CUDA(cudaEventSynchronize(p.second.second));
        float t = 0.f;
        CSB_CUDA(cudaEventElapsedTime(&t, p.second.first, p.second.second));
        ms[p.first] += t;
        launches[p.first] += 1;
    }
    return CS_OK;
}

int cs_solver_autotune(cs_solver *s, const double *q, int reps, int choice[2][3], void *stream) {
    if (!s || !q || reps < 1) return set_error(CS_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t bytes = (size_t)5 * s->d.lmx * sizeof(double);
    double *scratch = nullptr;
    if (cudaMalloc(&scratch, bytes) != cudaSuccess) return set_error(CS_ERR_ALLOC, "autotune scratch allocation failed");
    const int saved_tile[2][3] = {{s->tile[0][0], s->tile[0][1], s->tile[0][2]},
                                  {s->tile[1][0], s->tile[1][1], s->tile[1][2]}};
    const int saved_pl[2][3] = {{s->pl[0][0], s->pl[0][1], s->pl[0][2]}, {s->pl[1][0], s->pl[1][1], s->pl[1][2]}};
    const int saved_tma[3] = {s->tma[0], s->tma[1], s->tma[2]};
    if (s->graph) { cudaGraphExecDestroy(s->graph); s->graph = nullptr; }
    // candidates, applied to every pass where feasible: tile 8, tile 16, pipelined, TMA-staged (gradients)
    double best[2][3];
    int pick[2][3];
    for (int k = 0; k < 2; ++k)
        for (int a = 0; a < 3; ++a) { best[k][a] = 1e300; pick[k][a] = 8; }
    int rc = CS_OK;
    double dt = 0.0;
    CSB_CUDA(cudaMemcpyAsync(scratch, q, bytes, cudaMemcpyDeviceToDevice, st));
    if ((rc = run_step(s, scratch, 0.0, st)) == CS_OK) {
        CSB_CUDA(cudaStreamSynchronize(st));
        cs_solver_last_dt(s, &dt);
    }
    // per-point metrics run the one-phase kernels, or the TMA gradient passes
    // (the metric-reading CFL reduction of the first then stays one-phase)
    const int allowed = s->fm.xim ? 11 : 15;
    for (int c = 0; c < 4 && rc == CS_OK && dt > 0.0; ++c) {
        const int bit = 1 << c;
        if (!(allowed & bit)) continue;
        for (int k = 0; k < 2; ++k)
            for (int a = 0; a < 3; ++a) {
                const bool ok = (s->can[k][a] & bit) != 0;
                s->pl[k][a] = ok && c == 2;
                if (k == 0) s->tma[a] = ok && c == 3;
                s->tile[k][a] = ok && c == 1 ? 16 : 8;
                if (!(s->can[k][a] & 1) && !s->pl[k][a]) s->tile[k][a] = saved_tile[k][a];
            }
        // one untimed step first: the first launch of a kernel may load its
        // module (lazy loading), which must not count against the schedule
        rc = run_step(s, scratch, dt, st);
        if (rc) break;
        cs_solver_profile_begin(s);
        for (int r = 0; r < reps + 1 && rc == CS_OK; ++r) rc = run_step(s, scratch, dt, st);
        double ms[kPassKinds];
        int n[kPassKinds];
        if (rc == CS_OK) rc = cs_solver_profile_end(s, ms, n);
        if (rc) break;
        for (int k = 0; k < 2; ++k)
            for (int a = 0; a < 3; ++a) {
                const int kind = (k == 0 ? kPassGradX : kPassFluxX) + a;
                if (!(s->can[k][a] & bit) || !n[kind]) continue;
                const double t = ms[kind] / n[kind];
                if (t < best[k][a]) { best[k][a] = t; pick[k][a] = c == 3 ? 1 : (c == 2 ? 0 : (c == 1 ? 16 : 8)); }
            }
    }
    cudaFree(scratch);
    if (rc || !(dt > 0.0)) {
        for (int k = 0; k < 2; ++k)
            for (int a = 0; a < 3; ++a) {
                s->tile[k][a] = saved_tile[k][a];
                s->pl[k][a] = saved_pl[k][a];
                if (k == 0) s->tma[a] = saved_tma[a];
            }
        return rc ? rc : set_error(CS_ERR_STATE, "autotune: no time step from the state");
    }
    for (int k = 0; k < 2; ++k)
        for (int a = 0; a < 3; ++a) {
            s->pl[k][a] = pick[k][a] == 0;
            if (k == 0) s->tma[a] = pick[k][a] == 1;
            s->tile[k][a] = pick[k][a] <= 1 ? 8 : pick[k][a];
            if (choice) choice[k][a] = pick[k][a];
        }
    return CS_OK;
}

int cs_solver_schedule(const cs_solver *s, int choice[2][3]) {
    if (!s || !choice) return set_error(CS_ERR_INVALID, "null argument");
    for (int k = 0; k < 2; ++k)
        for (int a = 0; a < 3; ++a)
            choice[k][a] = s->pl[k][a] ? 0 : (k == 0 && s->tma[a] ? 1 : s->tile[k][a]);
    return CS_OK;
}

int cs_solver_set_metrics(cs_solver *s, const double *xim, const double *etm, const double *zem,
                          const double *yaco) {
    if (!s) return set_error(CS_ERR_INVALID, "null argument");
    const int given = (xim != nullptr) + (etm != nullptr) + (zem != nullptr) + (yaco != nullptr);
    if (given != 0 && given != 4) return set_error(CS_ERR_INVALID, "give all four metric arrays or none");
    if (given && s->mixed) return set_error(CS_ERR_UNSUPPORTED, "per-point metrics run in FP64 only");
    if (given && s->cfg.schedule == CS_SCHED_PIPELINE)
        return set_error(CS_ERR_UNSUPPORTED, "per-point metrics run the one-phase kernels only");
    if (given)
        for (int k = 0; k < 2; ++k)
            for (int a = 0; a < 3; ++a)
                if (s->active[a] && s->pl[k][a])
                    return set_error(CS_ERR_UNSUPPORTED, "axis %d: per-point metrics run the one-phase kernels "
                                     "only", a);
    if (s->graph) { cudaGraphExecDestroy(s->graph); s->graph = nullptr; }
    s->fm = FieldMet{xim, etm, zem, yaco};
    return CS_OK;
}

int cs_solver_destroy(cs_solver *s) {
    if (!s) return CS_OK;
    for (auto &p : s->prof) {
        cudaEventDestroy(p.second.first);
        cudaEventDestroy(p.second.second);
    }
    for (auto e : s->event_pool) cudaEventDestroy(e);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    for (void *p : {(void *)s->q1, (void *)s->grad, (void *)s->rhs, (void *)s->drva, (void *)s->dtacc,
                    (void *)s->dt_dev, (void *)s->qhost_dev, (void *)s->sh32, (void *)s->grad32,
                    (void *)s->rhs32, (void *)s->err})
        if (p) cudaFree(p);
    delete s;
    return CS_OK;
}

__global__ void k_widen(const float *__restrict__ a, double *__restrict__ b, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i];
}

int cs_solver_rhs(cs_solver *s, const double *q, double *rhs, void *stream) {
    if (!s || !q || !rhs) return set_error(CS_ERR_INVALID, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (s->mixed) {
        // build the shadow from q, assemble the FP32 RHS, widen it to FP64
        if (int rc = run_stage_mx(s, q, q, nullptr, true, nullptr, true, false, st)) return rc;
        const int64_t n = 5 * s->d.lmx;
        k_widen<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(s->rhs32, rhs, n);
        CSB_CUDA(cudaGetLastError());
        return CS_OK;
    }
    return run_stage(s, q, q, nullptr, rhs, nullptr, false, st);
}

int cs_solver_stage(cs_solver *s, int k, const double *qn, const double *qin, double *qout, double dt,
                    void *stream) {
    if (!s || !qn || !qin || !qout || k < 0 || k > 3 || !(dt > 0.0))
        return set_error(CS_ERR_INVALID, "bad argument");
    RkParams rk{};
    rk.div = 4 - k;
    rk.dt_fixed = dt;
    rk.cfl = s->cfg.cfl;
    rk.dtacc = s->dtacc;
    if (s->mixed) return run_stage_mx(s, qin, qn, qout, false, &rk, true, false, (cudaStream_t)stream);
    return run_stage(s, qin, qn, qout, nullptr, &rk, false, (cudaStream_t)stream);
}

int cs_solver_step(cs_solver *s, double *q, double dt, void *stream) {
    if (!s || !q) return set_error(CS_ERR_INVALID, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (s->cfg.use_graph && !s->profiling) {
        if (!s->graph || s->graph_q != q || s->graph_dt != dt || s->graph_stream != st) {
            if (s->graph) { cudaGraphExecDestroy(s->graph); s->graph = nullptr; }
            cudaStream_t cap;
            CSB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            cudaGraph_t g;
            CSB_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
            int rc = run_step(s, q, dt, cap);
            cudaError_t e = cudaStreamEndCapture(cap, &g);
            cudaStreamDestroy(cap);
            if (rc) return rc;
            if (e != cudaSuccess) return check_cuda(e, "cudaStreamEndCapture");
            e = cudaGraphInstantiate(&s->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) { s->graph = nullptr; return check_cuda(e, "cudaGraphInstantiate"); }
            s->graph_q = q;
            s->graph_dt = dt;
            s->graph_stream = st;
        }
        CSB_CUDA(cudaGraphLaunch(s->graph, st));
        return CS_OK;
    }
    return run_step(s, q, dt, st);
}

int cs_solver_step_host(cs_solver *s, const double *q_in_host, double *q_out_host, double dt,
                        void *stream) {
    if (!s || !q_in_host || !q_out_host) return set_error(CS_ERR_INVALID, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t bytes = (size_t)5 * s->d.lmx * sizeof(double);
    if (!s->qhost_dev && cudaMalloc(&s->qhost_dev, bytes) != cudaSuccess) {
        s->qhost_dev = nullptr;
        return set_error(CS_ERR_ALLOC, "state allocation failed");
    }
    CSB_CUDA(cudaMemcpyAsync(s->qhost_dev, q_in_host, bytes, cudaMemcpyHostToDevice, st));
    if (int rc = cs_solver_step(s, s->qhost_dev, dt, stream)) return rc;
    CSB_CUDA(cudaMemcpyAsync(q_out_host, s->qhost_dev, bytes, cudaMemcpyDeviceToHost, st));
    CSB_CUDA(cudaStreamSynchronize(st));
    return CS_OK;
}

int cs_solver_last_dt(cs_solver *s, double *dt) {
    if (!s || !dt) return set_error(CS_ERR_INVALID, "null argument");
    CSB_CUDA(cudaMemcpy(dt, s->dt_dev, sizeof(double), cudaMemcpyDeviceToHost));
    int e = 0;
    CSB_CUDA(cudaMemcpy(&e, s->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return set_error(CS_ERR_TIMEOUT, "a TMA staging copy of a gradient pass did not complete (code %#x)", e);
    return CS_OK;
}

int cs_solver_dt_device(cs_solver *s, double **dt_dev) {
    if (!s || !dt_dev) return set_error(CS_ERR_INVALID, "null argument");
    *dt_dev = s->dt_dev;
    return CS_OK;
}

int cs_tgv_init(double *q, int lxi, int let, int lze, double mach, double noise_amp, uint64_t seed,
                void *stream) {
    if (!q || lxi < 1 || let < 1 || lze < 1) return set_error(CS_ERR_INVALID, "bad argument");
    const int64_t lmx = (int64_t)lxi * let * lze;
    const double tp = 6.283185307179586476925286766559;
    k_tgv<<<(unsigned)((lmx + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        q, lxi, let, lmx, mach, noise_amp, seed, tp / lxi, tp / let, tp / lze);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

}  // extern "C"
