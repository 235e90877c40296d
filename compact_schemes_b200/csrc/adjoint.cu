// adjoint.cu -- tangent-linear and adjoint RHS / RK step, checkpointed
// reverse sweep (cs_rhs_jvp, cs_rhs_vjp, cs_step_jvp, cs_step_vjp,
// cs_adjoint_gradient) and host-side pointwise linearizations.
//
// With q^(-1) = q^n and c_k = dt J / (4 - k), the RK step is
//     q^(k) = q^n - c_k R(q^(k-1)),  k = 0..3,  q^(n+1) = q^(3),
// with dt held fixed (the time steps of the reference trajectory).  Its
// adjoint, given lambda_3 = dJ/dq^(n+1):
//     lambda_n = sum_k lambda_k - c_0 R'(q^n)^T lambda_0,
//     lambda_(k-1) = -c_k R'(q^(k-1))^T lambda_k.
// R(q) = sum_a D_a F_a(q, G), G_b = D_b phi(q), so
//     R'(q) dq = sum_a D_a [F_q dq + F_G dG],  dG_b = D_b (phi_q dq),
//     R'(q)^T l = F_q^T mu + phi_q^T sum_b D_b^T (F_G^T mu)_b,  mu_a = D_a^T l.
#include <cstring>
#include <vector>

#include "adjoint.cuh"

struct cs_adjoint {
    cs_solver_config cfg{};
    cs_solver *fwd = nullptr;
    cs_dcomp d{};
    int64_t lmx = 0;
    int64_t F[3] = {0, 0, 0};
    int ndf[2][3] = {{0, 0, 0}, {0, 0, 0}};
    int active[3] = {0, 0, 0};
    int amask = 0;
    int nsm = 1;
    csb::TableCache tables;
    const csb::DeviceTables *tab[3] = {nullptr, nullptr, nullptr};
    const csb::DeviceTables *tabT[3] = {nullptr, nullptr, nullptr};
    csb::Coeffs cf{};
    csb::Phys ph{};
    csb::AdjPoint ap{};
    // scratch: G, dG / Gbar [12], phi4 [4], F15 [15], qbar [5], t1, t2, t3 [5], partial sums
    double *G = nullptr, *G2 = nullptr, *phi4 = nullptr, *F15 = nullptr, *qbar = nullptr;
    double *t1 = nullptr, *t2 = nullptr, *t3 = nullptr, *partial = nullptr;
    unsigned long long *dtacc = nullptr;
    // non-reflective GCBC on the x faces: face mask, forward / tangent x-derivative
    // terms at the faces [2][5][F], face adjoint of q, lambda for the x solve [5][lmx]
    int gcbc_mask = 0;
    double *rf = nullptr, *drf = nullptr, *qbf = nullptr, *lamx = nullptr;
    // sweep buffer of cs_adjoint_gradient, kept for the next call
    double *sweep = nullptr;
    size_t sweep_bytes = 0;
};

namespace csb {

constexpr int kPointBlocks = 148 * 8;

static int lines(cs_adjoint *a, int axis, bool trans, const double *in, int64_t in_fs, double *out, int64_t out_fs,
                 int nf, bool accum, double scale, cudaStream_t st) {
    const DeviceTables *t = trans ? a->tabT[axis] : a->tab[axis];
    const dim3 grid((unsigned)((a->F[axis] + 7) / 8), (unsigned)nf);
    const int nstart = a->ndf[0][axis], nend = a->ndf[1][axis];
#define CSB_LINES(LT, AX)                                                                                    \
    do {                                                                                                     \
        if (trans)                                                                                           \
            k_lines<LT, AX, true><<<grid, 256, 0, st>>>(in, in_fs, out, out_fs, accum, scale, t->t64,         \
                                                        a->d.lxi, a->d.let, a->F[AX], nstart, nend, a->cf); \
        else                                                                                                 \
            k_lines<LT, AX, false><<<grid, 256, 0, st>>>(in, in_fs, out, out_fs, accum, scale, t->t64,        \
                                                         a->d.lxi, a->d.let, a->F[AX], nstart, nend, a->cf); \
    } while (0)
#define CSB_LINES_AX(LT)                       \
    do {                                       \
        if (axis == 0) CSB_LINES(LT, 0);       \
        else if (axis == 1) CSB_LINES(LT, 1);  \
        else CSB_LINES(LT, 2);                 \
    } while (0)
    switch (t->lt) {
        case 2: CSB_LINES_AX(2); break;
        case 4: CSB_LINES_AX(4); break;
        case 8: CSB_LINES_AX(8); break;
        case 16: CSB_LINES_AX(16); break;
        default: return set_error(CS_ERR_UNSUPPORTED, "adjoint: lines of more than 512 points");
    }
#undef CSB_LINES_AX
#undef CSB_LINES
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

// The compact filter (Gaitonde-Visbal, filter_rhs) or its transpose along axis.
static int filter_lines(cs_adjoint *a, int axis, bool trans, double af, const double *in, double *out, int nf,
                        bool accum, cudaStream_t st) {
    const int n = axis == 0 ? a->d.lxi : (axis == 1 ? a->d.let : a->d.lze);
    const int nstart = a->ndf[0][axis], nend = a->ndf[1][axis];
    const DeviceTables *t = a->tables.get(n, trans ? kFilterT : kFilter, nstart, nend, af);
    if (!t) return CS_ERR_UNSUPPORTED;
    const dim3 grid((unsigned)((a->F[axis] + 7) / 8), (unsigned)nf);
    const int64_t lmx = a->lmx;
#define CSB_FLINES(LT, AX)                                                                                      \
    do {                                                                                                        \
        if (trans)                                                                                              \
            k_lines<LT, AX, true, true><<<grid, 256, 0, st>>>(in, lmx, out, lmx, accum, 1.0, t->t64, a->d.lxi,   \
                                                              a->d.let, a->F[AX], nstart, nend, a->cf, af);     \
        else                                                                                                    \
            k_lines<LT, AX, false, true><<<grid, 256, 0, st>>>(in, lmx, out, lmx, accum, 1.0, t->t64, a->d.lxi,  \
                                                               a->d.let, a->F[AX], nstart, nend, a->cf, af);    \
    } while (0)
#define CSB_FLINES_AX(LT)                       \
    do {                                        \
        if (axis == 0) CSB_FLINES(LT, 0);       \
        else if (axis == 1) CSB_FLINES(LT, 1);  \
        else CSB_FLINES(LT, 2);                 \
    } while (0)
    switch (t->lt) {
        case 2: CSB_FLINES_AX(2); break;
        case 4: CSB_FLINES_AX(4); break;
        case 8: CSB_FLINES_AX(8); break;
        case 16: CSB_FLINES_AX(16); break;
        default: return set_error(CS_ERR_UNSUPPORTED, "adjoint: lines of more than 512 points");
    }
#undef CSB_FLINES_AX
#undef CSB_FLINES
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

static int grads(cs_adjoint *a, const double *q, cudaStream_t st) {
    for (int ax = 0; ax < 3; ++ax) {
        if (!a->active[ax]) continue;
        PassArgs p{};
        p.lmx = a->lmx;
        p.lxi = a->d.lxi;
        p.let = a->d.let;
        p.F = a->F[ax];
        p.nstart = a->ndf[0][ax];
        p.nend = a->ndf[1][ax];
        p.tl = 8;
        p.pl = 0;
        p.nsm = a->nsm;
        p.viscous = a->cfg.viscous;
        p.tab = a->tab[ax];
        p.cf = a->cf;
        p.ph = a->ph;
        p.grad = a->G;
        p.rhs = nullptr;
        p.dtacc = a->dtacc;
        int rc = ax == 0 ? launch_grad<0>(p, q, false, st) : (ax == 1 ? launch_grad<1>(p, q, false, st)
                                                                      : launch_grad<2>(p, q, false, st));
        if (rc) return rc;
    }
    return CS_OK;
}

static unsigned face_blocks(const cs_adjoint *a) { return (unsigned)((2 * a->F[0] + 127) / 128); }

// rf = (d/dxi F_x(q, G)) at the x faces; G must be current (viscous).
static int gcbc_forward_faces(cs_adjoint *a, const double *q, cudaStream_t st) {
    const int64_t lmx = a->lmx;
    if (a->cfg.viscous) k_flux_x_eval<true><<<kPointBlocks, 256, 0, st>>>(q, a->G, a->F15, a->ap);
    else k_flux_x_eval<false><<<kPointBlocks, 256, 0, st>>>(q, nullptr, a->F15, a->ap);
    CSB_CUDA(cudaGetLastError());
    if (int rc = lines(a, 0, false, a->F15, lmx, a->F15 + 5 * lmx, lmx, 5, false, 1.0, st)) return rc;
    k_xface_extract<<<face_blocks(a), 128, 0, st>>>(a->F15 + 5 * lmx, a->rf, a->d.lxi, lmx, a->F[0]);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

static int rhs_jvp(cs_adjoint *a, const double *q, const double *dq, double *dR, cudaStream_t st) {
    const int64_t lmx = a->lmx;
    const bool visc = a->cfg.viscous != 0;
    if (visc) {
        if (int rc = grads(a, q, st)) return rc;
        k_prim_tan<<<kPointBlocks, 256, 0, st>>>(q, dq, a->phi4, lmx);
        CSB_CUDA(cudaGetLastError());
        for (int b = 0; b < 3; ++b)
            if (a->active[b])
                if (int rc = lines(a, b, false, a->phi4, lmx, a->G2 + 4 * b * lmx, lmx, 4, false, 1.0, st)) return rc;
        k_flux_tan<true><<<kPointBlocks, 256, 0, st>>>(q, a->G, dq, a->G2, a->F15, a->ap, a->amask);
    } else {
        k_flux_tan<false><<<kPointBlocks, 256, 0, st>>>(q, nullptr, dq, nullptr, a->F15, a->ap, a->amask);
    }
    CSB_CUDA(cudaGetLastError());
    bool first = true;
    for (int ax = 0; ax < 3; ++ax) {
        if (!a->active[ax]) continue;
        if (int rc = lines(a, ax, false, a->F15 + 5 * ax * lmx, lmx, dR, lmx, 5, !first, 1.0, st)) return rc;
        if (ax == 0 && a->gcbc_mask) {
            k_xface_extract<<<face_blocks(a), 128, 0, st>>>(dR, a->drf, a->d.lxi, lmx, a->F[0]);
            CSB_CUDA(cudaGetLastError());
        }
        first = false;
    }
    if (first) CSB_CUDA(cudaMemsetAsync(dR, 0, 5 * lmx * sizeof(double), st));
    if (a->gcbc_mask) {
        if (int rc = gcbc_forward_faces(a, q, st)) return rc;
        k_gcbc_tan<<<face_blocks(a), 128, 0, st>>>(q, a->rf, dq, a->drf, dR, a->d.lxi, lmx, a->F[0], a->gcbc_mask,
                                                   a->ap.ph);
        CSB_CUDA(cudaGetLastError());
    }
    return CS_OK;
}

// w = scale * R'(q)^T lam; out = w (if set); acc_out = (acc_in or acc_out) + w (if set)
static int rhs_vjp(cs_adjoint *a, const double *q, const double *lam, double *out, double scale, cudaStream_t st,
                   const double *acc_in = nullptr, double *acc_out = nullptr) {
    const int64_t lmx = a->lmx;
    const bool visc = a->cfg.viscous != 0;
    if (visc)
        if (int rc = grads(a, q, st)) return rc;
    const double *lam_x = lam;
    if (a->gcbc_mask) {
        // the x-derivative term at the faces also feeds the GCBC correction
        if (int rc = gcbc_forward_faces(a, q, st)) return rc;
        CSB_CUDA(cudaMemcpyAsync(a->lamx, lam, 5 * lmx * sizeof(double), cudaMemcpyDeviceToDevice, st));
        k_gcbc_adj<<<face_blocks(a), 128, 0, st>>>(q, a->rf, lam, a->lamx, a->qbf, a->d.lxi, lmx, a->F[0],
                                                   a->gcbc_mask, a->ap.ph);
        CSB_CUDA(cudaGetLastError());
        lam_x = a->lamx;
    }
    for (int ax = 0; ax < 3; ++ax)
        if (a->active[ax])
            if (int rc = lines(a, ax, true, ax == 0 ? lam_x : lam, lmx, a->F15 + 5 * ax * lmx, lmx, 5, false, 1.0, st))
                return rc;
    if (visc) k_flux_adj<true><<<kPointBlocks, 256, 0, st>>>(q, a->G, a->F15, a->qbar, a->G2, a->ap, a->amask);
    else k_flux_adj<false><<<kPointBlocks, 256, 0, st>>>(q, nullptr, a->F15, a->qbar, nullptr, a->ap, a->amask);
    CSB_CUDA(cudaGetLastError());
    if (a->gcbc_mask) {
        k_xface_add<<<face_blocks(a), 128, 0, st>>>(a->qbf, a->qbar, a->d.lxi, lmx, a->F[0], a->gcbc_mask);
        CSB_CUDA(cudaGetLastError());
    }
    bool have_pb = false;
    if (visc) {
        for (int b = 0; b < 3; ++b) {
            if (!a->active[b]) continue;
            if (int rc = lines(a, b, true, a->G2 + 4 * b * lmx, lmx, a->phi4, lmx, 4, have_pb, 1.0, st)) return rc;
            have_pb = true;
        }
    }
    k_prim_adj<<<kPointBlocks, 256, 0, st>>>(q, a->qbar, a->phi4, out, scale, lmx, have_pb ? 1 : 0, acc_in,
                                             acc_out);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

static double stage_c(const cs_adjoint *a, int k, double dt) { return dt / (4 - k) * a->ph.J; }


}  // namespace csb

using namespace csb;

extern "C" {

int cs_adjoint_destroy(cs_adjoint *a) {
    if (!a) return set_error(CS_ERR_INVALID, "null argument");
    if (a->fwd) cs_solver_destroy(a->fwd);
    for (double *p : {a->G, a->G2, a->phi4, a->F15, a->qbar, a->t1, a->t2, a->t3, a->partial, a->rf, a->drf, a->qbf,
                      a->lamx, a->sweep})
        cudaFree(p);
    cudaFree(a->dtacc);
    delete a;
    return CS_OK;
}

int cs_adjoint_create(cs_adjoint **out, const cs_solver_config *cfg) {
    if (!out || !cfg) return set_error(CS_ERR_INVALID, "null argument");
    *out = nullptr;
    if (cfg->precision != CS_PREC_FP64) return set_error(CS_ERR_UNSUPPORTED, "adjoint: FP64 only");
    if (cfg->filter != CS_FILTER_NONE)
        return set_error(CS_ERR_UNSUPPORTED, "adjoint: the step map has no filter (cs_adjoint_filter applies it)");
    auto *a = new cs_adjoint();
    a->cfg = *cfg;
    a->cfg.use_graph = 0;  // the stages run with per-step time steps
    if (int rc = cs_solver_create(&a->fwd, &a->cfg)) { delete a; return rc; }
    a->d = cs_dcomp{cfg->lxi * cfg->let * cfg->lze, cfg->lxi, cfg->let, cfg->lze};
    a->lmx = (int64_t)cfg->lxi * cfg->let * cfg->lze;
    const int n[3] = {cfg->lxi, cfg->let, cfg->lze};
    a->F[0] = (int64_t)cfg->let * cfg->lze;
    a->F[1] = (int64_t)cfg->lxi * cfg->lze;
    a->F[2] = (int64_t)cfg->lxi * cfg->let;
    for (int ax = 0; ax < 3; ++ax) {
        a->ndf[0][ax] = bc_ndf(cfg->nbc[0][ax]);
        a->ndf[1][ax] = bc_ndf(cfg->nbc[1][ax]);
        if (n[ax] == 1) continue;
        if (n[ax] > 512) { cs_adjoint_destroy(a); return set_error(CS_ERR_UNSUPPORTED, "adjoint: lines of at most 512 points"); }
        a->tab[ax] = a->tables.get(n[ax], kDeriv, a->ndf[0][ax], a->ndf[1][ax], 0.0);
        a->tabT[ax] = a->tables.get(n[ax], kDerivT, a->ndf[0][ax], a->ndf[1][ax], 0.0);
        if (!a->tab[ax] || !a->tabT[ax]) { cs_adjoint_destroy(a); return CS_ERR_UNSUPPORTED; }
        a->active[ax] = 1;
        a->amask |= 1 << ax;
    }
    compute_interface_coeffs(a->cf);
    uniform_phys(a->cfg, a->ph);
    std::memcpy(a->ap.ph.M, a->ph.M, sizeof a->ph.M);
    a->ap.ph.J = a->ph.J;
    a->ap.ph.mu = a->ph.mu;
    for (int c = 0; c < 3; ++c) a->ap.ph.umf[c] = a->ph.umf[c];
    a->ap.lmx = a->lmx;
    a->ap.viscous = cfg->viscous;
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&a->nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) a->nsm = 1;
    const int64_t lmx = a->lmx;
    auto alloc = [&](double **p, int64_t nf) { return cudaMalloc(p, nf * lmx * sizeof(double)) == cudaSuccess; };
    const bool ok = alloc(&a->G, 12) && alloc(&a->G2, 12) && alloc(&a->phi4, 4) && alloc(&a->F15, 15) &&
                    alloc(&a->qbar, 5) && alloc(&a->t1, 5) && alloc(&a->t2, 5) && alloc(&a->t3, 5) &&
                    cudaMalloc(&a->partial, kPointBlocks * sizeof(double)) == cudaSuccess &&
                    cudaMalloc(&a->dtacc, 2 * sizeof(unsigned long long)) == cudaSuccess;
    if (!ok) {
        cs_adjoint_destroy(a);
        return set_error(CS_ERR_ALLOC, "adjoint scratch allocation failed");
    }
    cudaMemset(a->G, 0, 12 * lmx * sizeof(double));
    if (cfg->gcbc && a->active[0])
        a->gcbc_mask = (cfg->nbc[0][0] == CS_BC_NON_REFLECTIVE ? 1 : 0) | (cfg->nbc[1][0] == CS_BC_NON_REFLECTIVE ? 2 : 0);
    if (a->gcbc_mask) {
        const size_t fb = 10 * a->F[0] * sizeof(double);
        if (cudaMalloc(&a->rf, fb) != cudaSuccess || cudaMalloc(&a->drf, fb) != cudaSuccess ||
            cudaMalloc(&a->qbf, fb) != cudaSuccess || !alloc(&a->lamx, 5)) {
            cs_adjoint_destroy(a);
            return set_error(CS_ERR_ALLOC, "adjoint face scratch allocation failed");
        }
    }
    *out = a;
    return CS_OK;
}

int cs_adjoint_deriv(cs_adjoint *a, int axis, int transpose, const double *in, double *out, int nfields,
                     int accumulate, void *stream) {
    if (!a || !in || !out || axis < 0 || axis > 2 || nfields < 1) return set_error(CS_ERR_INVALID, "bad argument");
    if (!a->active[axis]) return set_error(CS_ERR_INVALID, "axis %d has a single point", axis);
    return lines(a, axis, transpose != 0, in, a->lmx, out, a->lmx, nfields, accumulate != 0, 1.0,
                 (cudaStream_t)stream);
}

int cs_adjoint_filter(cs_adjoint *a, int axis, int transpose, double alpha_f, const double *in, double *out,
                      int nfields, int accumulate, void *stream) {
    if (!a || !in || !out || axis < 0 || axis > 2 || nfields < 1) return set_error(CS_ERR_INVALID, "bad argument");
    if (!a->active[axis]) return set_error(CS_ERR_INVALID, "axis %d has a single point", axis);
    if (!(alpha_f > -0.5 && alpha_f < 0.5)) return set_error(CS_ERR_INVALID, "alpha_f %g outside (-1/2, 1/2)", alpha_f);
    return filter_lines(a, axis, transpose != 0, alpha_f, in, out, nfields, accumulate != 0, (cudaStream_t)stream);
}

int cs_rhs_jvp(cs_adjoint *a, const double *q, const double *dq, double *dR, void *stream) {
    if (!a || !q || !dq || !dR) return set_error(CS_ERR_INVALID, "null argument");
    return rhs_jvp(a, q, dq, dR, (cudaStream_t)stream);
}

int cs_rhs_vjp(cs_adjoint *a, const double *q, const double *lam, double *out, void *stream) {
    if (!a || !q || !lam || !out) return set_error(CS_ERR_INVALID, "null argument");
    return rhs_vjp(a, q, lam, out, 1.0, (cudaStream_t)stream);
}

int cs_adjoint_stages(cs_adjoint *a, const double *qn, double dt, double *const stages[4], double *q_next,
                      void *stream) {
    if (!a || !qn || !stages || !(dt > 0.0)) return set_error(CS_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t bytes = 5 * a->lmx * sizeof(double);
    if (stages[0] != qn) CSB_CUDA(cudaMemcpyAsync(stages[0], qn, bytes, cudaMemcpyDeviceToDevice, st));
    for (int k = 0; k < 4; ++k) {
        double *qout = k < 3 ? stages[k + 1] : (q_next ? q_next : a->t3);
        if (int rc = cs_solver_stage(a->fwd, k, stages[0], stages[k], qout, dt, stream)) return rc;
    }
    return CS_OK;
}

int cs_step_jvp(cs_adjoint *a, const double *const stages[4], double dt, const double *dq_n, double *dq_next,
                void *stream) {
    if (!a || !stages || !dq_n || !dq_next) return set_error(CS_ERR_INVALID, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t n5 = 5 * a->lmx;
    const double *cur = dq_n;
    for (int k = 0; k < 4; ++k) {
        double *nxt = k == 3 ? dq_next : (k % 2 == 0 ? a->t1 : a->t2);
        if (int rc = rhs_jvp(a, stages[k], cur, a->t3, st)) return rc;
        // nxt = dq_n - c_k dR
        k_xpay<<<kPointBlocks, 256, 0, st>>>(dq_n, -stage_c(a, k, dt), a->t3, nxt, n5);
        CSB_CUDA(cudaGetLastError());
        cur = nxt;
    }
    return CS_OK;
}

int cs_step_vjp(cs_adjoint *a, const double *const stages[4], double dt, const double *lam_next, double *lam_n,
                void *stream) {
    if (!a || !stages || !lam_next || !lam_n || lam_next == lam_n) return set_error(CS_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    // lam_n = lam_next + w_3 + w_2 + w_1 + w_0, w_k = -c_k R'(q^(k-1))^T lam_k, lam_(k-1) = w_k
    const double *cur = lam_next;
    for (int k = 3; k >= 0; --k) {
        double *w = k == 0 ? nullptr : (k % 2 == 1 ? a->t1 : a->t2);
        if (int rc = rhs_vjp(a, stages[k], cur, w, -stage_c(a, k, dt), st, k == 3 ? lam_next : nullptr, lam_n))
            return rc;
        cur = w;
    }
    return CS_OK;
}

int cs_kinetic_energy(cs_adjoint *a, const double *q, double *J_host, double *dJdq, void *stream) {
    if (!a || !q) return set_error(CS_ERR_INVALID, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    const double dv = a->cfg.dx * a->cfg.dy * a->cfg.dz;
    k_kinetic<<<kPointBlocks, 256, 0, st>>>(q, a->lmx, dv, a->partial, dJdq);
    CSB_CUDA(cudaGetLastError());
    if (J_host) {
        std::vector<double> part(kPointBlocks);
        CSB_CUDA(cudaMemcpyAsync(part.data(), a->partial, kPointBlocks * sizeof(double), cudaMemcpyDeviceToHost, st));
        CSB_CUDA(cudaStreamSynchronize(st));
        double s = 0.0;
        for (double v : part) s += v;
        *J_host = s;
    }
    return CS_OK;
}

int cs_adjoint_gradient_bytes(const cs_adjoint *a, int nsteps, int every, size_t *bytes) {
    if (!a || !bytes || nsteps < 1 || every < 1) return set_error(CS_ERR_INVALID, "bad argument");
    const int nseg = (nsteps + every - 1) / every, segmax = every < nsteps ? every : nsteps;
    *bytes = (size_t)(nseg + 1 + 4LL * segmax + 2) * 5 * a->lmx * sizeof(double);
    return CS_OK;
}

int cs_adjoint_gradient(cs_adjoint *a, const double *q0, int nsteps, const double *dt_host, int every,
                        double *grad_q0, double *J_host, void *stream) {
    if (!a || !q0 || !dt_host || !grad_q0 || nsteps < 1 || every < 1) return set_error(CS_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    const int64_t n5 = 5 * a->lmx;
    const size_t bytes = n5 * sizeof(double);
    const int nseg = (nsteps + every - 1) / every;
    const int segmax = every < nsteps ? every : nsteps;
    // checkpoints, the running state, the stage states of one segment, two adjoint states
    const int64_t nbuf = (int64_t)nseg + 1 + 4LL * segmax + 2;
    if (a->sweep_bytes < (size_t)nbuf * bytes) {
        // a larger sweep than any before: replace the kept buffer (a 4 GB
        // allocation costs far more than a reverse step, so it is reused)
        if (a->sweep) cudaFree(a->sweep);
        a->sweep = nullptr;
        a->sweep_bytes = 0;
        if (cudaMalloc(&a->sweep, nbuf * bytes) != cudaSuccess) {
            a->sweep = nullptr;
            return set_error(CS_ERR_ALLOC, "adjoint checkpoint allocation");
        }
        a->sweep_bytes = (size_t)nbuf * bytes;
    }
    double *buf = a->sweep;
    double *ckpt = buf, *qrun = buf + nseg * n5, *seg = qrun + n5, *lamA = seg + 4LL * segmax * n5, *lamB = lamA + n5;
    int rc = CS_OK;
    auto fail = [&](int r) { return r; };
    // forward sweep: checkpoint every `every` steps
    if (cudaMemcpyAsync(qrun, q0, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return fail(set_error(CS_ERR_CUDA, "state copy"));
    for (int s = 0; s < nsteps; ++s) {
        if (s % every == 0)
            if (cudaMemcpyAsync(ckpt + (s / every) * n5, qrun, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
                return fail(set_error(CS_ERR_CUDA, "checkpoint copy"));
        if ((rc = cs_solver_step(a->fwd, qrun, dt_host[s], stream))) return fail(rc);
    }
    double J = 0.0;
    if ((rc = cs_kinetic_energy(a, qrun, &J, lamA, stream))) return fail(rc);
    // reverse sweep, segment by segment, recomputing the stage states
    double *lam = lamA, *lam_out = lamB;
    for (int g = nseg - 1; g >= 0; --g) {
        const int s0 = g * every, s1 = s0 + every < nsteps ? s0 + every : nsteps;
        for (int s = s0; s < s1; ++s) {
            double *const st4[4] = {seg + (4LL * (s - s0)) * n5, seg + (4LL * (s - s0) + 1) * n5,
                                    seg + (4LL * (s - s0) + 2) * n5, seg + (4LL * (s - s0) + 3) * n5};
            const double *qn = s == s0 ? ckpt + g * n5 : nullptr;
            if (s == s0 && cudaMemcpyAsync(st4[0], qn, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
                return fail(set_error(CS_ERR_CUDA, "segment copy"));
            double *next = s + 1 < s1 ? seg + (4LL * (s + 1 - s0)) * n5 : nullptr;
            if ((rc = cs_adjoint_stages(a, st4[0], dt_host[s], st4, next, stream))) return fail(rc);
        }
        for (int s = s1 - 1; s >= s0; --s) {
            const double *const st4[4] = {seg + (4LL * (s - s0)) * n5, seg + (4LL * (s - s0) + 1) * n5,
                                          seg + (4LL * (s - s0) + 2) * n5, seg + (4LL * (s - s0) + 3) * n5};
            if ((rc = cs_step_vjp(a, st4, dt_host[s], lam, lam_out, stream))) return fail(rc);
            double *t = lam;
            lam = lam_out;
            lam_out = t;
        }
    }
    if (cudaMemcpyAsync(grad_q0, lam, bytes, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return fail(set_error(CS_ERR_CUDA, "gradient copy"));
    if (cudaStreamSynchronize(st) != cudaSuccess) return fail(set_error(CS_ERR_CUDA, "adjoint sweep"));
    if (J_host) *J_host = J;
    return CS_OK;
}

// ---------------------------------------------------------------- host-side pointwise linearizations
static PointPhys point_phys(const double M[9], double J, double mu, const double umf[3]) {
    PointPhys p{};
    for (int i = 0; i < 9; ++i) p.M[i / 3][i % 3] = M[i];
    p.J = J;
    p.mu = mu;
    for (int c = 0; c < 3; ++c) p.umf[c] = umf[c];
    return p;
}

int cs_point_flux(int axis, int viscous, const double q[5], const double G[12], const double M[9], double J,
                  double mu, const double umf[3], double F[5]) {
    if (axis < 0 || axis > 2 || !q || !G || !M || !umf || !F) return set_error(CS_ERR_INVALID, "bad argument");
    const PointPhys p = point_phys(M, J, mu, umf);
    if (viscous) flux_eval<true>(axis, q, G, p, F);
    else flux_eval<false>(axis, q, G, p, F);
    return CS_OK;
}

int cs_point_flux_jvp(int axis, int viscous, const double q[5], const double G[12], const double dq[5],
                      const double dG[12], const double M[9], double J, double mu, const double umf[3], double dF[5]) {
    if (axis < 0 || axis > 2 || !q || !G || !dq || !dG || !M || !umf || !dF) return set_error(CS_ERR_INVALID, "bad argument");
    const PointPhys p = point_phys(M, J, mu, umf);
    if (viscous) flux_tan<true>(axis, q, G, dq, dG, p, dF);
    else flux_tan<false>(axis, q, G, dq, dG, p, dF);
    return CS_OK;
}

int cs_point_flux_vjp(int axis, int viscous, const double q[5], const double G[12], const double Fbar[5],
                      const double M[9], double J, double mu, const double umf[3], double qbar[5], double Gbar[12]) {
    if (axis < 0 || axis > 2 || !q || !G || !Fbar || !M || !umf || !qbar || !Gbar)
        return set_error(CS_ERR_INVALID, "bad argument");
    const PointPhys p = point_phys(M, J, mu, umf);
    for (int m = 0; m < 5; ++m) qbar[m] = 0.0;
    for (int k = 0; k < 12; ++k) Gbar[k] = 0.0;
    if (viscous) flux_adj<true>(axis, q, G, Fbar, p, qbar, Gbar);
    else flux_adj<false>(axis, q, G, Fbar, p, qbar, Gbar);
    return CS_OK;
}

int cs_point_prim(const double q[5], double phi[4]) {
    if (!q || !phi) return set_error(CS_ERR_INVALID, "bad argument");
    prim_eval(q, phi);
    return CS_OK;
}

int cs_point_prim_jvp(const double q[5], const double dq[5], double dphi[4]) {
    if (!q || !dq || !dphi) return set_error(CS_ERR_INVALID, "bad argument");
    prim_tan(q, dq, dphi);
    return CS_OK;
}

int cs_point_prim_vjp(const double q[5], const double phibar[4], double qbar[5]) {
    if (!q || !phibar || !qbar) return set_error(CS_ERR_INVALID, "bad argument");
    for (int m = 0; m < 5; ++m) qbar[m] = 0.0;
    prim_adj(q, phibar, qbar);
    return CS_OK;
}

}  // extern "C"
