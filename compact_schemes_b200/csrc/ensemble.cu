// ensemble.cu -- host side of the batched ensemble (cs_ensemble_*): packed
// state and scratch, work-queue segment lists, the captured step graph and
// the autotuner.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "ensemble.cuh"

using csb::EnsBox;
using csb::EnsSeg;

struct cs_ensemble {
    int nbox = 0;
    bool viscous = true;
    std::vector<cs_solver_config> cfg;
    std::vector<EnsBox> hbox;
    EnsBox *dbox = nullptr;
    csb::TableCache tables;
    csb::Coeffs cf{};
    std::vector<int64_t> qoff;
    int64_t nq = 0, ng = 0, nr = 0;  // packed lengths in doubles
    double *q1 = nullptr, *grad = nullptr, *rhs = nullptr;
    unsigned long long *dtacc = nullptr;
    double *dt = nullptr;
    int *ctl = nullptr;  // [0] error word, [1] queue head, [2..] done[nbox][kEnsPhases]
    csb::Coeffs *cf_dev = nullptr;
    int lt_max = 2;
    int nsm = 1;
    cs_ensemble_tuning tune{0, 8, 0, 4};
    // work lists of the current tuning: [0] stage 0, [1] stages 1-3
    EnsSeg *segs[2] = {nullptr, nullptr};
    int nseg[2] = {0, 0}, nitems[2] = {0, 0};
    // captured step graph
    cudaGraphExec_t graph = nullptr;
    const double *graph_q = nullptr;
    cudaStream_t graph_stream = nullptr;
    // dependency wait: poll limit and extra required items (cs_ensemble_set_wait)
    long long poll_limit = csb::kEnsWaitPolls;
    int wait_bias = 0;
};

namespace csb {

static void ens_free_lists(cs_ensemble *e) {
    for (int i = 0; i < 2; ++i) {
        if (e->segs[i]) cudaFree(e->segs[i]);
        e->segs[i] = nullptr;
        e->nseg[i] = e->nitems[i] = 0;
    }
    if (e->graph) cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
    e->graph_q = nullptr;
}

// Segment lists for the current tuning.  Boxes are ranked largest first, and
// phase p of the box of rank r is queued at slot r + p * lag (ties by rank):
// lag = number of boxes gives all boxes' gradients, then all x fluxes, ...;
// a small lag queues a box's next phase soon after its previous one, while
// the phases of `lag` other boxes fill the gap, so a box's gradients and RHS
// are still in L2 when its next phase reads them.
static int ens_build_lists(cs_ensemble *e) {
    ens_free_lists(e);
    const int TL = e->tune.tile;
    std::vector<int> order(e->nbox);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return e->hbox[a].lmx > e->hbox[b].lmx; });
    const int lag = e->tune.window > 0 && e->tune.window < e->nbox ? e->tune.window : e->nbox;
    struct Key { int slot, rank, phase; };
    std::vector<Key> keys;
    for (int r = 0; r < e->nbox; ++r)
        for (int p = 0; p < kEnsPhases; ++p) keys.push_back({r + p * lag, r, p});
    std::stable_sort(keys.begin(), keys.end(), [](const Key &x, const Key &y) {
        return x.slot != y.slot ? x.slot < y.slot : x.rank < y.rank;
    });
    for (int list = 0; list < 2; ++list) {
        std::vector<EnsSeg> segs;
        std::vector<int> count(e->nbox * kEnsPhases, 0);
        int item = 0;
        for (const Key &k : keys) {
            const int b = order[k.rank], phase = k.phase;
            int kinds[3], nk = 0;
            if (phase == 0) {
                if (e->viscous) { kinds[0] = 0; kinds[1] = 1; kinds[2] = 2; nk = 3; }
                else if (list == 0) { kinds[0] = 0; nk = 1; }  // CFL maxima only
            } else {
                kinds[0] = 2 + phase;
                nk = 1;
            }
            for (int i = 0; i < nk; ++i) {
                EnsSeg sg{};
                sg.start = item;
                sg.ntiles = (int)((e->hbox[b].F[kinds[i] % 3] + TL - 1) / TL);
                sg.box = b;
                sg.kind = kinds[i];
                sg.phase = phase;
                sg.wait_count = phase > 0 ? count[b * kEnsPhases + phase - 1] : 0;
                segs.push_back(sg);
                const int nit = (sg.ntiles + e->tune.chunk - 1) / e->tune.chunk;
                item += nit;
                count[b * kEnsPhases + phase] += nit;
            }
        }
        if (cudaMalloc(&e->segs[list], segs.size() * sizeof(EnsSeg)) != cudaSuccess) {
            e->segs[list] = nullptr;
            return set_error(CS_ERR_ALLOC, "ensemble work list allocation failed");
        }
        CSB_CUDA(cudaMemcpy(e->segs[list], segs.data(), segs.size() * sizeof(EnsSeg), cudaMemcpyHostToDevice));
        e->nseg[list] = (int)segs.size();
        e->nitems[list] = item;
    }
    return CS_OK;
}

static int ens_tile_doubles(const cs_ensemble *e) { return 5 * e->tune.tile * (32 * e->lt_max + 1); }

// tile buffer, then the segment starts of the larger of the two work lists
static size_t ens_smem(const cs_ensemble *e) {
    const int nseg = std::max(e->nseg[0], e->nseg[1]);
    return (size_t)ens_tile_doubles(e) * sizeof(double) + (nseg <= kEnsSmemStarts ? (size_t)nseg * sizeof(int) : 0);
}

static int ens_run_step(cs_ensemble *e, double *q, cudaStream_t st) {
    CSB_CUDA(cudaMemsetAsync(e->dtacc, 0, 2 * sizeof(unsigned long long) * e->nbox, st));
    EnsArgs a{};
    a.boxes = e->dbox;
    a.err = e->ctl;
    a.poll_limit = e->poll_limit;
    a.wait_bias = e->wait_bias;
    a.queue = e->ctl + 1;
    a.done = e->ctl + 2;
    a.q = q;
    a.q1 = e->q1;
    a.grad = e->grad;
    a.rhs = e->rhs;
    a.dtacc = e->dtacc;
    a.dt = e->dt;
    a.cf = e->cf;
    a.cf_dev = e->cf_dev;
    a.chunk = e->tune.chunk;
    a.tile_doubles = ens_tile_doubles(e);
    const size_t smem = ens_smem(e);
    for (int k = 0; k < 4; ++k) {
        const int list = k == 0 ? 0 : 1;
        a.segs = e->segs[list];
        a.nseg = e->nseg[list];
        a.nitems = e->nitems[list];
        a.stage = k;
        CSB_CUDA(cudaMemsetAsync(e->ctl + 1, 0, sizeof(int) * (1 + kEnsPhases * e->nbox), st));
        const int rc = e->tune.tile == 4 ? ens_launch_tl4(a, e->viscous, e->tune.ctas_per_sm, e->nsm, smem, st, e->nbox)
                                         : ens_launch_tl8(a, e->viscous, e->tune.ctas_per_sm, e->nsm, smem, st, e->nbox);
        if (rc) return rc;
    }
    return CS_OK;
}

static int ens_check_tuning(const cs_ensemble *e, const cs_ensemble_tuning &t) {
    if (t.tile != 4 && t.tile != 8) return set_error(CS_ERR_INVALID, "ensemble tile %d: 4 or 8", t.tile);
    if (t.window < 0 || t.ctas_per_sm < 0 || t.chunk < 1 || t.chunk > 64)
        return set_error(CS_ERR_INVALID, "ensemble tuning");
    int smem_max = 0, dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        smem_max = 227 * 1024;
    const size_t need = (size_t)5 * t.tile * (32 * e->lt_max + 1) * sizeof(double) + kEnsSmemStarts * sizeof(int);
    if (need > (size_t)smem_max) return set_error(CS_ERR_UNSUPPORTED, "ensemble tile %d needs %zu bytes", t.tile, need);
    return CS_OK;
}

}  // namespace csb

using namespace csb;

extern "C" {

int cs_ensemble_destroy(cs_ensemble *e) {
    if (!e) return set_error(CS_ERR_INVALID, "null argument");
    ens_free_lists(e);
    cudaFree(e->dbox);
    cudaFree(e->q1);
    cudaFree(e->grad);
    cudaFree(e->rhs);
    cudaFree(e->dtacc);
    cudaFree(e->dt);
    cudaFree(e->ctl);
    cudaFree(e->cf_dev);
    delete e;
    return CS_OK;
}

int cs_ensemble_create(cs_ensemble **out, int nbox, const cs_solver_config *boxes) {
    if (!out || !boxes || nbox < 1) return set_error(CS_ERR_INVALID, "null argument or no boxes");
    if (nbox > kEnsMaxBoxes)
        return set_error(CS_ERR_UNSUPPORTED, "ensemble of %d boxes: at most %d per ensemble", nbox, kEnsMaxBoxes);
    *out = nullptr;
    auto *e = new cs_ensemble();
    e->nbox = nbox;
    e->cfg.assign(boxes, boxes + nbox);
    e->viscous = boxes[0].viscous != 0;
    compute_interface_coeffs(e->cf);
    e->hbox.resize(nbox);
    e->qoff.resize(nbox);
    for (int b = 0; b < nbox; ++b) {
        const cs_solver_config &c = boxes[b];
        EnsBox &bx = e->hbox[b];
        std::memset(&bx, 0, sizeof bx);
        auto fail = [&](int code, const char *what) {
            cs_ensemble_destroy(e);
            return set_error(code, "ensemble box %d: %s", b, what);
        };
        if ((c.viscous != 0) != e->viscous) return fail(CS_ERR_UNSUPPORTED, "all boxes viscous or all inviscid");
        if (c.precision != CS_PREC_FP64) return fail(CS_ERR_UNSUPPORTED, "FP64 only");
        if (c.gcbc) return fail(CS_ERR_UNSUPPORTED, "no characteristic boundary closure");
        if (c.filter != CS_FILTER_NONE) return fail(CS_ERR_UNSUPPORTED, "no filter in the ensemble step");
        if (!(c.dx > 0 && c.dy > 0 && c.dz > 0)) return fail(CS_ERR_INVALID, "grid spacing");
        const int n[3] = {c.lxi, c.let, c.lze};
        bx.lxi = c.lxi;
        bx.let = c.let;
        bx.lze = c.lze;
        bx.lmx = (int64_t)c.lxi * c.let * c.lze;
        bx.F[0] = (int64_t)c.let * c.lze;
        bx.F[1] = (int64_t)c.lxi * c.lze;
        bx.F[2] = (int64_t)c.lxi * c.let;
        for (int a = 0; a < 3; ++a) {
            if (n[a] < 8 || n[a] > 32 * kEnsMaxLt) return fail(CS_ERR_UNSUPPORTED, "every axis 8..256 points");
            const int s0 = bc_ndf(c.nbc[0][a]), s1 = bc_ndf(c.nbc[1][a]);
            if (s0 < 0 || s1 < 0) return fail(CS_ERR_INVALID, "boundary code");
            if (s0 != s1) return fail(CS_ERR_UNSUPPORTED, "both faces of an axis periodic or both physical");
            // lines of up to 64 points in chunks of 4 (at most 16 lanes): the
            // work items then solve two fields per half-warp (fewer PCR steps
            // per field than 2-point chunks over 32 lanes)
            const DeviceTables *t = e->tables.get(n[a], kDeriv, s0, s1, 0.0, n[a] <= 64 ? 4 : 2);
            if (!t) { cs_ensemble_destroy(e); return CS_ERR_UNSUPPORTED; }
            bx.tab[a] = t->t64;
            bx.lt[a] = t->lt;
            bx.nstart[a] = s0;
            bx.nend[a] = s1;
            e->lt_max = std::max(e->lt_max, t->lt);
        }
        uniform_phys(c, bx.ph);
        bx.cfl = c.cfl;
        bx.qoff = e->nq;
        bx.goff = e->ng;
        bx.roff = e->nr;
        e->qoff[b] = e->nq;
        e->nq += 5 * bx.lmx;
        e->ng += 12 * bx.lmx;
        e->nr += 5 * bx.lmx;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&e->nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) e->nsm = 1;
    const bool ok = cudaMalloc(&e->dbox, nbox * sizeof(EnsBox)) == cudaSuccess &&
                    cudaMalloc(&e->q1, e->nq * sizeof(double)) == cudaSuccess &&
                    cudaMalloc(&e->grad, e->ng * sizeof(double)) == cudaSuccess &&
                    cudaMalloc(&e->rhs, e->nr * sizeof(double)) == cudaSuccess &&
                    cudaMalloc(&e->dtacc, 2 * nbox * sizeof(unsigned long long)) == cudaSuccess &&
                    cudaMalloc(&e->dt, nbox * sizeof(double)) == cudaSuccess &&
                    cudaMalloc(&e->ctl, (2 + kEnsPhases * nbox) * sizeof(int)) == cudaSuccess &&
                    cudaMalloc(&e->cf_dev, sizeof(Coeffs)) == cudaSuccess;
    if (!ok) {
        cs_ensemble_destroy(e);
        return set_error(CS_ERR_ALLOC, "ensemble scratch allocation failed");
    }
    cudaMemcpy(e->dbox, e->hbox.data(), nbox * sizeof(EnsBox), cudaMemcpyHostToDevice);
    cudaMemcpy(e->cf_dev, &e->cf, sizeof(Coeffs), cudaMemcpyHostToDevice);
    cudaMemset(e->grad, 0, e->ng * sizeof(double));
    cudaMemset(e->dt, 0, nbox * sizeof(double));
    cudaMemset(e->ctl, 0, (2 + kEnsPhases * nbox) * sizeof(int));
    if (e->lt_max > 4) e->tune.tile = 4;  // 8-line tiles of 256-point lines need 82 KB
    if (int rc = ens_check_tuning(e, e->tune)) { cs_ensemble_destroy(e); return rc; }
    if (int rc = ens_build_lists(e)) { cs_ensemble_destroy(e); return rc; }
    if (cudaDeviceSynchronize() != cudaSuccess) {
        cs_ensemble_destroy(e);
        return set_error(CS_ERR_CUDA, "ensemble setup");
    }
    *out = e;
    return CS_OK;
}

int cs_ensemble_state_size(const cs_ensemble *e, int64_t *n_doubles) {
    if (!e || !n_doubles) return set_error(CS_ERR_INVALID, "null argument");
    *n_doubles = e->nq;
    return CS_OK;
}

int cs_ensemble_box_offset(const cs_ensemble *e, int box, int64_t *offset) {
    if (!e || !offset || box < 0 || box >= e->nbox) return set_error(CS_ERR_INVALID, "bad argument");
    *offset = e->qoff[box];
    return CS_OK;
}

int cs_ensemble_step(cs_ensemble *e, double *q, void *stream) {
    if (!e || !q) return set_error(CS_ERR_INVALID, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (!e->graph || e->graph_q != q || e->graph_stream != st) {
        if (e->graph) { cudaGraphExecDestroy(e->graph); e->graph = nullptr; }
        cudaStream_t cap;
        CSB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaGraph_t g;
        CSB_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        const int rc = ens_run_step(e, q, cap);
        cudaError_t err = cudaStreamEndCapture(cap, &g);
        cudaStreamDestroy(cap);
        if (rc) return rc;
        if (err != cudaSuccess) return check_cuda(err, "cudaStreamEndCapture");
        err = cudaGraphInstantiate(&e->graph, g, 0);
        cudaGraphDestroy(g);
        if (err != cudaSuccess) { e->graph = nullptr; return check_cuda(err, "cudaGraphInstantiate"); }
        e->graph_q = q;
        e->graph_stream = st;
    }
    CSB_CUDA(cudaGraphLaunch(e->graph, st));
    return CS_OK;
}

int cs_ensemble_last_dt(cs_ensemble *e, double *dt_host) {
    if (!e || !dt_host) return set_error(CS_ERR_INVALID, "null argument");
    CSB_CUDA(cudaDeviceSynchronize());
    CSB_CUDA(cudaMemcpy(dt_host, e->dt, e->nbox * sizeof(double), cudaMemcpyDeviceToHost));
    int err = 0;
    CSB_CUDA(cudaMemcpy(&err, e->ctl, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
        CSB_CUDA(cudaMemset(e->ctl, 0, sizeof(int)));
        return set_error(CS_ERR_TIMEOUT, "ensemble: the dependency wait of work item %d ran out", err - 1);
    }
    return CS_OK;
}

int cs_ensemble_set_wait(cs_ensemble *e, long long poll_limit, int extra) {
    if (!e) return set_error(CS_ERR_INVALID, "null argument");
    if (poll_limit < 1 || extra < 0) return set_error(CS_ERR_INVALID, "poll_limit %lld, extra %d", poll_limit, extra);
    e->poll_limit = poll_limit;
    e->wait_bias = extra;
    if (e->graph) { cudaGraphExecDestroy(e->graph); e->graph = nullptr; }
    return CS_OK;
}

int cs_ensemble_set_tuning(cs_ensemble *e, const cs_ensemble_tuning *t) {
    if (!e || !t) return set_error(CS_ERR_INVALID, "null argument");
    if (int rc = ens_check_tuning(e, *t)) return rc;
    e->tune = *t;
    return ens_build_lists(e);
}

int cs_ensemble_get_tuning(const cs_ensemble *e, cs_ensemble_tuning *t) {
    if (!e || !t) return set_error(CS_ERR_INVALID, "null argument");
    *t = e->tune;
    return CS_OK;
}

int cs_ensemble_autotune(cs_ensemble *e, const double *q, int reps, cs_ensemble_tuning *best, double *best_ms,
                         void *stream) {
    if (!e || !q || reps < 1) return set_error(CS_ERR_INVALID, "bad argument");
    cudaStream_t st = (cudaStream_t)stream;
    double *scratch = nullptr;
    if (cudaMalloc(&scratch, e->nq * sizeof(double)) != cudaSuccess)
        return set_error(CS_ERR_ALLOC, "autotune scratch allocation failed");
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    std::vector<int> windows = {0};
    for (int w : {8, 4, 2, 1})
        if (w < e->nbox) windows.push_back(w);
    std::vector<int> tiles = e->lt_max > 4 ? std::vector<int>{4} : std::vector<int>{8, 4};
    const int chunks[] = {2, 4, 8, 16};
    const cs_ensemble_tuning saved = e->tune;
    cs_ensemble_tuning win = saved;
    double win_ms = 1e300;
    int rc = CS_OK;
    for (int tile : tiles) {
        for (int ci = 0; ci < 4 && !rc; ++ci)
        for (int w : windows) {
            cs_ensemble_tuning t{w, tile, 0, chunks[ci]};
            if ((rc = cs_ensemble_set_tuning(e, &t))) break;
            if (cudaMemcpyAsync(scratch, q, e->nq * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
                rc = set_error(CS_ERR_CUDA, "autotune copy");
                break;
            }
            if ((rc = cs_ensemble_step(e, scratch, stream))) break;  // capture + warm-up
            cudaEventRecord(t0, st);
            for (int r = 0; r < reps && !rc; ++r) rc = cs_ensemble_step(e, scratch, stream);
            cudaEventRecord(t1, st);
            if (rc) break;
            if (cudaEventSynchronize(t1) != cudaSuccess) { rc = set_error(CS_ERR_CUDA, "autotune timing"); break; }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, t0, t1);
            if (ms / reps < win_ms) {
                win_ms = ms / reps;
                win = t;
            }
        }
        if (rc) break;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    int err = 0;
    cudaStreamSynchronize(st);
    cudaMemcpy(&err, e->ctl, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(scratch);
    if (rc) {
        cs_ensemble_set_tuning(e, &saved);
        return rc;
    }
    if (err) {
        cudaMemset(e->ctl, 0, sizeof(int));
        cs_ensemble_set_tuning(e, &saved);
        return set_error(CS_ERR_TIMEOUT, "ensemble autotune: a dependency wait ran out");
    }
    if ((rc = cs_ensemble_set_tuning(e, &win))) return rc;
    if (best) *best = win;
    if (best_ms) *best_ms = win_ms;
    return CS_OK;
}

}  // extern "C"
