// pipeline.cuh -- persistent two-role form of the fused passes.
//
// One CTA per SM walks its tiles t_k = blockIdx.x + k * gridDim.x of a pass,
// with two shared-memory staging buffers (tile k uses buffer k & 1).  The
// first NM threads (memory role) do all the HBM traffic: they stage a tile
// (load the state, form primitives or fluxes, write them in the line layout)
// and later store or accumulate its solved lines.  The other NS threads (solve
// role) only solve the lines of staged tiles.  At step k the memory role
// stores tile k-2 and stages tile k in buffer k & 1 while the solve role
// solves tile k-1 in the other buffer, so the latency-bound line solves
// overlap the HBM traffic instead of alternating with it.
//
// Hand-off by named barriers (count NM + NS):
//   FULL[b]    memory role bar.arrive after staging tile k, solve role bar.sync
//              before solving it;
//   SOLVED[b]  solve role bar.arrive after solving tile k, memory role bar.sync
//              before storing it (two steps later).
// Every tile of the CTA is arrived at and waited for exactly once on each
// barrier, so every use completes with NM + NS threads and no wait is left
// open at exit.  Within the memory role a thread stores exactly the positions
// it staged (same traversal), so reusing a buffer needs no further barrier.
// Same arithmetic, in the same order, as the one-phase kernels of
// fused_kernels.cuh / fused_mixed.cuh: results are bit-identical to them.
#pragma once

#include "fused_mixed.cuh"

#ifndef CSB_PL_NM
#define CSB_PL_NM 256  // memory-role threads per CTA
#endif
#ifndef CSB_PL_NS
#define CSB_PL_NS 256  // solve-role threads per CTA
#endif
#ifndef CSB_PL_LOAD_UNROLL
#define CSB_PL_LOAD_UNROLL 2
#endif

namespace csb {

constexpr int kBarSolved0 = 3;  // + buffer (FULL[b] is kBarFull0 + b)

template <int NM, int NS, typename Stage, typename Store, typename Solve>
__device__ __forceinline__ void run_pipeline(int64_t ntiles, Stage &&stage, Store &&store, Solve &&solve) {
    constexpr int kAll = NM + NS;
    const int64_t G = gridDim.x;
    const int64_t K = ntiles > (int64_t)blockIdx.x ? (ntiles - 1 - blockIdx.x) / G + 1 : 0;  // tiles of this CTA
    if ((int)threadIdx.x < NM) {
        for (int64_t k = 0; k < K + 2; ++k) {
            const int b = (int)(k & 1);
            if (k >= 2) {
                named_bar_sync(kBarSolved0 + b, kAll);
                store(blockIdx.x + (k - 2) * G, b, (int)threadIdx.x);
            }
            if (k < K) {
                stage(blockIdx.x + k * G, b, (int)threadIdx.x);
                named_bar_arrive(kBarFull0 + b, kAll);
            }
        }
    } else {
        for (int64_t k = 0; k < K; ++k) {
            const int b = (int)(k & 1);
            named_bar_sync(kBarFull0 + b, kAll);
            solve(blockIdx.x + k * G, b, (int)threadIdx.x - NM);
            named_bar_arrive(kBarSolved0 + b, kAll);
        }
    }
}

// Solve fields c0 .. c0+G-1 (< NF) of one line of an FP64 tile in place;
// ROWS as in solve_fields (the TMA gradient pass forms its closure rows on 8
// lanes per line, measured faster there).
template <int LT, int TL, int G, bool ROWS = false>
__device__ __forceinline__ void solve_group(double *sm, int line, int c0, int nf, int lane,
                                            const DevTables<double> &tab, int nstart, int nend, const Coeffs &cf) {
    double d[G][LT];
    double *lines[G];
#pragma unroll
    for (int g = 0; g < G; ++g) lines[g] = field_line<LT, TL>(sm, c0 + g < nf ? c0 + g : c0, line);
    const bool sums = ROWS && (nstart != 0 || nend != 0);
    const double rows = sums ? group_closure_rows<LT, double, double, G>(lines, nf - c0, tab.n, lane, cf) : 0.0;
#pragma unroll
    for (int g = 0; g < G; ++g) {
        double own2[2];
        if (sums) take_closure_rows(rows, g, lane, own2);
        if (c0 + g < nf) deriv_rhs<LT, double, double>(lines[g], tab.n, lane, nstart, nend, nullptr, cf, d[g],
                                                       sums ? own2 : nullptr);
        else {
#pragma unroll
            for (int t = 0; t < LT; ++t) d[g][t] = 0.0;
        }
    }
    warp_solve<LT, G, double>(tab, d, lane);
    __syncwarp();
#pragma unroll
    for (int g = 0; g < G; ++g) {
        if (c0 + g >= nf) continue;
        double *ln = field_line<LT, TL>(sm, c0 + g, line);
#pragma unroll
        for (int t = 0; t < LT; ++t)
            if (lane * LT + t < tab.n) ln[LineLayout<LT>::pos_ct(lane, t)] = d[g][t];
    }
}

// The solve-role warps share the (line, field group) solves of a tile;
// after(l, c0, lane) runs warp-wide once the group of line l starting at field
// c0 is solved.
template <int LT, int TL, int NF, int G, int NS, typename Fn>
__device__ __forceinline__ void consume_solve64(double *sm, int stid, int64_t line0, int64_t F,
                                                const DevTables<double> &tab, int nstart, int nend,
                                                const Coeffs &cf, Fn &&after) {
    constexpr int NG = (NF + G - 1) / G;
    const int cw = stid >> 5, lane = stid & 31;
#pragma unroll 1
    for (int p = cw; p < TL * NG; p += NS / 32) {
        const int l = p % TL, c0 = (p / TL) * G;
        if (line0 + l < F) {
            solve_group<LT, TL, G>(sm, l, c0, NF, lane, tab, nstart, nend, cf);
            __syncwarp();
            after(l, c0, lane);
        }
    }
}

// ----------------------------------------------------------------------------
// FP64 gradient pass (as k_grad)
// ----------------------------------------------------------------------------
template <int LT, int AXIS, int TL, bool DTRED, int NM, int NS>
__global__ void __launch_bounds__(NM + NS, 1)
k_grad_pl(const double *__restrict__ q, double *__restrict__ g, DevTables<double> tab, int lxi, int let,
          int64_t lmx, int64_t F, int nstart, int nend, Coeffs cf, Phys ph,
          unsigned long long *__restrict__ dtacc) {
    using L = LineLayout<LT>;
    constexpr int kBuf = 4 * TL * L::kSlot;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *const smb = reinterpret_cast<double *>(smem_raw);
    const int n = tab.n;
    double m1 = 0.0, m2 = 0.0;
    run_pipeline<NM, NS>(
        (F + TL - 1) / TL,
        [&](int64_t t, int b, int rtid) {
            double *sm = smb + b * kBuf;
            tile_for_each_r<AXIS, TL, NM, CSB_PL_LOAD_UNROLL>(rtid, t * TL, F, n, lxi, let,
                                                               [&](int l, int j, int64_t gi) {
                const Prim s = primitives(__ldg(q + gi), __ldg(q + lmx + gi), __ldg(q + 2 * lmx + gi),
                                          __ldg(q + 3 * lmx + gi), __ldg(q + 4 * lmx + gi));
                const int pj = L::pos(j);
                field_line<LT, TL>(sm, 0, l)[pj] = s.u;
                field_line<LT, TL>(sm, 1, l)[pj] = s.v;
                field_line<LT, TL>(sm, 2, l)[pj] = s.w;
                field_line<LT, TL>(sm, 3, l)[pj] = s.T;
                if (DTRED) {
                    // calc_time_step_kernel (src/cuda/kernels/physics.hpp:335-427)
                    const double uu = s.u + ph.umf[0], vv = s.v + ph.umf[1], ww = s.w + ph.umf[2];
                    double rr2 = 0.0;
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        rr2 += fabs(xmul(ph.M[a][0], uu) + xmul(ph.M[a][1], vv) + xmul(ph.M[a][2], ww));
                    const double ssi = fabs(ph.J);
                    m1 = fmax(m1, xmul(sqrt(xmul(s.T, ph.rr1)) + rr2, ssi));
                    m2 = fmax(m2, s.ri * ph.mu * ph.rr1 * ssi * ssi);
                }
            });
        },
        [&](int64_t t, int b, int rtid) {
            const double *sm = smb + b * kBuf;
            tile_for_each_r<AXIS, TL, NM, CSB_STORE_UNROLL>(rtid, t * TL, F, n, lxi, let,
                                                            [&](int l, int j, int64_t gi) {
                const int pj = L::pos(j);
#pragma unroll
                for (int c = 0; c < 4; ++c) g[c * lmx + gi] = sm[(c * TL + l) * L::kSlot + pj];
            });
        },
        [&](int64_t t, int b, int stid) {
            consume_solve64<LT, TL, 4, CSB_SOLVE_GROUP, NS>(smb + b * kBuf, stid, t * TL, F, tab, nstart, nend, cf,
                                                            [](int, int, int) {});
        });
    if (DTRED && (int)threadIdx.x < NM) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
            m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMax(dtacc, (unsigned long long)__double_as_longlong(m1));
            atomicMax(dtacc + 1, (unsigned long long)__double_as_longlong(m2));
        }
    }
}

// ----------------------------------------------------------------------------
// FP64 flux pass (as k_flux)
// ----------------------------------------------------------------------------
template <int LT, int AXIS, int TL, int MODE, bool VISC, int NM, int NS>
__global__ void __launch_bounds__(NM + NS, 1)
k_flux_pl(const double *__restrict__ q, const double *__restrict__ g, double *__restrict__ rhs,
          const double *__restrict__ qn, double *__restrict__ qout, double *__restrict__ drva,
          DevTables<double> tab, int lxi, int let, int64_t lmx, int64_t F, int nstart, int nend, Coeffs cf,
          Phys ph, RkParams rk) {
    using L = LineLayout<LT>;
    constexpr int kBuf = 5 * TL * L::kSlot;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *const smb = reinterpret_cast<double *>(smem_raw);
    const int n = tab.n;
    double dtk = 0.0;
    if (MODE >= kAccumRk) {
        const double dt = rk_dt(rk);
        dtk = xmul(dt / rk.div, ph.J);
        if (rk.dt_out && blockIdx.x == 0 && threadIdx.x == 0) *rk.dt_out = dt;
    }
    run_pipeline<NM, NS>(
        (F + TL - 1) / TL,
        [&](int64_t t, int b, int rtid) {
            double *sm = smb + b * kBuf;
            tile_for_each_r<AXIS, TL, NM, CSB_FLUX_UNROLL>(rtid, t * TL, F, n, lxi, let,
                                                            [&](int l, int j, int64_t gi) {
                double fl[5];
                point_flux<AXIS, VISC>(q, g, lmx, gi, ph, fl);
                const int pj = L::pos(j);
#pragma unroll
                for (int m = 0; m < 5; ++m) field_line<LT, TL>(sm, m, l)[pj] = fl[m];
            });
        },
        [&](int64_t t, int b, int rtid) {
            const double *sm = smb + b * kBuf;
            const int64_t line0 = t * TL;
            if (MODE == kWrite) {
                tile_for_each_r<AXIS, TL, NM, CSB_STORE_UNROLL>(rtid, line0, F, n, lxi, let,
                                                                [&](int l, int j, int64_t gi) {
                    const int pj = L::pos(j);
#pragma unroll
                    for (int m = 0; m < 5; ++m) rhs[m * lmx + gi] = sm[(m * TL + l) * L::kSlot + pj];
                });
            } else {
                constexpr int P = MODE == kAccum ? CSB_RMW_CHUNK : CSB_RMW_CHUNK_RK;
                double rv[P][5], qv[P][5];
                tile_for_each_r_chunked<AXIS, TL, NM, P>(
                    rtid, line0, F, n, lxi, let,
                    [&](int p, int l, int j, int64_t gi) {
#pragma unroll
                        for (int m = 0; m < 5; ++m) {
                            rv[p][m] = MODE == kWriteRk ? 0.0 : rhs[m * lmx + gi];
                            if (MODE >= kAccumRk) qv[p][m] = qn[m * lmx + gi];
                        }
                    },
                    [&](int p, int l, int j, int64_t gi) {
                        const int pj = L::pos(j);
#pragma unroll
                        for (int m = 0; m < 5; ++m) {
                            const double dfv = sm[(m * TL + l) * L::kSlot + pj];
                            if (MODE == kAccum) {
                                rhs[m * lmx + gi] = rv[p][m] + dfv;
                            } else {
                                const double r = MODE == kAccumRk ? rv[p][m] + dfv : dfv;
                                qout[m * lmx + gi] = qv[p][m] - xmul(dtk, r);
                            }
                        }
                    });
            }
        },
        [&](int64_t t, int b, int stid) {
            double *sm = smb + b * kBuf;
            const int64_t line0 = t * TL;
            consume_solve64<LT, TL, 5, CSB_SOLVE_GROUP, NS>(
                sm, stid, line0, F, tab, nstart, nend, cf, [&](int l, int c0, int lane) {
                    if (drva && lane < 2 * CSB_SOLVE_GROUP) {
                        // line-end derivatives for the characteristic boundary closure
                        // (drva of deriv_kernel_2d, src/cuda/kernels/numerics_pc.hpp:237-248)
                        const int m = c0 + lane % CSB_SOLVE_GROUP, face = lane / CSB_SOLVE_GROUP;
                        if (m < 5)
                            drva[(int64_t)(face * 5 + m) * F + line0 + l] =
                                field_line<LT, TL>(sm, m, l)[L::pos(face ? n - 1 : 0)];
                    }
                });
        });
}

// ----------------------------------------------------------------------------
// mixed-precision passes (as k_grad_mx / k_flux_mx)
// ----------------------------------------------------------------------------
// The solve-role warps share the (line, field) solves of an FP32 tile.
template <int LT, int TL, int NF, int NS, typename Fn>
__device__ __forceinline__ void consume_solve32(float *sm, int stid, int64_t line0, int64_t F,
                                                const DevTables<float> &tab, int nstart, int nend,
                                                const Coeffs &cf, int refine, Fn &&after) {
    const int cw = stid >> 5, lane = stid & 31;
#pragma unroll 1
    for (int p = cw; p < TL * NF; p += NS / 32) {
        const int l = p % TL, c = p / TL;
        if (line0 + l < F) {
            solve_line_mx<LT>(field_line32<LT, TL>(sm, c, l), lane, tab, nstart, nend, cf, refine);
            __syncwarp();
            after(l, c, lane);
        }
    }
}

template <int LT, int AXIS, int TL, bool FIRST, int NM, int NS>
__global__ void __launch_bounds__(NM + NS, 1)
k_grad_mx_pl(const double *__restrict__ q, float *__restrict__ sh, float *__restrict__ g,
             DevTables<float> tab, int lxi, int let, int64_t lmx, int64_t F, int nstart, int nend, Coeffs cf,
             Phys ph, unsigned long long *__restrict__ dtacc, int refine) {
    using L = LineLayout<LT>;
    constexpr int kBuf = 4 * TL * L::kSlot;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *const smb = reinterpret_cast<float *>(smem_raw);
    const int n = tab.n;
    double m1 = 0.0, m2 = 0.0;
    run_pipeline<NM, NS>(
        (F + TL - 1) / TL,
        [&](int64_t t, int b, int rtid) {
            float *sm = smb + b * kBuf;
            tile_for_each_r<AXIS, TL, NM, CSB_PL_LOAD_UNROLL>(rtid, t * TL, F, n, lxi, let,
                                                               [&](int l, int j, int64_t gi) {
                float u, v, wv, tp;
                if (FIRST) {
                    float s5[5];
                    Prim s;
                    shadow_from_q(__ldg(q + gi), __ldg(q + lmx + gi), __ldg(q + 2 * lmx + gi),
                                  __ldg(q + 3 * lmx + gi), __ldg(q + 4 * lmx + gi), s5, s);
#pragma unroll
                    for (int k = 0; k < 5; ++k) sh[k * lmx + gi] = s5[k];
                    u = s5[1];
                    v = s5[2];
                    wv = s5[3];
                    tp = s5[4];
                    const double uu = s.u + ph.umf[0], vv = s.v + ph.umf[1], ww = s.w + ph.umf[2];
                    double rr2 = 0.0;
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        rr2 += fabs(xmul(ph.M[a][0], uu) + xmul(ph.M[a][1], vv) + xmul(ph.M[a][2], ww));
                    const double ssi = fabs(ph.J);
                    m1 = fmax(m1, xmul(sqrt(xmul(s.T, ph.rr1)) + rr2, ssi));
                    m2 = fmax(m2, s.ri * ph.mu * ph.rr1 * ssi * ssi);
                } else {
                    const float dt = __ldg(sh + 4 * lmx + gi);
                    u = __ldg(sh + lmx + gi);
                    v = __ldg(sh + 2 * lmx + gi);
                    wv = __ldg(sh + 3 * lmx + gi);
                    tp = dt;
                }
                const int pj = L::pos(j);
                field_line32<LT, TL>(sm, 0, l)[pj] = u;
                field_line32<LT, TL>(sm, 1, l)[pj] = v;
                field_line32<LT, TL>(sm, 2, l)[pj] = wv;
                field_line32<LT, TL>(sm, 3, l)[pj] = tp;
            });
        },
        [&](int64_t t, int b, int rtid) {
            const float *sm = smb + b * kBuf;
            tile_for_each_r<AXIS, TL, NM, CSB_STORE_UNROLL>(rtid, t * TL, F, n, lxi, let,
                                                            [&](int l, int j, int64_t gi) {
                const int pj = L::pos(j);
#pragma unroll
                for (int c = 0; c < 4; ++c) g[c * lmx + gi] = sm[(c * TL + l) * L::kSlot + pj];
            });
        },
        [&](int64_t t, int b, int stid) {
            consume_solve32<LT, TL, 4, NS>(smb + b * kBuf, stid, t * TL, F, tab, nstart, nend, cf, refine,
                                           [](int, int, int) {});
        });
    if (FIRST && (int)threadIdx.x < NM) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            m1 = fmax(m1, __shfl_xor_sync(0xffffffffu, m1, o));
            m2 = fmax(m2, __shfl_xor_sync(0xffffffffu, m2, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMax(dtacc, (unsigned long long)__double_as_longlong(m1));
            atomicMax(dtacc + 1, (unsigned long long)__double_as_longlong(m2));
        }
    }
}

template <int LT, int AXIS, int TL, int MODE, bool VISC, bool SHADOW_OUT, int NM, int NS>
__global__ void __launch_bounds__(NM + NS, 1)
k_flux_mx_pl(const float *__restrict__ sh, const float *__restrict__ g, float *__restrict__ rhs,
             const double *__restrict__ qn, double *__restrict__ qout, float *__restrict__ sh_out,
             double *__restrict__ drva, DevTables<float> tab, int lxi, int let, int64_t lmx, int64_t F,
             int nstart, int nend, Coeffs cf, Phys ph, RkParams rk, int refine) {
    using L = LineLayout<LT>;
    constexpr int kBuf = 5 * TL * L::kSlot;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *const smb = reinterpret_cast<float *>(smem_raw);
    const int n = tab.n;
    double dtk = 0.0;
    if (MODE >= kAccumRk) {
        const double dt = rk_dt(rk);
        dtk = xmul(dt / rk.div, ph.J);
        if (rk.dt_out && blockIdx.x == 0 && threadIdx.x == 0) *rk.dt_out = dt;
    }
    run_pipeline<NM, NS>(
        (F + TL - 1) / TL,
        [&](int64_t t, int b, int rtid) {
            float *sm = smb + b * kBuf;
            tile_for_each_r<AXIS, TL, NM, CSB_FLUX_UNROLL>(rtid, t * TL, F, n, lxi, let,
                                                            [&](int l, int j, int64_t gi) {
                float fl[5];
                point_flux_mx<AXIS, VISC>(sh, g, lmx, gi, ph, fl);
                const int pj = L::pos(j);
#pragma unroll
                for (int m = 0; m < 5; ++m) field_line32<LT, TL>(sm, m, l)[pj] = fl[m];
            });
        },
        [&](int64_t t, int b, int rtid) {
            const float *sm = smb + b * kBuf;
            const int64_t line0 = t * TL;
            if (MODE == kWrite) {
                tile_for_each_r<AXIS, TL, NM, CSB_STORE_UNROLL>(rtid, line0, F, n, lxi, let,
                                                                [&](int l, int j, int64_t gi) {
                    const int pj = L::pos(j);
#pragma unroll
                    for (int m = 0; m < 5; ++m) rhs[m * lmx + gi] = sm[(m * TL + l) * L::kSlot + pj];
                });
            } else {
                constexpr int P = MODE == kAccum ? CSB_RMW_CHUNK : CSB_RMW_CHUNK_RK;
                float rv[P][5];
                double qv[P][5];
                tile_for_each_r_chunked<AXIS, TL, NM, P>(
                    rtid, line0, F, n, lxi, let,
                    [&](int p, int l, int j, int64_t gi) {
#pragma unroll
                        for (int m = 0; m < 5; ++m) {
                            rv[p][m] = MODE == kWriteRk ? 0.0f : rhs[m * lmx + gi];
                            if (MODE >= kAccumRk) qv[p][m] = qn[m * lmx + gi];
                        }
                    },
                    [&](int p, int l, int j, int64_t gi) {
                        const int pj = L::pos(j);
                        if (MODE == kAccum) {
#pragma unroll
                            for (int m = 0; m < 5; ++m)
                                rhs[m * lmx + gi] = rv[p][m] + sm[(m * TL + l) * L::kSlot + pj];
                        } else {
                            double qo[5];
#pragma unroll
                            for (int m = 0; m < 5; ++m) {
                                const double r = (double)rv[p][m] + (double)sm[(m * TL + l) * L::kSlot + pj];
                                qo[m] = qv[p][m] - xmul(dtk, r);
                                qout[m * lmx + gi] = qo[m];
                            }
                            if (SHADOW_OUT) {
                                float s5[5];
                                Prim s;
                                shadow_from_q(qo[0], qo[1], qo[2], qo[3], qo[4], s5, s);
#pragma unroll
                                for (int m = 0; m < 5; ++m) sh_out[m * lmx + gi] = s5[m];
                            }
                        }
                    });
            }
        },
        [&](int64_t t, int b, int stid) {
            float *sm = smb + b * kBuf;
            const int64_t line0 = t * TL;
            consume_solve32<LT, TL, 5, NS>(sm, stid, line0, F, tab, nstart, nend, cf, refine,
                                           [&](int l, int m, int lane) {
                if (drva && lane < 2) {
                    drva[(int64_t)(lane * 5 + m) * F + line0 + l] =
                        (double)field_line32<LT, TL>(sm, m, l)[L::pos(lane ? n - 1 : 0)];
                }
            });
        });
}

// ----------------------------------------------------------------------------
// launch templates
// ----------------------------------------------------------------------------
// Persistent grid: as many CTAs as fit on the device at once, at most one per tile.
template <typename KernelT>
inline unsigned pl_grid(KernelT kern, int threads, size_t smem, int64_t ntiles, int nsm) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, threads, smem) != cudaSuccess || nb < 1) nb = 1;
    const int64_t g = (int64_t)(nsm > 0 ? nsm : 1) * nb;
    return (unsigned)(ntiles < g ? ntiles : g);
}

template <int LT, int AXIS>
int launch_grad_pl_t(const PassArgs &a, const double *q, bool dtred, cudaStream_t st) {
    constexpr int TL = pl_tile<LT, double>(), NM = CSB_PL_NM, NS = CSB_PL_NS;
    const size_t smem = (size_t)2 * 4 * TL * LineLayout<LT>::kSlot * sizeof(double);
    auto kern = dtred ? k_grad_pl<LT, AXIS, TL, true, NM, NS> : k_grad_pl<LT, AXIS, TL, false, NM, NS>;
    if (int rc = set_smem(kern, smem)) return rc;
    const unsigned grid = pl_grid(kern, NM + NS, smem, (a.F + TL - 1) / TL, a.nsm);
    kern<<<grid, NM + NS, smem, st>>>(q, a.grad + (int64_t)AXIS * 4 * a.lmx, a.tab->t64, a.lxi, a.let, a.lmx, a.F,
                                      a.nstart, a.nend, a.cf, a.ph, a.dtacc);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

template <int LT, int AXIS, int MODE>
int launch_flux_pl_t(const PassArgs &a, const double *q, const double *qn, double *qout, double *drva,
                     const RkParams &rk, cudaStream_t st) {
    constexpr int TL = pl_tile<LT, double>(), NM = CSB_PL_NM, NS = CSB_PL_NS;
    const size_t smem = (size_t)2 * 5 * TL * LineLayout<LT>::kSlot * sizeof(double);
    auto kern = a.viscous ? k_flux_pl<LT, AXIS, TL, MODE, true, NM, NS> : k_flux_pl<LT, AXIS, TL, MODE, false, NM, NS>;
    if (int rc = set_smem(kern, smem)) return rc;
    const unsigned grid = pl_grid(kern, NM + NS, smem, (a.F + TL - 1) / TL, a.nsm);
    kern<<<grid, NM + NS, smem, st>>>(q, a.grad, a.rhs, qn, qout, drva, a.tab->t64, a.lxi, a.let, a.lmx, a.F,
                                      a.nstart, a.nend, a.cf, a.ph, rk);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

template <int LT, int AXIS>
int launch_grad_mx_pl_t(const MixedArgs &m, const double *q, bool first, cudaStream_t st) {
    constexpr int TL = pl_tile<LT, float>(), NM = CSB_PL_NM, NS = CSB_PL_NS;
    const PassArgs &a = m.base;
    const size_t smem = (size_t)2 * 4 * TL * LineLayout<LT>::kSlot * sizeof(float);
    auto kern = first ? k_grad_mx_pl<LT, AXIS, TL, true, NM, NS> : k_grad_mx_pl<LT, AXIS, TL, false, NM, NS>;
    if (int rc = set_smem(kern, smem)) return rc;
    const unsigned grid = pl_grid(kern, NM + NS, smem, (a.F + TL - 1) / TL, a.nsm);
    kern<<<grid, NM + NS, smem, st>>>(q, m.shadow, m.grad + (int64_t)AXIS * 4 * a.lmx, a.tab->t32, a.lxi, a.let,
                                      a.lmx, a.F, a.nstart, a.nend, a.cf, a.ph, a.dtacc, m.refine);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

template <int LT, int AXIS, int MODE>
int launch_flux_mx_pl_t(const MixedArgs &m, const double *qn, double *qout, bool shadow_out, double *drva,
                        const RkParams &rk, cudaStream_t st) {
    constexpr int TL = pl_tile<LT, float>(), NM = CSB_PL_NM, NS = CSB_PL_NS;
    const PassArgs &a = m.base;
    const size_t smem = (size_t)2 * 5 * TL * LineLayout<LT>::kSlot * sizeof(float);
    constexpr bool kRk = MODE >= kAccumRk;
    auto kern = a.viscous ? (shadow_out && kRk ? k_flux_mx_pl<LT, AXIS, TL, MODE, true, kRk, NM, NS>
                                               : k_flux_mx_pl<LT, AXIS, TL, MODE, true, false, NM, NS>)
                          : (shadow_out && kRk ? k_flux_mx_pl<LT, AXIS, TL, MODE, false, kRk, NM, NS>
                                               : k_flux_mx_pl<LT, AXIS, TL, MODE, false, false, NM, NS>);
    if (int rc = set_smem(kern, smem)) return rc;
    const unsigned grid = pl_grid(kern, NM + NS, smem, (a.F + TL - 1) / TL, a.nsm);
    kern<<<grid, NM + NS, smem, st>>>(m.shadow, m.grad, m.rhs, qn, qout, m.shadow, drva, a.tab->t32, a.lxi, a.let,
                                      a.lmx, a.F, a.nstart, a.nend, a.cf, a.ph, rk, m.refine);
    CSB_CUDA(cudaGetLastError());
    return CS_OK;
}

#define CSB_PL_LT_SWITCH(CALL)                                  \
    switch (lt) {                                               \
        case 2: return CALL(2);                                 \
        case 4: return CALL(4);                                 \
        case 8: return CALL(8);                                 \
        case 16: return CALL(16);                               \
    }                                                           \
    return set_error(CS_ERR_UNSUPPORTED, "chunk length");

template <int AXIS>
int launch_grad_pl_impl(const PassArgs &a, const double *q, bool dtred, cudaStream_t st) {
    const int lt = a.tab->lt;
#define CSB_CALL(LT) launch_grad_pl_t<LT, AXIS>(a, q, dtred, st)
    CSB_PL_LT_SWITCH(CSB_CALL)
#undef CSB_CALL
}

template <int AXIS, int MODE>
int launch_flux_pl_m(const PassArgs &a, const double *q, const double *qn, double *qout, double *drva,
                     const RkParams &rk, cudaStream_t st) {
    const int lt = a.tab->lt;
#define CSB_CALL(LT) launch_flux_pl_t<LT, AXIS, MODE>(a, q, qn, qout, drva, rk, st)
    CSB_PL_LT_SWITCH(CSB_CALL)
#undef CSB_CALL
}

template <int AXIS>
int launch_flux_pl_impl(const PassArgs &a, int mode, const double *q, const double *qn, double *qout,
                        double *drva, const RkParams &rk, cudaStream_t st) {
    switch (mode) {
        case kWrite: return launch_flux_pl_m<AXIS, kWrite>(a, q, qn, qout, drva, rk, st);
        case kAccum: return launch_flux_pl_m<AXIS, kAccum>(a, q, qn, qout, drva, rk, st);
        case kAccumRk: return launch_flux_pl_m<AXIS, kAccumRk>(a, q, qn, qout, drva, rk, st);
        default: return launch_flux_pl_m<AXIS, kWriteRk>(a, q, qn, qout, drva, rk, st);
    }
}

template <int AXIS>
int launch_grad_mx_pl_impl(const MixedArgs &m, const double *q, bool first, cudaStream_t st) {
    const int lt = m.base.tab->lt;
#define CSB_CALL(LT) launch_grad_mx_pl_t<LT, AXIS>(m, q, first, st)
    CSB_PL_LT_SWITCH(CSB_CALL)
#undef CSB_CALL
}

template <int AXIS, int MODE>
int launch_flux_mx_pl_m(const MixedArgs &m, const double *qn, double *qout, bool shadow_out, double *drva,
                        const RkParams &rk, cudaStream_t st) {
    const int lt = m.base.tab->lt;
#define CSB_CALL(LT) launch_flux_mx_pl_t<LT, AXIS, MODE>(m, qn, qout, shadow_out, drva, rk, st)
    CSB_PL_LT_SWITCH(CSB_CALL)
#undef CSB_CALL
}

template <int AXIS>
int launch_flux_mx_pl_impl(const MixedArgs &m, int mode, const double *qn, double *qout, bool shadow_out,
                           double *drva, const RkParams &rk, cudaStream_t st) {
    switch (mode) {
        case kWrite: return launch_flux_mx_pl_m<AXIS, kWrite>(m, qn, qout, shadow_out, drva, rk, st);
        case kAccum: return launch_flux_mx_pl_m<AXIS, kAccum>(m, qn, qout, shadow_out, drva, rk, st);
        case kAccumRk: return launch_flux_mx_pl_m<AXIS, kAccumRk>(m, qn, qout, shadow_out, drva, rk, st);
        default: return launch_flux_mx_pl_m<AXIS, kWriteRk>(m, qn, qout, shadow_out, drva, rk, st);
    }
}

// Per-axis entry points of the mixed-precision passes (pipeline_mixed_axis{0,1,2}.cu).
template <int AXIS>
int launch_grad_mx_pl(const MixedArgs &m, const double *q, bool first, cudaStream_t st);
template <int AXIS>
int launch_flux_mx_pl(const MixedArgs &m, int mode, const double *qn, double *qout, bool shadow_out,
                      double *drva, const RkParams &rk, cudaStream_t st);

}  // namespace csb
