// C ABI of the numeric phase (include/sdsb200.h): plan creation, the
// factorization program interpreter, the solve with iterative refinement and
// the output accessors.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"
#include "plan.h"
#include "solve.cuh"

using namespace sds;

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& msg) {
    g_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* where) {
    return fail(SDSB200_CUDA_ERROR, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(expr, where)                              \
    do {                                             \
        cudaError_t _e = (expr);                     \
        if (_e != cudaSuccess) return cuda_fail(_e, where); \
    } while (0)

double default_eps(const Plan* P) { return P->elsize == 8 ? 1e-13 : 1e-5; }

bool interrupted(const Plan* P) { return P->interrupt && *P->interrupt != 0; }

// profiling mode: an event pair around every launch, resolved at the end of the phase
void prof_begin(Plan* P, cudaStream_t st) {
    P->launches_done++;
    if (!P->profile) return;
    size_t k = P->prof_next;
    while (P->events.size() < k + 2) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        P->events.push_back(e);
    }
    cudaEventRecord(P->events[k], st);
}

void prof_end(Plan* P, cudaStream_t st, int kind, double flops, double bytes) {
    if (!P->profile) return;
    size_t k = P->prof_next;
    cudaEventRecord(P->events[k + 1], st);
    P->pending.push_back({kind, {flops, bytes}});
    P->pending_level.push_back(P->cur_level);
    P->prof_next += 2;
}

void prof_resolve(Plan* P) {
    if (!P->profile) return;
    for (size_t q = 0; q < P->pending.size(); ++q) {
        float ms = 0, at = 0;
        cudaEventSynchronize(P->events[2 * q + 1]);
        cudaEventElapsedTime(&ms, P->events[2 * q], P->events[2 * q + 1]);
        cudaEventElapsedTime(&at, P->events[0], P->events[2 * q]);
        ProfAcc& a = P->prof[P->pending[q].first];
        P->records.push_back({P->pending[q].first, P->pending_level[q], (double)ms, (double)at,
                              P->pending[q].second.first});
        a.ms += ms;
        a.flops += P->pending[q].second.first;
        a.bytes += P->pending[q].second.second;
        a.launches++;
    }
    P->pending.clear();
    P->pending_level.clear();
    P->prof_next = 0;
}

const char* const PROF_NAMES[PK_COUNT] = {"small", "assemble", "panel", "gemm", "pivot", "scale",
                                          "stats", "fwd", "bwd", "diag", "permute", "residual", "inv"};

int prof_kind_of(LaunchKind k) {
    switch (k) {
        case L_SMALL: return PK_SMALL;
        case L_SUBTREE: return PK_SMALL;
        case L_ASSEMBLE: return PK_ASSEMBLE;
        case L_CHOL_STEP: return PK_PANEL;
        case L_CHOL_FLOW: return PK_PANEL;
        case L_GEMM: return PK_GEMM;
        case L_PIVOT_FRONT: return PK_PIVOT;
        case L_SCALE: return PK_SCALE;
        case L_DFINV: return PK_INV;
        case L_PINV: return PK_INV;
        default: return PK_STATS;
    }
}

// Run `body` (launches only, no host synchronization) captured as a CUDA graph on the plan's own
// stream, replayed while `key` is unchanged. Without graphs (or when profiling) it runs eagerly.
template <class F>
int run_graph(Plan* P, Plan::CachedGraph& g, const std::vector<uint64_t>& key, cudaStream_t st, F body) {
    if (!P->use_graphs || P->profile) return body(st);
    CK(cudaEventRecord(P->join_in, st), "join");
    CK(cudaStreamWaitEvent(P->own, P->join_in, 0), "join");
    if (!g.exec || g.key != key) {
        if (g.exec) {
            cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
        }
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(P->own, cudaStreamCaptureModeThreadLocal), "begin capture");
        const int64_t before = P->launches_done;
        int rc = body(P->own);
        cudaError_t e = cudaStreamEndCapture(P->own, &graph);
        if (rc != SDSB200_OK) {
            if (e == cudaSuccess && graph) cudaGraphDestroy(graph);
            return rc;
        }
        CK(e, "end capture");
        g.launches = P->launches_done - before;
        P->launches_done = before;
        // kernel nodes keep the priority of the stream they were captured from (the side launches' is
        // the lowest)
        e = cudaGraphInstantiateWithFlags(&g.exec, graph, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(graph);
        CK(e, "graph instantiate");
        g.key = key;
    }
    CK(cudaGraphLaunch(g.exec, P->own), "graph launch");
    P->launches_done += g.launches;
    CK(cudaEventRecord(P->join_out, P->own), "join");
    CK(cudaStreamWaitEvent(st, P->join_out, 0), "join");
    return SDSB200_OK;
}

uint64_t bits(double x) {
    uint64_t u;
    memcpy(&u, &x, sizeof(u));
    return u;
}

__global__ void absmax_kernel(const double* x, int64_t len, double* out) {
    __shared__ double red[256];
    double m = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, fabs(x[i]));
    red[threadIdx.x] = m;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + h]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        // max of nonnegative doubles: their bit patterns order the same way
        atomicMax(reinterpret_cast<unsigned long long*>(out), (unsigned long long)__double_as_longlong(red[0]));
    }
}

template <typename T>
int run_factor(Plan* P, const double* nzval, double eps, double u, int pivot, int lu_pivot, cudaStream_t st) {
    const int nm = P->nact;
    const int32_t* members = P->all_members ? nullptr : P->d_members;
    T* factor = static_cast<T*>(P->d_factor);
    T* ufactor = static_cast<T*>(P->d_ufactor);
    T* cb = static_cast<T*>(P->d_cb);
    T* work = static_cast<T*>(P->d_work);
    int last_level = -2;   // the fused subtrees' launches are level -1
    const cudaStream_t main_st = st;
    bool on_side = false, any_side = false;
    cudaStream_t last_main = main_st;
    // the extra factorization streams start after the caller's prior work on `st`
    for (int g = 1; g < P->nfstreams; ++g) {
        if (g == 1) CK(cudaEventRecord(P->fstream_fork, main_st), "stream fork");
        CK(cudaStreamWaitEvent(P->fstreams[g - 1], P->fstream_fork, 0), "stream fork");
    }
    // every stream rejoins the caller's (a capture must end joined)
    auto join_all = [&]() {
        for (int g = 1; g < P->nfstreams; ++g) {
            cudaEventRecord(P->fevents[P->nfevents + g - 1], P->fstreams[g - 1]);
            cudaStreamWaitEvent(main_st, P->fevents[P->nfevents + g - 1], 0);
        }
        if (any_side) {
            cudaEventRecord(P->side_join, P->side);
            cudaStreamWaitEvent(main_st, P->side_join, 0);
        }
    };
    for (const ProgLaunch& L : P->prog) {
        if (L.kind != L_STATS && !L.side && L.level != last_level) {
            if (interrupted(P)) {
                join_all();
                return fail(SDSB200_INTERRUPTED, "interrupted by user_host_interrupt");
            }
            last_level = L.level;
        }
        // side launches: the side stream waits for the launches so far of the stream of the batch
        // they follow, then runs them beside the following levels of the factorization
        if (L.side && !on_side) {
            CK(cudaEventRecord(P->side_fork, last_main), "side fork");
            CK(cudaStreamWaitEvent(P->side, P->side_fork, 0), "side fork");
        }
        on_side = L.side != 0;
        any_side = any_side || on_side;
        if (!on_side) last_main = L.fstream > 0 ? P->fstreams[L.fstream - 1] : main_st;
        st = on_side ? P->side : last_main;
        for (int q = 0; q < L.wait_count; ++q)
            CK(cudaStreamWaitEvent(st, P->fevents[P->fwaits[L.wait_begin + q]], 0), "stream wait");
        cudaError_t e = cudaSuccess;
        P->cur_level = L.level;
        prof_begin(P, st);
        switch (L.kind) {
            case L_SMALL:
            case L_SUBTREE: {
                SmallArgs<T> a{};
                a.maps = P->maps;
                a.list = P->d_lists + (L.kind == L_SUBTREE ? L.list2 : L.list);
                a.sub_ptr = L.kind == L_SUBTREE ? P->d_lists + L.list : nullptr;
                a.members = members;
                a.nzval = nzval;
                a.factor = factor; a.ufactor = ufactor; a.cb = cb;
                a.d = P->d_d; a.piv = P->d_piv; a.kind = P->d_kind; a.stats = P->d_stats; a.finfo = P->d_finfo;
                a.psign = P->d_psign;
                a.nnz = P->nnz; a.factor_len = P->factor_len; a.cb_len = P->cb_len; a.n = P->n;
                a.ns = (int32_t)P->ns; a.pivot = pivot; a.lu_pivot = lu_pivot; a.u = u; a.eps = eps;
                e = launch_small<T>(P->structure, a, L.count, nm, L.cls, st);
                break;
            }
            case L_ASSEMBLE: {
                LargeAsmArgs<T> a{};
                a.maps = P->maps;
                a.tasks = P->d_coltasks + L.list;
                a.count = L.count;
                a.members = members;
                a.nzval = nzval;
                a.factor = factor; a.ufactor = ufactor; a.cb = cb;
                a.nnz = P->nnz; a.factor_len = P->factor_len; a.cb_len = P->cb_len;
                e = launch_assemble_large<T>(P->structure, a, nm, st);
                break;
            }
            case L_GEMM: {
                GemmArgs<T> a{};
                a.tiles = P->d_tiles + L.list;
                a.count = L.count;
                a.members = members;
                auto buf = [&](BufId b, int64_t& stride) -> T* {
                    switch (b) {
                        case BUF_FACTOR: stride = P->factor_len; return factor;
                        case BUF_UFACTOR: stride = P->factor_len; return ufactor;
                        case BUF_CB: stride = P->cb_len; return cb;
                        case BUF_INV: stride = P->inv_len; return static_cast<T*>(P->d_inv);
                        default: stride = P->work_len; return work;
                    }
                };
                a.abuf = buf(L.abuf, a.astride);
                a.bbuf = buf(L.bbuf, a.bstride);
                a.cbuf = buf(L.cbuf, a.cstride);
                a.finfo = P->d_finfo;
                a.ns = (int32_t)P->ns;
                a.status = P->d_solve_status;
                a.copy_src = static_cast<const T*>(P->d_inv);
                a.copy_stride = P->inv_len;
                a.exact = sizeof(T) == 8 ? L.exact : 0;
                // FP32: the panel steps' rank-32 updates (C in the factor) on the SIMT pipes; the
                // contribution-block (Schur complement) updates on the tensor cores
                a.simt = (sizeof(T) == 4 && L.cbuf == BUF_FACTOR) ? 1 : 0;
                e = launch_gemm<T>(a, nm, st);
                break;
            }
            case L_CHOL_STEP: {
                CholStepArgs<T> a{};
                a.fronts = P->d_fronts;
                a.tasks = P->d_steptasks + L.list;
                a.count = L.count;
                a.members = members;
                a.factor = factor;
                a.scratch = static_cast<T*>(P->d_inv);
                a.scr_len = P->inv_len;
                a.finfo = P->d_finfo; a.stats = P->d_stats;
                a.factor_len = P->factor_len; a.ns = (int32_t)P->ns; a.kb = L.cls; a.eps = eps;
                e = launch_chol_step<T>(a, nm, st);
                break;
            }
            case L_CHOL_FLOW: {
                // single-system plans only (member 0)
                unsigned int* cnt = P->d_flow_cnt + L.list2;
                e = cudaMemsetAsync(cnt, 0, sizeof(unsigned int) * (size_t)(L.count2 + 1), st);
                if (e != cudaSuccess) break;
                CholFlowArgs<T> a{};
                a.tasks = P->d_flow_tasks + L.list;
                a.ntasks = L.count;
                a.factor = factor;
                a.scratch = static_cast<T*>(P->d_inv);
                a.finfo = P->d_finfo;
                a.stats = P->d_stats;
                a.eps = eps;
                a.cnt = cnt;
                a.ncnt = L.count2;
                a.status = P->d_flow_status;
                a.trace = P->profile ? P->d_flow_trace + 4 * L.list : nullptr;
                e = launch_chol_flow<T>(a, st);
                break;
            }
            case L_PIVOT_FRONT: {
                LargePivotArgs<T> a{};
                a.fronts = P->d_fronts;
                a.list = P->d_lists + L.list;
                a.count = L.count;
                a.members = members;
                a.factor = factor; a.ufactor = ufactor;
                a.scratch = P->d_scratch; a.scr_off = P->d_scr_off + L.cls; a.scr_len = P->scr_len;
                a.d = P->d_d; a.piv = P->d_piv; a.kind = P->d_kind; a.stats = P->d_stats; a.finfo = P->d_finfo;
                a.psign = P->d_psign; a.perm = P->d_perm0;
                a.factor_len = P->factor_len; a.n = P->n; a.ns = (int32_t)P->ns;
                a.pivot = pivot; a.lu_pivot = lu_pivot; a.u = u; a.eps = eps;
                if (L.coop >= 0 && nm == 1 && !members) {
                    e = cudaMemsetAsync(P->d_coop_bar, 0, sizeof(unsigned int) * L.count, st);
                    CoopGroups g{P->d_coop_first + L.coop, P->d_coop_bar, P->d_solve_status};
                    if (e == cudaSuccess) e = launch_large_pivot_coop<T>(P->structure, a, g, L.coop_grid, st);
                } else {
                    e = launch_large_pivot<T>(P->structure, a, nm, st);
                }
                break;
            }
            case L_SCALE: {
                ScaleArgs<T> a{};
                a.fronts = P->d_fronts;
                a.list = P->d_lists + L.list;
                a.count = L.count;
                a.woff = P->d_woff + L.cls;
                a.members = members;
                a.factor = factor; a.d = P->d_d; a.kind = P->d_kind; a.work = work;
                a.factor_len = P->factor_len; a.n = P->n; a.work_len = P->work_len;
                e = launch_scale_ld_front<T>(P->structure, a, L.maxw, nm, st);
                break;
            }
            case L_DFINV: {
                // the dataflow solve's inverses: L11^-1 of the warp fronts, 64 x 64 diagonal blocks of
                // the tiled fronts (of the L panels, and of the U^T panels for LU)
                for (int side = 0; side < (P->structure == STRUCT_G ? 2 : 1) && e == cudaSuccess; ++side) {
                    const T* panels = side ? ufactor : factor;
                    T* inv = static_cast<T*>(side ? P->d_dfinv_U : P->d_dfinv_L);
                    SmallInvArgs<T> a{};
                    a.fronts = P->d_fronts;
                    a.list = P->d_df_small + L.list;
                    a.count = L.count;
                    a.inv_off = P->d_df_inv_off;
                    a.members = members;
                    a.panels = panels;
                    a.inv = inv;
                    a.factor_len = P->factor_len;
                    a.inv_len = P->df_inv_len;
                    a.finfo = P->d_finfo;
                    a.ns = (int32_t)P->ns;
                    e = launch_small_inv<T>(a, nm, L.cls, st);
                    if (e != cudaSuccess) break;
                    BlockInvArgs<T> b{};
                    b.fronts = P->d_fronts;
                    b.tasks = P->d_df_blkinv + 2 * L.list2;
                    b.count = L.count2;
                    b.dinv_off = P->d_df_inv_off;
                    b.members = members;
                    b.panels = panels;
                    b.dinv = inv;
                    b.factor_len = P->factor_len;
                    b.dinv_len = P->df_inv_len;
                    b.finfo = P->d_finfo;
                    b.ns = (int32_t)P->ns;
                    b.panel_layout = P->df_pinv ? 1 : 0;
                    e = launch_block_inv<T>(b, nm, st);
                }
                break;
            }
            case L_PINV: {
                // one launch of the inverse-panel GEMMs (cls 1: T = L[C, A] X[A, A] into the scratch;
                // 2: X[C, A] = -X[C, C] T; 3: L21 X), for each panel set
                const int sides = P->structure == STRUCT_G ? 2 : 1;
                for (int side = 0; side < sides && e == cudaSuccess; ++side) {
                    const T* panels = side ? ufactor : factor;
                    T* pinv = static_cast<T*>(side ? P->d_dfinv_U : P->d_dfinv_L);
                    T* work = static_cast<T*>(P->d_pwork) + (int64_t)side * P->pwork_len * P->nbatch;
                    PinvGemmArgs<T> a{};
                    a.tiles = P->d_pinv_tiles + L.list;
                    a.count = L.count;
                    a.members = members;
                    a.finfo = P->d_finfo;
                    a.ns = (int32_t)P->ns;
                    a.part = static_cast<T*>(P->d_psplit);
                    a.cnt = P->d_pcnt;
                    if (L.cls == 1) {
                        a.abuf = panels; a.astride = P->factor_len;
                        a.bbuf = pinv; a.bstride = P->df_inv_len;
                        a.cbuf = work; a.cstride = P->pwork_len;
                    } else if (L.cls == 2) {
                        a.abuf = pinv; a.astride = P->df_inv_len;
                        a.bbuf = work; a.bstride = P->pwork_len;
                        a.cbuf = pinv; a.cstride = P->df_inv_len;
                    } else {
                        a.abuf = panels; a.astride = P->factor_len;
                        a.bbuf = pinv; a.bstride = P->df_inv_len;
                        a.cbuf = pinv; a.cstride = P->df_inv_len;
                    }
                    e = launch_pinv_gemm<T>(a, nm, st);
                }
                break;
            }
            case L_STATS: {
                StatsArgs a{};
                a.stats = P->d_stats;
                a.members = members;
                a.super_ptr0 = P->d_super0;
                a.perm0 = P->d_perm0;
                a.totals = P->d_totals;
                a.info = P->d_info;
                a.ns = (int32_t)P->ns;
                e = launch_stats(a, nm, st);
                break;
            }
        }
        prof_end(P, st, prof_kind_of(L.kind), L.flops * nm, L.bytes * nm);
        if (e != cudaSuccess) {
            join_all();
            return cuda_fail(e, "factorization launch");
        }
        if (L.record >= 0) CK(cudaEventRecord(P->fevents[L.record], st), "stream record");
    }
    st = main_st;
    join_all();   // the factorization ends when every stream's launches are done
    return SDSB200_OK;
}

template <typename T>
// which: 1 forward sweep, 2 diagonal, 4 backward sweep (or-ed). The unfactored Schur root (its own
// last level) is only pulled into by the forward sweep and skipped by the backward one.
int run_sweeps(Plan* P, int nrhs, bool transpose, cudaStream_t st, int which) {
    const int nm = P->nact;
    const int32_t* members = P->all_members ? nullptr : P->d_members;
    const bool gen = P->structure == STRUCT_G, ldl = P->structure == STRUCT_S;
    const T* factor = static_cast<const T*>(P->d_factor);
    const T* ufactor = static_cast<const T*>(P->d_ufactor);
    SweepArgs<T> a{};
    a.fronts = P->d_fronts;
    a.members = members;
    a.Y = P->d_Y;
    a.U = P->d_U;
    a.uoff = P->d_uoff;
    a.child_list = P->maps.child_list;
    a.relind = P->maps.relind;
    a.rowval = P->maps.rowval;
    a.n = P->n; a.factor_len = P->factor_len; a.ulen = P->ulen;
    a.nrhs = nrhs;
    a.unit = P->structure != STRUCT_SPD;
    // forward: L (reordered) or, for A^T of "G", U^T (no reordering)
    a.fac = (gen && transpose) ? ufactor : factor;
    a.piv = P->d_piv;
    a.reorder = ldl || (gen && !transpose);
    a.tiles = P->d_rect_tiles;
    auto level_sweep = [&](bool fwd, int L) -> int {
        P->cur_level = L;
        const int64_t off = P->level_list_off[L];
        const int ns_ = P->level_nsmall[L], nl_ = P->level_nlarge[L];
        double ent = P->level_panel_entries[L];   // booked on the first launch of the level
        const int pk = fwd ? PK_FWD : PK_BWD;
        const bool schur = L == P->schur_level;
        if (schur && !fwd) return SDSB200_OK;   // the Schur block of Y holds its solution already
        if (!fwd && P->level_nbtile[L]) {
            SweepArgs<T> t = a;
            t.tiles = P->d_rect_tiles + 2 * P->level_btile_off[L];
            prof_begin(P, st);
            cudaError_t e = launch_sweep_rect<T>(false, t, P->level_nbtile[L], nm, P->level_maxw_large[L], st);
            prof_end(P, st, pk, 2.0 * ent * nrhs * nm, (double)sizeof(T) * ent * nm);
            ent = 0;
            if (e != cudaSuccess) return cuda_fail(e, "backward sweep (rectangular)");
        }
        for (int part = 0; part < 2; ++part) {
            const int cnt = part == 0 ? ns_ : nl_;
            if (!cnt) continue;
            SweepArgs<T> t = a;
            t.list = P->d_level_lists + off + (part == 0 ? 0 : ns_);
            t.count = cnt;
            t.rect = part == 0;
            t.pull_only = schur;
            prof_begin(P, st);
            cudaError_t e = launch_sweep<T>(fwd, t, nm, part == 0 ? P->level_maxw_small[L] : P->level_maxw_large[L], st);
            prof_end(P, st, pk, 2.0 * ent * nrhs * nm, (double)sizeof(T) * ent * nm);
            ent = 0;
            if (e != cudaSuccess) return cuda_fail(e, fwd ? "forward sweep" : "backward sweep");
        }
        if (fwd && P->level_nftile[L]) {
            SweepArgs<T> t = a;
            t.tiles = P->d_rect_tiles + 2 * P->level_ftile_off[L];
            prof_begin(P, st);
            cudaError_t e = launch_sweep_rect<T>(true, t, P->level_nftile[L], nm, P->level_maxw_large[L], st);
            prof_end(P, st, pk, 0.0, 0.0);
            if (e != cudaSuccess) return cuda_fail(e, "forward sweep (rectangular)");
        }
        return SDSB200_OK;
    };
    for (int L = 0; (which & 1) && L < P->nlevels; ++L) {
        int rc = level_sweep(true, L);
        if (rc) return rc;
    }
    if ((which & 2) && P->structure != STRUCT_SPD) {
        DiagArgs d{};
        d.members = members; d.d = P->d_d; d.kind = P->d_kind; d.Y = P->d_Y; d.n = P->n; d.nrhs = nrhs; d.two = ldl;
        prof_begin(P, st);
        cudaError_t e = launch_diag(d, nm, st);
        prof_end(P, st, PK_DIAG, (double)P->n * nrhs * nm, 24.0 * P->n * nrhs * nm);
        if (e != cudaSuccess) return cuda_fail(e, "diagonal sweep");
    }
    a.fac = (gen && !transpose) ? ufactor : factor;
    a.reorder = ldl || (gen && transpose);
    for (int L = P->nlevels - 1; (which & 4) && L >= 0; --L) {
        int rc = level_sweep(false, L);
        if (rc) return rc;
    }
    return SDSB200_OK;
}

// the whole solve as dataflow tasks in one persistent launch per group of up to DF_MAX_NRHS
// right-hand sides (solve_dataflow.cu)
template <typename T>
int run_dataflow(Plan* P, int nrhs, bool transpose, const double* in, int64_t ldin, double* out, int64_t ldout,
                 int mode, cudaStream_t st) {
    const bool gen = P->structure == STRUCT_G, ldl = P->structure == STRUCT_S;
    const T* factor = static_cast<const T*>(P->d_factor);
    const T* ufactor = static_cast<const T*>(P->d_ufactor);
    const T* iL = static_cast<const T*>(P->d_dfinv_L);
    const T* iU = static_cast<const T*>(P->d_dfinv_U);
    DataflowArgs<T> a{};
    a.tasks = P->d_df_tasks;
    a.ntasks = P->n_df_tasks;
    a.fronts = P->d_fronts;
    a.df = P->d_df;
    a.bundles = P->d_df_bundles;
    a.rptr = P->d_df_rptr;
    a.csrc = P->d_df_csrc;
    a.facf = (gen && transpose) ? ufactor : factor;
    a.facb = (gen && !transpose) ? ufactor : factor;
    a.invf = (gen && transpose) ? iU : iL;
    a.invb = (gen && !transpose) ? iU : iL;
    a.rowval = P->maps.rowval;
    a.piv = P->d_piv;
    a.perm = P->d_perm0;
    a.d = P->d_d;
    a.kind = P->d_kind;
    a.n = P->n;
    a.Y = P->d_Y;
    a.U = P->d_U;
    a.xtmp = P->d_xtmp;
    a.part = P->d_df_part;
    unsigned int* fl = P->d_df_flags;
    const int64_t ns = P->ns;
    a.fcnt = fl;
    a.bdone = fl + ns;
    a.xflag = fl + 2 * ns;
    a.pcnt = fl + 2 * ns + P->df_nblk;
    a.tcnt = fl + 2 * ns + 2 * (int64_t)P->df_nblk;
    a.ccnt = a.tcnt + P->df_ntcnt;
    a.head = fl + P->df_flags_len * P->nbatch;   // one task counter after every member's flags
    a.status = P->d_solve_status;
    a.reorder_fw = ldl || (gen && !transpose);
    a.reorder_bw = ldl || (gen && transpose);
    a.diag_mode = P->structure == STRUCT_SPD ? 0 : (ldl ? 2 : 1);
    a.mode = mode;
    a.ldin = ldin;
    a.ldout = ldout;
    // batch members: every task once per active member, member-dependent arrays by stride
    a.nmembers = P->nact;
    a.members = P->all_members ? nullptr : P->d_members;
    a.s_fac = P->factor_len;
    a.s_inv = P->df_inv_len;
    a.s_piv = P->n;
    a.s_d = 2 * P->n;
    a.s_in = ldin * nrhs;
    a.s_out = ldout * nrhs;
    a.s_y = P->n * P->max_nrhs;
    a.s_u = P->ulen;
    a.s_part = P->df_part_len;
    a.s_flags = P->df_flags_len;
    a.trace = (P->profile && P->nact == 1) ? P->d_df_trace : nullptr;
    double ent = 0.0;
    for (double v : P->level_panel_entries) ent += v;
    for (int r0 = 0; r0 < nrhs; r0 += DF_MAX_NRHS) {
        a.nrhs = std::min(DF_MAX_NRHS, nrhs - r0);
        // shared memory: per warp of a bundle f x nrhs doubles; a tiled task 2 x 64 + DF_CHUNK rows of
        // nrhs doubles; an inverse-panel forward task DF_PCOLS + 5 x 64 rows
        a.warp_smem = (int32_t)(((int64_t)P->df_fwarp_max * a.nrhs + 1) & ~int64_t(1));
        const size_t smem = sizeof(double) * std::max<size_t>({(size_t)a.warp_smem * (DF_THREADS / 32),
                                                               (2 * DF_BLK + DF_CHUNK) * (size_t)DF_MAX_NRHS,
                                                               (DF_PCOLS + 5 * DF_BLK) * (size_t)DF_MAX_NRHS});
        const int grid = dataflow_solve_grid<T>(a.nrhs, smem);
        if (grid <= 0) return fail(SDSB200_CUDA_ERROR, "no co-resident grid for the dataflow solve");
        a.in = in + (int64_t)r0 * ldin;
        a.out = out + (int64_t)r0 * ldout;
        CK(cudaMemsetAsync(P->d_df_flags, 0, sizeof(unsigned int) * (P->df_flags_len * P->nbatch + 1), st),
           "dataflow flag reset");
        prof_begin(P, st);
        cudaError_t e = launch_dataflow_solve<T>(a, grid, smem, st);
        // algorithmic work: every stored panel entry read once per sweep (2 flops per entry and rhs
        // each way), the right-hand side read and the solution written, per member
        prof_end(P, st, PK_FWD, 4.0 * ent * a.nrhs * P->nact,
                 (2.0 * sizeof(T) * ent + 24.0 * P->n * a.nrhs) * P->nact);
        if (e != cudaSuccess) return cuda_fail(e, "dataflow solve");
    }
    return SDSB200_OK;
}

// the one-launch solve of the active members
int run_one_launch(Plan* P, int nrhs, bool transpose, const double* in, int64_t ldin, double* out, int64_t ldout,
                   int mode, cudaStream_t st) {
    return P->elsize == 8 ? run_dataflow<double>(P, nrhs, transpose, in, ldin, out, ldout, mode, st)
                          : run_dataflow<float>(P, nrhs, transpose, in, ldin, out, ldout, mode, st);
}

bool use_persistent(const Plan* P) { return P->persistent; }

int sweeps(Plan* P, int nrhs, bool transpose, cudaStream_t st, int which = 7) {
    return P->elsize == 8 ? run_sweeps<double>(P, nrhs, transpose, st, which)
                          : run_sweeps<float>(P, nrhs, transpose, st, which);
}

// mode 0: Y = in[perm], 1: out[perm] = Y, 2: out[perm] += Y; identity: factor order, no permutation
int permute(Plan* P, int mode, const double* in, int64_t ldin, double* out, int64_t ldout, int nrhs, cudaStream_t st,
            bool identity = false) {
    PermArgs a{};
    a.members = P->all_members ? nullptr : P->d_members;
    a.perm = identity ? nullptr : P->d_perm0;
    a.Y = P->d_Y;
    a.in = in; a.out = out; a.ldin = ldin; a.ldout = ldout;
    a.n = P->n; a.nrhs = nrhs; a.mode = mode;
    prof_begin(P, st);
    cudaError_t e = launch_permute(a, P->nact, st);
    prof_end(P, st, PK_PERMUTE, 0.0, (mode == 2 ? 32.0 : 20.0) * P->n * nrhs * P->nact);
    return e == cudaSuccess ? SDSB200_OK : cuda_fail(e, "permute");
}

}  // namespace

extern "C" {

const char* sdsb200_last_error(void) { return g_error.c_str(); }

void sdsb200_default_opts(sdsb200_opts* o) {
    memset(o, 0, sizeof(*o));
    o->pivot_type = PIVOT_AUTO;
    o->pivot_epsilon_alg = 0;
    o->pivot_threshold = 0.01;
    o->pivot_epsilon = -1.0;
    o->ir_n_steps = 0;
    o->ir_mode = 0;
    o->ir_tol = 0.0;
    o->solve_mode = 0;
    o->deterministic_mode = 0;
}

int sdsb200_plan_create(sdsb200_plan** plan, const sdsb200_symbolic* sym, const sdsb200_plan_options* popts,
                        void* stream) {
    if (!plan) return fail(SDSB200_INVALID_VALUE, "plan is NULL");
    *plan = nullptr;
    try {
        Plan* P = build_plan(sym, popts, (cudaStream_t)stream);
        *plan = reinterpret_cast<sdsb200_plan*>(P);
        return SDSB200_OK;
    } catch (const PlanError& e) {
        return fail(e.code, e.msg);
    } catch (const std::exception& e) {
        return fail(SDSB200_ALLOC_FAILED, e.what());
    }
}

int sdsb200_plan_destroy(sdsb200_plan* plan) {
    free_plan(reinterpret_cast<Plan*>(plan));
    return SDSB200_OK;
}

int sdsb200_factor(sdsb200_plan* plan, const double* nzval, const int8_t* h_psign, const sdsb200_opts* opts,
                   int64_t* h_info, void* stream) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P) return fail(SDSB200_INVALID_VALUE, "plan is NULL");
    if (!nzval && P->nnz > 0) return fail(SDSB200_INVALID_VALUE, "nzval is NULL");
    sdsb200_opts o;
    if (opts) o = *opts;
    else sdsb200_default_opts(&o);
    cudaStream_t st = (cudaStream_t)stream;
    int pivot = o.pivot_type;
    int lu_pivot = 1;
    if (P->structure == STRUCT_S) {
        if (pivot == PIVOT_AUTO || pivot == PIVOT_LOCAL || pivot == PIVOT_BK) pivot = PIVOT_BK;
        else if (pivot != PIVOT_NONE && pivot != PIVOT_DIAGONAL)
            return fail(SDSB200_NOT_SUPPORTED, "pivot_type is not supported by LDLT");
    } else if (P->structure == STRUCT_G) {
        if (pivot == PIVOT_NONE || pivot == PIVOT_DIAGONAL) lu_pivot = 0;
        else if (pivot != PIVOT_AUTO && pivot != PIVOT_LOCAL && pivot != PIVOT_BK)
            return fail(SDSB200_NOT_SUPPORTED, "pivot_type is not supported by LU");
    }
    double eps = o.pivot_epsilon < 0 ? default_eps(P) : o.pivot_epsilon;
    if (!(o.pivot_threshold >= 0) || !std::isfinite(o.pivot_threshold))
        return fail(SDSB200_INVALID_VALUE, "pivot_threshold must be finite and nonnegative");
    if (o.pivot_epsilon_alg == 1 && P->structure != STRUCT_SPD) {
        // scaled epsilon: eps * max |a_ij| of the first active member (one host read)
        int m0 = P->all_members ? 0 : -1;
        std::vector<int32_t> mem(1, 0);
        if (m0 < 0) CK(cudaMemcpyAsync(mem.data(), P->d_members, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "members");
        CK(cudaMemsetAsync(P->d_amax, 0, sizeof(double), st), "memset");
        absmax_kernel<<<256, 256, 0, st>>>(nzval + (int64_t)(m0 < 0 ? mem[0] : 0) * P->nnz, P->nnz, P->d_amax);
        double amax = 0;
        CK(cudaMemcpyAsync(&amax, P->d_amax, sizeof(double), cudaMemcpyDeviceToHost, st), "amax");
        CK(cudaStreamSynchronize(st), "amax sync");
        if (amax > 0) eps *= amax;
    }
    if (h_psign) CK(cudaMemcpyAsync(P->d_psign, h_psign, P->n, cudaMemcpyHostToDevice, st), "psign");
    else CK(cudaMemsetAsync(P->d_psign, 0, P->n, st), "psign");
    P->launches_done = 0;
    P->factored = false;
    if (interrupted(P)) return fail(SDSB200_INTERRUPTED, "interrupted by user_host_interrupt");
    std::vector<uint64_t> key = {(uint64_t)(uintptr_t)nzval, bits(eps), bits(o.pivot_threshold), (uint64_t)pivot,
                                 (uint64_t)lu_pivot, (uint64_t)P->nact, (uint64_t)P->all_members};
    int rc = run_graph(P, P->g_factor, key, st, [&](cudaStream_t s) -> int {
        CK(cudaMemsetAsync(P->d_finfo, 0, sizeof(int32_t) * P->ns * P->nbatch, s), "memset finfo");
        CK(cudaMemsetAsync(P->d_stats, 0, sizeof(int64_t) * NSTAT * P->ns * P->nbatch, s), "memset stats");
        return P->elsize == 8 ? run_factor<double>(P, nzval, eps, o.pivot_threshold, pivot, lu_pivot, s)
                              : run_factor<float>(P, nzval, eps, o.pivot_threshold, pivot, lu_pivot, s);
    });
    if (rc != SDSB200_OK) return rc;
    // the phase's one host synchronization: the reduced info of the active members
    CK(cudaMemcpyAsync(P->h_info_pinned, P->d_info, sizeof(int64_t) * P->nact, cudaMemcpyDeviceToHost, st), "info");
    int32_t* h_flow_status = reinterpret_cast<int32_t*>(P->h_info_pinned + P->nbatch);
    CK(cudaMemcpyAsync(h_flow_status, P->d_flow_status, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "status");
    CK(cudaStreamSynchronize(st), "factorization");
    prof_resolve(P);
    if (*h_flow_status != 0) {
        cudaMemsetAsync(P->d_flow_status, 0, sizeof(int32_t), st);
        return fail(SDSB200_TIMEOUT, "a bounded wait of the factorization's step tasks gave up");
    }
    if (h_info) {
        if (P->all_members) {
            for (int k = 0; k < P->nact; ++k) h_info[k] = P->h_info_pinned[k];
        } else {
            std::vector<int32_t> mem(P->nact);
            CK(cudaMemcpy(mem.data(), P->d_members, sizeof(int32_t) * P->nact, cudaMemcpyDeviceToHost), "members");
            for (int k = 0; k < P->nact; ++k) h_info[mem[k]] = P->h_info_pinned[k];
        }
    }
    P->factored = true;
    return SDSB200_OK;
}

int sdsb200_solve(sdsb200_plan* plan, double* X, int64_t ldx, const double* B, int64_t ldb, int32_t nrhs,
                  const double* nzval, const sdsb200_opts* opts, int32_t* h_ir_steps, void* stream) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P) return fail(SDSB200_INVALID_VALUE, "plan is NULL");
    if (!P->factored) return fail(SDSB200_PHASE_ORDER, "solve before a successful factorization");
    if (P->schur_front >= 0)
        return fail(SDSB200_NOT_SUPPORTED, "Schur complement mode: the factorization is partial; use the solve "
                                           "phases (sdsb200_solve_phase)");
    if (nrhs < 1 || nrhs > P->max_nrhs) return fail(SDSB200_INVALID_VALUE, "nrhs outside 1:max_nrhs of the plan");
    if (ldx < P->n || ldb < P->n) return fail(SDSB200_INVALID_VALUE, "leading dimension smaller than n");
    if (!X || !B) return fail(SDSB200_INVALID_VALUE, "X or B is NULL");
    sdsb200_opts o;
    if (opts) o = *opts;
    else sdsb200_default_opts(&o);
    if (o.solve_mode < 0 || o.solve_mode > 2) return fail(SDSB200_INVALID_VALUE, "solve_mode must be 0, 1 or 2");
    if (o.ir_n_steps < 0) return fail(SDSB200_INVALID_VALUE, "ir_n_steps must be nonnegative");
    const bool transpose = P->structure == STRUCT_G && o.solve_mode != 0;
    if (o.ir_n_steps > 0) {
        if (!P->has_full) return fail(SDSB200_INVALID_VALUE, "refinement needs the residual map of the plan");
        if (!nzval) return fail(SDSB200_INVALID_VALUE, "refinement needs nzval");
        if ((const double*)X == B) return fail(SDSB200_INVALID_VALUE, "X and B must differ with refinement");
    }
    cudaStream_t st = (cudaStream_t)stream;
    // max shared memory of a sweep CTA: the widest front times nrhs (chunks of right-hand sides beyond it)
    int maxw = 1;
    for (int w : P->level_maxw) maxw = std::max(maxw, w);
    if ((size_t)maxw * nrhs * sizeof(double) > 200 * 1024)
        return fail(SDSB200_NOT_SUPPORTED, "front too wide for this many right-hand sides in one solve");
    P->launches_done = 0;
    const uint64_t common = ((uint64_t)nrhs << 32) | ((uint64_t)transpose << 8) | ((uint64_t)P->all_members << 4);
    std::vector<uint64_t> key = {(uint64_t)(uintptr_t)X, (uint64_t)ldx, (uint64_t)(uintptr_t)B, (uint64_t)ldb, common,
                                 (uint64_t)P->nact};
    int rc = run_graph(P, P->g_solve, key, st, [&](cudaStream_t s) -> int {
        if (use_persistent(P)) return run_one_launch(P, nrhs, transpose, B, ldb, X, ldx, 0, s);
        int r = permute(P, 0, B, ldb, nullptr, 0, nrhs, s);
        if (r) return r;
        r = sweeps(P, nrhs, transpose, s);
        if (r) return r;
        return permute(P, 1, nullptr, 0, X, ldx, nrhs, s);
    });
    if (rc) return rc;
    int steps = 0;
    const bool check = o.ir_tol > 0;
    const int ncols = nrhs * P->nact;
    for (int it = 0; it < o.ir_n_steps; ++it) {
        if (interrupted(P)) {
            if (h_ir_steps) *h_ir_steps = steps;
            return fail(SDSB200_INTERRUPTED, "interrupted by user_host_interrupt");
        }
        std::vector<uint64_t> rkey = key;
        rkey.push_back((uint64_t)(uintptr_t)nzval);
        rkey.push_back(check);
        rc = run_graph(P, P->g_resid, rkey, st, [&](cudaStream_t s) -> int {
            ResidualArgs r{};
            r.members = P->all_members ? nullptr : P->d_members;
            if (transpose) {
                r.rowptr = P->d_fullT_rowptr; r.colval = P->d_fullT_colval; r.srcptr = P->d_fullT_srcptr;
                r.src = P->d_fullT_src;
            } else {
                r.rowptr = P->d_full_rowptr; r.colval = P->d_full_colval; r.srcptr = P->d_full_srcptr;
                r.src = P->d_full_src;
            }
            r.nzval = nzval; r.X = X; r.B = B; r.R = P->d_R;
            r.n = P->n; r.nnz = P->nnz; r.ldx = ldx; r.ldb = ldb; r.nrhs = nrhs;
            r.entries = P->full_nnz;
            prof_begin(P, s);
            cudaError_t re = launch_residual(r, P->nact, s);
            prof_end(P, s, PK_RESIDUAL, 2.0 * P->full_nnz * nrhs * P->nact,
                     (16.0 * P->full_nnz + 16.0 * P->full_nsrc) * P->nact + 24.0 * P->n * nrhs * P->nact);
            CK(re, "residual");
            if (check) {
                NormArgs na{};
                na.members = r.members; na.R = P->d_R; na.B = B; na.out = P->d_norms; na.n = P->n; na.ldb = ldb;
                na.nrhs = nrhs;
                prof_begin(P, s);
                CK(launch_norms(na, ncols, s), "norms");
                prof_end(P, s, PK_RESIDUAL, 0.0, 16.0 * P->n * ncols);
                CK(cudaMemcpyAsync(P->h_norms, P->d_norms, sizeof(double) * 2 * ncols, cudaMemcpyDeviceToHost, s),
                   "norms");
            }
            return SDSB200_OK;
        });
        if (rc) return rc;
        if (check) {
            CK(cudaStreamSynchronize(st), "norms sync");
            double rel = 0;
            for (int c = 0; c < ncols; ++c) {
                double rr = sqrt(P->h_norms[2 * c]), bb = sqrt(P->h_norms[2 * c + 1]);
                rel = std::max(rel, bb > 0 ? rr / bb : rr);
            }
            if (rel <= o.ir_tol) break;
        }
        std::vector<uint64_t> ckey = key;
        rc = run_graph(P, P->g_corr, ckey, st, [&](cudaStream_t s) -> int {
            if (use_persistent(P)) return run_one_launch(P, nrhs, transpose, P->d_R, P->n, X, ldx, 2, s);
            int r = permute(P, 0, P->d_R, P->n, nullptr, 0, nrhs, s);
            if (r) return r;
            r = sweeps(P, nrhs, transpose, s);
            if (r) return r;
            return permute(P, 2, nullptr, 0, X, ldx, nrhs, s);
        });
        if (rc) return rc;
        steps++;
    }
    if (h_ir_steps) *h_ir_steps = steps;
    CK(cudaGetLastError(), "solve");
    if (P->profile) {
        CK(cudaStreamSynchronize(st), "solve");
        prof_resolve(P);
    }
    return SDSB200_OK;
}

int sdsb200_solve_phase(sdsb200_plan* plan, int32_t phase, double* X, int64_t ldx, const double* B, int64_t ldb,
                        int32_t nrhs, const sdsb200_opts* opts, void* stream) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P) return fail(SDSB200_INVALID_VALUE, "plan is NULL");
    if (phase < SDSB200_PHASE_FWD_PERM || phase > SDSB200_PHASE_STORE)
        return fail(SDSB200_INVALID_VALUE, "unknown solve phase");
    if (!P->factored) return fail(SDSB200_PHASE_ORDER, "solve phase before a successful factorization");
    if (nrhs < 1 || nrhs > P->max_nrhs) return fail(SDSB200_INVALID_VALUE, "nrhs outside 1:max_nrhs of the plan");
    const bool reads_b = phase == SDSB200_PHASE_FWD_PERM || phase == SDSB200_PHASE_LOAD;
    const bool writes_x = phase == SDSB200_PHASE_BWD_PERM || phase == SDSB200_PHASE_STORE;
    if (reads_b && (!B || ldb < P->n)) return fail(SDSB200_INVALID_VALUE, "B is NULL or its leading dimension < n");
    if (writes_x && (!X || ldx < P->n)) return fail(SDSB200_INVALID_VALUE, "X is NULL or its leading dimension < n");
    sdsb200_opts o;
    if (opts) o = *opts;
    else sdsb200_default_opts(&o);
    if (o.solve_mode < 0 || o.solve_mode > 2) return fail(SDSB200_INVALID_VALUE, "solve_mode must be 0, 1 or 2");
    const bool transpose = P->structure == STRUCT_G && o.solve_mode != 0;
    int maxw = 1;
    for (int w : P->level_maxw) maxw = std::max(maxw, w);
    if ((size_t)maxw * nrhs * sizeof(double) > 200 * 1024)
        return fail(SDSB200_NOT_SUPPORTED, "front too wide for this many right-hand sides in one solve");
    cudaStream_t st = (cudaStream_t)stream;
    P->launches_done = 0;
    int rc = SDSB200_OK;
    switch (phase) {
        case SDSB200_PHASE_FWD_PERM: rc = permute(P, 0, B, ldb, nullptr, 0, nrhs, st); break;
        case SDSB200_PHASE_FWD: rc = sweeps(P, nrhs, transpose, st, 1); break;
        case SDSB200_PHASE_DIAG: rc = sweeps(P, nrhs, transpose, st, 2); break;
        case SDSB200_PHASE_BWD: rc = sweeps(P, nrhs, transpose, st, 4); break;
        case SDSB200_PHASE_BWD_PERM: rc = permute(P, 1, nullptr, 0, X, ldx, nrhs, st); break;
        case SDSB200_PHASE_LOAD: rc = permute(P, 0, B, ldb, nullptr, 0, nrhs, st, true); break;
        default: rc = permute(P, 1, nullptr, 0, X, ldx, nrhs, st, true); break;
    }
    if (rc) return rc;
    CK(cudaGetLastError(), "solve phase");
    if (P->profile) {
        CK(cudaStreamSynchronize(st), "solve phase");
        prof_resolve(P);
    }
    return SDSB200_OK;
}

int sdsb200_schur_matrix(sdsb200_plan* plan, int32_t member, double* D, int64_t ldd, int32_t transposed,
                         void* stream) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P) return fail(SDSB200_INVALID_VALUE, "plan is NULL");
    if (P->schur_front < 0) return fail(SDSB200_INVALID_VALUE, "the analysis has no Schur complement (schur_mode = 0)");
    if (!P->factored) return fail(SDSB200_PHASE_ORDER, "Schur complement before a successful factorization");
    if (member < 0 || member >= P->nbatch) return fail(SDSB200_INVALID_VALUE, "member out of range");
    const DFront& R = P->fronts[P->schur_front];
    if (!D || ldd < R.w) return fail(SDSB200_INVALID_VALUE, "D is NULL or its leading dimension is below the Schur order");
    cudaStream_t st = (cudaStream_t)stream;
    const bool gen = P->structure == STRUCT_G;
    cudaError_t e;
    if (P->elsize == 8) {
        const double* fac = static_cast<const double*>(P->d_factor) + (int64_t)member * P->factor_len;
        const double* ufac = gen ? static_cast<const double*>(P->d_ufactor) + (int64_t)member * P->factor_len : nullptr;
        e = launch_schur_dense<double>(fac, ufac, R.panel, R.w, D, ldd, transposed != 0, st);
    } else {
        const float* fac = static_cast<const float*>(P->d_factor) + (int64_t)member * P->factor_len;
        const float* ufac = gen ? static_cast<const float*>(P->d_ufactor) + (int64_t)member * P->factor_len : nullptr;
        e = launch_schur_dense<float>(fac, ufac, R.panel, R.w, D, ldd, transposed != 0, st);
    }
    CK(e, "Schur complement export");
    return SDSB200_OK;
}

int sdsb200_get_stats(sdsb200_plan* plan, int32_t member, int64_t* h_stats, int64_t* h_totals) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P || member < 0 || member >= P->nbatch) return fail(SDSB200_INVALID_VALUE, "bad plan or member");
    if (h_stats)
        CK(cudaMemcpy(h_stats, P->d_stats + (int64_t)member * NSTAT * P->ns, sizeof(int64_t) * NSTAT * P->ns,
                      cudaMemcpyDeviceToHost), "stats");
    if (h_totals) {
        // totals are reduced per active slot; recompute from the statistics for any member
        std::vector<int64_t> st(NSTAT * P->ns);
        CK(cudaMemcpy(st.data(), P->d_stats + (int64_t)member * NSTAT * P->ns, sizeof(int64_t) * NSTAT * P->ns,
                      cudaMemcpyDeviceToHost), "stats");
        for (int q = 0; q < NSTAT; ++q) h_totals[q] = 0;
        for (int64_t s = 0; s < P->ns; ++s) {
            for (int q = 0; q < NSTAT - 1; ++q) h_totals[q] += st[s * NSTAT + q];
            if (st[s * NSTAT + ST_INFO] != 0) h_totals[ST_INFO] += 1;
        }
    }
    return SDSB200_OK;
}

int sdsb200_get_pivots(sdsb200_plan* plan, int32_t member, int32_t* h_piv, int8_t* h_kind, double* h_d) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P || member < 0 || member >= P->nbatch) return fail(SDSB200_INVALID_VALUE, "bad plan or member");
    if (h_piv) CK(cudaMemcpy(h_piv, P->d_piv + (int64_t)member * P->n, sizeof(int32_t) * P->n, cudaMemcpyDeviceToHost), "piv");
    if (h_kind) CK(cudaMemcpy(h_kind, P->d_kind + (int64_t)member * P->n, P->n, cudaMemcpyDeviceToHost), "kind");
    if (h_d) CK(cudaMemcpy(h_d, P->d_d + (int64_t)member * 2 * P->n, sizeof(double) * 2 * P->n, cudaMemcpyDeviceToHost), "d");
    return SDSB200_OK;
}

int sdsb200_get_factor(sdsb200_plan* plan, int32_t member, double* h_factor, double* h_ufactor) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P || member < 0 || member >= P->nbatch) return fail(SDSB200_INVALID_VALUE, "bad plan or member");
    const int64_t len = P->factor_len;
    auto get = [&](const void* src, double* dst) -> int {
        if (!dst) return SDSB200_OK;
        if (P->elsize == 8) {
            CK(cudaMemcpy(dst, static_cast<const double*>(src) + member * len, sizeof(double) * len, cudaMemcpyDeviceToHost), "factor");
        } else {
            std::vector<float> tmp(len);
            CK(cudaMemcpy(tmp.data(), static_cast<const float*>(src) + member * len, sizeof(float) * len, cudaMemcpyDeviceToHost), "factor");
            for (int64_t k = 0; k < len; ++k) dst[k] = tmp[k];
        }
        return SDSB200_OK;
    };
    int rc = get(P->d_factor, h_factor);
    if (rc) return rc;
    if (h_ufactor) {
        if (!P->d_ufactor) return fail(SDSB200_INVALID_VALUE, "no U^T panels: structure is not G");
        return get(P->d_ufactor, h_ufactor);
    }
    return SDSB200_OK;
}

int sdsb200_set_members(sdsb200_plan* plan, const int32_t* h_members, int32_t nact) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P) return fail(SDSB200_INVALID_VALUE, "plan is NULL");
    if (nact < 0 || !h_members) {
        P->all_members = true;
        P->nact = P->nbatch;
        return SDSB200_OK;
    }
    if (nact == 0 || nact > P->nbatch) return fail(SDSB200_INVALID_VALUE, "nact outside 1:nbatch");
    std::vector<char> seen(P->nbatch, 0);
    for (int k = 0; k < nact; ++k) {
        if (h_members[k] < 0 || h_members[k] >= P->nbatch || seen[h_members[k]])
            return fail(SDSB200_INVALID_VALUE, "members must be distinct indices in 0:nbatch-1");
        seen[h_members[k]] = 1;
    }
    CK(cudaMemcpy(P->d_members, h_members, sizeof(int32_t) * nact, cudaMemcpyHostToDevice), "members");
    P->all_members = false;
    P->nact = nact;
    return SDSB200_OK;
}

int64_t sdsb200_get_trace(sdsb200_plan* plan, int64_t* h_out, int64_t cap) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P || !h_out) return -1;
    if (cap < 0) {
        // the factorization's Cholesky step tasks of its last profiled call, in the plan's task order
        const int64_t nt = std::min<int64_t>(-cap, P->n_flow_tasks);
        if (nt > 0 && cudaMemcpy(h_out, P->d_flow_trace, sizeof(int64_t) * 4 * nt, cudaMemcpyDeviceToHost) != cudaSuccess)
            return -1;
        return nt;
    }
    // the dataflow solve's task trace of its last profiled launch: 6 int64 per task (start and end of the
    // task and the end of its dependency wait in %globaltimer ns, CTA, kind, a | b << 32)
    const int64_t nt = std::min<int64_t>(cap, P->n_df_tasks);
    if (cudaMemcpy(h_out, P->d_df_trace, sizeof(int64_t) * 6 * nt, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return nt;
}

int sdsb200_set_persistent(sdsb200_plan* plan, int32_t on) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P) return fail(SDSB200_INVALID_VALUE, "plan is NULL");
    P->persistent = on != 0;
    for (Plan::CachedGraph* g : {&P->g_solve, &P->g_corr})
        g->key.clear();
    return SDSB200_OK;
}

int sdsb200_set_graphs(sdsb200_plan* plan, int32_t on) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P) return fail(SDSB200_INVALID_VALUE, "plan is NULL");
    P->use_graphs = on != 0;
    return SDSB200_OK;
}

int sdsb200_set_profiling(sdsb200_plan* plan, int32_t on) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P) return fail(SDSB200_INVALID_VALUE, "plan is NULL");
    P->profile = on != 0;
    P->records.clear();
    cudaMemset(P->d_df_trace, 0, sizeof(int64_t) * 6 * std::max<int64_t>(1, P->n_df_tasks));
    for (int k = 0; k < PK_COUNT; ++k) P->prof[k] = ProfAcc();
    P->pending.clear();
    P->prof_next = 0;
    return SDSB200_OK;
}

int sdsb200_set_interrupt(sdsb200_plan* plan, const volatile int32_t* h_flag) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P) return fail(SDSB200_INVALID_VALUE, "plan is NULL");
    P->interrupt = h_flag;
    return SDSB200_OK;
}

double sdsb200_plan_stat(const sdsb200_plan* plan, const char* name) {
    const Plan* P = reinterpret_cast<const Plan*>(plan);
    if (!P || !name) return -1;
    std::string nm(name);
    if (nm == "ns") return (double)P->ns;
    if (nm == "nlevels") return P->nlevels;
    if (nm == "factor_len") return (double)P->factor_len;
    if (nm == "cb_len") return (double)P->cb_len;
    if (nm == "launches_factor") return P->launches_factor;
    if (nm == "launches_solve") return 2.0 * P->nlevels + 3;
    if (nm == "device_bytes") return (double)P->device_bytes;
    if (nm == "flops") return P->flops;
    if (nm == "elsize") return P->elsize;
    if (nm == "launches_done") return (double)P->launches_done;
    if (nm == "schur_n") return P->schur_front >= 0 ? (double)P->fronts[P->schur_front].w : 0.0;
    if (nm == "schur_level") return (double)P->schur_level;
    if (nm == "subtrees") return (double)P->nsubtrees;
    if (nm == "subtree_fronts") return (double)P->nsubtree_fronts;
    if (nm == "solve_status") {
        int32_t v = 0;
        cudaDeviceSynchronize();
        cudaMemcpy(&v, P->d_solve_status, sizeof(v), cudaMemcpyDeviceToHost);
        return v;
    }
    if (nm == "prof_records") return (double)P->records.size();
    if (nm.rfind("prof_record:", 0) == 0) {
        // "prof_record:<i>:kind|level|ms|start|flops" (start: ms after the phase's first launch began)
        size_t a = nm.find(':', 12);
        if (a == std::string::npos) return -1;
        size_t i = (size_t)atol(nm.substr(12, a - 12).c_str());
        if (i >= P->records.size()) return -1;
        std::string f = nm.substr(a + 1);
        if (f == "kind") return P->records[i].kind;
        if (f == "level") return P->records[i].level;
        if (f == "ms") return P->records[i].ms;
        if (f == "start") return P->records[i].start;
        if (f == "flops") return P->records[i].flops;
        return -1;
    }
    for (int k = 0; k < PK_COUNT; ++k) {
        std::string kn(PROF_NAMES[k]);
        if (nm == "prof_ms:" + kn) return P->prof[k].ms;
        if (nm == "prof_flops:" + kn) return P->prof[k].flops;
        if (nm == "prof_bytes:" + kn) return P->prof[k].bytes;
        if (nm == "prof_launches:" + kn) return (double)P->prof[k].launches;
    }
    return -1;
}

}  // extern "C"

extern "C" int sdsb200_residual(sdsb200_plan* plan, double* R, const double* X, int64_t ldx, const double* B,
                                int64_t ldb, int32_t nrhs, const double* nzval, int32_t solve_mode, void* stream) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P) return fail(SDSB200_INVALID_VALUE, "plan is NULL");
    if (!P->has_full) return fail(SDSB200_INVALID_VALUE, "the residual needs the full-pattern map of the plan");
    if (nrhs < 1) return fail(SDSB200_INVALID_VALUE, "nrhs must be positive");
    if (ldx < P->n || ldb < P->n) return fail(SDSB200_INVALID_VALUE, "leading dimension smaller than n");
    if (!R || !X || !B || !nzval) return fail(SDSB200_INVALID_VALUE, "NULL array");
    if (solve_mode < 0 || solve_mode > 2) return fail(SDSB200_INVALID_VALUE, "solve_mode must be 0, 1 or 2");
    const bool transpose = P->structure == STRUCT_G && solve_mode != 0;
    ResidualArgs r{};
    r.members = P->all_members ? nullptr : P->d_members;
    if (transpose) {
        r.rowptr = P->d_fullT_rowptr; r.colval = P->d_fullT_colval; r.srcptr = P->d_fullT_srcptr; r.src = P->d_fullT_src;
    } else {
        r.rowptr = P->d_full_rowptr; r.colval = P->d_full_colval; r.srcptr = P->d_full_srcptr; r.src = P->d_full_src;
    }
    r.nzval = nzval; r.X = X; r.B = B; r.R = R;
    r.n = P->n; r.nnz = P->nnz; r.ldx = ldx; r.ldb = ldb; r.nrhs = nrhs;
    r.entries = P->full_nnz;
    cudaError_t e = launch_residual(r, P->nact, (cudaStream_t)stream);
    return e == cudaSuccess ? SDSB200_OK : cuda_fail(e, "residual");
}

extern "C" int sdsb200_sampled_outer(int64_t n, int64_t nnz, const void* rowptr, const void* colval,
                                     int32_t index_width, int32_t index_base, int32_t structure, int32_t view,
                                     const double* U, int64_t ldu, const double* V, int64_t ldv, int32_t ncols,
                                     int32_t nbatch, double alpha, double* out, void* stream) {
    if (n < 0 || nnz < 0 || ncols < 1 || nbatch < 1) return fail(SDSB200_INVALID_VALUE, "sampled_outer: bad sizes");
    if (index_width != 4 && index_width != 8) return fail(SDSB200_INVALID_VALUE, "index_width must be 4 or 8");
    if (index_base != 0 && index_base != 1) return fail(SDSB200_INVALID_VALUE, "index_base must be 0 or 1");
    if (structure != STRUCT_G && structure != STRUCT_S && structure != STRUCT_SPD)
        return fail(SDSB200_INVALID_VALUE, "structure must be 0 (G), 1 (S) or 3 (SPD)");
    if (view != 'F' && view != 'L' && view != 'U') return fail(SDSB200_INVALID_VALUE, "view must be 'F', 'L' or 'U'");
    if (ldu < n || ldv < n) return fail(SDSB200_INVALID_VALUE, "leading dimension smaller than n");
    if (n > 0 && (!rowptr || !U || !V || (nnz > 0 && (!colval || !out))))
        return fail(SDSB200_INVALID_VALUE, "NULL array");
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    if (index_width == 4) {
        OuterArgs<int32_t> a{static_cast<const int32_t*>(rowptr), static_cast<const int32_t*>(colval), index_base, n,
                             nnz, structure, view, U, V, ldu, ldv, ncols, alpha, out};
        e = launch_sampled_outer(a, nbatch, st);
    } else {
        OuterArgs<int64_t> a{static_cast<const int64_t*>(rowptr), static_cast<const int64_t*>(colval), index_base, n,
                             nnz, structure, view, U, V, ldu, ldv, ncols, alpha, out};
        e = launch_sampled_outer(a, nbatch, st);
    }
    return e == cudaSuccess ? SDSB200_OK : cuda_fail(e, "sampled outer product");
}

// ---------------------------------------------------------------------------
// sdsb200_solve_noalloc: the dataflow solve with its working vectors in a static device array, for
// callers that may not allocate device memory after set-up. In host code the array's name is only a
// host-side stand-in: its device address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[SDSB200_NOALLOC_SCRATCH_BYTES];

#include <mutex>

namespace {

constexpr int NOALLOC_MAX_DEVICES = 64;
constexpr size_t NOALLOC_HEADER = 512;   // the fallback status word at 256 (the first bytes unused)
std::mutex g_noalloc_mu;
void* g_noalloc_base[NOALLOC_MAX_DEVICES] = {};

// device address of the static array on the current device (looked up on the first call there)
int noalloc_base(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "sdsb200_solve_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(SDSB200_NOT_SUPPORTED, "sdsb200_solve_noalloc: device index above 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_base[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "sdsb200_solve_noalloc: cudaGetSymbolAddress of the static scratch");
        g_noalloc_base[dev] = p;
    }
    *out = g_noalloc_base[dev];
    return SDSB200_OK;
}

// Points the plan's solve working vectors at the static array for the duration of one launch and
// puts the plan's own pointers back afterwards (the launch code reads them when it builds its
// arguments, on the host, before this returns).
struct ScratchSwap {
    Plan* P;
    double* Y; double* U; double* xtmp; int32_t* status;
    ScratchSwap(Plan* p, double* y, double* u, double* xt, int32_t* st)
        : P(p), Y(p->d_Y), U(p->d_U), xtmp(p->d_xtmp), status(p->d_solve_status) {
        P->d_Y = y; P->d_U = u; P->d_xtmp = xt; P->d_solve_status = st;
    }
    ~ScratchSwap() { P->d_Y = Y; P->d_U = U; P->d_xtmp = xtmp; P->d_solve_status = status; }
};

}  // namespace

extern "C" {

int sdsb200_solve_noalloc(sdsb200_plan* plan, double* X, int64_t ldx, const double* B, int64_t ldb, int32_t nrhs,
                          int32_t solve_mode, int32_t* status, void* stream) {
    Plan* P = reinterpret_cast<Plan*>(plan);
    if (!P) return fail(SDSB200_INVALID_VALUE, "plan is NULL");
    if (!P->factored) return fail(SDSB200_PHASE_ORDER, "solve before a successful factorization");
    if (P->schur_front >= 0)
        return fail(SDSB200_NOT_SUPPORTED, "Schur complement mode: the factorization is partial; use the solve "
                                           "phases (sdsb200_solve_phase)");
    if (nrhs < 1 || nrhs > P->max_nrhs) return fail(SDSB200_INVALID_VALUE, "nrhs outside 1:max_nrhs of the plan");
    if (ldx < P->n || ldb < P->n) return fail(SDSB200_INVALID_VALUE, "leading dimension smaller than n");
    if (!X || !B) return fail(SDSB200_INVALID_VALUE, "X or B is NULL");
    if (solve_mode < 0 || solve_mode > 2) return fail(SDSB200_INVALID_VALUE, "solve_mode must be 0, 1 or 2");
    if (!(P->nact == 1 && P->all_members))
        return fail(SDSB200_NOT_SUPPORTED, "sdsb200_solve_noalloc solves a plan with exactly one batch member");
    int maxw = 1;
    for (int w : P->level_maxw) maxw = std::max(maxw, w);
    if ((size_t)maxw * nrhs * sizeof(double) > 200 * 1024)
        return fail(SDSB200_NOT_SUPPORTED, "front too wide for this many right-hand sides in one solve");
    const size_t vec = (size_t)P->n * (size_t)nrhs;
    const size_t need = NOALLOC_HEADER + sizeof(double) * (2 * vec + (size_t)P->ulen);
    if (need > SDSB200_NOALLOC_SCRATCH_BYTES)
        return fail(SDSB200_INVALID_VALUE,
                    "sdsb200_solve_noalloc: the working vectors need " + std::to_string(need) +
                        " bytes (512 + 8 * (2 * n * nrhs + ulen)), above the static scratch of " +
                        std::to_string((unsigned long long)SDSB200_NOALLOC_SCRATCH_BYTES) + " bytes");
    void* base = nullptr;
    int rc = noalloc_base(&base);
    if (rc) return rc;
    unsigned char* b = static_cast<unsigned char*>(base);
    int32_t* st_word = status ? status : reinterpret_cast<int32_t*>(b + 256);
    double* Y = reinterpret_cast<double*>(b + NOALLOC_HEADER);
    double* xt = Y + vec;
    double* U = xt + vec;
    cudaStream_t st = (cudaStream_t)stream;
    // only the status word must start at zero here (the launch sequence zeroes the plan's flags and
    // counters); Y, xtmp and the update vectors are written before they are read in every solve
    CK(cudaMemsetAsync(st_word, 0, sizeof(int32_t), st), "sdsb200_solve_noalloc: status reset");
    const bool transpose = P->structure == STRUCT_G && solve_mode != 0;
    P->launches_done = 0;
    {
        ScratchSwap swap(P, Y, U, xt, st_word);
        rc = run_one_launch(P, nrhs, transpose, B, ldb, X, ldx, 0, st);
    }
    if (rc || status) return rc;
    // no status word of the caller's: read the fallback word back (a plain copy into a host variable,
    // which allocates nothing) so that a wait that gave up is not lost
    int32_t word = 0;
    CK(cudaMemcpyAsync(&word, st_word, sizeof(word), cudaMemcpyDeviceToHost, st), "sdsb200_solve_noalloc: status read");
    CK(cudaStreamSynchronize(st), "sdsb200_solve_noalloc: status read");
    if (word != 0) return fail(SDSB200_TIMEOUT, "sdsb200_solve_noalloc: a bounded wait of the solve gave up");
    return SDSB200_OK;
}

}  // extern "C"
