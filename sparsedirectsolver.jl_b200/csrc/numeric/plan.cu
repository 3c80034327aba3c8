// Plan construction (host): validates the reference's Symbolic maps, derives the
// level schedule, classifies fronts (shared-memory fused kernel vs. large-front
// dense path), places the contribution blocks in one arena by lifetime, builds
// the launch program of the factorization and allocates every device buffer.
// Replaces allocate_numeric (src/numeric/storage.jl:205-256), NumericPlan
// (:36-104) and allocate_solve (src/solve/sweeps.jl:164-173) of the reference;
// the schedule is this library's own (levels of the supernodal tree, fronts
// binned by size), not the reference's regime A/B/C schedule.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <functional>
#include <map>
#include <queue>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "plan.h"
#include "solve.cuh"

namespace sds {
constexpr int RECT_ROWS_PLAN = RECT_ROWS, RECT_COLS_PLAN = RECT_COLS;
}

namespace sds {

namespace {

struct BuildError : std::runtime_error {
    int code;
    BuildError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

std::vector<int64_t> read_map(const void* p, int64_t len, int width, const char* name) {
    if (len < 0) throw BuildError(SDSB200_INVALID_VALUE, std::string("negative length of ") + name);
    std::vector<int64_t> out(len);
    if (len == 0) return out;
    if (!p) throw BuildError(SDSB200_INVALID_VALUE, std::string("map ") + name + " is NULL");
    if (width == 4) {
        const int32_t* q = static_cast<const int32_t*>(p);
        for (int64_t k = 0; k < len; ++k) out[k] = q[k];
    } else {
        const int64_t* q = static_cast<const int64_t*>(p);
        for (int64_t k = 0; k < len; ++k) out[k] = q[k];
    }
    return out;
}

template <class X>
X* dalloc(Plan* P, size_t count) {
    if (count == 0) count = 1;
    void* ptr = nullptr;
    cudaError_t e = cudaMalloc(&ptr, count * sizeof(X));
    if (e != cudaSuccess) throw BuildError(SDSB200_ALLOC_FAILED, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    P->allocations.push_back(ptr);
    P->device_bytes += (int64_t)(count * sizeof(X));
    return static_cast<X*>(ptr);
}

template <class X>
X* upload(Plan* P, const std::vector<X>& v, cudaStream_t st) {
    X* d = dalloc<X>(P, v.size());
    if (!v.empty()) {
        cudaError_t e = cudaMemcpyAsync(d, v.data(), v.size() * sizeof(X), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) throw BuildError(SDSB200_CUDA_ERROR, cudaGetErrorString(e));
    }
    return d;
}

int32_t to_i32(int64_t v, const char* what) {
    if (v < INT32_MIN || v > INT32_MAX) throw BuildError(SDSB200_INVALID_VALUE, std::string(what) + " overflows int32");
    return (int32_t)v;
}

// first-fit placement of intervals [start, end] of `len` elements on one arena
// Contribution-block arena: blocks live over an interval of levels [start, end] and are placed in
// order of start. Released space is kept as free segments (by offset, coalesced with neighbours, and
// by length for a best-fit search), so a placement costs O(log blocks) even with hundreds of
// thousands of blocks alive at once (uneven batches).
struct Arena {
    std::map<int64_t, int64_t> by_off;             // free segment offset -> length
    std::multimap<int64_t, int64_t> by_len;        // free segment length -> offset
    std::priority_queue<std::tuple<int, int64_t, int64_t>, std::vector<std::tuple<int, int64_t, int64_t>>,
                        std::greater<std::tuple<int, int64_t, int64_t>>> live;   // (end, offset, length)
    int64_t top = 0;
    void erase_len(int64_t len, int64_t off) {
        auto r = by_len.equal_range(len);
        for (auto it = r.first; it != r.second; ++it)
            if (it->second == off) { by_len.erase(it); return; }
    }
    void add_free(int64_t off, int64_t len) {
        auto next = by_off.lower_bound(off);
        if (next != by_off.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                off = prev->first;
                len += prev->second;
                erase_len(prev->second, prev->first);
                by_off.erase(prev);
            }
        }
        next = by_off.lower_bound(off);
        if (next != by_off.end() && off + len == next->first) {
            len += next->second;
            erase_len(next->second, next->first);
            by_off.erase(next);
        }
        by_off[off] = len;
        by_len.emplace(len, off);
    }
    int64_t place(int64_t len, int start, int end) {
        while (!live.empty() && std::get<0>(live.top()) < start) {
            add_free(std::get<1>(live.top()), std::get<2>(live.top()));
            live.pop();
        }
        int64_t at = -1;
        for (auto it = by_len.lower_bound(len); it != by_len.end(); ++it) {
            const int64_t off = it->second, seg = it->first;
            const int64_t a = (off + 31) & ~int64_t(31);
            if (a + len > off + seg) continue;
            by_len.erase(it);
            by_off.erase(off);
            if (a > off) add_free(off, a - off);
            if (a + len < off + seg) add_free(a + len, off + seg - (a + len));
            at = a;
            break;
        }
        if (at < 0) {
            at = (top + 31) & ~int64_t(31);
            top = at + len;
        }
        live.emplace(end, at, len);
        return at;
    }
};

}  // namespace

Plan* build_plan(const sdsb200_symbolic* sym, const sdsb200_plan_options* popts, cudaStream_t st) {
    Plan* P = new Plan();
    try {
        if (!sym) throw BuildError(SDSB200_INVALID_VALUE, "symbolic is NULL");
        const int width = sym->index_width;
        if (width != 4 && width != 8) throw BuildError(SDSB200_INVALID_VALUE, "index_width must be 4 or 8");
        if (sym->structure != STRUCT_G && sym->structure != STRUCT_S && sym->structure != STRUCT_SPD)
            throw BuildError(SDSB200_NOT_SUPPORTED, "structure must be G, S or SPD");
        P->n = sym->n;
        P->nnz = sym->nnz;
        P->ns = sym->ns;
        P->structure = sym->structure;
        P->nbatch = popts ? std::max(1, popts->nbatch) : 1;
        P->precision = popts ? popts->precision : SDSB200_PRECISION_FP64;
        if (P->precision != SDSB200_PRECISION_FP64 && P->precision != SDSB200_PRECISION_FP32)
            throw BuildError(SDSB200_NOT_SUPPORTED, "precision must be FP64 or FP32");
        P->elsize = P->precision == SDSB200_PRECISION_FP64 ? 8 : 4;
        P->max_nrhs = popts ? std::max(1, popts->max_nrhs) : 1;
        P->nact = P->nbatch;
        const int64_t n = P->n, ns = P->ns, nnz = P->nnz;
        if (n < 0 || ns < 0 || nnz < 0) throw BuildError(SDSB200_INVALID_VALUE, "negative size");

        std::vector<int64_t> perm = read_map(sym->perm, n, width, "perm");
        std::vector<int64_t> super_ptr = read_map(sym->super_ptr, ns + 1, width, "super_ptr");
        std::vector<int64_t> snparent = read_map(sym->snparent, ns, width, "snparent");
        std::vector<int64_t> rowptr = read_map(sym->rowptr, ns + 1, width, "rowptr");
        std::vector<int64_t> front_ptr = read_map(sym->front_ptr, ns + 1, width, "front_ptr");
        std::vector<int64_t> child_ptr = read_map(sym->child_ptr, ns + 1, width, "child_ptr");
        std::vector<int64_t> relind_ptr = read_map(sym->relind_ptr, ns + 1, width, "relind_ptr");
        std::vector<int64_t> amap_ptr = read_map(sym->amap_ptr, ns + 1, width, "amap_ptr");
        if (ns > 0 && (super_ptr[0] != 1 || super_ptr[ns] != n + 1))
            throw BuildError(SDSB200_INVALID_VALUE, "super_ptr does not cover 1:n");
        std::vector<int64_t> rowval = read_map(sym->rowval, ns ? rowptr[ns] - 1 : 0, width, "rowval");
        std::vector<int64_t> child_list = read_map(sym->child_list, ns ? child_ptr[ns] - 1 : 0, width, "child_list");
        std::vector<int64_t> relind = read_map(sym->relind, ns ? relind_ptr[ns] - 1 : 0, width, "relind");
        std::vector<int64_t> amap = read_map(sym->amap, nnz, width, "amap");
        std::vector<int64_t> amap_src = read_map(sym->amap_src, ns ? amap_ptr[ns] - 1 : 0, width, "amap_src");
        P->factor_len = ns ? front_ptr[ns] - 1 : 0;
        const bool gen = P->structure == STRUCT_G;

        // fronts
        P->fronts.resize(ns);
        for (int64_t s = 0; s < ns; ++s) {
            DFront& F = P->fronts[s];
            int64_t f = rowptr[s + 1] - rowptr[s], w = super_ptr[s + 1] - super_ptr[s];
            if (w < 1 || f < w) throw BuildError(SDSB200_INVALID_VALUE, "front with w < 1 or f < w");
            if (front_ptr[s + 1] - front_ptr[s] != f * w)
                throw BuildError(SDSB200_INVALID_VALUE, "front_ptr does not match the panel sizes");
            F.panel = front_ptr[s] - 1;
            F.cb = -1;
            F.f = to_i32(f, "front rows");
            F.w = to_i32(w, "front width");
            F.c0 = to_i32(super_ptr[s] - 1, "column");
            F.parent = to_i32(snparent[s] - 1, "snparent");
            if (F.parent >= 0 && F.parent <= s)
                throw BuildError(SDSB200_INVALID_VALUE, "supernodes must be numbered children before parents");
            F.ch_begin = to_i32(child_ptr[s] - 1, "child_ptr");
            F.ch_end = to_i32(child_ptr[s + 1] - 1, "child_ptr");
            F.ri_begin = to_i32(relind_ptr[s] - 1, "relind_ptr");
            int64_t nri = relind_ptr[s + 1] - relind_ptr[s];
            if (nri != (F.parent >= 0 ? f - w : 0))
                throw BuildError(SDSB200_INVALID_VALUE, "relind length does not match the front");
            F.am_begin = to_i32(amap_ptr[s] - 1, "amap_ptr");
            F.am_end = to_i32(amap_ptr[s + 1] - 1, "amap_ptr");
            F.row_begin = to_i32(rowptr[s] - 1, "rowptr");
            F.level = 0;
            F.rc_begin = -1;
        }
        // Schur complement mode (schedule.schur, src/symbolic/schedule.jl:351-360): a dense root
        // supernode that the factorization assembles and does not factor
        if (sym->schur != 0) {
            const int64_t r = sym->schur - 1;
            if (r < 0 || r >= ns) throw BuildError(SDSB200_INVALID_VALUE, "schur is not a supernode");
            if (P->nbatch > 1)
                throw BuildError(SDSB200_NOT_SUPPORTED, "Schur complement mode does not support uniform batches");
            const DFront& R = P->fronts[r];
            if (R.parent >= 0 || R.f != R.w)
                throw BuildError(SDSB200_INVALID_VALUE, "the Schur front must be a root with no rows below its columns");
            P->schur_front = (int)r;
        }
        // levels: height above the leaves (children are numbered first)
        for (int64_t s = 0; s < ns; ++s) {
            int p = P->fronts[s].parent;
            if (p >= 0) P->fronts[p].level = std::max(P->fronts[p].level, P->fronts[s].level + 1);
        }
        if (P->schur_front >= 0) {
            // the Schur root gets the last level to itself (src/symbolic/schedule.jl:457-458)
            int top = 0;
            for (int64_t s = 0; s < ns; ++s)
                if (s != P->schur_front) top = std::max(top, P->fronts[s].level + 1);
            P->fronts[P->schur_front].level = top;
            P->schur_level = top;
        }
        P->nlevels = 0;
        for (auto& F : P->fronts) P->nlevels = std::max(P->nlevels, F.level + 1);
        P->level_fronts.assign(P->nlevels, {});
        for (int64_t s = 0; s < ns; ++s) P->level_fronts[P->fronts[s].level].push_back((int)s);
        for (auto& F : P->fronts) {
            double f = F.f;
            for (int k = 0; k < F.w; ++k) P->flops += (f - k) * (f - k);
        }

        // assembly entries: 0-based source, signed local position, per-column starts
        std::vector<int32_t> am_src(amap_src.size()), am_loc(amap_src.size());
        std::vector<int32_t> amcol;
        for (int64_t s = 0; s < ns; ++s) {
            DFront& F = P->fronts[s];
            F.amcol_begin = (int32_t)amcol.size();
            int64_t f = F.f;
            int j = 0;
            for (int64_t k = F.am_begin; k < F.am_end; ++k) {
                int64_t p = amap_src[k] - 1;
                if (p < 0 || p >= nnz) throw BuildError(SDSB200_INVALID_VALUE, "amap_src out of range");
                int64_t off = amap[p];
                int64_t loc = (off < 0 ? -off : off) - front_ptr[s];
                if (loc < 0 || loc >= f * F.w) throw BuildError(SDSB200_INVALID_VALUE, "amap offset outside its panel");
                am_src[k] = (int32_t)p;
                am_loc[k] = (gen && off < 0) ? -(int32_t)(loc + 1) : (int32_t)(loc + 1);
                while (j <= loc / f) { amcol.push_back((int32_t)k); ++j; }
            }
            while (j <= F.w) { amcol.push_back(F.am_end); ++j; }
        }

        // small / large classification
        std::vector<int> classes = P->elsize == 8 ? std::vector<int>{32, 64, 96, 128, 160}
                                                  : std::vector<int>{32, 64, 96, 128, 160, 224};
        const int tune_fsmall = popts ? (popts->tuning & 0x1FF) : 0;
        const int tune_wide = popts ? ((popts->tuning >> 9) & 0x7FF) : 0;
        const int tune_rsv = popts ? ((popts->tuning >> 20) & 0x3F) : 0;
        const int tune_sub = popts ? ((popts->tuning >> 26) & 0xF) : 0;
        if (popts && (popts->tuning >> 30) != 0)
            throw BuildError(SDSB200_INVALID_VALUE, "tuning: bits 30 and 31 must be zero");
        if (tune_fsmall) {
            if (std::find(classes.begin(), classes.end(), tune_fsmall) == classes.end())
                throw BuildError(SDSB200_INVALID_VALUE, "tuning: fsmall must be one of the front classes");
            while (classes.back() > tune_fsmall) classes.pop_back();
        }
        if (tune_wide && (tune_wide < 16 || tune_wide > DF_WARP_F))
            throw BuildError(SDSB200_INVALID_VALUE, "tuning: wide (the tallest warp front of the solve) must lie in 16..128");
        const int tune_chains = tune_rsv & 1, tune_streams = (tune_rsv >> 1) & 15, tune_steps = (tune_rsv >> 5) & 1;
        const int warp_f = tune_wide ? tune_wide : DF_WARP_F;
        // tiled fronts solved through inverse panels (single-system plans; batches use block chains)
        const bool pinv_mode = tune_chains == 0 && P->nbatch == 1;
        P->fsmall_max = classes.back();
        auto class_of = [&](int f) {
            for (int c : classes)
                if (f <= c) return c;
            return 0;
        };

        // Factorization streams (single-system Cholesky plans): the level-batched launches run per
        // (level, stream). Walking down from the roots, a front's heaviest child subtree (by its
        // critical path of 32-column steps) stays on the front's stream and every other child subtree
        // with a critical path of at least FSTREAM_MIN_CP steps starts a new stream while fewer than
        // `streams` are in use, so that independent subtrees factor concurrently instead of level by
        // level. A front waits for its children on other streams through events.
        std::vector<int> fstream(ns, 0);
        P->nfstreams = 1;
        {
            const int want = tune_streams ? tune_streams : FSTREAM_DEFAULT;
            if (P->structure == STRUCT_SPD && P->nbatch == 1 && P->schur_front < 0 && want > 1) {
                std::vector<int64_t> cp(ns, 0);
                for (int64_t s = 0; s < ns; ++s) {   // children precede parents
                    const DFront& F = P->fronts[s];
                    cp[s] += 1 + (class_of(F.f) ? 0 : (F.w + CHOL_NB - 1) / CHOL_NB);
                    if (F.parent >= 0) cp[F.parent] = std::max(cp[F.parent], cp[s]);
                }
                for (int64_t s = ns - 1; s >= 0; --s) {
                    const DFront& F = P->fronts[s];
                    std::vector<int> kids;
                    for (int q = F.ch_begin; q < F.ch_end; ++q) kids.push_back((int)(child_list[q] - 1));
                    std::stable_sort(kids.begin(), kids.end(), [&](int a, int b) { return cp[a] > cp[b]; });
                    for (size_t q = 0; q < kids.size(); ++q) {
                        const int c = kids[q];
                        if (q > 0 && cp[c] >= FSTREAM_MIN_CP && P->nfstreams < want) fstream[c] = P->nfstreams++;
                        else fstream[c] = fstream[s];
                    }
                }
            }
        }

        // Fused subtrees (the reference's regime A, src/symbolic/schedule.jl:331-345): the maximal
        // subtrees of shared-memory fronts, on one factorization stream, with at most `maxfronts` fronts
        // and at most 1/SMs of the flops, so that a subtree's serial chain stays short and the subtrees
        // fill the device. One CTA factors each, front after front in a postorder whose children come
        // by decreasing (stack peak - contribution block) (Liu's order, as the reference's), so that the
        // subtree's stack of contribution blocks stays small; they are launched before the stream's
        // first level. tuning subtree: 1..14: subtrees of up to 2^subtree fronts; 0 and 15 (default):
        // none. A subtree runs its fronts one after another, so it pays only where the bottom levels
        // are throughput-bound (far more tiny fronts than resident CTAs: batches of small systems; the
        // autotuner tries it) and costs where a level's launch is latency-bound (lap3d 48^3, lap2d 64^2);
        // the warp-per-front launches of such batches are faster still where the fronts have at most
        // 32 rows (1024 uneven 2-D systems: 6.40 against 6.79 ms with 16-front subtrees).
        std::vector<int> sub_of(ns, -1);
        struct Sub { int root, stream, cls; int64_t stack; std::vector<int> order; std::vector<int64_t> off; };
        std::vector<Sub> subs;
        if (tune_sub != 15 && tune_sub != 0 && ns > 0) {
            const int64_t maxfronts = int64_t(1) << tune_sub;
            int dev0 = 0, sms0 = 148;
            cudaGetDevice(&dev0);
            cudaDeviceGetAttribute(&sms0, cudaDevAttrMultiProcessorCount, dev0);
            std::vector<double> work(ns, 0.0);
            double total = 0;
            for (int64_t s = 0; s < ns; ++s) {
                const double f = P->fronts[s].f;
                for (int k = 0; k < P->fronts[s].w; ++k) work[s] += (f - k) * (f - k);
                total += work[s];
            }
            std::vector<int64_t> nfr(ns, 1), peak(ns, 0), cbsz(ns, 0);
            std::vector<char> elig(ns, 0);
            std::vector<std::vector<int>> kids(ns);
            for (int64_t s = 0; s < ns; ++s) {
                const DFront& F = P->fronts[s];
                const int64_t m = F.f - F.w;
                cbsz[s] = (F.parent >= 0 && m > 0) ? ((m * m + 31) & ~int64_t(31)) : 0;
                bool e = s != P->schur_front && class_of(F.f) != 0;
                for (int q = F.ch_begin; q < F.ch_end; ++q) {
                    const int c = (int)(child_list[q] - 1);
                    kids[s].push_back(c);
                    e = e && elig[c] && fstream[c] == fstream[s];
                    nfr[s] += nfr[c];
                    work[s] += work[c];
                }
                // stack peak of the subtree below s (its own contribution block not counted)
                std::stable_sort(kids[s].begin(), kids[s].end(), [&](int a, int b) {
                    return std::max(peak[a], cbsz[a]) - cbsz[a] > std::max(peak[b], cbsz[b]) - cbsz[b];
                });
                int64_t acc = 0, pk = 0;
                for (int c : kids[s]) {
                    pk = std::max(pk, acc + std::max(peak[c], cbsz[c]));
                    acc += cbsz[c];
                }
                peak[s] = pk;
                elig[s] = e && nfr[s] <= maxfronts && work[s] <= total / std::max(sms0, 1);
            }
            for (int64_t s = 0; s < ns; ++s) {
                const DFront& F = P->fronts[s];
                if (!elig[s] || (F.parent >= 0 && elig[F.parent])) continue;
                Sub t;
                t.root = (int)s;
                t.stream = fstream[s];
                t.cls = 0;
                t.stack = 0;
                // postorder, children in the sorted order; stack offsets of the contribution blocks:
                // a front's children's blocks lie on top of the stack when it runs, and its own block
                // (written after it has read theirs) replaces them from the first one's offset
                int64_t top = 0;
                std::vector<std::pair<int, size_t>> st2{{(int)s, 0}};
                std::vector<int64_t> base{0};
                while (!st2.empty()) {
                    auto& fr = st2.back();
                    const int x = fr.first;
                    if (fr.second < kids[x].size()) {
                        const int c = kids[x][fr.second++];
                        st2.push_back({c, 0});
                        base.push_back(top);
                        continue;
                    }
                    top = base.back();
                    st2.pop_back();
                    base.pop_back();
                    sub_of[x] = (int)subs.size();
                    t.order.push_back(x);
                    t.cls = std::max(t.cls, class_of(P->fronts[x].f));
                    if (x != (int)s && cbsz[x] > 0) {
                        t.off.push_back(top);
                        top += cbsz[x];
                        t.stack = std::max(t.stack, top);
                    } else {
                        t.off.push_back(-1);
                    }
                }
                P->nsubtree_fronts += (int64_t)t.order.size();
                subs.push_back(std::move(t));
            }
            P->nsubtrees = (int64_t)subs.size();
        }

        // contribution blocks on one arena per stream, by lifetime [start, end] in the stream's launch
        // order: 0 for its fused subtrees, L + 1 for its level L. A stream's launches run in that order,
        // and the only fronts whose parent is on another stream are the tops of their streams' subtrees
        // (nothing on their stream comes after them). A fused subtree's inner blocks live on its stack
        // region (lifetime [0, 0]); its root's block lives until the root's parent's level.
        {
            std::vector<Arena> arenas(P->nfstreams);
            auto t_of = [&](int s) { return sub_of[s] >= 0 ? 0 : P->fronts[s].level + 1; };
            for (Sub& t : subs) {
                const int64_t region = t.stack > 0 ? arenas[t.stream].place(t.stack, 0, 0) : 0;
                for (size_t q = 0; q < t.order.size(); ++q)
                    if (t.off[q] >= 0) P->fronts[t.order[q]].cb = region + t.off[q];
                DFront& R = P->fronts[t.root];
                const int64_t m = R.f - R.w;
                if (R.parent >= 0 && m > 0) R.cb = arenas[t.stream].place(m * m, 0, t_of(R.parent));
            }
            for (int L = 0; L < P->nlevels; ++L)
                for (int s : P->level_fronts[L]) {
                    DFront& F = P->fronts[s];
                    int64_t m = F.f - F.w;
                    if (F.parent < 0 || m == 0 || sub_of[s] >= 0) continue;
                    F.cb = arenas[fstream[s]].place(m * m, L + 1, t_of(F.parent));
                }
            int64_t base = 0;
            for (int g = 0; g < P->nfstreams; ++g) {
                const int64_t len = (arenas[g].top + 31) & ~int64_t(31);
                for (int64_t s = 0; s < ns; ++s)
                    if (fstream[s] == g && P->fronts[s].cb >= 0) P->fronts[s].cb += base;
                base += len;
            }
            P->cb_len = base;
        }

        // column-owner extend-add lists of the large fronts
        // and each child's row-chunk starts: the parent's rows are built ASM_ROWS at a time, and the
        // child's contribution rows that land in chunk k are ii in [rchunk[k], rchunk[k + 1])
        std::vector<int32_t> ea, eacol, rchunk;
        for (int64_t s = 0; s < ns; ++s) {
            DFront& F = P->fronts[s];
            F.eacol_begin = (int32_t)eacol.size();
            if (class_of(F.f) != 0 && s != P->schur_front) continue;
            std::vector<std::vector<std::pair<int, int>>> per(F.f);
            const int nchunk = (F.f + ASM_ROWS - 1) / ASM_ROWS;
            for (int q = F.ch_begin; q < F.ch_end; ++q) {
                int c = (int)child_list[q] - 1;
                if (c < 0 || c >= ns || P->fronts[c].parent != s)
                    throw BuildError(SDSB200_INVALID_VALUE, "child_list is inconsistent with snparent");
                DFront& C = P->fronts[c];
                int mc = C.f - C.w;
                if (mc <= 0 || C.cb < 0) continue;
                C.rc_begin = (int32_t)rchunk.size();
                int prev = -1;
                for (int t = 0; t < mc; ++t) {
                    int p = (int)relind[C.ri_begin + t] - 1;
                    if (p < 0 || p >= F.f) throw BuildError(SDSB200_INVALID_VALUE, "relind out of range");
                    if (p <= prev) throw BuildError(SDSB200_INVALID_VALUE, "relind of a front is not increasing");
                    for (int k = prev < 0 ? 0 : prev / ASM_ROWS + 1; k <= p / ASM_ROWS; ++k)
                        rchunk.push_back(t);
                    prev = p;
                    per[p].push_back({c, t});
                }
                for (int k = prev / ASM_ROWS + 1; k <= nchunk; ++k) rchunk.push_back(mc);
                if ((int64_t)rchunk.size() - C.rc_begin != nchunk + 1)
                    throw BuildError(SDSB200_INVALID_VALUE, "row-chunk table of a front has the wrong length");
            }
            for (int p = 0; p < F.f; ++p) {
                eacol.push_back((int32_t)(ea.size() / 2));
                for (auto& ct : per[p]) { ea.push_back(ct.first); ea.push_back(ct.second); }
            }
            eacol.push_back((int32_t)(ea.size() / 2));
        }

        // launch program of the factorization
        std::vector<int32_t> lists;
        std::vector<CholStepTask> steptasks;
        std::vector<ColTask> coltasks;
        std::vector<GemmTile> tiles;
        std::vector<int64_t> scr_off, woff;
        // tiles of the contribution-block updates: 128 rows in FP32 (the full M of a tcgen05 MMA), 64 in
        // FP64 (the DMMA kernel's tile)
        const int cb_bm = P->elsize == 4 ? GEMM_BM_TC : GEMM_BM;
        auto add_gemm_tiles = [&](int64_t a, int lda, int64_t b, int ldb, int64_t c, int ldc, int M, int N, int K,
                                  bool lower, int front, int bm = GEMM_BM) -> double {
            // algorithmic flops: 2 K per entry of C that is written (the lower trapezoid for SYRK-like updates)
            double entries = 0;
            for (int j = 0; j < N; ++j) entries += lower ? std::max(0, M - j) : M;
            for (int ti = 0; ti < M; ti += bm)
                for (int tj = 0; tj < N; tj += GEMM_BN) {
                    int mm = std::min(bm, M - ti), nn = std::min(GEMM_BN, N - tj);
                    if (lower && ti + mm - 1 < tj) continue;
                    GemmTile t;
                    t.a = a + ti;
                    t.b = b + tj;
                    t.c = c + ti + (int64_t)tj * ldc;
                    t.lda = lda; t.ldb = ldb; t.ldc = ldc;
                    t.m = mm; t.n = nn; t.k = K;
                    t.diag = lower ? ti - tj : (1 << 29);
                    t.front = front;
                    t.mode = 0;
                    t.pad = 0;
                    tiles.push_back(t);
                }
            return 2.0 * K * entries;
        };
        // per batch (level, stream): its first and last launch, and the step scratch of each stream
        struct Batch { int level, stream; size_t first, last; };
        std::vector<Batch> batches;
        std::vector<int> batch_of(ns, -1);
        std::vector<int64_t> scr_stream(P->nfstreams, 0);   // each stream's step scratch size
        // step tasks and copy tiles whose scratch slots move to their stream's part of the scratch
        std::vector<std::vector<size_t>> step_rebase(P->nfstreams), tile_rebase(P->nfstreams);
        std::vector<std::vector<size_t>> flow_rebase(P->nfstreams);
        std::vector<FlowTask> flowtasks;
        int64_t ncnt_total = 0;
        // single-system Cholesky plans with tuning steps = 1: a batch's steps as one dataflow launch
        // (default: one launch per step and kernel, measured faster on lap3d 48^3)
        const bool flow_mode = P->nbatch == 1 && tune_steps == 1;
        // each stream's fused subtrees first, one launch per size class (a batch of level -1): per
        // launch the subtrees' starts (count + 1 entries, relative to the fronts) and then the fronts
        for (int sg = 0; sg < P->nfstreams; ++sg) {
            std::map<int, std::vector<int>> bycls;
            for (size_t t = 0; t < subs.size(); ++t)
                if (subs[t].stream == sg) bycls[subs[t].cls].push_back((int)t);
            if (bycls.empty()) continue;
            const size_t first = P->prog.size();
            for (auto& kv : bycls) {
                ProgLaunch pl{};
                pl.kind = L_SUBTREE; pl.level = -1; pl.cls = kv.first; pl.fstream = sg;
                pl.count = (int)kv.second.size();
                pl.list = (int64_t)lists.size();
                pl.list2 = pl.list + pl.count + 1;
                int32_t at = 0;
                for (int t : kv.second) {
                    lists.push_back(at);
                    at += (int32_t)subs[t].order.size();
                }
                lists.push_back(at);
                double tri = (P->structure == STRUCT_G) ? 1.0 : 0.5;
                for (int t : kv.second)
                    for (int s : subs[t].order) {
                        lists.push_back(s);
                        const DFront& F = P->fronts[s];
                        double f = F.f, w = F.w, m = F.f - F.w;
                        for (int k = 0; k < F.w; ++k) pl.flops += (f - k) * (f - k);
                        pl.bytes += P->elsize * (f * w * (gen ? 2 : 1) + (F.cb >= 0 ? tri * m * m : 0.0));
                        pl.bytes += 12.0 * (F.am_end - F.am_begin);
                        for (int q = F.ch_begin; q < F.ch_end; ++q) {
                            const DFront& C = P->fronts[child_list[q] - 1];
                            double mc = C.f - C.w;
                            pl.bytes += P->elsize * tri * mc * mc + 4.0 * mc;
                        }
                    }
                P->prog.push_back(pl);
            }
            for (size_t t = 0; t < subs.size(); ++t)
                if (subs[t].stream == sg)
                    for (int s : subs[t].order) batch_of[s] = (int)batches.size();
            batches.push_back({-1, sg, first, P->prog.size() - 1});
        }
        for (int L = 0; L < P->nlevels; ++L)
          for (int sg = 0; sg < P->nfstreams; ++sg) {
            std::map<int, std::vector<int>> small;
            std::vector<int> large;
            for (int s : P->level_fronts[L]) {
                if (fstream[s] != sg || sub_of[s] >= 0) continue;
                int c = s == P->schur_front ? 0 : class_of(P->fronts[s].f);
                if (c) small[c].push_back(s);
                else large.push_back(s);
            }
            if (small.empty() && large.empty()) continue;
            const size_t prog_first = P->prog.size();
            struct BatchEnd {   // closes the batch whatever path the body leaves by
                std::vector<Batch>& b; std::vector<int>& of; Plan* P; int L, sg; size_t first;
                const std::map<int, std::vector<int>>& sm; const std::vector<int>& lg;
                ~BatchEnd() {
                    if (P->prog.size() == first) return;
                    for (auto& kv : sm) for (int s : kv.second) of[s] = (int)b.size();
                    for (int s : lg) of[s] = (int)b.size();
                    for (size_t q = first; q < P->prog.size(); ++q) P->prog[q].fstream = sg;
                    b.push_back({L, sg, first, P->prog.size() - 1});
                }
            } batch_end{batches, batch_of, P, L, sg, prog_first, small, large};
            for (auto& kv : small) {
                ProgLaunch pl{};
                pl.kind = L_SMALL; pl.level = L; pl.count = (int)kv.second.size(); pl.cls = kv.first;
                pl.list = (int64_t)lists.size();
                lists.insert(lists.end(), kv.second.begin(), kv.second.end());
                for (int s : kv.second) {
                    const DFront& F = P->fronts[s];
                    double f = F.f, w = F.w, m = F.f - F.w;
                    for (int k = 0; k < F.w; ++k) pl.flops += (f - k) * (f - k);
                    double tri = (P->structure == STRUCT_G) ? 1.0 : 0.5;
                    pl.bytes += P->elsize * (f * w * (gen ? 2 : 1) + (F.cb >= 0 ? tri * m * m : 0.0));
                    pl.bytes += 12.0 * (F.am_end - F.am_begin);
                    for (int q = F.ch_begin; q < F.ch_end; ++q) {
                        const DFront& C = P->fronts[child_list[q] - 1];
                        double mc = C.f - C.w;
                        pl.bytes += P->elsize * tri * mc * mc + 4.0 * mc;
                    }
                }
                P->prog.push_back(pl);
            }
            if (large.empty()) continue;
            {
                ProgLaunch pl{};
                pl.kind = L_ASSEMBLE; pl.level = L; pl.list = (int64_t)coltasks.size();
                for (int s : large) {
                    const DFront& F = P->fronts[s];
                    for (int p = 0; p < F.f; ++p)
                        if (p < F.w || F.cb >= 0) coltasks.push_back({s, p});
                }
                pl.count = (int)(coltasks.size() - pl.list);
                P->prog.push_back(pl);
            }
            if (L == P->schur_level) continue;   // the Schur root is assembled, not factored
            if (P->structure == STRUCT_SPD && flow_mode) {
                // the steps as dataflow tasks in one persistent launch (kernels.cuh, FlowTask), then the
                // contribution-block update. Per front: counters of the steps' tasks done (sd), of the
                // column blocks' tiles updated by their previous step (cr), of tile 0 substituted (hd),
                // and per (block, row tile) the steps applied (tf).
                const int NB = CHOL_NB;
                ProgLaunch fl{};
                fl.kind = L_CHOL_FLOW;
                fl.level = L;
                fl.list = (int64_t)flowtasks.size();
                fl.list2 = ncnt_total;
                int32_t nc = 0;
                int64_t scr = 0;
                struct FS { int s, K; int32_t sd, cr, hd, tf; std::vector<int32_t> tf_off; std::vector<int> nt; int64_t slot0; };
                std::vector<FS> fs;
                int Kmax = 0;
                for (int s : large) {
                    const DFront& F = P->fronts[s];
                    FS x{};
                    x.s = s;
                    x.K = (F.w + NB - 1) / NB;
                    Kmax = std::max(Kmax, x.K);
                    x.sd = nc; nc += x.K;
                    x.cr = nc; nc += x.K;
                    x.hd = nc; nc += x.K;
                    x.tf = nc;
                    for (int j = 0; j < x.K; ++j) {
                        x.tf_off.push_back(nc - x.tf);
                        nc += (F.f - NB * j + 63) / 64;
                    }
                    for (int k = 0; k < x.K; ++k) {
                        const int nbb = std::min(NB, F.w - NB * k), rows = F.f - (NB * k + nbb);
                        x.nt.push_back(rows > 0 ? (rows + 63) / 64 : 1);
                    }
                    x.slot0 = scr;
                    scr += (int64_t)NB * NB * x.K;
                    fs.push_back(std::move(x));
                }
                // the update of step k on column block j (j >= k + 2; block k + 1 is updated by the
                // step's own tasks), every row tile of the block
                auto upd = [&](const FS& x, int k, int j) {
                    const DFront& F = P->fronts[x.s];
                    const int nr = (F.f - NB * j + 63) / 64;
                    for (int r = 0; r < nr; ++r) {
                        FlowTask t{};
                        t.kind = FLOW_UPD; t.front = x.s; t.kb = NB * k; t.a = NB * j; t.b = NB * j + 64 * r;
                        t.w1 = x.sd + k; t.v1 = x.nt[k];
                        t.w2 = k > 0 ? x.tf + x.tf_off[j] + r : -1; t.v2 = k;
                        t.sig_store = x.tf + x.tf_off[j] + r; t.sig_val = k + 1;
                        t.sig_add = -1; t.sig_mid = -1; t.sig_head = -1; t.w_mid = -1;
                        t.f = F.f; t.w = F.w; t.panel = F.panel; t.scr = 0;
                        flowtasks.push_back(t);
                        fl.flops += 2.0 * std::min(64, F.f - t.b) * std::min(NB, F.w - t.a) * NB;
                    }
                };
                for (int k = 0; k < Kmax; ++k) {
                    for (const FS& x : fs)   // the previous step's updates of this step's next block
                        if (k >= 1 && k + 1 < x.K) upd(x, k - 1, k + 1);
                    for (const FS& x : fs) {
                        if (k >= x.K) continue;
                        const DFront& F = P->fronts[x.s];
                        const int nbb = std::min(NB, F.w - NB * k), rows = F.f - (NB * k + nbb);
                        const bool next = k + 1 < x.K;   // STEPN: the step also updates block k + 1
                        for (int t = 0; t < x.nt[k]; ++t) {
                            FlowTask ft{};
                            ft.kind = next ? FLOW_STEPN : FLOW_STEP; ft.front = x.s; ft.kb = NB * k;
                            ft.a = rows > 0 ? t : -1; ft.b = 0;
                            ft.w1 = k > 0 ? x.cr + k : -1;
                            ft.v1 = k > 0 ? (F.f - NB * k + 63) / 64 : 0;
                            ft.w2 = next && k > 0 ? x.tf + x.tf_off[k + 1] + t : -1;
                            ft.v2 = k;
                            if (next) {
                                ft.sig_mid = x.sd + k;
                                ft.sig_head = t == 0 ? x.hd + k : -1;
                                ft.w_mid = t > 0 ? x.hd + k : -1;
                                ft.sig_store = x.tf + x.tf_off[k + 1] + t; ft.sig_val = k + 1;
                                ft.sig_add = x.cr + k + 1;
                            } else {
                                ft.sig_mid = -1; ft.sig_head = -1; ft.w_mid = -1; ft.sig_store = -1;
                                ft.sig_add = x.sd + k;
                            }
                            ft.f = F.f; ft.w = F.w; ft.panel = F.panel;
                            ft.scr = rows > 0 ? x.slot0 + (int64_t)NB * NB * k : 0;
                            if (rows > 0) flow_rebase[sg].push_back(flowtasks.size());
                            flowtasks.push_back(ft);
                        }
                        fl.flops += 2.0 * nbb * nbb * nbb / 3.0 + 2.0 * (double)std::max(rows, 0) * nbb * nbb;
                        if (next) fl.flops += 2.0 * (F.f - NB * (k + 1)) * std::min(NB, F.w - NB * (k + 1)) * NB;
                        if (rows > 0) {
                            FlowTask ct{};
                            ct.kind = FLOW_COPY; ct.front = x.s; ct.kb = NB * k;
                            ct.w1 = x.sd + k; ct.v1 = x.nt[k]; ct.w2 = -1;
                            ct.sig_add = -1; ct.sig_store = -1; ct.sig_mid = -1; ct.sig_head = -1; ct.w_mid = -1;
                            ct.f = F.f; ct.w = F.w; ct.panel = F.panel;
                            ct.scr = x.slot0 + (int64_t)NB * NB * k;
                            flow_rebase[sg].push_back(flowtasks.size());
                            flowtasks.push_back(ct);
                        }
                    }
                    for (const FS& x : fs)   // the previous step's updates beyond
                        for (int j = k + 2; k >= 1 && j < x.K; ++j) upd(x, k - 1, j);
                }
                fl.count = to_i32((int64_t)flowtasks.size() - fl.list, "flow tasks");
                fl.count2 = nc;
                ncnt_total += nc + 1;
                scr_stream[sg] = std::max(scr_stream[sg], scr);
                if (fl.count) P->prog.push_back(fl);
                ProgLaunch cl{};
                cl.kind = L_GEMM; cl.level = L; cl.list = (int64_t)tiles.size();
                cl.abuf = cl.bbuf = BUF_FACTOR; cl.cbuf = BUF_CB;
                for (int s : large) {
                    const DFront& F = P->fronts[s];
                    int m = F.f - F.w;
                    if (F.cb < 0 || m == 0) continue;
                    cl.flops += add_gemm_tiles(F.panel + F.w, F.f, F.panel + F.w, F.f, F.cb, m, m, m, F.w, true, s, cb_bm);
                }
                cl.count = (int)(tiles.size() - cl.list);
                if (cl.count) P->prog.push_back(cl);
            } else if (P->structure == STRUCT_SPD) {
                const int NB = CHOL_NB;
                int maxw = 0;
                for (int s : large) maxw = std::max(maxw, P->fronts[s].w);
                // L11 of every (front, step) of the level gets its own scratch slot; it reaches the
                // panel through a copy tile of the step's update GEMM, or of the contribution-block
                // GEMM for a front's last step
                int64_t scr = 0;
                std::vector<std::pair<int, int64_t>> last_copy;
                auto copy_tile = [&](int s, int64_t slot, int kb) {
                    const DFront& F = P->fronts[s];
                    const int nbb = std::min(NB, F.w - kb);
                    GemmTile t{};
                    t.a = slot; t.lda = NB;
                    t.b = 0; t.ldb = 1;
                    t.c = F.panel + kb + (int64_t)kb * F.f; t.ldc = F.f;
                    t.m = nbb; t.n = nbb; t.k = 0;
                    t.diag = 1 << 29;
                    t.front = -1;
                    t.mode = 2;
                    tile_rebase[sg].push_back(tiles.size());
                    tiles.push_back(t);
                };
                for (int kb = 0; kb < maxw; kb += NB) {
                    ProgLaunch sl{};
                    sl.kind = L_CHOL_STEP; sl.level = L; sl.cls = kb; sl.nb = NB;
                    sl.list = (int64_t)steptasks.size();
                    std::vector<std::pair<int, int64_t>> step_copy;
                    for (int s : large) {
                        const DFront& F = P->fronts[s];
                        if (F.w <= kb) continue;
                        const int nbb = std::min(NB, F.w - kb), r1 = kb + nbb, rows = F.f - r1;
                        if (rows <= 0) {
                            steptasks.push_back({s, -1, 0, F.panel, F.f, F.w});
                        } else {
                            const int64_t slot = scr;
                            scr += (int64_t)NB * NB;
                            for (int t = 0; t * 64 < rows; ++t) {
                                step_rebase[sg].push_back(steptasks.size());
                                steptasks.push_back({s, t, slot, F.panel, F.f, F.w});
                            }
                            if (F.w > kb + NB) step_copy.push_back({s, slot});
                            else last_copy.push_back({s, slot});
                        }
                        sl.flops += 2.0 * nbb * nbb * nbb / 3.0 + 2.0 * (double)std::max(rows, 0) * nbb * nbb;
                        sl.bytes += P->elsize * (2.0 * nbb * nbb + 2.0 * std::max(rows, 0) * (double)nbb);
                    }
                    sl.count = (int)(steptasks.size() - sl.list);
                    P->prog.push_back(sl);
                    ProgLaunch gl{};
                    gl.kind = L_GEMM; gl.level = L; gl.list = (int64_t)tiles.size();
                    gl.abuf = gl.bbuf = gl.cbuf = BUF_FACTOR;
                    for (int s : large) {
                        const DFront& F = P->fronts[s];
                        if (F.w <= kb + NB) continue;
                        int k1 = kb + NB;
                        int64_t f = F.f;
                        gl.flops += add_gemm_tiles(F.panel + k1 + (int64_t)kb * f, F.f, F.panel + k1 + (int64_t)kb * f,
                                                   F.f, F.panel + k1 + (int64_t)k1 * f, F.f, F.f - k1, F.w - k1, NB,
                                                   true, s);
                    }
                    for (auto& sc2 : step_copy) copy_tile(sc2.first, sc2.second, kb);
                    gl.count = (int)(tiles.size() - gl.list);
                    if (gl.count) P->prog.push_back(gl);
                }
                scr_stream[sg] = std::max(scr_stream[sg], scr);
                ProgLaunch cl{};
                cl.kind = L_GEMM; cl.level = L; cl.list = (int64_t)tiles.size();
                cl.abuf = cl.bbuf = BUF_FACTOR; cl.cbuf = BUF_CB;
                for (int s : large) {
                    const DFront& F = P->fronts[s];
                    int m = F.f - F.w;
                    if (F.cb < 0 || m == 0) continue;
                    cl.flops += add_gemm_tiles(F.panel + F.w, F.f, F.panel + F.w, F.f, F.cb, m, m, m, F.w, true, s, cb_bm);
                }
                cl.count = (int)(tiles.size() - cl.list);
                if (cl.count) P->prog.push_back(cl);
                if (!last_copy.empty()) {
                    // the last diagonal blocks go to the panel (factor buffer), not to the CB arena
                    ProgLaunch ql{};
                    ql.kind = L_GEMM; ql.level = L; ql.list = (int64_t)tiles.size();
                    ql.abuf = ql.bbuf = ql.cbuf = BUF_FACTOR;
                    for (auto& lc2 : last_copy) {
                        const DFront& F = P->fronts[lc2.first];
                        copy_tile(lc2.first, lc2.second, ((F.w - 1) / NB) * NB);
                    }
                    ql.count = (int)(tiles.size() - ql.list);
                    P->prog.push_back(ql);
                }
            } else {
                ProgLaunch pl{};
                pl.kind = L_PIVOT_FRONT; pl.level = L; pl.list = (int64_t)lists.size(); pl.count = (int)large.size();
                pl.cls = (int)scr_off.size();
                int64_t so = 0;
                for (int s : large) {
                    const DFront& F = P->fronts[s];
                    lists.push_back(s);
                    scr_off.push_back(so);
                    so += pivot_scratch_len(F.f, F.w);
                }
                P->scr_len = std::max(P->scr_len, so);
                P->prog.push_back(pl);
                std::vector<int> withcb;
                for (int s : large)
                    if (P->fronts[s].cb >= 0) withcb.push_back(s);
                if (!withcb.empty()) {
                    ProgLaunch sl{};
                    sl.kind = L_SCALE;
                    sl.level = L; sl.list = (int64_t)lists.size(); sl.count = (int)withcb.size();
                    sl.cls = (int)woff.size();
                    int64_t wo = 0;
                    int maxw = 0;
                    ProgLaunch gl{};
                    gl.kind = L_GEMM; gl.level = L;
                    gl.abuf = BUF_WORK; gl.bbuf = gen ? BUF_UFACTOR : BUF_FACTOR; gl.cbuf = BUF_CB;
                    gl.exact = gen ? 2 : 1;
                    gl.list = (int64_t)tiles.size();
                    for (int s : withcb) {
                        const DFront& F = P->fronts[s];
                        int m = F.f - F.w;
                        lists.push_back(s);
                        woff.push_back(wo);
                        gl.flops += add_gemm_tiles(wo, m, F.panel + F.w, F.f, F.cb, m, m, m, F.w, !gen, s, cb_bm);
                        wo += ((int64_t)m * F.w + 31) & ~int64_t(31);
                        maxw = std::max(maxw, F.w);
                    }
                    sl.maxw = maxw;
                    P->work_len = std::max(P->work_len, wo);
                    P->prog.push_back(sl);
                    gl.count = (int)(tiles.size() - gl.list);
                    P->prog.push_back(gl);
                }
            }
        }
        // the streams' step scratch side by side; events between the streams' batches: a batch waits for
        // the batches of its fronts' children on other streams (each the top of its stream's subtree)
        {
            int64_t base = 0;
            for (int g = 0; g < P->nfstreams; ++g) {
                for (size_t i : step_rebase[g]) steptasks[i].scr += base;
                for (size_t i : tile_rebase[g]) tiles[i].a += base;
                for (size_t i : flow_rebase[g]) flowtasks[i].scr += base;
                base += scr_stream[g];
            }
            P->d_flow_tasks = upload(P, flowtasks, st);
            P->n_flow_tasks = (int64_t)flowtasks.size();
            P->d_flow_trace = dalloc<int64_t>(P, 4 * std::max<int64_t>(1, P->n_flow_tasks));
            P->flow_cnt_len = ncnt_total;
            P->inv_len = std::max(P->inv_len, base);
            std::vector<int> ev_of_batch(batches.size(), -1);
            std::vector<std::vector<int>> waits(batches.size());
            int nev = 0;
            for (int64_t s = 0; s < ns; ++s) {
                const int p = P->fronts[s].parent;
                if (p < 0 || batch_of[s] < 0 || batch_of[p] < 0 || fstream[s] == fstream[p]) continue;
                const int cb_ = batch_of[s], pb = batch_of[p];
                if (ev_of_batch[cb_] < 0) {
                    ev_of_batch[cb_] = nev++;
                    P->prog[batches[cb_].last].record = ev_of_batch[cb_];
                }
                if (std::find(waits[pb].begin(), waits[pb].end(), ev_of_batch[cb_]) == waits[pb].end())
                    waits[pb].push_back(ev_of_batch[cb_]);
            }
            for (size_t bi = 0; bi < batches.size(); ++bi) {
                if (waits[bi].empty()) continue;
                ProgLaunch& first = P->prog[batches[bi].first];
                first.wait_begin = (int32_t)P->fwaits.size();
                first.wait_count = (int32_t)waits[bi].size();
                P->fwaits.insert(P->fwaits.end(), waits[bi].begin(), waits[bi].end());
            }
            P->nfevents = nev;
        }
        // dataflow solve: front classes, task list, inverse layout, contribution lists (solve.cuh)
        {
            std::vector<DfFront> df(ns);
            std::vector<int64_t> inv_off(ns, -1);
            std::vector<int32_t> small_list, blkinv;
            int64_t il = 0;
            int32_t nblk = 0, npart = 0, ntcnt = 0, nccnt = 0;
            for (int64_t s = 0; s < ns; ++s) {
                const DFront& F = P->fronts[s];
                DfFront& d = df[s];
                d = DfFront{};
                if (s == P->schur_front) continue;
                const int m = F.f - F.w;
                d.tiled = !(F.w <= DF_WARP_W && F.f <= warp_f);
                d.inv = inv_off[s] = il;
                d.bsig = 1;
                if (!d.tiled) {
                    il += ((int64_t)F.w * F.w + 1) & ~int64_t(1);
                    d.fsig = 1;
                    small_list.push_back((int32_t)s);
                    P->df_fwarp_max = std::max(P->df_fwarp_max, F.f);
                } else if (pinv_mode) {
                    // the f x w inverse panel; its diagonal blocks come from the block-inverse launch
                    d.pinv = 1;
                    d.nblk = (F.w + DF_BLK - 1) / DF_BLK;
                    d.ntile = (F.f + DF_BLK - 1) / DF_BLK;
                    d.pbblk = (F.w + DF_PBCOLS - 1) / DF_PBCOLS;
                    d.fsig = d.ntile;
                    d.bsig = d.pbblk;
                    d.tcnt = ntcnt;
                    d.ccnt = nccnt;
                    ntcnt += d.ntile;
                    nccnt += d.pbblk;
                    il += ((int64_t)F.f * F.w + 1) & ~int64_t(1);
                    for (int b = 0; b < d.nblk; ++b) {
                        blkinv.push_back((int32_t)s);
                        blkinv.push_back(b);
                    }
                } else {
                    d.nblk = (F.w + DF_BLK - 1) / DF_BLK;
                    d.ntile = (F.f + DF_BLK - 1) / DF_BLK;
                    d.nchunk = m > DF_CHUNK ? (m + DF_CHUNK - 1) / DF_CHUNK : 0;
                    d.blk = nblk;
                    d.part = npart;
                    d.fsig = d.ntile;
                    nblk += d.nblk;
                    npart += d.nblk * d.nchunk;
                    il += (int64_t)d.nblk * DF_BLK * DF_BLK;
                    for (int b = 0; b < d.nblk; ++b) {
                        blkinv.push_back((int32_t)s);
                        blkinv.push_back(b);
                    }
                }
            }
            for (int64_t s = 0; s < ns; ++s)
                if (s != P->schur_front && P->fronts[s].parent >= 0) df[P->fronts[s].parent].fneed += df[s].fsig;
            // global update rows (U of the dataflow solve is (update row) x nrhs, row-major) and the
            // per-row contribution lists: for every front row, the children's update rows that land on
            // it, in child order (the order of the level kernels' pulls)
            std::vector<int32_t> rptr, csrc;
            {
                int64_t ur = 0, rb = 0;
                for (int64_t s = 0; s < ns; ++s) {
                    df[s].urow = to_i32(ur, "update rows");
                    df[s].rbase = to_i32(rb, "front rows");
                    ur += P->fronts[s].f - P->fronts[s].w;
                    rb += P->fronts[s].f + 1;
                }
                rptr.assign(rb, 0);
                std::vector<std::pair<int32_t, int32_t>> hits;   // (front row, global update row)
                for (int64_t s = 0; s < ns; ++s) {
                    const DFront& F = P->fronts[s];
                    hits.clear();
                    for (int cq = F.ch_begin; cq < F.ch_end; ++cq) {
                        const int c = (int)(child_list[cq] - 1);
                        const DFront& Cf = P->fronts[c];
                        const int mc = Cf.f - Cf.w;
                        for (int i2 = 0; i2 < mc; ++i2)
                            hits.push_back({(int32_t)(relind[Cf.ri_begin + i2] - 1), df[c].urow + i2});
                    }
                    std::stable_sort(hits.begin(), hits.end(),
                                     [](const std::pair<int32_t, int32_t>& x, const std::pair<int32_t, int32_t>& y) {
                                         return x.first < y.first;
                                     });
                    const int64_t base = df[s].rbase;
                    size_t h = 0;
                    for (int p2 = 0; p2 <= F.f; ++p2) {
                        rptr[base + p2] = to_i32((int64_t)csrc.size(), "contributions");
                        if (p2 == F.f) break;
                        while (h < hits.size() && hits[h].first == p2) csrc.push_back(hits[h++].second);
                    }
                    if (h != hits.size()) throw BuildError(SDSB200_INVALID_VALUE, "relind outside the parent's rows");
                }
            }
            std::vector<DfTask> tasks;
            std::vector<int32_t> bundles;
            // a level's warp fronts in bundles of at least DF_BUNDLE, more when the level has more fronts
            // than 8 per resident CTA: a bundle's warps take its fronts in turn, so a warp whose front
            // waits long holds up fewer others, and the CTAs spend fewer task switches
            int dev_ = 0, sms_ = 148;
            cudaGetDevice(&dev_);
            cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev_);
            const size_t df_ctas = 2 * (size_t)std::max(sms_, 1);
            auto push_bundles = [&](int L, int kind) {
                std::vector<int32_t> wl;
                for (int s : P->level_fronts[L])
                    if (s != P->schur_front && !df[s].tiled) wl.push_back(s);
                const size_t bsz = std::max<size_t>(DF_BUNDLE, (wl.size() + df_ctas - 1) / df_ctas);
                for (size_t o = 0; o < wl.size(); o += bsz) {
                    const int cnt = (int)std::min<size_t>(bsz, wl.size() - o);
                    tasks.push_back(DfTask{kind, (int32_t)bundles.size(), cnt, 0});
                    bundles.insert(bundles.end(), wl.begin() + o, wl.begin() + o + cnt);
                }
            };
            // partial-product slots of the inverse-panel tasks: one per task of a tile (block) that has
            // more than one; the task record carries the tile's (block's) first slot
            int64_t npslot = 0;
            auto slot_field = [&](int chunk, int nchunks) {
                if (nchunks > 1 && npslot + nchunks > (int64_t(1) << 22))
                    throw BuildError(SDSB200_INVALID_VALUE, "dataflow solve: too many partial slots");
                return (int32_t)(chunk | ((nchunks > 1 ? npslot : 0) << 8));
            };
            for (int L = 0; L < P->nlevels; ++L) {
                for (int s : P->level_fronts[L]) {
                    if (s == P->schur_front || !df[s].tiled) continue;
                    if (df[s].pinv) {
                        const int w = P->fronts[s].w;
                        if ((w + DF_PCOLS - 1) / DF_PCOLS > 255)
                            throw BuildError(SDSB200_INVALID_VALUE, "dataflow solve: front too wide for the inverse panels");
                        for (int t = 0; t < df[s].ntile; ++t) {
                            const int nk = df_pf_chunks(w, t);
                            for (int k = 0; k < nk; ++k) tasks.push_back(DfTask{DF_FW_PINV, s, t, slot_field(k, nk)});
                            if (nk > 1) npslot += nk;
                        }
                    } else {
                        for (int t = 0; t < df[s].ntile; ++t) tasks.push_back(DfTask{DF_FW_TILE, s, t, 0});
                    }
                }
                push_bundles(L, DF_FW_BUNDLE);
            }
            for (int L = P->nlevels - 1; L >= 0; --L) {
                for (int s : P->level_fronts[L]) {
                    if (s == P->schur_front || !df[s].tiled) continue;
                    if (df[s].pinv) {
                        const int f = P->fronts[s].f;
                        if ((f + DF_PROWS - 1) / DF_PROWS > 255)
                            throw BuildError(SDSB200_INVALID_VALUE, "dataflow solve: front too tall for the inverse panels");
                        for (int b = df[s].pbblk - 1; b >= 0; --b) {
                            const int nr = df_pb_chunks(f, b), r0 = df_pb_first(b);
                            for (int k = 0; k < nr; ++k)
                                tasks.push_back(DfTask{DF_BW_PINV, s, b, slot_field(r0 + k, nr)});
                            if (nr > 1) npslot += nr;
                        }
                    } else {
                        for (int b = 0; b < df[s].nblk; ++b)
                            for (int c = 0; c < df[s].nchunk; ++c) tasks.push_back(DfTask{DF_BW_PART, s, b, c});
                        for (int b = df[s].nblk - 1; b >= 0; --b) tasks.push_back(DfTask{DF_BW_OWNER, s, b, 0});
                    }
                }
                push_bundles(L, DF_BW_BUNDLE);
            }
            P->df_inv_len = std::max<int64_t>(il, 2);
            P->df_nblk = nblk;
            P->df_ntcnt = ntcnt;
            P->df_nccnt = nccnt;
            P->df_pinv = pinv_mode;
            // fcnt, bdone (ns each), xflag, pcnt (nblk each), tcnt, ccnt, the task counter
            P->df_flags_len = 2 * ns + 2 * (int64_t)nblk + ntcnt + nccnt + 8;
            P->n_df_tasks = (int32_t)tasks.size();
            P->n_df_small = (int32_t)small_list.size();
            P->n_df_blkinv = (int32_t)(blkinv.size() / 2);
            P->d_df = upload(P, df, st);
            P->d_df_tasks = upload(P, tasks, st);
            P->d_df_bundles = upload(P, bundles, st);
            P->d_df_inv_off = upload(P, inv_off, st);

            P->d_df_rptr = upload(P, rptr, st);
            P->d_df_csrc = upload(P, csrc, st);
            P->df_part_len = std::max<int64_t>(1, std::max<int64_t>(npart, npslot) * DF_BLK * DF_MAX_NRHS);
            P->d_df_part = dalloc<double>(P, P->df_part_len * P->nbatch);
            P->d_df_flags = dalloc<unsigned int>(P, P->df_flags_len * P->nbatch + 1);
            P->d_df_trace = dalloc<int64_t>(P, 6 * (int64_t)std::max<int32_t>(1, P->n_df_tasks));
            // The inverses are built level by level on the side stream, each level's right after its
            // factorization launches (single-system plans only: a batch is solved by the per-level
            // sweeps). Per level: the warp fronts' L11^-1 and the tiled fronts' 64 x 64 diagonal-block
            // inverses; then for the inverse-panel fronts L11^-1 by recursive doubling over those blocks
            // (at each doubling level, for every pair of adjacent aligned block ranges A (full, h blocks)
            // and C (up to h blocks): T = L[C, A] X[A, A] into the scratch, X[C, A] = -X[C, C] T) and
            // the update rows L21 X. X lives in the inverse panel (ld f).
            if (P->nbatch == 1) {
                std::map<std::pair<int, int>, std::vector<ProgLaunch>> side;   // per batch (level, stream)
                std::vector<int32_t> small_sorted, blk_sorted;
                std::vector<PinvTile> pt;
                auto bw_of = [](int w, int b) { return std::min(DF_BLK, w - DF_BLK * b); };
                int64_t pwork = 0;
                // batch "level" -1: the stream's fused subtrees
                for (int L = -1; L < P->nlevels; ++L)
                  for (int sg = 0; sg < P->nfstreams; ++sg) {
                    std::vector<int> lf;
                    if (L < 0) {
                        for (int L2 = 0; L2 < P->nlevels; ++L2)
                            for (int s : P->level_fronts[L2])
                                if (sub_of[s] >= 0) lf.push_back(s);
                    } else {
                        for (int s : P->level_fronts[L])
                            if (sub_of[s] < 0) lf.push_back(s);
                    }
                    if (lf.empty()) continue;
                    std::vector<ProgLaunch>& side_b = side[{L, sg}];
                    std::vector<int> pf;   // the batch's inverse-panel fronts
                    // the warp fronts' L11^-1 in one launch per width class (8, 16, 32: the narrow
                    // kernels hold far fewer registers); the first also takes the diagonal blocks
                    std::vector<int32_t> by_w[3];
                    const int64_t blk0 = (int64_t)blk_sorted.size() / 2;
                    for (int s : lf) {
                        if (s == P->schur_front || fstream[s] != sg) continue;
                        if (!df[s].tiled) {
                            const int w = P->fronts[s].w;
                            by_w[w <= 8 ? 0 : w <= 16 ? 1 : 2].push_back(s);
                            continue;
                        }
                        for (int b = 0; b < df[s].nblk; ++b) {
                            blk_sorted.push_back(s);
                            blk_sorted.push_back(b);
                        }
                        if (df[s].pinv) pf.push_back(s);
                    }
                    bool blk_done = false;
                    for (int c = 0; c < 3; ++c) {
                        ProgLaunch il_{};
                        il_.kind = L_DFINV;
                        il_.level = L;
                        il_.side = 1;
                        il_.cls = 8 << c;
                        il_.list = (int64_t)small_sorted.size();
                        il_.list2 = blk0;
                        il_.count = to_i32((int64_t)by_w[c].size(), "inverse launch");
                        il_.count2 = blk_done ? 0 : to_i32((int64_t)blk_sorted.size() / 2 - blk0, "inverse launch");
                        small_sorted.insert(small_sorted.end(), by_w[c].begin(), by_w[c].end());
                        if (il_.count + il_.count2 > 0) {
                            side_b.push_back(il_);
                            blk_done = true;
                        }
                    }
                    // one launch of tiles; a tile with a long inner dimension becomes nsplit CTAs
                    auto push_launch = [&](std::vector<PinvTile>& v, int cls) {
                        ProgLaunch pl{};
                        pl.kind = L_PINV;
                        pl.level = L;
                        pl.side = 1;
                        pl.cls = cls;
                        pl.list = (int64_t)pt.size();
                        int32_t slots = 0, cnts = 0;
                        for (const PinvTile& t0 : v) {
                            pl.flops += 2.0 * t0.m * t0.n * t0.k;
                            const int ns_ = (t0.k + PINV_KSPLIT - 1) / PINV_KSPLIT;
                            if (ns_ <= 1) {
                                PinvTile t = t0;
                                t.nsplit = 1;
                                pt.push_back(t);
                                continue;
                            }
                            for (int sp = 0; sp < ns_; ++sp) {
                                PinvTile t = t0;
                                const int k0 = sp * PINV_KSPLIT;
                                t.a += (int64_t)k0 * t0.lda;
                                t.b += k0;
                                t.k = std::min(PINV_KSPLIT, t0.k - k0);
                                t.nsplit = ns_;
                                t.split = sp;
                                t.slot = slots;
                                t.cnt = cnts;
                                pt.push_back(t);
                            }
                            slots += ns_;
                            cnts += 1;
                        }
                        P->psplit_slots = std::max(P->psplit_slots, (int64_t)slots);
                        P->psplit_cnts = std::max(P->psplit_cnts, (int64_t)cnts);
                        pl.count = to_i32((int64_t)(pt.size() - pl.list), "inverse-panel tiles");
                        if (pl.count > 0) side_b.push_back(pl);
                        v.clear();
                    };
                    int maxK = 0;
                    for (int s : pf) maxK = std::max(maxK, df[s].nblk);
                    for (int h = 1; h < maxK; h *= 2) {
                        std::vector<PinvTile> g1, g2;
                        int64_t toff = 0;
                        for (int s : pf) {
                            const DFront& F = P->fronts[s];
                            const int K = df[s].nblk, f = F.f, w = F.w;
                            const int64_t po = inv_off[s], pa = F.panel;
                            for (int a0 = 0; a0 + h < K; a0 += 2 * h) {
                                const int c0 = a0 + h, c1 = std::min(a0 + 2 * h, K);
                                const int rowsC = std::min(w, DF_BLK * c1) - DF_BLK * c0;
                                for (int ci = c0; ci < c1; ++ci)
                                    for (int aj = a0; aj < c0; ++aj) {
                                        PinvTile t1{};
                                        t1.a = pa + DF_BLK * ci + (int64_t)DF_BLK * aj * f;
                                        t1.lda = f;
                                        t1.b = po + DF_BLK * aj + (int64_t)DF_BLK * aj * f;
                                        t1.ldb = f;
                                        t1.c = toff + DF_BLK * (ci - c0) + (int64_t)DF_BLK * (aj - a0) * rowsC;
                                        t1.ldc = rowsC;
                                        t1.m = bw_of(w, ci);
                                        t1.n = DF_BLK;
                                        t1.k = DF_BLK * (c0 - aj);
                                        t1.front = (int32_t)s;
                                        g1.push_back(t1);
                                        PinvTile t2{};
                                        t2.a = po + DF_BLK * ci + (int64_t)DF_BLK * c0 * f;
                                        t2.lda = f;
                                        t2.b = toff + (int64_t)DF_BLK * (aj - a0) * rowsC;
                                        t2.ldb = rowsC;
                                        t2.c = po + DF_BLK * ci + (int64_t)DF_BLK * aj * f;
                                        t2.ldc = f;
                                        t2.m = bw_of(w, ci);
                                        t2.n = DF_BLK;
                                        t2.k = DF_BLK * (ci - c0) + bw_of(w, ci);
                                        t2.front = (int32_t)s;
                                        t2.neg = 1;
                                        g2.push_back(t2);
                                    }
                                toff += (int64_t)rowsC * DF_BLK * h;
                            }
                        }
                        pwork = std::max(pwork, toff);
                        push_launch(g1, 1);
                        push_launch(g2, 2);
                    }
                    std::vector<PinvTile> gw;
                    for (int s : pf) {
                        const DFront& F = P->fronts[s];
                        const int K = df[s].nblk, f = F.f, w = F.w, m = f - w;
                        const int64_t po = inv_off[s], pa = F.panel;
                        for (int r0 = 0; r0 < m; r0 += DF_BLK)
                            for (int aj = 0; aj < K; ++aj) {
                                PinvTile t{};
                                t.a = pa + w + r0 + (int64_t)DF_BLK * aj * f;
                                t.lda = f;
                                t.b = po + DF_BLK * aj + (int64_t)DF_BLK * aj * f;
                                t.ldb = f;
                                t.c = po + w + r0 + (int64_t)DF_BLK * aj * f;
                                t.ldc = f;
                                t.m = std::min(DF_BLK, m - r0);
                                t.n = bw_of(w, aj);
                                t.k = w - DF_BLK * aj;
                                t.front = (int32_t)s;
                                gw.push_back(t);
                            }
                    }
                    push_launch(gw, 3);
                }
                P->d_df_small = upload(P, small_sorted, st);
                P->d_df_blkinv = upload(P, blk_sorted, st);
                P->pwork_len = pinv_mode ? std::max<int64_t>(pwork, 2) : 0;
                P->d_pinv_tiles = upload(P, pt, st);
                // every batch's side launches right after the batch's last launch of the factorization
                std::vector<ProgLaunch> merged;
                for (size_t q = 0; q < P->prog.size(); ++q) {
                    merged.push_back(P->prog[q]);
                    const std::pair<int, int> key{P->prog[q].level, P->prog[q].fstream};
                    const bool last_of_batch = q + 1 == P->prog.size() || P->prog[q + 1].level != key.first ||
                                               P->prog[q + 1].fstream != key.second;
                    auto it = side.find(key);
                    if (last_of_batch && it != side.end()) {
                        merged.insert(merged.end(), it->second.begin(), it->second.end());
                        side.erase(it);
                    }
                }
                for (auto& kv : side) merged.insert(merged.end(), kv.second.begin(), kv.second.end());
                P->prog.swap(merged);
            } else {
                // uniform batches: launches after the factorization build every member's warp-front
                // L11^-1 (one launch per width class 8, 16, 32) and 64 x 64 diagonal-block inverses
                // (the tiled fronts run as block chains)
                std::vector<int32_t> small_all, blk_all;
                std::vector<int32_t> by_w[3];
                for (int L = 0; L < P->nlevels; ++L)
                    for (int s : P->level_fronts[L]) {
                        if (!df[s].tiled) {
                            const int w = P->fronts[s].w;
                            by_w[w <= 8 ? 0 : w <= 16 ? 1 : 2].push_back(s);
                            continue;
                        }
                        for (int b = 0; b < df[s].nblk; ++b) {
                            blk_all.push_back(s);
                            blk_all.push_back(b);
                        }
                    }
                const int wcls[3] = {8, 16, 32};
                std::vector<ProgLaunch> inv_l;
                for (int c = 0; c < 3; ++c) {
                    ProgLaunch il_{};
                    il_.kind = L_DFINV;
                    il_.level = P->nlevels;
                    il_.cls = wcls[c];
                    il_.list = (int64_t)small_all.size();
                    il_.list2 = 0;
                    il_.count = to_i32((int64_t)by_w[c].size(), "inverse launch");
                    il_.count2 = inv_l.empty() ? to_i32((int64_t)blk_all.size() / 2, "inverse launch") : 0;
                    small_all.insert(small_all.end(), by_w[c].begin(), by_w[c].end());
                    if (il_.count + il_.count2 > 0) inv_l.push_back(il_);
                }
                if (inv_l.empty() && !blk_all.empty()) {
                    ProgLaunch il_{};
                    il_.kind = L_DFINV;
                    il_.level = P->nlevels;
                    il_.count2 = to_i32((int64_t)blk_all.size() / 2, "inverse launch");
                    inv_l.push_back(il_);
                }
                P->d_df_small = upload(P, small_all, st);
                P->d_df_blkinv = upload(P, blk_all, st);
                P->prog.insert(P->prog.end(), inv_l.begin(), inv_l.end());
            }
        }
        {
            ProgLaunch pl{};
            pl.kind = L_STATS;
            P->prog.push_back(pl);
        }
        P->launches_factor = (int)P->prog.size();

        // solve: update vectors, per-level lists
        std::vector<int64_t> uoff(ns, -1);
        int64_t uo = 0;
        for (int64_t s = 0; s < ns; ++s) {
            int64_t m = P->fronts[s].f - P->fronts[s].w;
            if (m > 0) {
                uoff[s] = uo;
                uo += (m * P->max_nrhs + 3) & ~int64_t(3);
            }
        }
        P->ulen = std::max<int64_t>(uo, 1);
        std::vector<int32_t> level_lists, rect_tiles;
        P->level_maxw.assign(P->nlevels, 0);
        P->level_panel_entries.assign(P->nlevels, 0.0);
        P->level_nsmall.assign(P->nlevels, 0);
        P->level_nlarge.assign(P->nlevels, 0);
        P->level_maxw_small.assign(P->nlevels, 1);
        P->level_maxw_large.assign(P->nlevels, 1);
        P->level_nftile.assign(P->nlevels, 0);
        P->level_nbtile.assign(P->nlevels, 0);
        auto solve_large = [&](const DFront& F) { return (int64_t)(F.f - F.w) * F.w >= 16384; };
        for (int L = 0; L < P->nlevels; ++L) {
            P->level_list_off.push_back((int64_t)level_lists.size());
            for (int pass = 0; pass < 2; ++pass)
                for (int s : P->level_fronts[L]) {
                    const DFront& F = P->fronts[s];
                    if (solve_large(F) != (pass == 1)) continue;
                    level_lists.push_back(s);
                    if (pass == 0) {
                        P->level_nsmall[L]++;
                        P->level_maxw_small[L] = std::max(P->level_maxw_small[L], F.w);
                    } else {
                        P->level_nlarge[L]++;
                        P->level_maxw_large[L] = std::max(P->level_maxw_large[L], F.w);
                    }
                    P->level_maxw[L] = std::max(P->level_maxw[L], F.w);
                    P->level_panel_entries[L] += (double)F.f * F.w - 0.5 * (double)F.w * (F.w - 1);
                }
            P->level_ftile_off.push_back((int64_t)rect_tiles.size() / 2);
            for (int s : P->level_fronts[L]) {
                const DFront& F = P->fronts[s];
                if (!solve_large(F)) continue;
                for (int r0 = 0; r0 < F.f - F.w; r0 += RECT_ROWS_PLAN) {
                    rect_tiles.push_back(s);
                    rect_tiles.push_back(r0);
                    P->level_nftile[L]++;
                }
            }
            P->level_btile_off.push_back((int64_t)rect_tiles.size() / 2);
            for (int s : P->level_fronts[L]) {
                const DFront& F = P->fronts[s];
                if (!solve_large(F)) continue;
                for (int c0 = 0; c0 < F.w; c0 += RECT_COLS_PLAN) {
                    rect_tiles.push_back(s);
                    rect_tiles.push_back(c0);
                    P->level_nbtile[L]++;
                }
            }
        }

        // host maps kept for the outputs
        P->h_perm0.resize(n);
        for (int64_t k = 0; k < n; ++k) {
            if (perm[k] < 1 || perm[k] > n) throw BuildError(SDSB200_INVALID_VALUE, "perm out of range");
            P->h_perm0[k] = (int32_t)(perm[k] - 1);
        }
        P->h_super0.resize(ns);
        for (int64_t s = 0; s < ns; ++s) P->h_super0[s] = (int32_t)(super_ptr[s] - 1);
        std::vector<int32_t> rv0(rowval.size()), cl0(child_list.size()), ri0(relind.size());
        for (size_t k = 0; k < rowval.size(); ++k) rv0[k] = (int32_t)(rowval[k] - 1);
        for (size_t k = 0; k < child_list.size(); ++k) cl0[k] = (int32_t)(child_list[k] - 1);
        for (size_t k = 0; k < relind.size(); ++k) ri0[k] = (int32_t)(relind[k] - 1);

        // residual map (and its transpose for op(A) = A^T of "G")
        if (sym->full_rowptr && sym->full_colval && sym->full_srcptr && sym->full_src) {
            P->has_full = true;
            P->full_nnz = sym->full_nnz;
            P->full_nsrc = sym->full_nsrc;
            std::vector<int64_t> frp = read_map(sym->full_rowptr, n + 1, width, "full_rowptr");
            std::vector<int64_t> fcv = read_map(sym->full_colval, P->full_nnz, width, "full_colval");
            std::vector<int64_t> fsp = read_map(sym->full_srcptr, P->full_nnz + 1, width, "full_srcptr");
            std::vector<int64_t> fsr = read_map(sym->full_src, P->full_nsrc, width, "full_src");
            for (auto& v : frp) v -= 1;
            for (auto& v : fcv) v -= 1;
            for (auto& v : fsp) v -= 1;
            for (auto& v : fsr) v -= 1;
            P->d_full_rowptr = upload(P, frp, st);
            P->d_full_colval = upload(P, fcv, st);
            P->d_full_srcptr = upload(P, fsp, st);
            P->d_full_src = upload(P, fsr, st);
            if (gen) {
                // transpose: entries regrouped by column, each keeping its source list
                std::vector<int64_t> cnt(n + 1, 0);
                for (int64_t e = 0; e < P->full_nnz; ++e) cnt[fcv[e] + 1]++;
                std::vector<int64_t> trp(n + 1, 0);
                for (int64_t i = 0; i < n; ++i) trp[i + 1] = trp[i] + cnt[i + 1];
                std::vector<int64_t> tcv(P->full_nnz), tsp(P->full_nnz + 1), tsr;
                std::vector<int64_t> next(trp.begin(), trp.end() - 1);
                std::vector<int64_t> epos(P->full_nnz);
                for (int64_t r = 0; r < n; ++r)
                    for (int64_t e = frp[r]; e < frp[r + 1]; ++e) {
                        int64_t q = next[fcv[e]]++;
                        tcv[q] = r;
                        epos[q] = e;
                    }
                tsp[0] = 0;
                for (int64_t q = 0; q < P->full_nnz; ++q) {
                    int64_t e = epos[q];
                    for (int64_t k = fsp[e]; k < fsp[e + 1]; ++k) tsr.push_back(fsr[k]);
                    tsp[q + 1] = (int64_t)tsr.size();
                }
                P->d_fullT_rowptr = upload(P, trp, st);
                P->d_fullT_colval = upload(P, tcv, st);
                P->d_fullT_srcptr = upload(P, tsp, st);
                P->d_fullT_src = upload(P, tsr, st);
            }
        }

        // device copies
        P->d_fronts = upload(P, P->fronts, st);
        P->maps.fronts = P->d_fronts;
        P->maps.child_list = upload(P, cl0, st);
        P->maps.relind = upload(P, ri0, st);
        P->maps.am_src = upload(P, am_src, st);
        P->maps.am_loc = upload(P, am_loc, st);
        P->maps.amcol = upload(P, amcol, st);
        // cooperative pivot launches (single-member plans): a group of co-resident CTAs per wide front,
        // sized by the front's update work f w^2, at least one CTA and at most the update items of its
        // first step (row chunks x column groups; twice that for the U^T part of "G")
        std::vector<int32_t> coop_first;
        if (P->nbatch == 1) {
            const int cap = P->elsize == 8 ? large_pivot_coop_capacity<double>(P->structure)
                                           : large_pivot_coop_capacity<float>(P->structure);
            for (ProgLaunch& L : P->prog) {
                if (L.kind != L_PIVOT_FRONT || L.count <= 0 || 2 * L.count > cap) continue;
                double total = 0;
                for (int i = 0; i < L.count; ++i) {
                    const DFront& F = P->fronts[lists[L.list + i]];
                    total += (double)F.f * F.w * F.w;
                }
                L.coop = (int32_t)coop_first.size();
                int first = 0;
                for (int i = 0; i < L.count; ++i) {
                    const DFront& F = P->fronts[lists[L.list + i]];
                    const double share = total > 0 ? (double)cap * ((double)F.f * F.w * F.w) / total : 1.0;
                    const int64_t items = (int64_t)((F.f + COOP_ROWS - 1) / COOP_ROWS) *
                                          ((F.w + COOP_COLS - 1) / COOP_COLS) * (gen ? 2 : 1);
                    const int64_t most = std::max<int64_t>(1, items);
                    const int g = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)share, most));
                    coop_first.push_back(first);
                    first += g;
                }
                coop_first.push_back(first);
                L.coop_grid = first;
                P->coop_bar_len = std::max(P->coop_bar_len, L.count);
            }
        }
        P->d_coop_first = upload(P, coop_first, st);
        if (P->coop_bar_len) P->d_coop_bar = dalloc<unsigned int>(P, P->coop_bar_len);
        P->maps.ea = upload(P, ea, st);
        P->maps.eacol = upload(P, eacol, st);
        P->maps.rchunk = upload(P, rchunk, st);
        P->maps.rowval = upload(P, rv0, st);
        P->d_perm0 = upload(P, P->h_perm0, st);
        P->maps.perm = P->d_perm0;
        P->d_super0 = upload(P, P->h_super0, st);
        P->d_lists = upload(P, lists, st);
        P->d_coltasks = upload(P, coltasks, st);
        P->d_steptasks = upload(P, steptasks, st);
        P->d_tiles = upload(P, tiles, st);
        P->d_scr_off = upload(P, scr_off, st);
        P->d_woff = upload(P, woff, st);
        P->d_uoff = upload(P, uoff, st);
        P->d_level_lists = upload(P, level_lists, st);
        P->d_rect_tiles = upload(P, rect_tiles, st);

        const int64_t nb = P->nbatch;
        const size_t es = P->elsize;
        auto alloc_bytes = [&](size_t bytes) -> void* {
            return (void*)dalloc<unsigned char>(P, bytes);
        };
        P->d_factor = alloc_bytes(es * std::max<int64_t>(P->factor_len, 1) * nb);
        if (gen) P->d_ufactor = alloc_bytes(es * std::max<int64_t>(P->factor_len, 1) * nb);
        P->d_cb = alloc_bytes(es * std::max<int64_t>(P->cb_len, 1) * nb);
        P->d_d = dalloc<double>(P, 2 * n * nb);
        P->d_piv = dalloc<int32_t>(P, n * nb);
        P->d_kind = dalloc<int8_t>(P, n * nb);
        P->d_stats = dalloc<int64_t>(P, NSTAT * ns * nb);
        P->d_finfo = dalloc<int32_t>(P, ns * nb);
        P->d_totals = dalloc<int64_t>(P, NSTAT * nb);
        P->d_info = dalloc<int64_t>(P, nb);
        P->d_psign = dalloc<int8_t>(P, n);
        P->d_members = dalloc<int32_t>(P, nb);
        P->d_amax = dalloc<double>(P, 1);
        if (P->scr_len) P->d_scratch = dalloc<double>(P, P->scr_len * nb);
        if (P->work_len) P->d_work = alloc_bytes(es * P->work_len * nb);
        if (P->inv_len) P->d_inv = alloc_bytes(es * P->inv_len * nb);
        P->d_dfinv_L = alloc_bytes(es * P->df_inv_len * nb);
        if (gen) P->d_dfinv_U = alloc_bytes(es * P->df_inv_len * nb);
        if (P->pwork_len) P->d_pwork = alloc_bytes(es * P->pwork_len * nb * (gen ? 2 : 1));
        if (P->flow_cnt_len) P->d_flow_cnt = dalloc<unsigned int>(P, P->flow_cnt_len);
        P->d_flow_status = dalloc<int32_t>(P, 1);
        cudaMemsetAsync(P->d_flow_status, 0, sizeof(int32_t), st);
        if (P->psplit_slots) {
            P->d_psplit = alloc_bytes(es * P->psplit_slots * 64 * 64);
            P->d_pcnt = dalloc<unsigned int>(P, P->psplit_cnts);
            cudaMemsetAsync(P->d_pcnt, 0, sizeof(unsigned int) * P->psplit_cnts, st);
        }
        P->d_xtmp = dalloc<double>(P, n * P->max_nrhs * nb);
        P->d_solve_status = dalloc<int32_t>(P, 1);
        cudaMemsetAsync(P->d_solve_status, 0, sizeof(int32_t), st);
        P->d_Y = dalloc<double>(P, n * P->max_nrhs * nb);
        P->d_U = dalloc<double>(P, P->ulen * nb);
        P->d_R = dalloc<double>(P, n * P->max_nrhs * nb);
        P->d_norms = dalloc<double>(P, 2 * P->max_nrhs * nb);
        if (cudaMallocHost(&P->h_norms, sizeof(double) * 2 * P->max_nrhs * nb) != cudaSuccess)
            throw BuildError(SDSB200_ALLOC_FAILED, "cudaMallocHost");
        // info of every member, then the step tasks' status word
        if (cudaMallocHost(&P->h_info_pinned, sizeof(int64_t) * (nb + 1)) != cudaSuccess)
            throw BuildError(SDSB200_ALLOC_FAILED, "cudaMallocHost");
        {
            int dev = 0, optin = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
            cudaError_t ke = prepare_factor_kernels(optin);
            if (ke == cudaSuccess) ke = prepare_dense_kernels(optin);
            if (ke == cudaSuccess) ke = prepare_solve_kernels(optin);
            if (ke == cudaSuccess) ke = prepare_dataflow_kernels(optin);
            if (ke == cudaSuccess) ke = prepare_tc_kernels();
            if (ke != cudaSuccess)
                throw BuildError(SDSB200_CUDA_ERROR, std::string("kernel attribute setup failed: ") + cudaGetErrorString(ke));
            if ((int64_t)small_front_smem(P->fsmall_max, P->elsize) > optin)
                throw BuildError(SDSB200_NOT_SUPPORTED, "shared memory per block too small for the front classes");
        }
        // the capture stream at the highest priority, the side stream (the solve's inverses, beside the
        // factorization) at the lowest
        int prio_low = 0, prio_high = 0;
        cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
        if (cudaStreamCreateWithPriority(&P->own, cudaStreamNonBlocking, prio_high) != cudaSuccess ||
            cudaStreamCreateWithPriority(&P->side, cudaStreamNonBlocking, prio_low) != cudaSuccess ||
            cudaEventCreateWithFlags(&P->join_in, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&P->join_out, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&P->side_fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&P->side_join, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&P->fstream_fork, cudaEventDisableTiming) != cudaSuccess)
            throw BuildError(SDSB200_CUDA_ERROR, "stream or event creation failed");
        // the factorization's extra streams and their events (the cross-stream ones, then one join per
        // extra stream)
        for (int g = 1; g < P->nfstreams; ++g) {
            cudaStream_t fs = nullptr;
            if (cudaStreamCreateWithPriority(&fs, cudaStreamNonBlocking, prio_high) != cudaSuccess)
                throw BuildError(SDSB200_CUDA_ERROR, "stream creation failed");
            P->fstreams.push_back(fs);
        }
        for (int q = 0; q < P->nfevents + P->nfstreams - 1; ++q) {
            cudaEvent_t ev = nullptr;
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
                throw BuildError(SDSB200_CUDA_ERROR, "event creation failed");
            P->fevents.push_back(ev);
        }
        cudaMemsetAsync(P->d_psign, 0, n, st);
        cudaMemsetAsync(P->d_kind, 0, n * nb, st);
        cudaMemsetAsync(P->d_d, 0, sizeof(double) * 2 * n * nb, st);
        cudaMemsetAsync(P->d_piv, 0, sizeof(int32_t) * n * nb, st);
        std::vector<int32_t> spiv;
        std::vector<int8_t> skind;
        std::vector<double> sd;
        if (P->schur_front >= 0) {
            // the Schur root's columns: identity local order, unit 1x1 pivots, d = 1 and no 2x2 part
            // (src/numeric/schur.jl:15-29); no kernel writes them, so they are set once here
            const DFront& R = P->fronts[P->schur_front];
            for (int k = 0; k < R.w; ++k) spiv.push_back(R.c0 + k + 1);
            skind.assign(R.w, (int8_t)KIND_1X1);
            sd.assign(R.w, 1.0);
            for (int64_t mb = 0; mb < nb; ++mb) {
                cudaMemcpyAsync(P->d_piv + mb * n + R.c0, spiv.data(), sizeof(int32_t) * R.w, cudaMemcpyHostToDevice, st);
                cudaMemcpyAsync(P->d_kind + mb * n + R.c0, skind.data(), R.w, cudaMemcpyHostToDevice, st);
                cudaMemcpyAsync(P->d_d + mb * 2 * n + R.c0, sd.data(), sizeof(double) * R.w, cudaMemcpyHostToDevice, st);
            }
        }
        cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) throw BuildError(SDSB200_CUDA_ERROR, cudaGetErrorString(e));
        return P;
    } catch (const BuildError& be) {
        free_plan(P);
        throw PlanError{be.code, be.what()};
    }
}

void free_plan(Plan* P) {
    if (!P) return;
    for (void* p : P->allocations) cudaFree(p);
    for (cudaEvent_t e : P->events) cudaEventDestroy(e);
    for (Plan::CachedGraph* g : {&P->g_factor, &P->g_solve, &P->g_resid, &P->g_corr})
        if (g->exec) cudaGraphExecDestroy(g->exec);
    if (P->join_in) cudaEventDestroy(P->join_in);
    if (P->join_out) cudaEventDestroy(P->join_out);
    if (P->side_fork) cudaEventDestroy(P->side_fork);
    if (P->side_join) cudaEventDestroy(P->side_join);
    if (P->own) cudaStreamDestroy(P->own);
    if (P->side) cudaStreamDestroy(P->side);
    if (P->fstream_fork) cudaEventDestroy(P->fstream_fork);
    for (cudaStream_t fs : P->fstreams) cudaStreamDestroy(fs);
    for (cudaEvent_t ev : P->fevents) cudaEventDestroy(ev);
    if (P->h_norms) cudaFreeHost(P->h_norms);
    if (P->h_info_pinned) cudaFreeHost(P->h_info_pinned);
    delete P;
}

}  // namespace sds
