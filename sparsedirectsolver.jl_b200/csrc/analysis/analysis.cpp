// Host analysis of the numeric phase: from a CSR pattern to the Symbolic maps.
//
// Restates, step by step, the reference's host analysis (SparseDirectSolver.jl,
// src/symbolic/*.jl) so that callers without Julia obtain the same maps the
// reference would hand to its numeric phase. Internally 1-based, as the
// reference, so that every index expression can be checked against it line by
// line; the orderings (AMD, nested dissection) are this file's own, the
// reference's come from third-party packages (CliqueTrees.jl 1.x, AMD.jl 0.5,
// Metis.jl 1).
#include "../../../include/sdsb200_analysis.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <tuple>
#include <numeric>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

using std::vector;
typedef int64_t i64;

namespace {

thread_local std::string g_err;

struct AnalysisError : std::runtime_error {
    explicit AnalysisError(const std::string& m) : std::runtime_error(m) {}
};

// ---------------------------------------------------------------------------
// Symmetric pattern (src/symbolic/pattern.jl:17-171): 1-based adjacency, sorted,
// unique, no diagonal, both triangles. colptr has n + 2 slots (index 0 unused).
struct Pattern {
    int n = 0;
    vector<int> colptr;  // colptr[1..n+1]
    vector<int> rowval;  // rowval[1..nnz]
    int deg(int j) const { return colptr[j + 1] - colptr[j]; }
    const int* nb_begin(int j) const { return rowval.data() + colptr[j]; }
    const int* nb_end(int j) const { return rowval.data() + colptr[j + 1]; }
};

// column-sorted, duplicate-free CSC of (I[k], J[k]) (src/symbolic/pattern.jl:180-213, `_csc_unique`)
Pattern csc_unique(int n, const vector<int>& I, const vector<int>& J) {
    vector<int> count(n + 2, 0);
    for (int j : J) count[j + 1]++;
    vector<int> colptr(n + 2, 0);
    colptr[1] = 1;
    for (int j = 1; j <= n; ++j) colptr[j + 1] = colptr[j] + count[j + 1];
    vector<int> rowval(I.size() + 1, 0);
    vector<int> next(colptr.begin(), colptr.end());
    for (size_t k = 0; k < I.size(); ++k) rowval[next[J[k]]++] = I[k];
    Pattern P;
    P.n = n;
    P.colptr.assign(n + 2, 0);
    P.colptr[1] = 1;
    P.rowval.assign(1, 0);
    for (int j = 1; j <= n; ++j) {
        std::sort(rowval.begin() + colptr[j], rowval.begin() + colptr[j + 1]);
        int prev = 0;
        for (int p = colptr[j]; p < colptr[j + 1]; ++p) {
            if (rowval[p] != prev) P.rowval.push_back(rowval[p]);
            prev = rowval[p];
        }
        P.colptr[j + 1] = (int)P.rowval.size();
    }
    return P;
}

// entry filter of the view (src/symbolic/pattern.jl:103-110)
inline bool keep_entry(int structure, int view, i64 r, i64 c) {
    if (structure == SDSA_STRUCTURE_G) return true;
    if (view == 'U') return c >= r;
    return c <= r;
}

struct Csr {
    int n;
    vector<i64> rp;  // 1-based, rp[1..n+1]
    vector<i64> cv;  // 1-based columns, cv[1..nnz]
};

Csr host_pattern(i64 n, const i64* rowptr, const i64* colval, int index_base) {
    Csr A;
    A.n = (int)n;
    i64 shift = index_base == 0 ? 1 : 0;
    A.rp.assign(n + 2, 0);
    for (i64 r = 0; r <= n; ++r) A.rp[r + 1] = rowptr[r] + shift;
    if (A.rp[1] != 1) throw AnalysisError("rowptr must start at the index base");
    i64 nnz = A.rp[n + 1] - 1;
    if (nnz < 0) throw AnalysisError("rowptr must end at nnz + base");
    for (i64 r = 1; r <= n; ++r)
        if (A.rp[r] > A.rp[r + 1]) throw AnalysisError("rowptr is not nondecreasing");
    A.cv.assign(nnz + 1, 0);
    for (i64 p = 0; p < nnz; ++p) {
        i64 c = colval[p] + shift;
        if (c < 1 || c > n) throw AnalysisError("column index out of range");
        A.cv[p + 1] = c;
    }
    return A;
}

Pattern symmetric_pattern(const Csr& A, int structure, int view) {
    vector<int> I, J;
    for (int r = 1; r <= A.n; ++r)
        for (i64 p = A.rp[r]; p < A.rp[r + 1]; ++p) {
            int c = (int)A.cv[p];
            if (!keep_entry(structure, view, r, c) || r == c) continue;
            I.push_back(r); J.push_back(c);
            I.push_back(c); J.push_back(r);
        }
    return csc_unique(A.n, I, J);
}

// ---------------------------------------------------------------------------
// Approximate minimum degree (Amestoy, Davis & Duff, SIAM J. Matrix Anal. Appl.
// 17(4), 1996): quotient graph of variables and elements, approximate external
// degrees d_i = |A_i \ i| + |L_p \ i| + sum_{e in E_i \ p} |L_e \ L_p|,
// supervariable detection by hashing, aggressive element absorption.
// 0-based; returns the elimination order (order[k] = vertex eliminated k-th).
vector<int> amd_order0(int n, const vector<vector<int>>& adj) {
    vector<vector<int>> A(adj), E(n), L(n), members(n);
    vector<int> nv(n, 1), deg(n, 0), status(n, 0);  // status 0 variable, 1 element, 2 absorbed supervariable
    vector<char> elive(n, 0);
    vector<i64> esize(n, 0), w(n, 0);
    vector<int> wflag(n, 0), mark(n, 0);
    int stamp = 0, wstamp = 0;
    // the variables by (degree, index): a binary min-heap whose entries carry the variable's version;
    // an erase bumps the version, so stale entries are skipped when they surface, and the entry taken
    // is always the least (degree, index) among the variables present, as an ordered set would give
    struct Entry { int d, i, ver; };
    auto later = [](const Entry& a, const Entry& b) { return a.d != b.d ? a.d > b.d : a.i > b.i; };
    vector<Entry> heap;
    heap.reserve(4 * (size_t)n + 16);
    vector<int> ver(n, 0);
    vector<char> present(n, 0);
    auto push = [&](int i) {
        present[i] = 1;
        heap.push_back({deg[i], i, ++ver[i]});
        std::push_heap(heap.begin(), heap.end(), later);
    };
    auto erase = [&](int i) { present[i] = 0; ++ver[i]; };
    for (int i = 0; i < n; ++i) {
        members[i].push_back(i);
        deg[i] = (int)A[i].size();
        push(i);
    }
    vector<int> order;
    order.reserve(n);
    int nelim = 0;
    vector<int> Lp, g;
    vector<std::pair<i64, int>> hashed;
    while (true) {
        while (!heap.empty() && !(present[heap.front().i] && heap.front().ver == ver[heap.front().i])) {
            std::pop_heap(heap.begin(), heap.end(), later);
            heap.pop_back();
        }
        if (heap.empty()) break;
        int p = heap.front().i;
        std::pop_heap(heap.begin(), heap.end(), later);
        heap.pop_back();
        erase(p);
        ++stamp;
        mark[p] = stamp;
        Lp.clear();
        for (int e : E[p]) {
            if (!elive[e]) continue;
            for (int v : L[e])
                if (status[v] == 0 && mark[v] != stamp) { mark[v] = stamp; Lp.push_back(v); }
            elive[e] = 0;
            vector<int>().swap(L[e]);
        }
        for (int v : A[p])
            if (status[v] == 0 && mark[v] != stamp) { mark[v] = stamp; Lp.push_back(v); }
        status[p] = 1;
        elive[p] = 1;
        for (int m : members[p]) order.push_back(m);
        nelim += nv[p];
        vector<int>().swap(A[p]);
        vector<int>().swap(E[p]);
        i64 lpw = 0;
        for (int v : Lp) { lpw += nv[v]; erase(v); }
        L[p] = Lp;
        esize[p] = lpw;
        // |L_e \ L_p| for the elements adjacent to L_p
        ++wstamp;
        for (int v : Lp)
            for (int e : E[v]) {
                if (!elive[e] || e == p) continue;
                if (wflag[e] != wstamp) { wflag[e] = wstamp; w[e] = esize[e]; }
                w[e] -= nv[v];
            }
        // prune the lists and update the degrees
        for (int i : Lp) {
            vector<int>& Ei = E[i];
            size_t q = 0;
            i64 d = 0;
            for (int e : Ei) {
                if (!elive[e] || e == p) continue;
                i64 we = (wflag[e] == wstamp) ? w[e] : esize[e];
                if (we <= 0) { elive[e] = 0; continue; }  // aggressive absorption: L_e inside L_p
                d += we;
                Ei[q++] = e;
            }
            Ei.resize(q);
            Ei.push_back(p);
            vector<int>& Ai = A[i];
            q = 0;
            for (int v : Ai) {
                if (status[v] != 0 || mark[v] == stamp) continue;
                d += nv[v];
                Ai[q++] = v;
            }
            Ai.resize(q);
            d += lpw - nv[i];
            i64 bound = (i64)n - nelim - nv[i];
            i64 d2 = (i64)deg[i] + lpw - nv[i];
            d = std::min(d, d2);
            d = std::min(d, bound);
            deg[i] = (int)std::max<i64>(d, 0);
        }
        // supervariables: identical element and variable lists
        if (Lp.size() > 1) {
            // hash groups (each in Lp order; the groups are disjoint, so their order is immaterial)
            hashed.clear();
            for (int i : Lp) {
                i64 h = 0;
                for (int e : E[i]) h += e;
                for (int v : A[i]) h += v;
                hashed.push_back({h, i});
            }
            std::stable_sort(hashed.begin(), hashed.end(),
                             [](const std::pair<i64, int>& a, const std::pair<i64, int>& b) { return a.first < b.first; });
            for (size_t g0 = 0; g0 < hashed.size();) {
                size_t g1 = g0 + 1;
                while (g1 < hashed.size() && hashed[g1].first == hashed[g0].first) ++g1;
                g.clear();
                for (size_t t = g0; t < g1; ++t) g.push_back(hashed[t].second);
                g0 = g1;
                if (g.size() < 2) continue;
                for (size_t a = 0; a < g.size(); ++a) {
                    int i = g[a];
                    if (status[i] != 0) continue;
                    vector<int> Ei(E[i]), Ai(A[i]);
                    std::sort(Ei.begin(), Ei.end());
                    std::sort(Ai.begin(), Ai.end());
                    for (size_t b = a + 1; b < g.size(); ++b) {
                        int j = g[b];
                        if (status[j] != 0 || E[j].size() != Ei.size() || A[j].size() != Ai.size()) continue;
                        vector<int> Ej(E[j]), Aj(A[j]);
                        std::sort(Ej.begin(), Ej.end());
                        std::sort(Aj.begin(), Aj.end());
                        if (Ej != Ei || Aj != Ai) continue;
                        nv[i] += nv[j];
                        deg[i] = std::max(0, deg[i] - nv[j]);
                        nv[j] = 0;
                        status[j] = 2;
                        members[i].insert(members[i].end(), members[j].begin(), members[j].end());
                        vector<int>().swap(members[j]);
                        vector<int>().swap(A[j]);
                        vector<int>().swap(E[j]);
                    }
                }
            }
        }
        for (int i : Lp)
            if (status[i] == 0) push(i);
    }
    return order;
}

vector<vector<int>> adjacency0(const Pattern& P) {
    vector<vector<int>> adj(P.n);
    for (int j = 1; j <= P.n; ++j)
        for (const int* q = P.nb_begin(j); q != P.nb_end(j); ++q) adj[j - 1].push_back(*q - 1);
    return adj;
}

// 1-based perm (perm[k] = original column eliminated k-th), perm[0] unused
vector<int> amd_perm(const Pattern& P) {
    vector<int> o = amd_order0(P.n, adjacency0(P));
    vector<int> perm(P.n + 1, 0);
    for (int k = 0; k < P.n; ++k) perm[k + 1] = o[k] + 1;
    return perm;
}

// Nested dissection by breadth-first level structures (George & Liu, "Computer
// Solution of Large Sparse Positive Definite Systems", 1981, ch. 8): from a
// pseudo-peripheral vertex, the level with the fewest vertices among the
// balanced middle levels is a vertex separator (edges only join adjacent
// levels); both sides are dissected recursively and ordered before it. Parts
// of at most `leaf` vertices are ordered by AMD.
struct NestedDissection {
    const vector<vector<int>>& adj;
    vector<int> where, level, order;
    int stamp = 0;
    int leaf;
    NestedDissection(const vector<vector<int>>& a, int leaf_) : adj(a), where(a.size(), 0), level(a.size(), -1), leaf(leaf_) {}

    void order_leaf(const vector<int>& vs) {
        int m = (int)vs.size();
        if (m == 0) return;
        int tag = ++stamp;
        std::unordered_map<int, int> loc;
        loc.reserve(m * 2);
        for (int k = 0; k < m; ++k) { where[vs[k]] = tag; loc[vs[k]] = k; }
        vector<vector<int>> sub(m);
        for (int k = 0; k < m; ++k)
            for (int u : adj[vs[k]])
                if (where[u] == tag) sub[k].push_back(loc[u]);
        vector<int> o = amd_order0(m, sub);
        for (int k : o) order.push_back(vs[k]);
    }

    // BFS inside the vertices tagged `tag`; returns the levels
    vector<vector<int>> bfs(int start, int tag) {
        vector<vector<int>> lv;
        vector<int> cur{start}, nxt;
        int vstamp = ++stamp;
        level[start] = vstamp;
        while (!cur.empty()) {
            lv.push_back(cur);
            nxt.clear();
            for (int v : cur)
                for (int u : adj[v])
                    if (where[u] == tag && level[u] != vstamp) { level[u] = vstamp; nxt.push_back(u); }
            std::swap(cur, nxt);
        }
        return lv;
    }

    void dissect(vector<int> vs) {
        if ((int)vs.size() <= leaf) { order_leaf(vs); return; }
        int tag = ++stamp;
        for (int v : vs) where[v] = tag;
        // connected components
        vector<vector<int>> comps;
        {
            int cstamp = ++stamp;
            vector<int> seen_stamp;
            for (int v : vs) {
                if (level[v] == cstamp) continue;
                vector<int> comp{v};
                level[v] = cstamp;
                for (size_t h = 0; h < comp.size(); ++h)
                    for (int u : adj[comp[h]])
                        if (where[u] == tag && level[u] != cstamp) { level[u] = cstamp; comp.push_back(u); }
                comps.push_back(std::move(comp));
            }
        }
        if (comps.size() > 1) {
            for (auto& c : comps) dissect(std::move(c));
            return;
        }
        // pseudo-peripheral start vertex
        int start = vs[0];
        for (int v : vs)
            if (adj[v].size() < adj[start].size()) start = v;
        vector<vector<int>> lv = bfs(start, tag);
        for (int it = 0; it < 4; ++it) {
            const vector<int>& last = lv.back();
            int cand = last[0];
            for (int v : last)
                if (adj[v].size() < adj[cand].size()) cand = v;
            for (int v : vs) where[v] = tag;
            vector<vector<int>> lv2 = bfs(cand, tag);
            if (lv2.size() <= lv.size()) break;
            lv.swap(lv2);
            start = cand;
        }
        int nl = (int)lv.size();
        int total = (int)vs.size();
        if (nl < 3) { order_leaf(vs); return; }
        // the smallest level whose both sides hold at least 30% of the vertices
        vector<int> before(nl + 1, 0);
        for (int k = 0; k < nl; ++k) before[k + 1] = before[k] + (int)lv[k].size();
        int best = -1;
        for (int k = 1; k < nl - 1; ++k) {
            int a = before[k], b = total - before[k + 1];
            if (a < 0.3 * total || b < 0.3 * total) continue;
            if (best < 0 || lv[k].size() < lv[best].size()) best = k;
        }
        if (best < 0) {  // most balanced split
            int bd = total + 1;
            for (int k = 1; k < nl - 1; ++k) {
                int d = std::abs(before[k] - (total - before[k + 1]));
                if (d < bd) { bd = d; best = k; }
            }
        }
        vector<int> left, right, sep(lv[best]);
        for (int k = 0; k < best; ++k) left.insert(left.end(), lv[k].begin(), lv[k].end());
        for (int k = best + 1; k < nl; ++k) right.insert(right.end(), lv[k].begin(), lv[k].end());
        std::sort(sep.begin(), sep.end());
        dissect(std::move(left));
        dissect(std::move(right));
        for (int v : sep) order.push_back(v);
    }
};

vector<int> nd_perm(const Pattern& P) {
    vector<vector<int>> adj = adjacency0(P);
    NestedDissection nd(adj, 64);
    vector<int> all(P.n);
    std::iota(all.begin(), all.end(), 0);
    nd.dissect(all);
    vector<int> perm(P.n + 1, 0);
    for (int k = 0; k < P.n; ++k) perm[k + 1] = nd.order[k] + 1;
    return perm;
}

vector<int> invperm(const vector<int>& perm) {
    vector<int> ip(perm.size(), 0);
    for (size_t k = 1; k < perm.size(); ++k) ip[perm[k]] = (int)k;
    return ip;
}

// ---------------------------------------------------------------------------
// Elimination tree, postorder, column counts (src/symbolic/etree.jl:14-178)
vector<int> etree(const Pattern& P, const vector<int>& perm) {
    int n = P.n;
    vector<int> ip = invperm(perm), parent(n + 1, 0), ancestor(n + 1, 0);
    for (int k = 1; k <= n; ++k)
        for (const int* q = P.nb_begin(perm[k]); q != P.nb_end(perm[k]); ++q) {
            int i = ip[*q];
            if (i >= k) continue;
            while (i != 0 && i < k) {
                int inext = ancestor[i];
                ancestor[i] = k;
                if (inext == 0) parent[i] = k;
                i = inext;
            }
        }
    return parent;
}

vector<int> postorder(const vector<int>& parent) {
    int n = (int)parent.size() - 1;
    vector<int> head(n + 1, 0), next(n + 1, 0), post(n + 1, 0), stack;
    for (int j = n; j >= 1; --j) {
        int p = parent[j];
        if (p == 0) continue;
        next[j] = head[p];
        head[p] = j;
    }
    int k = 0;
    for (int root = 1; root <= n; ++root) {
        if (parent[root] != 0) continue;
        stack.push_back(root);
        while (!stack.empty()) {
            int p = stack.back();
            int c = head[p];
            if (c == 0) {
                stack.pop_back();
                post[++k] = p;
            } else {
                head[p] = next[c];
                stack.push_back(c);
            }
        }
    }
    if (k != n) throw AnalysisError("parent does not describe a forest");
    return post;
}

vector<int> colcounts(const Pattern& P, const vector<int>& perm, const vector<int>& parent, const vector<int>& post) {
    int n = P.n;
    vector<int> ip = invperm(perm);
    vector<int> delta(n + 1, 0), first(n + 1, 0), maxfirst(n + 1, 0), prevleaf(n + 1, 0), ancestor(n + 1);
    for (int i = 0; i <= n; ++i) ancestor[i] = i;
    for (int k = 1; k <= n; ++k) {
        int j = post[k];
        delta[j] = first[j] == 0 ? 1 : 0;
        while (j != 0 && first[j] == 0) {
            first[j] = k;
            j = parent[j];
        }
    }
    for (int k = 1; k <= n; ++k) {
        int j = post[k];
        if (parent[j] != 0) delta[parent[j]] -= 1;
        for (const int* q = P.nb_begin(perm[j]); q != P.nb_end(perm[j]); ++q) {
            int i = ip[*q];
            // Gilbert-Ng-Peyton leaf test (etree.jl:80-97)
            if (i <= j || first[j] <= maxfirst[i]) continue;
            maxfirst[i] = first[j];
            int jprev = prevleaf[i];
            prevleaf[i] = j;
            if (jprev == 0) { delta[j] += 1; continue; }
            int qq = jprev;
            while (qq != ancestor[qq]) qq = ancestor[qq];
            int s = jprev;
            while (s != qq) {
                int sp = ancestor[s];
                ancestor[s] = qq;
                s = sp;
            }
            delta[j] += 1;
            delta[qq] -= 1;
        }
        if (parent[j] != 0) ancestor[j] = parent[j];
    }
    vector<int> counts(delta);
    for (int k = 1; k <= n; ++k) {
        int j = post[k];
        if (parent[j] != 0) counts[parent[j]] += counts[j];
    }
    return counts;
}

int tree_height(const vector<int>& parent) {
    int n = (int)parent.size() - 1;
    if (n == 0) return 0;
    vector<int> h(n + 1, 1);
    vector<int> post = postorder(parent);
    int mx = 0;
    for (int k = 1; k <= n; ++k) {
        int j = post[k];
        if (parent[j] != 0) h[parent[j]] = std::max(h[parent[j]], h[j] + 1);
    }
    for (int j = 1; j <= n; ++j) mx = std::max(mx, h[j]);
    return mx;
}

// ---------------------------------------------------------------------------
// Supernodes (src/symbolic/supernodes.jl:204-383)
struct ColumnPartition {
    vector<int> order;      // order[1..n]
    vector<int> super_ptr;  // super_ptr[1..ns+1]
    vector<int> snparent;   // snparent[1..ns]
    int ns() const { return (int)super_ptr.size() - 2; }
};

inline i64 trapezoid(i64 w, i64 f) { return w * f - (w * (w - 1)) / 2; }

vector<int> col2sn_of(const vector<int>& super_ptr) {
    int ns = (int)super_ptr.size() - 2;
    vector<int> c(super_ptr[ns + 1], 0);
    for (int s = 1; s <= ns; ++s)
        for (int j = super_ptr[s]; j < super_ptr[s + 1]; ++j) c[j] = s;
    return c;
}

vector<int> relabel_parent(const vector<int>& parent, const vector<int>& order) {
    vector<int> inv = invperm(order);
    int n = (int)order.size() - 1;
    vector<int> par(n + 1, 0);
    for (int k = 1; k <= n; ++k) {
        int j = order[k];
        par[k] = parent[j] == 0 ? 0 : inv[parent[j]];
    }
    return par;
}

ColumnPartition fundamental_supernodes(const vector<int>& parent, const vector<int>& post, const vector<int>& counts) {
    int n = (int)parent.size() - 1;
    vector<int> par = relabel_parent(parent, post);
    vector<int> cnt(n + 1, 0), nchild(n + 1, 0);
    for (int k = 1; k <= n; ++k) cnt[k] = counts[post[k]];
    for (int k = 1; k <= n; ++k)
        if (par[k] != 0) nchild[par[k]]++;
    ColumnPartition cp;
    cp.super_ptr = {0, 1};
    for (int k = 2; k <= n; ++k) {
        bool joins = par[k - 1] == k && nchild[k] == 1 && cnt[k - 1] == cnt[k] + 1;
        if (!joins) cp.super_ptr.push_back(k);
    }
    if (n > 0) cp.super_ptr.push_back(n + 1);
    else cp.super_ptr = {0, 1};
    vector<int> c2s = col2sn_of(cp.super_ptr);
    int ns = cp.ns();
    cp.snparent.assign(ns + 1, 0);
    for (int s = 1; s <= ns; ++s) {
        int last = cp.super_ptr[s + 1] - 1;
        cp.snparent[s] = par[last] == 0 ? 0 : c2s[par[last]];
    }
    cp.order = post;
    return cp;
}

ColumnPartition amalgamate(const ColumnPartition& sn, const vector<int>& parent, const vector<int>& counts,
                           int max_width, double zero_fraction, int min_width) {
    int n = (int)sn.order.size() - 1;
    vector<int> cnt(n + 1, 0);
    for (int k = 1; k <= n; ++k) cnt[k] = counts[sn.order[k]];
    vector<int> uptr = {0, 1};
    for (int s = 1; s <= sn.ns(); ++s) {
        int first = sn.super_ptr[s], last = sn.super_ptr[s + 1] - 1;
        for (int j = first; j <= last; ++j)
            if (cnt[j] != cnt[first] - (j - first)) throw AnalysisError("amalgamate needs exact supernodes");
        uptr.push_back(last + 1);
    }
    int nu = (int)uptr.size() - 2;
    vector<int> par = relabel_parent(parent, sn.order);
    vector<int> col2u = col2sn_of(uptr);
    vector<int> uparent(nu + 1, 0);
    for (int u = 1; u <= nu; ++u) {
        int last = uptr[u + 1] - 1;
        uparent[u] = par[last] == 0 ? 0 : col2u[par[last]];
    }
    vector<i64> width(nu + 1), rows(nu + 1), truennz(nu + 1), zeros_(nu + 1, 0);
    i64 total_true = 0;
    for (int u = 1; u <= nu; ++u) {
        width[u] = uptr[u + 1] - uptr[u];
        rows[u] = cnt[uptr[u]];
        truennz[u] = trapezoid(width[u], rows[u]);
        total_true += truennz[u];
    }
    i64 budget = (i64)std::floor(zero_fraction * (double)total_true);
    i64 used = 0;
    vector<int> into(nu + 1, 0);
    vector<vector<int>> children(nu + 1);
    for (int u = 1; u <= nu; ++u)
        if (uparent[u] != 0) children[uparent[u]].push_back(u);
    for (int p = 1; p <= nu; ++p) {
        vector<int>& kids = children[p];
        std::sort(kids.begin(), kids.end(), [&](int a, int b) {
            i64 ka = -(rows[a] - width[a]), kb = -(rows[b] - width[b]);
            if (ka != kb) return ka < kb;
            if (width[a] != width[b]) return width[a] < width[b];
            return a < b;
        });
        for (int c : kids) {
            i64 w = width[c] + width[p];
            if (w > max_width) continue;
            i64 added = width[c] * (width[c] + rows[p] - rows[c]);
            if (used + added > budget) continue;
            i64 z = zeros_[c] + zeros_[p] + added;
            i64 t = truennz[c] + truennz[p];
            if (!((double)z <= zero_fraction * (double)t || w <= min_width)) continue;
            into[c] = p;
            used += added;
            width[p] = w;
            rows[p] += width[c];
            zeros_[p] = z;
            truennz[p] = t;
        }
    }
    vector<int> rep(nu + 1);
    for (int u = 0; u <= nu; ++u) rep[u] = u;
    for (int u = nu; u >= 1; --u)
        if (into[u] != 0) rep[u] = rep[into[u]];
    vector<int> ids(nu + 1, 0);
    int ns = 0;
    for (int u = 1; u <= nu; ++u)
        if (into[u] == 0) ids[u] = ++ns;
    vector<int> gparent(ns + 1, 0);
    vector<vector<int>> mem(ns + 1);
    for (int u = 1; u <= nu; ++u) {
        mem[ids[rep[u]]].push_back(u);
        if (into[u] == 0 && uparent[u] != 0) gparent[ids[u]] = ids[rep[uparent[u]]];
    }
    vector<int> gpost = postorder(gparent);
    ColumnPartition out;
    vector<int> neworder = {0};
    out.super_ptr = {0, 1};
    for (int k = 1; k <= ns; ++k) {
        int g = gpost[k];
        for (int u : mem[g])
            for (int j = uptr[u]; j < uptr[u + 1]; ++j) neworder.push_back(j);
        out.super_ptr.push_back((int)neworder.size());
    }
    vector<int> gpos = invperm(gpost);
    out.snparent.assign(ns + 1, 0);
    for (int k = 1; k <= ns; ++k) {
        int g = gpost[k];
        out.snparent[k] = gparent[g] == 0 ? 0 : gpos[gparent[g]];
    }
    out.order.assign(n + 1, 0);
    for (int k = 1; k <= n; ++k) out.order[k] = sn.order[neworder[k]];
    return out;
}

struct SupernodePartition {
    int n = 0;
    vector<int> perm, iperm, parent, counts, super_ptr, col2sn, snparent, snpost, rowptr, rowval;
    i64 nnz_stored = 0, nnz_L = 0;
    double flops = 0;
    int ns() const { return (int)super_ptr.size() - 2; }
    int width(int s) const { return super_ptr[s + 1] - super_ptr[s]; }
    int nrows(int s) const { return rowptr[s + 1] - rowptr[s]; }
};

SupernodePartition supernode_partition(const Pattern& P, const vector<int>& perm, const vector<int>& parent,
                                       const vector<int>& counts, const ColumnPartition& cp) {
    SupernodePartition sp;
    int n = P.n;
    sp.n = n;
    sp.perm.assign(n + 1, 0);
    for (int k = 1; k <= n; ++k) sp.perm[k] = perm[cp.order[k]];
    sp.iperm = invperm(sp.perm);
    sp.parent = relabel_parent(parent, cp.order);
    sp.counts.assign(n + 1, 0);
    for (int k = 1; k <= n; ++k) sp.counts[k] = counts[cp.order[k]];
    int ns = cp.ns();
    sp.super_ptr = cp.super_ptr;
    sp.col2sn = col2sn_of(sp.super_ptr);
    sp.snparent = cp.snparent;
    vector<vector<int>> children(ns + 1);
    for (int s = 1; s <= ns; ++s)
        if (sp.snparent[s] != 0) children[sp.snparent[s]].push_back(s);
    sp.rowptr.assign(ns + 2, 0);
    sp.rowptr[1] = 1;
    sp.rowval.assign(1, 0);
    vector<int> mark(n + 1, 0), below;
    for (int s = 1; s <= ns; ++s) {
        int first = sp.super_ptr[s], last = sp.super_ptr[s + 1] - 1;
        below.clear();
        for (int j = first; j <= last; ++j)
            for (const int* q = P.nb_begin(sp.perm[j]); q != P.nb_end(sp.perm[j]); ++q) {
                int i = sp.iperm[*q];
                if (i > last && mark[i] != s) { mark[i] = s; below.push_back(i); }
            }
        for (int c : children[s])
            for (int p = sp.rowptr[c]; p < sp.rowptr[c + 1]; ++p) {
                int i = sp.rowval[p];
                if (i > last && mark[i] != s) { mark[i] = s; below.push_back(i); }
            }
        if ((i64)below.size() * 16 > (i64)(n - last)) {
            // dense: the marked rows in increasing order (the rows of the top fronts, where a sort
            // would cost |below| log |below| per front)
            below.clear();
            for (int i = last + 1; i <= n; ++i)
                if (mark[i] == s) below.push_back(i);
        } else {
            std::sort(below.begin(), below.end());
        }
        for (int j = first; j <= last; ++j) sp.rowval.push_back(j);
        sp.rowval.insert(sp.rowval.end(), below.begin(), below.end());
        sp.rowptr[s + 1] = (int)sp.rowval.size();
        i64 w = last - first + 1, f = w + (i64)below.size();
        sp.nnz_stored += trapezoid(w, f);
        for (i64 k = 0; k < w; ++k) sp.flops += (double)(f - k) * (double)(f - k);
    }
    sp.snpost = postorder(sp.snparent);
    for (int k = 1; k <= n; ++k) sp.nnz_L += sp.counts[k];
    return sp;
}

// ---------------------------------------------------------------------------
// 2x2 pivot pairs (src/symbolic/pairs.jl)
struct PairCandidates {
    vector<char> candidate;  // [1..n]
    vector<double> w;        // aligned with P.rowval
    vector<double> amax;     // [1..n]
};

PairCandidates pivot_candidates(const Pattern& P, const Csr& A, const double* nz, int structure, int view,
                                double tolerance) {
    int n = P.n;
    vector<double> dval(n + 1, 0.0), wval(P.rowval.size(), 0.0);
    vector<char> dpresent(n + 1, 0);
    for (int r = 1; r <= n; ++r)
        for (i64 p = A.rp[r]; p < A.rp[r + 1]; ++p) {
            int c = (int)A.cv[p];
            if (!keep_entry(structure, view, r, c)) continue;
            double v = nz[p - 1];
            if (r == c) {
                dval[r] += v;
                dpresent[r] = 1;
            } else {
                const int* b = P.nb_begin(c);
                int k1 = (int)(std::lower_bound(b, P.nb_end(c), r) - b);
                wval[P.colptr[c] + k1] += v;
                b = P.nb_begin(r);
                int k2 = (int)(std::lower_bound(b, P.nb_end(r), c) - b);
                wval[P.colptr[r] + k2] += v;
            }
        }
    PairCandidates pc;
    pc.w.resize(wval.size());
    for (size_t k = 0; k < wval.size(); ++k) pc.w[k] = std::fabs(wval[k]);
    pc.amax.assign(n + 1, 0.0);
    pc.candidate.assign(n + 1, 0);
    for (int i = 1; i <= n; ++i) {
        double m = 0.0;
        for (int p = P.colptr[i]; p < P.colptr[i + 1]; ++p) m = std::max(m, pc.w[p]);
        pc.amax[i] = m;
        pc.candidate[i] = !dpresent[i] || std::fabs(dval[i]) <= tolerance * m;
    }
    return pc;
}

typedef std::pair<int, int> IPair;  // (partner, candidate)

vector<IPair> all_pivot_pairs(const Pattern& P, const PairCandidates& cands) {
    int n = P.n;
    auto eligible = [&](int p) { return !cands.candidate[P.rowval[p]] && cands.w[p] > 0; };
    vector<std::pair<int, int>> keyed;  // (nelig, candidate)
    for (int i = 1; i <= n; ++i) {
        if (!cands.candidate[i]) continue;
        int ne = 0;
        for (int p = P.colptr[i]; p < P.colptr[i + 1]; ++p) ne += eligible(p);
        keyed.push_back({ne, i});
    }
    std::sort(keyed.begin(), keyed.end());
    vector<char> matched(n + 1, 0);
    vector<IPair> pairs;
    for (auto& kv : keyed) {
        int i = kv.second, best = 0;
        for (int p = P.colptr[i]; p < P.colptr[i + 1]; ++p) {
            int j = P.rowval[p];
            if (!eligible(p) || matched[j]) continue;
            if (best == 0 || cands.w[p] > cands.w[best] ||
                (cands.w[p] == cands.w[best] && P.deg(j) < P.deg(P.rowval[best])))
                best = p;
        }
        if (best == 0) continue;
        matched[P.rowval[best]] = 1;
        pairs.push_back({P.rowval[best], i});
    }
    std::stable_sort(pairs.begin(), pairs.end(), [](const IPair& a, const IPair& b) { return a.second < b.second; });
    return pairs;
}

vector<int> structural_zero_pivots(const PairCandidates& cands, const Pattern& P, const vector<int>& perm,
                                   const vector<IPair>& pairs) {
    // The search runs in elimination positions. Each row's edges with a nonzero value come in the
    // row's own order, with the diagonal of a non-candidate last, every column replaced by its
    // position. The depth-first order is the reference's, and so is every augmenting path and every
    // failure; a column's test is then one comparison with k and one seen mark.
    const int n = P.n;
    vector<int> pos = invperm(perm), mate(n + 1, 0);
    for (auto& ab : pairs) { mate[ab.first] = ab.second; mate[ab.second] = ab.first; }
    vector<int> aptr(n + 2, 0), adj;
    adj.reserve(P.rowval.size());
    for (int k = 1; k <= n; ++k) {
        const int r = perm[k];
        aptr[k] = (int)adj.size();
        for (int p = P.colptr[r]; p < P.colptr[r + 1]; ++p)
            if (cands.w[p] > 0) adj.push_back(pos[P.rowval[p]]);
        if (!cands.candidate[r]) adj.push_back(k);
    }
    aptr[n + 1] = (int)adj.size();
    vector<int> colm(n + 1, 0), seen(n + 1, 0), srow, sptr, scol, out;
    for (int k = 1; k <= n; ++k) {
        const int v = perm[k], m = mate[v];
        if (m != 0 && pos[m] == k - 1) { colm[k] = k - 1; colm[k - 1] = k; continue; }
        if (!cands.candidate[v] || m != 0) { colm[k] = k; continue; }
        srow.assign(1, k); sptr.assign(1, aptr[k]); scol.assign(1, 0);
        bool found = false;
        while (!srow.empty()) {
            const int r = srow.back(), q = sptr.back();
            if (q >= aptr[r + 1]) { srow.pop_back(); sptr.pop_back(); scol.pop_back(); continue; }
            sptr.back() = q + 1;
            const int j = adj[q];
            if (!(j <= k && seen[j] != k)) continue;
            seen[j] = k;
            scol.back() = j;
            if (j == k) {
                for (size_t t = 0; t < srow.size(); ++t) colm[scol[t]] = srow[t];
                found = true;
                break;
            }
            srow.push_back(colm[j]); sptr.push_back(aptr[colm[j]]); scol.push_back(0);
        }
        if (!found) { out.push_back(v); colm[k] = k; }
    }
    return out;
}

int zero_pivot_pairs(vector<IPair>& pairs, const PairCandidates& cands, const Pattern& P, const vector<int>& perm,
                     double u) {
    vector<int> zs = structural_zero_pivots(cands, P, perm, pairs);
    int n = P.n;
    vector<char> inpair(n + 1, 0);
    for (auto& ab : pairs) inpair[ab.first] = inpair[ab.second] = 1;
    vector<int> pos = invperm(perm);
    auto eligible = [&](int i, int p) {
        return !inpair[P.rowval[p]] && cands.w[p] > 0 && cands.w[p] >= u * cands.amax[i];
    };
    vector<std::tuple<int, int, int>> keyed;  // (nfree, pos, index in zs)
    for (size_t t = 0; t < zs.size(); ++t) {
        int i = zs[t], nf = 0;
        for (int p = P.colptr[i]; p < P.colptr[i + 1]; ++p) nf += eligible(i, p);
        keyed.emplace_back(nf, pos[i], (int)t);
    }
    std::sort(keyed.begin(), keyed.end());
    int added = 0;
    for (auto& kt : keyed) {
        int i = zs[std::get<2>(kt)];
        if (inpair[i]) continue;
        int best = 0;
        for (int p = P.colptr[i]; p < P.colptr[i + 1]; ++p) {
            if (!eligible(i, p)) continue;
            if (best == 0 || cands.w[p] > cands.w[best] ||
                (cands.w[p] == cands.w[best] && pos[P.rowval[p]] < pos[P.rowval[best]]))
                best = p;
        }
        if (best == 0) continue;
        int j = P.rowval[best];
        inpair[j] = inpair[i] = 1;
        pairs.push_back({j, i});
        added++;
    }
    std::stable_sort(pairs.begin(), pairs.end(), [](const IPair& a, const IPair& b) { return a.second < b.second; });
    return added;
}

void pair_groups(int n, const vector<IPair>& pairs, vector<int>& ptr, vector<int>& members) {
    vector<int> mate(n + 1, 0);
    vector<char> paired(n + 1, 0);
    for (auto& ab : pairs) {
        if (ab.first < 1 || ab.first > n || ab.second < 1 || ab.second > n || ab.first == ab.second ||
            paired[ab.first] || paired[ab.second])
            throw AnalysisError("pivot pairs must be disjoint pairs of distinct indices");
        mate[ab.first] = ab.second;
        paired[ab.first] = paired[ab.second] = 1;
    }
    ptr.assign(1, 0);
    ptr.push_back(1);
    members.assign(1, 0);
    for (int v = 1; v <= n; ++v) {
        if (mate[v] != 0) { members.push_back(v); members.push_back(mate[v]); }
        else if (!paired[v]) members.push_back(v);
        else continue;
        ptr.push_back((int)members.size());
    }
}

Pattern compressed_pattern(const Pattern& P, const vector<IPair>& pairs, vector<int>& gptr, vector<int>& members) {
    int n = P.n;
    pair_groups(n, pairs, gptr, members);
    int ng = (int)gptr.size() - 2;
    vector<int> group(n + 1, 0);
    for (int g = 1; g <= ng; ++g)
        for (int k = gptr[g]; k < gptr[g + 1]; ++k) group[members[k]] = g;
    vector<int> I, J;
    for (int j = 1; j <= n; ++j)
        for (const int* q = P.nb_begin(j); q != P.nb_end(j); ++q) {
            int gi = group[*q], gj = group[j];
            if (gi == gj) continue;
            I.push_back(gi); J.push_back(gj);
        }
    return csc_unique(ng, I, J);
}

vector<int> expand_permutation(const vector<int>& cperm, const vector<int>& gptr, const vector<int>& members) {
    vector<int> perm = {0};
    for (size_t k = 1; k < cperm.size(); ++k) {
        int g = cperm[k];
        for (int q = gptr[g]; q < gptr[g + 1]; ++q) perm.push_back(members[q]);
    }
    return perm;
}

Pattern pair_pattern(const Pattern& P, const vector<IPair>& pairs) {
    if (pairs.empty()) return P;
    vector<int> gptr, members;
    Pattern Pc = compressed_pattern(P, pairs, gptr, members);
    vector<int> I, J;
    for (int g = 1; g <= Pc.n; ++g) {
        for (int a = gptr[g]; a < gptr[g + 1]; ++a)
            for (int b = gptr[g]; b < gptr[g + 1]; ++b)
                if (a != b) { I.push_back(members[a]); J.push_back(members[b]); }
        for (const int* q = Pc.nb_begin(g); q != Pc.nb_end(g); ++q) {
            int h = *q;
            for (int a = gptr[g]; a < gptr[g + 1]; ++a)
                for (int b = gptr[h]; b < gptr[h + 1]; ++b) { I.push_back(members[b]); J.push_back(members[a]); }
        }
    }
    return csc_unique(P.n, I, J);
}

// ---------------------------------------------------------------------------
// ordering choice (src/symbolic/ordering.jl:118-317)
vector<int> ordering_perm(const Pattern& P, int alg) {
    if (alg == SDSA_REORDER_NATURAL) {
        vector<int> p(P.n + 1);
        for (int k = 0; k <= P.n; ++k) p[k] = k;
        return p;
    }
    if (alg == SDSA_REORDER_AMD) return amd_perm(P);
    if (alg == SDSA_REORDER_ND) return nd_perm(P);
    throw AnalysisError("unknown ordering algorithm");
}

struct Evaluated {
    double flops = 0, cost = 0;
    i64 nnz_L = 0;
    int sdepth = 0;
};

Evaluated evaluate_ordering(const Pattern& P, const vector<int>& perm, bool amalg, int mw, double zf, int minw) {
    vector<int> parent = etree(P, perm), post = postorder(parent), counts = colcounts(P, perm, parent, post);
    ColumnPartition cp = fundamental_supernodes(parent, post, counts);
    if (amalg) cp = amalgamate(cp, parent, counts, mw, zf, minw);
    Evaluated e;
    e.sdepth = tree_height(cp.snparent);
    for (size_t k = 1; k < counts.size(); ++k) {
        e.flops += (double)counts[k] * (double)counts[k];
        e.nnz_L += counts[k];
    }
    e.cost = e.flops + 1.0e8 * e.sdepth;
    return e;
}

struct Ordered {
    int alg;
    vector<int> perm;
    vector<IPair> pairs;
    int rounds = 0;
};

Ordered pair_ordering(const Pattern& P, int alg, const PairCandidates& cands, double u) {
    Ordered o;
    o.alg = alg;
    o.perm = ordering_perm(P, alg);
    while (o.rounds < 8) {
        int added = zero_pivot_pairs(o.pairs, cands, P, o.perm, u);
        if (added == 0) break;
        o.rounds++;
        vector<int> gptr, members;
        Pattern Pc = compressed_pattern(P, o.pairs, gptr, members);
        o.perm = expand_permutation(ordering_perm(Pc, alg), gptr, members);
    }
    return o;
}

// ---------------------------------------------------------------------------
// Schur complement mode (src/symbolic/ordering.jl:330-470, src/symbolic/supernodes.jl:380-425)

// the pattern of P restricted to `vertices` (increasing), renumbered 1..|vertices| in their order
// (induced_pattern, src/symbolic/ordering.jl:355-371)
Pattern induced_pattern(const Pattern& P, const vector<int>& vertices) {
    vector<int> loc(P.n + 1, 0);
    for (size_t k = 0; k < vertices.size(); ++k) loc[vertices[k]] = (int)k + 1;
    Pattern Q;
    Q.n = (int)vertices.size();
    Q.colptr.assign(Q.n + 2, 0);
    Q.colptr[1] = 1;
    Q.rowval.assign(1, 0);
    for (int k = 1; k <= Q.n; ++k) {
        const int v = vertices[k - 1];
        for (const int* q = P.nb_begin(v); q != P.nb_end(v); ++q)
            if (loc[*q] > 0) Q.rowval.push_back(loc[*q]);
        Q.colptr[k + 1] = (int)Q.rowval.size();
    }
    return Q;
}

// The column partition of Schur complement mode (schur_supernode_partition,
// src/symbolic/supernodes.jl:391-425): the last ns columns of perm form one dense root supernode, the
// last, whose etree is the chain of its columns with the dense column counts ns, ns - 1, ..., 1; the
// other columns are partitioned as usual on their own elimination forest (fundamental supernodes,
// then amalgamation), so nothing merges into the root; a supernode whose last column has its etree
// parent among the Schur columns becomes a child of the root.
SupernodePartition schur_supernode_partition(const Pattern& P, const vector<int>& perm, int ns, bool amalg, int mw,
                                             double zf, int minw, int& sdepth) {
    const int n = P.n, m = n - ns;
    if (ns < 1 || ns > n) throw AnalysisError("the Schur complement must have between 1 and n rows");
    vector<int> parent = etree(P, perm), post = postorder(parent), counts = colcounts(P, perm, parent, post);
    vector<int> subparent(m + 1, 0);
    for (int j = 1; j <= m; ++j) subparent[j] = parent[j] > m ? 0 : parent[j];
    for (int j = m + 1; j <= n; ++j) {
        parent[j] = j < n ? j + 1 : 0;
        counts[j] = n - j + 1;
    }
    vector<int> subcounts(counts.begin(), counts.begin() + m + 1);
    ColumnPartition cp;
    if (m > 0) {
        cp = fundamental_supernodes(subparent, postorder(subparent), subcounts);
        if (amalg) cp = amalgamate(cp, subparent, subcounts, mw, zf, minw);
    } else {
        cp.order.assign(1, 0);
        cp.super_ptr = {0, 1};
        cp.snparent.assign(1, 0);
    }
    const int nsub = cp.ns();
    ColumnPartition full = cp;
    for (int j = m + 1; j <= n; ++j) full.order.push_back(j);
    full.super_ptr.push_back(n + 1);
    for (int s = 1; s <= nsub; ++s)
        if (full.snparent[s] == 0 && parent[cp.order[cp.super_ptr[s + 1] - 1]] > m) full.snparent[s] = nsub + 1;
    full.snparent.push_back(0);
    sdepth = tree_height(full.snparent);
    return supernode_partition(P, perm, parent, counts, full);
}

// The pattern of S = A22 - A21 A11^{-1} A12 over the flagged vertices in increasing order (schur_pattern,
// src/symbolic/ordering.jl:424-470): (i, j) when i == j, when (i, j) is in P, or when both are adjacent
// to one connected component of the graph of the other vertices. 1-based CSR, sorted columns.
void schur_pattern(const Pattern& P, const vector<char>& flag, vector<i64>& rowptr, vector<i64>& colval) {
    const int n = P.n;
    vector<int> loc(n + 1, 0);
    int ns = 0;
    for (int v = 1; v <= n; ++v)
        if (flag[v]) loc[v] = ++ns;
    vector<vector<int>> adj(ns + 1);
    for (int k = 1; k <= ns; ++k) adj[k].push_back(k);
    for (int v = 1; v <= n; ++v) {
        if (!loc[v]) continue;
        for (const int* q = P.nb_begin(v); q != P.nb_end(v); ++q)
            if (loc[*q]) adj[loc[v]].push_back(loc[*q]);
    }
    vector<char> seen(n + 1, 0);
    vector<int> mark(ns + 1, 0), stack, nbrs;
    int ncomp = 0;
    for (int v0 = 1; v0 <= n; ++v0) {
        if (loc[v0] || seen[v0]) continue;
        ++ncomp;
        nbrs.clear();
        seen[v0] = 1;
        stack.push_back(v0);
        while (!stack.empty()) {
            const int v = stack.back();
            stack.pop_back();
            for (const int* q = P.nb_begin(v); q != P.nb_end(v); ++q) {
                const int i = *q;
                if (loc[i]) {
                    if (mark[loc[i]] != ncomp) {
                        mark[loc[i]] = ncomp;
                        nbrs.push_back(loc[i]);
                    }
                } else if (!seen[i]) {
                    seen[i] = 1;
                    stack.push_back(i);
                }
            }
        }
        for (int a : nbrs)
            for (int b : nbrs)
                if (a != b) adj[a].push_back(b);
    }
    rowptr.assign(ns + 1, 0);
    rowptr[0] = 1;
    colval.clear();
    for (int k = 1; k <= ns; ++k) {
        vector<int>& c = adj[k];
        std::sort(c.begin(), c.end());
        c.erase(std::unique(c.begin(), c.end()), c.end());
        colval.insert(colval.end(), c.begin(), c.end());
        rowptr[k] = (i64)colval.size() + 1;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
struct sdsa_result {
    int n = 0;
    i64 nnz = 0;
    int structure = 0;
    int alg_used = 0;
    int pair_rounds = 0;
    int sdepth = 0;
    SupernodePartition sp;
    vector<IPair> pairs;
    vector<i64> panel_ptr, front_nrows, front_ncols, child_ptr, child_list, relind_ptr, relind, amap, amap_ptr,
        amap_src;
    vector<i64> full_rowptr, full_colval, full_srcptr, full_src, full_conj;
    int schur = 0;       // Schur complement mode: the root supernode (1-based), 0 = off
    vector<i64> schur_rowptr, schur_colval;
    vector<int> ordering;  // the ordering algorithm's permutation (1-based, slot 0 unused), before the
                           // supernodal renumbering that `perm` composes with it
};

namespace {

// assembly map and its owner-pull grouping (src/symbolic/maps.jl:146-186)
void build_maps(sdsa_result& R, const Csr& A, int structure, int view) {
    const SupernodePartition& sp = R.sp;
    int ns = sp.ns();
    R.panel_ptr.assign(ns + 1, 0);
    R.front_nrows.assign(ns, 0);
    R.front_ncols.assign(ns, 0);
    R.panel_ptr[0] = 1;
    for (int s = 1; s <= ns; ++s) {
        i64 f = sp.nrows(s), w = sp.width(s);
        R.front_nrows[s - 1] = f;
        R.front_ncols[s - 1] = w;
        R.panel_ptr[s] = R.panel_ptr[s - 1] + f * w;
    }
    i64 nnz = (i64)A.cv.size() - 1;
    R.amap.assign(nnz, 0);
    vector<int> owner(nnz, 0);                 // the front of each kept entry (1-based), 0 = dropped
    bool neg = structure == SDSA_STRUCTURE_G;  // real element types: only "G" mirrors into Uᵀ
    for (int r = 1; r <= A.n; ++r)
        for (i64 p = A.rp[r]; p < A.rp[r + 1]; ++p) {
            int c = (int)A.cv[p];
            if (!keep_entry(structure, view, r, c)) continue;
            int i = sp.iperm[r], j = sp.iperm[c];
            bool flip = i < j;
            if (flip) std::swap(i, j);
            int s = sp.col2sn[j];
            const int* rb = sp.rowval.data() + sp.rowptr[s];
            const int* re = sp.rowval.data() + sp.rowptr[s + 1];
            const int* q = std::lower_bound(rb, re, i);
            if (q == re || *q != i) throw AnalysisError("entry outside the symbolic factor");
            i64 f = re - rb;
            i64 off = R.panel_ptr[s - 1] + (i64)(j - sp.super_ptr[s]) * f + (q - rb);
            R.amap[p - 1] = (flip && neg) ? -off : off;
            owner[p - 1] = s;
        }
    // grouping: the kept entries ordered by (|off|, off < 0 [G only], p). The fronts own disjoint,
    // increasing ranges of offsets, so the entries are bucketed by front (a counting sort, in p order)
    // and each front's bucket is sorted by that key: the same strict order as one sort of all entries.
    vector<i64> cnt(ns + 1, 0);
    for (i64 p = 0; p < nnz; ++p) cnt[owner[p]]++;
    R.amap_ptr.assign(ns + 1, 0);
    R.amap_ptr[0] = 1;
    for (int s = 1; s <= ns; ++s) R.amap_ptr[s] = R.amap_ptr[s - 1] + cnt[s];
    R.amap_src.assign(R.amap_ptr[ns] - 1, 0);
    {
        vector<i64> next(R.amap_ptr.begin(), R.amap_ptr.end() - 1);
        for (i64 p = 0; p < nnz; ++p)
            if (owner[p]) R.amap_src[next[owner[p] - 1]++ - 1] = p;
    }
    bool signed_ = structure == SDSA_STRUCTURE_G;
    for (int s = 1; s <= ns; ++s)
        std::sort(R.amap_src.begin() + (R.amap_ptr[s - 1] - 1), R.amap_src.begin() + (R.amap_ptr[s] - 1),
                  [&](i64 a, i64 b) {
                      i64 oa = std::llabs(R.amap[a]), ob = std::llabs(R.amap[b]);
                      if (oa != ob) return oa < ob;
                      if (signed_) {
                          bool na = R.amap[a] < 0, nb = R.amap[b] < 0;
                          if (na != nb) return !na;
                      }
                      return a < b;
                  });
    for (i64& q : R.amap_src) q += 1;
    // children in increasing id (maps.jl:209-223)
    R.child_ptr.assign(ns + 1, 0);
    R.child_ptr[0] = 1;
    vector<i64> nch(ns + 1, 0);
    for (int s = 1; s <= ns; ++s)
        if (sp.snparent[s] != 0) nch[sp.snparent[s]]++;
    for (int s = 1; s <= ns; ++s) R.child_ptr[s] = R.child_ptr[s - 1] + nch[s];
    R.child_list.assign(R.child_ptr[ns] - 1, 0);
    vector<i64> next(R.child_ptr.begin(), R.child_ptr.end() - 1);
    for (int s = 1; s <= ns; ++s) {
        int p = sp.snparent[s];
        if (p == 0) continue;
        R.child_list[next[p - 1] - 1] = s;
        next[p - 1]++;
    }
    // relative indices (maps.jl:110-132)
    // (each parent's row positions are tabulated once and read by all of its children)
    R.relind_ptr.assign(ns + 1, 0);
    R.relind_ptr[0] = 1;
    for (int c = 1; c <= ns; ++c)
        R.relind_ptr[c] = R.relind_ptr[c - 1] + (sp.snparent[c] != 0 ? sp.nrows(c) - sp.width(c) : 0);
    R.relind.assign(R.relind_ptr[ns] - 1, 0);
    {
        vector<int> at(sp.n + 1, 0), stamp(sp.n + 1, 0);
        for (int p = 1; p <= ns; ++p) {
            if (R.child_ptr[p] == R.child_ptr[p - 1]) continue;
            for (int k = 0, q = sp.rowptr[p]; q < sp.rowptr[p + 1]; ++q, ++k) {
                at[sp.rowval[q]] = k;
                stamp[sp.rowval[q]] = p;
            }
            for (i64 t = R.child_ptr[p - 1]; t < R.child_ptr[p]; ++t) {
                const int c = (int)R.child_list[t - 1];
                i64 o = R.relind_ptr[c - 1] - 1;
                for (int q = sp.rowptr[c] + sp.width(c); q < sp.rowptr[c + 1]; ++q) {
                    const int i = sp.rowval[q];
                    if (stamp[i] != p) throw AnalysisError("row missing from the parent");
                    R.relind[o++] = at[i] + 1;
                }
            }
        }
    }
    // full-pattern map of the residual (src/symbolic/pattern.jl:249-290)
    // the contributions (r, c, p) ordered by (r, c, p): bucketed by row (a counting sort), then each
    // row's few entries sorted by (c, p), the same strict order as one sort of all of them
    struct Contrib { i64 r, c, p; char cj; };
    vector<i64> rstart(A.n + 2, 0);
    for (int r = 1; r <= A.n; ++r)
        for (i64 p = A.rp[r]; p < A.rp[r + 1]; ++p) {
            int c = (int)A.cv[p];
            if (!keep_entry(structure, view, r, c)) continue;
            rstart[r + 1]++;
            if (structure != SDSA_STRUCTURE_G && r != c) rstart[c + 1]++;
        }
    for (int r = 1; r <= A.n; ++r) rstart[r + 1] += rstart[r];
    vector<Contrib> con(rstart[A.n + 1]);
    {
        vector<i64> next(rstart.begin(), rstart.end());
        for (int r = 1; r <= A.n; ++r)
            for (i64 p = A.rp[r]; p < A.rp[r + 1]; ++p) {
                int c = (int)A.cv[p];
                if (!keep_entry(structure, view, r, c)) continue;
                con[next[r]++] = {r, c, p, 0};
                if (structure != SDSA_STRUCTURE_G && r != c) con[next[c]++] = {c, r, p, 0};
            }
    }
    for (int r = 1; r <= A.n; ++r)
        std::sort(con.begin() + rstart[r], con.begin() + rstart[r + 1], [](const Contrib& a, const Contrib& b) {
            if (a.c != b.c) return a.c < b.c;
            return a.p < b.p;
        });
    R.full_rowptr.assign(A.n + 1, 0);
    R.full_colval.clear();
    R.full_srcptr.assign(1, 1);
    R.full_src.clear();
    R.full_conj.clear();
    vector<i64> nrow(A.n + 2, 0);
    i64 pr = 0, pc = 0;
    for (size_t t = 0; t < con.size(); ++t) {
        if (con[t].r != pr || con[t].c != pc) {
            if (t > 0) R.full_srcptr.push_back((i64)t + 1);
            R.full_colval.push_back(con[t].c);
            nrow[con[t].r]++;
            pr = con[t].r;
            pc = con[t].c;
        }
        R.full_src.push_back(con[t].p);
        R.full_conj.push_back(con[t].cj);
    }
    if (!con.empty()) R.full_srcptr.push_back((i64)con.size() + 1);
    R.full_rowptr[0] = 1;
    for (int r = 1; r <= A.n; ++r) R.full_rowptr[r] = R.full_rowptr[r - 1] + nrow[r];
}

// ---------------------------------------------------------------------------
// Matching and scaling: MC64 (Duff & Koster 2001) as the reference restates it
// (src/matching/mc64.jl). Rows of the square matrix are matched to columns from
// |a_ij|, on the host, from the values. 0-based in this section.

// Row-wise |a| of the matrix the matching reads (`_abs_csr`, mc64.jl:216-239): "G" the stored rows;
// the symmetric structures the full matrix rebuilt from the view's triangle. Duplicates are summed
// (in input order) before the absolute value; explicit zeros stay (job 1 counts them). Columns of a
// row ascending.
struct AbsCsr {
    vector<i64> ptr;
    vector<int> adj;
    vector<double> w;
};

AbsCsr abs_csr(const Csr& A, const double* nz, int structure, int view) {
    const int n = A.n;
    struct Entry {
        int r, c;
        double x;
    };
    vector<Entry> e;
    for (int r = 1; r <= n; ++r)
        for (i64 p = A.rp[r]; p < A.rp[r + 1]; ++p) {
            const int c = (int)A.cv[p];
            if (!keep_entry(structure, view, r, c)) continue;
            const double x = nz[p - 1];
            e.push_back({r - 1, c - 1, x});
            if (structure != SDSA_STRUCTURE_G && r != c) e.push_back({c - 1, r - 1, x});
        }
    std::stable_sort(e.begin(), e.end(), [](const Entry& a, const Entry& b) { return a.r != b.r ? a.r < b.r : a.c < b.c; });
    AbsCsr M;
    M.ptr.assign(n + 1, 0);
    for (size_t k = 0; k < e.size();) {
        size_t q = k;
        double sum = 0.0;
        for (; q < e.size() && e[q].r == e[k].r && e[q].c == e[k].c; ++q) sum += e[q].x;
        M.adj.push_back(e[k].c);
        M.w.push_back(std::fabs(sum));
        M.ptr[e[k].r + 1]++;
        k = q;
    }
    for (int i = 0; i < n; ++i) M.ptr[i + 1] += M.ptr[i];
    return M;
}

// Binary min-heap of (key, vertex) with lazy deletion. Equal keys keep the order of the sift rules
// below (parent wins ties going up, the left child wins ties going down), so the matching's choices
// among equal distances are reproducible.
struct MinHeap {
    vector<double> key;
    vector<int> val;
    void clear() { key.clear(); val.clear(); }
    bool empty() const { return key.empty(); }
    void push(double k, int v) {
        key.push_back(k);
        val.push_back(v);
        size_t i = key.size() - 1;
        while (i > 0) {
            const size_t p = (i - 1) / 2;
            if (key[p] <= key[i]) break;
            std::swap(key[p], key[i]);
            std::swap(val[p], val[i]);
            i = p;
        }
    }
    void pop(double& k, int& v) {
        k = key[0];
        v = val[0];
        const double lk = key.back();
        const int lv = val.back();
        key.pop_back();
        val.pop_back();
        const size_t m = key.size();
        if (m == 0) return;
        key[0] = lk;
        val[0] = lv;
        size_t i = 0;
        while (true) {
            const size_t l = 2 * i + 1;
            if (l >= m) break;
            const size_t c = (l + 1 < m && key[l + 1] < key[l]) ? l + 1 : l;
            if (key[i] <= key[c]) break;
            std::swap(key[i], key[c]);
            std::swap(val[i], val[c]);
            i = c;
        }
    }
};

// Minimum-cost matching of maximum cardinality between rows 0..n-1 and columns 0..n-1 (costs >= 0 on
// the edges adj[ptr[i]..ptr[i+1]), by successive shortest augmenting paths: Dijkstra on the reduced
// costs cost - u[i] - v[j] >= 0 (min_cost_matching, mc64.jl:109-189). lmate[i] = the column matched to
// row i or -1; u + v <= cost on every edge, with equality on the matched ones.
void min_cost_matching(const vector<i64>& ptr, const vector<int>& adj, const vector<double>& cost, int n,
                       vector<int>& lmate, vector<double>& u, vector<double>& v) {
    const double inf = std::numeric_limits<double>::infinity();
    lmate.assign(n, -1);
    vector<int> rmate(n, -1);
    u.assign(n, 0.0);
    v.assign(n, 0.0);
    // feasible start (u = min(0, row minimum) = 0 for nonnegative costs, v = 0), then a cheap
    // matching of the tight edges
    for (int i = 0; i < n; ++i) {
        double mn = 0.0;
        for (i64 p = ptr[i]; p < ptr[i + 1]; ++p) mn = std::min(mn, cost[p]);
        u[i] = mn;
        for (i64 p = ptr[i]; p < ptr[i + 1]; ++p) {
            const int j = adj[p];
            if (rmate[j] < 0 && cost[p] - u[i] <= 0.0) {
                lmate[i] = j;
                rmate[j] = i;
                break;
            }
        }
    }
    vector<double> dist(n, inf);
    vector<int> pred(n, -1);
    vector<char> done(n, 0);
    vector<int> touched, finals;
    MinHeap heap;
    for (int i0 = 0; i0 < n; ++i0) {
        if (lmate[i0] >= 0) continue;
        touched.clear();
        finals.clear();
        heap.clear();
        int cur = i0, jfree = -1;
        double dcur = 0.0, len = inf;
        while (true) {
            for (i64 p = ptr[cur]; p < ptr[cur + 1]; ++p) {
                const int j = adj[p];
                if (done[j]) continue;
                const double nd = dcur + std::max(cost[p] - u[cur] - v[j], 0.0);
                if (nd < dist[j]) {
                    if (std::isinf(dist[j])) touched.push_back(j);
                    dist[j] = nd;
                    pred[j] = cur;
                    heap.push(nd, j);
                }
            }
            int j = -1;
            while (!heap.empty()) {
                double d;
                int jj;
                heap.pop(d, jj);
                if (done[jj] || d > dist[jj]) continue;
                j = jj;
                break;
            }
            if (j < 0) break;   // no augmenting path: row i0 stays unmatched
            done[j] = 1;
            finals.push_back(j);
            if (rmate[j] < 0) {
                jfree = j;
                len = dist[j];
                break;
            }
            cur = rmate[j];     // the matched edge has reduced cost 0
            dcur = dist[j];
        }
        if (jfree >= 0) {
            u[i0] += len;
            for (int j : finals) {
                if (j == jfree) continue;
                u[rmate[j]] += len - dist[j];
                v[j] -= len - dist[j];
            }
            int j = jfree;
            while (true) {      // flip the alternating path
                const int i = pred[j];
                const int nj = lmate[i];
                lmate[i] = j;
                rmate[j] = i;
                if (i == i0) break;
                j = nj;
            }
        }
        for (int j : touched) {
            dist[j] = inf;
            done[j] = 0;
        }
    }
}

int matched_count(const vector<int>& lmate) {
    int c = 0;
    for (int j : lmate) c += j >= 0;
    return c;
}

// maximum cardinality matching on the edges with keep[p] (zero costs)
vector<int> cardinality_matching(const AbsCsr& M, int n, const vector<char>& keep) {
    vector<i64> sp(n + 1, 0);
    vector<int> sa;
    for (int i = 0; i < n; ++i) {
        for (i64 p = M.ptr[i]; p < M.ptr[i + 1]; ++p)
            if (keep[p]) sa.push_back(M.adj[p]);
        sp[i + 1] = (i64)sa.size();
    }
    vector<int> lmate;
    vector<double> u, v;
    min_cost_matching(sp, sa, vector<double>(sa.size(), 0.0), n, lmate, u, v);
    return lmate;
}

// jobs 2 and 3: maximize the smallest matched |a_ij| (bottleneck), by bisection over the distinct
// nonzero values (`_bottleneck_matching`, mc64.jl:258-279)
vector<int> bottleneck_matching(const AbsCsr& M, int n) {
    const size_t ne = M.w.size();
    vector<int> full = cardinality_matching(M, n, vector<char>(ne, 1));
    const int target = matched_count(full);
    vector<double> vals;
    for (double x : M.w)
        if (x > 0) vals.push_back(x);
    std::sort(vals.begin(), vals.end());
    vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
    if (vals.empty()) return full;
    auto at_least = [&](double t) {
        vector<char> keep(ne);
        for (size_t p = 0; p < ne; ++p) keep[p] = M.w[p] >= t;
        return cardinality_matching(M, n, keep);
    };
    vector<int> best = at_least(vals[0]);
    if (matched_count(best) != target) return full;
    size_t lo = 0, hi = vals.size() - 1;   // the largest threshold index that keeps `target` matches
    while (lo < hi) {
        const size_t mid = (lo + hi + 1) >> 1;
        vector<int> m = at_least(vals[mid]);
        if (matched_count(m) == target) {
            lo = mid;
            best = std::move(m);
        } else {
            hi = mid - 1;
        }
    }
    return best;
}

void finite_scaling(vector<double>& s) {
    for (double& x : s)
        if (!(std::isfinite(x) && x > 0)) x = 1.0;
}

// 2x2 pivot pairs of "S" from the cycles of a symmetric matching (`matching_pairs`, mc64.jl:380-441;
// Duff & Pralet 2005). perm is the 1-based matching permutation, d the symmetric scaling. Cycles of
// matched indices of length >= 2 are split into pairs of consecutive indices (a_{i, perm(i)} != 0):
// an even cycle takes the alternative with the larger product of scaled |a|, an odd one leaves out
// the index with the largest scaled diagonal. A pair is kept when one of its indices is a 2x2
// candidate (scaled |a_ii| <= tol * max_{j != i} scaled |a_ij|), or always with keep_all; its
// candidate is the index with the smaller scaled-diagonal ratio. Pairs (partner, candidate), 1-based,
// sorted by candidate.
vector<std::pair<i64, i64>> matching_pairs(const AbsCsr& M, int n, const i64* perm, const int8_t* matched,
                                           const double* d, double tol, bool keep_all) {
    vector<double> dg(n, 0.0), offmax(n, 0.0);
    for (int i = 0; i < n; ++i)
        for (i64 p = M.ptr[i]; p < M.ptr[i + 1]; ++p) {
            const int j = M.adj[p];
            const double x = d[i] * M.w[p] * d[j];
            if (j == i) dg[i] = x;
            else offmax[i] = std::max(offmax[i], x);
        }
    auto entry = [&](int i, int j) {
        for (i64 p = M.ptr[i]; p < M.ptr[i + 1]; ++p)
            if (M.adj[p] == j) return d[i] * M.w[p] * d[j];
        return 0.0;
    };
    auto ratio = [&](int i) { return offmax[i] > 0 ? dg[i] / offmax[i] : std::numeric_limits<double>::infinity(); };
    auto candidate = [&](int i) { return dg[i] <= tol * offmax[i]; };
    vector<char> seen(n, 0);
    vector<std::pair<i64, i64>> pairs;
    vector<int> cyc;
    for (int i0 = 0; i0 < n; ++i0) {
        if (seen[i0] || !matched[i0]) continue;
        cyc.clear();
        int i = i0;
        bool ok = true;
        while (!seen[i]) {
            seen[i] = 1;
            cyc.push_back(i);
            if (!matched[i]) ok = false;
            i = (int)perm[i] - 1;
        }
        const int L = (int)cyc.size();
        if (!(ok && i == i0 && L >= 2)) continue;
        int start;   // 0-based position of the first pair's first index
        if (L % 2 == 0) {
            double p0 = 1.0, p1 = 1.0;
            for (int k = 0; k < L; k += 2) {
                p0 *= entry(cyc[k], cyc[k + 1]);
                p1 *= entry(cyc[k + 1], cyc[(k + 2) % L]);
            }
            start = p1 > p0 ? 1 : 0;
        } else {
            int big = 0;   // the first largest scaled diagonal stays a singleton
            for (int k = 1; k < L; ++k)
                if (dg[cyc[k]] > dg[cyc[big]]) big = k;
            start = (big + 1) % L;
        }
        for (int t = 0; t + 1 < L; t += 2) {
            const int a = cyc[(start + t) % L], b = cyc[(start + t + 1) % L];
            if (!(keep_all || candidate(a) || candidate(b))) continue;
            if (ratio(a) < ratio(b)) pairs.push_back({b + 1, a + 1});
            else pairs.push_back({a + 1, b + 1});
        }
    }
    std::stable_sort(pairs.begin(), pairs.end(), [](const std::pair<i64, i64>& x, const std::pair<i64, i64>& y) {
        return x.second < y.second;
    });
    return pairs;
}

// MC64 jobs 1-5 (`mc64`, mc64.jl:302-333): lmate and the row / column scalings (ones except job 5,
// r_i = exp(u_i) / max_k |a_ik|, c_j = exp(v_j) from the assignment on log max_k |a_ik| - log |a_ij|,
// so that |r_i a_ij c_j| <= 1 with equality on the matched entries)
void mc64(const AbsCsr& M, int n, int job, vector<int>& lmate, vector<double>& rs, vector<double>& cs) {
    rs.assign(n, 1.0);
    cs.assign(n, 1.0);
    if (job == 1) {
        lmate = cardinality_matching(M, n, vector<char>(M.w.size(), 1));
        return;
    }
    if (job == 2 || job == 3) {
        lmate = bottleneck_matching(M, n);
        return;
    }
    vector<double> rowmax(n, 0.0);
    for (int i = 0; i < n; ++i)
        for (i64 p = M.ptr[i]; p < M.ptr[i + 1]; ++p) rowmax[i] = std::max(rowmax[i], M.w[p]);
    vector<i64> sp(n + 1, 0);
    vector<int> sa;
    vector<double> cost;
    for (int i = 0; i < n; ++i) {
        for (i64 p = M.ptr[i]; p < M.ptr[i + 1]; ++p) {
            if (!(M.w[p] > 0)) continue;
            sa.push_back(M.adj[p]);
            cost.push_back(job == 5 ? std::log(rowmax[i]) - std::log(M.w[p]) : rowmax[i] - M.w[p]);
        }
        sp[i + 1] = (i64)sa.size();
    }
    vector<double> u, v;
    min_cost_matching(sp, sa, cost, n, lmate, u, v);
    if (job == 5) {
        for (int i = 0; i < n; ++i) {
            rs[i] = rowmax[i] > 0 ? std::exp(u[i]) / rowmax[i] : 1.0;
            cs[i] = std::exp(v[i]);
        }
        finite_scaling(rs);
        finite_scaling(cs);
    }
}

}  // namespace

extern "C" {

void sdsa_default_options(sdsa_options* o, int structure) {
    std::memset(o, 0, sizeof(*o));
    o->structure = structure;
    o->view = 'F';
    o->index_base = 1;
    o->reordering = SDSA_REORDER_DEFAULT;
    o->user_perm = nullptr;
    o->pivot_pairs = SDSA_PAIRS_DEFAULT;
    o->pivot_pair_tolerance = 1e-6;
    o->pivot_threshold = 0.01;
    o->use_superpanels = 1;
    o->amalg_max_width = 32;
    o->amalg_zero_fraction = 0.25;
    o->amalg_min_width = 8;
}

const char* sdsa_last_error(void) { return g_err.c_str(); }

int sdsa_analyze(int64_t n, const int64_t* rowptr, const int64_t* colval, const double* nzval,
                 const sdsa_options* opts, sdsa_result** out) {
    *out = nullptr;
    try {
        if (n < 0) throw AnalysisError("n must be nonnegative");
        int structure = opts->structure;
        if (structure != SDSA_STRUCTURE_G && structure != SDSA_STRUCTURE_S && structure != SDSA_STRUCTURE_SPD)
            throw AnalysisError("structure must be G, S or SPD");
        int view = opts->view;
        if (view != 'L' && view != 'U' && view != 'F') throw AnalysisError("view must be 'L', 'U' or 'F'");
        Csr A = host_pattern(n, rowptr, colval, opts->index_base);
        Pattern P = symmetric_pattern(A, structure, view);
        bool amalg = opts->use_superpanels != 0;
        int mw = opts->amalg_max_width, minw = opts->amalg_min_width;
        double zf = opts->amalg_zero_fraction;
        if (mw < 1) throw AnalysisError("amalgamation max_width must be >= 1");

        std::unique_ptr<sdsa_result> R(new sdsa_result());
        R->n = (int)n;
        R->nnz = (i64)A.cv.size() - 1;
        R->structure = structure;
        auto user_perm = [&]() {
            vector<int> perm(n + 1, 0);
            vector<char> seen(n + 2, 0);
            bool zero_based = false;
            for (i64 k = 0; k < n; ++k) if (opts->user_perm[k] == 0) zero_based = true;
            for (i64 k = 0; k < n; ++k) {
                i64 v = opts->user_perm[k] + (zero_based ? 1 : 0);
                if (v < 1 || v > n || seen[v]) throw AnalysisError("user_perm is not a permutation");
                seen[v] = 1;
                perm[k + 1] = (int)v;
            }
            return perm;
        };
        // Schur complement mode: the flagged rows and columns (schur_flags, src/symbolic/ordering.jl:339-346)
        vector<char> sflag;
        int nschur = 0;
        if (opts->user_schur_indices) {
            sflag.assign(n + 1, 0);
            for (i64 k = 0; k < n; ++k)
                if (opts->user_schur_indices[k] != 0) {
                    sflag[k + 1] = 1;
                    ++nschur;
                }
            if (nschur == 0) throw AnalysisError("user_schur_indices selects no row: the Schur complement would be empty");
        }
        // ordering (with 2x2 pairs for "S")
        Ordered chosen;
        if (nschur > 0) {
            // compute_schur_ordering (src/symbolic/ordering.jl:386-415): the flagged vertices last in
            // increasing order; the others in the user permutation's relative order, or by the fill-reducing
            // ordering of the pattern they induce; no 2x2 pivot pairs
            vector<int> inner, perm(1, 0);
            for (int v = 1; v <= (int)n; ++v)
                if (!sflag[v]) inner.push_back(v);
            if (opts->user_perm) {
                const vector<int> up = user_perm();
                for (int k = 1; k <= (int)n; ++k)
                    if (!sflag[up[k]]) perm.push_back(up[k]);
                chosen.alg = 4;
            } else {
                Pattern Q = induced_pattern(P, inner);
                const int requested = opts->reordering;
                vector<int> algs = requested == SDSA_REORDER_DEFAULT ? vector<int>{SDSA_REORDER_AMD, SDSA_REORDER_ND}
                                                                      : vector<int>{requested};
                vector<int> best;
                double best_cost = 0;
                for (int a : algs) {
                    vector<int> q = ordering_perm(Q, a);
                    const double c = evaluate_ordering(Q, q, amalg, mw, zf, minw).cost;
                    if (best.empty() || c < best_cost) {
                        best = q;
                        best_cost = c;
                        chosen.alg = a;
                    }
                }
                for (int k = 1; k <= Q.n; ++k) perm.push_back(inner[best[k] - 1]);
            }
            for (int v = 1; v <= (int)n; ++v)
                if (sflag[v]) perm.push_back(v);
            chosen.perm = perm;
        } else if (opts->user_perm) {
            chosen.alg = 4;
            chosen.perm = user_perm();
        } else {
            int requested = opts->reordering;
            bool search = structure == SDSA_STRUCTURE_S && opts->pivot_pairs != SDSA_PAIRS_NONE &&
                          requested != SDSA_REORDER_NATURAL && nzval != nullptr;
            PairCandidates cands;
            vector<IPair> fixed;
            if (structure == SDSA_STRUCTURE_S && opts->user_pairs && opts->n_user_pairs > 0) {
                // pairs chosen by the caller (the cycles of a matching): the ordering keeps each pair
                // adjacent, with no value-based search
                for (i64 k = 0; k < opts->n_user_pairs; ++k) {
                    const i64 a = opts->user_pairs[2 * k], b = opts->user_pairs[2 * k + 1];
                    if (a < 1 || a > n || b < 1 || b > n || a == b) throw AnalysisError("user_pairs out of range");
                    fixed.push_back({(int)a, (int)b});
                }
                search = false;
            }
            if (search) {
                cands = pivot_candidates(P, A, nzval, structure, view, opts->pivot_pair_tolerance);
                if (opts->pivot_pairs == SDSA_PAIRS_ALL) {
                    fixed = all_pivot_pairs(P, cands);
                    search = false;
                }
            }
            vector<int> algs;
            if (requested == SDSA_REORDER_DEFAULT) algs = {SDSA_REORDER_AMD, SDSA_REORDER_ND};
            else algs = {requested};
            vector<Ordered> cands_o;
            for (int a : algs) {
                if (search) {
                    cands_o.push_back(pair_ordering(P, a, cands, opts->pivot_threshold));
                } else if (fixed.empty()) {
                    Ordered o;
                    o.alg = a;
                    o.perm = ordering_perm(P, a);
                    cands_o.push_back(o);
                } else {
                    vector<int> gptr, members;
                    Pattern Pc = compressed_pattern(P, fixed, gptr, members);
                    Ordered o;
                    o.alg = a;
                    o.perm = expand_permutation(ordering_perm(Pc, a), gptr, members);
                    o.pairs = fixed;
                    cands_o.push_back(o);
                }
            }
            int best = -1;
            size_t best_zeros = 0;
            double best_cost = 0;
            for (size_t k = 0; k < cands_o.size(); ++k) {
                Pattern Q = pair_pattern(P, cands_o[k].pairs);
                Evaluated e = evaluate_ordering(Q, cands_o[k].perm, amalg, mw, zf, minw);
                size_t zl = (search && cands_o.size() > 1)
                                ? structural_zero_pivots(cands, P, cands_o[k].perm, cands_o[k].pairs).size()
                                : 0;
                if (best < 0 || zl < best_zeros || (zl == best_zeros && e.cost < best_cost)) {
                    best = (int)k;
                    best_zeros = zl;
                    best_cost = e.cost;
                }
            }
            chosen = cands_o[best];
        }
        R->alg_used = chosen.alg;
        R->ordering = chosen.perm;
        R->pairs = chosen.pairs;
        R->pair_rounds = chosen.rounds;
        Pattern F = pair_pattern(P, chosen.pairs);
        if (nschur > 0) {
            R->sp = schur_supernode_partition(F, chosen.perm, nschur, amalg, mw, zf, minw, R->sdepth);
            R->schur = R->sp.ns();
            schur_pattern(P, sflag, R->schur_rowptr, R->schur_colval);
        } else {
            vector<int> parent = etree(F, chosen.perm), post = postorder(parent),
                        counts = colcounts(F, chosen.perm, parent, post);
            ColumnPartition cp = fundamental_supernodes(parent, post, counts);
            if (amalg) cp = amalgamate(cp, parent, counts, mw, zf, minw);
            R->sdepth = tree_height(cp.snparent);
            R->sp = supernode_partition(F, chosen.perm, parent, counts, cp);
        }
        build_maps(*R, A, structure, view);
        *out = R.release();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

static const vector<int>* int_field(const sdsa_result* r, const std::string& nm, int& skip) {
    skip = 1;  // 1-based vectors with slot 0 unused
    const SupernodePartition& sp = r->sp;
    if (nm == "perm") return &sp.perm;
    if (nm == "iperm") return &sp.iperm;
    if (nm == "counts") return &sp.counts;
    if (nm == "super_ptr") return &sp.super_ptr;
    if (nm == "snparent") return &sp.snparent;
    if (nm == "snpost") return &sp.snpost;
    if (nm == "rowptr") return &sp.rowptr;
    if (nm == "rowval") return &sp.rowval;
    if (nm == "ordering") return &r->ordering;
    return nullptr;
}

static const vector<i64>* i64_field(const sdsa_result* r, const std::string& nm) {
    if (nm == "front_ptr") return &r->panel_ptr;
    if (nm == "front_nrows") return &r->front_nrows;
    if (nm == "front_ncols") return &r->front_ncols;
    if (nm == "child_ptr") return &r->child_ptr;
    if (nm == "child_list") return &r->child_list;
    if (nm == "relind_ptr") return &r->relind_ptr;
    if (nm == "relind") return &r->relind;
    if (nm == "amap") return &r->amap;
    if (nm == "amap_ptr") return &r->amap_ptr;
    if (nm == "amap_src") return &r->amap_src;
    if (nm == "full_rowptr") return &r->full_rowptr;
    if (nm == "full_colval") return &r->full_colval;
    if (nm == "full_srcptr") return &r->full_srcptr;
    if (nm == "full_src") return &r->full_src;
    if (nm == "full_conj") return &r->full_conj;
    if (nm == "schur_rowptr") return &r->schur_rowptr;
    if (nm == "schur_colval") return &r->schur_colval;
    return nullptr;
}

int64_t sdsa_len(const sdsa_result* r, const char* name) {
    std::string nm(name);
    int skip;
    if (nm == "pairs") return 2 * (int64_t)r->pairs.size();
    if (const vector<int>* v = int_field(r, nm, skip)) return (int64_t)v->size() - skip;
    if (const vector<i64>* v = i64_field(r, nm)) return (int64_t)v->size();
    return -1;
}

int sdsa_get(const sdsa_result* r, const char* name, int64_t* out) {
    std::string nm(name);
    int skip;
    if (nm == "pairs") {
        for (size_t k = 0; k < r->pairs.size(); ++k) {
            out[2 * k] = r->pairs[k].first;
            out[2 * k + 1] = r->pairs[k].second;
        }
        return 0;
    }
    if (const vector<int>* v = int_field(r, nm, skip)) {
        for (size_t k = skip; k < v->size(); ++k) out[k - skip] = (*v)[k];
        return 0;
    }
    if (const vector<i64>* v = i64_field(r, nm)) {
        std::copy(v->begin(), v->end(), out);
        return 0;
    }
    g_err = "unknown map " + nm;
    return -1;
}

double sdsa_stat(const sdsa_result* r, const char* name) {
    std::string nm(name);
    if (nm == "n") return r->n;
    if (nm == "nnz") return (double)r->nnz;
    if (nm == "ns") return r->sp.ns();
    if (nm == "nnz_stored") return (double)r->sp.nnz_stored;
    if (nm == "nnz_L") return (double)r->sp.nnz_L;
    if (nm == "flops") return r->sp.flops;
    if (nm == "factor_len") return r->panel_ptr.empty() ? 0.0 : (double)(r->panel_ptr.back() - 1);
    if (nm == "sdepth") return r->sdepth;
    if (nm == "alg_used") return r->alg_used;
    if (nm == "npairs") return (double)r->pairs.size();
    if (nm == "pair_rounds") return r->pair_rounds;
    if (nm == "schur") return r->schur;
    if (nm == "schur_n") return r->schur ? r->sp.width(r->schur) : 0;
    return NAN;
}

void sdsa_free(sdsa_result* r) { delete r; }

int sdsa_matching_pairs(int64_t n, const int64_t* rowptr, const int64_t* colval, const double* nzval, int view,
                        int index_base, const int64_t* perm, const int8_t* matched, const double* d, int pivot_pairs,
                        double pivot_pair_tolerance, int64_t* pairs, int64_t* npairs) {
    try {
        *npairs = 0;
        if (n < 0) throw AnalysisError("n must be nonnegative");
        if (view != 'L' && view != 'U' && view != 'F') throw AnalysisError("view must be 'L', 'U' or 'F'");
        if (pivot_pairs == SDSA_PAIRS_NONE || n == 0) return 0;
        Csr A = host_pattern(n, rowptr, colval, index_base);
        const int nn = (int)n;
        for (int i = 0; i < nn; ++i)
            if (perm[i] < 1 || perm[i] > n) throw AnalysisError("perm out of range");
        AbsCsr M = abs_csr(A, nzval, SDSA_STRUCTURE_S, view);
        auto pr = matching_pairs(M, nn, perm, matched, d, pivot_pair_tolerance, pivot_pairs == SDSA_PAIRS_ALL);
        for (size_t k = 0; k < pr.size(); ++k) {
            pairs[2 * k] = pr[k].first;
            pairs[2 * k + 1] = pr[k].second;
        }
        *npairs = (int64_t)pr.size();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

int sdsa_matching(int64_t n, const int64_t* rowptr, const int64_t* colval, const double* nzval, int structure,
                  int view, int index_base, int job, int64_t* perm, int8_t* matched, double* rscale,
                  double* cscale) {
    try {
        if (n < 0) throw AnalysisError("n must be nonnegative");
        if (structure != SDSA_STRUCTURE_G && structure != SDSA_STRUCTURE_S && structure != SDSA_STRUCTURE_SPD)
            throw AnalysisError("structure must be G, S or SPD");
        if (view != 'L' && view != 'U' && view != 'F') throw AnalysisError("view must be 'L', 'U' or 'F'");
        if (job == 6) job = 5;   // "algo6" (automatic) runs job 5
        if (job < 1 || job > 5) throw AnalysisError("unknown matching job; expected 1 to 6");
        if (n > 0 && (!rowptr || !colval || !nzval || !perm || !matched || !rscale || !cscale))
            throw AnalysisError("NULL array");
        Csr A = host_pattern(n, rowptr, colval, index_base);
        const int nn = (int)n;
        AbsCsr M = abs_csr(A, nzval, structure, view);
        vector<int> lmate;
        vector<double> rs, cs;
        mc64(M, nn, job, lmate, rs, cs);
        // the matching permutation (`_complete_matching`, mc64.jl:344-357): unmatched rows take the
        // unmatched columns in increasing order
        vector<char> used(nn, 0);
        for (int j : lmate)
            if (j >= 0) used[j] = 1;
        int next_free = 0;
        for (int i = 0; i < nn; ++i) {
            matched[i] = lmate[i] >= 0 ? 1 : 0;
            int j = lmate[i];
            if (j < 0) {
                while (used[next_free]) ++next_free;
                j = next_free++;
            }
            perm[i] = j + 1;
        }
        if (structure == SDSA_STRUCTURE_G) {
            for (int i = 0; i < nn; ++i) {
                rscale[i] = rs[i];
                cscale[i] = cs[i];
            }
            return 0;
        }
        // symmetric scaling d = sqrt(r c) (Duff & Pralet 2005); an unmatched index takes
        // 1 / max_j |a_ij| d_j over its matched neighbours (compute_matching, mc64.jl:378-398)
        vector<double> d(nn);
        for (int i = 0; i < nn; ++i) d[i] = std::sqrt(rs[i] * cs[i]);
        for (int i = 0; i < nn; ++i) {
            if (matched[i]) continue;
            double m = 0.0;
            for (i64 p = M.ptr[i]; p < M.ptr[i + 1]; ++p)
                if (matched[M.adj[p]]) m = std::max(m, M.w[p] * d[M.adj[p]]);
            d[i] = m > 0 ? 1.0 / m : 1.0;
        }
        finite_scaling(d);
        for (int i = 0; i < nn; ++i) rscale[i] = cscale[i] = d[i];
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

}  // extern "C"
