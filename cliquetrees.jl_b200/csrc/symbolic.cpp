// Host-side symbolic analysis for the multifrontal numeric phase.
//
// This is integer work that runs once per sparsity pattern and is uploaded
// to the GPU afterwards.  It restates, in C++, the steps CliqueTrees.jl takes
// from an elimination order to a `ChordalSymbolic`:
//
//   eliminationtree_impl!          src/trees.jl:127-138
//   etree_impl! (Liu, path compr.) src/parent.jl:54-90
//   supcnt_impl! (column counts)   src/parent.jl:201-297
//   stree_impl!  (Maximal)         src/supernode_types.jl:41-88
//   postorder_impl! / invpermute   src/parent.jl:420-458, :527-598
//   supernodetree_impl! relabel    src/supernode_trees.jl:107-180
//   cliquetree_impl! separators    src/clique_trees.jl:146-234
//   ChordalSymbolic(res,sep,tree)  src/Multifrontal.jl/src/chordal_symbolic.jl:302-378
//
// Everything is 0-based here; the reference is 1-based.  The column counts
// are computed with the Gilbert-Ng-Peyton skeleton/LCA algorithm (the same
// mathematical quantity supcnt_impl! produces), everything else follows the
// reference's traversal orders so that the supernode partition, postorder,
// relabelling and separators come out identical.
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <algorithm>
#include <new>
#include <string>

#include "../../include/cliquetrees_symbolic.h"

typedef int64_t I;

struct ct_symbolic {
    I n = 0, nfr = 0;
    std::vector<I> order;   // order[i] = original vertex placed at position i
    std::vector<I> invp;    // invp[v]  = position of original vertex v
    std::vector<I> resptr;  // nfr+1
    std::vector<I> sepptr;  // nfr+1
    std::vector<I> septgt;  // sepptr[nfr]
    std::vector<I> reltgt;  // sepptr[nfr]
    std::vector<I> pnt;     // nfr, -1 for roots
    std::vector<I> chdptr;  // nfr+2, list nfr holds the roots
    std::vector<I> chdtgt;  // nfr
    std::vector<I> idx;     // n, column -> front
    std::vector<I> Dptr;    // nfr+1
    std::vector<I> Lptr;    // nfr+1
    I nMptr = 0, nMval = 0, nNval = 0, nFval = 0;
};

static thread_local std::string g_err;

extern "C" const char* ct_last_error(void) { return g_err.c_str(); }
void ct_set_error(const std::string& msg) { g_err = msg; }

// ---------------------------------------------------------------------------
// graph helpers
// ---------------------------------------------------------------------------

// upper[k] = neighbours of (new) vertex k with smaller new label, self loops
// dropped.  Mirrors sympermute!_impl! with the Forward ordering
// (src/bipartite_graphs.jl:275-334): the count and fill passes walk the
// original vertices in increasing order and each undirected edge once.
static void sympermute_forward(I n, const I* colptr, const I* rowval, const I* index,
                               std::vector<I>& ptr, std::vector<I>& tgt) {
    ptr.assign(n + 1, 0);
    for (I j = 0; j < n; ++j) {
        I jj = index[j];
        for (I p = colptr[j]; p < colptr[j + 1]; ++p) {
            I i = rowval[p];
            if (i < j) {
                I ii = index[i], kk = jj;
                if (kk < ii) kk = ii;
                ptr[kk + 1] += 1;
            }
        }
    }
    for (I k = 0; k < n; ++k) ptr[k + 1] += ptr[k];
    tgt.assign(ptr[n], 0);
    std::vector<I> pos(ptr.begin(), ptr.end() - 1);
    for (I j = 0; j < n; ++j) {
        I jj = index[j];
        for (I p = colptr[j]; p < colptr[j + 1]; ++p) {
            I i = rowval[p];
            if (i < j) {
                I ii = index[i], kk = jj;
                if (kk < ii) std::swap(ii, kk);
                tgt[pos[kk]++] = ii;
            }
        }
    }
}

// transpose of a graph on n vertices; adjacency lists come out sorted
// (reverse!_impl!, src/bipartite_graphs.jl:360-391).
static void transpose_graph(I n, const std::vector<I>& ptr, const std::vector<I>& tgt,
                            std::vector<I>& rptr, std::vector<I>& rtgt) {
    rptr.assign(n + 1, 0);
    for (I j = 0; j < n; ++j)
        for (I p = ptr[j]; p < ptr[j + 1]; ++p) rptr[tgt[p] + 1] += 1;
    for (I k = 0; k < n; ++k) rptr[k + 1] += rptr[k];
    rtgt.assign(rptr[n], 0);
    std::vector<I> pos(rptr.begin(), rptr.end() - 1);
    for (I j = 0; j < n; ++j)
        for (I p = ptr[j]; p < ptr[j + 1]; ++p) rtgt[pos[tgt[p]]++] = j;
}

// Liu's elimination tree with path compression (src/parent.jl:54-90).
static void etree(I n, const std::vector<I>& uptr, const std::vector<I>& utgt, std::vector<I>& parent) {
    parent.assign(n, -1);
    std::vector<I> ancestor(n, -1);
    for (I i = 0; i < n; ++i) {
        for (I p = uptr[i]; p < uptr[i + 1]; ++p) {
            I r = utgt[p];
            if (r < i) {
                while (ancestor[r] != -1 && ancestor[r] != i) {
                    I t = ancestor[r];
                    ancestor[r] = i;
                    r = t;
                }
                if (ancestor[r] == -1) {
                    ancestor[r] = i;
                    parent[r] = i;
                }
            }
        }
    }
}

// children lists in increasing order (reverse!_impl!, src/parent.jl:151-193);
// list n holds the roots.
static void children_lists(I n, const std::vector<I>& parent, std::vector<I>& ptr, std::vector<I>& tgt) {
    ptr.assign(n + 2, 0);
    for (I i = 0; i < n; ++i) {
        I j = parent[i] < 0 ? n : parent[i];
        ptr[j + 1] += 1;
    }
    for (I k = 0; k <= n; ++k) ptr[k + 1] += ptr[k];
    tgt.assign(n, 0);
    std::vector<I> pos(ptr.begin(), ptr.end() - 1);
    for (I i = 0; i < n; ++i) {
        I j = parent[i] < 0 ? n : parent[i];
        tgt[pos[j]++] = i;
    }
}

// Postorder of a forest following postorder_impl! (src/parent.jl:420-458):
// children are visited in increasing order; the roots are pushed on the
// stack in increasing order, so the largest root is traversed first.
// Returns index[v] = postorder position of v.
static void postorder_like_reference(I n, const std::vector<I>& parent, std::vector<I>& index) {
    std::vector<I> brother(n, -1), child(n, -1), stack;
    stack.reserve(n);
    I root = -1;
    for (I i = n - 1; i >= 0; --i) {
        I j = parent[i];
        if (j < 0) { brother[i] = root; root = i; }
        else { brother[i] = child[j]; child[j] = i; }
    }
    for (I r = root; r != -1; r = brother[r]) stack.push_back(r);
    index.assign(n, -1);
    for (I i = 0; i < n; ++i) {
        I j = stack.back(); stack.pop_back();
        while (child[j] != -1) {
            stack.push_back(j);
            I c = child[j];
            child[j] = brother[c];
            j = c;
        }
        index[j] = i;
    }
}

// Column counts of the Cholesky factor (diagonal included) from the
// elimination tree and the higher-neighbour lists, by the row-subtree
// skeleton method of Gilbert, Ng and Peyton.  This is the quantity that
// supcnt_impl! computes (src/parent.jl:201-297).
static void column_counts(I n, const std::vector<I>& parent, const std::vector<I>& lptr,
                          const std::vector<I>& ltgt, std::vector<I>& cc) {
    // any postorder works for this computation
    std::vector<I> post(n), head(n, -1), next(n, -1), stack;
    for (I j = n - 1; j >= 0; --j) {
        if (parent[j] >= 0) { next[j] = head[parent[j]]; head[parent[j]] = j; }
    }
    I k = 0;
    stack.reserve(n);
    for (I r = 0; r < n; ++r) {
        if (parent[r] >= 0) continue;
        stack.push_back(r);
        while (!stack.empty()) {
            I p = stack.back();
            I c = head[p];
            if (c == -1) { stack.pop_back(); post[k++] = p; }
            else { head[p] = next[c]; stack.push_back(c); }
        }
    }
    std::vector<I> first(n, -1), maxfirst(n, -1), prevleaf(n, -1), ancestor(n);
    cc.assign(n, 0);
    for (k = 0; k < n; ++k) {
        I j = post[k];
        cc[j] = (first[j] == -1) ? 1 : 0;
        for (; j != -1 && first[j] == -1; j = parent[j]) first[j] = k;
    }
    for (I i = 0; i < n; ++i) ancestor[i] = i;
    for (k = 0; k < n; ++k) {
        I j = post[k];
        if (parent[j] != -1) cc[parent[j]] -= 1;
        for (I p = lptr[j]; p < lptr[j + 1]; ++p) {
            I i = ltgt[p];
            // is j a leaf of the i-th row subtree?
            if (i <= j || first[j] <= maxfirst[i]) continue;
            maxfirst[i] = first[j];
            I jprev = prevleaf[i];
            prevleaf[i] = j;
            cc[j] += 1;
            if (jprev == -1) continue;
            I q = jprev;
            while (q != ancestor[q]) q = ancestor[q];
            for (I s = jprev; s != q;) { I sp = ancestor[s]; ancestor[s] = q; s = sp; }
            cc[q] -= 1;
        }
        if (parent[j] != -1) ancestor[j] = parent[j];
    }
    for (k = 0; k < n; ++k) {
        I j = post[k];
        if (parent[j] != -1) cc[parent[j]] += cc[j];
    }
}

// ---------------------------------------------------------------------------
// main driver
// ---------------------------------------------------------------------------

static int build(ct_symbolic* S, I n, const I* colptr, const I* rowval, const I* order_in) {
    S->n = n;
    std::vector<I> order(order_in, order_in + n), index(n, -1);
    for (I i = 0; i < n; ++i) {
        I v = order[i];
        if (v < 0 || v >= n || index[v] != -1) { g_err = "order is not a permutation"; return -2; }
        index[v] = i;
    }
    for (I j = 0; j < n; ++j) {
        if (colptr[j] > colptr[j + 1]) { g_err = "colptr is not monotone"; return -2; }
        for (I p = colptr[j]; p < colptr[j + 1]; ++p)
            if (rowval[p] < 0 || rowval[p] >= n) { g_err = "rowval out of range"; return -2; }
    }

    // upper: smaller neighbours in elimination labels; lower: larger ones.
    std::vector<I> uptr, utgt, lptr, ltgt;
    sympermute_forward(n, colptr, rowval, index.data(), uptr, utgt);
    std::vector<I> eparent;
    etree(n, uptr, utgt, eparent);
    transpose_graph(n, uptr, utgt, lptr, ltgt);

    std::vector<I> cc;
    column_counts(n, eparent, lptr, ltgt, cc);

    // maximal supernode partition (stree_impl!, Maximal)
    std::vector<I> cptr, ctgt;
    children_lists(n, eparent, cptr, ctgt);
    std::vector<I> nic(n), newv, sparent, sanc;
    newv.reserve(n); sparent.reserve(n); sanc.reserve(n);
    for (I v = 0; v < n; ++v) {
        I u = -1;
        for (I p = cptr[v]; p < cptr[v + 1]; ++p) {
            I s = ctgt[p];
            if (cc[s] == cc[v] + 1) { u = s; break; }
        }
        if (u >= 0) {
            nic[v] = nic[u];
            for (I p = cptr[v]; p < cptr[v + 1]; ++p) {
                I s = ctgt[p];
                if (s != u) { sparent[nic[s]] = nic[v]; sanc[nic[s]] = v; }
            }
        } else {
            nic[v] = (I)newv.size();
            newv.push_back(v); sparent.push_back(-1); sanc.push_back(-1);
            for (I p = cptr[v]; p < cptr[v + 1]; ++p) {
                I s = ctgt[p];
                sparent[nic[s]] = nic[v]; sanc[nic[s]] = v;
            }
        }
    }
    I h = (I)newv.size();
    S->nfr = h;

    // postorder the supernode tree and relabel it (postorder!_impl!)
    std::vector<I> sidx;
    postorder_like_reference(h, sparent, sidx);
    std::vector<I> pnt(h), old_of(h);
    for (I i = 0; i < h; ++i) {
        pnt[sidx[i]] = sparent[i] < 0 ? -1 : sidx[sparent[i]];
        old_of[sidx[i]] = i;
    }

    // relabel vertices: each supernode becomes a run of consecutive labels
    // (src/supernode_trees.jl:151-166)
    std::vector<I> label(n, -1), resptr(h + 1), seplen(h);
    resptr[0] = 0;
    for (I i = 0; i < h; ++i) {
        I j = old_of[i], u = newv[j];
        I p = resptr[i];
        label[u] = p;
        for (I v = eparent[u]; v != -1; v = eparent[v]) {
            if (v == sanc[j]) break;
            label[v] = ++p;
        }
        I nn = p - resptr[i] + 1;
        seplen[i] = cc[u] - nn;
        resptr[i + 1] = p + 1;
    }
    if (resptr[h] != n) { g_err = "internal: supernodes do not cover all vertices"; return -3; }

    S->order.assign(n, 0);
    for (I v = 0; v < n; ++v) S->order[label[v]] = order[v];
    S->invp.assign(n, 0);
    for (I i = 0; i < n; ++i) S->invp[S->order[i]] = i;

    // higher neighbours in final labels: for every edge of the elimination
    // graph, both labels preserve the ancestor order, so these lists come out
    // sorted (sympermute!_impl! with Reverse, src/clique_trees.jl:154).
    std::vector<I> hptr(n + 1, 0), htgt;
    for (I j = 0; j < n; ++j)
        for (I p = lptr[j]; p < lptr[j + 1]; ++p) {
            I a = label[j], b = label[ltgt[p]];
            hptr[std::min(a, b) + 1] += 1;
        }
    for (I k = 0; k < n; ++k) hptr[k + 1] += hptr[k];
    htgt.assign(hptr[n], 0);
    {
        std::vector<I> pos(hptr.begin(), hptr.end() - 1);
        for (I j = 0; j < n; ++j)
            for (I p = lptr[j]; p < lptr[j + 1]; ++p) {
                I a = label[j], b = label[ltgt[p]];
                htgt[pos[std::min(a, b)]++] = std::max(a, b);
            }
    }

    // supernode children lists (ascending, roots in list h)
    std::vector<I> chdptr, chdtgt;
    children_lists(h, pnt, chdptr, chdtgt);

    // separators (cliquetree_impl!): adjacency of the first residual column
    // merged with the children's separators, all restricted to labels past
    // the residual.
    std::vector<I> sepptr(h + 1, 0);
    for (I i = 0; i < h; ++i) sepptr[i + 1] = sepptr[i] + seplen[i];
    std::vector<I> septgt(sepptr[h]);
    std::vector<I> cache;
    cache.reserve(n);
    for (I j = 0; j < h; ++j) {
        I q0 = resptr[j], q1 = resptr[j + 1];
        I pstrt = sepptr[j];
        I p = pstrt;
        I r = hptr[q0], rstop = hptr[q0 + 1];
        while (r < rstop && htgt[r] < q1) ++r;
        while (r < rstop) {
            if (p >= sepptr[j + 1]) { g_err = "internal: separator overflow"; return -3; }
            septgt[p++] = htgt[r++];
        }
        I p1 = p;
        for (I c = chdptr[j]; c < chdptr[j + 1]; ++c) {
            I i = chdtgt[c];
            I a = pstrt, aend = p1;
            I b = sepptr[i], bend = sepptr[i + 1];
            while (b < bend && septgt[b] < q1) ++b;
            cache.clear();
            while (a < aend && b < bend) {
                I va = septgt[a], vb = septgt[b];
                if (va == vb) { cache.push_back(va); ++a; ++b; }
                else if (va < vb) { cache.push_back(va); ++a; }
                else { cache.push_back(vb); ++b; }
            }
            while (a < aend) cache.push_back(septgt[a++]);
            while (b < bend) cache.push_back(septgt[b++]);
            if ((I)cache.size() > seplen[j]) { g_err = "internal: separator overflow"; return -3; }
            for (size_t t = 0; t < cache.size(); ++t) septgt[pstrt + (I)t] = cache[t];
            p1 = pstrt + (I)cache.size();
        }
        if (p1 != sepptr[j + 1]) { g_err = "internal: separator size disagrees with column count"; return -3; }
    }

    // ChordalSymbolic(res, sep, tree) (chordal_symbolic.jl:302-378), 0-based
    std::vector<I> reltgt(sepptr[h]), idx(n), Dptr(h + 1), Lptr(h + 1);
    I jMptr = 1, jMval = 0, jNval = 0;
    I nMptr = 1, nMval = 0, nNval = 0, nFval = 0, Dp = 0, Lp = 0;
    for (I j = 0; j < h; ++j) {
        Dptr[j] = Dp; Lptr[j] = Lp;
        I nn = resptr[j + 1] - resptr[j];
        I na = sepptr[j + 1] - sepptr[j];
        I nj = nn + na;
        for (I w = resptr[j]; w < resptr[j + 1]; ++w) idx[w] = j;
        for (I c = chdptr[j]; c < chdptr[j + 1]; ++c) {
            I i = chdtgt[c];
            // position of each sep(i) row inside bag(j) = res(j) ++ sep(j)
            I q = 0;
            I w = resptr[j];
            for (I p = sepptr[i]; p < sepptr[i + 1]; ++p) {
                I v = septgt[p];
                while (w < v && q < nn - 1) { ++q; w = resptr[j] + q; }
                while (w < v) { ++q; w = septgt[sepptr[j] + q - nn]; }
                reltgt[p] = q;
            }
            I ma = sepptr[i + 1] - sepptr[i];
            jMptr -= 1; jMval -= ma * ma; jNval -= ma;
        }
        if (na > 0) {
            jMptr += 1; jMval += na * na; jNval += na;
            nMptr = std::max(nMptr, jMptr);
            nMval = std::max(nMval, jMval);
            nNval = std::max(nNval, jNval);
        }
        nFval = std::max(nFval, nj);
        Dp += nn * nn;
        Lp += nn * na;
    }
    Dptr[h] = Dp; Lptr[h] = Lp;

    S->resptr.swap(resptr);
    S->sepptr.swap(sepptr);
    S->septgt.swap(septgt);
    S->reltgt.swap(reltgt);
    S->pnt.swap(pnt);
    S->chdptr.swap(chdptr);
    S->chdtgt.swap(chdtgt);
    S->idx.swap(idx);
    S->Dptr.swap(Dptr);
    S->Lptr.swap(Lptr);
    S->nMptr = nMptr; S->nMval = nMval; S->nNval = nNval; S->nFval = nFval;
    return 0;
}

extern "C" int ct_symbolic_create(int64_t n, const int64_t* colptr, const int64_t* rowval,
                                  const int64_t* order, ct_symbolic** out) {
    if (!out || n < 0 || (n > 0 && (!colptr || !rowval || !order))) { g_err = "bad arguments"; return -1; }
    *out = nullptr;
    ct_symbolic* S = new (std::nothrow) ct_symbolic();
    if (!S) { g_err = "out of memory"; return -4; }
    int rc;
    try {
        rc = build(S, n, colptr, rowval, order);
    } catch (const std::bad_alloc&) {
        g_err = "out of memory"; rc = -4;
    }
    if (rc != 0) { delete S; return rc; }
    *out = S;
    return 0;
}

extern "C" void ct_symbolic_destroy(ct_symbolic* S) { delete S; }

extern "C" int ct_symbolic_sizes(const ct_symbolic* S, int64_t* out) {
    // out[0..7] = n, nfr, nsep (=len septgt), ndz, nlz, nMptr, nMval, nNval; out[8] = nFval
    if (!S || !out) return -1;
    out[0] = S->n; out[1] = S->nfr; out[2] = (int64_t)S->septgt.size();
    out[3] = S->Dptr.empty() ? 0 : S->Dptr.back();
    out[4] = S->Lptr.empty() ? 0 : S->Lptr.back();
    out[5] = S->nMptr; out[6] = S->nMval; out[7] = S->nNval; out[8] = S->nFval;
    return 0;
}

static void copy_out(const std::vector<I>& v, int64_t* dst) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(I));
}

extern "C" int ct_symbolic_arrays(const ct_symbolic* S, int64_t* order, int64_t* invp, int64_t* resptr,
                                  int64_t* sepptr, int64_t* septgt, int64_t* reltgt, int64_t* pnt,
                                  int64_t* chdptr, int64_t* chdtgt, int64_t* idx, int64_t* Dptr, int64_t* Lptr) {
    if (!S) return -1;
    copy_out(S->order, order); copy_out(S->invp, invp);
    copy_out(S->resptr, resptr); copy_out(S->sepptr, sepptr);
    copy_out(S->septgt, septgt); copy_out(S->reltgt, reltgt);
    copy_out(S->pnt, pnt); copy_out(S->chdptr, chdptr); copy_out(S->chdtgt, chdtgt);
    copy_out(S->idx, idx); copy_out(S->Dptr, Dptr); copy_out(S->Lptr, Lptr);
    return 0;
}

// ---------------------------------------------------------------------------
// Geometric nested dissection for regular grids.  The reference would call
// METIS (ext/MetisExt.jl:64) for a nested-dissection order; it is not
// available offline, so grid problems get an explicit order from recursive
// coordinate bisection, which the reference accepts as `alg = order`
// (src/elimination_algorithms.jl:776-779).
// Vertex (x, y, z) has id x + nx*(y + ny*z).  Separators are planes through
// the middle of the longest box side; leaves below `leaf` vertices are
// numbered in natural order.  Eliminated last = top separator.
// ---------------------------------------------------------------------------
namespace {
struct Box { I x0, x1, y0, y1, z0, z1; };
}

static void nd_box(I nx, I ny, const Box& b, I leaf, std::vector<I>& out, I& pos) {
    I sx = b.x1 - b.x0, sy = b.y1 - b.y0, sz = b.z1 - b.z0;
    if (sx <= 0 || sy <= 0 || sz <= 0) return;
    // iterative is unnecessary: recursion depth is O(log n)
    if (sx * sy * sz <= leaf || (sx <= 2 && sy <= 2 && sz <= 2)) {
        for (I z = b.z0; z < b.z1; ++z)
            for (I y = b.y0; y < b.y1; ++y)
                for (I x = b.x0; x < b.x1; ++x) out[pos++] = x + nx * (y + ny * z);
        return;
    }
    Box a = b, c = b, s = b;
    if (sx >= sy && sx >= sz) {
        I m = b.x0 + sx / 2;
        a.x1 = m; s.x0 = m; s.x1 = m + 1; c.x0 = m + 1;
    } else if (sy >= sz) {
        I m = b.y0 + sy / 2;
        a.y1 = m; s.y0 = m; s.y1 = m + 1; c.y0 = m + 1;
    } else {
        I m = b.z0 + sz / 2;
        a.z1 = m; s.z0 = m; s.z1 = m + 1; c.z0 = m + 1;
    }
    nd_box(nx, ny, a, leaf, out, pos);
    nd_box(nx, ny, c, leaf, out, pos);
    for (I z = s.z0; z < s.z1; ++z)
        for (I y = s.y0; y < s.y1; ++y)
            for (I x = s.x0; x < s.x1; ++x) out[pos++] = x + nx * (y + ny * z);
}

extern "C" int ct_grid_nd_order(int64_t nx, int64_t ny, int64_t nz, int64_t leaf, int64_t* order) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || !order) { g_err = "bad arguments"; return -1; }
    I n = nx * ny * nz;
    std::vector<I> out(n);
    I pos = 0;
    nd_box(nx, ny, Box{0, nx, 0, ny, 0, nz}, leaf < 1 ? 1 : leaf, out, pos);
    if (pos != n) { g_err = "internal: nd order incomplete"; return -3; }
    std::memcpy(order, out.data(), n * sizeof(I));
    return 0;
}
