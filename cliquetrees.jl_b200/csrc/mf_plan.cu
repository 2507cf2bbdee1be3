// Host-side plan: per-front device metadata, level schedule and the grouped
// work lists each kernel launch consumes.  Built once per sparsity pattern.
//
// The reference walks the fronts in postorder with one LIFO stack of update
// matrices (chol_impl!, src/Multifrontal.jl/src/cholesky.jl:361-392).  Here
// fronts are grouped by height in the tree: all fronts of one level depend
// only on lower levels, so each level is a handful of grouped launches.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>

#include "mf_internal.cuh"

namespace mf {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

std::recursive_mutex& device_mutex() {
    static std::recursive_mutex mu;
    return mu;
}
const char* last_error() { return g_last_error.c_str(); }

int cuda_fail(cudaError_t e, const char* where) {
    g_last_error = std::string(where) + ": " + cudaGetErrorString(e);
    return -3;
}

static inline int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Best-fit allocator over one device pool (offsets in elements).  Blocks
// are 32-element aligned; freed neighbours are coalesced.  Used to give the
// update matrices (and the forward-solve updates) of each front a slot that
// lives from the level that produces it to the level of its parent, so the
// pool holds only the live frontier instead of every front at once.
class PoolAllocator {
  public:
    int64_t alloc(int64_t size) {
        size = (size + 31) & ~int64_t(31);
        if (size == 0) return 0;
        auto it = by_size_.lower_bound({size, -1});
        if (it != by_size_.end()) {
            int64_t off = it->second, bsz = it->first;
            by_size_.erase(it);
            by_off_.erase(off);
            if (bsz > size) insert_free(off + size, bsz - size);
            return off;
        }
        // grow: extend a free block that touches the end, else append
        if (!by_off_.empty()) {
            auto last = std::prev(by_off_.end());
            if (last->first + last->second == top_) {
                int64_t off = last->first;
                by_size_.erase({last->second, off});
                by_off_.erase(last);
                top_ = off + size;
                return off;
            }
        }
        int64_t off = top_;
        top_ += size;
        return off;
    }
    void release(int64_t off, int64_t size) {
        size = (size + 31) & ~int64_t(31);
        if (size == 0) return;
        auto nx = by_off_.lower_bound(off);
        if (nx != by_off_.end() && nx->first == off + size) {
            size += nx->second;
            by_size_.erase({nx->second, nx->first});
            nx = by_off_.erase(nx);
        }
        if (nx != by_off_.begin()) {
            auto pv = std::prev(nx);
            if (pv->first + pv->second == off) {
                off = pv->first;
                size += pv->second;
                by_size_.erase({pv->second, pv->first});
                by_off_.erase(pv);
            }
        }
        insert_free(off, size);
    }
    int64_t high_water() const { return top_; }

  private:
    void insert_free(int64_t off, int64_t size) {
        by_off_[off] = size;
        by_size_.insert({size, off});
    }
    std::map<int64_t, int64_t> by_off_;
    std::set<std::pair<int64_t, int64_t>> by_size_;
    int64_t top_ = 0;
};

int build_plan(mf_handle* h, const int64_t* resptr, const int64_t* sepptr, const int64_t* septgt,
               const int64_t* reltgt, const int64_t* chdptr, const int64_t* chdtgt, const int64_t* Dptr,
               const int64_t* Lptr) {
    const int64_t nfr = h->nfr, n = h->n;
    // ---- validate the symbolic input (a corrupted pattern must not reach a kernel)
    if (resptr[0] != 0 || resptr[nfr] != n) { set_error("resptr does not cover 0..n"); return -2; }
    if (sepptr[0] != 0) { set_error("sepptr must start at 0"); return -2; }
    if (chdptr[0] != 0 || chdptr[nfr + 1] != nfr) { set_error("chdptr must cover nfr children"); return -2; }
    h->nsep = sepptr[nfr];
    std::vector<int32_t> parent(nfr, -1);
    for (int64_t j = 0; j < nfr; ++j) {
        if (resptr[j + 1] <= resptr[j]) { set_error("empty residual"); return -2; }
        if (sepptr[j + 1] < sepptr[j]) { set_error("sepptr not monotone"); return -2; }
        if (resptr[j + 1] - resptr[j] + sepptr[j + 1] - sepptr[j] > (int64_t)1 << 30) {
            set_error("front too large"); return -2;
        }
    }
    for (int64_t j = 0; j <= nfr; ++j) {
        if (chdptr[j + 1] < chdptr[j]) { set_error("chdptr not monotone"); return -2; }
        for (int64_t p = chdptr[j]; p < chdptr[j + 1]; ++p) {
            int64_t c = chdtgt[p];
            if (c < 0 || c >= nfr) { set_error("child index out of range"); return -2; }
            if (j < nfr && c >= j) { set_error("tree is not postordered (child >= parent)"); return -2; }
            if (parent[c] != -1) { set_error("front has two parents"); return -2; }
            parent[c] = (int32_t)(j < nfr ? j : -1);
        }
    }
    for (int64_t j = 0; j < nfr; ++j) {
        int64_t nn = resptr[j + 1] - resptr[j], na = sepptr[j + 1] - sepptr[j];
        int64_t prev = resptr[j + 1] - 1;
        for (int64_t p = sepptr[j]; p < sepptr[j + 1]; ++p) {
            if (septgt[p] <= prev || septgt[p] >= n) { set_error("separator rows not increasing past res"); return -2; }
            prev = septgt[p];
        }
        int64_t pj = parent[j];
        if (na > 0 && pj < 0) { set_error("root front with a separator"); return -2; }
        if (pj >= 0) {
            int64_t pn = resptr[pj + 1] - resptr[pj] + sepptr[pj + 1] - sepptr[pj];
            int64_t prevr = -1;
            for (int64_t p = sepptr[j]; p < sepptr[j + 1]; ++p) {
                int64_t r = reltgt[p];
                if (r <= prevr || r >= pn) { set_error("rel index outside the parent bag"); return -2; }
                // rel must point at the same global row in the parent's bag
                int64_t pnn = resptr[pj + 1] - resptr[pj];
                int64_t row = r < pnn ? resptr[pj] + r : septgt[sepptr[pj] + r - pnn];
                if (row != septgt[p]) { set_error("rel index does not match the parent's bag"); return -2; }
                prevr = r;
            }
        }
        if (Dptr[j + 1] - Dptr[j] != nn * nn || Lptr[j + 1] - Lptr[j] != nn * na) {
            set_error("Dptr/Lptr disagree with the front sizes"); return -2;
        }
        (void)nn;
    }
    h->ndz = Dptr[nfr];
    h->nlz = Lptr[nfr];
    h->h_resptr.assign(resptr, resptr + nfr + 1);
    h->h_sepptr.assign(sepptr, sepptr + nfr + 1);
    h->h_septgt.assign(septgt, septgt + sepptr[nfr]);
    h->h_Dptr.assign(Dptr, Dptr + nfr + 1);
    h->h_Lptr.assign(Lptr, Lptr + nfr + 1);

    // ---- execution fronts (relaxed amalgamation of last-child chains)
    //
    // The reference's maximal supernodes (supernode_types.jl:41-88) leave
    // long chains of thin fronts, each materialising an update matrix that
    // its parent immediately re-reads.  The GPU plan merges a front into its
    // parent when the front is the parent's last child (its columns end
    // where the parent's begin, so the merged residual stays contiguous) and
    // the merge adds few explicit zeros (the thresholds of CHOLMOD's relaxed
    // amalgamation).  Structural zeros of L stay exact zeros in floating
    // point, so every entry of the reference layout is still computed; the
    // merged panels are converted back to the reference's Dval/Lval layout
    // on download.  MF_AMALGAMATE=0 in the environment disables merging.
    std::vector<int32_t> exec_of(nfr, -1);
    struct EF { int32_t top; int64_t c0, c1, truth; };
    std::vector<EF> ef;
    ef.reserve(nfr);
    const char* env = getenv("MF_AMALGAMATE");
    const bool amalg = !(env && env[0] == '0');
    for (int64_t j = 0; j < nfr; ++j) {
        int64_t nn = resptr[j + 1] - resptr[j], na = sepptr[j + 1] - sepptr[j];
        int64_t truth = nn * (nn + 1) / 2 + nn * na;
        if (amalg && chdptr[j + 1] > chdptr[j]) {
            int64_t c = chdtgt[chdptr[j + 1] - 1];
            EF& E = ef[exec_of[c]];
            if (E.top == c && E.c1 == resptr[j]) {
                int64_t N = E.c1 - E.c0 + nn;
                int64_t merged = N * (N + 1) / 2 + N * na;
                int64_t tot = E.truth + truth;
                double z = (double)(merged - tot) / (double)merged;
                bool ok = (N <= 4) || (N <= 16 && z < 0.8) || (N <= 48 && z < 0.1) || (z < 0.05);
                if (ok) {
                    E.top = (int32_t)j;
                    E.c1 = resptr[j + 1];
                    E.truth = tot;
                    exec_of[j] = exec_of[c];
                    continue;
                }
            }
        }
        exec_of[j] = (int32_t)ef.size();
        ef.push_back(EF{(int32_t)j, resptr[j], resptr[j + 1], truth});
    }
    const int64_t nex = (int64_t)ef.size();
    h->nexec = nex;
    std::vector<int32_t> eparent(nex, -1);
    for (int64_t e = 0; e < nex; ++e) {
        int64_t pt = parent[ef[e].top];
        eparent[e] = pt < 0 ? -1 : exec_of[pt];
    }
    // children CSR of the execution tree (ascending)
    std::vector<int64_t> echdptr(nex + 1, 0);
    for (int64_t e = 0; e < nex; ++e)
        if (eparent[e] >= 0) echdptr[eparent[e] + 1]++;
    for (int64_t e = 0; e < nex; ++e) echdptr[e + 1] += echdptr[e];
    h->h_exec_chd.assign(std::max<int64_t>(echdptr[nex], 1), 0);
    {
        std::vector<int64_t> pos(echdptr.begin(), echdptr.end() - 1);
        for (int64_t e = 0; e < nex; ++e)
            if (eparent[e] >= 0) h->h_exec_chd[pos[eparent[e]]++] = (int32_t)e;
    }
    // position of a global row in the bag of execution front e
    auto bagpos = [&](int64_t e, int64_t row) -> int64_t {
        const EF& E = ef[e];
        if (row >= E.c0 && row < E.c1) return row - E.c0;
        const int64_t* s0 = septgt + sepptr[E.top];
        const int64_t* s1 = septgt + sepptr[E.top + 1];
        const int64_t* it = std::lower_bound(s0, s1, row);
        if (it == s1 || *it != row) return -1;
        return (E.c1 - E.c0) + (it - s0);
    };
    // rel of execution fronts (into the parent's bag), indexed like septgt
    h->h_exec_rel.assign(std::max<int64_t>(h->nsep, 1), -1);
    for (int64_t e = 0; e < nex; ++e) {
        if (eparent[e] < 0) continue;
        int64_t t = ef[e].top;
        for (int64_t p = sepptr[t]; p < sepptr[t + 1]; ++p) {
            int64_t q = bagpos(eparent[e], septgt[p]);
            if (q < 0) { set_error("internal: separator row missing from the parent bag"); return -3; }
            h->h_exec_rel[p] = (int32_t)q;
        }
    }
    // reference front -> rows of its block inside the execution panel
    h->h_sepmap.assign(std::max<int64_t>(h->nsep, 1), -1);
    h->h_ref.resize(nfr);
    for (int64_t j = 0; j < nfr; ++j) {
        int64_t e = exec_of[j];
        for (int64_t p = sepptr[j]; p < sepptr[j + 1]; ++p) {
            int64_t q = bagpos(e, septgt[p]);
            if (q < 0) { set_error("internal: reference separator row missing from its execution bag"); return -3; }
            h->h_sepmap[p] = (int32_t)q;
        }
        RefFront& r = h->h_ref[j];
        r.Dptr = Dptr[j];
        r.Lptr = Lptr[j];
        r.nn = (int32_t)(resptr[j + 1] - resptr[j]);
        r.na = (int32_t)(sepptr[j + 1] - sepptr[j]);
        r.res0 = (int32_t)resptr[j];
        r.sep0 = (int32_t)sepptr[j];
        r.exec = (int32_t)e;
    }
    h->h_exec_of = exec_of;

    // ---- execution fronts: levels and offsets
    h->h_fronts.resize(nex);
    int64_t poff = 0;
    int max_level = 0;
    std::vector<int32_t> level(nex, 0);
    for (int64_t e = 0; e < nex; ++e) {
        int64_t pe = eparent[e];
        if (pe >= 0) level[pe] = std::max(level[pe], level[e] + 1);
    }
    int64_t ioff = 0, ioff2 = 0;
    for (int64_t e = 0; e < nex; ++e) {
        Front& f = h->h_fronts[e];
        int64_t t = ef[e].top;
        int64_t nn = ef[e].c1 - ef[e].c0, na = sepptr[t + 1] - sepptr[t];
        f.nn = (int32_t)nn; f.na = (int32_t)na;
        f.col0 = (int32_t)ef[e].c0;
        f.sep0 = (int32_t)sepptr[t];
        f.chd0 = (int32_t)echdptr[e]; f.chd1 = (int32_t)echdptr[e + 1];
        f.parent = eparent[e];
        f.level = level[e];
        f.ldp = (int32_t)((nn + na + 3) & ~int64_t(3));
        f.ldm = (int32_t)((na + 3) & ~int64_t(3));
        f.poff = poff; poff += (int64_t)f.ldp * nn;
        f.moff = 0;
        f.roff = 0;
        f.ioff = 0;
        if (nn + na > kSmallMax) { f.ioff = ioff; ioff += cdiv(nn, kNB) * kNB * kNB; }
        f.i2off = -1;
        if (!solve_small(f)) {
            const int64_t nK = cdiv(nn, kSolveNB), wL = nn - (nK - 1) * kSolveNB;
            f.i2off = ioff2;
            ioff2 += (nK - 1) * kSolveNB * kSolveNB + (int64_t)super_ld((int)wL) * wL;
        }
        max_level = std::max(max_level, level[e]);
    }
    h->npanel = poff;
    h->ninv = ioff;
    h->ninv2 = ioff2;
    // ---- subtrees of small fronts solved in one launch per direction
    // (k_s_sub_fwd / k_s_sub_bwd).  A front heads a task subtree when it
    // and all its descendants are solve-small, the subtree's cost (one unit
    // per front plus its panel entries / 256) is at most wmax, and its
    // parent's subtree is not such a subtree; consecutive heads are packed
    // into one task up to wmax.  wmax spreads the small part of the forest
    // over about 16 tasks per SM (148 SMs), at least 48 units.
    // Opt-in (MF_SUBTREE_SOLVE=1 in the environment): measured slower than
    // the per-level launches on the 80^3, 100^2 and batched 2D workloads --
    // a task's narrow levels leave most of its warps idle, while a level
    // launch keeps every front of the level in flight.
    std::vector<int32_t> task_of(nex, -1);
    std::vector<std::vector<int32_t>> task_heads;
    const char* stenv = getenv("MF_SUBTREE_SOLVE");
    if (stenv && stenv[0] == '1') {
        std::vector<char> allsmall(nex, 0);
        std::vector<double> cost(nex, 0.0);
        for (int L = 0; L <= max_level; ++L)
            for (int64_t e = 0; e < nex; ++e) {
                if (level[e] != L) continue;
                const Front& f = h->h_fronts[e];
                bool ok = solve_small(f);
                double c = 1.0 + (double)(f.nn + f.na) * f.nn / 256.0;
                for (int32_t p = f.chd0; p < f.chd1; ++p) {
                    const int32_t ch = h->h_exec_chd[(size_t)p];
                    ok = ok && allsmall[ch];
                    c += cost[ch];
                }
                allsmall[e] = ok;
                cost[e] = c;
            }
        double tot = 0.0;
        for (int64_t e = 0; e < nex; ++e)
            if (allsmall[e] && (eparent[e] < 0 || !allsmall[eparent[e]])) tot += cost[e];
        const double wmax = std::max(48.0, tot / (148.0 * 16.0));
        auto fits = [&](int64_t e) { return allsmall[e] && cost[e] <= wmax; };
        double acc = 0.0;
        for (int64_t e = 0; e < nex; ++e) {
            if (!fits(e) || (eparent[e] >= 0 && fits(eparent[e]))) continue;
            if (task_heads.empty() || acc + cost[e] > wmax) {
                task_heads.emplace_back();
                acc = 0.0;
            }
            task_heads.back().push_back((int32_t)e);
            acc += cost[e];
        }
        for (size_t t = 0; t < task_heads.size(); ++t) {
            std::vector<int32_t> stack(task_heads[t].begin(), task_heads[t].end());
            while (!stack.empty()) {
                const int32_t e = stack.back();
                stack.pop_back();
                task_of[e] = (int32_t)t;
                const Front& f = h->h_fronts[e];
                for (int32_t p = f.chd0; p < f.chd1; ++p) stack.push_back(h->h_exec_chd[(size_t)p]);
            }
        }
    }
    {
        // slot lifetimes: produced at level(e), read while level(parent(e))
        // is processed, reusable from the next level on.  The solve's update
        // blocks of task fronts live in a region of their own per task (its
        // CTA walks the task's levels at its own pace, concurrently with the
        // other tasks), reused inside the task by the same rule; a head's
        // block stays until its parent reads it.
        std::vector<std::vector<int32_t>> born(max_level + 1), dies(max_level + 1);
        for (int64_t e = 0; e < nex; ++e) {
            if (h->h_fronts[e].na == 0) continue;
            born[level[e]].push_back((int32_t)e);
            dies[level[eparent[e]]].push_back((int32_t)e);
        }
        PoolAllocator pm, pr;
        std::vector<PoolAllocator> ptask(task_heads.size());
        for (int L = 0; L <= max_level; ++L) {
            for (int32_t e : born[L]) {
                Front& f = h->h_fronts[e];
                f.moff = pm.alloc((int64_t)f.ldm * f.na);
                const int32_t t = task_of[e];
                f.roff = t < 0 ? pr.alloc((int64_t)f.na) : ptask[(size_t)t].alloc((int64_t)f.na);
            }
            for (int32_t e : dies[L]) {
                Front& f = h->h_fronts[e];
                pm.release(f.moff, (int64_t)f.ldm * f.na);
                const int32_t t = task_of[e];
                if (t < 0) pr.release(f.roff, (int64_t)f.na);
                else if (task_of[eparent[e]] == t) ptask[(size_t)t].release(f.roff, (int64_t)f.na);
            }
        }
        h->nmval = pm.high_water();
        int64_t rbase = pr.high_water();
        std::vector<int64_t> tbase(task_heads.size());
        for (size_t t = 0; t < task_heads.size(); ++t) {
            tbase[t] = rbase;
            rbase += ptask[t].high_water();
        }
        for (int64_t e = 0; e < nex; ++e)
            if (task_of[e] >= 0 && h->h_fronts[e].na > 0) h->h_fronts[e].roff += tbase[(size_t)task_of[e]];
        h->nrval_per_rhs = rbase;
    }

    // ---- work lists
    h->levels.assign(max_level + 1, Level());
    std::vector<std::vector<int32_t>> by_level(max_level + 1);
    for (int64_t e = 0; e < nex; ++e) by_level[level[e]].push_back((int32_t)e);
    std::vector<Item>& items = h->h_items;
    items.clear();
    auto begin = [&](ItemList& l) { l.off = (int64_t)items.size(); };
    auto end = [&](ItemList& l) { l.cnt = (int64_t)items.size() - l.off; };
    auto push = [&](int32_t f, int32_t a, int32_t b) { items.push_back(Item{f, a, b, 0}); };
    std::vector<Item> easeg; // extend-add segments, appended after them

    // the 32-row warp-per-front factor measured slower than k_small with its
    // per-level sizing (2D batch and 100^2 grid), so it is opt-in
    const char* w32env = getenv("MF_WARP_FRONT32");
    const bool warp32 = w32env && w32env[0] == '1';
    for (int L = 0; L <= max_level; ++L) {
        Level& lv = h->levels[L];
        const std::vector<int32_t>& fr = by_level[L];
        // factorization
        begin(lv.small_warp);
        for (int32_t j : fr) {
            const Front& f = h->h_fronts[j];
            if (f.nn + f.na <= kWarpSmallNJ) push(j, 0, 0);
        }
        end(lv.small_warp);
        begin(lv.small_warp2);
        for (int32_t j : fr) {
            const Front& f = h->h_fronts[j];
            if (warp32 && f.nn + f.na > kWarpSmallNJ && f.nn + f.na <= kWarpSmallNJ2) push(j, 0, 0);
        }
        end(lv.small_warp2);
        begin(lv.small);
        for (int32_t j : fr) {
            const Front& f = h->h_fronts[j];
            if (f.nn + f.na > (warp32 ? kWarpSmallNJ2 : kWarpSmallNJ) && f.nn + f.na <= kSmallMax) {
                push(j, 0, 0);
                lv.small_maxnj = std::max(lv.small_maxnj, f.nn + f.na);
            }
        }
        end(lv.small);
        int max_steps = 0;
        for (int part = 0; part < 2; ++part) {
            ItemList& el = part ? lv.ea_upd : lv.ea;
            begin(el);
            for (int32_t j : fr) {
                const Front& f = h->h_fronts[j];
                const int nj = f.nn + f.na;
                if (nj <= kSmallMax) continue;
                if (!part) {
                    max_steps = std::max<int>(max_steps, (int)cdiv(f.nn, kNB));
                    lv.max_nn_blocked = std::max(lv.max_nn_blocked, f.nn);
                }
                const int nch = f.chd1 - f.chd0;
                if (nch == 0) continue;
                for (int t = 0; t < cdiv(nj, kEAcols); ++t) {
                    const int c0 = t * kEAcols, c1 = std::min(c0 + kEAcols, nj);
                    const int pc0 = part ? std::max(c0, f.nn) : c0, pc1 = part ? c1 : std::min(c1, f.nn);
                    if (pc0 >= pc1) continue;
                    for (int q = 0; pc0 + q * kEArows < nj; ++q) {
                        const int r0 = pc0 + q * kEArows, r1 = std::min(r0 + kEArows, nj);
                        std::vector<Item> segs;
                        bool any = false;
                        for (int32_t pp = f.chd1 - 1; pp >= f.chd0; --pp) {
                            const int32_t c = h->h_exec_chd[(size_t)pp];
                            const Front& fc = h->h_fronts[(size_t)c];
                            const int32_t* rel = h->h_exec_rel.data() + fc.sep0;
                            const int32_t* rend = rel + fc.na;
                            const int b0 = (int)(std::lower_bound(rel, rend, pc0) - rel);
                            const int b1 = (int)(std::lower_bound(rel, rend, pc1) - rel);
                            const int a0 = (int)(std::lower_bound(rel, rend, r0) - rel);
                            const int a1 = (int)(std::lower_bound(rel, rend, r1) - rel);
                            // rows a >= b of a child column b (lower triangle)
                            if (b0 < b1 && a1 > std::max(a0, b0)) any = true;
                            segs.push_back(Item{c, b0, b1, 0});
                            segs.push_back(Item{a0, a1, 0, 0});
                        }
                        if (!any) continue;
                        items.push_back(Item{j, t, q, (int32_t)easeg.size()});
                        easeg.insert(easeg.end(), segs.begin(), segs.end());
                    }
                }
            }
            end(el);
        }
        // two-level blocking: outer blocks of kob columns, sub-panels of kNB;
        // levels with a very large front take wider outer blocks (trailing
        // updates with a longer K amortise the tile overheads)
        {
            const char* wenv = getenv("MF_WIDE_FRONT_NN");
            const int wide_nn = wenv ? atoi(wenv) : kWideFrontNN;
            lv.kob = (wide_nn > 0 && lv.max_nn_blocked >= wide_nn) ? kOBWide : kOB;
        }
        const int kob = lv.kob;
        for (int ob = 0; ob * kob < lv.max_nn_blocked; ++ob) {
            for (int sp = 0; sp < kob / kNB; ++sp) {
                const int c0 = ob * kob + sp * kNB;
                if (c0 >= lv.max_nn_blocked) break;
                PanelStep st;
                st.b = ob; st.s = sp;
                begin(st.left);
                if (sp > 0)
                    for (int32_t j : fr) {
                        const Front& f = h->h_fronts[j];
                        if (f.nn + f.na <= kSmallMax || f.nn <= c0) continue;
                        for (int t = 0; t < (int)cdiv(f.nn + f.na - c0, kTile); ++t) push(j, t, 0);
                    }
                end(st.left);
                begin(st.diag);
                for (int32_t j : fr) {
                    const Front& f = h->h_fronts[j];
                    if (f.nn + f.na <= kSmallMax || f.nn <= c0) continue;
                    push(j, 0, 0);
                }
                end(st.diag);
                begin(st.panel);
                for (int32_t j : fr) {
                    const Front& f = h->h_fronts[j];
                    if (f.nn + f.na <= kSmallMax || f.nn <= c0) continue;
                    int w = std::min(kNB, f.nn - c0);
                    for (int t = 0; t < (int)cdiv(f.nn + f.na - c0 - w, kTile); ++t) push(j, t, 0);
                }
                end(st.panel);
                // trailing update: first the tiles of the next outer block's
                // columns (what its sub-panels wait for), then the rest
                // (st.trail_ncrit / trail_tc_ncrit count the first part)
                begin(st.trail);
                const bool last_sub = (sp == kob / kNB - 1) || (c0 + kNB >= lv.max_nn_blocked);
                if (last_sub)
                    for (int part = 0; part < 2; ++part)
                        for (int32_t j : fr) {
                            const Front& f = h->h_fronts[j];
                            if (f.nn + f.na <= kSmallMax || f.nn <= ob * kob) continue;
                            const int e = std::min(f.nn, (ob + 1) * kob);
                            if (e >= f.nn) continue;  // no panel columns after this outer block
                            const int nj = f.nn + f.na;
                            for (int tj = 0; tj < (int)cdiv(f.nn - e, kTile); ++tj) {
                                if ((tj < kob / kTile) != (part == 0)) continue;
                                const int cs = e + tj * kTile;
                                for (int ti = 0; ti < (int)cdiv(nj - cs, kTile); ++ti) push(j, ti, tj);
                            }
                            if (part == 0) st.trail_ncrit = (int64_t)items.size() - st.trail.off;
                        }
                end(st.trail);
                // 128-row tiles for the tcgen05 kernels
                begin(st.left_tc);
                if (sp > 0)
                    for (int32_t j : fr) {
                        const Front& f = h->h_fronts[j];
                        if (f.nn + f.na <= kSmallMax || f.nn <= c0) continue;
                        for (int t = 0; t < (int)cdiv(f.nn + f.na - c0, kTM); ++t) push(j, t, 0);
                    }
                end(st.left_tc);
                begin(st.panel_tc);
                for (int32_t j : fr) {
                    const Front& f = h->h_fronts[j];
                    if (f.nn + f.na <= kSmallMax || f.nn <= c0) continue;
                    // rows from the 4-aligned row at or before the first one below the block
                    const int r0 = (c0 + std::min(kNB, f.nn - c0)) & ~3;
                    for (int t = 0; t < (int)cdiv(f.nn + f.na - r0, kTM); ++t) push(j, t, 0);
                }
                end(st.panel_tc);
                begin(st.trail_tc);
                std::vector<Item> split;
                int64_t units = 0;
                if (last_sub) {
                    std::vector<int64_t> ubase(fr.size(), -1);
                    for (size_t i = 0; i < fr.size(); ++i) {
                        const int32_t j = fr[i];
                        const Front& f = h->h_fronts[j];
                        if (f.nn + f.na <= kSmallMax || f.nn <= ob * kob) continue;
                        const int e = std::min(f.nn, (ob + 1) * kob);
                        if (e >= f.nn) continue;
                        const int nj = f.nn + f.na;
                        // split operand units of rows [e, nj) x columns [ob*kob, e)
                        const int nrb = (int)cdiv(nj - e, kSplitRows), nkc = (int)cdiv(e - ob * kob, kSplitK);
                        for (int rb = 0; rb < nrb; ++rb)
                            for (int kc = 0; kc < nkc; ++kc) split.push_back(Item{j, rb, kc, (int32_t)units});
                        ubase[i] = units;
                        units += (int64_t)nrb * nkc * (h->diag ? 2 : 1);
                    }
                    for (int part = 0; part < 2; ++part) {
                        for (size_t i = 0; i < fr.size(); ++i) {
                            if (ubase[i] < 0) continue;
                            const int32_t j = fr[i];
                            const Front& f = h->h_fronts[j];
                            const int e = std::min(f.nn, (ob + 1) * kob);
                            const int nj = f.nn + f.na;
                            for (int tj = 0; tj < (int)cdiv(f.nn - e, kTcTrailN); ++tj) {
                                if ((tj < kob / kTcTrailN) != (part == 0)) continue;
                                const int cs = e + tj * kTcTrailN;
                                // rows from the first 128-aligned tile that reaches the diagonal
                                for (int ti = 0; ti < (int)cdiv(nj - cs, kTM); ++ti)
                                    items.push_back(Item{j, ti, tj, (int32_t)ubase[i]});
                            }
                        }
                        if (part == 0) st.trail_tc_ncrit = (int64_t)items.size() - st.trail_tc.off;
                    }
                }
                end(st.trail_tc);
                begin(st.split_tc);
                items.insert(items.end(), split.begin(), split.end());
                end(st.split_tc);
                h->nsplit_units = std::max(h->nsplit_units, units);
                lv.steps.push_back(st);
            }
        }
        (void)max_steps;
        begin(lv.syrk);
        for (int32_t j : fr) {
            const Front& f = h->h_fronts[j];
            if (f.nn + f.na <= kSmallMax || f.na == 0) continue;
            int t = (int)cdiv(f.na, kTile);
            for (int tj = 0; tj < t; ++tj)
                for (int ti = tj; ti < t; ++ti) push(j, ti, tj);
        }
        end(lv.syrk);
        begin(lv.syrk_tc);
        std::vector<Item> ssplit;
        int64_t sunits = 0;
        for (int32_t j : fr) {
            const Front& f = h->h_fronts[j];
            if (f.nn + f.na <= kSmallMax || f.na == 0) continue;
            // tiles start at the 4-aligned panel row nn & ~3, delta rows before L21
            const int delta = f.nn & 3;
            const int tcn = (int)cdiv(f.na + delta, kTcSyrkN);
            for (int tj = 0; tj < tcn; ++tj)
                // 128-row tiles from the diagonal: L21 rows tj * N - delta + 128 ti
                for (int ti = 0; ti < (int)cdiv(f.na + delta - tj * kTcSyrkN, kTM); ++ti)
                    items.push_back(Item{j, ti, tj, (int32_t)sunits});
            // split operand units of rows [nn & ~3, nj) x columns [0, nn)
            const int nrb = (int)cdiv(f.na + delta, kSplitRows), nkc = (int)cdiv(f.nn, kSplitK);
            for (int rb = 0; rb < nrb; ++rb)
                for (int kc = 0; kc < nkc; ++kc) ssplit.push_back(Item{j, rb, kc, (int32_t)sunits});
            sunits += (int64_t)nrb * nkc * (h->diag ? 2 : 1);
        }
        end(lv.syrk_tc);
        begin(lv.split_syrk);
        items.insert(items.end(), ssplit.begin(), ssplit.end());
        end(lv.split_syrk);
        h->nsplit_units = std::max(h->nsplit_units, sunits);

        // solves: small fronts (solve_small) one warp each; blocked fronts in
        // 256-column super-block steps using the super-block inverses
        begin(lv.s_small);
        for (int32_t j : fr) {
            const Front& f = h->h_fronts[j];
            if (solve_small(f) && task_of[j] < 0 && f.nn + f.na > kTinyNJ2) push(j, 0, 0);
        }
        end(lv.s_small);
        begin(lv.s_tiny);
        for (int32_t j : fr) {
            const Front& f = h->h_fronts[j];
            if (solve_small(f) && task_of[j] < 0 && f.nn + f.na <= kTinyNJ) push(j, 0, 0);
        }
        end(lv.s_tiny);
        begin(lv.s_tiny2);
        for (int32_t j : fr) {
            const Front& f = h->h_fronts[j];
            const int nj = f.nn + f.na;
            if (solve_small(f) && task_of[j] < 0 && nj > kTinyNJ && nj <= kTinyNJ2) push(j, 0, 0);
        }
        end(lv.s_tiny2);
        // forward gather: item (front, row tile, first row pointer of the
        // front, 0).  Row q of a blocked front owns the list of the children's
        // update rows that land on it, children in reverse order (the order
        // the reference adds them): h_grow[base + q] .. h_grow[base + q + 1]
        // index h_gcon, one record (child roff, child row, child na) each
        begin(lv.s_gather);
        int max_sblocks = 0;
        int64_t max_l21 = 0;
        std::vector<int32_t> gfirst;  // per blocked front of the level: its first gather item
        for (int32_t j : fr) {
            const Front& f = h->h_fronts[j];
            if (solve_small(f)) continue;
            const int nj = f.nn + f.na;
            const int nt = (int)cdiv(nj, kSolveRows);
            gfirst.push_back((int32_t)items.size());
            max_l21 = std::max<int64_t>(max_l21, (int64_t)f.nn * f.na);
            std::vector<int32_t> cnt((size_t)nj + 1, 0);
            for (int32_t p = f.chd1 - 1; p >= f.chd0; --p) {
                const Front& fc = h->h_fronts[(size_t)h->h_exec_chd[(size_t)p]];
                const int32_t* rel = h->h_exec_rel.data() + fc.sep0;
                for (int a = 0; a < fc.na; ++a) cnt[(size_t)rel[a] + 1] += 1;
            }
            const int64_t base = (int64_t)h->h_grow.size(), c0 = (int64_t)h->h_gcon.size();
            if (base + nj + 1 > INT32_MAX) {
                set_error("plan: too many gather rows");
                return -3;
            }
            std::vector<int64_t> at((size_t)nj);
            int64_t run = c0;
            for (int q = 0; q <= nj; ++q) {
                run += cnt[(size_t)q];
                h->h_grow.push_back(run);
                if (q < nj) at[(size_t)q] = run;
            }
            h->h_gcon.resize((size_t)run);
            for (int32_t p = f.chd1 - 1; p >= f.chd0; --p) {
                const Front& fc = h->h_fronts[(size_t)h->h_exec_chd[(size_t)p]];
                const int32_t* rel = h->h_exec_rel.data() + fc.sep0;
                for (int a = 0; a < fc.na; ++a)
                    h->h_gcon[(size_t)at[(size_t)rel[a]]++] = GCon{fc.roff, a, fc.na};
            }
            for (int t = 0; t < nt; ++t) items.push_back(Item{j, t, (int32_t)base, 0});
            max_sblocks = std::max<int>(max_sblocks, (int)cdiv(f.nn, kSolveNB));
        }
        end(lv.s_gather);
        lv.s_steps.resize(max_sblocks);
        for (int k = 0; k < max_sblocks; ++k) {
            SolveStep& st = lv.s_steps[k];
            const int k0 = k * kSolveNB;
            begin(st.diag);
            for (int32_t j : fr) {
                const Front& f = h->h_fronts[j];
                if (solve_small(f) || f.nn <= k0) continue;
                push(j, 0, 0);
            }
            end(st.diag);
            begin(st.fwd);
            for (int32_t j : fr) {
                const Front& f = h->h_fronts[j];
                if (solve_small(f) || f.nn <= k0) continue;
                const int w = std::min(kSolveNB, f.nn - k0);
                // 64-row tiles of the diagonal block's rows below the super-block,
                // from the 4-aligned row at or before the first of them (the
                // L21 rows are updated once per level by s_fwd_l)
                const int below = f.nn - ((k0 + w) & ~3);
                if (f.nn > k0 + w)
                    for (int t = 0; t < (int)cdiv(below, kFwdRows); ++t) push(j, t, 0);
            }
            end(st.fwd);
            begin(st.bwd);
            for (int32_t j : fr) {
                const Front& f = h->h_fronts[j];
                if (solve_small(f) || f.nn <= k0) continue;
                for (int t = 0; t < (int)cdiv(k0, kNB); ++t) push(j, t, 0);
            }
            end(st.bwd);
        }
        // the same chain as k_s_chain items: per step K, kDiagSplit diagonal
        // parts of every front, then the tiles, the ones the next diagonal
        // step waits for first (forward: the rows just below the super-block;
        // backward: the columns just left of it).  Each front gets a
        // counter block per direction: [finished diagonal parts, steps applied
        // to each 64-row / 64-column tile of its diagonal block].
        if (max_sblocks > 0) {
            lv.chain_tk = h->nchain;
            h->nchain += 2;
            std::vector<int32_t> bf;
            for (int32_t j : fr)
                if (!solve_small(h->h_fronts[j])) bf.push_back(j);
            std::vector<int32_t> cbf(bf.size()), cbb(bf.size());
            for (size_t i = 0; i < bf.size(); ++i) {
                cbf[i] = (int32_t)h->nchain;
                h->nchain += 1 + cdiv(h->h_fronts[bf[i]].nn, kNB);
            }
            for (size_t i = 0; i < bf.size(); ++i) {
                cbb[i] = (int32_t)h->nchain;
                h->nchain += 1 + cdiv(h->h_fronts[bf[i]].nn, kNB);
            }
            const int nsplit = kSolveNB / 16;
            auto fwd_tiles = [&](const Front& f, int k0) {
                const int w = std::min(kSolveNB, f.nn - k0);
                return f.nn > k0 + w ? (int)cdiv(f.nn - ((k0 + w) & ~3), kFwdRows) : 0;
            };
            // Ticket order D(0) C(0) D(1) B(0) C(1) D(2) B(1) ...: D(k) the
            // diagonal parts of step k, C(k) its four tiles of the next
            // super-block (what D(k + 1) waits for), B(k) its other tiles.  The
            // next step's diagonal parts come right after the tiles they wait
            // for instead of behind the step's bulk, and every item still
            // waits only on smaller tickets (C(k + 1) on B(k) and D(k + 1)).
            auto diag_parts = [&](int k) {
                for (size_t i = 0; i < bf.size(); ++i)
                    if (h->h_fronts[bf[i]].nn > k * kSolveNB)
                        for (int q = 0; q < nsplit; ++q) items.push_back(Item{bf[i], -1 - q, k, cbf[i]});
            };
            auto fwd_range = [&](int k, int t0, int t1) {
                const int k0 = k * kSolveNB;
                int maxt = 0;
                for (size_t i = 0; i < bf.size(); ++i)
                    if (h->h_fronts[bf[i]].nn > k0) maxt = std::max(maxt, fwd_tiles(h->h_fronts[bf[i]], k0));
                for (int t = t0; t < std::min(t1, maxt); ++t)
                    for (size_t i = 0; i < bf.size(); ++i) {
                        const Front& f = h->h_fronts[bf[i]];
                        if (f.nn > k0 && t < fwd_tiles(f, k0)) items.push_back(Item{bf[i], t, k, cbf[i]});
                    }
            };
            begin(lv.s_chain_f);
            diag_parts(0);
            for (int k = 0; k < max_sblocks; ++k) {
                fwd_range(k, 0, 4);                                   // C(k)
                if (k + 1 < max_sblocks) diag_parts(k + 1);           // D(k + 1)
                fwd_range(k, 4, INT32_MAX);                           // B(k)
            }
            end(lv.s_chain_f);
            auto bdiag_parts = [&](int k) {
                for (size_t i = 0; i < bf.size(); ++i)
                    if (h->h_fronts[bf[i]].nn > k * kSolveNB)
                        for (int q = 0; q < nsplit; ++q) items.push_back(Item{bf[i], -1 - q, k, cbb[i]});
            };
            // tiles t1 - 1 down to t0 of step k (columns left of super-block k)
            auto bwd_range = [&](int k, int t0, int t1) {
                const int k0 = k * kSolveNB;
                for (int t = t1 - 1; t >= std::max(t0, 0); --t)
                    for (size_t i = 0; i < bf.size(); ++i)
                        if (h->h_fronts[bf[i]].nn > k0) items.push_back(Item{bf[i], t, k, cbb[i]});
            };
            begin(lv.s_chain_b);
            bdiag_parts(max_sblocks - 1);
            for (int k = max_sblocks - 1; k >= 0; --k) {
                const int nt = (int)cdiv(k * kSolveNB, kNB);
                bwd_range(k, nt - 4, nt);                             // C(k)
                if (k > 0) bdiag_parts(k - 1);                        // D(k - 1)
                bwd_range(k, 0, nt - 4);                              // B(k)
            }
            end(lv.s_chain_b);
            if (h->nchain > INT32_MAX) {
                set_error("plan: too many solve-chain counters");
                return -3;
            }
        }
        // forward R -= L21 x1 of the blocked fronts: items (front, 64-row tile of
        // L21 from the 4-aligned row at or before nn, 512-column chunk, slot),
        // then one reduction item per row tile adding the chunks in order
        begin(lv.s_fwd_l);
        int32_t fslot = 0;
        std::vector<Item> fred;
        for (int32_t j : fr) {
            const Front& f = h->h_fronts[j];
            if (solve_small(f) || f.na == 0) continue;
            const int rows = f.nn + f.na - (f.nn & ~3);
            const int nchunk = (int)cdiv(f.nn, kFwdCols);
            for (int t = 0; t < (int)cdiv(rows, kFwdRows); ++t) {
                fred.push_back(Item{j, t, fslot, nchunk});
                for (int q = 0; q < nchunk; ++q) items.push_back(Item{j, t, q, fslot++});
            }
        }
        end(lv.s_fwd_l);
        begin(lv.s_fwd_red);
        for (const Item& r : fred) items.push_back(r);
        end(lv.s_fwd_red);
        h->nbwd_part = std::max<int64_t>(h->nbwd_part, fslot);
        begin(lv.s_bwd_l);
        int32_t slot = 0;
        std::vector<Item> red;
        std::vector<int32_t> bfirst;  // per blocked front of the level: its first partial slot
        for (int32_t j : fr) {
            const Front& f = h->h_fronts[j];
            if (solve_small(f)) continue;
            bfirst.push_back(slot);
            const int nchunk = std::max<int>(1, (int)cdiv(f.na, kBwdRows));
            for (int t = 0; t < cdiv(f.nn, kNB); ++t) {
                red.push_back(Item{j, t, slot, 0});
                for (int q = 0; q < nchunk; ++q) items.push_back(Item{j, t, q, slot++});
            }
        }
        end(lv.s_bwd_l);
        h->nbwd_part = std::max<int64_t>(h->nbwd_part, slot);
        begin(lv.s_bwd_red);
        for (const Item& r : red) items.push_back(r);
        end(lv.s_bwd_red);
        // single-super-block levels with short L21s: one cluster per blocked
        // front (the gather items' segment offsets are made absolute below;
        // the mid items point at the gather items themselves)
        begin(lv.s_mid);
        if (max_sblocks == 1 && max_l21 <= kMidMaxL21) {
            size_t i = 0;
            for (int32_t j : fr) {
                const Front& f = h->h_fronts[j];
                if (solve_small(f)) continue;
                items.push_back(Item{j, gfirst[i], bfirst[i], (int32_t)cdiv(f.nn + f.na, kSolveRows)});
                ++i;
            }
        }
        end(lv.s_mid);
    }
    // task lists: task items {first level item, end}, level items {first
    // front item, end, height}, front items {front}; fronts of a task sorted
    // by height (a front's height exceeds its children's)
    {
        const int64_t ntask = (int64_t)task_heads.size();
        std::vector<std::vector<int32_t>> members((size_t)ntask);
        for (int64_t e = 0; e < nex; ++e)
            if (task_of[e] >= 0) members[(size_t)task_of[e]].push_back((int32_t)e);
        std::vector<Item> tlev, tfr;
        std::vector<Item> tasks((size_t)ntask);
        for (int64_t t = 0; t < ntask; ++t) {
            std::vector<int32_t>& m = members[(size_t)t];
            std::stable_sort(m.begin(), m.end(), [&](int32_t a, int32_t b) { return level[a] < level[b]; });
            tasks[(size_t)t].front = (int32_t)tlev.size();
            size_t i = 0;
            while (i < m.size()) {
                size_t k = i;
                while (k < m.size() && level[m[k]] == level[m[i]]) ++k;
                tlev.push_back(Item{(int32_t)tfr.size(), (int32_t)(tfr.size() + (k - i)), level[m[i]], 0});
                for (size_t q = i; q < k; ++q) tfr.push_back(Item{m[q], 0, 0, 0});
                i = k;
            }
            tasks[(size_t)t].a = (int32_t)tlev.size();
        }
        // absolute item indices: tasks, then levels, then fronts
        const int64_t tb = (int64_t)items.size(), lb = tb + ntask, fb = lb + (int64_t)tlev.size();
        if (fb + (int64_t)tfr.size() > INT32_MAX) {
            set_error("plan: too many work items");
            return -3;
        }
        for (Item& t : tasks) { t.front += (int32_t)lb; t.a += (int32_t)lb; }
        for (Item& l : tlev) { l.front += (int32_t)fb; l.a += (int32_t)fb; }
        h->sub_tasks.off = tb;
        h->sub_tasks.cnt = ntask;
        items.insert(items.end(), tasks.begin(), tasks.end());
        items.insert(items.end(), tlev.begin(), tlev.end());
        items.insert(items.end(), tfr.begin(), tfr.end());
    }
    {
        const int64_t ebase = (int64_t)items.size();
        if (ebase + (int64_t)easeg.size() > INT32_MAX) {
            set_error("plan: too many work items");
            return -3;
        }
        for (const Level& lv : h->levels)
            for (const ItemList* el : {&lv.ea, &lv.ea_upd})
                for (int64_t i = el->off; i < el->off + el->cnt; ++i) items[(size_t)i].pad += (int32_t)ebase;
        items.insert(items.end(), easeg.begin(), easeg.end());
    }
    begin(h->inv2_items);
    for (int64_t e = 0; e < (int64_t)h->h_fronts.size(); ++e) {
        const Front& f = h->h_fronts[(size_t)e];
        if (f.i2off < 0) continue;
        for (int K = 0; K < (int)cdiv(f.nn, kSolveNB); ++K) push((int32_t)e, K, 0);
    }
    end(h->inv2_items);
    return 0;
}

}  // namespace mf
