// Minimum-degree elimination order on the quotient graph with approximate
// external degrees and element absorption, restated from the published
// algorithm of Amestoy, Davis & Duff, "An approximate minimum degree
// ordering algorithm", SIAM J. Matrix Anal. Appl. 17(4):886-905, 1996
// (degree bound of their eq. (4); aggressive absorption of elements whose
// variables all lie in the new element).  Supervariables are not detected.
//
// This is the general-purpose ordering of this package: the reference's
// default, AMF (src/AMFLib.jl, approximate minimum fill), is not restated;
// it differs in the score it minimises (fill instead of degree), not in the
// quotient-graph mechanics.
#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

extern "C" const char* ct_last_error(void);
void ct_set_error(const std::string& msg);

namespace {

using I = int64_t;

struct Buckets {  // doubly linked degree lists
    std::vector<I> head, next, prev, deg;
    I mindeg = 0;
    explicit Buckets(I n) : head(n + 1, -1), next(n, -1), prev(n, -1), deg(n, 0) {}
    void insert(I i, I d) {
        deg[i] = d;
        prev[i] = -1;
        next[i] = head[d];
        if (head[d] >= 0) prev[head[d]] = i;
        head[d] = i;
        if (d < mindeg) mindeg = d;
    }
    void remove(I i) {
        const I d = deg[i];
        if (prev[i] >= 0) next[prev[i]] = next[i]; else head[d] = next[i];
        if (next[i] >= 0) prev[next[i]] = prev[i];
        next[i] = prev[i] = -1;
    }
    I pop_min(I n) {
        while (mindeg <= n && head[mindeg] < 0) ++mindeg;
        if (mindeg > n) return -1;
        const I i = head[mindeg];
        remove(i);
        return i;
    }
};

}  // namespace

extern "C" int ct_mindeg_order(int64_t n, const int64_t* colptr, const int64_t* rowval, int64_t* order) {
    if (n < 0 || (n > 0 && (!colptr || !order))) {
        ct_set_error("ct_mindeg_order: bad arguments");
        return -1;
    }
    try {
        // symmetric adjacency without self loops
        std::vector<std::vector<I>> adj((size_t)n);
        for (I j = 0; j < n; ++j)
            for (I p = colptr[j]; p < colptr[j + 1]; ++p) {
                const I i = rowval[p];
                if (i < 0 || i >= n) {
                    ct_set_error("ct_mindeg_order: row index out of range");
                    return -2;
                }
                if (i == j) continue;
                adj[(size_t)i].push_back(j);
                adj[(size_t)j].push_back(i);
            }
        for (auto& a : adj) {
            std::sort(a.begin(), a.end());
            a.erase(std::unique(a.begin(), a.end()), a.end());
        }
        // status: 0 variable, 1 element (eliminated, live), 2 absorbed element
        std::vector<char> status((size_t)n, 0);
        std::vector<std::vector<I>> elems((size_t)n);  // E_i of a variable
        std::vector<std::vector<I>> Le((size_t)n);     // variables of a live element
        std::vector<I> w((size_t)n, -1), mark((size_t)n, -1);
        Buckets bk(n);
        for (I i = 0; i < n; ++i) bk.insert(i, (I)adj[(size_t)i].size());
        std::vector<I> Lp;
        for (I k = 0; k < n; ++k) {
            const I p = bk.pop_min(n);
            if (p < 0) {
                ct_set_error("ct_mindeg_order: degree lists exhausted early");
                return -3;
            }
            order[k] = p;
            status[(size_t)p] = 1;
            // L_p = (A_p U union of L_e over E_p) \ {p}; the elements of E_p are absorbed
            Lp.clear();
            mark[(size_t)p] = k;
            for (I j : adj[(size_t)p])
                if (status[(size_t)j] == 0 && mark[(size_t)j] != k) { mark[(size_t)j] = k; Lp.push_back(j); }
            for (I e : elems[(size_t)p]) {
                if (status[(size_t)e] != 1) continue;
                for (I j : Le[(size_t)e])
                    if (status[(size_t)j] == 0 && mark[(size_t)j] != k) { mark[(size_t)j] = k; Lp.push_back(j); }
                status[(size_t)e] = 2;
                std::vector<I>().swap(Le[(size_t)e]);
            }
            std::vector<I>().swap(adj[(size_t)p]);
            std::vector<I>().swap(elems[(size_t)p]);
            // prune the neighbours: variables of L_p are now reached through element p
            for (I i : Lp) {
                bk.remove(i);
                auto& A = adj[(size_t)i];
                A.erase(std::remove_if(A.begin(), A.end(),
                                       [&](I j) { return status[(size_t)j] != 0 || mark[(size_t)j] == k; }),
                        A.end());
                auto& E = elems[(size_t)i];
                E.erase(std::remove_if(E.begin(), E.end(), [&](I e) { return status[(size_t)e] != 1; }), E.end());
            }
            // |L_e \ L_p| for the other elements adjacent to L_p
            std::vector<I> touched;
            for (I i : Lp)
                for (I e : elems[(size_t)i]) {
                    if (w[(size_t)e] < 0) { w[(size_t)e] = (I)Le[(size_t)e].size(); touched.push_back(e); }
                    w[(size_t)e] -= 1;
                }
            // aggressive absorption: an element inside L_p adds nothing
            for (I e : touched)
                if (w[(size_t)e] == 0) { status[(size_t)e] = 2; std::vector<I>().swap(Le[(size_t)e]); }
            const I lp = (I)Lp.size();
            for (I i : Lp) {
                auto& E = elems[(size_t)i];
                E.erase(std::remove_if(E.begin(), E.end(), [&](I e) { return status[(size_t)e] != 1; }), E.end());
                I ext = 0;
                for (I e : E) ext += w[(size_t)e];
                E.push_back(p);
                const I d1 = bk.deg[(size_t)i] + lp - 1;
                const I d2 = (I)adj[(size_t)i].size() + lp - 1 + ext;
                I d = std::min(std::min(d1, d2), n - k - 1);
                if (d < 0) d = 0;
                bk.insert(i, d);
            }
            for (I e : touched) w[(size_t)e] = -1;
            Le[(size_t)p] = Lp;
        }
    } catch (const std::bad_alloc&) {
        ct_set_error("ct_mindeg_order: out of memory");
        return -4;
    }
    return 0;
}
