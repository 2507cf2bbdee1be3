// Approximate minimum fill (AMF) ordering: the reference's default
// elimination algorithm, restated in C++ so that the host symbolic analysis
// orders a matrix exactly as CliqueTrees.jl does.
//
// Reference (paths relative to the CliqueTrees.jl root):
//   AMFLib.amf(weights, graph)     src/elimination_algorithms.jl:1556-1559
//                                  (simplegraph, then amf on its CSR arrays)
//   amf(n, vwght, xadj, adjncy)    src/AMFLib.jl/src/AMFLib.jl:56-91
//   amf_impl!                      src/AMFLib.jl/src/AMFLib.jl:93-155
//   hamf_impl!                     src/AMFLib.jl/src/AMFLib.jl:703-1525
//   default algorithm AMF()        src/elimination_algorithms.jl:2380
//
// Provenance and licence of the algorithm.  hamf_impl! is the HAMF4 routine
// (halo approximate minimum fill with supervariables, version 20190828) of
// Patrick Amestoy, adapted by Francois Pellegrini for Scotch
// (hall_order_hf.c) and from there to Julia; HAMF4 is itself a modification
// of AMD (Amestoy, Davis and Duff, "An approximate minimum degree ordering
// algorithm", SIAM J. Matrix Anal. Appl. 17 (1996) 886-905).  Those sources
// are distributed under the BSD 3-clause licence:
//   Copyright 2004,2007,2010,2012,2018-2020,2023,2024 IPB, Universite de
//   Bordeaux, INRIA & CNRS & others; AMD Copyright (c) 1996-2016 Timothy A.
//   Davis, Patrick R. Amestoy and Iain S. Duff.  All rights reserved.
//   THIS SOFTWARE IS PROVIDED BY THE COPYRIGHT HOLDERS AND CONTRIBUTORS "AS
//   IS" AND ANY EXPRESS OR IMPLIED WARRANTIES, INCLUDING, BUT NOT LIMITED TO,
//   THE IMPLIED WARRANTIES OF MERCHANTABILITY AND FITNESS FOR A PARTICULAR
//   PURPOSE ARE DISCLAIMED.  IN NO EVENT SHALL THE COPYRIGHT HOLDERS OR
//   CONTRIBUTORS BE LIABLE FOR ANY DIRECT, INDIRECT, INCIDENTAL, SPECIAL,
//   EXEMPLARY, OR CONSEQUENTIAL DAMAGES ARISING IN ANY WAY OUT OF THE USE OF
//   THIS SOFTWARE, EVEN IF ADVISED OF THE POSSIBILITY OF SUCH DAMAGE.
//
// The ordering must come out identical to the reference's, so the pivot
// selection, tie breaking, hashing, list orders, aggressive absorption,
// workspace compression and the floating-point fill score follow
// hamf_impl! step by step.  Only the graph form the reference uses for
// AMF() is supported: a plain graph of unit-weight variables, no elements
// and no halo (nbelts = 0, every len(i) >= 0, norig = n), so the halo
// branches of hamf_impl! (degree(i) = n2) are never taken and are left out.
// Arrays are 1-based inside this file, as in the reference, which keeps
// every index expression comparable line by line.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cliquetrees_symbolic.h"

void ct_set_error(const std::string& msg);

namespace {

typedef int64_t I;

// floor(x + 1/2) as an integer (anint, AMFLib.jl:52-54)
inline I anint(double x) { return (I)std::floor(x + 0.5); }

struct Amf {
    // problem
    I n = 0, norig = 0, nbbuck = 0, iwlen = 0, pfree = 0;
    // 1-based work arrays (index 0 unused), named as in hamf_impl!
    std::vector<I> pe, len, iw, nv, elen, last, degree, wf, next, w, head;

    // bucket of a fill score: scores above norig share buckets of width pas
    inline I bucket(I score, I pas) const {
        if (score > norig) {
            I d = (score - norig) / pas + norig;
            return d < nbbuck ? d : nbbuck;
        }
        return score;
    }

    // remove variable i from its degree list (AMFLib.jl:1028-1047)
    inline void unlink(I i, I pas) {
        I ilast = last[i], inext = next[i];
        if (inext != 0) last[inext] = ilast;
        if (ilast != 0) {
            next[ilast] = inext;
        } else {
            head[bucket(wf[i], pas) + 1] = inext;
        }
    }

    // hamf_impl! (AMFLib.jl:703-1525) for a graph without elements or halo.
    void run() {
        for (I i = 1; i <= n; ++i) {
            elen[i] = 0; last[i] = 0; degree[i] = 0; wf[i] = 0; next[i] = 0; w[i] = 0;
        }
        for (I i = 1; i <= nbbuck + 2; ++i) head[i] = 0;

        const I idummy = std::numeric_limits<I>::max() - 1;
        const double dummy = (double)idummy;
        const I pas = std::max<I>(norig / 8, 1);
        I wflg = 2;
        const I maxint_n = std::numeric_limits<I>::max() - norig;
        I nel = 0, totel = 0;
        const I hmod = std::max<I>(1, nbbuck - 1);
        I dmax = 0;
        I mem = pfree - 1;
        I maxmem = mem;
        I mindeg = 0;

        // AMFLib.jl:840-867: no elements; unit weights so degree = len
        for (I i = 1; i <= n; ++i) {
            w[i] = 1;
            totel += nv[i];
            degree[i] = len[i];
        }

        // AMFLib.jl:913-955: degree lists; isolated variables go first
        for (I i = 1; i <= n; ++i) {
            if (elen[i] < 0) continue;
            I deg = degree[i];
            if (deg > 0) {
                wf[i] = deg;
                deg = bucket(deg, pas);
                I inext = head[deg + 1];
                if (inext != 0) last[inext] = i;
                next[i] = inext;
                head[deg + 1] = i;
            } else {
                nel += nv[i];
                elen[i] = -nel;
                pe[i] = 0;
                w[i] = 0;
            }
        }

        I nleft = totel - nel;
        (void)nleft;

        while (nel < totel) {
            // pivot: first nonempty bucket at or above mindeg (AMFLib.jl:960-1005)
            I deg = mindeg - 1, me = 0;
            while (deg < nbbuck && me <= 0) {
                deg += 1;
                me = head[deg + 1];
            }
            mindeg = deg;
            if (me <= 0) throw std::runtime_error("amf: no pivot found");
            if (deg > norig) {
                // shared bucket: the variable of smallest score, first seen wins
                I j = next[me];
                I k = wf[me];
                while (j > 0) {
                    if (wf[j] < k) { me = j; k = wf[me]; }
                    j = next[j];
                }
                I ilast = last[me], inext = next[me];
                if (inext != 0) last[inext] = ilast;
                if (ilast != 0) next[ilast] = inext;
                else head[deg + 1] = inext;
            } else {
                I inext = next[me];
                if (inext != 0) last[inext] = 0;
                head[deg + 1] = inext;
            }

            // AMFLib.jl:1007-1012
            const I elenme = elen[me];
            elen[me] = -1 - nel;
            I nvpiv = nv[me];
            nel += nvpiv;
            nv[me] = -nvpiv;
            I degme = 0;
            I pme1, pme2, newmem;

            if (elenme == 0) {
                // new element in place (AMFLib.jl:1014-1051)
                pme1 = pe[me];
                pme2 = pme1 - 1;
                for (I p = pme1; p <= pme1 + len[me] - 1; ++p) {
                    I i = iw[p];
                    I nvi = nv[i];
                    if (nvi > 0) {
                        degme += nvi;
                        nv[i] = -nvi;
                        pme2 += 1;
                        iw[pme2] = i;
                        unlink(i, pas);
                    }
                }
                newmem = 0;
            } else {
                // new element in the free space iw[pfree...] (AMFLib.jl:1052-1179)
                I p = pe[me];
                pme1 = pfree;
                const I slenme = len[me] - elenme;
                I knt1_updated = 0;
                for (I knt1 = 1; knt1 <= elenme + 1; ++knt1) {
                    knt1_updated += 1;
                    I e, pj, ln;
                    if (knt1 > elenme) {
                        e = me; pj = p; ln = slenme;
                    } else {
                        e = iw[p]; p += 1;
                        pj = pe[e]; ln = len[e];
                    }
                    I knt2_updated = 0;
                    for (I knt2 = 1; knt2 <= ln; ++knt2) {
                        knt2_updated += 1;
                        I i = iw[pj]; pj += 1;
                        I nvi = nv[i];
                        if (nvi > 0) {
                            if (pfree > iwlen) {
                                // compress iw (AMFLib.jl:1079-1140)
                                pe[me] = p;
                                len[me] -= knt1_updated;
                                knt1_updated = 0;
                                if (len[me] == 0) pe[me] = 0;
                                pe[e] = pj;
                                len[e] = ln - knt2_updated;
                                knt2_updated = 0;
                                if (len[e] == 0) pe[e] = 0;
                                for (I j = 1; j <= n; ++j) {
                                    I pn = pe[j];
                                    if (pn > 0) { pe[j] = iw[pn]; iw[pn] = -j; }
                                }
                                I pdst = 1, psrc = 1;
                                const I pend = pme1 - 1;
                                while (psrc <= pend) {
                                    I j = -iw[psrc];
                                    psrc += 1;
                                    if (j > 0) {
                                        iw[pdst] = pe[j];
                                        pe[j] = pdst;
                                        pdst += 1;
                                        const I lenj = len[j];
                                        for (I knt3 = 0; knt3 <= lenj - 2; ++knt3) iw[pdst + knt3] = iw[psrc + knt3];
                                        pdst += lenj - 1;
                                        psrc += lenj - 1;
                                    }
                                }
                                const I p1 = pdst;
                                for (I ps = pme1; ps <= pfree - 1; ++ps) { iw[pdst] = iw[ps]; pdst += 1; }
                                pme1 = p1;
                                pfree = pdst;
                                pj = pe[e];
                                p = pe[me];
                            }
                            degme += nvi;
                            nv[i] = -nvi;
                            iw[pfree] = i; pfree += 1;
                            unlink(i, pas);
                        }
                    }
                    if (e != me) { pe[e] = -me; w[e] = 0; }
                }
                pme2 = pfree - 1;
                newmem = pfree - pme1;
                mem += newmem;
                maxmem = std::max(maxmem, mem);
            }

            degree[me] = degme;
            pe[me] = pme1;
            len[me] = pme2 - pme1 + 1;

            if (wflg > maxint_n) {
                for (I x = 1; x <= n; ++x)
                    if (w[x] != 0) w[x] = 1;
                wflg = 2;
            }

            // |Le \ Lme| for every element e met (AMFLib.jl:1195-1218)
            for (I pme = pme1; pme <= pme2; ++pme) {
                const I i = iw[pme];
                const I eln = elen[i];
                if (eln > 0) {
                    const I nvi = -nv[i];
                    const I wnvi = wflg - nvi;
                    for (I p = pe[i]; p <= pe[i] + eln - 1; ++p) {
                        const I e = iw[p];
                        I we = w[e];
                        if (we >= wflg) {
                            we -= nvi;
                        } else if (we != 0) {
                            we = degree[e] + wnvi;
                            wf[e] = 0;
                        }
                        w[e] = we;
                    }
                }
            }

            // degree update and element absorption (AMFLib.jl:1220-1308)
            for (I pme = pme1; pme <= pme2; ++pme) {
                const I i = iw[pme];
                const I p1 = pe[i];
                const I p2 = p1 + elen[i] - 1;
                I pn = p1;
                I hash = 0;
                I dg = 0, wf3 = 0, wf4 = 0;
                I nvi = -nv[i];
                for (I p = p1; p <= p2; ++p) {
                    const I e = iw[p];
                    const I dext = w[e] - wflg;
                    if (dext > 0) {
                        if (wf[e] == 0) wf[e] = dext * (2 * degree[e] - dext - 1);
                        wf4 += wf[e];
                        dg += dext;
                        iw[pn] = e; pn += 1;
                        hash += e;
                    } else if (dext == 0) {
                        pe[e] = -me;
                        w[e] = 0;
                    }
                }
                elen[i] = pn - p1 + 1;
                const I p3 = pn;
                for (I p = p2 + 1; p <= p1 + len[i] - 1; ++p) {
                    const I j = iw[p];
                    const I nvj = nv[j];
                    if (nvj > 0) {
                        dg += nvj;
                        wf3 += nvj;
                        iw[pn] = j; pn += 1;
                        hash += j;
                    }
                }
                if (dg == 0) {
                    // mass elimination
                    pe[i] = -me;
                    nvi = -nv[i];
                    degme -= nvi;
                    nvpiv += nvi;
                    nel += nvi;
                    nv[i] = 0;
                    elen[i] = 0;
                } else {
                    if (degree[i] < dg) {
                        wf4 = 0;
                        wf3 = 0;
                    } else {
                        degree[i] = dg;
                    }
                    wf[i] = wf4 + 2 * nvi * wf3;
                    iw[pn] = iw[p3];
                    iw[p3] = iw[p1];
                    iw[p1] = me;
                    len[i] = pn - p1 + 1;
                    hash = (hash % hmod) + 1;
                    const I j = head[hash + 1];
                    if (j <= 0) {
                        next[i] = -j;
                        head[hash + 1] = -i;
                    } else {
                        next[i] = last[j];
                        last[j] = i;
                    }
                    last[i] = hash;
                }
            }

            degree[me] = degme;
            if (degme > dmax) dmax = degme;
            wflg += dmax;
            if (wflg > maxint_n) {
                for (I x = 1; x <= n; ++x)
                    if (w[x] != 0) w[x] = 1;
                wflg = 2;
            }

            // supervariable detection (AMFLib.jl:1328-1392)
            for (I pme = pme1; pme <= pme2; ++pme) {
                I i = iw[pme];
                if (nv[i] < 0) {
                    const I hash = last[i];
                    I j = head[hash + 1];
                    if (j == 0) continue;
                    if (j < 0) {
                        i = -j;
                        head[hash + 1] = 0;
                    } else {
                        i = last[j];
                        last[j] = 0;
                    }
                    while (i != 0 && next[i] != 0) {
                        const I ln = len[i];
                        const I eln = elen[i];
                        for (I p = pe[i] + 1; p <= pe[i] + ln - 1; ++p) w[iw[p]] = wflg;
                        I jlast = i;
                        j = next[i];
                        while (j != 0) {
                            bool differ = len[j] != ln || elen[j] != eln;
                            if (!differ) {
                                for (I p = pe[j] + 1; p <= pe[j] + ln - 1; ++p) {
                                    if (w[iw[p]] != wflg) { differ = true; break; }
                                }
                            }
                            if (differ) {
                                jlast = j;
                                j = next[j];
                            } else {
                                pe[j] = -i;
                                if (wf[j] > wf[i]) wf[i] = wf[j];
                                nv[i] += nv[j];
                                nv[j] = 0;
                                elen[j] = 0;
                                j = next[j];
                                next[jlast] = j;
                            }
                        }
                        wflg += 1;
                        i = next[i];
                    }
                }
            }

            // restore degree lists with the new fill scores (AMFLib.jl:1394-1455)
            I p = pme1;
            nleft = totel - nel;
            for (I pme = pme1; pme <= pme2; ++pme) {
                const I i = iw[pme];
                const I nvi = -nv[i];
                if (nvi > 0) {
                    nv[i] = nvi;
                    I dg = degree[i];
                    double rmf;
                    if (degree[i] + degme > nleft) {
                        const double rmf1 = (double)dg * (double)(dg - 1 + 2 * degme) - (double)wf[i];
                        degree[i] = nleft - nvi;
                        dg = degree[i];
                        rmf = (double)dg * (double)(dg - 1) - (double)(degme - nvi) * (double)(degme - nvi - 1);
                        rmf = std::min(rmf, rmf1);
                    } else {
                        degree[i] += degme - nvi;
                        rmf = (double)dg * (double)(dg - 1 + 2 * degme) - (double)wf[i];
                    }
                    rmf /= (double)(nvi + 1);
                    if (rmf < dummy) {
                        wf[i] = anint(rmf);
                    } else if (rmf / (double)n < dummy) {
                        wf[i] = anint(rmf / (double)n);
                    } else {
                        wf[i] = idummy;
                    }
                    if (wf[i] <= 0) wf[i] = 1;
                    const I bk = bucket(wf[i], pas);
                    const I inext = head[bk + 1];
                    if (inext != 0) last[inext] = i;
                    next[i] = inext;
                    last[i] = 0;
                    head[bk + 1] = i;
                    if (mindeg > bk) mindeg = bk;
                    iw[p] = i; p += 1;
                }
            }

            // finalise the element (AMFLib.jl:1457-1468)
            nv[me] = nvpiv + degme;
            len[me] = p - pme1;
            if (len[me] == 0) { pe[me] = 0; w[me] = 0; }
            if (newmem != 0) {
                pfree = p;
                mem = mem - newmem + len[me];
            }
        }

        // pivot order of every variable from the assembly tree (AMFLib.jl:1497-1522)
        for (I i = 1; i <= n; ++i) {
            if (elen[i] == 0) {
                I j = -pe[i];
                while (elen[j] >= 0) j = -pe[j];
                const I e = j;
                I k = -elen[e];
                j = i;
                while (elen[j] >= 0) {
                    const I jnext = -pe[j];
                    pe[j] = -e;
                    if (elen[j] == 0) { elen[j] = k; k += 1; }
                    j = jnext;
                }
                elen[e] = -k;
            }
        }
    }
};

}  // namespace

extern "C" int ct_amf_order(int64_t n, const int64_t* colptr, const int64_t* rowval, int64_t* order) {
    if (n < 0 || (n > 0 && (!colptr || !rowval || !order))) {
        ct_set_error("ct_amf_order: bad arguments");
        return -1;
    }
    if (n == 0) return 0;
    try {
        // simplegraph (bipartite_graphs.jl:393-413): the adjacency lists in
        // their stored order with self loops dropped, as 1-based CSR
        for (I j = 0; j < n; ++j) {
            if (colptr[j + 1] < colptr[j]) { ct_set_error("ct_amf_order: colptr decreases"); return -2; }
            for (I p = colptr[j]; p < colptr[j + 1]; ++p)
                if (rowval[p] < 0 || rowval[p] >= n) { ct_set_error("ct_amf_order: row index out of range"); return -2; }
        }
        std::vector<I> xadj(n + 2), adjncy;
        adjncy.reserve((size_t)(colptr[n] - colptr[0]) + 1);
        adjncy.push_back(0);  // 1-based
        for (I j = 0; j < n; ++j) {
            xadj[j + 1] = (I)adjncy.size();
            for (I p = colptr[j]; p < colptr[j + 1]; ++p)
                if (rowval[p] != j) adjncy.push_back(rowval[p] + 1);
        }
        xadj[n + 1] = (I)adjncy.size();

        // amf / amf_impl! set-up (AMFLib.jl:61-129)
        Amf a;
        a.n = n;
        a.norig = n;  // unit weights
        a.nbbuck = 2 * a.norig;
        const I mm = xadj[n + 1];
        const I m = mm - 1;
        a.iwlen = m + 4 * n + 10000;
        a.pe.assign(n + 2, 0);
        a.len.assign(n + 1, 0);
        a.iw.assign(a.iwlen + 1, 0);
        a.nv.assign(n + 1, 0);
        a.elen.assign(n + 1, 0);
        a.last.assign(n + 1, 0);
        a.degree.assign(n + 1, 0);
        a.wf.assign(n + 1, 0);
        a.next.assign(n + 1, 0);
        a.w.assign(n + 1, 0);
        a.head.assign(a.nbbuck + 3, 0);
        for (I p = 1; p <= m; ++p) a.iw[p] = adjncy[p];
        a.pfree = mm;
        I p = a.pe[1] = xadj[1];
        for (I i = 1; i <= n; ++i) {
            const I pp = a.pe[i + 1] = xadj[i + 1];
            a.nv[i] = 1;
            a.len[i] = pp - p;
            p = pp;
        }
        a.run();

        // AMFLib.jl:134-154: elen holds each variable's position
        std::vector<I> pos(a.norig + 1, 0);
        for (I i = 1; i <= n; ++i) {
            const I j = a.elen[i] < 0 ? -a.elen[i] : a.elen[i];
            pos[j] = i;
        }
        I k = 0;
        for (I j = 1; j <= a.norig; ++j) {
            const I i = pos[j];
            if (i > 0) {
                order[k] = i - 1;
                k += 1;
            }
        }
        if (k != n) { ct_set_error("ct_amf_order: internal error (positions are not a permutation)"); return -3; }
        return 0;
    } catch (const std::bad_alloc&) {
        ct_set_error("ct_amf_order: out of memory");
        return -4;
    } catch (const std::exception& ex) {
        ct_set_error(std::string("ct_amf_order: ") + ex.what());
        return -3;
    }
}
