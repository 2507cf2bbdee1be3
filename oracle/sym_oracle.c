/*
 * sym_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of CliqueTrees.jl's symbolic analysis for the checker and
 * the reference arm of the benchmark: the default elimination order (AMF)
 * and the chain from an elimination order to a ChordalSymbolic.  It shares
 * no code with the product's host symbolic library; the tests compare the
 * two on many graphs, and both are pinned by the reference's known answers
 * (the AMFLib README order of the 8-vertex graph, the Maximal clique tree of
 * the 17-vertex graph of test/core.jl, the README 5x5 factorizations).
 *
 * Followed (paths relative to the reference root):
 *   AMFLib.amf / amf_impl! / hamf_impl!   src/AMFLib.jl/src/AMFLib.jl:56-155, :703-1525
 *       (HAMF4 of P. Amestoy via Scotch, BSD 3-clause licence: Copyright
 *        2004-2024 IPB, Universite de Bordeaux, INRIA & CNRS & others; AMD
 *        Copyright (c) 1996-2016 T. A. Davis, P. R. Amestoy, I. S. Duff.
 *        Provided "as is", without warranty of any kind.)
 *   simplegraph                          src/bipartite_graphs.jl:393-413
 *   supernodetree_impl!                  src/supernode_trees.jl:107-180
 *     etree_impl! (Liu)                  src/parent.jl:54-90
 *     column counts (supcnt_impl!)       src/parent.jl:201-297; computed
 *                                        here by row-subtree traversal, which
 *                                        yields the same numbers
 *     stree_impl! (Maximal)              src/supernode_types.jl:41-88
 *     postorder!_impl! / lcrs_impl!      src/parent.jl:94-119, :420-458, :527-598
 *   cliquetree_impl! (separators)        src/clique_trees.jl:146-234
 *   ChordalSymbolic(res, sep, tree)      src/Multifrontal.jl/src/chordal_symbolic.jl:302-378
 *
 * Arrays crossing the interface are 0-based int64; 1-based inside the AMF
 * restatement, as in the reference.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef int64_t I;

/* ------------------------------------------------------------------------ */
/* AMF (hamf_impl! without elements or halo: unit weights, nbelts = 0)       */
/* ------------------------------------------------------------------------ */

typedef struct {
    I n, norig, nbbuck, iwlen, pfree, pas;
    I *pe, *len, *iw, *nv, *elen, *last, *degree, *wf, *next, *w, *head;
} amf_ws;

static I amf_bucket(const amf_ws* a, I score) {
    if (score > a->norig) {
        I d = (score - a->norig) / a->pas + a->norig;
        return d < a->nbbuck ? d : a->nbbuck;
    }
    return score;
}

static void amf_unlink(amf_ws* a, I i) {
    I ilast = a->last[i], inext = a->next[i];
    if (inext != 0) a->last[inext] = ilast;
    if (ilast != 0) a->next[ilast] = inext;
    else a->head[amf_bucket(a, a->wf[i]) + 1] = inext;
}

static int amf_run(amf_ws* a) {
    I *pe = a->pe, *len = a->len, *iw = a->iw, *nv = a->nv, *elen = a->elen, *last = a->last;
    I *degree = a->degree, *wf = a->wf, *next = a->next, *w = a->w, *head = a->head;
    const I n = a->n, norig = a->norig, nbbuck = a->nbbuck, iwlen = a->iwlen;
    const I idummy = INT64_MAX - 1;
    const double dummy = (double)idummy;
    const I maxint_n = INT64_MAX - norig;
    const I hmod = nbbuck - 1 > 1 ? nbbuck - 1 : 1;
    I wflg = 2, nel = 0, totel = 0, dmax = 0, mindeg = 0, nleft;
    I pfree = a->pfree;
    a->pas = norig / 8 > 1 ? norig / 8 : 1;

    for (I i = 1; i <= n; ++i) { elen[i] = last[i] = degree[i] = wf[i] = next[i] = w[i] = 0; }
    for (I i = 1; i <= nbbuck + 2; ++i) head[i] = 0;
    for (I i = 1; i <= n; ++i) { w[i] = 1; totel += nv[i]; degree[i] = len[i]; }
    for (I i = 1; i <= n; ++i) {
        I deg = degree[i];
        if (deg > 0) {
            wf[i] = deg;
            deg = amf_bucket(a, deg);
            I inext = head[deg + 1];
            if (inext != 0) last[inext] = i;
            next[i] = inext;
            head[deg + 1] = i;
        } else {
            nel += nv[i]; elen[i] = -nel; pe[i] = 0; w[i] = 0;
        }
    }

    while (nel < totel) {
        I deg = mindeg - 1, me = 0;
        while (deg < nbbuck && me <= 0) { deg += 1; me = head[deg + 1]; }
        mindeg = deg;
        if (me <= 0) return -3;
        if (deg > norig) {
            I j = next[me], k = wf[me];
            while (j > 0) {
                if (wf[j] < k) { me = j; k = wf[me]; }
                j = next[j];
            }
            I ilast = last[me], inext = next[me];
            if (inext != 0) last[inext] = ilast;
            if (ilast != 0) next[ilast] = inext; else head[deg + 1] = inext;
        } else {
            I inext = next[me];
            if (inext != 0) last[inext] = 0;
            head[deg + 1] = inext;
        }
        const I elenme = elen[me];
        elen[me] = -1 - nel;
        I nvpiv = nv[me];
        nel += nvpiv;
        nv[me] = -nvpiv;
        I degme = 0, pme1, pme2, newmem;
        if (elenme == 0) {
            pme1 = pe[me];
            pme2 = pme1 - 1;
            for (I p = pme1; p <= pme1 + len[me] - 1; ++p) {
                I i = iw[p], nvi = nv[i];
                if (nvi > 0) {
                    degme += nvi; nv[i] = -nvi; pme2 += 1; iw[pme2] = i;
                    amf_unlink(a, i);
                }
            }
            newmem = 0;
        } else {
            I p = pe[me];
            pme1 = pfree;
            const I slenme = len[me] - elenme;
            I knt1_updated = 0;
            for (I knt1 = 1; knt1 <= elenme + 1; ++knt1) {
                knt1_updated += 1;
                I e, pj, ln;
                if (knt1 > elenme) { e = me; pj = p; ln = slenme; }
                else { e = iw[p]; p += 1; pj = pe[e]; ln = len[e]; }
                I knt2_updated = 0;
                for (I knt2 = 1; knt2 <= ln; ++knt2) {
                    knt2_updated += 1;
                    I i = iw[pj]; pj += 1;
                    I nvi = nv[i];
                    if (nvi > 0) {
                        if (pfree > iwlen) {
                            pe[me] = p; len[me] -= knt1_updated; knt1_updated = 0;
                            if (len[me] == 0) pe[me] = 0;
                            pe[e] = pj; len[e] = ln - knt2_updated; knt2_updated = 0;
                            if (len[e] == 0) pe[e] = 0;
                            for (I j = 1; j <= n; ++j) {
                                I pn = pe[j];
                                if (pn > 0) { pe[j] = iw[pn]; iw[pn] = -j; }
                            }
                            I pdst = 1, psrc = 1;
                            const I pend = pme1 - 1;
                            while (psrc <= pend) {
                                I j = -iw[psrc]; psrc += 1;
                                if (j > 0) {
                                    iw[pdst] = pe[j]; pe[j] = pdst; pdst += 1;
                                    const I lenj = len[j];
                                    for (I t = 0; t <= lenj - 2; ++t) iw[pdst + t] = iw[psrc + t];
                                    pdst += lenj - 1; psrc += lenj - 1;
                                }
                            }
                            const I p1 = pdst;
                            for (I ps = pme1; ps <= pfree - 1; ++ps) { iw[pdst] = iw[ps]; pdst += 1; }
                            pme1 = p1; pfree = pdst; pj = pe[e]; p = pe[me];
                        }
                        degme += nvi; nv[i] = -nvi; iw[pfree] = i; pfree += 1;
                        amf_unlink(a, i);
                    }
                }
                if (e != me) { pe[e] = -me; w[e] = 0; }
            }
            pme2 = pfree - 1;
            newmem = pfree - pme1;
        }
        degree[me] = degme;
        pe[me] = pme1;
        len[me] = pme2 - pme1 + 1;
        if (wflg > maxint_n) {
            for (I x = 1; x <= n; ++x) if (w[x] != 0) w[x] = 1;
            wflg = 2;
        }
        for (I pme = pme1; pme <= pme2; ++pme) {
            const I i = iw[pme], eln = elen[i];
            if (eln > 0) {
                const I nvi = -nv[i], wnvi = wflg - nvi;
                for (I p = pe[i]; p <= pe[i] + eln - 1; ++p) {
                    const I e = iw[p];
                    I we = w[e];
                    if (we >= wflg) we -= nvi;
                    else if (we != 0) { we = degree[e] + wnvi; wf[e] = 0; }
                    w[e] = we;
                }
            }
        }
        for (I pme = pme1; pme <= pme2; ++pme) {
            const I i = iw[pme], p1 = pe[i], p2 = p1 + elen[i] - 1;
            I pn = p1, hash = 0, dg = 0, wf3 = 0, wf4 = 0, nvi = -nv[i];
            for (I p = p1; p <= p2; ++p) {
                const I e = iw[p], dext = w[e] - wflg;
                if (dext > 0) {
                    if (wf[e] == 0) wf[e] = dext * (2 * degree[e] - dext - 1);
                    wf4 += wf[e]; dg += dext; iw[pn] = e; pn += 1; hash += e;
                } else if (dext == 0) {
                    pe[e] = -me; w[e] = 0;
                }
            }
            elen[i] = pn - p1 + 1;
            const I p3 = pn;
            for (I p = p2 + 1; p <= p1 + len[i] - 1; ++p) {
                const I j = iw[p], nvj = nv[j];
                if (nvj > 0) { dg += nvj; wf3 += nvj; iw[pn] = j; pn += 1; hash += j; }
            }
            if (dg == 0) {
                pe[i] = -me; nvi = -nv[i]; degme -= nvi; nvpiv += nvi; nel += nvi; nv[i] = 0; elen[i] = 0;
            } else {
                if (degree[i] < dg) { wf4 = 0; wf3 = 0; } else degree[i] = dg;
                wf[i] = wf4 + 2 * nvi * wf3;
                iw[pn] = iw[p3]; iw[p3] = iw[p1]; iw[p1] = me;
                len[i] = pn - p1 + 1;
                hash = (hash % hmod) + 1;
                const I j = head[hash + 1];
                if (j <= 0) { next[i] = -j; head[hash + 1] = -i; }
                else { next[i] = last[j]; last[j] = i; }
                last[i] = hash;
            }
        }
        degree[me] = degme;
        if (degme > dmax) dmax = degme;
        wflg += dmax;
        if (wflg > maxint_n) {
            for (I x = 1; x <= n; ++x) if (w[x] != 0) w[x] = 1;
            wflg = 2;
        }
        for (I pme = pme1; pme <= pme2; ++pme) {
            I i = iw[pme];
            if (nv[i] >= 0) continue;
            const I hash = last[i];
            I j = head[hash + 1];
            if (j == 0) continue;
            if (j < 0) { i = -j; head[hash + 1] = 0; }
            else { i = last[j]; last[j] = 0; }
            while (i != 0 && next[i] != 0) {
                const I ln = len[i], eln = elen[i];
                for (I p = pe[i] + 1; p <= pe[i] + ln - 1; ++p) w[iw[p]] = wflg;
                I jlast = i;
                j = next[i];
                while (j != 0) {
                    int differ = len[j] != ln || elen[j] != eln;
                    for (I p = pe[j] + 1; !differ && p <= pe[j] + ln - 1; ++p) differ = w[iw[p]] != wflg;
                    if (differ) { jlast = j; j = next[j]; }
                    else {
                        pe[j] = -i;
                        if (wf[j] > wf[i]) wf[i] = wf[j];
                        nv[i] += nv[j]; nv[j] = 0; elen[j] = 0;
                        j = next[j]; next[jlast] = j;
                    }
                }
                wflg += 1;
                i = next[i];
            }
        }
        I p = pme1;
        nleft = totel - nel;
        for (I pme = pme1; pme <= pme2; ++pme) {
            const I i = iw[pme], nvi = -nv[i];
            if (nvi <= 0) continue;
            nv[i] = nvi;
            I dg = degree[i];
            double rmf;
            if (degree[i] + degme > nleft) {
                double rmf1 = (double)dg * (double)(dg - 1 + 2 * degme) - (double)wf[i];
                degree[i] = nleft - nvi;
                dg = degree[i];
                rmf = (double)dg * (double)(dg - 1) - (double)(degme - nvi) * (double)(degme - nvi - 1);
                if (rmf1 < rmf) rmf = rmf1;
            } else {
                degree[i] += degme - nvi;
                rmf = (double)dg * (double)(dg - 1 + 2 * degme) - (double)wf[i];
            }
            rmf /= (double)(nvi + 1);
            if (rmf < dummy) wf[i] = (I)floor(rmf + 0.5);
            else if (rmf / (double)n < dummy) wf[i] = (I)floor(rmf / (double)n + 0.5);
            else wf[i] = idummy;
            if (wf[i] <= 0) wf[i] = 1;
            const I bk = amf_bucket(a, wf[i]);
            const I inext = head[bk + 1];
            if (inext != 0) last[inext] = i;
            next[i] = inext; last[i] = 0; head[bk + 1] = i;
            if (mindeg > bk) mindeg = bk;
            iw[p] = i; p += 1;
        }
        nv[me] = nvpiv + degme;
        len[me] = p - pme1;
        if (len[me] == 0) { pe[me] = 0; w[me] = 0; }
        if (newmem != 0) pfree = p;
    }
    for (I i = 1; i <= n; ++i) {
        if (elen[i] != 0) continue;
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
    a->pfree = pfree;
    return 0;
}

/* order[k] = vertex eliminated k-th (0-based) by AMF() on the symmetric
 * pattern (colptr, rowval) (both triangles, rows ascending). */
int mfo_amf_order(I n, const I* colptr, const I* rowval, I* order) {
    if (n <= 0) return 0;
    I m = 0;
    for (I j = 0; j < n; ++j)
        for (I p = colptr[j]; p < colptr[j + 1]; ++p) m += rowval[p] != j;
    amf_ws a;
    memset(&a, 0, sizeof a);
    a.n = n; a.norig = n; a.nbbuck = 2 * n; a.iwlen = m + 4 * n + 10000;
    I** arrs[] = {&a.pe, &a.len, &a.nv, &a.elen, &a.last, &a.degree, &a.wf, &a.next, &a.w};
    int bad = 0;
    for (size_t t = 0; t < sizeof arrs / sizeof arrs[0]; ++t) bad |= !(*arrs[t] = calloc(n + 2, sizeof(I)));
    bad |= !(a.iw = calloc(a.iwlen + 1, sizeof(I)));
    bad |= !(a.head = calloc(a.nbbuck + 3, sizeof(I)));
    int rc = -4;
    if (!bad) {
        /* simplegraph: stored order, self loops dropped; pe/len (amf_impl!) */
        I q = 1;
        for (I j = 0; j < n; ++j) {
            a.pe[j + 1] = q;
            for (I p = colptr[j]; p < colptr[j + 1]; ++p)
                if (rowval[p] != j) a.iw[q++] = rowval[p] + 1;
            a.len[j + 1] = q - a.pe[j + 1];
            a.nv[j + 1] = 1;
        }
        a.pe[n + 1] = q;
        a.pfree = q;
        rc = amf_run(&a);
        if (rc == 0) {
            I* pos = a.head; /* amf_impl! reuses head for the positions */
            for (I j = 1; j <= n; ++j) pos[j] = 0;
            for (I i = 1; i <= n; ++i) pos[a.elen[i] < 0 ? -a.elen[i] : a.elen[i]] = i;
            I k = 0;
            for (I j = 1; j <= n; ++j)
                if (pos[j] > 0) order[k++] = pos[j] - 1;
            if (k != n) rc = -3;
        }
    }
    for (size_t t = 0; t < sizeof arrs / sizeof arrs[0]; ++t) free(*arrs[t]);
    free(a.iw);
    free(a.head);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* elimination order -> ChordalSymbolic                                      */
/* ------------------------------------------------------------------------ */

typedef struct {
    I n, nfr;
    I *perm, *resptr, *sepptr, *septgt, *reltgt, *pnt, *chdptr, *chdtgt, *idx, *Dptr, *Lptr;
    I nMptr, nMval, nNval, nFval;
} mfo_sym;

static int cmp_i64(const void* x, const void* y) {
    I a = *(const I*)x, b = *(const I*)y;
    return (a > b) - (a < b);
}

void mfo_symbolic_free(mfo_sym* S) {
    if (!S) return;
    free(S->perm); free(S->resptr); free(S->sepptr); free(S->septgt); free(S->reltgt); free(S->pnt);
    free(S->chdptr); free(S->chdtgt); free(S->idx); free(S->Dptr); free(S->Lptr);
    free(S);
}

/* Symbolic factorization of the symmetric pattern (colptr, rowval) under the
 * elimination order `order` (order[k] = vertex eliminated k-th), Maximal
 * supernodes.  Returns NULL on failure. */
mfo_sym* mfo_symbolic_create(I n, const I* colptr, const I* rowval, const I* order) {
    mfo_sym* S = calloc(1, sizeof(mfo_sym));
    if (!S) return NULL;
    S->n = n;
    I *index = malloc(sizeof(I) * (n + 1)), *lptr = calloc(n + 2, sizeof(I)), *ltgt = NULL;
    I *par = malloc(sizeof(I) * (n + 1)), *anc = malloc(sizeof(I) * (n + 1)), *cc = calloc(n + 1, sizeof(I));
    I *mark = malloc(sizeof(I) * (n + 1)), *cptr = calloc(n + 2, sizeof(I)), *ctgt = malloc(sizeof(I) * (n + 1));
    I *snd_of = malloc(sizeof(I) * (n + 1)), *first = malloc(sizeof(I) * (n + 1));
    I *spar = malloc(sizeof(I) * (n + 1)), *sanc = malloc(sizeof(I) * (n + 1));
    I *post = malloc(sizeof(I) * (n + 1)), *newpos = malloc(sizeof(I) * (n + 1));
    I *child = NULL, *brother = NULL, *stack = NULL, *oldsnd = NULL;
    if (!index || !lptr || !par || !anc || !cc || !mark || !cptr || !ctgt || !snd_of || !first || !spar || !sanc ||
        !post || !newpos)
        goto fail;
    /* positions: vertex order[k] is eliminated k-th; 1-based labels below */
    for (I k = 0; k < n; ++k) index[order[k]] = k + 1;
    /* lower adjacency in elimination labels: for label i, the labels k < i of its neighbours */
    for (I j = 0; j < n; ++j)
        for (I p = colptr[j]; p < colptr[j + 1]; ++p) {
            I a = index[j], b = index[rowval[p]];
            if (a != b) lptr[(a > b ? a : b) + 1]++;
        }
    for (I i = 1; i <= n; ++i) lptr[i + 1] += lptr[i];
    ltgt = malloc(sizeof(I) * (lptr[n + 1] + 1));
    if (!ltgt) goto fail;
    {
        I* pos = mark;
        for (I i = 1; i <= n; ++i) pos[i] = lptr[i];
        for (I j = 0; j < n; ++j)
            for (I p = colptr[j]; p < colptr[j + 1]; ++p) {
                I a = index[j], b = index[rowval[p]];
                if (a > b) ltgt[pos[a]++] = b;
                else if (b > a) ltgt[pos[b]++] = a;
            }
    }
    /* elimination tree (Liu, path compression) */
    for (I i = 1; i <= n; ++i) {
        par[i] = 0; anc[i] = 0;
        for (I p = lptr[i]; p < lptr[i + 1]; ++p) {
            I r = ltgt[p];
            while (anc[r] != 0 && anc[r] != i) { I t = anc[r]; anc[r] = i; r = t; }
            if (anc[r] == 0) { anc[r] = i; par[r] = i; }
        }
    }
    /* column counts (diagonal included) by row subtrees: row i of L holds
     * every column on the tree paths from its lower neighbours up to i */
    for (I i = 1; i <= n; ++i) { mark[i] = 0; cc[i] = 1; }
    for (I i = 1; i <= n; ++i) {
        mark[i] = i;
        for (I p = lptr[i]; p < lptr[i + 1]; ++p)
            for (I c = ltgt[p]; c != 0 && mark[c] != i; c = par[c]) { mark[c] = i; cc[c]++; }
    }
    /* children lists, ascending */
    for (I i = 1; i <= n; ++i) if (par[i]) cptr[par[i] + 1]++;
    cptr[1] = 1;
    for (I i = 1; i <= n; ++i) cptr[i + 1] += cptr[i];
    {
        I* pos = mark;
        for (I i = 1; i <= n; ++i) pos[i] = cptr[i];
        for (I i = 1; i <= n; ++i) if (par[i]) ctgt[pos[par[i]]++] = i;
    }
    /* Maximal supernodes: v continues the supernode of its first child s
     * (ascending) with cc[s] == cc[v] + 1 */
    I ns = 0;
    for (I v = 1; v <= n; ++v) {
        I u = 0;
        for (I p = cptr[v]; p < cptr[v + 1]; ++p)
            if (cc[ctgt[p]] == cc[v] + 1) { u = ctgt[p]; break; }
        if (u) snd_of[v] = snd_of[u];
        else { snd_of[v] = ++ns; first[ns] = v; spar[ns] = 0; sanc[ns] = 0; }
        for (I p = cptr[v]; p < cptr[v + 1]; ++p) {
            I s = ctgt[p];
            if (s != u) { spar[snd_of[s]] = snd_of[v]; sanc[snd_of[s]] = v; }
        }
    }
    /* postorder of the supernode tree: children ascending; the roots are
     * stacked ascending, so the largest root's subtree comes first */
    child = calloc(ns + 1, sizeof(I)); brother = calloc(ns + 1, sizeof(I));
    stack = malloc(sizeof(I) * (ns + 1)); oldsnd = malloc(sizeof(I) * (ns + 1));
    if (!child || !brother || !stack || !oldsnd) goto fail;
    {
        I root = 0;
        for (I i = ns; i >= 1; --i) {
            I j = spar[i];
            if (!j) { brother[i] = root; root = i; }
            else { brother[i] = child[j]; child[j] = i; }
        }
        I top = 0;
        for (I r = root; r; r = brother[r]) stack[++top] = r;
        for (I i = 1; i <= ns; ++i) {
            I j = stack[top--];
            while (child[j]) { stack[++top] = j; I c = child[j]; child[j] = brother[c]; j = c; }
            post[j] = i;
        }
    }
    for (I s = 1; s <= ns; ++s) oldsnd[post[s]] = s;
    /* residuals in postorder: the chain from first[s] up the elimination
     * tree until the vertex where s attaches to its parent supernode */
    S->nfr = ns;
    S->resptr = malloc(sizeof(I) * (ns + 1));
    S->sepptr = malloc(sizeof(I) * (ns + 1));
    S->pnt = malloc(sizeof(I) * (ns > 0 ? ns : 1));
    S->perm = malloc(sizeof(I) * (n > 0 ? n : 1));
    S->idx = malloc(sizeof(I) * (n > 0 ? n : 1));
    if (!S->resptr || !S->sepptr || !S->pnt || !S->perm || !S->idx) goto fail;
    {
        I p = 0;
        S->resptr[0] = 0;
        S->sepptr[0] = 0;
        for (I t = 1; t <= ns; ++t) {
            I s = oldsnd[t], u = first[s], nn = 0;
            for (I v = u; v != 0 && v != sanc[s]; v = par[v]) { newpos[v] = p + nn; nn++; }
            S->resptr[t] = p + nn;
            S->sepptr[t] = S->sepptr[t - 1] + (cc[u] - nn);
            S->pnt[t - 1] = spar[s] ? post[spar[s]] - 1 : -1;
            p += nn;
        }
        if (p != n) goto fail;
    }
    for (I v = 1; v <= n; ++v) S->perm[newpos[v]] = order[v - 1];
    for (I t = 0; t < ns; ++t)
        for (I c = S->resptr[t]; c < S->resptr[t + 1]; ++c) S->idx[c] = t;
    /* separators: rows below the residual of the first residual column of L
     * (its lower neighbours joined with the children's separators) */
    S->septgt = malloc(sizeof(I) * (S->sepptr[ns] + 1));
    S->reltgt = malloc(sizeof(I) * (S->sepptr[ns] + 1));
    S->chdptr = calloc(ns + 2, sizeof(I));
    S->chdtgt = malloc(sizeof(I) * (ns + 1));
    if (!S->septgt || !S->reltgt || !S->chdptr || !S->chdtgt) goto fail;
    for (I t = 0; t < ns; ++t) S->chdptr[(S->pnt[t] < 0 ? ns : S->pnt[t]) + 1]++;
    for (I t = 0; t <= ns; ++t) S->chdptr[t + 1] += S->chdptr[t];
    {
        I* pos = stack;  /* ns + 1 entries */
        for (I t = 0; t <= ns; ++t) pos[t] = S->chdptr[t];
        for (I t = 0; t < ns; ++t) S->chdtgt[pos[S->pnt[t] < 0 ? ns : S->pnt[t]]++] = t;
    }
    {
        /* new labels of the lower neighbours: the old label v is newpos[v] */
        for (I c = 0; c < n; ++c) mark[c + 1] = -1;
        I* buf = anc;  /* scratch, n + 1 entries */
        for (I t = 0; t < ns; ++t) {
            const I r1 = S->resptr[t + 1];
            I cnt = 0;
            /* the old label of new column r0 is first[oldsnd[t + 1]] */
            const I v0 = first[oldsnd[t + 1]];
            /* neighbours of v0 with a larger new label (both triangles of A) */
            const I orig = order[v0 - 1];
            for (I p = colptr[orig]; p < colptr[orig + 1]; ++p) {
                I w = newpos[index[rowval[p]]];
                if (w >= r1 && mark[w + 1] != t) { mark[w + 1] = t; buf[cnt++] = w; }
            }
            for (I q = S->chdptr[t]; q < S->chdptr[t + 1]; ++q) {
                I c = S->chdtgt[q];
                for (I e = S->sepptr[c]; e < S->sepptr[c + 1]; ++e) {
                    I w = S->septgt[e];
                    if (w >= r1 && mark[w + 1] != t) { mark[w + 1] = t; buf[cnt++] = w; }
                }
            }
            if (cnt != S->sepptr[t + 1] - S->sepptr[t]) goto fail;
            qsort(buf, (size_t)cnt, sizeof(I), cmp_i64);
            memcpy(S->septgt + S->sepptr[t], buf, sizeof(I) * cnt);
        }
    }
    /* rel, Dptr, Lptr and the stack bounds (chordal_symbolic.jl:302-378) */
    S->Dptr = malloc(sizeof(I) * (ns + 1));
    S->Lptr = malloc(sizeof(I) * (ns + 1));
    if (!S->Dptr || !S->Lptr) goto fail;
    {
        I jMptr = 1, jMval = 0, jNval = 0, Dp = 0, Lp = 0;
        S->nMptr = 1; S->nMval = 0; S->nNval = 0; S->nFval = 0;
        for (I t = 0; t < ns; ++t) {
            S->Dptr[t] = Dp; S->Lptr[t] = Lp;
            const I r0 = S->resptr[t], nn = S->resptr[t + 1] - r0, na = S->sepptr[t + 1] - S->sepptr[t];
            const I* jsep = S->septgt + S->sepptr[t];
            for (I q = S->chdptr[t]; q < S->chdptr[t + 1]; ++q) {
                I c = S->chdtgt[q];
                /* position (0-based) of each row of sep(c) in res(t) ++ sep(t) */
                I k = 0;
                for (I e = S->sepptr[c]; e < S->sepptr[c + 1]; ++e) {
                    I v = S->septgt[e];
                    if (v < r0 + nn) S->reltgt[e] = v - r0;
                    else {
                        while (k < na && jsep[k] < v) k++;
                        S->reltgt[e] = nn + k;
                    }
                }
                I ma = S->sepptr[c + 1] - S->sepptr[c];
                jMptr -= 1; jMval -= ma * ma; jNval -= ma;
            }
            if (na > 0) {
                jMptr += 1; jMval += na * na; jNval += na;
                if (jMptr > S->nMptr) S->nMptr = jMptr;
                if (jMval > S->nMval) S->nMval = jMval;
                if (jNval > S->nNval) S->nNval = jNval;
            }
            if (nn + na > S->nFval) S->nFval = nn + na;
            Dp += nn * nn; Lp += nn * na;
        }
        S->Dptr[ns] = Dp; S->Lptr[ns] = Lp;
    }
    free(index); free(lptr); free(ltgt); free(par); free(anc); free(cc); free(mark); free(cptr); free(ctgt);
    free(snd_of); free(first); free(spar); free(sanc); free(post); free(newpos); free(child); free(brother);
    free(stack); free(oldsnd);
    return S;
fail:
    free(index); free(lptr); free(ltgt); free(par); free(anc); free(cc); free(mark); free(cptr); free(ctgt);
    free(snd_of); free(first); free(spar); free(sanc); free(post); free(newpos); free(child); free(brother);
    free(stack); free(oldsnd);
    mfo_symbolic_free(S);
    return NULL;
}

/* sizes: n, nfr, nsep, nMptr, nMval, nNval, nFval */
void mfo_symbolic_sizes(const mfo_sym* S, I* out) {
    out[0] = S->n; out[1] = S->nfr; out[2] = S->sepptr[S->nfr];
    out[3] = S->nMptr; out[4] = S->nMval; out[5] = S->nNval; out[6] = S->nFval;
}

/* copy out; lengths: perm, idx n; resptr, sepptr, Dptr, Lptr nfr+1; septgt,
 * reltgt nsep; pnt nfr; chdptr nfr+2; chdtgt nfr */
void mfo_symbolic_arrays(const mfo_sym* S, I* perm, I* resptr, I* sepptr, I* septgt, I* reltgt, I* pnt, I* chdptr,
                         I* chdtgt, I* idx, I* Dptr, I* Lptr) {
    const I n = S->n, nf = S->nfr, ns = S->sepptr[nf];
    memcpy(perm, S->perm, sizeof(I) * n);
    memcpy(resptr, S->resptr, sizeof(I) * (nf + 1));
    memcpy(sepptr, S->sepptr, sizeof(I) * (nf + 1));
    memcpy(septgt, S->septgt, sizeof(I) * ns);
    memcpy(reltgt, S->reltgt, sizeof(I) * ns);
    memcpy(pnt, S->pnt, sizeof(I) * nf);
    memcpy(chdptr, S->chdptr, sizeof(I) * (nf + 2));
    memcpy(chdtgt, S->chdtgt, sizeof(I) * nf);
    memcpy(idx, S->idx, sizeof(I) * n);
    memcpy(Dptr, S->Dptr, sizeof(I) * (nf + 1));
    memcpy(Lptr, S->Lptr, sizeof(I) * (nf + 1));
}
