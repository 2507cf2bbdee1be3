/*
 * cliquetrees_symbolic.h -- host-side symbolic analysis (integer, run once
 * per sparsity pattern).  C ABI, no CUDA.
 *
 * Replaces the Julia chain that turns an elimination order into a
 * `ChordalSymbolic`:
 *   symbolic(graph; alg=order)        src/Multifrontal.jl/src/chordal_symbolic.jl:88-91
 *   cliquetree(weights, graph, alg)   src/clique_trees.jl:106-144
 *   supernodetree_impl!               src/supernode_trees.jl:107-180
 *   ChordalSymbolic(res, sep, tree)   src/Multifrontal.jl/src/chordal_symbolic.jl:302-378
 *
 * Conventions: every index is 0-based int64 (the reference is 1-based).
 * Return codes: 0 ok, -1 bad argument, -2 invalid input, -3 internal
 * inconsistency, -4 out of memory; ct_last_error() describes the last one.
 */
#ifndef CLIQUETREES_SYMBOLIC_H
#define CLIQUETREES_SYMBOLIC_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ct_symbolic ct_symbolic;

/* Build the symbolic factorization of the symmetric pattern (colptr,
 * rowval) (both triangles or one; self loops ignored) under the elimination
 * order `order` (order[i] = vertex eliminated i-th).  The final order after
 * supernode relabelling is returned by ct_symbolic_arrays.
 * Reference: cliquetree(graph; alg=order, snd=Maximal()), clique_trees.jl:106. */
int ct_symbolic_create(int64_t n, const int64_t* colptr, const int64_t* rowval,
                       const int64_t* order, ct_symbolic** out);

void ct_symbolic_destroy(ct_symbolic* S);

/* out[0..8] = n, nfr, nsep, ndz (= sum nn^2), nlz (= sum nn*na),
 *             nMptr, nMval, nNval, nFval   (ChordalSymbolic fields,
 *             chordal_symbolic.jl:15-28). */
int ct_symbolic_sizes(const ct_symbolic* S, int64_t* out);

/* Copy the arrays out (any pointer may be NULL).  Lengths:
 * order, invp, idx: n;  resptr, sepptr, Dptr, Lptr: nfr+1;
 * septgt, reltgt: nsep;  pnt: nfr (-1 = root);  chdptr: nfr+2;  chdtgt: nfr
 * (children lists ascending; list nfr holds the roots, as Tree.graph does,
 * src/trees.jl:7-32). */
int ct_symbolic_arrays(const ct_symbolic* S, int64_t* order, int64_t* invp, int64_t* resptr,
                       int64_t* sepptr, int64_t* septgt, int64_t* reltgt, int64_t* pnt,
                       int64_t* chdptr, int64_t* chdtgt, int64_t* idx, int64_t* Dptr, int64_t* Lptr);

/* Nested-dissection elimination order of an nx*ny*nz grid by recursive
 * coordinate bisection (vertex id x + nx*(y + ny*z)).  Stands in for the
 * METIS order of ext/MetisExt.jl:64, which the reference accepts as an
 * explicit permutation (src/elimination_algorithms.jl:776-779). */
int ct_grid_nd_order(int64_t nx, int64_t ny, int64_t nz, int64_t leaf, int64_t* order);

/* Approximate-minimum-fill elimination order of the symmetric pattern
 * (colptr, rowval) (both triangles, rows of each column in stored order;
 * self loops ignored): the reference's default ordering AMF(), i.e.
 * AMFLib.amf(weights, graph) (src/elimination_algorithms.jl:1556-1559 ->
 * src/AMFLib.jl/src/AMFLib.jl:56-155, hamf_impl! :703-1525) with unit
 * weights, restated step by step so that the order is identical.
 * order[k] = vertex eliminated k-th (0-based). */
int ct_amf_order(int64_t n, const int64_t* colptr, const int64_t* rowval, int64_t* order);

/* Minimum-degree elimination order of the symmetric pattern (colptr,
 * rowval) (either or both triangles; self loops ignored): quotient graph
 * with approximate external degrees and element absorption (Amestoy, Davis
 * & Duff 1996).  An optional ordering; the reference's default is AMF
 * (ct_amf_order). */
int ct_mindeg_order(int64_t n, const int64_t* colptr, const int64_t* rowval, int64_t* order);

const char* ct_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
