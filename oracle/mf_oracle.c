/*
 * mf_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of CliqueTrees.jl's multifrontal numeric phase, used as
 * the checker for the CUDA implementation and as the timed CPU baseline.
 * It is never linked into, loaded by, or called from the product path.
 *
 * The reference (AlgebraicJulia/CliqueTrees.jl v1.19.4) is pure Julia and
 * delegates its dense arithmetic to BLAS/LAPACK (OpenBLAS via
 * libblastrampoline).  Julia is not installed here, so the reference cannot
 * be run: parity of this restatement is pinned by the in-repository
 * known-answer examples (5x5 Cholesky and LDLt factors and solves) and by
 * residual/backward-error checks; bit-level parity with a Julia run is
 * unpinned.  The BLAS here is the OpenBLAS 0.3.30 that ships inside the
 * scipy wheel (symbols prefixed `scipy_`), loaded with dlopen by the caller.
 *
 * Followed line by line (paths relative to the reference root):
 *   chol_impl!            src/Multifrontal.jl/src/cholesky.jl:361-392
 *   chol_loop_snd!        src/Multifrontal.jl/src/cholesky.jl:434-556
 *   chol_loop_nod!        src/Multifrontal.jl/src/cholesky.jl:560-692
 *   chol_factor!          src/Multifrontal.jl/src/cholesky.jl:694-737
 *   chol_send!            src/Multifrontal.jl/src/cholesky.jl:950-983
 *   potrf! (LAPACK)       src/Multifrontal.jl/src/blas/potrf.jl:87-103
 *   potrf!/potrf2! (LDLt) src/Multifrontal.jl/src/blas/potrf.jl:3-41, :135-178
 *   syrk! / trrk! / syr!  src/Multifrontal.jl/src/blas/syrk.jl:137-159, trrk.jl:5-8, syr.jl:3-11
 *   zerotri!, addscattertri!, cdiv!, cmul!
 *                         src/Multifrontal.jl/src/utils.jl:280-303, :555-579, :677-727
 *   regularize(::NoRegularization)
 *                         src/Multifrontal.jl/src/regularization/no_regularization.jl:27-42
 *   div_impl!             src/Multifrontal.jl/src/divide.jl:417-450
 *   div_fwd_loop_snd!/nod! src/Multifrontal.jl/src/divide.jl:493-659, :662-821
 *   div_bwd_loop_snd!/nod! src/Multifrontal.jl/src/divide.jl:864-1038, :1041-1204
 *   div_fwd_update!/div_bwd_update!
 *                         src/Multifrontal.jl/src/divide.jl:1206-1293
 *   ldiv!(W, ::NaturalFactorization, B)
 *                         src/Multifrontal.jl/src/divide.jl:191-199
 *   selinv! / selinv_impl! / selinv_loop_snd! / selinv_loop_nod! / selinv_send!
 *                         src/Multifrontal.jl/src/selinv.jl:38-424
 *   trrk! -> syr2k(alpha/2) src/Multifrontal.jl/src/blas/trrk.jl:5-8; trtri! -> LAPACK
 *                         src/Multifrontal.jl/src/blas/trtri.jl:3-6
 *
 * All symbolic arrays are 0-based (see include/cliquetrees_symbolic.h).
 */
#include <dlfcn.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int blasint; /* LP64 OpenBLAS */
typedef int64_t I;

static void (*x_dpotrf)(const char*, const blasint*, double*, const blasint*, blasint*, size_t);
static void (*x_dtrsm)(const char*, const char*, const char*, const char*, const blasint*, const blasint*,
                       const double*, const double*, const blasint*, double*, const blasint*, size_t, size_t,
                       size_t, size_t);
static void (*x_dsyrk)(const char*, const char*, const blasint*, const blasint*, const double*, const double*,
                       const blasint*, const double*, double*, const blasint*, size_t, size_t);
static void (*x_dsyr2k)(const char*, const char*, const blasint*, const blasint*, const double*, const double*,
                        const blasint*, const double*, const blasint*, const double*, double*, const blasint*,
                        size_t, size_t);
static void (*x_dsyr)(const char*, const blasint*, const double*, const double*, const blasint*, double*,
                      const blasint*, size_t);
static void (*x_dgemm)(const char*, const char*, const blasint*, const blasint*, const blasint*, const double*,
                       const double*, const blasint*, const double*, const blasint*, const double*, double*,
                       const blasint*, size_t, size_t);
static void (*x_dgemv)(const char*, const blasint*, const blasint*, const double*, const double*, const blasint*,
                       const double*, const blasint*, const double*, double*, const blasint*, size_t);
static void (*x_dger)(const blasint*, const blasint*, const double*, const double*, const blasint*, const double*,
                      const blasint*, double*, const blasint*);
static void (*x_dtrsv)(const char*, const char*, const char*, const blasint*, const double*, const blasint*,
                       double*, const blasint*, size_t, size_t, size_t);
static void (*x_set_threads)(int);
static void (*x_dsymm)(const char*, const char*, const blasint*, const blasint*, const double*, const double*,
                       const blasint*, const double*, const blasint*, const double*, double*, const blasint*,
                       size_t, size_t);
static void (*x_dsymv)(const char*, const blasint*, const double*, const double*, const blasint*, const double*,
                       const blasint*, const double*, double*, const blasint*, size_t);
static double (*x_ddot)(const blasint*, const double*, const blasint*, const double*, const blasint*);
static void (*x_dtrtri)(const char*, const char*, const blasint*, double*, const blasint*, blasint*, size_t, size_t);

static void* g_blas = NULL;

static void* sym(const char* name) {
    char buf[128];
    void* p = dlsym(g_blas, name);
    if (p) return p;
    snprintf(buf, sizeof buf, "scipy_%s", name);
    return dlsym(g_blas, buf);
}

/* Load BLAS from `path` (the scipy-bundled OpenBLAS).  Returns 0 on success. */
int mfo_init(const char* path, int nthreads) {
    if (!g_blas) {
        g_blas = dlopen(path, RTLD_NOW | RTLD_LOCAL);
        if (!g_blas) return -1;
        x_dpotrf = sym("dpotrf_");
        x_dtrsm = sym("dtrsm_");
        x_dsyrk = sym("dsyrk_");
        x_dsyr2k = sym("dsyr2k_");
        x_dsyr = sym("dsyr_");
        x_dgemm = sym("dgemm_");
        x_dgemv = sym("dgemv_");
        x_dger = sym("dger_");
        x_dtrsv = sym("dtrsv_");
        x_set_threads = sym("openblas_set_num_threads");
        x_dsymm = sym("dsymm_");
        x_dsymv = sym("dsymv_");
        x_ddot = sym("ddot_");
        x_dtrtri = sym("dtrtri_");
        if (!x_dsymm || !x_dsymv || !x_ddot || !x_dtrtri) return -2;
        if (!x_dpotrf || !x_dtrsm || !x_dsyrk || !x_dsyr2k || !x_dsyr || !x_dgemm || !x_dgemv || !x_dger ||
            !x_dtrsv)
            return -2;
    }
    if (x_set_threads && nthreads > 0) x_set_threads(nthreads);
    return 0;
}

/* ---------------------------------------------------------------------- */
/* pivot acceptance (no_regularization.jl:27-42): with sign s != 0 the     */
/* pivot must have the sign of s; with s == 0 anything is kept.  A         */
/* rejected pivot becomes zero, which the callers report as a failure.    */
static int g_reg_mode = 0;           /* 0 NoRegularization, 1 DynamicRegularization */
static double g_reg_delta = 0.0, g_reg_eps = 0.0;

/* The pivot rule for the following factorizations: mode 0 is
 * NoRegularization, mode 1 DynamicRegularization(delta, epsilon)
 * (dynamic_regularization.jl:75-90; negative values take the defaults
 * cbrt(eps) and sqrt(eps), :58-72). */
void mfo_set_regularization(int mode, double delta, double epsilon) {
    g_reg_mode = mode;
    g_reg_delta = delta < 0 ? cbrt(2.220446049250313e-16) : delta;
    g_reg_eps = epsilon < 0 ? sqrt(2.220446049250313e-16) : epsilon;
}

static double regularize(double s, double djj) {
    if (g_reg_mode == 1) return (s * djj < g_reg_eps) ? g_reg_delta * s : djj;
    if (s != 0.0 && !(s * djj > 0.0)) return 0.0;
    return djj;
}

/* potrf2!(Val(:L), A, d, S, R, Val(:U)) -- unblocked LDLt (potrf.jl:3-41) */
static I potrf2_ldlt(double* A, I n, I lda, double* d, const double* S) {
    for (I j = 0; j < n; ++j) {
        double Ajj = regularize(S[j], A[j + j * lda]);
        if (Ajj == 0.0) return j + 1;
        d[j] = Ajj;
        double iD = 1.0 / Ajj;
        for (I i = j + 1; i < n; ++i) A[i + j * lda] *= iD;
        for (I k = j + 1; k < n; ++k) {
            double Akj = A[k + j * lda];
            A[k + k * lda] -= Ajj * (Akj * Akj);
            for (I i = k + 1; i < n; ++i) A[i + k * lda] -= A[i + j * lda] * Ajj * Akj;
        }
    }
    return 0;
}

/* B <- B diag(d)^{-1}: cdiv!(Val(:R), Val(:U), B, d) (utils.jl:681-691) */
static void cdiv_r(double* B, I m, I n, I ldb, const double* d) {
    for (I j = 0; j < n; ++j) {
        double idj = 1.0 / d[j];
        for (I i = 0; i < m; ++i) B[i + j * ldb] *= idj;
    }
}

/* C <- alpha * B diag(d) B^T + beta C (lower) for LDLt:
 * syrk!(..., Val(:U)) = copy, cmul!, trrk! -> syr2k(alpha/2) (syrk.jl:147-159, trrk.jl:5-8) */
static void syrk_ldlt(double alpha, const double* B, I m, I k, I ldb, const double* d, double beta, double* C,
                      I ldc, double* W) {
    for (I j = 0; j < k; ++j)
        for (I i = 0; i < m; ++i) W[i + j * m] = B[i + j * ldb] * d[j];
    blasint bm = (blasint)m, bk = (blasint)k, lw = (blasint)(m > 0 ? m : 1), lb = (blasint)ldb, lc = (blasint)ldc;
    double a2 = alpha / 2;
    if (m > 0 && k > 0) x_dsyr2k("L", "N", &bm, &bk, &a2, W, &lw, B, &lb, &beta, C, &lc, 1, 1);
}

/* recursive potrf! for LDLt (potrf.jl:135-178), THRESHOLD = 64 (Multifrontal.jl:34) */
static I potrf_ldlt(double* A, I n, I lda, double* d, const double* S, double* W) {
    if (n <= 64) return potrf2_ldlt(A, n, lda, d, S);
    I n1 = 1;
    while (n1 * 2 <= n) n1 *= 2; /* 2^floor(log2 n) */
    n1 /= 2;
    double* A11 = A;
    double* A22 = A + n1 + n1 * lda;
    double* B = A + n1; /* rows n1.., cols 0..n1 */
    I info = potrf_ldlt(A11, n1, lda, d, S, W);
    if (info != 0) return info;
    blasint m = (blasint)(n - n1), k = (blasint)n1, la = (blasint)lda;
    double one = 1.0;
    x_dtrsm("R", "L", "T", "U", &m, &k, &one, A11, &la, B, &la, 1, 1, 1, 1);
    cdiv_r(B, n - n1, n1, lda, d);
    syrk_ldlt(-1.0, B, n - n1, n1, lda, d, 1.0, A22, lda, W);
    info = potrf_ldlt(A22, n - n1, lda, d + n1, S + n1, W);
    if (info != 0) return n1 + info;
    return 0;
}

/* potrf2!(Val(:L), A, d, S, R, Val(:N)) -- unblocked Cholesky with the
 * pivot rule (potrf.jl:3-41) */
static I potrf2_chol(double* A, I n, I lda, const double* S) {
    for (I j = 0; j < n; ++j) {
        double Ajj = regularize(S[j], A[j + j * lda]);
        if (Ajj == 0.0) return j + 1;
        A[j + j * lda] = Ajj = sqrt(Ajj);
        double iD = 1.0 / Ajj;
        for (I i = j + 1; i < n; ++i) A[i + j * lda] *= iD;
        for (I k = j + 1; k < n; ++k) {
            double Akj = A[k + j * lda];
            A[k + k * lda] -= Akj * Akj;
            for (I i = k + 1; i < n; ++i) A[i + k * lda] -= A[i + j * lda] * Akj;
        }
    }
    return 0;
}

/* generic recursive potrf! for Cholesky with a regularization
 * (potrf.jl:135-178 with Val(:N)), THRESHOLD = 64 */
static I potrf_chol(double* A, I n, I lda, const double* S) {
    if (n <= 64) return potrf2_chol(A, n, lda, S);
    I n1 = 1;
    while (n1 * 2 <= n) n1 *= 2;
    n1 /= 2;
    double* A22 = A + n1 + n1 * lda;
    double* B = A + n1;
    I info = potrf_chol(A, n1, lda, S);
    if (info != 0) return info;
    blasint m = (blasint)(n - n1), k = (blasint)n1, la = (blasint)lda;
    double one = 1.0, mone = -1.0;
    x_dtrsm("R", "L", "T", "N", &m, &k, &one, A, &la, B, &la, 1, 1, 1, 1);
    x_dsyrk("L", "N", &m, &k, &mone, B, &la, &one, A22, &la, 1, 1);
    info = potrf_chol(A22, n - n1, lda, S + n1);
    if (info != 0) return n1 + info;
    return 0;
}

/* chol_factor! (cholesky.jl:694-737) */
static I chol_factor(double* D, I nn, double* L, I na, double* d, const double* S, int diag, double* W) {
    I info;
    if (diag == 0 && g_reg_mode == 0) {
        /* LAPACK path for Float64 + NoRegularization (potrf.jl:101-103, :87-90) */
        blasint bn = (blasint)nn, binfo = 0;
        x_dpotrf("L", &bn, D, &bn, &binfo, 1);
        info = binfo;
    } else if (diag == 0) {
        /* any other regularization: the generic recursive potrf! */
        info = potrf_chol(D, nn, nn, S);
    } else {
        info = potrf_ldlt(D, nn, nn, d, S, W);
    }
    if (info == 0 && na > 0 && nn > 0) {
        blasint m = (blasint)na, k = (blasint)nn;
        double one = 1.0;
        x_dtrsm("R", "L", "T", diag ? "U" : "N", &m, &k, &one, D, &k, L, &m, 1, 1, 1, 1);
        if (diag) cdiv_r(L, na, nn, na, d);
    }
    return info;
}

typedef struct {
    I* Mptr;   /* stack of offsets into Mval */
    double* Mval;
    double* F; /* nFval^2 */
    double* W; /* nFval^2, LDLt scratch */
} fws;

/* addscattertri!(F, M, inj, Val(:L)) (utils.jl:555-579) */
static void addscattertri(double* F, I ldf, const double* M, I m, const I* inj) {
    for (I j = 0; j < m; ++j) {
        I cj = inj[j];
        for (I i = j; i < m; ++i) F[inj[i] + cj * ldf] += M[i + j * m];
    }
}

/* Multifrontal Cholesky (diag = 0) or LDLt (diag = 1) following chol_impl!.
 * Dval/Lval hold the assembled matrix on entry and the factor on exit.
 * d: n pivots (LDLt only, may be NULL for Cholesky).  S: n signs (NULL =
 * ones for Cholesky, zeros for LDLt).  Returns info: 0 ok; k > 0 = 1-based
 * permuted column of the first rejected pivot; < 0 allocation failure. */
int64_t mfo_chol_impl(I n, I nfr, const I* resptr, const I* sepptr, const I* reltgt, const I* chdptr,
                      const I* chdtgt, const I* Dptr, const I* Lptr, I nMptr, I nMval, I nFval, int diag,
                      double* Dval, double* Lval, double* d, const double* S_in) {
    double* S = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    fws w;
    size_t fsz = (size_t)(nFval * nFval > 2 ? nFval * nFval : 2);
    w.Mptr = (I*)malloc(sizeof(I) * (size_t)(nMptr + 2));
    w.Mval = (double*)malloc(sizeof(double) * (size_t)(nMval > 0 ? nMval : 1));
    w.F = (double*)malloc(sizeof(double) * fsz);
    w.W = (double*)malloc(sizeof(double) * fsz);
    if (!S || !w.Mptr || !w.Mval || !w.F || !w.W) {
        free(S); free(w.Mptr); free(w.Mval); free(w.F); free(w.W);
        return -1;
    }
    for (I i = 0; i < n; ++i) S[i] = S_in ? S_in[i] : (diag ? 0.0 : 1.0);

    I ns = 0; /* number of update matrices on the stack */
    w.Mptr[0] = 0;
    I result = 0;
    for (I j = 0; j < nfr && result == 0; ++j) {
        I r0 = resptr[j];
        I nn = resptr[j + 1] - r0;
        I na = sepptr[j + 1] - sepptr[j];
        I nj = nn + na;
        double* F = w.F;
        double* D = Dval + Dptr[j];
        double* L = Lval + Lptr[j];
        /* F <- 0 (lower triangle) */
        for (I c = 0; c < nj; ++c)
            for (I r = c; r < nj; ++r) F[r + c * nj] = 0.0;
        /* pop the children's update matrices in reverse order */
        for (I p = chdptr[j + 1] - 1; p >= chdptr[j]; --p) {
            I i = chdtgt[p];
            I ma = sepptr[i + 1] - sepptr[i];
            addscattertri(F, nj, w.Mval + w.Mptr[ns - 1], ma, reltgt + sepptr[i]);
            ns -= 1;
        }
        if (nn == 1) {
            /* chol_loop_nod! (cholesky.jl:560-692) */
            double d11 = D[0] + F[0];
            for (I a = 0; a < na; ++a) L[a] += F[1 + a];
            d11 = regularize(S[r0], d11);
            if (d11 == 0.0) { result = 1 + r0; break; }
            if (diag == 0) { d11 = sqrt(d11); D[0] = d11; }
            else d[r0] = d11;
            if (na > 0) {
                ns += 1;
                I strt = w.Mptr[ns - 1];
                w.Mptr[ns] = strt + na * na;
                double* M = w.Mval + strt;
                for (I c = 0; c < na; ++c)
                    for (I r = c; r < na; ++r) M[r + c * na] = F[(1 + r) + (1 + c) * nj];
                for (I a = 0; a < na; ++a) L[a] /= d11;
                blasint bn = (blasint)na, one_i = 1;
                double alpha = diag ? -d11 : -1.0;
                x_dsyr("L", &bn, &alpha, L, &one_i, M, &bn, 1);
            }
            continue;
        }
        /* chol_loop_snd! (cholesky.jl:434-556): L <- L + F */
        for (I c = 0; c < nn; ++c) {
            for (I r = c; r < nn; ++r) D[r + c * nn] += F[r + c * nj];
            for (I a = 0; a < na; ++a) L[a + c * na] += F[(nn + a) + c * nj];
        }
        I info = chol_factor(D, nn, L, na, diag ? d + r0 : NULL, S + r0, diag, w.W);
        if (info != 0) { result = info + r0; break; }
        if (na > 0) {
            ns += 1;
            I strt = w.Mptr[ns - 1];
            w.Mptr[ns] = strt + na * na;
            double* M = w.Mval + strt;
            for (I c = 0; c < na; ++c)
                for (I r = c; r < na; ++r) M[r + c * na] = F[(nn + r) + (nn + c) * nj];
            if (diag == 0) {
                blasint bm = (blasint)na, bk = (blasint)nn;
                double alpha = -1.0, beta = 1.0;
                x_dsyrk("L", "N", &bm, &bk, &alpha, L, &bm, &beta, M, &bm, 1, 1);
            } else {
                syrk_ldlt(-1.0, L, na, nn, na, d + r0, 1.0, M, na, w.W);
            }
        }
    }
    free(S); free(w.Mptr); free(w.Mval); free(w.F); free(w.W);
    return result;
}

/* ---------------------------------------------------------------------- */
/* supernodal solves                                                       */

/* Forward pass C <- L^{-1} C (div_impl! with isforward, divide.jl:439-442).
 * C is n x nrhs column major with leading dimension ldc; vec != 0 selects
 * the AbstractVector code path (trsv/gemv) used for a single vector.    */
static int fwd(I nfr, const I* resptr, const I* sepptr, const I* reltgt, const I* chdptr, const I* chdtgt,
               const I* Dptr, const I* Lptr, I nMptr, I nNval, I nFval, int diag, const double* Dval,
               const double* Lval, double* C, I nrhs, I ldc, int vec) {
    I* Mptr = (I*)malloc(sizeof(I) * (size_t)(nMptr + 2));
    double* Mval = (double*)malloc(sizeof(double) * (size_t)(nNval * nrhs > 0 ? nNval * nrhs : 1));
    double* F = (double*)malloc(sizeof(double) * (size_t)(nFval * nrhs > 0 ? nFval * nrhs : 1));
    if (!Mptr || !Mval || !F) { free(Mptr); free(Mval); free(F); return -1; }
    I ns = 0;
    Mptr[0] = 0;
    for (I j = 0; j < nfr; ++j) {
        I r0 = resptr[j];
        I nn = resptr[j + 1] - r0;
        I na = sepptr[j + 1] - sepptr[j];
        I nj = nn + na;
        const double* D = Dval + Dptr[j];
        const double* L = Lval + Lptr[j];
        double* C1 = C + r0;
        for (I k = 0; k < nj * nrhs; ++k) F[k] = 0.0;
        for (I p = chdptr[j + 1] - 1; p >= chdptr[j]; --p) {
            I i = chdtgt[p];
            I ma = sepptr[i + 1] - sepptr[i];
            const I* inj = reltgt + sepptr[i];
            const double* M = Mval + Mptr[ns - 1];
            for (I c = 0; c < nrhs; ++c)
                for (I a = 0; a < ma; ++a) F[inj[a] + c * nj] += M[a + c * ma];
            ns -= 1;
        }
        for (I c = 0; c < nrhs; ++c)
            for (I a = 0; a < nn; ++a) C1[a + c * ldc] += F[a + c * nj];
        if (nn == 1) {
            /* div_fwd_loop_nod! (divide.jl:662-821) */
            if (diag == 0)
                for (I c = 0; c < nrhs; ++c) C1[c * ldc] /= D[0];
        } else {
            blasint bn = (blasint)nn, br = (blasint)nrhs, bl = (blasint)ldc, one_i = 1;
            double one = 1.0;
            if (vec) x_dtrsv("L", "N", diag ? "U" : "N", &bn, D, &bn, C1, &one_i, 1, 1, 1);
            else x_dtrsm("L", "L", "N", diag ? "U" : "N", &bn, &br, &one, D, &bn, C1, &bl, 1, 1, 1, 1);
        }
        if (na > 0) {
            ns += 1;
            I strt = Mptr[ns - 1];
            Mptr[ns] = strt + na * nrhs;
            double* M2 = Mval + strt;
            for (I c = 0; c < nrhs; ++c)
                for (I a = 0; a < na; ++a) M2[a + c * na] = F[(nn + a) + c * nj];
            blasint bm = (blasint)na, bn = (blasint)nn, br = (blasint)nrhs, bl = (blasint)ldc, one_i = 1;
            double mone = -1.0, one = 1.0;
            if (nn == 1) {
                if (vec) {
                    double c1 = C1[0];
                    for (I a = 0; a < na; ++a) M2[a] += -c1 * L[a]; /* axpy!(-c1, l21, M2) */
                } else {
                    x_dger(&bm, &br, &mone, L, &one_i, C1, &bl, M2, &bm);
                }
            } else if (vec) {
                x_dgemv("N", &bm, &bn, &mone, L, &bm, C1, &one_i, &one, M2, &one_i, 1);
            } else {
                x_dgemm("N", "N", &bm, &br, &bn, &mone, L, &bm, C1, &bl, &one, M2, &bm, 1, 1);
            }
        }
    }
    free(Mptr); free(Mval); free(F);
    return 0;
}

/* Backward pass C <- L^{-T} C (divide.jl:443-446, :864-1204). */
static int bwd(I nfr, const I* resptr, const I* sepptr, const I* reltgt, const I* chdptr, const I* chdtgt,
               const I* Dptr, const I* Lptr, I nMptr, I nNval, I nFval, int diag, const double* Dval,
               const double* Lval, double* C, I nrhs, I ldc, int vec) {
    I* Mptr = (I*)malloc(sizeof(I) * (size_t)(nMptr + 2));
    double* Mval = (double*)malloc(sizeof(double) * (size_t)(nNval * nrhs > 0 ? nNval * nrhs : 1));
    double* F = (double*)malloc(sizeof(double) * (size_t)(nFval * nrhs > 0 ? nFval * nrhs : 1));
    if (!Mptr || !Mval || !F) { free(Mptr); free(Mval); free(F); return -1; }
    I ns = 0;
    Mptr[0] = 0;
    for (I j = nfr - 1; j >= 0; --j) {
        I r0 = resptr[j];
        I nn = resptr[j + 1] - r0;
        I na = sepptr[j + 1] - sepptr[j];
        I nj = nn + na;
        const double* D = Dval + Dptr[j];
        const double* L = Lval + Lptr[j];
        double* C1 = C + r0;
        const double* M2 = NULL;
        blasint bm = (blasint)na, bn = (blasint)nn, br = (blasint)nrhs, bl = (blasint)ldc, one_i = 1;
        double mone = -1.0, one = 1.0;
        if (na > 0) {
            M2 = Mval + Mptr[ns - 1];
            ns -= 1;
            if (nn == 1) {
                for (I c = 0; c < nrhs; ++c) {
                    /* c1 -= dot(l21, M2[:, c]) via gemv/ger-free loop as in the nod path */
                    double s = 0.0;
                    for (I a = 0; a < na; ++a) s += L[a] * M2[a + c * na];
                    C1[c * ldc] -= s;
                }
            } else if (vec) {
                x_dgemv("T", &bm, &bn, &mone, L, &bm, M2, &one_i, &one, C1, &one_i, 1);
            } else {
                x_dgemm("T", "N", &bn, &br, &bm, &mone, L, &bm, M2, &bm, &one, C1, &bl, 1, 1);
            }
        }
        if (nn == 1) {
            if (diag == 0)
                for (I c = 0; c < nrhs; ++c) C1[c * ldc] /= D[0];
        } else if (vec) {
            x_dtrsv("L", "T", diag ? "U" : "N", &bn, D, &bn, C1, &one_i, 1, 1, 1);
        } else {
            x_dtrsm("L", "L", "T", diag ? "U" : "N", &bn, &br, &one, D, &bn, C1, &bl, 1, 1, 1, 1);
        }
        for (I c = 0; c < nrhs; ++c) {
            for (I a = 0; a < nn; ++a) F[a + c * nj] = C1[a + c * ldc];
            for (I a = 0; a < na; ++a) F[(nn + a) + c * nj] = M2[a + c * na];
        }
        for (I p = chdptr[j]; p < chdptr[j + 1]; ++p) {
            I i = chdtgt[p];
            I ma = sepptr[i + 1] - sepptr[i];
            const I* inj = reltgt + sepptr[i];
            ns += 1;
            I strt = Mptr[ns - 1];
            Mptr[ns] = strt + ma * nrhs;
            double* Mi = Mval + strt;
            for (I c = 0; c < nrhs; ++c)
                for (I a = 0; a < ma; ++a) Mi[a + c * ma] = F[inj[a] + c * nj];
        }
    }
    free(Mptr); free(Mval); free(F);
    return 0;
}

/* ldiv!(W, NaturalFactorization(F), C): L solve, D solve (LDLt), L^T solve
 * (divide.jl:191-199).  The permutation is applied by the caller. */
int mfo_div_impl(I n, I nfr, const I* resptr, const I* sepptr, const I* reltgt, const I* chdptr,
                 const I* chdtgt, const I* Dptr, const I* Lptr, I nMptr, I nNval, I nFval, int diag,
                 const double* Dval, const double* Lval, const double* d, double* C, I nrhs, I ldc, int vec) {
    int rc = fwd(nfr, resptr, sepptr, reltgt, chdptr, chdtgt, Dptr, Lptr, nMptr, nNval, nFval, diag, Dval, Lval,
                 C, nrhs, ldc, vec);
    if (rc) return rc;
    if (diag) {
        for (I c = 0; c < nrhs; ++c)
            for (I i = 0; i < n; ++i) C[i + c * ldc] /= d[i];
    }
    return bwd(nfr, resptr, sepptr, reltgt, chdptr, chdtgt, Dptr, Lptr, nMptr, nNval, nFval, diag, Dval, Lval, C,
               nrhs, ldc, vec);
}

/* ---------------------------------------------------------------------- */
/* selected inversion of a Cholesky factor (selinv!, selinv.jl:38-424):    */
/* Dval/Lval hold L on entry and the entries of A^{-1} on the pattern of L */
/* on exit (lower triangle of each diagonal block).  Returns 0, or -1 on   */
/* an allocation failure.                                                  */
int mfo_selinv(I n, I nfr, const I* resptr, const I* sepptr, const I* reltgt, const I* chdptr, const I* chdtgt,
               const I* Dptr, const I* Lptr, I nMptr, I nMval, I nFval, double* Dval, double* Lval) {
    (void)n;
    I* Mptr = (I*)malloc(sizeof(I) * (size_t)(nMptr + 2));
    double* Mval = (double*)malloc(sizeof(double) * (size_t)(nMval > 0 ? nMval : 1));
    double* F = (double*)malloc(sizeof(double) * (size_t)(nFval * nFval > 0 ? nFval * nFval : 1));
    if (!Mptr || !Mval || !F) { free(Mptr); free(Mval); free(F); return -1; }
    I ns = 0;
    Mptr[0] = 0;
    for (I j = nfr - 1; j >= 0; --j) {
        const I nn = resptr[j + 1] - resptr[j];
        const I na = sepptr[j + 1] - sepptr[j];
        const I nj = nn + na;
        double* D = Dval + Dptr[j];
        double* L = Lval + Lptr[j];
        if (nn == 1) {
            /* selinv_loop_nod! (selinv.jl:258-376) */
            double d11 = D[0];
            double f11 = 0.0;
            if (na > 0) {
                const double* M = Mval + Mptr[ns - 1];
                ns -= 1;
                for (I c = 0; c < na; ++c)
                    for (I r = c; r < na; ++r) F[(1 + r) + (1 + c) * nj] = M[r + c * na];
                for (I a = 0; a < na; ++a) L[a] /= d11;
                blasint bn = (blasint)na, one_i = 1, ldm = (blasint)na;
                double alpha = -1.0, beta = 0.0;
                x_dsymv("L", &bn, &alpha, M, &ldm, L, &one_i, &beta, F + 1, &one_i, 1);
                f11 -= x_ddot(&bn, L, &one_i, F + 1, &one_i);
            }
            d11 = 1.0 / d11;
            f11 += d11 * d11;
            D[0] = f11;
            F[0] = f11;
            for (I a = 0; a < na; ++a) L[a] = F[1 + a];
        } else {
            /* selinv_loop_snd! (selinv.jl:130-256) */
            for (I c = 0; c < nn; ++c)
                for (I r = 0; r < nn; ++r) F[r + c * nj] = 0.0;
            if (na > 0) {
                const double* M = Mval + Mptr[ns - 1];
                ns -= 1;
                for (I c = 0; c < na; ++c)
                    for (I r = c; r < na; ++r) F[(nn + r) + (nn + c) * nj] = M[r + c * na];
                blasint bm = (blasint)na, bk = (blasint)nn, bj = (blasint)nj;
                double one = 1.0, mone = -1.0, zero = 0.0, mhalf = -0.5;
                /* L21 <- L21 D11^{-1} */
                x_dtrsm("R", "L", "N", "N", &bm, &bk, &one, D, &bk, L, &bm, 1, 1, 1, 1);
                /* F21 <- -M22 L21 */
                x_dsymm("L", "L", &bm, &bk, &mone, M, &bm, L, &bm, &zero, F + nn, &bj, 1, 1);
                /* F11 <- F11 - L21^T F21 (trrk: syr2k with alpha / 2) */
                x_dsyr2k("L", "T", &bk, &bm, &mhalf, L, &bm, F + nn, &bj, &one, F, &bj, 1, 1);
            }
            /* D11 <- D11^{-1}; tril!; F11 <- F11 + D11^T D11 */
            blasint bk = (blasint)nn, bj = (blasint)nj, info = 0;
            x_dtrtri("L", "N", &bk, D, &bk, &info, 1, 1);
            for (I c = 0; c < nn; ++c)
                for (I r = 0; r < c; ++r) D[r + c * nn] = 0.0;
            double one = 1.0;
            x_dsyrk("L", "T", &bk, &bk, &one, D, &bk, &one, F, &bj, 1, 1);
            /* D11 <- F11; L21 <- F21 */
            for (I c = 0; c < nn; ++c)
                for (I r = 0; r < nn; ++r) D[r + c * nn] = F[r + c * nj];
            for (I c = 0; c < nn; ++c)
                for (I a = 0; a < na; ++a) L[a + c * na] = F[(nn + a) + c * nj];
        }
        /* send the update matrices to the children (selinv_send!, copygathertri!) */
        for (I p = chdptr[j]; p < chdptr[j + 1]; ++p) {
            const I i = chdtgt[p];
            const I ma = sepptr[i + 1] - sepptr[i];
            const I* inj = reltgt + sepptr[i];
            ns += 1;
            const I strt = Mptr[ns - 1];
            Mptr[ns] = strt + ma * ma;
            double* Mi = Mval + strt;
            for (I b = 0; b < ma; ++b)
                for (I a = b; a < ma; ++a) Mi[a + b * ma] = F[inj[a] + inj[b] * nj];
        }
    }
    free(Mptr); free(Mval); free(F);
    return 0;
}
