// Selected inversion of a Cholesky factor on the GPU: the entries of A^{-1}
// on the sparsity pattern of L, written over the factor (selinv!,
// src/Multifrontal.jl/src/selinv.jl:38-424).  FP64, Cholesky handles.
//
// The reference walks the fronts in reverse postorder with a LIFO stack of
// update matrices: front j receives M = Z[sep(j), sep(j)] gathered from its
// parent's frontal matrix, and computes
//     W   = L21 L11^{-1}                      (trsm!)
//     Z21 = -M W                              (symm!)
//     Z11 = L11^{-T} L11^{-1} - W^T Z21       (trtri!, syrk!, trrk!)
// then hands Z[sep(i), sep(i)] of its frontal matrix [Z11; Z21 M] to each
// child i.  Here the fronts (the execution fronts of the device plan; their
// extra structural zeros do not change the result on the reference pattern)
// are processed by depth: all fronts of one depth are independent, and each
// keeps its M (= Z22) in a pool slot until its children, one depth further
// down, have gathered from it, so two depth pools alternate.  Fronts with
// nj <= 96 run one CTA each, the whole computation in shared memory; larger
// fronts gather M with a grouped kernel and then run the dense steps as
// cuBLAS level-3 calls (dtrsm, dsymm, dsyr2k, dsyrk) on the handle's stream.
#include <cublas_v2.h>

#include <algorithm>
#include <vector>

#include "mf_internal.cuh"

namespace mf {

constexpr int kSelSmall = 96;  // fronts with nj <= kSelSmall: one CTA in shared memory

// M (na x na, lower triangle, leading dimension na) of front j gathered from
// its parent's frontal matrix: columns of the parent's residual from its
// panel (Z11 / Z21 after its own selected inversion), the rest from the
// parent's M slot.
__device__ __forceinline__ double parent_entry(const Front& fp, const double* Pp, const double* Mp, int r, int c) {
    if (c < fp.nn) return Pp[r + (int64_t)c * fp.ldp];
    return Mp[(r - fp.nn) + (int64_t)(c - fp.nn) * fp.na];
}

// Gather M of the big fronts of one depth: item (front, 64-column tile).
__global__ void __launch_bounds__(256) k_sel_gather(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                    const int32_t* __restrict__ reltgt,
                                                    const int64_t* __restrict__ slot, const double* __restrict__ P,
                                                    double* __restrict__ pool) {
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const Front fp = fronts[f.parent];
    const int na = f.na;
    const int32_t* rel = reltgt + f.sep0;
    const double* Pp = P + fp.poff;
    const double* Mp = pool + slot[f.parent];
    double* M = pool + slot[it.front];
    const int b0 = it.a * 64, b1 = min(b0 + 64, na);
    for (int b = b0 + (threadIdx.x >> 5); b < b1; b += 8) {
        const int c = rel[b];
        for (int a = b + (threadIdx.x & 31); a < na; a += 32) M[a + (int64_t)b * na] = parent_entry(fp, Pp, Mp, rel[a], c);
    }
}

// One small front (nj <= kSelSmall) per CTA.  Shared memory: F (nj x nj,
// the frontal Z), Lp (nj x nn, the factor panel, W over its L21 rows), X
// (nn x nn, L11^{-1}).
__global__ void __launch_bounds__(256) k_sel_small(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                   const int32_t* __restrict__ reltgt,
                                                   const int64_t* __restrict__ slot, double* __restrict__ P,
                                                   double* __restrict__ pool) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp;
    double* F = reinterpret_cast<double*>(sm_raw);  // F[r + c * nj]
    double* Lp = F + nj * nj;                         // Lp[r + c * nj], r < nj, c < nn
    double* X = Lp + nj * nn;                         // X[r + c * nn]
    const int tid = threadIdx.x, nt = blockDim.x;
    double* Pj = P + f.poff;
    for (int i = tid; i < nj * nn; i += nt) {
        const int r = i % nj, c = i / nj;
        Lp[i] = Pj[r + (int64_t)c * ld];
    }
    for (int i = tid; i < nj * nj; i += nt) F[i] = 0.0;
    __syncthreads();
    if (na > 0) {
        // M from the parent into F22 (lower) and into this front's slot
        const Front fp = fronts[f.parent];
        const int32_t* rel = reltgt + f.sep0;
        const double* Pp = P + fp.poff;
        const double* Mp = pool + slot[f.parent];
        double* M = pool + slot[it.front];
        for (int i = tid; i < na * na; i += nt) {
            const int a = i % na, b = i / na;
            if (a >= b) {
                const double v = parent_entry(fp, Pp, Mp, rel[a], rel[b]);
                F[(nn + a) + (nn + b) * nj] = v;
                M[a + (int64_t)b * na] = v;
            }
        }
        __syncthreads();
        // W = L21 L11^{-1}: row a solves W L11 = L21 from the last column back
        for (int a = tid; a < na; a += nt) {
            double* w = Lp + nn + a;  // W[a, c] at w[c * nj]
            for (int c = nn - 1; c >= 0; --c) {
                double s = w[c * nj];
                for (int k = c + 1; k < nn; ++k) s -= w[k * nj] * Lp[k + c * nj];
                w[c * nj] = s / Lp[c + c * nj];
            }
        }
        __syncthreads();
        // Z21 = -M W (M symmetric, lower triangle in F22)
        for (int i = tid; i < na * nn; i += nt) {
            const int a = i % na, c = i / na;
            double s = 0.0;
            for (int b = 0; b < na; ++b) {
                const double m = a >= b ? F[(nn + a) + (nn + b) * nj] : F[(nn + b) + (nn + a) * nj];
                s += m * Lp[(nn + b) + c * nj];
            }
            F[(nn + a) + c * nj] = -s;
        }
    }
    // X = L11^{-1}: column c solves L11 x = e_c
    for (int c = tid; c < nn; c += nt) {
        for (int r = 0; r < c; ++r) X[r + c * nn] = 0.0;
        for (int r = c; r < nn; ++r) {
            double s = r == c ? 1.0 : 0.0;
            for (int k = c; k < r; ++k) s -= Lp[r + k * nj] * X[k + c * nn];
            X[r + c * nn] = s / Lp[r + r * nj];
        }
    }
    __syncthreads();
    // Z11 = X^T X - W^T Z21 (lower triangle; the upper triangle stays zero)
    for (int i = tid; i < nn * nn; i += nt) {
        const int r = i % nn, c = i / nn;
        if (r < c) continue;
        double s = 0.0;
        for (int k = r; k < nn; ++k) s += X[k + r * nn] * X[k + c * nn];
        for (int a = 0; a < na; ++a) s -= Lp[(nn + a) + r * nj] * F[(nn + a) + c * nj];
        F[r + c * nj] = s;
    }
    __syncthreads();
    for (int i = tid; i < nj * nn; i += nt) {
        const int r = i % nj, c = i / nj;
        Pj[r + (int64_t)c * ld] = (r >= nn || r >= c) ? F[i] : 0.0;
    }
}

// Big fronts: after cuBLAS has left Z11 (lower, nn x nn, leading dimension
// nn) and Z21 (na x nn, leading dimension na) in scratch, write them into
// the panel (the upper triangle of the diagonal block zero).
__global__ void k_sel_store(double* __restrict__ Pj, int ld, int nn, int na, const double* __restrict__ Z11,
                            const double* __restrict__ Z21) {
    const int nj = nn + na;
    const int64_t tot = (int64_t)nj * nn;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(i % nj), c = (int)(i / nj);
        double v;
        if (r < nn) v = r >= c ? Z11[r + (int64_t)c * nn] : 0.0;
        else v = Z21[(r - nn) + (int64_t)c * na];
        Pj[r + (int64_t)c * ld] = v;
    }
}

// X = identity (nn x nn) for the triangular inverse by dtrsm
__global__ void k_sel_eye(double* __restrict__ X, int nn) {
    const int64_t tot = (int64_t)nn * nn;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < tot; i += (int64_t)gridDim.x * blockDim.x)
        X[i] = (i % nn) == (i / nn) ? 1.0 : 0.0;
}

static int cublas_fail(cublasStatus_t s, const char* where) {
    set_error(std::string(where) + ": cuBLAS status " + std::to_string((int)s));
    return -3;
}

#define MF_CUBLAS(call)                                                  \
    do {                                                                 \
        cublasStatus_t _s = (call);                                      \
        if (_s != CUBLAS_STATUS_SUCCESS) return cublas_fail(_s, #call);  \
    } while (0)

int launch_selinv(mf_handle* h) {
    // allocations, frees and cuBLAS setup below must not meet another
    // thread's stream capture
    std::lock_guard<std::recursive_mutex> lk(device_mutex());
    if (h->diag) { set_error("mf_selinv: selected inversion is defined for Cholesky factorizations"); return -1; }
    if (!have_fp64(h) || (h->mixed && !h->fp64_current)) {
        set_error("mf_selinv: needs the FP64 factor of the current matrix (mf_factorize)");
        return -1;
    }
    const int64_t nex = h->nexec;
    if (nex == 0) return 0;
    // depths (root 0) and, per depth, the small and the big fronts
    std::vector<int> depth((size_t)nex, 0);
    int maxd = 0;
    for (int64_t e = nex - 1; e >= 0; --e) {  // postorder: parents after children
        const int p = h->h_fronts[(size_t)e].parent;
        depth[(size_t)e] = p < 0 ? 0 : depth[(size_t)p] + 1;
        maxd = std::max(maxd, depth[(size_t)e]);
    }
    std::vector<std::vector<int32_t>> small((size_t)maxd + 1), big((size_t)maxd + 1);
    for (int64_t e = 0; e < nex; ++e) {
        const Front& f = h->h_fronts[(size_t)e];
        (f.nn + f.na <= kSelSmall ? small : big)[(size_t)depth[(size_t)e]].push_back((int32_t)e);
    }
    // M slots: depth parity pools, each sized for its largest depth
    std::vector<int64_t> slot((size_t)nex, 0);
    int64_t psize[2] = {0, 0};
    for (int d = 0; d <= maxd; ++d) {
        int64_t off = 0;
        for (auto* lst : {&small[(size_t)d], &big[(size_t)d]})
            for (int32_t e : *lst) {
                const Front& f = h->h_fronts[(size_t)e];
                slot[(size_t)e] = off;
                off += ((int64_t)f.na * f.na + 31) & ~int64_t(31);
            }
        psize[d & 1] = std::max(psize[d & 1], off);
    }
    for (int d = 0; d <= maxd; ++d)
        for (auto* lst : {&small[(size_t)d], &big[(size_t)d]})
            for (int32_t e : *lst)
                if (d & 1) slot[(size_t)e] += psize[0];
    // scratch of the largest big front: Z21 (na x nn), Z11 and X (nn x nn)
    int64_t scratch = 1;
    std::vector<Item> items;
    std::vector<int64_t> small_off((size_t)maxd + 2), gather_off((size_t)maxd + 2);
    for (int d = 0; d <= maxd; ++d) {
        small_off[(size_t)d] = (int64_t)items.size();
        for (int32_t e : small[(size_t)d]) items.push_back(Item{e, 0, 0, 0});
        gather_off[(size_t)d] = (int64_t)items.size();
        for (int32_t e : big[(size_t)d]) {
            const Front& f = h->h_fronts[(size_t)e];
            scratch = std::max(scratch, (int64_t)f.na * f.nn + 2 * (int64_t)f.nn * f.nn);
            if (f.na > 0)
                for (int t = 0; t < (f.na + 63) / 64; ++t) items.push_back(Item{e, t, 0, 0});
        }
    }
    small_off[(size_t)maxd + 1] = gather_off[(size_t)maxd + 1] = (int64_t)items.size();
    const int64_t pool_doubles = std::max<int64_t>(psize[0] + psize[1], 1);
    double *pool = nullptr, *scr = nullptr;
    int64_t* dslot = nullptr;
    Item* ditems = nullptr;
    auto cleanup = [&]() {
        cudaStreamSynchronize(h->stream);
        if (pool) cudaFree(pool);
        if (scr) cudaFree(scr);
        if (dslot) cudaFree(dslot);
        if (ditems) cudaFree(ditems);
    };
    cudaError_t e = cudaMalloc((void**)&pool, sizeof(double) * pool_doubles);
    if (e == cudaSuccess) e = cudaMalloc((void**)&scr, sizeof(double) * scratch);
    if (e == cudaSuccess) e = cudaMalloc((void**)&dslot, sizeof(int64_t) * nex);
    if (e == cudaSuccess) e = cudaMalloc((void**)&ditems, sizeof(Item) * std::max<size_t>(items.size(), 1));
    if (e == cudaSuccess) e = cudaMemcpy(dslot, slot.data(), sizeof(int64_t) * nex, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !items.empty())
        e = cudaMemcpy(ditems, items.data(), sizeof(Item) * items.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        set_error(std::string("mf_selinv: device allocation failed: ") + cudaGetErrorString(e));
        return -4;
    }
    if (!h->cublas) {
        cublasHandle_t cb = nullptr;
        if (cublasCreate(&cb) != CUBLAS_STATUS_SUCCESS) { cleanup(); set_error("mf_selinv: cublasCreate failed"); return -3; }
        h->cublas = cb;
    }
    cublasHandle_t cb = static_cast<cublasHandle_t>(h->cublas);
    int rc = 0;
    auto body = [&]() -> int {
        MF_CUBLAS(cublasSetStream(cb, h->stream));
        MF_CUBLAS(cublasSetPointerMode(cb, CUBLAS_POINTER_MODE_HOST));
        const int smem_max = (kSelSmall * kSelSmall * 3) * (int)sizeof(double);
        MF_CUDA(cudaFuncSetAttribute(k_sel_small, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max));
        const double one = 1.0, zero = 0.0, mone = -1.0, mhalf = -0.5;
        for (int d = 0; d <= maxd; ++d) {
            const int64_t ns = gather_off[(size_t)d] - small_off[(size_t)d];
            if (ns > 0) {
                k_sel_small<<<(unsigned)ns, 256, smem_max, h->stream>>>(h->d_fronts, ditems + small_off[(size_t)d],
                                                                         h->d_reltgt, dslot, h->d_P, pool);
                MF_CUDA(cudaGetLastError());
            }
            const int64_t ng = small_off[(size_t)d + 1] - gather_off[(size_t)d];
            if (ng > 0) {
                k_sel_gather<<<(unsigned)ng, 256, 0, h->stream>>>(h->d_fronts, ditems + gather_off[(size_t)d],
                                                                  h->d_reltgt, dslot, h->d_P, pool);
                MF_CUDA(cudaGetLastError());
            }
            for (int32_t ef : big[(size_t)d]) {
                const Front& f = h->h_fronts[(size_t)ef];
                const int nn = f.nn, na = f.na, ld = f.ldp;
                double* Pj = h->d_P + f.poff;
                double* Z21 = scr;
                double* Z11 = scr + (int64_t)na * nn;
                double* X = Z11 + (int64_t)nn * nn;
                double* M = pool + slot[(size_t)ef];
                if (na > 0) {
                    // W = L21 L11^{-1} in place of L21
                    MF_CUBLAS(cublasDtrsm(cb, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N,
                                          CUBLAS_DIAG_NON_UNIT, na, nn, &one, Pj, ld, Pj + nn, ld));
                    // Z21 = -M W
                    MF_CUBLAS(cublasDsymm(cb, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, na, nn, &mone, M, na,
                                          Pj + nn, ld, &zero, Z21, na));
                    // Z11 = -(W^T Z21 + Z21^T W) / 2 (lower)
                    MF_CUBLAS(cublasDsyr2k(cb, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, nn, na, &mhalf, Pj + nn, ld, Z21,
                                           na, &zero, Z11, nn));
                }
                // X = L11^{-1}; Z11 += X^T X
                k_sel_eye<<<296, 256, 0, h->stream>>>(X, nn);
                MF_CUDA(cudaGetLastError());
                MF_CUBLAS(cublasDtrsm(cb, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT,
                                      nn, nn, &one, Pj, ld, X, nn));
                const double beta = na > 0 ? 1.0 : 0.0;
                MF_CUBLAS(cublasDsyrk(cb, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, nn, nn, &one, X, nn, &beta, Z11, nn));
                k_sel_store<<<296, 256, 0, h->stream>>>(Pj, ld, nn, na, Z11, Z21);
                MF_CUDA(cudaGetLastError());
            }
        }
        return 0;
    };
    rc = body();
    cleanup();
    if (rc) return rc;
    h->fp64_current = false;  // the panels now hold the selected inverse, not a factor
    h->selinv_done = true;
    release_graphs(h);
    return 0;
}

}  // namespace mf
