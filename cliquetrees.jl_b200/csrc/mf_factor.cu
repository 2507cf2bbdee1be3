// Numeric factorization kernels (FP64) for the B200 multifrontal solver.
//
// Per tree level (see mf_plan.cu):
//   k_small   : fronts with nj <= kSmallMax.  One CTA holds the whole frontal
//               matrix in shared memory: load the assembled panel, extend-add
//               the children's update matrices, partial LDL^T/Cholesky of the
//               first nn columns, write panel + update matrix.  This fuses
//               chol_loop_snd!/chol_loop_nod! (cholesky.jl:434-692) for the
//               many tiny fronts of a maximal-supernode tree.
//   k_ea      : extend-add for larger fronts, one CTA per (front, 16 parent
//               columns); each CTA owns its target columns, so the children
//               are added in a fixed order without atomics (addscattertri!,
//               utils.jl:555-579 via chol_send!, cholesky.jl:950-983).
//   k_diag    : per 64-column sub-panel, one CTA per front factors the
//               diagonal block in shared memory, writes it back and stores
//               the inverse of the factored block (potrf! of chol_factor!,
//               cholesky.jl:694-737);
//   k_gemm    : grouped 64x64 DMMA (mma.sync m8n8k4 f64) tile GEMM with a
//               cp.async double-buffered K loop, in four roles: left-looking
//               update of a sub-panel from its outer block, trailing update
//               of the panel after an outer block (K = 256), the TRSM of a
//               sub-panel as a product with the inverse of its diagonal
//               block, and M = F22 - L21 D L21^T with K = nn (syrk!,
//               blas/syrk.jl:137-159).
#include <climits>
#include <cstdio>

#include "mf_internal.cuh"

namespace mf {

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------

// pivot acceptance of NoRegularization (no_regularization.jl:27-42):
// a pivot whose sign disagrees with a nonzero requested sign is rejected,
// and a zero pivot is always rejected.
__device__ __forceinline__ bool pivot_ok(double s, double p) {
    if (s != 0.0 && !(s * p > 0.0)) return false;
    return p != 0.0;
}

__device__ __forceinline__ double pivot_sign(const double* signs, int ldlt, int64_t col) {
    if (!ldlt) return 1.0;
    return signs ? signs[col] : 0.0;
}

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// ---------------------------------------------------------------------------
// assembly and layout conversion
// ---------------------------------------------------------------------------

__global__ void k_scatter(double* __restrict__ P, const int64_t* __restrict__ slot, const double* __restrict__ v,
                          int64_t nnz) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < nnz; i += stride) P[slot[i]] = v[i];
}

// one warp per column: copy between the reference layout (Dval nn x nn,
// Lval na x nn of reference front j) and the panel of the execution front
// that holds j (nj x nn, ld nj): the D rows keep their order, the L rows go
// to sepmap positions.
template <bool TO_PANEL>
__global__ void k_dl_panel(const Front* __restrict__ fronts, const RefFront* __restrict__ ref,
                           const int32_t* __restrict__ colref, const int32_t* __restrict__ sepmap,
                           double* __restrict__ Dv, double* __restrict__ Lv, double* __restrict__ P, int64_t n) {
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const RefFront rf = ref[colref[warp]];
    const Front f = fronts[rf.exec];
    const int c = (int)(warp - rf.res0);
    const int off = rf.res0 - f.col0;
    double* pc = P + f.poff + (int64_t)(off + c) * f.ldp;
    double* dc = Dv + rf.Dptr + (int64_t)c * rf.nn;
    double* lc = Lv + rf.Lptr + (int64_t)c * rf.na;
    const int32_t* map = sepmap + rf.sep0;
    for (int r = lane; r < rf.nn; r += 32) {
        if (TO_PANEL) pc[off + r] = dc[r]; else dc[r] = pc[off + r];
    }
    for (int r = lane; r < rf.na; r += 32) {
        if (TO_PANEL) pc[map[r]] = lc[r]; else lc[r] = pc[map[r]];
    }
}

// ---------------------------------------------------------------------------
// small fronts: whole frontal matrix in shared memory
// ---------------------------------------------------------------------------
template <int LDLT>
__global__ void __launch_bounds__(256) k_small(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                               const int32_t* __restrict__ reltgt,
                                               const int32_t* __restrict__ chdtgt, double* __restrict__ P,
                                               double* __restrict__ M, double* __restrict__ d,
                                               const double* __restrict__ signs, long long* __restrict__ info) {
    extern __shared__ double F[];
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp;
    const int tid = threadIdx.x, nt = blockDim.x;
    double* Pj = P + f.poff;
    for (int i = tid; i < nj * nn; i += nt) {
        int r = i % nj, c = i / nj;
        F[i] = Pj[r + (int64_t)c * ld];
    }
    for (int i = tid; i < nj * na; i += nt) F[nj * nn + i] = 0.0;
    __syncthreads();
    // extend-add, children popped in reverse (cholesky.jl:506-514)
    for (int p = f.chd1 - 1; p >= f.chd0; --p) {
        const Front fc = fronts[chdtgt[p]];
        const int ma = fc.na, lm = fc.ldm;
        const int32_t* rel = reltgt + fc.sep0;
        const double* Mc = M + fc.moff;
        for (int i = tid; i < ma * ma; i += nt) {
            int a = i % ma, b = i / ma;
            if (a >= b) F[rel[a] + rel[b] * nj] += Mc[a + b * lm];
        }
        __syncthreads();
    }
    // right-looking partial factorization of the first nn columns
    for (int k = 0; k < nn; ++k) {
        double piv = F[k + k * nj];
        double s = pivot_sign(signs, LDLT, f.col0 + k);
        if (!pivot_ok(s, piv) || (!LDLT && !(piv > 0.0))) {
            if (tid == 0) atomicMin(info, (long long)(f.col0 + k + 1));
            return;  // uniform across the block
        }
        double dk = LDLT ? piv : sqrt(piv);
        double inv = 1.0 / dk;
        __syncthreads();
        if (tid == 0) {
            if (LDLT) d[f.col0 + k] = piv; else F[k + k * nj] = dk;
        }
        for (int i = k + 1 + tid; i < nj; i += nt) F[i + k * nj] *= inv;
        __syncthreads();
        const int m = nj - k - 1;
        for (int i = tid; i < m * m; i += nt) {
            int r = k + 1 + i % m, c = k + 1 + i / m;
            if (r >= c) {
                double lc = F[c + k * nj];
                if (LDLT) lc *= piv;
                F[r + c * nj] -= F[r + k * nj] * lc;
            }
        }
        __syncthreads();
    }
    for (int i = tid; i < nj * nn; i += nt) {
        int r = i % nj, c = i / nj;
        Pj[r + (int64_t)c * ld] = F[i];
    }
    double* Mj = M + f.moff;
    const int lm = f.ldm;
    for (int i = tid; i < na * na; i += nt) {
        int a = i % na, b = i / na;
        Mj[a + b * lm] = F[(nn + a) + (nn + b) * nj];
    }
}

// ---------------------------------------------------------------------------
// extend-add for blocked fronts
// ---------------------------------------------------------------------------
__device__ __forceinline__ int lower_bound_i32(const int32_t* a, int n, int v) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(256) k_ea(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                            const int32_t* __restrict__ reltgt, const int32_t* __restrict__ chdtgt,
                                            double* __restrict__ P, double* __restrict__ M) {
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp, lm = f.ldm;
    const int c0 = it.a * kEAcols, c1 = min(c0 + kEAcols, nj);
    const int tid = threadIdx.x, nt = blockDim.x;
    double* Pj = P + f.poff;
    double* Mj = M + f.moff;
    // zero the update-matrix columns this CTA owns
    for (int c = max(c0, nn); c < c1; ++c)
        for (int r = tid; r < na; r += nt) Mj[r + (int64_t)(c - nn) * lm] = 0.0;
    __syncthreads();
    for (int p = f.chd1 - 1; p >= f.chd0; --p) {
        const Front fc = fronts[chdtgt[p]];
        const int ma = fc.na, lmc = fc.ldm;
        const int32_t* rel = reltgt + fc.sep0;
        const double* Mc = M + fc.moff;
        const int b0 = lower_bound_i32(rel, ma, c0);
        const int b1 = lower_bound_i32(rel, ma, c1);
        for (int b = b0; b < b1; ++b) {
            const int col = rel[b];
            const double* mc = Mc + (int64_t)b * lmc;
            if (col < nn) {
                double* pc = Pj + (int64_t)col * ld;
                for (int a = b + tid; a < ma; a += nt) pc[rel[a]] += mc[a];
            } else {
                double* dst = Mj + (int64_t)(col - nn) * lm - nn;
                for (int a = b + tid; a < ma; a += nt) dst[rel[a]] += mc[a];
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// diagonal block: factor + inverse
// ---------------------------------------------------------------------------
constexpr int LDS = kNB + 4;  // shared-memory leading dimension (bank spread for DMMA fragments)

// Factor the w x w diagonal block in shared memory (lower, ld LDS).
// Returns the local failing column (0-based) or -1.  Must be called by all
// threads of the block.
template <int LDLT>
__device__ int factor_diag_block(double* Dk, double* piv, int w, const double* signs, int64_t col0) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int k = 0; k < w; ++k) {
        double p = Dk[k + k * LDS];
        double s = pivot_sign(signs, LDLT, col0 + k);
        if (!pivot_ok(s, p) || (!LDLT && !(p > 0.0))) return k;
        double dk = LDLT ? p : sqrt(p);
        double inv = 1.0 / dk;
        __syncthreads();
        if (tid == 0) {
            piv[k] = LDLT ? p : dk;
            if (!LDLT) Dk[k + k * LDS] = dk;
        }
        for (int i = k + 1 + tid; i < w; i += nt) Dk[i + k * LDS] *= inv;
        __syncthreads();
        const int m = w - k - 1;
        for (int i = tid; i < m * m; i += nt) {
            int r = k + 1 + i % m, c = k + 1 + i / m;
            if (r >= c) {
                double lc = Dk[c + k * LDS];
                if (LDLT) lc *= p;
                Dk[r + c * LDS] -= Dk[r + k * LDS] * lc;
            }
        }
        __syncthreads();
    }
    return -1;
}

// Inverse of the factored lower-triangular block (unit diagonal for LDLt)
// by row sweeps: X[i][j] = -(sum_{k=j}^{i-1} L[i][k] X[k][j]) / L[i][i].
template <int LDLT>
__device__ void invert_lower(const double* Dk, double* X, int w) {
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int i = tid; i < kNB * kNB; i += nt) X[i] = 0.0;
    __syncthreads();
    for (int i = 0; i < w; ++i) {
        const double lii = LDLT ? 1.0 : Dk[i + i * LDS];
        for (int j = tid; j <= i; j += nt) {
            double v;
            if (j == i) {
                v = 1.0 / lii;
            } else {
                double acc = 0.0;
                for (int k = j; k < i; ++k) acc += Dk[i + k * LDS] * X[k + j * kNB];
                v = -acc / lii;
            }
            X[i + j * kNB] = v;
        }
        __syncthreads();
    }
}

// Blocked factorization of a 64 x 64 diagonal block held in shared memory
// (lower, ld LDS; columns >= w are padded with the identity).  Four 16-wide
// steps: warp 0 factors the 16 x 16 diagonal sub-block with warp
// synchronisation only, then all threads solve the rows below it and apply
// the rank-16 update to the trailing block.  piv[k] receives sqrt(pivot)
// (Cholesky) or the pivot (LDLt).  Returns the first rejected local column
// (< w) or -1; called by all threads.
template <int LDLT>
__device__ int factor_diag64(double* Dk, double* piv, int w, const double* signs, int64_t col0, int* flag) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    for (int p = 0; p < 4; ++p) {
        const int pb = p * 16;
        if (warp == 0) {
            int bad = -1;
            for (int k = 0; k < 16; ++k) {
                const int c = pb + k;
                const double pv = Dk[c + c * LDS];
                if (c < w) {
                    const double sg = pivot_sign(signs, LDLT, col0 + c);
                    if (!pivot_ok(sg, pv) || (!LDLT && !(pv > 0.0))) { bad = c; break; }
                }
                const double dk = LDLT ? pv : sqrt(pv);
                const double inv = 1.0 / dk;
                __syncwarp();
                if (lane > k && lane < 16) Dk[(pb + lane) + c * LDS] *= inv;
                if (lane == 0) {
                    piv[c] = dk;
                    if (!LDLT) Dk[c + c * LDS] = dk;
                }
                __syncwarp();
                // rank-1 update of the rest of the 16 x 16 sub-block
                for (int e = lane; e < 256; e += 32) {
                    const int i = e & 15, j = e >> 4;
                    if (j > k && i >= j) {
                        double lj = Dk[(pb + j) + c * LDS];
                        if (LDLT) lj *= pv;
                        Dk[(pb + i) + (pb + j) * LDS] -= Dk[(pb + i) + c * LDS] * lj;
                    }
                }
                __syncwarp();
            }
            if (lane == 0) *flag = bad;
        }
        __syncthreads();
        if (*flag >= 0) return *flag;
        // rows below the sub-block: X <- X Lpp^{-T} (Cholesky) or X Lpp^{-T} D^{-1} (LDLt)
        for (int r = pb + 16 + tid; r < 64; r += nt) {
            for (int c = 0; c < 16; ++c) {
                double v = Dk[r + (pb + c) * LDS];
                for (int q = 0; q < c; ++q) v -= Dk[r + (pb + q) * LDS] * Dk[(pb + c) + (pb + q) * LDS];
                if (!LDLT) v /= piv[pb + c];
                Dk[r + (pb + c) * LDS] = v;
            }
            if (LDLT)
                for (int c = 0; c < 16; ++c) Dk[r + (pb + c) * LDS] /= piv[pb + c];
        }
        __syncthreads();
        // trailing update: rank 16
        const int m = 64 - pb - 16;
        for (int e = tid; e < m * m; e += nt) {
            const int i = pb + 16 + e % m, j = pb + 16 + e / m;
            if (i >= j) {
                double acc = 0.0;
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    double lj = Dk[j + (pb + q) * LDS];
                    if (LDLT) lj *= piv[pb + q];
                    acc += Dk[i + (pb + q) * LDS] * lj;
                }
                Dk[i + j * LDS] -= acc;
            }
        }
        __syncthreads();
    }
    return -1;
}

// Inverse X (ld 64) of the factored 64 x 64 lower block (unit diagonal for
// LDLt) in 16 x 16 blocks: the four diagonal blocks by one warp each, then
// X_ij = -X_ii (sum_{k=j}^{i-1} L_ik X_kj) along the block sub-diagonals.
template <int LDLT>
__device__ void invert_lower64(const double* Dk, double* X, double* T) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < kNB * kNB; i += nt) X[i] = 0.0;
    __syncthreads();
    if (warp < 4 && lane < 16) {
        const int b = warp * 16, j = lane;
        const double* L = Dk + b + b * LDS;
        double* Xb = X + b + b * kNB;
        Xb[j + j * kNB] = LDLT ? 1.0 : 1.0 / L[j + j * LDS];
        for (int i = j + 1; i < 16; ++i) {
            double acc = 0.0;
            for (int k = j; k < i; ++k) acc += L[i + k * LDS] * Xb[k + j * kNB];
            Xb[i + j * kNB] = LDLT ? -acc : -acc / L[i + i * LDS];
        }
    }
    __syncthreads();
    for (int dist = 1; dist < 4; ++dist) {
        const int nb = 4 - dist;  // blocks (jb + dist, jb) for jb = 0 .. nb-1
        // T_ij = sum_{k=j}^{i-1} L_ik X_kj   (16 x 16 per block)
        for (int e = tid; e < nb * 256; e += nt) {
            const int blk = e >> 8, r = (e >> 4) & 15, c = e & 15;
            const int ib = (blk + dist) * 16, jb = blk * 16;
            double acc = 0.0;
            for (int k = jb; k < ib; ++k) acc += Dk[(ib + r) + k * LDS] * X[k + (jb + c) * kNB];
            T[e] = acc;
        }
        __syncthreads();
        // X_ij = -X_ii T_ij
        for (int e = tid; e < nb * 256; e += nt) {
            const int blk = e >> 8, r = (e >> 4) & 15, c = e & 15;
            const int ib = (blk + dist) * 16, jb = blk * 16;
            double acc = 0.0;
            for (int k = 0; k <= r; ++k) acc += X[(ib + r) + (ib + k) * kNB] * T[(blk << 8) + (k << 4) + c];
            X[(ib + r) + (jb + c) * kNB] = -acc;
        }
        __syncthreads();
    }
}

template <int LDLT>
__global__ void __launch_bounds__(256) k_diag(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                              int c0, double* __restrict__ P, double* __restrict__ inv,
                                              double* __restrict__ d, const double* __restrict__ signs,
                                              long long* __restrict__ info) {
    extern __shared__ double smem[];
    double* Dk = smem;                 // kNB * LDS
    double* X = Dk + kNB * LDS;        // kNB * kNB
    double* T = X + kNB * kNB;         // 3 * 256
    double* piv = T + 3 * 256;         // kNB
    __shared__ int flag;
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, ld = f.ldp;
    const int w = min(kNB, nn - c0);
    const int tid = threadIdx.x, nt = blockDim.x;
    double* Pj = P + f.poff;
    for (int i = tid; i < kNB * kNB; i += nt) {
        int r = i & (kNB - 1), c = i >> 6;
        double v;
        if (r < w && c < w) v = Pj[(c0 + r) + (int64_t)(c0 + c) * ld];
        else v = (r == c) ? 1.0 : 0.0;
        Dk[r + c * LDS] = v;
    }
    __syncthreads();
    int bad = factor_diag64<LDLT>(Dk, piv, w, signs, (int64_t)f.col0 + c0, &flag);
    if (bad >= 0) {
        if (tid == 0) atomicMin(info, (long long)(f.col0 + c0 + bad + 1));
        return;
    }
    for (int i = tid; i < w * w; i += nt) {
        int r = i % w, c = i / w;
        if (r >= c) Pj[(c0 + r) + (int64_t)(c0 + c) * ld] = Dk[r + c * LDS];
    }
    if (LDLT)
        for (int i = tid; i < w; i += nt) d[f.col0 + c0 + i] = piv[i];
    invert_lower64<LDLT>(Dk, X, T);
    double* dst = inv + f.ioff + (int64_t)(c0 / kNB) * kNB * kNB;
    for (int i = tid; i < kNB * kNB; i += nt) {
        int r = i & (kNB - 1), c = i >> 6;
        dst[i] = (r < w && c < w) ? X[i] : 0.0;
    }
}

// ---------------------------------------------------------------------------
// DMMA tile GEMM with a cp.async double-buffered K loop.
// acc(64x64) += A(64 x K) * B(64 x K)^T, 8 warps; warp w owns rows
// (w&1)*32..+32 and columns (w>>1)*16..+16 as 4 x 2 fragments of 8 x 8.
// Shared tiles are [k][m] with m contiguous (leading dimension LDS).
// ---------------------------------------------------------------------------
constexpr int KC = 32;                   // K chunk per pipeline stage
constexpr int STAGE = KC * LDS;          // doubles per matrix per stage
constexpr int kGemmSmem = (4 * STAGE + 2 * KC) * (int)sizeof(double);

struct Acc {
    double c[4][2][2];
};

__device__ __forceinline__ void acc_zero(Acc& a) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) a.c[i][j][0] = a.c[i][j][1] = 0.0;
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool valid) {
    unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
    int n = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(src), "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// Stage one K chunk: rows ra..ra+63 of A (clamped at amax) and rows
// rb..rb+63 of B (clamped at bmax), columns k..k+kc-1, zero fill outside.
__device__ __forceinline__ void stage_chunk(double* As, double* Bs, const double* A, int64_t lda, int ra, int amax,
                                            const double* B, int64_t ldb, int rb, int bmax, int k, int kc) {
    for (int i = threadIdx.x; i < 64 * KC; i += blockDim.x) {
        int m = i & 63, kk = i >> 6;
        bool va = (ra + m < amax) && kk < kc;
        bool vb = (rb + m < bmax) && kk < kc;
        const double* sa = A + (va ? (ra + m) + (int64_t)(k + kk) * lda : 0);
        const double* sb = B + (vb ? (rb + m) + (int64_t)(k + kk) * ldb : 0);
        cp_async8(As + m + kk * LDS, sa, va);
        cp_async8(Bs + m + kk * LDS, sb, vb);
    }
}

__device__ __forceinline__ void mma_chunk(Acc& acc, const double* As, const double* Bs, const double* dsc, int kc) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wr = (warp & 1) * 32, wc = (warp >> 1) * 16;
    const int fr = lane >> 2, fk = lane & 3;
    for (int k = 0; k < kc; k += 4) {
        double a[4], b[2];
        const double s = dsc ? dsc[k + fk] : 1.0;
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[(wr + i * 8 + fr) + (k + fk) * LDS] * s;
#pragma unroll
        for (int j = 0; j < 2; ++j) b[j] = Bs[(wc + j * 8 + fr) + (k + fk) * LDS];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) dmma(acc.c[i][j][0], acc.c[i][j][1], a[i], b[j]);
    }
}

// acc += A[ra.., kbeg..kend) * B[rb.., kbeg..kend)^T (optionally D-scaled)
__device__ void gemm_k_loop(Acc& acc, double* smem, const double* A, int64_t lda, int ra, int amax, const double* B,
                            int64_t ldb, int rb, int bmax, int kbeg, int kend, const double* dvec) {
    double* As[2] = {smem, smem + STAGE};
    double* Bs[2] = {smem + 2 * STAGE, smem + 3 * STAGE};
    double* Ds[2] = {smem + 4 * STAGE, smem + 4 * STAGE + KC};
    const int nchunk = (kend - kbeg + KC - 1) / KC;
    if (nchunk <= 0) return;
    auto load = [&](int c, int st) {
        int k = kbeg + c * KC;
        int kc = min(KC, kend - k);
        stage_chunk(As[st], Bs[st], A, lda, ra, amax, B, ldb, rb, bmax, k, kc);
        if (dvec)
            for (int i = threadIdx.x; i < KC; i += blockDim.x) Ds[st][i] = i < kc ? dvec[k + i] : 0.0;
        cp_commit();
    };
    load(0, 0);
    for (int c = 0; c < nchunk; ++c) {
        const int st = c & 1;
        if (c + 1 < nchunk) {
            load(c + 1, st ^ 1);
            cp_wait<1>();
        } else {
            cp_wait<0>();
        }
        __syncthreads();
        int kc = min(KC, kend - (kbeg + c * KC));
        mma_chunk(acc, As[st], Bs[st], dvec ? Ds[st] : nullptr, (kc + 3) & ~3);
        __syncthreads();
    }
}

// C(rbase+r, cbase+c) -= acc (or = acc * colscale when OVERWRITE), for
// r < rmax, c < cmax; on a diagonal tile only row >= col is written.
template <bool OVERWRITE>
__device__ __forceinline__ void acc_store(const Acc& acc, double* C, int64_t ldc, int rbase, int cbase, int rmax,
                                          int cmax, bool diag_tile, const double* colscale) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wr = (warp & 1) * 32, wc = (warp >> 1) * 16;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                int r = wr + i * 8 + (lane >> 2);
                int c = wc + j * 8 + (lane & 3) * 2 + e;
                if (r < rmax && c < cmax && (!diag_tile || rbase + r >= cbase + c)) {
                    double* p = C + (rbase + r) + (int64_t)(cbase + c) * ldc;
                    if (OVERWRITE) *p = colscale ? acc.c[i][j][e] * colscale[c] : acc.c[i][j][e];
                    else *p -= acc.c[i][j][e];
                }
            }
}

enum GemmRole { G_LEFT = 0, G_TRAIL = 1, G_SYRK = 2, G_TRSM = 3 };

template <int ROLE, int LDLT>
__global__ void __launch_bounds__(256) k_gemm(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                              int ob, int c0, double* __restrict__ P, double* __restrict__ M,
                                              const double* __restrict__ d, const double* __restrict__ inv) {
    extern __shared__ double smem[];
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp;
    double* Pj = P + f.poff;
    const double* dj = LDLT ? d + f.col0 : nullptr;
    Acc acc;
    acc_zero(acc);
    if (ROLE == G_LEFT) {
        // sub-panel [c0, c0+w) rows [c0 + 64 a, ..) -= panel cols [ob*kOB, c0)
        const int w = min(kNB, nn - c0);
        const int rs = c0 + it.a * kTile;
        gemm_k_loop(acc, smem, Pj, ld, rs, nj, Pj, ld, c0, c0 + w, ob * kOB, c0, dj);
        acc_store<false>(acc, Pj, ld, rs, c0, nj - rs, w, it.a == 0, nullptr);
    } else if (ROLE == G_TRAIL) {
        const int e = min(nn, (ob + 1) * kOB);
        const int cs = e + it.b * kTile, rs = cs + it.a * kTile;
        gemm_k_loop(acc, smem, Pj, ld, rs, nj, Pj, ld, cs, nn, ob * kOB, e, dj);
        acc_store<false>(acc, Pj, ld, rs, cs, nj - rs, nn - cs, it.a == 0, nullptr);
    } else if (ROLE == G_SYRK) {
        const int rs = it.a * kTile, cs = it.b * kTile;
        gemm_k_loop(acc, smem, Pj + nn, ld, rs, na, Pj + nn, ld, cs, na, 0, nn, dj);
        acc_store<false>(acc, M + f.moff, f.ldm, rs, cs, na - rs, na - cs, it.a == it.b, nullptr);
    } else {
        // X (rows below the diagonal block, cols [c0, c0+w)) = X * Linv^T (* D^-1)
        const int w = min(kNB, nn - c0);
        const int rs = c0 + w + it.a * kTile;
        const double* Li = inv + f.ioff + (int64_t)(c0 / kNB) * kNB * kNB;
        gemm_k_loop(acc, smem, Pj + (int64_t)c0 * ld, ld, rs, nj, Li - 0, kNB, 0, w, 0, w, nullptr);
        __syncthreads();
        double* sc = smem;  // reuse: reciprocal pivots for LDLt
        if (LDLT) {
            for (int i = threadIdx.x; i < w; i += blockDim.x) sc[i] = 1.0 / dj[c0 + i];
            __syncthreads();
        }
        acc_store<true>(acc, Pj + (int64_t)c0 * ld, ld, rs, 0, nj - rs, w, false, LDLT ? sc : nullptr);
    }
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
Timer::Timer(mf_handle* h_, int k_) : h(h_), k(k_) {
    if (!h->profile) return;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, h->stream);
}

Timer::~Timer() {
    if (!h->profile) return;
    cudaEventRecord(b, h->stream);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    h->times.ms[k] += ms;
    h->times.launches[k] += 1;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
}

static inline unsigned grid_for(int64_t cnt) { return (unsigned)cnt; }

int launch_assemble(mf_handle* h, const double* dnz) {
    Timer t(h, K_ASSEMBLE);
    MF_CUDA(cudaMemsetAsync(h->d_P, 0, sizeof(double) * h->npanel, h->stream));
    if (h->nnz > 0) {
        int64_t blocks = (h->nnz + 255) / 256;
        if (blocks > 148 * 16) blocks = 148 * 16;
        k_scatter<<<(unsigned)blocks, 256, 0, h->stream>>>(h->d_P, h->d_pslot, dnz, h->nnz);
        MF_CUDA(cudaGetLastError());
    }
    return 0;
}

int launch_dl_to_panel(mf_handle* h, const double* dD, const double* dL) {
    Timer t(h, K_OTHER);
    if (h->n == 0) return 0;
    int64_t threads = h->n * 32;
    unsigned blocks = (unsigned)((threads + 255) / 256);
    MF_CUDA(cudaMemsetAsync(h->d_P, 0, sizeof(double) * h->npanel, h->stream));
    k_dl_panel<true><<<blocks, 256, 0, h->stream>>>(h->d_fronts, h->d_ref, h->d_colfront, h->d_sepmap,
                                                     const_cast<double*>(dD), const_cast<double*>(dL), h->d_P, h->n);
    MF_CUDA(cudaGetLastError());
    return 0;
}

int launch_panel_to_dl(mf_handle* h, double* dD, double* dL) {
    Timer t(h, K_OTHER);
    if (h->n == 0) return 0;
    int64_t threads = h->n * 32;
    unsigned blocks = (unsigned)((threads + 255) / 256);
    k_dl_panel<false><<<blocks, 256, 0, h->stream>>>(h->d_fronts, h->d_ref, h->d_colfront, h->d_sepmap, dD, dL,
                                                      h->d_P, h->n);
    MF_CUDA(cudaGetLastError());
    return 0;
}

constexpr int kDiagSmem = (kNB * LDS + kNB * kNB + 3 * 256 + kNB) * (int)sizeof(double);

template <int LDLT>
static int factor_impl(mf_handle* h) {
    MF_CUDA(cudaFuncSetAttribute(k_small<LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kSmallMax * kSmallMax * (int)sizeof(double)));
    MF_CUDA(cudaFuncSetAttribute(k_diag<LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDiagSmem));
    MF_CUDA(cudaFuncSetAttribute(k_gemm<G_LEFT, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem));
    MF_CUDA(cudaFuncSetAttribute(k_gemm<G_TRAIL, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem));
    MF_CUDA(cudaFuncSetAttribute(k_gemm<G_SYRK, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem));
    MF_CUDA(cudaFuncSetAttribute(k_gemm<G_TRSM, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem));
    const Item* items = h->d_items;
    for (const Level& lv : h->levels) {
        if (lv.small.cnt) {
            Timer t(h, K_SMALL);
            k_small<LDLT><<<grid_for(lv.small.cnt), 256, kSmallMax * kSmallMax * sizeof(double), h->stream>>>(
                h->d_fronts, items + lv.small.off, h->d_reltgt, h->d_chdtgt, h->d_P, h->d_M, h->d_d, h->d_signs,
                h->d_info);
            MF_CUDA(cudaGetLastError());
        }
        if (lv.ea.cnt) {
            Timer t(h, K_EA);
            k_ea<<<grid_for(lv.ea.cnt), 256, 0, h->stream>>>(h->d_fronts, items + lv.ea.off, h->d_reltgt,
                                                             h->d_chdtgt, h->d_P, h->d_M);
            MF_CUDA(cudaGetLastError());
        }
        for (const PanelStep& st : lv.steps) {
            const int c0 = st.b * kOB + st.s * kNB;
            if (st.left.cnt) {
                Timer t(h, K_UPDATE);
                k_gemm<G_LEFT, LDLT><<<grid_for(st.left.cnt), 256, kGemmSmem, h->stream>>>(
                    h->d_fronts, items + st.left.off, st.b, c0, h->d_P, h->d_M, h->d_d, h->d_inv);
                MF_CUDA(cudaGetLastError());
            }
            if (st.diag.cnt) {
                Timer t(h, K_PANEL);
                k_diag<LDLT><<<grid_for(st.diag.cnt), 256, kDiagSmem, h->stream>>>(
                    h->d_fronts, items + st.diag.off, c0, h->d_P, h->d_inv, h->d_d, h->d_signs, h->d_info);
                MF_CUDA(cudaGetLastError());
            }
            if (st.panel.cnt) {
                Timer t(h, K_PANEL);
                k_gemm<G_TRSM, LDLT><<<grid_for(st.panel.cnt), 256, kGemmSmem, h->stream>>>(
                    h->d_fronts, items + st.panel.off, st.b, c0, h->d_P, h->d_M, h->d_d, h->d_inv);
                MF_CUDA(cudaGetLastError());
            }
            if (st.trail.cnt) {
                Timer t(h, K_UPDATE);
                k_gemm<G_TRAIL, LDLT><<<grid_for(st.trail.cnt), 256, kGemmSmem, h->stream>>>(
                    h->d_fronts, items + st.trail.off, st.b, c0, h->d_P, h->d_M, h->d_d, h->d_inv);
                MF_CUDA(cudaGetLastError());
            }
        }
        if (lv.syrk.cnt) {
            Timer t(h, K_SYRK);
            k_gemm<G_SYRK, LDLT><<<grid_for(lv.syrk.cnt), 256, kGemmSmem, h->stream>>>(
                h->d_fronts, items + lv.syrk.off, 0, 0, h->d_P, h->d_M, h->d_d, h->d_inv);
            MF_CUDA(cudaGetLastError());
        }
    }
    return 0;
}

int launch_factor(mf_handle* h) {
    return h->diag ? factor_impl<1>(h) : factor_impl<0>(h);
}

}  // namespace mf
