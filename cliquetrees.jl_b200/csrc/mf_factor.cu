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
//   k_panel   : per 64-column panel step: factor the diagonal block in
//               shared memory (every CTA of the front redundantly; CTA 0
//               writes it) and solve a 64-row tile of the panel below it
//               (potrf! + trsm! + cdiv! of chol_factor!, cholesky.jl:694-737).
//   k_update  : trailing update of the remaining panel columns with DMMA
//               (mma.sync m8n8k4 f64) 64x64 tiles.
//   k_syrk    : M = F22 - L21 D L21^T for the whole front at once, K = nn
//               (syrk!, blas/syrk.jl:137-159), DMMA 64x64 tiles.
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
// Lval na x nn) and the stacked panel (nj x nn, ld nj).
template <bool TO_PANEL>
__global__ void k_dl_panel(const Front* __restrict__ fronts, const int32_t* __restrict__ colfront,
                           const int64_t* __restrict__ Dptr, const int64_t* __restrict__ Lptr, double* __restrict__ Dv,
                           double* __restrict__ Lv, double* __restrict__ P, int64_t n) {
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= n) return;
    int j = colfront[warp];
    Front f = fronts[j];
    int c = (int)(warp - f.col0);
    int nj = f.nn + f.na;
    double* pc = P + f.poff + (int64_t)c * nj;
    double* dc = Dv + Dptr[j] + (int64_t)c * f.nn;
    double* lc = Lv + Lptr[j] + (int64_t)c * f.na;
    for (int r = lane; r < f.nn; r += 32) {
        if (TO_PANEL) pc[r] = dc[r]; else dc[r] = pc[r];
    }
    for (int r = lane; r < f.na; r += 32) {
        if (TO_PANEL) pc[f.nn + r] = lc[r]; else lc[r] = pc[f.nn + r];
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
    const int nn = f.nn, na = f.na, nj = nn + na;
    const int tid = threadIdx.x, nt = blockDim.x;
    double* Pj = P + f.poff;
    for (int i = tid; i < nj * nn; i += nt) F[i] = Pj[i];
    for (int i = tid; i < nj * na; i += nt) F[nj * nn + i] = 0.0;
    __syncthreads();
    // extend-add, children popped in reverse (cholesky.jl:506-514)
    for (int p = f.chd1 - 1; p >= f.chd0; --p) {
        const Front fc = fronts[chdtgt[p]];
        const int ma = fc.na;
        const int32_t* rel = reltgt + fc.sep0;
        const double* Mc = M + fc.moff;
        for (int i = tid; i < ma * ma; i += nt) {
            int a = i % ma, b = i / ma;
            if (a >= b) F[rel[a] + rel[b] * nj] += Mc[i];
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
    for (int i = tid; i < nj * nn; i += nt) Pj[i] = F[i];
    double* Mj = M + f.moff;
    for (int i = tid; i < na * na; i += nt) {
        int a = i % na, b = i / na;
        Mj[i] = F[(nn + a) + (nn + b) * nj];
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
    const int nn = f.nn, na = f.na, nj = nn + na;
    const int c0 = it.a * kEAcols, c1 = min(c0 + kEAcols, nj);
    const int tid = threadIdx.x, nt = blockDim.x;
    double* Pj = P + f.poff;
    double* Mj = M + f.moff;
    // zero the update-matrix columns this CTA owns
    for (int c = max(c0, nn); c < c1; ++c)
        for (int r = tid; r < na; r += nt) Mj[r + (int64_t)(c - nn) * na] = 0.0;
    __syncthreads();
    for (int p = f.chd1 - 1; p >= f.chd0; --p) {
        const Front fc = fronts[chdtgt[p]];
        const int ma = fc.na;
        const int32_t* rel = reltgt + fc.sep0;
        const double* Mc = M + fc.moff;
        const int b0 = lower_bound_i32(rel, ma, c0);
        const int b1 = lower_bound_i32(rel, ma, c1);
        // flatten (column b, row a >= b) pairs of the owned columns
        for (int b = b0; b < b1; ++b) {
            const int col = rel[b];
            const double* mc = Mc + (int64_t)b * ma;
            if (col < nn) {
                double* pc = Pj + (int64_t)col * nj;
                for (int a = b + tid; a < ma; a += nt) pc[rel[a]] += mc[a];
            } else {
                double* dst = Mj + (int64_t)(col - nn) * na - nn;
                for (int a = b + tid; a < ma; a += nt) dst[rel[a]] += mc[a];
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// blocked path: panel step (diag factor + panel solve)
// ---------------------------------------------------------------------------
constexpr int LDS = kNB + 4;  // shared-memory leading dimension (bank spread for DMMA fragments)
constexpr int kPanelSmem = (kNB * LDS + kTile * LDS + kNB) * (int)sizeof(double);
constexpr int kTileSmem = (2 * kTile * LDS + kNB) * (int)sizeof(double);

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

template <int LDLT>
__global__ void __launch_bounds__(256) k_panel(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                               int step, double* __restrict__ P, double* __restrict__ d,
                                               const double* __restrict__ signs, long long* __restrict__ info) {
    extern __shared__ double smem[];
    double* Dk = smem;
    double* X = Dk + kNB * LDS;
    double* piv = X + kTile * LDS;
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, nj = nn + f.na;
    const int k0 = step * kNB;
    const int w = min(kNB, nn - k0);
    const int tid = threadIdx.x, nt = blockDim.x;
    double* Pj = P + f.poff;
    for (int i = tid; i < w * w; i += nt) {
        int r = i % w, c = i / w;
        Dk[r + c * LDS] = Pj[(k0 + r) + (int64_t)(k0 + c) * nj];
    }
    __syncthreads();
    int bad = factor_diag_block<LDLT>(Dk, piv, w, signs, (int64_t)f.col0 + k0);
    if (bad >= 0) {
        if (it.a == 0 && tid == 0) atomicMin(info, (long long)(f.col0 + k0 + bad + 1));
        return;
    }
    __syncthreads();
    if (it.a == 0) {
        for (int i = tid; i < w * w; i += nt) {
            int r = i % w, c = i / w;
            if (r >= c) Pj[(k0 + r) + (int64_t)(k0 + c) * nj] = Dk[r + c * LDS];
        }
        if (LDLT)
            for (int i = tid; i < w; i += nt) d[f.col0 + k0 + i] = piv[i];
        return;
    }
    const int r0 = k0 + w + (it.a - 1) * kTile;
    const int nr = min(kTile, nj - r0);
    for (int i = tid; i < nr * w; i += nt) {
        int r = i % nr, c = i / nr;
        X[r + c * LDS] = Pj[(r0 + r) + (int64_t)(k0 + c) * nj];
    }
    __syncthreads();
    // X <- X Dk^{-T}  (Cholesky) or X <- X Dk^{-T} diag(piv)^{-1} (LDLt, unit Dk)
    for (int c = 0; c < w; ++c) {
        if (!LDLT) {
            double inv = 1.0 / piv[c];
            for (int r = tid; r < nr; r += nt) X[r + c * LDS] *= inv;
            __syncthreads();
        }
        const int m = w - c - 1;
        for (int i = tid; i < nr * m; i += nt) {
            int r = i % nr, cc = c + 1 + i / nr;
            X[r + cc * LDS] -= X[r + c * LDS] * Dk[cc + c * LDS];
        }
        __syncthreads();
    }
    if (LDLT) {
        for (int i = tid; i < nr * w; i += nt) {
            int r = i % nr, c = i / nr;
            X[r + c * LDS] *= 1.0 / piv[c];
        }
        __syncthreads();
    }
    for (int i = tid; i < nr * w; i += nt) {
        int r = i % nr, c = i / nr;
        Pj[(r0 + r) + (int64_t)(k0 + c) * nj] = X[r + c * LDS];
    }
}

// ---------------------------------------------------------------------------
// DMMA tile core: acc(64x64) += A(64 x kc) * B(64 x kc)^T, smem column major
// with leading dimension LDS.  8 warps; warp w owns rows (w&1)*32..+32 and
// columns (w>>1)*16..+16 as 4 x 2 fragments of 8 x 8.
// ---------------------------------------------------------------------------
struct Acc {
    double c[4][2][2];
};

__device__ __forceinline__ void acc_zero(Acc& a) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) a.c[i][j][0] = a.c[i][j][1] = 0.0;
}

__device__ __forceinline__ void mma_tile(Acc& acc, const double* As, const double* Bs, int kc) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wr = (warp & 1) * 32, wc = (warp >> 1) * 16;
    const int fr = lane >> 2, fk = lane & 3;
    for (int k = 0; k < kc; k += 4) {
        double a[4], b[2];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[(wr + i * 8 + fr) + (k + fk) * LDS];
#pragma unroll
        for (int j = 0; j < 2; ++j) b[j] = Bs[(wc + j * 8 + fr) + (k + fk) * LDS];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) dmma(acc.c[i][j][0], acc.c[i][j][1], a[i], b[j]);
    }
}

// C(rows, cols) -= acc for the rows/cols inside the matrix; on a diagonal
// tile only the lower triangle (row >= col) is written.
__device__ __forceinline__ void acc_sub_store(const Acc& acc, double* C, int64_t ldc, int rbase, int cbase, int rmax,
                                              int cmax, bool diag_tile) {
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
                if (r < rmax && c < cmax && (!diag_tile || rbase + r >= cbase + c))
                    C[(rbase + r) + (int64_t)(cbase + c) * ldc] -= acc.c[i][j][e];
            }
}

// load a (64 x kc) block of a column-major matrix (rows r0.., cols c0..)
// into smem (ld LDS), zero-filling rows >= rmax; optionally scale column c
// by scale[c].
__device__ __forceinline__ void load_block(double* S, const double* G, int64_t ldg, int r0, int rmax, int c0, int kc,
                                           const double* scale) {
    for (int i = threadIdx.x; i < kTile * kc; i += blockDim.x) {
        int r = i % kTile, c = i / kTile;
        double v = 0.0;
        if (r0 + r < rmax) {
            v = G[(r0 + r) + (int64_t)(c0 + c) * ldg];
            if (scale) v *= scale[c];
        }
        S[r + c * LDS] = v;
    }
}

// trailing update inside the panel after step `step`
template <int LDLT>
__global__ void __launch_bounds__(256) k_update(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                int step, double* __restrict__ P, const double* __restrict__ d) {
    extern __shared__ double smem[];
    double* As = smem;
    double* Bs = As + kTile * LDS;
    double* sc = Bs + kTile * LDS;
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, nj = nn + f.na;
    const int k0 = step * kNB;
    const int w = min(kNB, nn - k0);
    const int cs = k0 + w + it.b * kTile;   // first column of the tile
    const int rs = cs + it.a * kTile;       // first row of the tile
    double* Pj = P + f.poff;
    if (LDLT) {
        for (int i = threadIdx.x; i < w; i += blockDim.x) sc[i] = d[f.col0 + k0 + i];
        __syncthreads();
    }
    load_block(As, Pj, nj, rs, nj, k0, w, nullptr);
    load_block(Bs, Pj, nj, cs, nn, k0, w, LDLT ? sc : nullptr);
    // pad k to a multiple of 4 with zeros
    int kc = (w + 3) & ~3;
    for (int i = threadIdx.x; i < kTile * (kc - w); i += blockDim.x) {
        int r = i % kTile, c = w + i / kTile;
        As[r + c * LDS] = 0.0; Bs[r + c * LDS] = 0.0;
    }
    __syncthreads();
    Acc acc;
    acc_zero(acc);
    mma_tile(acc, As, Bs, kc);
    acc_sub_store(acc, Pj, nj, rs, cs, nj - rs, nn - cs, it.a == 0);
}

// M -= L D L^T over the whole front (K = nn), K in chunks of 32
template <int LDLT>
__global__ void __launch_bounds__(256) k_syrk(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                              const double* __restrict__ P, double* __restrict__ M,
                                              const double* __restrict__ d) {
    constexpr int KC = 32;
    extern __shared__ double smem[];
    double* As = smem;
    double* Bs = As + kTile * LDS;
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, na = f.na, nj = nn + na;
    const int rs = it.a * kTile, cs = it.b * kTile;
    const double* Pj = P + f.poff;
    const double* dj = LDLT ? d + f.col0 : nullptr;
    Acc acc;
    acc_zero(acc);
    for (int k = 0; k < nn; k += KC) {
        int kc = min(KC, nn - k);
        int kp = (kc + 3) & ~3;
        for (int i = threadIdx.x; i < kTile * kp; i += blockDim.x) {
            int r = i % kTile, c = i / kTile;
            double a = 0.0, b = 0.0;
            if (c < kc) {
                if (rs + r < na) a = Pj[(nn + rs + r) + (int64_t)(k + c) * nj];
                if (cs + r < na) {
                    b = Pj[(nn + cs + r) + (int64_t)(k + c) * nj];
                    if (LDLT) b *= dj[k + c];
                }
            }
            As[r + c * LDS] = a;
            Bs[r + c * LDS] = b;
        }
        __syncthreads();
        mma_tile(acc, As, Bs, kp);
        __syncthreads();
    }
    acc_sub_store(acc, M + f.moff, na, rs, cs, na - rs, na - cs, it.a == it.b);
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
    k_dl_panel<true><<<blocks, 256, 0, h->stream>>>(h->d_fronts, h->d_colfront, h->d_Dptr, h->d_Lptr,
                                                     const_cast<double*>(dD), const_cast<double*>(dL), h->d_P, h->n);
    MF_CUDA(cudaGetLastError());
    return 0;
}

int launch_panel_to_dl(mf_handle* h, double* dD, double* dL) {
    Timer t(h, K_OTHER);
    if (h->n == 0) return 0;
    int64_t threads = h->n * 32;
    unsigned blocks = (unsigned)((threads + 255) / 256);
    k_dl_panel<false><<<blocks, 256, 0, h->stream>>>(h->d_fronts, h->d_colfront, h->d_Dptr, h->d_Lptr, dD, dL,
                                                      h->d_P, h->n);
    MF_CUDA(cudaGetLastError());
    return 0;
}

template <int LDLT>
static int factor_impl(mf_handle* h) {
    MF_CUDA(cudaFuncSetAttribute(k_small<LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kSmallMax * kSmallMax * (int)sizeof(double)));
    MF_CUDA(cudaFuncSetAttribute(k_panel<LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPanelSmem));
    MF_CUDA(cudaFuncSetAttribute(k_update<LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem));
    MF_CUDA(cudaFuncSetAttribute(k_syrk<LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem));
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
        for (size_t k = 0; k < lv.steps.size(); ++k) {
            const PanelStep& st = lv.steps[k];
            if (st.panel.cnt) {
                Timer t(h, K_PANEL);
                k_panel<LDLT><<<grid_for(st.panel.cnt), 256, kPanelSmem, h->stream>>>(
                    h->d_fronts, items + st.panel.off, (int)k, h->d_P, h->d_d, h->d_signs, h->d_info);
                MF_CUDA(cudaGetLastError());
            }
            if (st.update.cnt) {
                Timer t(h, K_UPDATE);
                k_update<LDLT><<<grid_for(st.update.cnt), 256, kTileSmem, h->stream>>>(h->d_fronts, items + st.update.off,
                                                                               (int)k, h->d_P, h->d_d);
                MF_CUDA(cudaGetLastError());
            }
        }
        if (lv.syrk.cnt) {
            Timer t(h, K_SYRK);
            k_syrk<LDLT><<<grid_for(lv.syrk.cnt), 256, kTileSmem, h->stream>>>(h->d_fronts, items + lv.syrk.off, h->d_P,
                                                                       h->d_M, h->d_d);
            MF_CUDA(cudaGetLastError());
        }
    }
    return 0;
}

int launch_factor(mf_handle* h) {
    return h->diag ? factor_impl<1>(h) : factor_impl<0>(h);
}

}  // namespace mf
