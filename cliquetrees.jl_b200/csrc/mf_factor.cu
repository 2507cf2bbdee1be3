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
//               columns, 1024 parent rows); each CTA owns its target entries,
//               so the children are added in a fixed order without atomics
//               (addscattertri!, utils.jl:555-579 via chol_send!,
//               cholesky.jl:950-983).  The panel columns are done before the
//               front is factored, the update-matrix columns after the SYRK.
//   k_diag    : per 64-column sub-panel, one CTA per front factors the
//               diagonal block in shared memory, writes it back and stores
//               the inverse of the factored block (potrf! of chol_factor!,
//               cholesky.jl:694-737);
//   k_gemm    : grouped 64x64 DMMA (mma.sync m8n8k4 f64) tile GEMM with a
//               cp.async double-buffered K loop, in four roles: left-looking
//               update of a sub-panel from its outer block, trailing update
//               of the panel after an outer block (K = 256), the TRSM of a
//               sub-panel as a product with the inverse of its diagonal
//               block, and M = -L21 D L21^T with K = nn (syrk!,
//               blas/syrk.jl:137-159; the children's F22 is added to M
//               after it, which reorders the reference's sum F22 - L21 L21^T).
#include <climits>
#include <cstdio>
#include <type_traits>

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

__device__ __forceinline__ double reg_pivot(const Reg& r, double s, double p) {
    return (s * p < r.eps) ? r.delta * s : p;
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

template <typename T>
__global__ void k_scatter(T* __restrict__ P, const int64_t* __restrict__ slot, const double* __restrict__ v,
                          int64_t nnz, const int32_t* __restrict__ rowi, const int32_t* __restrict__ coli,
                          const double* __restrict__ scale) {
    pdl_prologue();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < nnz; i += stride) {
        double x = v[i];
        if (scale) x *= scale[rowi[i]] * scale[coli[i]];
        P[slot[i]] = (T)x;
    }
}

// scale[i] = 1/sqrt(|a_ii|) (1 where a_ii = 0) from the assembled values
__global__ void k_diag_scale(double* __restrict__ scale, const int64_t* __restrict__ dslot,
                             const double* __restrict__ v, int64_t n) {
    pdl_prologue();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t k = dslot[i];
    double a = k >= 0 ? fabs(v[k]) : 0.0;
    scale[i] = a > 0.0 ? 1.0 / sqrt(a) : 1.0;
}

// one warp per column: copy between the reference layout (Dval nn x nn,
// Lval na x nn of reference front j) and the panel of the execution front
// that holds j (nj x nn, ld nj): the D rows keep their order, the L rows go
// to sepmap positions.
template <bool TO_PANEL>
__global__ void k_dl_panel(const Front* __restrict__ fronts, const RefFront* __restrict__ ref,
                           const int32_t* __restrict__ colref, const int32_t* __restrict__ sepmap,
                           double* __restrict__ Dv, double* __restrict__ Lv, double* __restrict__ P, int64_t n) {
    pdl_prologue();
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

// single-precision panels -> reference layout (mixed-mode factor download)
__global__ void k_panel32_to_dl(const Front* __restrict__ fronts, const RefFront* __restrict__ ref,
                                const int32_t* __restrict__ colref, const int32_t* __restrict__ sepmap,
                                double* __restrict__ Dv, double* __restrict__ Lv, const float* __restrict__ P,
                                int64_t n) {
    pdl_prologue();
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const RefFront rf = ref[colref[warp]];
    const Front f = fronts[rf.exec];
    const int c = (int)(warp - rf.res0);
    const int off = rf.res0 - f.col0;
    const float* pc = P + f.poff + (int64_t)(off + c) * f.ldp;
    double* dc = Dv + rf.Dptr + (int64_t)c * rf.nn;
    double* lc = Lv + rf.Lptr + (int64_t)c * rf.na;
    const int32_t* map = sepmap + rf.sep0;
    for (int r = lane; r < rf.nn; r += 32) dc[r] = pc[off + r];
    for (int r = lane; r < rf.na; r += 32) lc[r] = pc[map[r]];
}

// ---------------------------------------------------------------------------
// small fronts: whole frontal matrix in shared memory
// ---------------------------------------------------------------------------
// Thresholds of the single-precision factorization's pivot check (mixed form,
// whose matrix is scaled to unit diagonal): a pivot that lost more than five
// of FP32's seven digits to cancellation against its diagonal entry, or grew
// beyond 1e7 times the largest diagonal entry of its block, flags the front
// (or 64 x 64 diagonal block), which is then factored again in FP64.
constexpr double kRescueSmall = 1e-5;
constexpr double kRescueGrowth = 1e7;
constexpr int kSmallKids = 32;  // children whose records k_small fetches up front

// One small front held in shared memory as TC: load the assembled panel, add
// the children (in the reference's reverse order), factor the first nn
// columns right-looking.  Returns the first rejected pivot (front-local) or
// -1; with `check`, *flag is set when a pivot is small or grown (see above).
// Uniform across the block.
template <typename TC, typename T, int LDLT>
__device__ int small_front(TC* F, const Front& f, const Front* __restrict__ fronts,
                           const int32_t* __restrict__ reltgt, const int32_t* __restrict__ chdtgt,
                           const T* __restrict__ P, const T* __restrict__ M, const double* __restrict__ signs,
                           bool check, int* flag, Reg reg) {
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp;
    const int tid = threadIdx.x, nt = blockDim.x;
    const T* Pj = P + f.poff;
    // the children's records (first kSmallKids, in the order they are added),
    // fetched at once beside the panel load instead of one dependent pair of
    // loads per child
    __shared__ int kid_na[kSmallKids], kid_lm[kSmallKids], kid_sep0[kSmallKids];
    __shared__ int64_t kid_moff[kSmallKids];
    const int nch = f.chd1 - f.chd0;
    for (int q = tid; q < min(nch, kSmallKids); q += nt) {
        const Front fc = fronts[chdtgt[f.chd1 - 1 - q]];
        kid_na[q] = fc.na;
        kid_lm[q] = fc.ldm;
        kid_sep0[q] = fc.sep0;
        kid_moff[q] = fc.moff;
    }
    for (int i = tid; i < nj * nn; i += nt) {
        int r = i % nj, c = i / nj;
        F[i] = (TC)Pj[r + (int64_t)c * ld];
    }
    for (int i = tid; i < nj * na; i += nt) F[nj * nn + i] = TC(0);
    __syncthreads();
    // extend-add, children popped in reverse (cholesky.jl:506-514)
    for (int q = 0; q < nch; ++q) {
        int ma, lm, sep0;
        int64_t moff;
        if (q < kSmallKids) {
            ma = kid_na[q], lm = kid_lm[q], sep0 = kid_sep0[q], moff = kid_moff[q];
        } else {
            const Front fc = fronts[chdtgt[f.chd1 - 1 - q]];
            ma = fc.na, lm = fc.ldm, sep0 = fc.sep0, moff = fc.moff;
        }
        const int32_t* rel = reltgt + sep0;
        const T* Mc = M + moff;
        for (int i = tid; i < ma * ma; i += nt) {
            int a = i % ma, b = i / ma;
            if (a >= b) F[rel[a] + rel[b] * nj] += (TC)Mc[a + b * lm];
        }
        __syncthreads();
    }
    // right-looking partial factorization of the first nn columns, one
    // block barrier per column: step k reads column k unscaled and scales
    // its entries on the fly (the same rounded products the stored scaled
    // column holds), and column k is written back scaled -- with its
    // diagonal entry -- during step k + 1, which touches only columns > k
    TC pk = TC(0), ik = TC(0);  // the previous column's stored diagonal and reciprocal
    for (int k = 0; k < nn; ++k) {
        if (k > 0) {
            if (tid == 0) F[(k - 1) + (k - 1) * nj] = pk;
            for (int i = k + tid; i < nj; i += nt) F[i + (k - 1) * nj] *= ik;
        }
        TC piv = F[k + k * nj];
        double s = pivot_sign(signs, LDLT, f.col0 + k);
        if (reg.delta >= 0.0) {
            piv = (TC)reg_pivot(reg, s, (double)piv);
            if (piv == TC(0)) return k;  // uniform across the block
        } else if (!pivot_ok(s, (double)piv) || (!LDLT && !(piv > TC(0)))) {
            return k;  // uniform across the block
        }
        if (check && tid == 0) {
            // the original diagonal entry of column k is still in the panel
            const double a0 = fabs((double)Pj[k + (int64_t)k * ld]);
            const double ap = fabs((double)piv);
            if (ap < kRescueSmall * a0 || ap > kRescueGrowth * fmax(a0, 1.0)) *flag = 1;
        }
        TC dk = LDLT ? piv : sqrt(piv);
        TC inv = TC(1) / dk;
        const int m = nj - k - 1;
        for (int i = tid; i < m * m; i += nt) {
            int r = k + 1 + i % m, c = k + 1 + i / m;
            if (r >= c) {
                TC lc = F[c + k * nj] * inv;
                if (LDLT) lc *= piv;
                const TC lr = F[r + k * nj] * inv;
                F[r + c * nj] -= lr * lc;
            }
        }
        pk = LDLT ? piv : dk;
        ik = inv;
        __syncthreads();
    }
    if (nn > 0) {
        if (tid == 0) F[(nn - 1) + (nn - 1) * nj] = pk;
        for (int i = nn + tid; i < nj; i += nt) F[i + (nn - 1) * nj] *= ik;
        __syncthreads();
    }
    return -1;
}

// Write a factored small front back: panel, update matrix, LDLt pivots (the
// diagonal of the factored panel holds them: the unit diagonal of L is
// implied and the LDLt panel diagonal keeps d_k).
template <typename TC, typename T, int LDLT>
__device__ void small_front_store(const TC* F, const Front& f, T* __restrict__ P, T* __restrict__ M,
                                 T* __restrict__ d) {
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp;
    const int tid = threadIdx.x, nt = blockDim.x;
    T* Pj = P + f.poff;
    for (int i = tid; i < nj * nn; i += nt) {
        int r = i % nj, c = i / nj;
        Pj[r + (int64_t)c * ld] = (T)F[i];
    }
    if (LDLT)
        for (int k = tid; k < nn; k += nt) d[f.col0 + k] = (T)F[k + k * nj];
    T* Mj = M + f.moff;
    const int lm = f.ldm;
    for (int i = tid; i < na * na; i += nt) {
        int a = i % na, b = i / na;
        Mj[a + b * lm] = (T)F[(nn + a) + (nn + b) * nj];
    }
}

// small fronts (nj <= kSmallMax): one CTA holds the whole front in shared
// memory.  Single precision: a front whose factorization rejects a pivot or
// flags a small or grown pivot is factored again from its inputs in FP64 in
// the same shared memory (fronts of nj <= kSmallRescue, whose FP64 front fits
// the FP32 buffer; the panel and the children's update matrices are only
// read before the final store, so the inputs are intact), and the FP64
// result is stored rounded to FP32.  A rejection in FP64 -- or in FP32 for a
// larger front -- is reported through info.
constexpr int kSmallRescue = 67;  // 67^2 doubles <= kSmallMax^2 floats
constexpr int kSmallNarrowNJ = 48;     // levels whose small fronts all have nj <= this ...
constexpr int kSmallWideLevel = 4 * 148;  // ... and that hold at least this many run 128-thread CTAs,
constexpr int kSmallTinyNJ = 32;       // 64-thread CTAs when nj <= this

template <typename T, int LDLT>
__global__ void __launch_bounds__(256) k_small(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                               const int32_t* __restrict__ reltgt,
                                               const int32_t* __restrict__ chdtgt, T* __restrict__ P,
                                               T* __restrict__ M, T* __restrict__ d,
                                               const double* __restrict__ signs, long long* __restrict__ info,
                                               int* __restrict__ rescued, Reg reg) {
    pdl_prologue();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int flag;
    T* F = reinterpret_cast<T*>(smem_raw);
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nj = f.nn + f.na;
    constexpr bool single = sizeof(T) == 4;
    if (threadIdx.x == 0) flag = 0;
    __syncthreads();
    int bad = small_front<T, T, LDLT>(F, f, fronts, reltgt, chdtgt, P, M, signs, single, &flag, reg);
    __syncthreads();
    if (single && (bad >= 0 || flag) && nj <= kSmallRescue) {
        double* F64 = reinterpret_cast<double*>(smem_raw);
        bad = small_front<double, T, LDLT>(F64, f, fronts, reltgt, chdtgt, P, M, signs, false, &flag, reg);
        if (bad < 0) {
            if (threadIdx.x == 0) atomicAdd(rescued, 1);
            small_front_store<double, T, LDLT>(F64, f, P, M, d);
            return;
        }
    }
    if (bad >= 0) {
        if (threadIdx.x == 0) atomicMin(info, (long long)(f.col0 + bad + 1));
        return;
    }
    small_front_store<T, T, LDLT>(F, f, P, M, d);
}

// ---------------------------------------------------------------------------
// Tiny fronts (nj <= ROWS, ROWS = 16 or 32): one WARP per front, kWarpFronts
// fronts per CTA, warp-synchronous (no block barriers).  Lane r holds row r of
// the front in the warp's slice of shared memory (leading dimension ROWS + 1,
// sized for FP64 so a flagged single-precision front can be redone in place).  The
// arithmetic is k_small's: the children added in the reference's reverse
// order, one addition per entry and child, then the right-looking partial
// factorization with the same update expression.
// ---------------------------------------------------------------------------
// ROWS = 16 (nj <= kWarpSmallNJ: lanes 16..31 idle, registers and shared
// memory small) or 32 (kWarpSmallNJ < nj <= kWarpSmallNJ2)
constexpr int kWarpFronts = 8;
template <int ROWS>
constexpr int warp_slice() { return (ROWS + 1) * ROWS * (int)sizeof(double); }  // bytes per warp

template <typename TC, typename T, int LDLT, int ROWS>
__device__ int warp_front(TC* F, const Front& f, const Front* __restrict__ fronts,
                          const int32_t* __restrict__ reltgt, const int32_t* __restrict__ chdtgt,
                          const T* __restrict__ P, const T* __restrict__ M, const double* __restrict__ signs,
                          bool check, bool* flag, Reg reg, int lane) {
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp;
    const T* Pj = P + f.poff;
    const bool row = lane < nj;
    // lane q fetches the record of the q-th child to add (children past 32
    // are read in the loop), beside the panel loads
    const int nch = f.chd1 - f.chd0;
    int kna = 0, klm = 0, ksep = 0;
    int64_t kmoff = 0;
    if (lane < nch) {
        const Front fc = fronts[chdtgt[f.chd1 - 1 - lane]];
        kna = fc.na, klm = fc.ldm, ksep = fc.sep0, kmoff = fc.moff;
    }
    {
        // every panel load of the lane in flight at once, then the stores
        T v[ROWS];
#pragma unroll
        for (int c = 0; c < ROWS; ++c) v[c] = (row && c < nn) ? Pj[lane + (int64_t)c * ld] : T(0);
#pragma unroll
        for (int c = 0; c < ROWS; ++c)
            if (row && c < nj) F[lane + c * (ROWS + 1)] = (TC)v[c];
    }
    __syncwarp();
    // extend-add, children popped in reverse (cholesky.jl:506-514)
    for (int q = 0; q < nch; ++q) {
        int ma = __shfl_sync(0xffffffffu, kna, q & 31), lm = __shfl_sync(0xffffffffu, klm, q & 31);
        int sep0 = __shfl_sync(0xffffffffu, ksep, q & 31);
        int64_t moff = __shfl_sync(0xffffffffu, kmoff, q & 31);
        if (q >= 32) {
            const Front fc = fronts[chdtgt[f.chd1 - 1 - q]];
            ma = fc.na, lm = fc.ldm, sep0 = fc.sep0, moff = fc.moff;
        }
        const int32_t* rel = reltgt + sep0;
        const T* Mc = M + moff;
        const int ra = lane < ma ? rel[lane] : 0;
        T mv[ROWS];
#pragma unroll
        for (int b = 0; b < ROWS; ++b) mv[b] = (b < ma && lane >= b && lane < ma) ? Mc[lane + b * lm] : T(0);
#pragma unroll
        for (int b = 0; b < ROWS; ++b) {
            const int rb = __shfl_sync(0xffffffffu, ra, b);
            if (b < ma && lane >= b && lane < ma) F[ra + rb * (ROWS + 1)] += (TC)mv[b];
        }
        __syncwarp();
    }
    // right-looking partial factorization of the first nn columns
    for (int k = 0; k < nn; ++k) {
        TC piv = F[k + k * (ROWS + 1)];
        const double s = pivot_sign(signs, LDLT, f.col0 + k);
        if (reg.delta >= 0.0) {
            piv = (TC)reg_pivot(reg, s, (double)piv);
            if (piv == TC(0)) return k;  // uniform across the warp
        } else if (!pivot_ok(s, (double)piv) || (!LDLT && !(piv > TC(0)))) {
            return k;  // uniform across the warp
        }
        if (check) {
            const double a0 = fabs((double)Pj[k + (int64_t)k * ld]);
            const double ap = fabs((double)piv);
            if (ap < kRescueSmall * a0 || ap > kRescueGrowth * fmax(a0, 1.0)) *flag = true;
        }
        const TC dk = LDLT ? piv : sqrt(piv);
        const TC inv = TC(1) / dk;
        __syncwarp();
        if (lane == k) F[k + k * (ROWS + 1)] = LDLT ? piv : dk;
        if (lane > k && row) F[lane + k * (ROWS + 1)] *= inv;
        __syncwarp();
        if (lane > k && row) {
            const TC lr = F[lane + k * (ROWS + 1)];
            for (int c = k + 1; c <= lane; ++c) {
                TC lc = F[c + k * (ROWS + 1)];
                if (LDLT) lc *= piv;
                F[lane + c * (ROWS + 1)] -= lr * lc;
            }
        }
        __syncwarp();
    }
    return -1;
}

template <typename TC, typename T, int LDLT, int ROWS>
__device__ void warp_front_store(const TC* F, const Front& f, T* __restrict__ P, T* __restrict__ M,
                                 T* __restrict__ d, int lane) {
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp;
    T* Pj = P + f.poff;
    if (lane < nj)
        for (int c = 0; c < nn; ++c) Pj[lane + (int64_t)c * ld] = (T)F[lane + c * (ROWS + 1)];
    if (LDLT && lane < nn) d[f.col0 + lane] = (T)F[lane + lane * (ROWS + 1)];
    T* Mj = M + f.moff;
    const int lm = f.ldm;
    if (lane < na)
        for (int b = 0; b < na; ++b) Mj[lane + b * lm] = (T)F[(nn + lane) + (nn + b) * (ROWS + 1)];
}

template <typename T, int LDLT, int ROWS>
__global__ void __launch_bounds__(kWarpFronts * 32) k_small_warp(const Front* __restrict__ fronts,
                                                                const Item* __restrict__ items, int64_t cnt,
                                                                const int32_t* __restrict__ reltgt,
                                                                const int32_t* __restrict__ chdtgt,
                                                                T* __restrict__ P, T* __restrict__ M,
                                                                T* __restrict__ d, const double* __restrict__ signs,
                                                                long long* __restrict__ info,
                                                                int* __restrict__ rescued, Reg reg) {
    pdl_prologue();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t w = (int64_t)blockIdx.x * kWarpFronts + wib;
    if (w >= cnt) return;  // whole warps only
    unsigned char* slice = smem_raw + (size_t)wib * warp_slice<ROWS>();
    const Front f = fronts[items[w].front];
    constexpr bool single = sizeof(T) == 4;
    bool flag = false;
    T* F = reinterpret_cast<T*>(slice);
    int bad = warp_front<T, T, LDLT, ROWS>(F, f, fronts, reltgt, chdtgt, P, M, signs, single, &flag, reg, lane);
    if (single && (bad >= 0 || flag)) {
        // the panel and the children's update matrices are only read before
        // the final store: refactor from the same inputs in FP64
        double* F64 = reinterpret_cast<double*>(slice);
        __syncwarp();
        bool unused = false;
        bad = warp_front<double, T, LDLT, ROWS>(F64, f, fronts, reltgt, chdtgt, P, M, signs, false, &unused, reg, lane);
        if (bad < 0) {
            if (lane == 0) atomicAdd(rescued, 1);
            __syncwarp();
            warp_front_store<double, T, LDLT, ROWS>(F64, f, P, M, d, lane);
            return;
        }
    }
    if (bad >= 0) {
        if (lane == 0) atomicMin(info, (long long)(f.col0 + bad + 1));
        return;
    }
    __syncwarp();
    warp_front_store<T, T, LDLT, ROWS>(F, f, P, M, d, lane);
}

// ---------------------------------------------------------------------------
// extend-add for blocked fronts
// ---------------------------------------------------------------------------

// One CTA per (front, 16 parent columns, kEArows parent rows); warp w owns
// parent columns c0 + w and c0 + w + 8.  The plan lists, per child in the
// reference's order (reverse, cholesky.jl:506-514), the child columns b0..b1
// and rows a0..a1 whose relative indices fall in the item's columns and rows,
// so the kernel does no searching.  Every parent entry belongs to one CTA and
// one warp, and the children are added in a fixed order: no atomics, no block
// barrier, deterministic sums.  PART 0 adds into the panel columns (before
// the front is factored), PART 1 into the update matrix, which the SYRK has
// already set to -L21 L21^T (so it is never zeroed or read twice).  A child
// column streams in chunks of up to 4 x 32 rows (ea_chunk).
// a chunk of U x 32 rows of a child column: the relative indices and child
// values of the chunk first, then the U parent entries they address, so U
// independent gather chains are in flight per lane; PRED drops rows >= a1
template <typename T, int U, bool PRED>
__device__ __forceinline__ void ea_chunk(const int32_t* __restrict__ rel, const T* mc, T* dst, int a, int a1) {
    int r[U];
    T v[U], o[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int aa = a + 32 * u;
        const bool in = !PRED || aa < a1;
        r[u] = in ? __ldg(rel + aa) : -1;
        v[u] = in ? mc[aa] : T(0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
        if (r[u] >= 0) o[u] = dst[r[u]];
#pragma unroll
    for (int u = 0; u < U; ++u)
        if (r[u] >= 0) dst[r[u]] = o[u] + v[u];
}

template <typename T, int PART>
__global__ void __launch_bounds__(256) k_ea(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                            const Item* __restrict__ all_items, const int32_t* __restrict__ reltgt,
                                            T* __restrict__ P, T* __restrict__ M) {
    pdl_prologue();
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, ld = f.ldp, lm = f.ldm;
    const int c0 = it.a * kEAcols;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T* Pj = P + f.poff;
    T* Mj = M + f.moff;
    const Item* seg = all_items + it.pad;  // segment offsets index the whole item buffer
    const int nch = f.chd1 - f.chd0;
    for (int s = 0; s < nch; ++s) {
        const Item s1 = seg[2 * s], s2 = seg[2 * s + 1];
        const int b0 = s1.a, b1 = s1.b, a0 = s2.front, a1 = s2.a;
        if (b0 >= b1 || a1 <= a0) continue;
        const Front fc = fronts[s1.front];
        const int32_t* __restrict__ rel = reltgt + fc.sep0;
        const T* Mc = M + fc.moff;
        for (int b = b0; b < b1; ++b) {
            const int col = __ldg(rel + b);
            if (((col - c0) & 7) != warp) continue;  // the owner warp of this parent column
            const T* mc = Mc + (int64_t)b * fc.ldm;
            T* dst = PART == 0 ? Pj + (int64_t)col * ld : Mj + (int64_t)(col - nn) * lm - nn;
            // full chunks of 4 x 32 rows, then one predicated chunk of at
            // most 4 x 32 rows (a single row per lane when the rest is that
            // short: many child columns are, and the predicated slots would
            // cost instructions for nothing).  Eight chains per lane measured
            // slower on long columns (more lines in flight than L1 keeps).
            int a = max(a0, b) + lane;
            for (; a + 96 < a1; a += 128) ea_chunk<T, 4, false>(rel, mc, dst, a, a1);
            if (a + 32 < a1) ea_chunk<T, 4, true>(rel, mc, dst, a, a1);
            else if (a < a1) dst[__ldg(rel + a)] += mc[a];
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// diagonal block: factor + inverse
// ---------------------------------------------------------------------------

// Diagonal block: factor + inverse, one CTA of 256 threads per front.
//
// The 64 x 64 block (columns >= w padded with the identity) sits in shared
// memory and is factored in four 16-column panels.  Per panel, warp 0
// factors the 16 x 16 diagonal block in registers (lane i < 16 owns row i;
// column k reaches the other lanes by shuffles, so the 16 dependent pivot
// steps use no barrier) and inverts it (lane j owns column j).  All threads
// then form the rows below as A L^-T (D^-1) with that inverse and apply the
// rank-16 update to the trailing block; both are fully unrolled 16-term dot
// products.  Finally the off-diagonal 16 x 16 blocks of X = L^-1 (unit
// diagonal for LDLt) follow along the block sub-diagonals,
// X_ij = -X_ii sum_{k=j}^{i-1} L_ik X_kj.  About 26 barriers in all.  This is
// diag_block_seq (the FP64 kernel); the FP32 kernel runs diag_block_la,
// which takes the inverses and the bulk updates off warp 0's chain.
constexpr int LDS = kNB + 4;  // shared-memory leading dimension of the GEMM stages
constexpr int LDA = kNB + 1;  // leading dimension of the block and its inverse in the diagonal kernel

// dynamic shared memory of k_diag: the FP64 layout in both precisions (the
// single-precision kernel refactors flagged blocks in FP64 in place)
template <typename T>
constexpr int diag_smem() { return (2 * kNB * LDA + 2 * kNB) * (int)sizeof(double); }

// The pivot's diagonal entry dk (sqrt(p) for Cholesky, p for LDLt) and its
// reciprocal.  FP32 (the mixed form, whose factor only preconditions the
// FP64 refinement) uses the hardware reciprocal square root / reciprocal;
// FP64 keeps the correctly rounded operations of the plain form.
template <typename T, int LDLT>
__device__ __forceinline__ void diag_pivot(T p, T& dk, T& ik);
template <>
__device__ __forceinline__ void diag_pivot<float, 0>(float p, float& dk, float& ik) {
    ik = rsqrtf(p);
    dk = p * ik;
}
template <>
__device__ __forceinline__ void diag_pivot<float, 1>(float p, float& dk, float& ik) {
    dk = p;
    ik = __frcp_rn(p);
}
template <>
__device__ __forceinline__ void diag_pivot<double, 0>(double p, double& dk, double& ik) {
    dk = sqrt(p);
    ik = 1.0 / dk;
}
template <>
__device__ __forceinline__ void diag_pivot<double, 1>(double p, double& dk, double& ik) {
    dk = p;
    ik = 1.0 / p;
}

// Factor and invert the 64 x 64 block held in shared memory as TC: A (block,
// identity beyond column w), X (inverse), pivs (L_kk or d_k), rinv (their
// reciprocals).  Returns the first rejected pivot (block-local) or -1,
// uniform across the block; bad_s is a shared scratch int.
//
// Four 16-column panels with look-ahead.  Panel p: warp 0 factors its 16 x 16
// diagonal block in registers (the pivot chain, by shuffles) while warps 1..7
// apply panel p-1's update to every entry below that block (the rows and
// columns the later panels read); then every thread with a row below solves
// that row against the panel's triangle (forward substitution in registers),
// and the next panel's 16 x 16 diagonal block takes panel p's update, so warp
// 0 can start on it at once.  The chain therefore waits for no bulk update.
// The 16 x 16 inverses (warps 0..3 at once) and the off-diagonal blocks of X
// follow the factorization.
template <typename TC, int LDLT>
__device__ __forceinline__ void diag_factor16(TC* A, TC* pivs, TC* rinv, int pb, int w,
                                              const double* __restrict__ signs, int64_t colbase, int* bad_s,
                                              const Reg& reg, int lane) {
    using T = TC;
    const int i = lane & 15;  // lanes 16..31 mirror 0..15
    T a[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) a[j] = j <= i ? A[(pb + i) + (pb + j) * LDA] : T(0);
    T mypiv = T(1), myrinv = T(1);
    int bad = -1;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        T pv = __shfl_sync(0xffffffffu, a[k], k);
        if (reg.delta >= 0.0) {
            if (pb + k < w) {
                pv = (T)reg_pivot(reg, pivot_sign(signs, LDLT, colbase + pb + k), (double)pv);
                if (i == k) a[k] = pv;
                if (bad < 0 && pv == T(0)) bad = pb + k;
            }
        } else if (bad < 0 && pb + k < w) {
            const double sg = pivot_sign(signs, LDLT, colbase + pb + k);
            if (!pivot_ok(sg, (double)pv) || (!LDLT && !(pv > T(0)))) bad = pb + k;
        }
        // after a rejected pivot the remaining steps run on junk and are discarded
        T dk, ik;
        diag_pivot<T, LDLT>(pv, dk, ik);
        const T aik = a[k];
        const T lik = aik * ik;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            if (j > k) {  // resolved at compile time once both loops are unrolled
                const T u = __shfl_sync(0xffffffffu, LDLT ? aik : lik, j);
                if (i >= j) a[j] -= lik * u;
            }
        }
        if (i > k) a[k] = lik;
        else if (i == k) {
            if (!LDLT) a[k] = dk;
            mypiv = dk;
            myrinv = ik;
        }
    }
    if (lane < 16) {
#pragma unroll
        for (int jj = 0; jj < 16; ++jj)
            if (jj <= i) A[(pb + i) + (pb + jj) * LDA] = a[jj];
        pivs[pb + i] = mypiv;
        rinv[pb + i] = myrinv;
    }
    if (lane == 0 && bad >= 0) (*bad_s) = bad;
}

// the inverse of the factored 16 x 16 diagonal block at pb (one warp): lane
// j owns column j
template <typename TC, int LDLT>
__device__ __forceinline__ void diag_inv16(const TC* A, TC* X, const TC* rinv, int pb, int lane) {
    using T = TC;
    const int i = lane & 15, j = i;
    T a[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) a[k] = k < i ? A[(pb + i) + (pb + k) * LDA] : T(0);
    const T myrinv = rinv[pb + i];
    T x[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) {
        T acc = T(0);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            if (k < r) {  // resolved at compile time once both loops are unrolled
                const T lrk = __shfl_sync(0xffffffffu, a[k], r);
                if (k >= j) acc += lrk * x[k];
            }
        }
        const T rr = __shfl_sync(0xffffffffu, myrinv, r);
        x[r] = r < j ? T(0) : (r == j ? (LDLT ? T(1) : rr) : (LDLT ? -acc : -acc * rr));
    }
    if (lane < 16)
#pragma unroll
        for (int r = 0; r < 16; ++r) X[(pb + r) + (pb + j) * LDA] = x[r];
}

// A[i, j] -= sum_q L[i, pb + q] (d_q) L[j, pb + q] over a rectangle of rows
// [r0, 64) x columns [c0, c1), lower triangle only, threads t0.. of the block
template <typename TC, int LDLT>
__device__ __forceinline__ void diag_update(TC* A, const TC* pivs, int pb, int r0, int c0, int c1, int t,
                                            int nt) {
    using T = TC;
    const int nr = kNB - r0, nc = c1 - c0;
    for (int e = t; e < nr * nc; e += nt) {
        const int i = r0 + e % nr, j = c0 + e / nr;
        if (i >= j) {
            T acc = T(0);
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                T lj = A[j + (pb + q) * LDA];
                if (LDLT) lj *= pivs[pb + q];
                acc += A[i + (pb + q) * LDA] * lj;
            }
            A[i + j * LDA] -= acc;
        }
    }
}

// The off-diagonal 16 x 16 blocks of X = L^-1 from the four diagonal
// inverses already in X, by block distance (the whole CTA).
template <typename TC>
__device__ __forceinline__ void diag_inv_offdiag(const TC* A, TC* X) {
    const int tid = threadIdx.x;
    using T = TC;
#pragma unroll 1
    for (int dist = 1; dist < 4; ++dist) {
        const int nb = 4 - dist;
        T tmp[3];
#pragma unroll
        for (int s = 0; s < 3; ++s) {  // T_ij = sum_{k=j}^{i-1} L_ik X_kj
            const int o = tid + 256 * s;
            tmp[s] = T(0);
            if (o < nb * 256) {
                const int bj = o >> 8, bi = bj + dist, r = (o >> 4) & 15, c = o & 15;
                T acc = T(0);
                for (int bk = bj; bk < bi; ++bk)
#pragma unroll
                    for (int q = 0; q < 16; ++q)
                        acc += A[(16 * bi + r) + (16 * bk + q) * LDA] * X[(16 * bk + q) + (16 * bj + c) * LDA];
                tmp[s] = acc;
            }
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            const int o = tid + 256 * s;
            if (o < nb * 256) {
                const int bj = o >> 8, bi = bj + dist, r = (o >> 4) & 15, c = o & 15;
                X[(16 * bi + r) + (16 * bj + c) * LDA] = tmp[s];
            }
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < 3; ++s) {  // X_ij = -X_ii T_ij
            const int o = tid + 256 * s;
            if (o < nb * 256) {
                const int bj = o >> 8, bi = bj + dist, r = (o >> 4) & 15, c = o & 15;
                T acc = T(0);
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    acc += X[(16 * bi + r) + (16 * bi + q) * LDA] * X[(16 * bi + q) + (16 * bj + c) * LDA];
                tmp[s] = -acc;
            }
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            const int o = tid + 256 * s;
            if (o < nb * 256) {
                const int bj = o >> 8, bi = bj + dist, r = (o >> 4) & 15, c = o & 15;
                X[(16 * bi + r) + (16 * bj + c) * LDA] = tmp[s];
            }
        }
        __syncthreads();
    }
}

template <typename TC, int LDLT>
__device__ int diag_block_la(TC* A, TC* X, TC* pivs, TC* rinv, int w, const double* __restrict__ signs,
                          int64_t colbase, int* bad_s, Reg reg) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    using T = TC;
    if (tid == 0) *bad_s = -1;
    __syncthreads();
    // the panel loop stays rolled: its body runs once per panel and block,
    // and four unrolled copies made the kernel wait on instruction fetches
#pragma unroll 1
    for (int p = 0; p < 4; ++p) {
        const int pb = p * 16;
        if (warp == 0) {
            diag_factor16<TC, LDLT>(A, pivs, rinv, pb, w, signs, colbase, bad_s, reg, lane);
        } else if (p > 0) {
            // panel p-1's update of everything below the diagonal block p
            // (rows >= pb + 16, columns pb .. row); the block itself took it
            // at the end of the previous panel
            diag_update<TC, LDLT>(A, pivs, pb - 16, pb + 16, pb, kNB, tid - 32, 224);
        }
        __syncthreads();
        if ((*bad_s) >= 0) break;  // uniform
        if (p == 3) break;
        // rows below: solve each row against the panel's triangle, in four
        // column groups (finish a group, then subtract it from the later
        // columns at once), which cuts the dependent chain of the
        // substitution to about a third
        const int r = pb + 16 + tid;
        if (r < kNB) {
            T y[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) y[c] = A[r + (pb + c) * LDA];
#pragma unroll
            for (int g = 0; g < 4; ++g) {
#pragma unroll
                for (int c = 4 * g; c < 4 * g + 4; ++c) {
#pragma unroll
                    for (int q = 4 * g; q < c; ++q) y[c] -= y[q] * A[(pb + c) + (pb + q) * LDA];
                    if (!LDLT) y[c] *= rinv[pb + c];
                }
#pragma unroll
                for (int c = 4 * g + 4; c < 16; ++c)
#pragma unroll
                    for (int q = 4 * g; q < 4 * g + 4; ++q) y[c] -= y[q] * A[(pb + c) + (pb + q) * LDA];
            }
#pragma unroll
            for (int c = 0; c < 16; ++c) A[r + (pb + c) * LDA] = LDLT ? y[c] * rinv[pb + c] : y[c];
        }
        __syncthreads();
        // the next diagonal block takes this panel's update now
        {
            const int e = tid;
            if (e < 256) {
                const int ii = e & 15, jj = e >> 4;
                const int gi = pb + 16 + ii, gj = pb + 16 + jj;
                if (ii >= jj) {
                    T acc = T(0);
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        T lj = A[gj + (pb + q) * LDA];
                        if (LDLT) lj *= pivs[pb + q];
                        acc += A[gi + (pb + q) * LDA] * lj;
                    }
                    A[gi + gj * LDA] -= acc;
                }
            }
        }
        __syncthreads();
    }
    if (*bad_s >= 0) return *bad_s;  // uniform
    // the four 16 x 16 diagonal inverses at once
    if (warp < 4) diag_inv16<TC, LDLT>(A, X, rinv, warp * 16, lane);
    __syncthreads();
    diag_inv_offdiag<TC>(A, X);
    return -1;
}

// The sequential version: per panel, warp 0 factors and inverts the 16 x 16
// diagonal block, then the CTA forms the rows below from that inverse and
// applies the panel's trailing update.
template <typename TC, int LDLT>
__device__ int diag_block_seq(TC* A, TC* X, TC* pivs, TC* rinv, int w, const double* __restrict__ signs,
                          int64_t colbase, int* bad_s, Reg reg) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    using T = TC;
    if (tid == 0) *bad_s = -1;
    __syncthreads();
#pragma unroll 1
    for (int p = 0; p < 4; ++p) {
        const int pb = p * 16;
        if (warp == 0) {
            const int i = lane & 15;  // lanes 16..31 mirror 0..15
            T a[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) a[j] = j <= i ? A[(pb + i) + (pb + j) * LDA] : T(0);
            T mypiv = T(1), myrinv = T(1);
            int bad = -1;
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                T pv = __shfl_sync(0xffffffffu, a[k], k);
                if (reg.delta >= 0.0) {
                    if (pb + k < w) {
                        pv = (T)reg_pivot(reg, pivot_sign(signs, LDLT, colbase + pb + k), (double)pv);
                        if (i == k) a[k] = pv;
                        if (bad < 0 && pv == T(0)) bad = pb + k;
                    }
                } else if (bad < 0 && pb + k < w) {
                    const double sg = pivot_sign(signs, LDLT, colbase + pb + k);
                    if (!pivot_ok(sg, (double)pv) || (!LDLT && !(pv > T(0)))) bad = pb + k;
                }
                // after a rejected pivot the remaining steps run on junk and are discarded
                T dk, ik;
                diag_pivot<T, LDLT>(pv, dk, ik);
                const T aik = a[k];
                const T lik = aik * ik;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    if (j > k) {  // resolved at compile time once both loops are unrolled
                        const T u = __shfl_sync(0xffffffffu, LDLT ? aik : lik, j);
                        if (i >= j) a[j] -= lik * u;
                    }
                }
                if (i > k) a[k] = lik;
                else if (i == k) {
                    if (!LDLT) a[k] = dk;
                    mypiv = dk;
                    myrinv = ik;
                }
            }
            // inverse of the 16 x 16 factor: lane j owns column j
            const int j = i;
            T x[16];
#pragma unroll
            for (int r = 0; r < 16; ++r) {
                T acc = T(0);
#pragma unroll
                for (int k = 0; k < 16; ++k) {
                    if (k < r) {  // resolved at compile time once both loops are unrolled
                        const T lrk = __shfl_sync(0xffffffffu, a[k], r);
                        if (k >= j) acc += lrk * x[k];
                    }
                }
                const T rr = __shfl_sync(0xffffffffu, myrinv, r);
                x[r] = r < j ? T(0) : (r == j ? (LDLT ? T(1) : rr) : (LDLT ? -acc : -acc * rr));
            }
            if (lane < 16) {
#pragma unroll
                for (int jj = 0; jj < 16; ++jj)
                    if (jj <= i) A[(pb + i) + (pb + jj) * LDA] = a[jj];
#pragma unroll
                for (int r = 0; r < 16; ++r) X[(pb + r) + (pb + j) * LDA] = x[r];
                pivs[pb + i] = mypiv;
                rinv[pb + i] = myrinv;
            }
            if (lane == 0 && bad >= 0) (*bad_s) = bad;
        }
        __syncthreads();
        if ((*bad_s) >= 0) break;  // uniform
        const int m = 48 - pb;  // rows / columns after the panel
        if (m == 0) break;
        // rows below: L_rc = sum_{q <= c} A_r,pb+q Xpp_c,q (/ d_c)
        T res[3];
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            const int o = tid + 256 * s;
            res[s] = T(0);
            if (o < m * 16) {
                const int r = pb + 16 + o % m, c = o / m;
                T acc = T(0);
#pragma unroll
                for (int q = 0; q < 16; ++q) acc += A[r + (pb + q) * LDA] * X[(pb + c) + (pb + q) * LDA];
                res[s] = LDLT ? acc * rinv[pb + c] : acc;
            }
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            const int o = tid + 256 * s;
            if (o < m * 16) A[(pb + 16 + o % m) + (pb + o / m) * LDA] = res[s];
        }
        __syncthreads();
        // trailing update A_ij -= sum_q L_iq (d_q) L_jq, pb+16 <= j <= i
        for (int e = tid; e < m * m; e += 256) {
            const int i = pb + 16 + e % m, j = pb + 16 + e / m;
            if (i >= j) {
                T acc = T(0);
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    T lj = A[j + (pb + q) * LDA];
                    if (LDLT) lj *= pivs[pb + q];
                    acc += A[i + (pb + q) * LDA] * lj;
                }
                A[i + j * LDA] -= acc;
            }
        }
        __syncthreads();
    }
    if (*bad_s >= 0) return *bad_s;  // uniform
    diag_inv_offdiag<TC>(A, X);
    return -1;
}

// FP32 (the mixed form) takes the look-ahead version; FP64 the sequential
// one, measured faster for doubles (the look-ahead's update warps compete
// with warp 0's pivot chain for the FP64 pipes, and the row substitution is
// a longer FP64 dependency chain than the product with the inverse).
template <typename TC, int LDLT>
__device__ int diag_block(TC* A, TC* X, TC* pivs, TC* rinv, int w, const double* __restrict__ signs,
                          int64_t colbase, int* bad_s, Reg reg) {
    if (sizeof(TC) == 4) return diag_block_la<TC, LDLT>(A, X, pivs, rinv, w, signs, colbase, bad_s, reg);
    return diag_block_seq<TC, LDLT>(A, X, pivs, rinv, w, signs, colbase, bad_s, reg);
}

// Write back a factored diagonal block: the factor into the panel, the LDLt
// pivots, the inverse into the inverse scratch.
template <typename TC, typename T, int LDLT>
__device__ void diag_block_store(const TC* A, const TC* X, const TC* pivs, int w, T* Pj, int64_t ld, int c0,
                                 T* __restrict__ d, int64_t dcol, T* dst) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int e = tid; e < kNB * kNB; e += 256) {
        const int r = e & (kNB - 1), c = e >> 6;
        if (r >= c && r < w && c < w) Pj[(c0 + r) + (int64_t)(c0 + c) * ld] = (T)A[r + c * LDA];
    }
    if (LDLT && tid < w) d[dcol + tid] = (T)pivs[tid];
#pragma unroll
    for (int e = tid; e < kNB * kNB; e += 256) {
        const int r = e & (kNB - 1), c = e >> 6;
        dst[e] = (r < w && c < w) ? (T)X[r + c * LDA] : T(0);
    }
}

template <typename TC, typename T>
__device__ void diag_block_load(TC* A, TC* X, const T* Pj, int64_t ld, int c0, int w) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int e = tid; e < kNB * kNB; e += 256) {
        const int r = e & (kNB - 1), c = e >> 6;
        TC v = (r == c) ? TC(1) : TC(0);
        if (r >= c && r < w && c < w) v = (TC)Pj[(c0 + r) + (int64_t)(c0 + c) * ld];
        A[r + c * LDA] = v;
        X[r + c * LDA] = TC(0);
    }
}

// Diagonal block kernel.  Single precision: when the FP32 factorization
// rejects a pivot, or a pivot lost more than five digits against its
// diagonal entry or grew beyond 1e7 times the block's largest diagonal entry,
// the block is loaded again and factored and inverted in FP64 (the dynamic
// shared memory is sized for that), and the FP64 result is stored rounded to
// FP32.  A rejection in FP64 is reported through info.
template <typename T, int LDLT>
__global__ void __launch_bounds__(256, 1) k_diag(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                              int c0, T* __restrict__ P, T* __restrict__ inv,
                                              T* __restrict__ d, const double* __restrict__ signs,
                                              long long* __restrict__ info, int* __restrict__ rescued, Reg reg) {
    pdl_prologue();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* A = reinterpret_cast<T*>(smem_raw);  // block, A[r + c * LDA]
    T* X = A + kNB * LDA;                   // inverse, same layout
    T* pivs = X + kNB * LDA;                // L_kk (Cholesky) or d_k (LDLt)
    T* rinv = pivs + kNB;                   // 1 / L_kk or 1 / d_k
    __shared__ int bad_s, flag_s;
    __shared__ double dmax_s;
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn;
    const int64_t ld = f.ldp;
    const int w = min(kNB, nn - c0);
    const int tid = threadIdx.x;
    T* Pj = P + f.poff;
    T* dst = inv + f.ioff + (int64_t)(c0 / kNB) * kNB * kNB;
    constexpr bool single = sizeof(T) == 4;
    if (tid == 0) { flag_s = 0; dmax_s = 0.0; }
    diag_block_load<T, T>(A, X, Pj, ld, c0, w);
    __syncthreads();
    // |a_kk| before the factorization and the block's largest (non-negative
    // doubles order like their bit patterns); diag_block starts with a barrier
    const double a0 = tid < w ? fabs((double)A[tid + tid * LDA]) : 0.0;
    if (single && tid < w)
        atomicMax(reinterpret_cast<unsigned long long*>(&dmax_s), (unsigned long long)__double_as_longlong(a0));
    int bad = diag_block<T, LDLT>(A, X, pivs, rinv, w, signs, (int64_t)f.col0 + c0, &bad_s, reg);
    if (single) {
        if (bad < 0 && tid < w) {
            const double dk = LDLT ? fabs((double)pivs[tid]) : (double)pivs[tid] * (double)pivs[tid];
            if (dk < kRescueSmall * a0 || dk > kRescueGrowth * fmax(dmax_s, 1.0)) flag_s = 1;
        }
        __syncthreads();
        if (bad >= 0 || flag_s) {
            double* A64 = reinterpret_cast<double*>(smem_raw);
            double* X64 = A64 + kNB * LDA;
            double* piv64 = X64 + kNB * LDA;
            double* rinv64 = piv64 + kNB;
            __syncthreads();
            diag_block_load<double, T>(A64, X64, Pj, ld, c0, w);
            bad = diag_block<double, LDLT>(A64, X64, piv64, rinv64, w, signs, (int64_t)f.col0 + c0, &bad_s, reg);
            if (bad < 0) {
                if (tid == 0) atomicAdd(rescued, 1);
                diag_block_store<double, T, LDLT>(A64, X64, piv64, w, Pj, ld, c0, d, f.col0 + c0, dst);
                return;
            }
        }
    }
    if (bad >= 0) {  // uniform
        if (tid == 0) atomicMin(info, (long long)(f.col0 + c0 + bad + 1));
        return;
    }
    diag_block_store<T, T, LDLT>(A, X, pivs, w, Pj, ld, c0, d, f.col0 + c0, dst);
}

// ---------------------------------------------------------------------------
// Tile GEMM with a cp.async double-buffered K loop:
// acc(64x64) += A(64 x K) * B(64 x K)^T.  Shared tiles are [k][m] with m
// contiguous (leading dimension LDS).
//   double: DMMA (mma.sync m8n8k4 f64), 8 warps; warp w owns rows
//           (w&1)*32..+32 and columns (w>>1)*16..+16 as 4 x 2 fragments.
//   float : FMA, thread t owns rows (t>>4)*4..+4 and columns (t&15)*4..+4.
// ---------------------------------------------------------------------------
constexpr int KC = 32;                   // K chunk per pipeline stage
constexpr int STAGE = KC * LDS;          // elements per matrix per stage

template <typename T>
constexpr int gemm_smem() { return (4 * STAGE + 2 * KC) * (int)sizeof(T); }

template <typename T>
struct Acc;
template <>
struct Acc<double> {
    double c[4][2][2];
};
template <>
struct Acc<float> {
    float c[4][4];
};

__device__ __forceinline__ void acc_zero(Acc<double>& a) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) a.c[i][j][0] = a.c[i][j][1] = 0.0;
}
__device__ __forceinline__ void acc_zero(Acc<float>& a) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) a.c[i][j] = 0.f;
}

template <typename T>
__device__ __forceinline__ void cp_async_el(T* dst, const T* src, bool valid) {
    unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
    int n = valid ? (int)sizeof(T) : 0;
    if (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(src), "r"(n));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(saddr), "l"(src), "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <typename T>
__device__ __forceinline__ void stage_chunk(T* As, T* Bs, const T* A, int64_t lda, int ra, int amax, const T* B,
                                            int64_t ldb, int rb, int bmax, int k, int kc) {
    for (int i = threadIdx.x; i < 64 * KC; i += blockDim.x) {
        int m = i & 63, kk = i >> 6;
        bool va = (ra + m < amax) && kk < kc;
        bool vb = (rb + m < bmax) && kk < kc;
        const T* sa = A + (va ? (ra + m) + (int64_t)(k + kk) * lda : 0);
        const T* sb = B + (vb ? (rb + m) + (int64_t)(k + kk) * ldb : 0);
        cp_async_el(As + m + kk * LDS, sa, va);
        cp_async_el(Bs + m + kk * LDS, sb, vb);
    }
}

__device__ __forceinline__ void mma_chunk(Acc<double>& acc, const double* As, const double* Bs, const double* dsc,
                                          int kc) {
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

__device__ __forceinline__ void mma_chunk(Acc<float>& acc, const float* As, const float* Bs, const float* dsc,
                                          int kc) {
    const int tr = (threadIdx.x >> 4) * 4, tc = (threadIdx.x & 15) * 4;
    for (int k = 0; k < kc; ++k) {
        const float4 a4 = *reinterpret_cast<const float4*>(As + tr + k * LDS);
        const float4 b4 = *reinterpret_cast<const float4*>(Bs + tc + k * LDS);
        const float s = dsc ? dsc[k] : 1.f;
        const float a[4] = {a4.x * s, a4.y * s, a4.z * s, a4.w * s};
        const float b[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc.c[i][j] = fmaf(a[i], b[j], acc.c[i][j]);
    }
}

// acc += A[ra.., kbeg..kend) * B[rb.., kbeg..kend)^T (optionally D-scaled)
template <typename T>
__device__ void gemm_k_loop(Acc<T>& acc, T* smem, const T* A, int64_t lda, int ra, int amax, const T* B,
                            int64_t ldb, int rb, int bmax, int kbeg, int kend, const T* dvec) {
    const int nchunk = (kend - kbeg + KC - 1) / KC;
    if (nchunk <= 0) return;
    auto buf_a = [&](int st) { return smem + st * STAGE; };
    auto buf_b = [&](int st) { return smem + (2 + st) * STAGE; };
    auto buf_d = [&](int st) { return smem + 4 * STAGE + st * KC; };
    auto load = [&](int c, int st) {
        int k = kbeg + c * KC;
        int kc = min(KC, kend - k);
        stage_chunk(buf_a(st), buf_b(st), A, lda, ra, amax, B, ldb, rb, bmax, k, kc);
        if (dvec)
            for (int i = threadIdx.x; i < KC; i += blockDim.x) buf_d(st)[i] = i < kc ? dvec[k + i] : T(0);
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
        mma_chunk(acc, buf_a(st), buf_b(st), dvec ? buf_d(st) : nullptr, (kc + 3) & ~3);
        __syncthreads();
    }
}

// visit every accumulator element as (row, col, value)
template <typename F>
__device__ __forceinline__ void acc_for_each(const Acc<double>& acc, F&& fn) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wr = (warp & 1) * 32, wc = (warp >> 1) * 16;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e)
                fn(wr + i * 8 + (lane >> 2), wc + j * 8 + (lane & 3) * 2 + e, acc.c[i][j][e]);
}
template <typename F>
__device__ __forceinline__ void acc_for_each(const Acc<float>& acc, F&& fn) {
    const int tr = (threadIdx.x >> 4) * 4, tc = (threadIdx.x & 15) * 4;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) fn(tr + i, tc + j, acc.c[i][j]);
}

// C(rbase+r, cbase+c) -= acc (or = acc * colscale when OVERWRITE), for
// r < rmax, c < cmax; on a diagonal tile only row >= col is written.
// Store an accumulator tile: MODE 0 C -= acc, MODE 1 C = acc (times the
// column scale if given), MODE 2 C = -acc (the SYRK writes M = -L21 L21^T;
// the children's extend-add follows it).
template <int MODE, typename T>
__device__ __forceinline__ void acc_store(const Acc<T>& acc, T* C, int64_t ldc, int rbase, int cbase, int rmax,
                                          int cmax, bool diag_tile, const T* colscale) {
    acc_for_each(acc, [&](int r, int c, T v) {
        if (r < rmax && c < cmax && (!diag_tile || rbase + r >= cbase + c)) {
            T* p = C + (rbase + r) + (int64_t)(cbase + c) * ldc;
            if (MODE == 1) *p = colscale ? v * colscale[c] : v;
            else if (MODE == 2) *p = -v;
            else *p -= v;
        }
    });
}

enum GemmRole { G_LEFT = 0, G_TRAIL = 1, G_SYRK = 2, G_TRSM = 3 };

template <typename T, int ROLE, int LDLT>
__global__ void __launch_bounds__(256) k_gemm(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                              int obs, int obw, int c0, T* __restrict__ P, T* __restrict__ M,
                                              const T* __restrict__ d, const T* __restrict__ inv) {
    pdl_prologue();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* smem = reinterpret_cast<T*>(smem_raw);
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp;
    T* Pj = P + f.poff;
    const T* dj = LDLT ? d + f.col0 : nullptr;
    Acc<T> acc;
    acc_zero(acc);
    if (ROLE == G_LEFT) {
        const int w = min(kNB, nn - c0);
        const int rs = c0 + it.a * kTile;
        gemm_k_loop<T>(acc, smem, Pj, ld, rs, nj, Pj, ld, c0, c0 + w, obs, c0, dj);
        acc_store<0>(acc, Pj, ld, rs, c0, nj - rs, w, it.a == 0, (const T*)nullptr);
    } else if (ROLE == G_TRAIL) {
        const int e = min(nn, obs + obw);
        const int cs = e + it.b * kTile, rs = cs + it.a * kTile;
        gemm_k_loop<T>(acc, smem, Pj, ld, rs, nj, Pj, ld, cs, nn, obs, e, dj);
        acc_store<0>(acc, Pj, ld, rs, cs, nj - rs, nn - cs, it.a == 0, (const T*)nullptr);
    } else if (ROLE == G_SYRK) {
        const int rs = it.a * kTile, cs = it.b * kTile;
        gemm_k_loop<T>(acc, smem, Pj + nn, ld, rs, na, Pj + nn, ld, cs, na, 0, nn, dj);
        acc_store<2>(acc, M + f.moff, f.ldm, rs, cs, na - rs, na - cs, it.a == it.b, (const T*)nullptr);
    } else {
        // X (rows below the diagonal block, cols [c0, c0+w)) = X * Linv^T (* D^-1)
        const int w = min(kNB, nn - c0);
        const int rs = c0 + w + it.a * kTile;
        const T* Li = inv + f.ioff + (int64_t)(c0 / kNB) * kNB * kNB;
        gemm_k_loop<T>(acc, smem, Pj + (int64_t)c0 * ld, ld, rs, nj, Li, kNB, 0, w, 0, w, (const T*)nullptr);
        __syncthreads();
        T* sc = smem;  // reuse: reciprocal pivots for LDLt
        if (LDLT) {
            for (int i = threadIdx.x; i < w; i += blockDim.x) sc[i] = T(1) / dj[c0 + i];
            __syncthreads();
        }
        acc_store<1>(acc, Pj + (int64_t)c0 * ld, ld, rs, 0, nj - rs, w, false, LDLT ? (const T*)sc : nullptr);
    }
}

// ---------------------------------------------------------------------------
// 256x256 diagonal super-block inverses for the blocked solves, once after
// the factorization.  Super-block K of a front (columns k0 = 256 K ..) is
// made of up to four 64-column blocks with stored inverses D_s; its inverse
// X follows by block forward substitution along the block sub-diagonals:
//   X_ss = D_s,   X_st = -D_s sum_{u=t}^{s-1} L_su X_ut   (s > t),
// 64 x 64 tile products in shared memory, 4 x 4 outputs per thread.
// ---------------------------------------------------------------------------
constexpr int ILD = kNB + 1;

template <typename T>
constexpr int inv256_smem() { return 3 * kNB * ILD * (int)sizeof(T); }

template <typename T>
__device__ __forceinline__ void tile_in(T* dst, const T* src, int64_t ld, int rows, int cols) {
    for (int e = threadIdx.x; e < kNB * kNB; e += blockDim.x) {
        const int r = e & (kNB - 1), c = e >> 6;
        dst[r + c * ILD] = (r < rows && c < cols) ? src[r + (int64_t)c * ld] : T(0);
    }
}

template <typename T>
__device__ __forceinline__ void tile_mma(T (&acc)[4][4], const T* A, const T* B) {
    const int tr = (threadIdx.x >> 4) * 4, tc = (threadIdx.x & 15) * 4;
#pragma unroll 8
    for (int k = 0; k < kNB; ++k) {
        T a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = A[(tr + i) + k * ILD];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = B[k + (tc + j) * ILD];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_inv256(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                const T* __restrict__ P, const T* __restrict__ inv,
                                                T* __restrict__ inv2) {
    pdl_prologue();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* As = reinterpret_cast<T*>(smem_raw);
    T* Bs = As + kNB * ILD;
    T* Cs = Bs + kNB * ILD;
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int K = it.a, k0 = K * kSolveNB, wK = min(kSolveNB, f.nn - k0), ns = (wK + kNB - 1) / kNB;
    const int ld2 = super_ld(wK), ld = f.ldp;
    T* X = inv2 + f.i2off + (int64_t)K * kSolveNB * kSolveNB;
    const T* Pj = P + f.poff;
    const int tid = threadIdx.x;
    for (int e = tid; e < ld2 * wK; e += blockDim.x) X[e] = T(0);
    __syncthreads();
    for (int s = 0; s < ns; ++s) {
        const int ws = min(kNB, wK - s * kNB);
        const T* D = inv + f.ioff + (int64_t)(k0 / kNB + s) * kNB * kNB;
        for (int e = tid; e < ws * ws; e += blockDim.x) {
            const int r = e % ws, c = e / ws;
            X[(s * kNB + r) + (int64_t)(s * kNB + c) * ld2] = D[r + c * kNB];
        }
    }
    __syncthreads();
    const int tr = (tid >> 4) * 4, tc = (tid & 15) * 4;
    for (int d = 1; d < ns; ++d)
        for (int s = d; s < ns; ++s) {
            const int t = s - d;
            const int ws = min(kNB, wK - s * kNB), wt = min(kNB, wK - t * kNB);
            T acc[4][4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
            for (int u = t; u < s; ++u) {  // T += L_su X_ut
                tile_in(As, Pj + (k0 + s * kNB) + (int64_t)(k0 + u * kNB) * ld, ld, ws, kNB);
                tile_in(Bs, X + u * kNB + (int64_t)(t * kNB) * ld2, ld2, kNB, wt);
                __syncthreads();
                tile_mma(acc, As, Bs);
                __syncthreads();
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) Cs[(tr + i) + (tc + j) * ILD] = acc[i][j];
            tile_in(As, inv + f.ioff + (int64_t)(k0 / kNB + s) * kNB * kNB, kNB, kNB, kNB);
            __syncthreads();
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
            tile_mma(acc, As, Cs);
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (tr + i < ws && tc + j < wt)
                        X[(s * kNB + tr + i) + (int64_t)(t * kNB + tc + j) * ld2] = -acc[i][j];
            __syncthreads();  // X_st is read by the next distance
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

template <typename T>
static int assemble_impl(mf_handle* h, const double* dnz, T* P, const double* scale) {
    Timer t(h, K_ASSEMBLE);
    MF_CUDA(cudaMemsetAsync(P, 0, sizeof(T) * h->npanel, h->stream));
    if (h->nnz > 0) {
        int64_t blocks = (h->nnz + 255) / 256;
        if (blocks > 148 * 16) blocks = 148 * 16;
        launch_k(k_scatter<T>, (unsigned)blocks, 256, 0, h->stream, P, h->d_pslot, dnz, h->nnz, h->d_nzrow, h->d_nzcol,
                                                               scale);
        MF_CUDA(cudaGetLastError());
    }
    return 0;
}

int launch_assemble(mf_handle* h, const double* dnz) {
    if (!have_fp64(h)) {
        set_error("no FP64 factor storage: a mixed handle has it only after an FP64 factorization");
        return -1;
    }
    return assemble_impl<double>(h, dnz, h->d_P, nullptr);
}

int launch_assemble_mixed(mf_handle* h, const double* dnz) {
    if (h->n > 0) {
        launch_k(k_diag_scale, (unsigned)((h->n + 255) / 256), 256, 0, h->stream, h->d_scale, h->d_dslot, dnz, h->n);
        MF_CUDA(cudaGetLastError());
    }
    return assemble_impl<float>(h, dnz, h->f32.P, h->d_scale);
}

int launch_dl_to_panel(mf_handle* h, const double* dD, const double* dL) {
    if (!have_fp64(h)) {
        set_error("no FP64 factor storage: a mixed handle has it only after an FP64 factorization");
        return -1;
    }
    Timer t(h, K_OTHER);
    if (h->n == 0) return 0;
    int64_t threads = h->n * 32;
    unsigned blocks = (unsigned)((threads + 255) / 256);
    MF_CUDA(cudaMemsetAsync(h->d_P, 0, sizeof(double) * h->npanel, h->stream));
    launch_k(k_dl_panel<true>, blocks, 256, 0, h->stream, h->d_fronts, h->d_ref, h->d_colfront, h->d_sepmap,
                                                     const_cast<double*>(dD), const_cast<double*>(dL), h->d_P, h->n);
    MF_CUDA(cudaGetLastError());
    return 0;
}

int launch_panel_to_dl(mf_handle* h, double* dD, double* dL) {
    if (!have_fp64(h)) {
        set_error("no FP64 factor storage: a mixed handle has it only after an FP64 factorization");
        return -1;
    }
    if (h->mixed && !h->fp64_current) {
        set_error("the FP64 factor storage does not hold the current matrix: the last mixed factorization "
                  "stayed in FP32");
        return -1;
    }
    Timer t(h, K_OTHER);
    if (h->n == 0) return 0;
    int64_t threads = h->n * 32;
    unsigned blocks = (unsigned)((threads + 255) / 256);
    launch_k(k_dl_panel<false>, blocks, 256, 0, h->stream, h->d_fronts, h->d_ref, h->d_colfront, h->d_sepmap, dD, dL,
                                                      h->d_P, h->n);
    MF_CUDA(cudaGetLastError());
    return 0;
}

int launch_panel32_to_dl(mf_handle* h, double* dD, double* dL) {
    if (h->n == 0) return 0;
    int64_t threads = h->n * 32;
    unsigned blocks = (unsigned)((threads + 255) / 256);
    launch_k(k_panel32_to_dl, blocks, 256, 0, h->stream, h->d_fronts, h->d_ref, h->d_colfront, h->d_sepmap, dD, dL,
                                                   h->f32.P, h->n);
    MF_CUDA(cudaGetLastError());
    return 0;
}


template <typename T, int LDLT>
static int factor_impl(mf_handle* h, const FactorBufs<T>& fb) {
    // the pivot rule applies to the FP64 factorization; the mixed form keeps
    // NoRegularization (its single-precision factor only preconditions)
    const Reg reg = std::is_same<T, double>::value ? h->reg : Reg();
    constexpr int gs = gemm_smem<T>();
    MF_CUDA(cudaFuncSetAttribute(k_small<T, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kSmallMax * kSmallMax * (int)sizeof(T)));
    MF_CUDA(cudaFuncSetAttribute(k_small_warp<T, LDLT, kWarpSmallNJ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kWarpFronts * warp_slice<kWarpSmallNJ>()));
    MF_CUDA(cudaFuncSetAttribute(k_small_warp<T, LDLT, kWarpSmallNJ2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kWarpFronts * warp_slice<kWarpSmallNJ2>()));
    MF_CUDA(cudaFuncSetAttribute(k_diag<T, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, diag_smem<T>()));
    MF_CUDA(cudaFuncSetAttribute(k_inv256<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, inv256_smem<T>()));
    MF_CUDA(cudaFuncSetAttribute(k_gemm<T, G_LEFT, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, gs));
    MF_CUDA(cudaFuncSetAttribute(k_gemm<T, G_TRAIL, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, gs));
    MF_CUDA(cudaFuncSetAttribute(k_gemm<T, G_SYRK, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, gs));
    MF_CUDA(cudaFuncSetAttribute(k_gemm<T, G_TRSM, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, gs));
    const Item* items = h->d_items;
    // per-level timing while autotuning (profile mode: no graph, synchronised)
    cudaEvent_t tev[3] = {nullptr, nullptr, nullptr};
    if (h->tuning) {
        for (auto& e : tev) MF_CUDA(cudaEventCreate(&e));
        h->tune_steps_ms.assign(h->levels.size(), 0.0);
        h->tune_syrk_ms.assign(h->levels.size(), 0.0);
    }
    for (size_t L = 0; L < h->levels.size(); ++L) {
        const Level& lv = h->levels[L];
        if (lv.small_warp.cnt) {
            Timer t(h, K_SMALL);
            const unsigned g = (unsigned)((lv.small_warp.cnt + kWarpFronts - 1) / kWarpFronts);
            launch_k(k_small_warp<T, LDLT, kWarpSmallNJ>, g, kWarpFronts * 32, kWarpFronts * warp_slice<kWarpSmallNJ>(),
                h->stream, h->d_fronts, items + lv.small_warp.off, lv.small_warp.cnt, h->d_reltgt, h->d_chdtgt, fb.P,
                fb.M, fb.d, h->d_signs, h->d_info, h->d_rescued, reg);
            MF_CUDA(cudaGetLastError());
        }
        if (lv.small_warp2.cnt) {
            Timer t(h, K_SMALL);
            const unsigned g = (unsigned)((lv.small_warp2.cnt + kWarpFronts - 1) / kWarpFronts);
            launch_k(k_small_warp<T, LDLT, kWarpSmallNJ2>, g, kWarpFronts * 32,
                kWarpFronts * warp_slice<kWarpSmallNJ2>(), h->stream, h->d_fronts, items + lv.small_warp2.off,
                lv.small_warp2.cnt, h->d_reltgt, h->d_chdtgt, fb.P, fb.M, fb.d, h->d_signs, h->d_info, h->d_rescued,
                reg);
            MF_CUDA(cudaGetLastError());
        }
        if (lv.small.cnt) {
            Timer t(h, K_SMALL);
            // shared memory for the level's largest front (as FP64 up to
            // kSmallRescue rows, for the in-place rescue of an FP32 front) and
            // 128 threads for levels of many narrow fronts: more fronts in
            // flight (a level of few fronts keeps 256 threads, for latency)
            const int mj = lv.small_maxnj;
            const int rj = std::min(mj, kSmallRescue);
            const size_t sm = std::max<size_t>((size_t)mj * mj * sizeof(T), sizeof(T) == 4 ? (size_t)rj * rj * 8 : 0);
            const bool wide = lv.small.cnt >= kSmallWideLevel;
            const unsigned nt = !wide || mj > kSmallNarrowNJ ? 256 : mj <= kSmallTinyNJ ? 64 : 128;
            launch_k(k_small<T, LDLT>, grid_for(lv.small.cnt), nt, sm, h->stream, 
                h->d_fronts, items + lv.small.off, h->d_reltgt, h->d_chdtgt, fb.P, fb.M, fb.d, h->d_signs,
                h->d_info, h->d_rescued, reg);
            MF_CUDA(cudaGetLastError());
        }
        if (lv.ea.cnt) {
            Timer t(h, K_EA);
            launch_k(k_ea<T, 0>, grid_for(lv.ea.cnt), 256, 0, h->stream, h->d_fronts, items + lv.ea.off, items,
                                                                   h->d_reltgt, fb.P, fb.M);
            MF_CUDA(cudaGetLastError());
        }
        if (h->tuning) MF_CUDA(cudaEventRecord(tev[0], h->stream));
        // Look-ahead: an outer block's trailing update runs its tiles of the
        // next outer block's columns on `stream` and the rest on `side`,
        // beside the next block's sub-panels (which touch only their own
        // columns); `stream` waits for `side` before the next trailing update
        // (its columns overlap, and it reuses the split operands) and before
        // the SYRK.  The persistent tensor-core kernel on `side` leaves
        // side_free_sms SMs to the sub-panel kernels.  Profile and tuning runs
        // stay on one stream.
        const bool la_on = h->lookahead && h->side && !h->profile && !h->tuning;
        bool pending = false;
        auto join = [&]() -> int {
            if (pending) MF_CUDA(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
            pending = false;
            return 0;
        };
        // launch `body` on `side` after the work queued on `stream` so far
        auto on_side = [&](const std::function<int()>& body) -> int {
            MF_CUDA(cudaEventRecord(h->ev_fork, h->stream));
            MF_CUDA(cudaStreamWaitEvent(h->side, h->ev_fork, 0));
            cudaStream_t main = h->stream;
            h->stream = h->side;
            h->grid_cap = std::max(1, (h->num_sms > 0 ? h->num_sms : 148) - h->side_free_sms);
            const int rc = body();
            h->grid_cap = 0;
            h->stream = main;
            if (rc) return rc;
            MF_CUDA(cudaEventRecord(h->ev_join, h->side));
            pending = true;
            return 0;
        };
        for (const PanelStep& st : lv.steps) {
            const int obs = st.b * lv.kob, obw = lv.kob;
            const int c0 = obs + st.s * kNB;
            if (std::is_same<T, float>::value && h->use_tc && lv.tc_steps) {
                // single precision: the GEMM roles run on the tcgen05 tensor cores
                const FactorBufs<float>& f32b = reinterpret_cast<const FactorBufs<float>&>(fb);
                int rc;
                if (st.left_tc.cnt) {
                    Timer t(h, K_LEFT);
                    if ((rc = tc_launch(h, 0, st.left_tc, obs, obw, c0, f32b))) return rc;
                }
                if (st.diag.cnt) {
                    Timer t(h, K_DIAG);
                    launch_kx(h->panel_pdl || pdl_enabled(), k_diag<T, LDLT>, grid_for(st.diag.cnt), 256,
                        diag_smem<T>(), h->stream, h->d_fronts, items + st.diag.off, c0, fb.P, fb.inv, fb.d,
                        h->d_signs, h->d_info, h->d_rescued, reg);
                    MF_CUDA(cudaGetLastError());
                }
                if (st.panel_tc.cnt) {
                    Timer t(h, K_PANEL);
                    if ((rc = tc_launch(h, 3, st.panel_tc, obs, obw, c0, f32b))) return rc;
                }
                if (st.trail_tc.cnt) {
                    Timer t(h, K_UPDATE);
                    if ((rc = join())) return rc;
                    const bool la = la_on && st.trail_tc_ncrit > 0 && st.trail_tc_ncrit < st.trail_tc.cnt;
                    const ItemList crit{st.trail_tc.off, la ? st.trail_tc_ncrit : st.trail_tc.cnt};
                    rc = h->tc_split ? tc_launch_split(h, 1, crit, st.split_tc, obs, obw, c0, f32b)
                                     : tc_launch(h, 1, crit, obs, obw, c0, f32b);
                    if (rc) return rc;
                    if (la) {
                        const ItemList bulk{st.trail_tc.off + st.trail_tc_ncrit, st.trail_tc.cnt - st.trail_tc_ncrit};
                        rc = on_side([&]() {
                            return h->tc_split ? tc_launch_split(h, 1, bulk, ItemList{}, obs, obw, c0, f32b)
                                               : tc_launch(h, 1, bulk, obs, obw, c0, f32b);
                        });
                        if (rc) return rc;
                    }
                }
                continue;
            }
            if (st.left.cnt) {
                Timer t(h, K_LEFT);
                launch_kx(h->panel_pdl || pdl_enabled(), k_gemm<T, G_LEFT, LDLT>, grid_for(st.left.cnt), 256, gs,
                    h->stream, h->d_fronts, items + st.left.off, obs, obw, c0, fb.P, fb.M, fb.d, fb.inv);
                MF_CUDA(cudaGetLastError());
            }
            if (st.diag.cnt) {
                Timer t(h, K_DIAG);
                launch_kx(h->panel_pdl || pdl_enabled(), k_diag<T, LDLT>, grid_for(st.diag.cnt), 256,
                    diag_smem<T>(), h->stream, h->d_fronts, items + st.diag.off, c0, fb.P, fb.inv, fb.d,
                    h->d_signs, h->d_info, h->d_rescued, reg);
                MF_CUDA(cudaGetLastError());
            }
            if (st.panel.cnt) {
                Timer t(h, K_PANEL);
                launch_kx(h->panel_pdl || pdl_enabled(), k_gemm<T, G_TRSM, LDLT>, grid_for(st.panel.cnt), 256, gs,
                    h->stream, h->d_fronts, items + st.panel.off, obs, obw, c0, fb.P, fb.M, fb.d, fb.inv);
                MF_CUDA(cudaGetLastError());
            }
            if (st.trail.cnt) {
                Timer t(h, K_UPDATE);
                if (int rc = join()) return rc;
                const bool la = la_on && st.trail_ncrit > 0 && st.trail_ncrit < st.trail.cnt;
                const int64_t ncrit = la ? st.trail_ncrit : st.trail.cnt;
                launch_k(k_gemm<T, G_TRAIL, LDLT>, grid_for(ncrit), 256, gs, h->stream,
                    h->d_fronts, items + st.trail.off, obs, obw, c0, fb.P, fb.M, fb.d, fb.inv);
                MF_CUDA(cudaGetLastError());
                if (la) {
                    const int rc = on_side([&]() -> int {
                        launch_k(k_gemm<T, G_TRAIL, LDLT>, grid_for(st.trail.cnt - ncrit), 256, gs, h->stream,
                            h->d_fronts, items + st.trail.off + ncrit, obs, obw, c0, fb.P, fb.M, fb.d, fb.inv);
                        MF_CUDA(cudaGetLastError());
                        return 0;
                    });
                    if (rc) return rc;
                }
            }
        }
        if (int rc = join()) return rc;
        if (h->tuning) MF_CUDA(cudaEventRecord(tev[1], h->stream));
        if (std::is_same<T, float>::value && h->use_tc && lv.tc_syrk) {
            if (lv.syrk_tc.cnt) {
                Timer t(h, K_SYRK);
                const FactorBufs<float>& f32b = reinterpret_cast<const FactorBufs<float>&>(fb);
                int rc = h->tc_split ? tc_launch_split(h, 2, lv.syrk_tc, lv.split_syrk, 0, 0, 0, f32b)
                                     : tc_launch(h, 2, lv.syrk_tc, 0, 0, 0, f32b);
                if (rc) return rc;
            }
        } else if (lv.syrk.cnt) {
            Timer t(h, K_SYRK);
            launch_k(k_gemm<T, G_SYRK, LDLT>, grid_for(lv.syrk.cnt), 256, gs, h->stream, 
                h->d_fronts, items + lv.syrk.off, 0, 0, 0, fb.P, fb.M, fb.d, fb.inv);
            MF_CUDA(cudaGetLastError());
        }
        if (lv.ea_upd.cnt) {
            Timer t(h, K_EA);
            launch_k(k_ea<T, 1>, grid_for(lv.ea_upd.cnt), 256, 0, h->stream, h->d_fronts, items + lv.ea_upd.off, items,
                                                                       h->d_reltgt, fb.P, fb.M);
            MF_CUDA(cudaGetLastError());
        }
        if (h->tuning) {
            MF_CUDA(cudaEventRecord(tev[2], h->stream));
            MF_CUDA(cudaEventSynchronize(tev[2]));
            float a = 0.f, b = 0.f;
            MF_CUDA(cudaEventElapsedTime(&a, tev[0], tev[1]));
            MF_CUDA(cudaEventElapsedTime(&b, tev[1], tev[2]));
            h->tune_steps_ms[L] += a;
            h->tune_syrk_ms[L] += b;
        }
    }
    if (h->tuning)
        for (auto& e : tev) cudaEventDestroy(e);
    if (h->inv2_items.cnt) {
        Timer t(h, K_OTHER);
        launch_k(k_inv256<T>, grid_for(h->inv2_items.cnt), 256, inv256_smem<T>(), h->stream, 
            h->d_fronts, items + h->inv2_items.off, fb.P, fb.inv, fb.inv2);
        MF_CUDA(cudaGetLastError());
    }
    return 0;
}

int run_captured(mf_handle* h, int64_t k0, int64_t k1, int64_t k2, int64_t k3, const std::function<int()>& body) {
    if (!h->use_graphs || h->profile || h->tuning || !h->stream) return body();
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    MF_CUDA(cudaStreamIsCapturing(h->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return body();
    for (const GraphEntry& g : h->graphs)
        if (g.key[0] == k0 && g.key[1] == k1 && g.key[2] == k2 && g.key[3] == k3) {
            MF_CUDA(cudaGraphLaunch(g.exec, h->stream));
            return 0;
        }
    std::lock_guard<std::recursive_mutex> lk(device_mutex());
    MF_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = body();
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    if (rc || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return rc ? rc : cuda_fail(e, "cudaStreamEndCapture");
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate");
    h->graphs.push_back(GraphEntry{{k0, k1, k2, k3}, exec});
    MF_CUDA(cudaGraphLaunch(exec, h->stream));
    return 0;
}

void release_graphs(mf_handle* h) {
    for (GraphEntry& g : h->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    h->graphs.clear();
}

// graph keys: kind (1 FP64 factor, 2 FP32 factor), then what the launch
// sequence reads through pointers that can change between calls
int launch_factor(mf_handle* h) {
    if (!have_fp64(h)) {
        set_error("no FP64 factor storage: a mixed handle has it only after an FP64 factorization");
        return -1;
    }
    FactorBufs<double> fb{h->d_P, h->d_M, h->d_inv, h->d_d, h->d_inv2};
    int rc = run_captured(h, 1, (int64_t)(uintptr_t)h->d_signs, 0, 0, [&]() {
        return h->diag ? factor_impl<double, 1>(h, fb) : factor_impl<double, 0>(h, fb);
    });
    h->fp64_current = rc == 0;
    h->selinv_done = false;
    return rc;
}

int launch_factor_mixed(mf_handle* h) {
    FactorBufs<float> fb{h->f32.P, h->f32.M, h->f32.inv, h->f32.d, h->f32.inv2};
    if (h->use_tc) {
        int rc = tc_prepare(h);
        if (rc) return rc;
    }
    return run_captured(h, 2, (int64_t)(uintptr_t)h->d_signs, h->use_tc ? 1 : 0, 0, [&]() {
        return h->diag ? factor_impl<float, 1>(h, fb) : factor_impl<float, 0>(h, fb);
    });
}

}  // namespace mf

// ---------------------------------------------------------------------------
// log|det| of the factored matrix, reduced on the device
// (LinearAlgebra.logabsdet / logdet / det of a ChordalFactorization,
// src/Multifrontal.jl/src/abstract_factorization.jl:156-179).  Cholesky: the
// terms are log of the squared diagonal of L; LDLt: log|d_j| and the sign of
// d_j.  A mixed handle without an FP64 factor uses its single-precision factor
// of S A S and adds -2 log s_j.  Each block reduces a contiguous range of
// columns in a fixed tree order and writes (sum, negatives, zeros); the host
// adds the block results in block order, so the result is bitwise repeatable.
// ---------------------------------------------------------------------------
namespace mf {

constexpr int kLogdetThreads = 256;
constexpr int kLogdetBlocks = 296;  // 2 x 148 SMs

template <typename T, int UNIT>
__global__ void __launch_bounds__(kLogdetThreads)
k_logdet(const Front* __restrict__ fronts, const RefFront* __restrict__ ref, const int32_t* __restrict__ colref,
         const T* __restrict__ P, const T* __restrict__ d, const double* __restrict__ scale, int64_t n,
         double* __restrict__ out) {
    pdl_prologue();
    __shared__ double s_sum[kLogdetThreads];
    __shared__ int s_neg[kLogdetThreads], s_zero[kLogdetThreads];
    const int64_t per = (n + gridDim.x - 1) / gridDim.x;
    const int64_t c0 = blockIdx.x * per;
    const int64_t c1 = c0 + per < n ? c0 + per : n;
    double acc = 0.0;
    int neg = 0, zero = 0;
    for (int64_t c = c0 + threadIdx.x; c < c1; c += kLogdetThreads) {
        double v;
        if (UNIT) {
            v = (double)d[c];
        } else {
            const RefFront rf = ref[colref[c]];
            const Front f = fronts[rf.exec];
            const int64_t k = c - f.col0;
            const double l = (double)P[f.poff + k + k * f.ldp];
            v = l * l;
        }
        if (scale) v /= scale[c] * scale[c];
        if (v == 0.0) zero += 1;
        if (v < 0.0) neg += 1;
        acc += log(fabs(v));
    }
    s_sum[threadIdx.x] = acc;
    s_neg[threadIdx.x] = neg;
    s_zero[threadIdx.x] = zero;
    __syncthreads();
    for (int w = kLogdetThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            s_sum[threadIdx.x] += s_sum[threadIdx.x + w];
            s_neg[threadIdx.x] += s_neg[threadIdx.x + w];
            s_zero[threadIdx.x] += s_zero[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[3 * blockIdx.x] = s_sum[0];
        out[3 * blockIdx.x + 1] = (double)s_neg[0];
        out[3 * blockIdx.x + 2] = (double)s_zero[0];
    }
}

int launch_logdet(mf_handle* h, double* logabsdet, double* sign) {
    const bool fp64 = have_fp64(h) && (!h->mixed || h->fp64_current);
    if (!fp64 && !h->mixed) {
        set_error("mf_logdet: no factor on the device");
        return -1;
    }
    if (!h->d_logdet) {
        std::lock_guard<std::recursive_mutex> lk(device_mutex());
        MF_CUDA(cudaMalloc((void**)&h->d_logdet, sizeof(double) * 3 * kLogdetBlocks));
        h->bytes += (int64_t)sizeof(double) * 3 * kLogdetBlocks;
    }
    double* part = h->d_logdet;
    const int64_t n = h->n;
    if (n > 0) {
        if (fp64) {
            if (h->diag)
                launch_k(k_logdet<double, 1>, kLogdetBlocks, kLogdetThreads, 0, h->stream, 
                    h->d_fronts, h->d_ref, h->d_colfront, h->d_P, h->d_d, nullptr, n, part);
            else
                launch_k(k_logdet<double, 0>, kLogdetBlocks, kLogdetThreads, 0, h->stream, 
                    h->d_fronts, h->d_ref, h->d_colfront, h->d_P, h->d_d, nullptr, n, part);
        } else {
            if (h->diag)
                launch_k(k_logdet<float, 1>, kLogdetBlocks, kLogdetThreads, 0, h->stream, 
                    h->d_fronts, h->d_ref, h->d_colfront, h->f32.P, h->f32.d, h->d_scale, n, part);
            else
                launch_k(k_logdet<float, 0>, kLogdetBlocks, kLogdetThreads, 0, h->stream, 
                    h->d_fronts, h->d_ref, h->d_colfront, h->f32.P, h->f32.d, h->d_scale, n, part);
        }
        MF_CUDA(cudaGetLastError());
    }
    std::vector<double> hp(3 * kLogdetBlocks, 0.0);
    cudaError_t e = cudaSuccess;
    if (n > 0)
        e = cudaMemcpyAsync(hp.data(), part, sizeof(double) * 3 * kLogdetBlocks, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "mf_logdet");
    double sum = 0.0, neg = 0.0, zero = 0.0;
    for (int b = 0; b < kLogdetBlocks; ++b) {
        sum += hp[3 * b];
        neg += hp[3 * b + 1];
        zero += hp[3 * b + 2];
    }
    *logabsdet = zero > 0 ? -INFINITY : sum;
    *sign = zero > 0 ? 0.0 : (fmod(neg, 2.0) == 0.0 ? 1.0 : -1.0);
    return 0;
}

}  // namespace mf
