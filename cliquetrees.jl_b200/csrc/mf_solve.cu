// Supernodal forward and backward solves (FP64) for the B200 multifrontal
// solver, with many right-hand sides.
//
// Reference: div_impl! (src/Multifrontal.jl/src/divide.jl:417-450), the
// forward loop div_fwd_loop_snd!/_nod! (:493-821) with div_fwd_update!
// (:1206-1248), the backward loop div_bwd_loop_snd!/_nod! (:864-1204) with
// div_bwd_update! (:1250-1293), and ldiv!(W, NaturalFactorization, B)
// (:191-199) for the L, D, L^T sequence.
//
// Layout: C (n x nrhs, ld n) holds the right-hand sides in elimination
// order and receives the solution.  Forward updates of front j (the
// reference's M2 = F2 - L21 C1 pushed on the stack) live at R + roff_j*nrhs
// (na x nrhs, ld na) and are pulled by the parent.  In the backward pass the
// reference pushes F restricted to sep(i) to each child; that vector is the
// already-final solution at rows sep(i), so children read it from C directly.
#include "mf_internal.cuh"

namespace mf {

constexpr int kMaxRhs = 16;   // right-hand sides per pass (larger counts are chunked)

// ---------------------------------------------------------------------------
// permutation (mul!(C, P, B), multiply.jl:277-280): C[i] = B[perm[i]]
// ---------------------------------------------------------------------------
template <bool IN>
__global__ void k_perm(double* __restrict__ C, double* B, const int64_t* __restrict__ perm, int64_t n,
                       int64_t ldb, int nrhs) {
    pdl_prologue();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n * nrhs; i += stride) {
        int64_t r = i / n, row = i % n;
        if (IN) C[row + r * n] = B[perm[row] + r * ldb];
        else B[perm[row] + r * ldb] = C[row + r * n];
    }
}

template <typename T>
__global__ void k_diag_div(T* __restrict__ C, const T* __restrict__ d, int64_t n, int nrhs) {
    pdl_prologue();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n * nrhs; i += stride) C[i] /= d[i % n];
}

// ---------------------------------------------------------------------------
// small fronts (nj <= 96, or nn <= 64 and na <= 256): one warp per front,
// kSmallWarps fronts per CTA, warp-synchronous (no block barriers).  The
// front's right-hand-side block C1 (nn x nrhs) lives in the warp's slice of
// shared memory; lane i holds rows i, i + 32, i + 64 in registers during the
// triangular solves.
// ---------------------------------------------------------------------------
constexpr int kSmallWarps = 4;
constexpr int kSmallRows = (kSmallMax + 31) / 32;  // rows per lane (3)

template <typename T, int NR>
constexpr int small_solve_smem() { return kSmallWarps * kSmallMax * NR * (int)sizeof(T); }

constexpr int kSmallChunk = 4;  // triangular-solve steps whose panel loads are issued together

// Resident 128-thread CTAs per SM the small-front solves are compiled for
// (a register budget): the per-front work is a chain of dependent loads, so
// warps in flight set the throughput; wide right-hand-side blocks need the
// registers instead.
template <typename T, int NR>
constexpr int small_min_blocks() { return sizeof(T) == 4 ? (NR <= 4 ? 6 : 4) : (NR <= 4 ? 4 : 2); }

// Loads for steps k0 .. k0 + kSmallChunk - 1 of a small front's triangular
// solve: lane i gets, for rows a = i + 32 s, the strictly lower entry L_ak of
// column k (forward, TRANS = 0) or the entry L_ka of row k left of the
// diagonal (backward, TRANS = 1), zero elsewhere, and the diagonal L_kk.
template <typename T, int UNIT, int TRANS = 0>
__device__ __forceinline__ void small_cols(T (&l)[kSmallChunk][kSmallRows], T (&dg)[kSmallChunk],
                                           const T* __restrict__ Pj, int ld, int nn, int k0, int lane) {
#pragma unroll
    for (int q = 0; q < kSmallChunk; ++q) {
        const int k = TRANS ? k0 - q : k0 + q;
        const bool kv = k >= 0 && k < nn;
#pragma unroll
        for (int s = 0; s < kSmallRows; ++s) {
            const int a = lane + 32 * s;
            const bool v = kv && (TRANS ? a < k : (a > k && a < nn));
            l[q][s] = v ? (TRANS ? Pj[k + (int64_t)a * ld] : Pj[a + (int64_t)k * ld]) : T(0);
        }
        dg[q] = (!UNIT && kv) ? Pj[k + (int64_t)k * ld] : T(1);
    }
}

// One small front's forward step, by one warp (C1: the warp's shared slice,
// C1[a + r * kSmallMax]).  The children's update blocks are read through L2
// (ld.cg): in k_s_sub_fwd another warp of the CTA wrote them.
template <typename T, int UNIT, int NR>
__device__ __forceinline__ void small_fwd_front(const Front& f, const Front* __restrict__ fronts,
                                                const int32_t* __restrict__ reltgt,
                                                const int32_t* __restrict__ chdtgt, const T* __restrict__ P,
                                                T* C, T* R, int64_t n, int nrhs, T* C1, int lane) {
    const int nn = f.nn, na = f.na, ld = f.ldp;
    const T* Pj = P + f.poff;
    T* Rj = R + f.roff * nrhs;
    for (int i = lane; i < nn * nrhs; i += 32) {
        const int a = i % nn, r = i / nn;
        C1[a + r * kSmallMax] = C[f.col0 + a + (int64_t)r * n];
    }
    for (int i = lane; i < na * nrhs; i += 32) Rj[i] = T(0);
    // lane q fetches the record of the q-th child to add (children past 32
    // are read in the loop)
    const int nch = f.chd1 - f.chd0;
    int kna = 0, ksep = 0;
    int64_t kroff = 0;
    if (lane < nch) {
        const Front fc = fronts[chdtgt[f.chd1 - 1 - lane]];
        kna = fc.na, ksep = fc.sep0, kroff = fc.roff;
    }
    __syncwarp();
    // child updates, children in reverse order (the reference pops its stack)
    for (int q = 0; q < nch; ++q) {
        int ma = __shfl_sync(0xffffffffu, kna, q & 31), sep0 = __shfl_sync(0xffffffffu, ksep, q & 31);
        int64_t roff = __shfl_sync(0xffffffffu, kroff, q & 31);
        if (q >= 32) {
            const Front fc = fronts[chdtgt[f.chd1 - 1 - q]];
            ma = fc.na, sep0 = fc.sep0, roff = fc.roff;
        }
        const int32_t* rel = reltgt + sep0;
        const T* Mc = R + roff * nrhs;
        // four loads per lane in flight before the adds (the child's rows
        // are distinct, so one child's adds never collide)
        for (int i0 = 0; i0 < ma * nrhs; i0 += 128) {
            int qv[4];
            T mv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int i = i0 + 32 * u + lane;
                qv[u] = -1;
                mv[u] = T(0);
                if (i < ma * nrhs) {
                    qv[u] = rel[i % ma];
                    mv[u] = __ldcg(Mc + i);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (qv[u] < 0) continue;
                const int r = (i0 + 32 * u + lane) / ma;
                if (qv[u] < nn) C1[qv[u] + r * kSmallMax] += mv[u];
                else Rj[(qv[u] - nn) + r * na] += mv[u];
            }
        }
        __syncwarp();
    }
    // forward substitution, column oriented: x_k = C1[k] / L_kk, then
    // rows a > k lose L_ak x_k
    T x[kSmallRows][NR];
#pragma unroll
    for (int s = 0; s < kSmallRows; ++s)
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const int a = lane + 32 * s;
            x[s][r] = (a < nn && r < nrhs) ? C1[a + r * kSmallMax] : T(0);
        }
    // The columns come in chunks of kSmallChunk: the next chunk's loads are
    // issued before the current chunk's steps, so the step chain waits on
    // shuffles and FMAs rather than on one load per column.
    T ln[kSmallChunk][kSmallRows], dn[kSmallChunk];
    small_cols<T, UNIT>(ln, dn, Pj, ld, nn, 0, lane);
    for (int k0 = 0; k0 < nn; k0 += kSmallChunk) {
        T lc[kSmallChunk][kSmallRows], dc[kSmallChunk];
#pragma unroll
        for (int q = 0; q < kSmallChunk; ++q) {
            dc[q] = dn[q];
#pragma unroll
            for (int s = 0; s < kSmallRows; ++s) lc[q][s] = ln[q][s];
        }
        small_cols<T, UNIT>(ln, dn, Pj, ld, nn, k0 + kSmallChunk, lane);
#pragma unroll
        for (int q = 0; q < kSmallChunk; ++q) {
            const int k = k0 + q;
            if (k >= nn) break;  // uniform across the warp
            const int ko = k & 31, ks = k >> 5;
            const T dinv = UNIT ? T(1) : T(1) / dc[q];
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                T own = ks == 0 ? x[0][r] : (ks == 1 ? x[1][r] : x[2][r]);
                const T xk = __shfl_sync(0xffffffffu, own, ko) * dinv;
#pragma unroll
                for (int s = 0; s < kSmallRows; ++s) x[s][r] -= lc[q][s] * xk;
                if (lane == ko) {
                    if (ks == 0) x[0][r] = xk; else if (ks == 1) x[1][r] = xk; else x[2][r] = xk;
                }
            }
        }
    }
#pragma unroll
    for (int s = 0; s < kSmallRows; ++s) {
        const int a = lane + 32 * s;
        if (a < nn)
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) {
                    C1[a + r * kSmallMax] = x[s][r];
                    C[f.col0 + a + (int64_t)r * n] = x[s][r];
                }
    }
    __syncwarp();
    // R_j -= L21 x: lanes own rows of L21 (coalesced along the panel
    // columns), two rows (a, a + 32) at a time with eight columns of both
    // loaded before their products: sixteen loads in flight per lane
    for (int a = lane; a < na; a += 64) {
        const bool two = a + 32 < na;
        T acc0[NR], acc1[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) acc0[r] = acc1[r] = T(0);
        const T* lr0 = Pj + nn + a;
        const T* lr1 = lr0 + 32;
        for (int k0 = 0; k0 < nn; k0 += 8) {
            T l0[8], l1[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int k = k0 + u;
                l0[u] = k < nn ? lr0[(int64_t)k * ld] : T(0);
                l1[u] = (two && k < nn) ? lr1[(int64_t)k * ld] : T(0);
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int k = k0 + u;
                if (k < nn)
#pragma unroll
                    for (int r = 0; r < NR; ++r) {
                        const T c = C1[k + r * kSmallMax];
                        acc0[r] += l0[u] * c;
                        acc1[r] += l1[u] * c;
                    }
            }
        }
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) {
                Rj[a + r * na] -= acc0[r];
                if (two) Rj[a + 32 + r * na] -= acc1[r];
            }
    }
}

template <typename T, int UNIT, int NR>
__global__ void __launch_bounds__(kSmallWarps * 32, small_min_blocks<T, NR>()) k_s_small_fwd(const Front* __restrict__ fronts,
                                                                  const Item* __restrict__ items, int64_t cnt,
                                                                  const int32_t* __restrict__ reltgt,
                                                                  const int32_t* __restrict__ chdtgt,
                                                                  const T* __restrict__ P, T* __restrict__ C,
                                                                  T* __restrict__ R, int64_t n, int nrhs) {
    pdl_prologue();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t w = (int64_t)blockIdx.x * kSmallWarps + wib;
    if (w >= cnt) return;  // whole warps only
    T* C1 = reinterpret_cast<T*>(sm_raw) + wib * kSmallMax * NR;
    const Front f = fronts[items[w].front];
    small_fwd_front<T, UNIT, NR>(f, fronts, reltgt, chdtgt, P, C, R, n, nrhs, C1, lane);
}

// One small front's backward step, by one warp.  x[sep] is read through L2
// (ld.cg): in k_s_sub_bwd the ancestors' warps of the same CTA wrote it.
template <typename T, int UNIT, int NR>
__device__ __forceinline__ void small_bwd_front(const Front& f, const int32_t* __restrict__ septgt,
                                                const T* __restrict__ P, T* C, int64_t n, int nrhs, int lane) {
    const int nn = f.nn, na = f.na, ld = f.ldp;
    const T* Pj = P + f.poff;
    const int32_t* sep = septgt + f.sep0;
    // C[res] - L21^T x[sep]: lanes own columns k and walk the rows a in
    // order, 32 rows at a time: lane i gathers x[sep[a0 + i]] for the chunk
    // (the next chunk's gather is issued before this chunk's products) and
    // the rows' x values reach the other lanes by shuffles
    T acc[kSmallRows][NR];
#pragma unroll
    for (int s = 0; s < kSmallRows; ++s)
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[s][r] = T(0);
    T xv[NR];
    {
        const bool v = lane < na;
        const int64_t row = v ? sep[lane] : 0;
#pragma unroll
        for (int r = 0; r < NR; ++r) xv[r] = (v && r < nrhs) ? __ldcg(C + row + (int64_t)r * n) : T(0);
    }
    for (int a0 = 0; a0 < na; a0 += 32) {
        T xn[NR];
        {
            const int a = a0 + 32 + lane;
            const bool v = a < na;
            const int64_t row = v ? sep[a] : 0;
#pragma unroll
            for (int r = 0; r < NR; ++r) xn[r] = (v && r < nrhs) ? __ldcg(C + row + (int64_t)r * n) : T(0);
        }
        const int m = min(32, na - a0);
        const T* pa = Pj + nn + a0;
#pragma unroll 8
        for (int j = 0; j < m; ++j) {
            T xb[NR];
#pragma unroll
            for (int r = 0; r < NR; ++r) xb[r] = __shfl_sync(0xffffffffu, xv[r], j);
#pragma unroll
            for (int s = 0; s < kSmallRows; ++s) {
                const int k = lane + 32 * s;
                if (k < nn) {
                    const T l = pa[j + (int64_t)k * ld];
#pragma unroll
                    for (int r = 0; r < NR; ++r) acc[s][r] += l * xb[r];
                }
            }
        }
#pragma unroll
        for (int r = 0; r < NR; ++r) xv[r] = xn[r];
    }
    // C1 in registers: lane i holds rows k = i + 32 s
    T c[kSmallRows][NR];
#pragma unroll
    for (int s = 0; s < kSmallRows; ++s) {
        const int k = lane + 32 * s;
#pragma unroll
        for (int r = 0; r < NR; ++r)
            c[s][r] = (k < nn && r < nrhs) ? C[f.col0 + k + (int64_t)r * n] - acc[s][r] : T(0);
    }
    // back substitution, column oriented on L^T: x_k = c_k / L_kk, k
    // descending, then rows j < k lose L_kj x_k; the rows of L for the next
    // kSmallChunk steps are loaded while the current ones are applied
    T ln[kSmallChunk][kSmallRows], dn[kSmallChunk];
    small_cols<T, UNIT, 1>(ln, dn, Pj, ld, nn, nn - 1, lane);
    for (int k0 = nn - 1; k0 >= 0; k0 -= kSmallChunk) {
        T lc[kSmallChunk][kSmallRows], dc[kSmallChunk];
#pragma unroll
        for (int q = 0; q < kSmallChunk; ++q) {
            dc[q] = dn[q];
#pragma unroll
            for (int s = 0; s < kSmallRows; ++s) lc[q][s] = ln[q][s];
        }
        small_cols<T, UNIT, 1>(ln, dn, Pj, ld, nn, k0 - kSmallChunk, lane);
#pragma unroll
        for (int q = 0; q < kSmallChunk; ++q) {
            const int k = k0 - q;
            if (k < 0) break;  // uniform across the warp
            const int ko = k & 31, ks = k >> 5;
            const T dinv = UNIT ? T(1) : T(1) / dc[q];
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                T own = ks == 0 ? c[0][r] : (ks == 1 ? c[1][r] : c[2][r]);
                const T xk = __shfl_sync(0xffffffffu, own, ko) * dinv;
#pragma unroll
                for (int s = 0; s < kSmallRows; ++s) c[s][r] -= lc[q][s] * xk;
                if (lane == ko) {
                    if (ks == 0) c[0][r] = xk; else if (ks == 1) c[1][r] = xk; else c[2][r] = xk;
                }
            }
        }
    }
#pragma unroll
    for (int s = 0; s < kSmallRows; ++s) {
        const int k = lane + 32 * s;
        if (k < nn)
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs) C[f.col0 + k + (int64_t)r * n] = c[s][r];
    }
}

template <typename T, int UNIT, int NR>
__global__ void __launch_bounds__(kSmallWarps * 32, small_min_blocks<T, NR>()) k_s_small_bwd(const Front* __restrict__ fronts,
                                                                  const Item* __restrict__ items, int64_t cnt,
                                                                  const int32_t* __restrict__ septgt,
                                                                  const T* __restrict__ P, T* __restrict__ C,
                                                                  int64_t n, int nrhs) {
    pdl_prologue();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t w = (int64_t)blockIdx.x * kSmallWarps + wib;
    if (w >= cnt) return;
    const Front f = fronts[items[w].front];
    small_bwd_front<T, UNIT, NR>(f, septgt, P, C, n, nrhs, lane);
}

// ---------------------------------------------------------------------------
// Tiny fronts (nj <= G, G = 16 or 32): G lanes per front (two fronts per warp
// for G = 16), lane g owning row g of its front (forward) or column g
// (backward).  Each lane
// issues all its panel loads at the start (row g of the panel forward,
// column g backward), so a front costs a few dependent memory trips instead
// of k_s_small_*'s chain of column steps, and for G = 16 twice as many
// fronts are in flight per warp.  Loops over columns run to the warp's
// largest front (shuffles take the whole warp) with the other front's steps
// predicated off.  Each entry gets the
// operations of k_s_small_fwd / _bwd in the same order, so the results are
// bitwise equal to them.
// ---------------------------------------------------------------------------
constexpr int kTinyWarps = 4;
template <int G>
constexpr int tiny_fronts() { return kTinyWarps * 32 / G; }  // fronts per CTA

// the larger of v and the other front's v in the warp (G = 16)
template <int G>
__device__ __forceinline__ int tiny_warp_max(int v) {
    return G == 32 ? v : max(v, __shfl_xor_sync(0xffffffffu, v, 16));
}

template <typename T, int NR, int G>
constexpr int tiny_min_blocks() {
    return G == 16 ? (sizeof(T) == 4 ? (NR <= 4 ? 10 : NR <= 8 ? 8 : 4) : (NR <= 2 ? 8 : NR <= 4 ? 6 : NR <= 8 ? 4 : 3))
                   : (sizeof(T) == 4 ? (NR <= 4 ? 8 : NR <= 8 ? 6 : 3) : (NR <= 4 ? 4 : NR <= 8 ? 3 : 2));
}

__device__ __forceinline__ Front tiny_front(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                            int64_t w, int64_t cnt) {
    Front f{};
    if (w < cnt) f = fronts[items[w].front];
    else f.chd0 = f.chd1 = 0;  // nn = na = 0: every step predicated off
    return f;
}

template <typename T, int UNIT, int NR, int G>
__global__ void __launch_bounds__(kTinyWarps * 32, tiny_min_blocks<T, NR, G>()) k_s_tiny_fwd(
    const Front* __restrict__ fronts, const Item* __restrict__ items, int64_t cnt, const int32_t* __restrict__ reltgt,
    const int32_t* __restrict__ chdtgt, const T* __restrict__ P, T* __restrict__ C, T* __restrict__ R, int64_t n,
    int nrhs) {
    pdl_prologue();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    constexpr unsigned kAll = 0xffffffffu;
    const int g = threadIdx.x & (G - 1), slot = threadIdx.x / G;
    const Front f = tiny_front(fronts, items, (int64_t)blockIdx.x * tiny_fronts<G>() + slot, cnt);
    T* Wv = reinterpret_cast<T*>(sm_raw) + slot * G * NR;  // Wv[row * NR + r]
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp;
    const T* Pj = P + f.poff;
    T lr[G];  // row g of the panel
#pragma unroll
    for (int k = 0; k < G; ++k) lr[k] = (g < nj && k < nn) ? Pj[g + (int64_t)k * ld] : T(0);
#pragma unroll
    for (int r = 0; r < NR; ++r) Wv[g * NR + r] = (g < nn && r < nrhs) ? C[f.col0 + g + (int64_t)r * n] : T(0);
    __syncwarp();
    // child updates, children in reverse order (one addition per entry and
    // child); lane g fetches child g's record up front (children past G
    // are read in the loop)
    const int nch = f.chd1 - f.chd0;
    const int nchw = tiny_warp_max<G>(nch);
    int kna = 0, ksep = 0;
    int64_t kroff = 0;
    if (g < nch) {
        const Front fc = fronts[chdtgt[f.chd1 - 1 - g]];
        kna = fc.na, ksep = fc.sep0, kroff = fc.roff;
    }
    for (int i = 0; i < nchw; ++i) {
        const int src = (threadIdx.x & ~(G - 1) & 31) + (i & (G - 1));
        int ma = __shfl_sync(kAll, kna, src);
        int sep0 = __shfl_sync(kAll, ksep, src);
        int64_t roff = __shfl_sync(kAll, kroff, src);
        if (i < nch) {
            if (i >= G) {
                const Front fc = fronts[chdtgt[f.chd1 - 1 - i]];
                ma = fc.na, sep0 = fc.sep0, roff = fc.roff;
            }
            if (g < ma) {
                const int q = reltgt[sep0 + g];
                const T* Mc = R + roff * nrhs + g;
#pragma unroll
                for (int r = 0; r < NR; ++r)
                    if (r < nrhs) Wv[q * NR + r] += Mc[r * ma];
            }
        }
        __syncwarp();
    }
    T x[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) x[r] = Wv[g * NR + r];
    const int nnw = tiny_warp_max<G>(nn);
    // forward substitution: x_k = w_k / L_kk, rows k < a < nn lose L_ak x_k
#pragma unroll
    for (int k = 0; k < G; ++k) {
        if (k >= nnw) break;  // uniform across the warp
        const T dk = __shfl_sync(kAll, lr[k], k, G);
        const T dinv = UNIT ? T(1) : T(1) / dk;
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const T xk = __shfl_sync(kAll, x[r], k, G) * dinv;
            if (k < nn) {
                if (g > k && g < nn) x[r] -= lr[k] * xk;
                if (g == k) x[r] = xk;
            }
        }
    }
    if (g < nn)
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) C[f.col0 + g + (int64_t)r * n] = x[r];
    // R_j = (child sums) - L21 x
    T acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = T(0);
#pragma unroll
    for (int k = 0; k < G; ++k) {
        if (k >= nnw) break;
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const T xk = __shfl_sync(kAll, x[r], k, G);
            if (k < nn) acc[r] += lr[k] * xk;
        }
    }
    if (g >= nn && g < nj) {
        T* Rj = R + f.roff * nrhs + (g - nn);
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) Rj[(int64_t)r * na] = x[r] - acc[r];
    }
}

template <typename T, int UNIT, int NR, int G>
__global__ void __launch_bounds__(kTinyWarps * 32, tiny_min_blocks<T, NR, G>()) k_s_tiny_bwd(
    const Front* __restrict__ fronts, const Item* __restrict__ items, int64_t cnt, const int32_t* __restrict__ septgt,
    const T* __restrict__ P, T* __restrict__ C, int64_t n, int nrhs) {
    pdl_prologue();
    constexpr unsigned kAll = 0xffffffffu;
    const int g = threadIdx.x & (G - 1), slot = threadIdx.x / G;
    const Front f = tiny_front(fronts, items, (int64_t)blockIdx.x * tiny_fronts<G>() + slot, cnt);
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp;
    const T* Pj = P + f.poff;
    T cv[G];  // column g of the panel
#pragma unroll
    for (int i = 0; i < G; ++i) cv[i] = (g < nn && i < nj) ? Pj[i + (int64_t)g * ld] : T(0);
    T xs[NR];  // lanes nn .. nj - 1: x of the separator rows
    {
        const bool v = g >= nn && g < nj;
        const int64_t row = v ? septgt[f.sep0 + g - nn] : 0;
#pragma unroll
        for (int r = 0; r < NR; ++r) xs[r] = (v && r < nrhs) ? __ldcg(C + row + (int64_t)r * n) : T(0);
    }
    // C1 - L21^T x[sep], separator rows in order
    T acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = T(0);
    const int njw = tiny_warp_max<G>(nj);
#pragma unroll
    for (int i = 0; i < G; ++i) {
        if (i >= njw) break;  // uniform across the warp
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const T xb = __shfl_sync(kAll, xs[r], i, G);
            if (i >= nn && i < nj) acc[r] += cv[i] * xb;
        }
    }
    T c[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) c[r] = (g < nn && r < nrhs) ? C[f.col0 + g + (int64_t)r * n] - acc[r] : T(0);
    // back substitution on L^T: x_k = c_k / L_kk, k descending; columns
    // j < k lose L_kj x_k
    const int nnw = tiny_warp_max<G>(nn);
#pragma unroll
    for (int k = G - 1; k >= 0; --k) {
        if (k >= nnw) continue;  // uniform across the warp
        const T dk = __shfl_sync(kAll, cv[k], k, G);
        const T dinv = UNIT ? T(1) : T(1) / dk;
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            const T xk = __shfl_sync(kAll, c[r], k, G) * dinv;
            if (k < nn) {
                if (g < k) c[r] -= cv[k] * xk;
                if (g == k) c[r] = xk;
            }
        }
    }
    if (g < nn)
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) C[f.col0 + g + (int64_t)r * n] = c[r];
}

// ---------------------------------------------------------------------------
// Subtrees of small fronts in ONE launch per direction: CTA b takes task
// items[task0 + b] = {first level item, end}; each level item {first front
// item, end} lists the task's fronts of one tree height.  The CTA's warps
// take the fronts of a height one per warp (the per-front code of
// k_s_small_fwd / _bwd) and a block barrier separates the heights, ascending
// forward (children before parents) and descending backward.  Tasks are
// disjoint subtrees, so CTAs never wait on one another; what would be one
// launch per tree level for these fronts is one launch in all.
// ---------------------------------------------------------------------------
constexpr int kSubWarps = 8;

template <typename T, int NR>
constexpr int sub_solve_smem() { return kSubWarps * kSmallMax * NR * (int)sizeof(T); }

template <typename T, int UNIT, int NR>
__global__ void __launch_bounds__(kSubWarps * 32, small_min_blocks<T, NR>() / 2) k_s_sub_fwd(const Front* __restrict__ fronts,
                                                              const Item* __restrict__ items, int64_t task0,
                                                              const int32_t* __restrict__ reltgt,
                                                              const int32_t* __restrict__ chdtgt,
                                                              const T* __restrict__ P, T* __restrict__ C,
                                                              T* __restrict__ R, int64_t n, int nrhs) {
    pdl_prologue();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    T* C1 = reinterpret_cast<T*>(sm_raw) + wib * kSmallMax * NR;
    const Item tk = items[task0 + blockIdx.x];
    for (int L = tk.front; L < tk.a; ++L) {
        const Item lv = items[L];
        for (int i = lv.front + wib; i < lv.a; i += kSubWarps) {
            const Front f = fronts[items[i].front];
            small_fwd_front<T, UNIT, NR>(f, fronts, reltgt, chdtgt, P, C, R, n, nrhs, C1, lane);
        }
        __syncthreads();
    }
}

template <typename T, int UNIT, int NR>
__global__ void __launch_bounds__(kSubWarps * 32, small_min_blocks<T, NR>() / 2) k_s_sub_bwd(const Front* __restrict__ fronts,
                                                              const Item* __restrict__ items, int64_t task0,
                                                              const int32_t* __restrict__ septgt,
                                                              const T* __restrict__ P, T* __restrict__ C,
                                                              int64_t n, int nrhs) {
    pdl_prologue();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const Item tk = items[task0 + blockIdx.x];
    for (int L = tk.a - 1; L >= tk.front; --L) {
        const Item lv = items[L];
        for (int i = lv.front + wib; i < lv.a; i += kSubWarps) {
            const Front f = fronts[items[i].front];
            small_bwd_front<T, UNIT, NR>(f, septgt, P, C, n, nrhs, lane);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// blocked fronts
// ---------------------------------------------------------------------------
// forward gather: W[res] = C[res] + child updates, R_j = child updates.
// One thread per (row, right-hand side) of the item's 256-row tile adds the
// row's own list of child contributions (h_grow / h_gcon, children in the
// reference's order), so no two threads touch one entry and the tile needs
// no barrier
template <typename T>
__device__ __forceinline__ void gather_run(const Item& it, const Front* __restrict__ fronts,
                                           const int64_t* __restrict__ grow, const GCon* __restrict__ gcon,
                                           const T* __restrict__ C, T* W, T* R, int64_t n, int nrhs) {
    const Front f = fronts[it.front];
    const int nn = f.nn, na = f.na, nj = nn + na;
    const int p0 = it.a * kSolveRows, p1 = min(p0 + kSolveRows, nj);
    const int w = p1 - p0;
    const int64_t* rp = grow + it.b;
    T* Rj = R + f.roff * nrhs;
    for (int i = threadIdx.x; i < w * nrhs; i += blockDim.x) {
        const int q = p0 + i % w, r = i / w;
        T v = q < nn ? C[f.col0 + q + (int64_t)r * n] : T(0);
        const int64_t e1 = rp[q + 1];
        for (int64_t e = rp[q]; e < e1; ++e) {
            const GCon g = gcon[e];
            v += R[g.roff * nrhs + g.a + (int64_t)r * g.ma];
        }
        if (q < nn) W[f.col0 + q + (int64_t)r * n] = v;
        else Rj[(q - nn) + (int64_t)r * na] = v;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_s_gather(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                  const int64_t* __restrict__ grow,
                                                  const GCon* __restrict__ gcon, const T* __restrict__ C,
                                                  T* __restrict__ W, T* __restrict__ R, int64_t n, int nrhs) {
    pdl_prologue();
    gather_run<T>(items[blockIdx.x], fronts, grow, gcon, C, W, R, n, nrhs);
}

// ---------------------------------------------------------------------------
// blocked diagonal solves in steps of a 256-column super-block K (columns
// k0 .. k0 + wK of a front), with the super-block inverse X_K stored by the
// factorization.  Per step and level:
//   forward : k_s_sdiag<.., 0>  x_K = X_K W_K    (kDiagSplit CTAs per front), then
//             k_s_ftile  rows below: W / R -= L[rows, K] x_K (64-row tiles);
//   backward: k_s_sdiag<.., 1>  x_K = X_K^T W_K  (kDiagSplit CTAs per front), then
//             k_s_btile  columns left: W[c] -= sum_i L[k0 + i, c] x_K[i] (64-column tiles).
// ---------------------------------------------------------------------------
template <typename T, int NR>
constexpr int sdiag_smem() { return (kSolveNB * NR + 16 * kSolveNB) * (int)sizeof(T); }

// element copy global -> shared that stays in flight (cp.async); a false
// `valid` writes zero and reads nothing
template <typename T>
__device__ __forceinline__ void cpa(T* dst, const T* src, bool valid) {
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
    const int nb = valid ? (int)sizeof(T) : 0;
    if (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(saddr), "l"(src), "r"(nb) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(saddr), "l"(src), "r"(nb) : "memory");
}
// 16 bytes global -> shared in flight (cp.async.cg); a false `valid` writes
// zeros and reads nothing; both addresses 16-byte aligned
__device__ __forceinline__ void cpa16(void* dst, const void* src, bool valid) {
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(saddr), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cpa_wait_all() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// x_K = X_K b_K (BWD = 0) or X_K^T b_K (BWD = 1), spread over kDiagSplit
// CTAs per front so that the 256 x 256 inverse streams through many SMs:
// CTA q owns outputs a in [16 q, 16 q + 16); its 16 rows (forward) or 16
// columns (backward) of X are staged in shared memory with every load in
// flight at once, then thread t takes output 16 q + t / 16 and every 16th
// input starting at t % 16, and half-warp shuffles add the partial sums.
constexpr int kDiagSplit = kSolveNB / 16;

// W and C go through L2 only (ld/st .cg): within one k_s_chain launch other
// CTAs write them, and L1 is not coherent across SMs.
// Each step function issues the loads that depend on nothing computed in
// this solve (the panel, the inverse) first, then calls wait() -- a no-op in
// the per-step kernels, the chain's bounded waits in k_s_chain; a false
// return (a timed-out wait, uniform across the CTA) skips the rest.
struct NoWait {
    __device__ bool operator()() const { return true; }
};
// the per-step kernels: wait for the previous grid of the stream (launched
// for programmatic dependence; a no-op otherwise)
struct PdlWait {
    __device__ bool operator()() const {
        asm volatile("griddepcontrol.wait;" ::: "memory");
        return true;
    }
};

template <typename T, int NR, int BWD, typename Wait = NoWait>
__device__ __forceinline__ void sdiag_run(const Front& f, int step, int q, const T* __restrict__ inv2, T* C,
                                          const T* W, int64_t n, int nrhs, unsigned char* sm_raw,
                                          Wait wait = Wait()) {
    T* b = reinterpret_cast<T*>(sm_raw);  // [r][c] : b[c + r * kSolveNB]
    T* xt = b + kSolveNB * NR;            // forward: xt[c * 16 + a - 16q]; backward: xt[(a - 16q) * 256 + c]
    const int k0 = step * kSolveNB, wK = min(kSolveNB, f.nn - k0), ld2 = super_ld(wK);
    if (16 * q >= wK) {  // whole CTA: nothing to compute, the wait still taken
        wait();
        return;
    }
    const T* X = inv2 + f.i2off + (int64_t)step * kSolveNB * kSolveNB;
    // 16-byte copies (X's columns and ld2 are multiples of 4 elements, so
    // every copy is aligned and stays inside the ld2 x wK block); entries
    // outside the triangle the products read come along and are never used
    constexpr int VWX = 16 / (int)sizeof(T);
    if (!BWD) {
        constexpr int G = 16 / VWX;  // copies per column: the CTA's 16 rows
        for (int e = threadIdx.x; e < G * kSolveNB; e += blockDim.x) {
            const int c = e / G, g = e % G, a0 = 16 * q + g * VWX;
            const bool v = c < wK && a0 < ld2;
            cpa16(xt + c * 16 + g * VWX, v ? X + a0 + (int64_t)c * ld2 : X, v);
        }
    } else {
        constexpr int G = kSolveNB / VWX;  // copies per staged column of X
        for (int e = threadIdx.x; e < 16 * G; e += blockDim.x) {
            const int al = e / G, c0 = (e % G) * VWX, a = 16 * q + al;
            const bool v = a < wK && c0 < ld2;
            cpa16(xt + al * kSolveNB + c0, v ? X + c0 + (int64_t)a * ld2 : X, v);
        }
    }
    if (!wait()) {
        cpa_wait_all();
        return;
    }
    for (int i = threadIdx.x; i < kSolveNB * NR; i += blockDim.x) {
        const int c = i % kSolveNB, r = i / kSolveNB;
        b[i] = (c < wK && r < nrhs) ? __ldcg(W + f.col0 + k0 + c + (int64_t)r * n) : T(0);
    }
    cpa_wait_all();
    __syncthreads();
    const int al = threadIdx.x >> 4, a = 16 * q + al, cl = threadIdx.x & 15;
    T acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = T(0);
    if (a < wK) {
        const int cb = BWD ? a : 0, ce = BWD ? wK : a + 1;
#pragma unroll 4
        for (int c = cb + cl; c < ce; c += 16) {
            const T x = BWD ? xt[al * kSolveNB + c] : xt[c * 16 + al];
#pragma unroll
            for (int r = 0; r < NR; ++r) acc[r] += x * b[c + r * kSolveNB];
        }
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        T v = acc[r];
        for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        acc[r] = v;
    }
    if (cl == 0 && a < wK)
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) __stcg(C + f.col0 + k0 + a + (int64_t)r * n, acc[r]);
}

template <typename T, int NR, int BWD>
__global__ void __launch_bounds__(256) k_s_sdiag(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                 int step, const T* __restrict__ inv2, T* __restrict__ C,
                                                 const T* __restrict__ W, int64_t n, int nrhs) {
    pdl_trigger();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const Front f = fronts[items[blockIdx.x / kDiagSplit].front];
    sdiag_run<T, NR, BWD>(f, step, (int)(blockIdx.x % kDiagSplit), inv2, C, W, n, nrhs, sm_raw, PdlWait());
}

constexpr int kColBatch = 16;  // 16-byte panel loads a lane issues before using them (step tiles: few CTAs)
constexpr int kColBatchL = 8;  // the same for the L21 products (many CTAs: occupancy hides the latency)

// 16 bytes of consecutive panel entries in one load: 4 floats or 2 doubles
template <typename T> struct Vec16;
template <> struct Vec16<float> {
    using type = float4;
    static constexpr int W = 4;
    __device__ static float at(const float4& v, int e) { return e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w; }
};
template <> struct Vec16<double> {
    using type = double2;
    static constexpr int W = 2;
    __device__ static double at(const double2& v, int e) { return e == 0 ? v.x : v.y; }
};

// forward rows below super-block K inside the diagonal block: W -= L[rows, K] x_K
// (the L21 rows are done once per level by k_s_fwd_l).
// Work item a covers the 64 rows from (k0 + wK rounded down to 4) + 64 a;
// rows of the block itself that fall in the first tile are computed and
// dropped.  Warp w streams columns 32 w .. 32 w + 31 of the block straight
// from the panel: a lane loads 16 bytes (4 float or 2 double rows) of a
// column, 64 / VW lanes cover the tile's rows and the warp takes VW / 2
// columns per load (coalesced runs of 256 / 512 bytes); x_K comes from
// shared memory as a broadcast.  Partial sums are added lane half by lane
// half, then warp by warp, in a fixed order.
template <typename T, int NR>
constexpr int ftile_smem() { return (kSolveNB * NR + 8 * NR * kFwdRows) * (int)sizeof(T); }

template <typename T, int NR, typename Wait = NoWait>
__device__ __forceinline__ void ftile_run(const Front& f, int step, int ta, const T* __restrict__ P, const T* C,
                                          T* W, int64_t n, int nrhs, unsigned char* sm_raw, Wait wait = Wait()) {
    using VT = Vec16<T>;
    using V = typename VT::type;
    constexpr int VW = VT::W;             // rows per load
    constexpr int LPC = kFwdRows / VW;    // lanes per column (16 float, 32 double)
    constexpr int CPL = 32 / LPC;         // columns per warp load (2 float, 1 double)
    T* xs = reinterpret_cast<T*>(sm_raw);  // xs[c * NR + r]
    T* red = xs + kSolveNB * NR;           // red[(w * NR + r) * kFwdRows + row]
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp;
    const int k0 = step * kSolveNB, wK = min(kSolveNB, nn - k0);
    const int rlo = k0 + wK;
    const int ra = (rlo & ~3) + ta * kFwdRows;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int rr = (lane % LPC) * VW, ch = lane / LPC;
    // row is a multiple of 4 below nj, so the 16-byte load ends inside the
    // column's ldp (a multiple of 4) rows
    const int row = ra + rr;
    const int cb = warp * 32;
    const int cn = min(32, wK - cb);
    const bool act = row < nj && cn > 0;
    const T* pc = P + f.poff + (int64_t)(k0 + cb) * ld + row;
    // the first batch of panel loads (all of a lane's for FP32) before x_K
    V lb[kColBatch];
    if (act)
#pragma unroll
        for (int u = 0; u < kColBatch; ++u) {
            const int c = ch + u * CPL;
            if (c < cn) lb[u] = *reinterpret_cast<const V*>(pc + (int64_t)c * ld);
        }
    if (!wait()) return;
    for (int i = tid; i < kSolveNB * NR; i += 256) {
        const int c = i & (kSolveNB - 1), r = i / kSolveNB;
        xs[c * NR + r] = (c < wK && r < nrhs) ? __ldcg(C + f.col0 + k0 + c + (int64_t)r * n) : T(0);
    }
    __syncthreads();
    T acc[VW][NR];
#pragma unroll
    for (int e = 0; e < VW; ++e)
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[e][r] = T(0);
    if (act) {
        // all of a batch's loads are issued before its products (one
        // memory round trip per 16 columns of a lane, in column order)
        for (int cb0 = ch; cb0 < cn; cb0 += kColBatch * CPL) {
            if (cb0 != ch)
#pragma unroll
                for (int u = 0; u < kColBatch; ++u) {
                    const int c = cb0 + u * CPL;
                    if (c < cn) lb[u] = *reinterpret_cast<const V*>(pc + (int64_t)c * ld);
                }
#pragma unroll
            for (int u = 0; u < kColBatch; ++u) {
                const int c = cb0 + u * CPL;
                if (c < cn) {
                    const T* xc = xs + (cb + c) * NR;
#pragma unroll
                    for (int r = 0; r < NR; ++r) {
                        const T x = xc[r];
#pragma unroll
                        for (int e = 0; e < VW; ++e) acc[e][r] += VT::at(lb[u], e) * x;
                    }
                }
            }
        }
    }
    if (CPL == 2) {
#pragma unroll
        for (int e = 0; e < VW; ++e)
#pragma unroll
            for (int r = 0; r < NR; ++r) acc[e][r] += __shfl_xor_sync(0xffffffffu, acc[e][r], 16);
    }
    if (ch == 0) {
#pragma unroll
        for (int r = 0; r < NR; ++r)
#pragma unroll
            for (int e = 0; e < VW; ++e) red[(warp * NR + r) * kFwdRows + rr + e] = acc[e][r];
    }
    __syncthreads();
    for (int o = tid; o < kFwdRows * NR; o += 256) {
        const int rl = o & (kFwdRows - 1), r = o / kFwdRows;
        const int q = ra + rl;
        if (r < nrhs && q >= rlo && q < nj) {
            T v = T(0);
#pragma unroll
            for (int w = 0; w < 8; ++w) v += red[(w * NR + r) * kFwdRows + rl];
            if (q < nn) {
                T* wp = W + f.col0 + q + (int64_t)r * n;
                __stcg(wp, __ldcg(wp) - v);
            }
        }
    }
}

template <typename T, int NR>
__global__ void __launch_bounds__(256) k_s_ftile(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                 int step, const T* __restrict__ P, const T* __restrict__ C,
                                                 T* __restrict__ W, int64_t n, int nrhs) {
    pdl_trigger();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    ftile_run<T, NR>(f, step, it.a, P, C, W, n, nrhs, sm_raw, PdlWait());
}

// forward R_j -= L21 x1 for the blocked fronts of a level, once all their
// diagonal-block steps are done (x1 = C over the front's columns).  Item
// (front, 64-row tile t of L21 from the 4-aligned row at or before nn,
// 512-column chunk q, slot): warp w streams columns 64 w .. 64 w + 63 of the
// chunk with 16-byte loads as in k_s_ftile, x1 is a shared-memory broadcast,
// and the chunk's sums for the tile's rows go to part[slot]; k_s_fwd_red adds
// the chunks of a tile in order.  This takes the L21 product (most of the
// forward data of a large front) out of the sequential step chain.
template <typename T, int NR>
constexpr int fwdl_smem() { return (kFwdCols * NR + 8 * NR * kFwdRows) * (int)sizeof(T); }

template <typename T, int NR>
__global__ void __launch_bounds__(256) k_s_fwd_l(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                 const T* __restrict__ P, const T* __restrict__ C,
                                                 T* __restrict__ part, int64_t n, int nrhs) {
    pdl_prologue();
    using VT = Vec16<T>;
    using V = typename VT::type;
    constexpr int VW = VT::W;             // rows per load
    constexpr int LPC = kFwdRows / VW;    // lanes per column (16 float, 32 double)
    constexpr int CPL = 32 / LPC;         // columns per warp load (2 float, 1 double)
    extern __shared__ __align__(16) unsigned char sm_raw[];
    T* xs = reinterpret_cast<T*>(sm_raw);  // xs[c * NR + r], c relative to the chunk
    T* red = xs + kFwdCols * NR;           // red[(w * NR + r) * kFwdRows + row]
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, nj = nn + f.na, ld = f.ldp;
    const int cq = it.b * kFwdCols, wq = min(kFwdCols, nn - cq);
    const int ra = (nn & ~3) + it.a * kFwdRows;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < kFwdCols * NR; i += 256) {
        const int c = i % kFwdCols, r = i / kFwdCols;
        xs[c * NR + r] = (c < wq && r < nrhs) ? C[f.col0 + cq + c + (int64_t)r * n] : T(0);
    }
    __syncthreads();
    const int rr = (lane % LPC) * VW, ch = lane / LPC;
    // row is a multiple of 4 below nj, so the 16-byte load ends inside the
    // column's ldp (a multiple of 4) rows
    const int row = ra + rr;
    const int cb = warp * (kFwdCols / 8);
    const int cn = min(kFwdCols / 8, wq - cb);
    T acc[VW][NR];
#pragma unroll
    for (int e = 0; e < VW; ++e)
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[e][r] = T(0);
    if (row < nj && cn > 0) {
        const T* pc = P + f.poff + (int64_t)(cq + cb) * ld + row;
        // all of a batch's loads are issued before its products (one
        // memory round trip per 16 columns of a lane, in column order)
        for (int cb0 = ch; cb0 < cn; cb0 += kColBatchL * CPL) {
            V lb[kColBatchL];
#pragma unroll
            for (int u = 0; u < kColBatchL; ++u) {
                const int c = cb0 + u * CPL;
                if (c < cn) lb[u] = *reinterpret_cast<const V*>(pc + (int64_t)c * ld);
            }
#pragma unroll
            for (int u = 0; u < kColBatchL; ++u) {
                const int c = cb0 + u * CPL;
                if (c < cn) {
                    const T* xc = xs + (cb + c) * NR;
#pragma unroll
                    for (int r = 0; r < NR; ++r) {
                        const T x = xc[r];
#pragma unroll
                        for (int e = 0; e < VW; ++e) acc[e][r] += VT::at(lb[u], e) * x;
                    }
                }
            }
        }
    }
    if (CPL == 2) {
#pragma unroll
        for (int e = 0; e < VW; ++e)
#pragma unroll
            for (int r = 0; r < NR; ++r) acc[e][r] += __shfl_xor_sync(0xffffffffu, acc[e][r], 16);
    }
    if (ch == 0) {
#pragma unroll
        for (int r = 0; r < NR; ++r)
#pragma unroll
            for (int e = 0; e < VW; ++e) red[(warp * NR + r) * kFwdRows + rr + e] = acc[e][r];
    }
    __syncthreads();
    T* dst = part + (int64_t)it.pad * (kFwdRows * kMaxRhs);
    for (int o = tid; o < kFwdRows * kMaxRhs; o += 256) {
        const int rl = o % kFwdRows, r = o / kFwdRows;
        T v = T(0);
        if (r < NR)
#pragma unroll
            for (int w = 0; w < 8; ++w) v += red[(w * NR + r) * kFwdRows + rl];
        dst[o] = v;
    }
}

// R_j[rows of tile t] -= the chunk sums of k_s_fwd_l, chunks in order.
template <typename T>
__global__ void __launch_bounds__(256) k_s_fwd_red(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                   const T* __restrict__ part, T* __restrict__ R, int nrhs) {
    pdl_prologue();
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, na = f.na;
    const int ra = (nn & ~3) + it.a * kFwdRows;
    T* Rj = R + f.roff * nrhs;
    for (int o = threadIdx.x; o < kFwdRows * kMaxRhs; o += blockDim.x) {
        const int rl = o % kFwdRows, r = o / kFwdRows;
        const int q = ra + rl;
        if (r >= nrhs || q < nn || q >= nn + na) continue;
        T s = T(0);
        for (int c = 0; c < it.pad; ++c) s += part[(int64_t)(it.b + c) * (kFwdRows * kMaxRhs) + o];
        Rj[(q - nn) + r * na] -= s;
    }
}

// backward columns left of super-block K (64-column tile it.a):
// W[c] -= sum_i L[k0 + i, c] x_K[i].  Thread (q, c) owns column c over the
// block rows 64 q .. 64 q + 63, loading 16 bytes (4 float or 2 double rows)
// at a time, eight loads in flight; the lanes of a warp sit on the same
// rows, so x_K is a shared-memory broadcast.  The four row quarters are
// added in order.
template <typename T, int NR>
constexpr int btile_smem() { return (kSolveNB * NR + 4 * NR * kNB) * (int)sizeof(T); }

template <typename T, int NR, typename Wait = NoWait>
__device__ __forceinline__ void btile_run(const Front& f, int step, int ta, const T* __restrict__ P, const T* C,
                                          T* W, int64_t n, int nrhs, unsigned char* sm_raw, Wait wait = Wait()) {
    using VT = Vec16<T>;
    using V = typename VT::type;
    constexpr int VW = VT::W;
    T* xs = reinterpret_cast<T*>(sm_raw);  // xs[i * NR + r]
    T* red = xs + kSolveNB * NR;           // red[(q * NR + r) * kNB + c]
    const int nn = f.nn, ld = f.ldp;
    const int k0 = step * kSolveNB, wK = min(kSolveNB, nn - k0);
    const int c0 = ta * kNB, wc = min(kNB, k0 - c0);
    const int tid = threadIdx.x;
    const int c = tid & (kNB - 1), q = tid >> 6;
    const int i0 = q * 64, ni = min(64, wK - i0);  // rows of this quarter inside the block
    const bool act = c < wc && ni > 0;
    // k0 + i0 + i is a multiple of 4 below nn <= nj, so each 16-byte load
    // ends inside the column's ldp rows; rows past the block are dropped by
    // the select below.  The first batch (all of a thread's for FP32) is
    // issued before x_K.
    const T* pc = P + f.poff + (int64_t)(c0 + c) * ld + k0 + i0;
    V l[kColBatch];
    if (act)
#pragma unroll
        for (int u = 0; u < kColBatch; ++u)
            if (u * VW < ni) l[u] = *reinterpret_cast<const V*>(pc + u * VW);
    if (!wait()) return;
    for (int i = tid; i < kSolveNB * NR; i += 256) {
        const int a = i & (kSolveNB - 1), r = i / kSolveNB;
        xs[a * NR + r] = (a < wK && r < nrhs) ? __ldcg(C + f.col0 + k0 + a + (int64_t)r * n) : T(0);
    }
    __syncthreads();
    T acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = T(0);
    if (act) {
        for (int i = 0; i < 64; i += kColBatch * VW) {
            if (i != 0)
#pragma unroll
                for (int u = 0; u < kColBatch; ++u)
                    if (i + u * VW < ni) l[u] = *reinterpret_cast<const V*>(pc + i + u * VW);
#pragma unroll
            for (int u = 0; u < kColBatch; ++u) {
                const int ib = i + u * VW;
                if (ib < ni) {
                    const T* xr = xs + (i0 + ib) * NR;
#pragma unroll
                    for (int e = 0; e < VW; ++e) {
                        const T lv = ib + e < ni ? VT::at(l[u], e) : T(0);
#pragma unroll
                        for (int r = 0; r < NR; ++r) acc[r] += lv * xr[e * NR + r];
                    }
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) red[(q * NR + r) * kNB + c] = acc[r];
    __syncthreads();
    for (int o = tid; o < kNB * NR; o += 256) {
        const int cc = o & (kNB - 1), r = o / kNB;
        if (cc < wc && r < nrhs) {
            const T v = red[(0 * NR + r) * kNB + cc] + red[(1 * NR + r) * kNB + cc] +
                        red[(2 * NR + r) * kNB + cc] + red[(3 * NR + r) * kNB + cc];
            T* wp = W + f.col0 + c0 + cc + (int64_t)r * n;
            __stcg(wp, __ldcg(wp) - v);
        }
    }
}

template <typename T, int NR>
__global__ void __launch_bounds__(256) k_s_btile(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                 int step, const T* __restrict__ P, const T* __restrict__ C,
                                                 T* __restrict__ W, int64_t n, int nrhs) {
    pdl_trigger();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    btile_run<T, NR>(f, step, it.a, P, C, W, n, nrhs, sm_raw, PdlWait());
}

// ---------------------------------------------------------------------------
// The super-block chain of a level's blocked fronts in ONE launch per
// direction (instead of two launches per step).  The plan lists the items
// in ticket order: per step K (ascending forward, descending backward) the
// kDiagSplit diagonal parts of every front (it.a = -1 - q), then the tiles
// (it.a = tile), those the next diagonal step waits for first.  CTAs take
// items in that order from a ticket counter.  Each front has a counter
// block in `ctl` at it.pad: [0] finished diagonal parts, [1 + g] steps
// applied to 64-row (forward) / 64-column (backward) tile g of its diagonal
// block.  A diagonal part of step K waits until the tiles of super-block K
// hold every earlier step; a tile item waits for x_K (all diagonal parts of
// step K) and for its tile's earlier steps.  Every wait is for items with
// smaller tickets, which running CTAs already hold, so each wait ends.  Each
// wait is still bounded (kChainWaitNs of %globaltimer): a timeout sets *err,
// after which every wait gives up at once and the items left do nothing.
// The arithmetic of each item is k_s_sdiag's / k_s_ftile's / k_s_btile's in
// the same order, so results equal the per-step launches bit for bit.
// ---------------------------------------------------------------------------
constexpr unsigned long long kChainWaitNs = 2000000000ull;

// the poll is a relaxed load (an acquire load would also drop the SM's L1
// lines on every poll, slowing the working CTAs beside it); the caller's
// fence after a successful wait orders the data reads that follow
__device__ __forceinline__ int ld_relaxed_gpu(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long chain_clock() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// bounded wait (one thread) until *p >= need; false on timeout or once *err is set
__device__ bool chain_wait(const int* p, int need, int* err) {
    if (ld_relaxed_gpu(p) >= need) return true;
    const unsigned long long t0 = chain_clock();
    unsigned ns = 32;
    for (;;) {
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
        if (ld_relaxed_gpu(p) >= need) return true;
        if (*reinterpret_cast<volatile int*>(err)) return false;
        if (chain_clock() - t0 > kChainWaitNs) {
            atomicExch(err, 2);
            return false;
        }
    }
}

template <typename T, int NR, int BWD>
constexpr int chain_smem() {
    return sdiag_smem<T, NR>() > (BWD ? btile_smem<T, NR>() : ftile_smem<T, NR>())
               ? sdiag_smem<T, NR>()
               : (BWD ? btile_smem<T, NR>() : ftile_smem<T, NR>());
}

template <typename T, int NR, int BWD>
__global__ void __launch_bounds__(256) k_s_chain(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                 int64_t cnt, int* ticket, int* ctl, const T* __restrict__ inv2,
                                                 const T* __restrict__ P, T* C, T* W, int64_t n, int nrhs,
                                                 int* err) {
    pdl_prologue();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    __shared__ int s_t, s_ok;
    for (;;) {
        __syncthreads();  // the previous item is finished by every thread
        if (threadIdx.x == 0) {
            s_t = atomicAdd(ticket, 1);
            s_ok = 1;
        }
        __syncthreads();
        const int64_t t = s_t;
        if (t >= cnt) return;
        const Item it = items[t];
        const Front f = fronts[it.front];
        const int S = (f.nn + kSolveNB - 1) / kSolveNB, K = it.b;
        const int done = BWD ? S - 1 - K : K;  // steps applied before step K
        int* xdone = ctl + it.pad;
        int* tiles = xdone + 1;
        // the waits run inside the step functions, after the loads of the
        // panel or the inverse (which depend on nothing in this solve)
        if (it.a < 0) {
            const int g0 = K * (kSolveNB / kNB);
            const int ng = min(kSolveNB / kNB, (f.nn - K * kSolveNB + kNB - 1) / kNB);
            auto wait = [&]() -> bool {
                if (threadIdx.x < ng) {
                    if (!chain_wait(tiles + g0 + threadIdx.x, done, err)) s_ok = 0;
                    __threadfence();
                }
                __syncthreads();
                return s_ok != 0;
            };
            sdiag_run<T, NR, BWD>(f, K, -1 - it.a, inv2, C, W, n, nrhs, sm_raw, wait);
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0 && s_ok) atomicAdd(xdone, 1);
        } else {
            const int g = BWD ? it.a : ((K + 1) * kSolveNB) / kNB + it.a;
            auto wait = [&]() -> bool {
                if (threadIdx.x == 0) {
                    if (!chain_wait(xdone, kDiagSplit * (done + 1), err) || !chain_wait(tiles + g, done, err))
                        s_ok = 0;
                    __threadfence();
                }
                __syncthreads();
                return s_ok != 0;
            };
            if (BWD) btile_run<T, NR>(f, K, it.a, P, C, W, n, nrhs, sm_raw, wait);
            else ftile_run<T, NR>(f, K, it.a, P, C, W, n, nrhs, sm_raw, wait);
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0 && s_ok) atomicAdd(tiles + g, 1);
        }
    }
}

// backward: W[res tile] = C[res tile] - L21^T x[sep].  Items are (front,
// 64-column tile, chunk of kBwdRows rows of L21); each writes its partial
// sums to part[item.pad] and k_s_bwd_red adds the chunks of a tile in a
// fixed order.  The chunk's x[sep] rows are gathered into shared memory
// once; thread (q, c) then owns column c over a quarter of the chunk's rows
// and streams them from the panel 16 bytes at a time (the rows are taken
// from the 4-aligned row at or before the chunk start; rows outside the
// chunk are dropped by a select), with x as a shared-memory broadcast.  The
// four quarters are added in order.
constexpr int kBwdAlignRows = kBwdRows + 16;  // staged rows: the chunk, its alignment lead-in, quarters of 4k rows

template <typename T, int NR>
constexpr int bwd_smem() { return (kBwdAlignRows * NR + 4 * NR * kNB) * (int)sizeof(T); }

// one work item (front f, 64-column tile it.a, row chunk it.b, slot it.pad);
// BATCH 16-byte loads of a thread are in flight at once (the order of the
// products does not depend on it)
template <typename T, int NR, int BATCH>
__device__ __forceinline__ void bwdl_run(const Front& f, const Item& it, const int32_t* __restrict__ septgt,
                                         const T* __restrict__ P, const T* __restrict__ C, T* part, int64_t n,
                                         int nrhs, unsigned char* sm_raw) {
    using VT = Vec16<T>;
    using V = typename VT::type;
    constexpr int VW = VT::W;
    T* xs = reinterpret_cast<T*>(sm_raw);  // xs[i * NR + r], i = panel row - row0
    T* red = xs + kBwdAlignRows * NR;      // red[(q * NR + r) * kNB + c]
    const int nn = f.nn, na = f.na, ld = f.ldp;
    const int tid = threadIdx.x;
    const int32_t* sep = septgt + f.sep0;
    const int c0 = it.a * kNB, wc = min(kNB, nn - c0);
    const int a_beg = it.b * kBwdRows, a_end = min(na, a_beg + kBwdRows);
    const int rlo = nn + a_beg, rhi = nn + a_end;  // panel rows of the chunk
    const int row0 = rlo & ~3;                     // 4-aligned start of the staged rows
    const int nrow = rhi - row0;                   // <= kBwdAlignRows
    for (int i = tid; i < kBwdAlignRows * NR; i += 256) {
        const int a = i % kBwdAlignRows, r = i / kBwdAlignRows;
        const int row = row0 + a;
        xs[a * NR + r] = (row >= rlo && row < rhi && r < nrhs) ? C[sep[row - nn] + (int64_t)r * n] : T(0);
    }
    __syncthreads();
    const int c = tid & (kNB - 1), q = tid >> 6;
    constexpr int QR = kBwdAlignRows / 4;      // rows per quarter (a multiple of 4)
    const int i0 = q * QR, ni = min(QR, nrow - i0);
    T acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = T(0);
    if (c < wc && ni > 0) {
        // row0 + i0 + i is a multiple of 4 below rhi <= nj, so each 16-byte
        // load ends inside the column's ldp rows
        const T* pc = P + f.poff + (int64_t)(c0 + c) * ld + row0 + i0;
        for (int i = 0; i < QR; i += BATCH * VW) {
            V l[BATCH];
#pragma unroll
            for (int u = 0; u < BATCH; ++u)
                if (i + u * VW < ni) l[u] = *reinterpret_cast<const V*>(pc + i + u * VW);
#pragma unroll
            for (int u = 0; u < BATCH; ++u) {
                const int ib = i + u * VW;
                if (ib < ni) {
                    const T* xr = xs + (i0 + ib) * NR;
#pragma unroll
                    for (int e = 0; e < VW; ++e) {
                        // rows before the chunk hold finite factor entries and meet
                        // x = 0; rows past it (up to ldp) are dropped here
                        const T lv = ib + e < ni ? VT::at(l[u], e) : T(0);
#pragma unroll
                        for (int r = 0; r < NR; ++r) acc[r] += lv * xr[e * NR + r];
                    }
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) red[(q * NR + r) * kNB + c] = acc[r];
    __syncthreads();
    T* dst = part + (int64_t)it.pad * (kNB * kMaxRhs);
    for (int o = tid; o < kNB * kMaxRhs; o += 256) {
        const int cc = o % kNB, r = o / kNB;
        T v = T(0);
        if (r < NR)
            v = red[(0 * NR + r) * kNB + cc] + red[(1 * NR + r) * kNB + cc] + red[(2 * NR + r) * kNB + cc] +
                red[(3 * NR + r) * kNB + cc];
        dst[o] = v;
    }
}

template <typename T, int NR>
__global__ void __launch_bounds__(256) k_s_bwd_l(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                 const int32_t* __restrict__ septgt, const T* __restrict__ P,
                                                 const T* __restrict__ C, T* __restrict__ part, int64_t n,
                                                 int nrhs) {
    pdl_prologue();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    bwdl_run<T, NR, kColBatchL>(f, it, septgt, P, C, part, n, nrhs, sm_raw);
}

// W[tile it.a of the front's columns] = C - (the chunk sums at part[it.b ...],
// chunks in order); part is read through L2 (in k_s_mid_bwd other CTAs of
// the cluster wrote it)
template <typename T>
__device__ __forceinline__ void bwdred_run(const Front& f, const Item& it, const T* part, const T* __restrict__ C,
                                           T* W, int64_t n, int nrhs) {
    const int c0 = it.a * kNB, wc = min(kNB, f.nn - c0);
    const int nchunk = (f.na + kBwdRows - 1) / kBwdRows;
    for (int o = threadIdx.x; o < kNB * kMaxRhs; o += blockDim.x) {
        const int c = o % kNB, r = o / kNB;
        if (c >= wc || r >= nrhs) continue;
        T s = T(0);
        for (int q = 0; q < nchunk; ++q) s += __ldcg(part + (int64_t)(it.b + q) * (kNB * kMaxRhs) + o);
        const int64_t idx = f.col0 + c0 + c + (int64_t)r * n;
        W[idx] = C[idx] - s;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_s_bwd_red(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                   const T* __restrict__ part, const T* __restrict__ C,
                                                   T* __restrict__ W, int64_t n, int nrhs) {
    pdl_prologue();
    const Item it = items[blockIdx.x];
    bwdred_run<T>(fronts[it.front], it, part, C, W, n, nrhs);
}

// ---------------------------------------------------------------------------
// Levels whose blocked fronts are single super-blocks (nn <= kSolveNB) with
// a short L21: one thread-block cluster of kMidCluster CTAs per front does
// the level's whole forward (or backward) work in one launch, instead of
// the four (three) dependent launches above.  Phases are separated by the
// cluster's hardware barrier (every CTA of a cluster is resident at once, so
// the barrier needs no bounded wait); data crossing CTAs goes through L2
// (stores, a gpu-scope fence before the barrier, .cg loads after it).
//   forward : gather tiles -> x = X W[res] (the 16 parts of k_s_sdiag) ->
//             R_j -= L21 x, one warp per 64-row tile of L21;
//   backward: L21^T x[sep] partial sums (k_s_bwd_l items) -> W = C - sums
//             (k_s_bwd_red) -> x = X^T W (the 16 parts of k_s_sdiag).
// Every entry gets the same operations in the same order as in the
// per-kernel launches, so the results are bitwise equal to them.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mid_cluster_sync() {
    __threadfence();
    asm volatile("barrier.cluster.arrive.release.aligned;\n"
                 "barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

template <typename T, int NR>
constexpr int midf_smem() {
    return sdiag_smem<T, NR>() > (kSolveNB * NR + 8 * NR * kFwdRows) * (int)sizeof(T)
               ? sdiag_smem<T, NR>()
               : (kSolveNB * NR + 8 * NR * kFwdRows) * (int)sizeof(T);
}
template <typename T, int NR>
constexpr int midb_smem() { return sdiag_smem<T, NR>() > bwd_smem<T, NR>() ? sdiag_smem<T, NR>() : bwd_smem<T, NR>(); }

// R_j[rows of 64-row L21 tile t] -= L21 x1 with one warp (nn <= kSolveNB):
// for each 64-column group g the warp does what warp g of k_s_fwd_l does for
// the tile (same lanes, same column order), and the group sums are added in
// group order in the warp's slice of shared memory, as k_s_fwd_l adds its
// warps' sums; the single chunk's sum is then taken from R as k_s_fwd_red does
template <typename T, int NR>
__device__ __forceinline__ void midf_tile(const Front& f, int t, const T* __restrict__ P, const T* xs, T* tot,
                                          T* R, int nrhs) {
    using VT = Vec16<T>;
    using V = typename VT::type;
    constexpr int VW = VT::W;
    constexpr int LPC = kFwdRows / VW;
    constexpr int CPL = 32 / LPC;
    constexpr int GC = kFwdCols / 8;  // columns per group: one warp's share in k_s_fwd_l
    const int lane = threadIdx.x & 31;
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp;
    const int ra = (nn & ~3) + t * kFwdRows;
    const int rr = (lane % LPC) * VW, ch = lane / LPC;
    const int row = ra + rr;
    const int ng = (nn + GC - 1) / GC;
    for (int g = 0; g < ng; ++g) {
        const int cb = g * GC, cn = min(GC, nn - cb);
        T acc[VW][NR];
#pragma unroll
        for (int e = 0; e < VW; ++e)
#pragma unroll
            for (int r = 0; r < NR; ++r) acc[e][r] = T(0);
        if (row < nj) {
            const T* pc = P + f.poff + (int64_t)cb * ld + row;
            for (int cb0 = ch; cb0 < cn; cb0 += kColBatch * CPL) {
                V lb[kColBatch];
#pragma unroll
                for (int u = 0; u < kColBatch; ++u) {
                    const int c = cb0 + u * CPL;
                    if (c < cn) lb[u] = *reinterpret_cast<const V*>(pc + (int64_t)c * ld);
                }
#pragma unroll
                for (int u = 0; u < kColBatch; ++u) {
                    const int c = cb0 + u * CPL;
                    if (c < cn) {
                        const T* xc = xs + (cb + c) * NR;
#pragma unroll
                        for (int r = 0; r < NR; ++r) {
                            const T x = xc[r];
#pragma unroll
                            for (int e = 0; e < VW; ++e) acc[e][r] += VT::at(lb[u], e) * x;
                        }
                    }
                }
            }
        }
        if (CPL == 2) {
#pragma unroll
            for (int e = 0; e < VW; ++e)
#pragma unroll
                for (int r = 0; r < NR; ++r) acc[e][r] += __shfl_xor_sync(0xffffffffu, acc[e][r], 16);
        }
        if (ch == 0) {
#pragma unroll
            for (int r = 0; r < NR; ++r)
#pragma unroll
                for (int e = 0; e < VW; ++e) {
                    T* tp = tot + r * kFwdRows + rr + e;
                    *tp = (g == 0 ? T(0) : *tp) + acc[e][r];
                }
        }
    }
    __syncwarp();
    T* Rj = R + f.roff * nrhs;
    for (int o = lane; o < kFwdRows * NR; o += 32) {
        const int rl = o % kFwdRows, r = o / kFwdRows;
        const int q = ra + rl;
        if (r < nrhs && q >= nn && q < nj) {
            T* rp = Rj + (q - nn) + (int64_t)r * na;
            *rp = __ldcg(rp) - (T(0) + tot[r * kFwdRows + rl]);
        }
    }
    __syncwarp();
}

// item (front, first gather item, first backward partial slot, gather tiles)
template <typename T, int NR>
__global__ void __cluster_dims__(kMidCluster, 1, 1) __launch_bounds__(256)
    k_s_mid_fwd(const Front* __restrict__ fronts, const Item* __restrict__ mid, const Item* __restrict__ all_items,
                const int64_t* __restrict__ grow, const GCon* __restrict__ gcon, const T* __restrict__ inv2,
                const T* __restrict__ P, T* C, T* W, T* R, int64_t n, int nrhs) {
    pdl_prologue();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const Item m = mid[blockIdx.x / kMidCluster];
    const int rank = (int)(blockIdx.x % kMidCluster);
    const Front f = fronts[m.front];
    for (int t = rank; t < m.pad; t += kMidCluster) gather_run<T>(all_items[m.a + t], fronts, grow, gcon, C, W, R, n, nrhs);
    mid_cluster_sync();
    for (int q = rank; q < kDiagSplit; q += kMidCluster) {
        sdiag_run<T, NR, 0>(f, 0, q, inv2, C, W, n, nrhs, sm_raw);
        __syncthreads();
    }
    mid_cluster_sync();
    if (f.na > 0) {
        T* xs = reinterpret_cast<T*>(sm_raw);  // xs[c * NR + r]
        T* tot = xs + kSolveNB * NR;           // per warp: tot[r * kFwdRows + row]
        for (int i = threadIdx.x; i < kSolveNB * NR; i += blockDim.x) {
            const int c = i % kSolveNB, r = i / kSolveNB;
            xs[c * NR + r] = (c < f.nn && r < nrhs) ? __ldcg(C + f.col0 + c + (int64_t)r * n) : T(0);
        }
        __syncthreads();
        const int warp = threadIdx.x >> 5;
        const int ntile = (f.nn + f.na - (f.nn & ~3) + kFwdRows - 1) / kFwdRows;
        for (int t = rank * 8 + warp; t < ntile; t += kMidCluster * 8)
            midf_tile<T, NR>(f, t, P, xs, tot + warp * NR * kFwdRows, R, nrhs);
    }
}

template <typename T, int NR>
__global__ void __cluster_dims__(kMidCluster, 1, 1) __launch_bounds__(256)
    k_s_mid_bwd(const Front* __restrict__ fronts, const Item* __restrict__ mid, const int32_t* __restrict__ septgt,
                const T* __restrict__ inv2, const T* __restrict__ P, T* C, T* W, T* part, int64_t n, int nrhs) {
    pdl_prologue();
    extern __shared__ __align__(16) unsigned char sm_raw[];
    const Item m = mid[blockIdx.x / kMidCluster];
    const int rank = (int)(blockIdx.x % kMidCluster);
    const Front f = fronts[m.front];
    const int nct = (f.nn + kNB - 1) / kNB;
    const int nchunk = max(1, (f.na + kBwdRows - 1) / kBwdRows);
    for (int u = rank; u < nct * nchunk; u += kMidCluster) {
        bwdl_run<T, NR, kColBatch>(f, Item{m.front, u / nchunk, u % nchunk, m.b + u}, septgt, P, C, part, n, nrhs,
                                   sm_raw);
        __syncthreads();
    }
    mid_cluster_sync();
    for (int t = rank; t < nct; t += kMidCluster) bwdred_run<T>(f, Item{m.front, t, m.b + t * nchunk, 0}, part, C, W, n, nrhs);
    mid_cluster_sync();
    for (int q = rank; q < kDiagSplit; q += kMidCluster) {
        sdiag_run<T, NR, 1>(f, 0, q, inv2, C, W, n, nrhs, sm_raw);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static unsigned grid_stride_blocks(int64_t work) {
    int64_t b = (work + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    if (b < 1) b = 1;
    return (unsigned)b;
}

int launch_permute_in(mf_handle* h, const double* B, int64_t ldb, const int64_t* perm, int64_t nrhs) {
    Timer t(h, K_PERM);
    launch_k(k_perm<true>, grid_stride_blocks(h->n * nrhs), 256, 0, h->stream, h->d_C, const_cast<double*>(B), perm, h->n,
                                                                         ldb, (int)nrhs);
    MF_CUDA(cudaGetLastError());
    return 0;
}

int launch_permute_out(mf_handle* h, double* B, int64_t ldb, const int64_t* perm, int64_t nrhs) {
    Timer t(h, K_PERM);
    launch_k(k_perm<false>, grid_stride_blocks(h->n * nrhs), 256, 0, h->stream, h->d_C, B, perm, h->n, ldb, (int)nrhs);
    MF_CUDA(cudaGetLastError());
    return 0;
}

int launch_permute_to(mf_handle* h, const double* B, int64_t ldb, const int64_t* perm, int64_t nrhs, double* dst) {
    Timer t(h, K_PERM);
    launch_k(k_perm<true>, grid_stride_blocks(h->n * nrhs), 256, 0, h->stream, dst, const_cast<double*>(B), perm, h->n, ldb,
                                                                         (int)nrhs);
    MF_CUDA(cudaGetLastError());
    return 0;
}

int launch_permute_from(mf_handle* h, double* B, int64_t ldb, const int64_t* perm, int64_t nrhs, const double* src) {
    Timer t(h, K_PERM);
    launch_k(k_perm<false>, grid_stride_blocks(h->n * nrhs), 256, 0, h->stream, const_cast<double*>(src), B, perm, h->n,
                                                                          ldb, (int)nrhs);
    MF_CUDA(cudaGetLastError());
    return 0;
}

// one k_s_chain launch: a persistent grid of at most (resident CTAs per SM)
// x SMs, fewer when the level has fewer items
template <typename T, int NR, int BWD>
static int chain_go(mf_handle* h, const Level& lv, const SolveBufs<T>& sb, int nrhs) {
    const ItemList& il = BWD ? lv.s_chain_b : lv.s_chain_f;
    constexpr int sm = chain_smem<T, NR, BWD>();
    MF_CUDA(cudaFuncSetAttribute(k_s_chain<T, NR, BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    int occ = 0;
    MF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_s_chain<T, NR, BWD>, 256, sm));
    const int64_t grid = std::min<int64_t>(il.cnt, (int64_t)std::max(occ, 1) * std::max(h->num_sms, 1));
    launch_k(k_s_chain<T, NR, BWD>, (unsigned)grid, 256, sm, h->stream, h->d_fronts, h->d_items + il.off, il.cnt,
                                                                  h->d_chain + lv.chain_tk + BWD, h->d_chain,
                                                                  sb.inv2, sb.P, sb.C, sb.W, h->n, nrhs, h->d_err);
    MF_CUDA(cudaGetLastError());
    return 0;
}

template <typename T, int BWD>
static int launch_chain(mf_handle* h, const Level& lv, const SolveBufs<T>& sb, int nrb, int nrhs) {
    switch (nrb) {
        case 1: return chain_go<T, 1, BWD>(h, lv, sb, nrhs);
        case 2: return chain_go<T, 2, BWD>(h, lv, sb, nrhs);
        case 4: return chain_go<T, 4, BWD>(h, lv, sb, nrhs);
        case 8: return chain_go<T, 8, BWD>(h, lv, sb, nrhs);
        default: return chain_go<T, 16, BWD>(h, lv, sb, nrhs);
    }
}

// one cluster launch for the blocked fronts of a single-super-block level
template <typename T, int NR, int BWD>
static int mid_go(mf_handle* h, const Level& lv, const SolveBufs<T>& sb, int nrhs) {
    const unsigned g = (unsigned)(lv.s_mid.cnt * kMidCluster);
    const Item* it = h->d_items + lv.s_mid.off;
    if (!BWD) {
        MF_CUDA(cudaFuncSetAttribute(k_s_mid_fwd<T, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, midf_smem<T, NR>()));
        launch_k(k_s_mid_fwd<T, NR>, g, 256, midf_smem<T, NR>(), h->stream, h->d_fronts, it, h->d_items, h->d_grow,
                 h->d_gcon, sb.inv2, sb.P, sb.C, sb.W, sb.R, h->n, nrhs);
    } else {
        MF_CUDA(cudaFuncSetAttribute(k_s_mid_bwd<T, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, midb_smem<T, NR>()));
        launch_k(k_s_mid_bwd<T, NR>, g, 256, midb_smem<T, NR>(), h->stream, h->d_fronts, it, h->d_septgt, sb.inv2,
                 sb.P, sb.C, sb.W, sb.part, h->n, nrhs);
    }
    MF_CUDA(cudaGetLastError());
    return 0;
}

template <typename T, int BWD>
static int launch_mid(mf_handle* h, const Level& lv, const SolveBufs<T>& sb, int nrb, int nrhs) {
    switch (nrb) {
        case 1: return mid_go<T, 1, BWD>(h, lv, sb, nrhs);
        case 2: return mid_go<T, 2, BWD>(h, lv, sb, nrhs);
        case 4: return mid_go<T, 4, BWD>(h, lv, sb, nrhs);
        case 8: return mid_go<T, 8, BWD>(h, lv, sb, nrhs);
        default: return mid_go<T, 16, BWD>(h, lv, sb, nrhs);
    }
}

// the tiny fronts of a level: k_s_tiny_* (16 lanes per front), or the
// warp-per-front k_s_small_* when switched off
template <typename T, int UNIT, int NR, int BWD, int G>
static int tiny_go(mf_handle* h, const ItemList& il, const SolveBufs<T>& sb, int nrhs) {
    const Item* it = h->d_items + il.off;
    const int64_t c = il.cnt;
    if (h->tiny_solve) {
        const unsigned g = (unsigned)((c + tiny_fronts<G>() - 1) / tiny_fronts<G>());
        constexpr int sm = tiny_fronts<G>() * G * NR * (int)sizeof(T);
        if (!BWD)
            launch_k(k_s_tiny_fwd<T, UNIT, NR, G>, g, kTinyWarps * 32, sm, h->stream, h->d_fronts, it, c,
                     h->d_reltgt, h->d_chdtgt, sb.P, sb.C, sb.R, h->n, nrhs);
        else
            launch_k(k_s_tiny_bwd<T, UNIT, NR, G>, g, kTinyWarps * 32, 0, h->stream, h->d_fronts, it, c,
                     h->d_septgt, sb.P, sb.C, h->n, nrhs);
    } else {
        const unsigned g = (unsigned)((c + kSmallWarps - 1) / kSmallWarps);
        if (!BWD)
            launch_k(k_s_small_fwd<T, UNIT, NR>, g, kSmallWarps * 32, small_solve_smem<T, NR>(), h->stream,
                     h->d_fronts, it, c, h->d_reltgt, h->d_chdtgt, sb.P, sb.C, sb.R, h->n, nrhs);
        else
            launch_k(k_s_small_bwd<T, UNIT, NR>, g, kSmallWarps * 32, 0, h->stream, h->d_fronts, it, c, h->d_septgt,
                     sb.P, sb.C, h->n, nrhs);
    }
    MF_CUDA(cudaGetLastError());
    return 0;
}

template <typename T, int UNIT, int BWD, int G>
static int launch_tiny(mf_handle* h, const ItemList& il, const SolveBufs<T>& sb, int nrb, int nrhs) {
    Timer t(h, K_S_SMALL);
    switch (nrb) {
        case 1: return tiny_go<T, UNIT, 1, BWD, G>(h, il, sb, nrhs);
        case 2: return tiny_go<T, UNIT, 2, BWD, G>(h, il, sb, nrhs);
        case 4: return tiny_go<T, UNIT, 4, BWD, G>(h, il, sb, nrhs);
        case 8: return tiny_go<T, UNIT, 8, BWD, G>(h, il, sb, nrhs);
        default: return tiny_go<T, UNIT, 16, BWD, G>(h, il, sb, nrhs);
    }
}

template <typename T, int UNIT>
static int solve_impl(mf_handle* h, const SolveBufs<T>& sb, int nrhs) {
    if (h->profile) {
        h->times.launches[K_SOLVE_PASS] += 1;
        h->times.launches[K_SOLVE_RHS] += nrhs;
    }
    MF_CUDA(cudaFuncSetAttribute(k_s_ftile<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, ftile_smem<T, 16>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_ftile<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, ftile_smem<T, 8>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_ftile<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, ftile_smem<T, 4>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_ftile<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, ftile_smem<T, 2>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_ftile<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, ftile_smem<T, 1>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_btile<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, btile_smem<T, 16>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_btile<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, btile_smem<T, 8>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_sdiag<T, 16, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, sdiag_smem<T, 16>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_sdiag<T, 16, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sdiag_smem<T, 16>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_sdiag<T, 8, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, sdiag_smem<T, 8>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_sdiag<T, 8, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sdiag_smem<T, 8>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_bwd_l<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, bwd_smem<T, 16>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_fwd_l<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, fwdl_smem<T, 16>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_fwd_l<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, fwdl_smem<T, 8>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_fwd_l<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, fwdl_smem<T, 4>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_bwd_l<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bwd_smem<T, 8>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_bwd_l<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bwd_smem<T, 4>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_small_fwd<T, UNIT, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 small_solve_smem<T, 16>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_sub_fwd<T, UNIT, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 sub_solve_smem<T, 16>()));
    MF_CUDA(cudaFuncSetAttribute(k_s_sub_fwd<T, UNIT, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 sub_solve_smem<T, 8>()));
    const int nrb = nrhs <= 1 ? 1 : nrhs <= 2 ? 2 : nrhs <= 4 ? 4 : nrhs <= 8 ? 8 : 16;
    const Item* items = h->d_items;
    const int64_t n = h->n;
    // the chain kernel for a level: every level (MF_SOLVE_CHAIN=1), none
    // (=0), or by default the levels of at least kChainMinSteps super-block
    // steps, where overlapping the steps' tiles outweighs the waits
    auto use_chain = [&](const Level& lv) {
        if (h->nchain <= 0 || h->solve_chain == 0) return false;
        return h->solve_chain == 1 || (int)lv.s_steps.size() >= kChainMinSteps;
    };
    bool any_chain = false;
    for (const Level& lv : h->levels) any_chain = any_chain || use_chain(lv);
    if (any_chain) MF_CUDA(cudaMemsetAsync(h->d_chain, 0, sizeof(int) * (size_t)h->nchain, h->stream));
    if (h->sub_tasks.cnt) {
        // the subtrees of small fronts, forward, in one launch
        Timer t(h, K_S_SMALL);
        const unsigned g = (unsigned)h->sub_tasks.cnt;
        const int64_t t0 = h->sub_tasks.off;
        switch (nrb) {
            case 1: launch_k(k_s_sub_fwd<T, UNIT, 1>, g, kSubWarps * 32, sub_solve_smem<T, 1>(), h->stream, 
                        h->d_fronts, items, t0, h->d_reltgt, h->d_chdtgt, sb.P, sb.C, sb.R, n, nrhs); break;
            case 2: launch_k(k_s_sub_fwd<T, UNIT, 2>, g, kSubWarps * 32, sub_solve_smem<T, 2>(), h->stream, 
                        h->d_fronts, items, t0, h->d_reltgt, h->d_chdtgt, sb.P, sb.C, sb.R, n, nrhs); break;
            case 4: launch_k(k_s_sub_fwd<T, UNIT, 4>, g, kSubWarps * 32, sub_solve_smem<T, 4>(), h->stream, 
                        h->d_fronts, items, t0, h->d_reltgt, h->d_chdtgt, sb.P, sb.C, sb.R, n, nrhs); break;
            case 8: launch_k(k_s_sub_fwd<T, UNIT, 8>, g, kSubWarps * 32, sub_solve_smem<T, 8>(), h->stream, 
                        h->d_fronts, items, t0, h->d_reltgt, h->d_chdtgt, sb.P, sb.C, sb.R, n, nrhs); break;
            default: launch_k(k_s_sub_fwd<T, UNIT, 16>, g, kSubWarps * 32, sub_solve_smem<T, 16>(), h->stream, 
                        h->d_fronts, items, t0, h->d_reltgt, h->d_chdtgt, sb.P, sb.C, sb.R, n, nrhs); break;
        }
        MF_CUDA(cudaGetLastError());
    }
    // forward: levels ascending
    for (const Level& lv : h->levels) {
        if (lv.s_tiny.cnt)
            if (int rc = launch_tiny<T, UNIT, 0, kTinyNJ>(h, lv.s_tiny, sb, nrb, nrhs)) return rc;
        if (lv.s_tiny2.cnt)
            if (int rc = launch_tiny<T, UNIT, 0, kTinyNJ2>(h, lv.s_tiny2, sb, nrb, nrhs)) return rc;
        if (lv.s_small.cnt) {
            Timer t(h, K_S_SMALL);
            const unsigned g = (unsigned)((lv.s_small.cnt + kSmallWarps - 1) / kSmallWarps);
            const Item* it = items + lv.s_small.off;
            const int64_t c = lv.s_small.cnt;
            switch (nrb) {
                case 1: launch_k(k_s_small_fwd<T, UNIT, 1>, g, kSmallWarps * 32, small_solve_smem<T, 1>(), h->stream, 
                            h->d_fronts, it, c, h->d_reltgt, h->d_chdtgt, sb.P, sb.C, sb.R, n, nrhs); break;
                case 2: launch_k(k_s_small_fwd<T, UNIT, 2>, g, kSmallWarps * 32, small_solve_smem<T, 2>(), h->stream, 
                            h->d_fronts, it, c, h->d_reltgt, h->d_chdtgt, sb.P, sb.C, sb.R, n, nrhs); break;
                case 4: launch_k(k_s_small_fwd<T, UNIT, 4>, g, kSmallWarps * 32, small_solve_smem<T, 4>(), h->stream, 
                            h->d_fronts, it, c, h->d_reltgt, h->d_chdtgt, sb.P, sb.C, sb.R, n, nrhs); break;
                case 8: launch_k(k_s_small_fwd<T, UNIT, 8>, g, kSmallWarps * 32, small_solve_smem<T, 8>(), h->stream, 
                            h->d_fronts, it, c, h->d_reltgt, h->d_chdtgt, sb.P, sb.C, sb.R, n, nrhs); break;
                default: launch_k(k_s_small_fwd<T, UNIT, 16>, g, kSmallWarps * 32, small_solve_smem<T, 16>(), h->stream, 
                            h->d_fronts, it, c, h->d_reltgt, h->d_chdtgt, sb.P, sb.C, sb.R, n, nrhs); break;
            }
            MF_CUDA(cudaGetLastError());
        }
        const bool mid = h->mid_solve && lv.s_mid.cnt;
        if (mid) {
            Timer t(h, K_S_FWD);
            if (int rc = launch_mid<T, 0>(h, lv, sb, nrb, nrhs)) return rc;
            continue;
        }
        if (lv.s_gather.cnt) {
            Timer t(h, K_S_GATHER);
            launch_k(k_s_gather<T>, (unsigned)lv.s_gather.cnt, 256, 0, h->stream, 
                h->d_fronts, items + lv.s_gather.off, h->d_grow, h->d_gcon, sb.C, sb.W, sb.R, n, nrhs);
            MF_CUDA(cudaGetLastError());
        }
        const bool chain = use_chain(lv);
        if (chain && lv.s_chain_f.cnt) {
            Timer t(h, K_S_FWD);
            if (int rc = launch_chain<T, 0>(h, lv, sb, nrb, nrhs)) return rc;
        }
        for (size_t k = 0; !chain && k < lv.s_steps.size(); ++k) {
            const SolveStep& st = lv.s_steps[k];
            if (!st.diag.cnt) continue;
            Timer t(h, K_S_FWD);
            const unsigned gd = (unsigned)st.diag.cnt;
            const Item* itd = items + st.diag.off;
            switch (nrb) {
                case 1: launch_kx(h->step_pdl, k_s_sdiag<T, 1, 0>, gd * kDiagSplit, 256, sdiag_smem<T, 1>(), h->stream, h->d_fronts, itd, (int)k, sb.inv2, sb.C, sb.W, n, nrhs); break;
                case 2: launch_kx(h->step_pdl, k_s_sdiag<T, 2, 0>, gd * kDiagSplit, 256, sdiag_smem<T, 2>(), h->stream, h->d_fronts, itd, (int)k, sb.inv2, sb.C, sb.W, n, nrhs); break;
                case 4: launch_kx(h->step_pdl, k_s_sdiag<T, 4, 0>, gd * kDiagSplit, 256, sdiag_smem<T, 4>(), h->stream, h->d_fronts, itd, (int)k, sb.inv2, sb.C, sb.W, n, nrhs); break;
                case 8: launch_kx(h->step_pdl, k_s_sdiag<T, 8, 0>, gd * kDiagSplit, 256, sdiag_smem<T, 8>(), h->stream, h->d_fronts, itd, (int)k, sb.inv2, sb.C, sb.W, n, nrhs); break;
                default: launch_kx(h->step_pdl, k_s_sdiag<T, 16, 0>, gd * kDiagSplit, 256, sdiag_smem<T, 16>(), h->stream, h->d_fronts, itd, (int)k, sb.inv2, sb.C, sb.W, n, nrhs); break;
            }
            MF_CUDA(cudaGetLastError());
            if (st.fwd.cnt) {
                const unsigned gf = (unsigned)st.fwd.cnt;
                const Item* itf = items + st.fwd.off;
                switch (nrb) {
                    case 1: launch_kx(h->step_pdl, k_s_ftile<T, 1>, gf, 256, ftile_smem<T, 1>(), h->stream, h->d_fronts, itf, (int)k, sb.P, sb.C, sb.W, n, nrhs); break;
                    case 2: launch_kx(h->step_pdl, k_s_ftile<T, 2>, gf, 256, ftile_smem<T, 2>(), h->stream, h->d_fronts, itf, (int)k, sb.P, sb.C, sb.W, n, nrhs); break;
                    case 4: launch_kx(h->step_pdl, k_s_ftile<T, 4>, gf, 256, ftile_smem<T, 4>(), h->stream, h->d_fronts, itf, (int)k, sb.P, sb.C, sb.W, n, nrhs); break;
                    case 8: launch_kx(h->step_pdl, k_s_ftile<T, 8>, gf, 256, ftile_smem<T, 8>(), h->stream, h->d_fronts, itf, (int)k, sb.P, sb.C, sb.W, n, nrhs); break;
                    default: launch_kx(h->step_pdl, k_s_ftile<T, 16>, gf, 256, ftile_smem<T, 16>(), h->stream, h->d_fronts, itf, (int)k, sb.P, sb.C, sb.W, n, nrhs); break;
                }
                MF_CUDA(cudaGetLastError());
            }
        }
        if (lv.s_fwd_l.cnt) {
            Timer t(h, K_S_FWD);
            const unsigned gl = (unsigned)lv.s_fwd_l.cnt;
            const Item* itl = items + lv.s_fwd_l.off;
            switch (nrb) {
                case 1: launch_k(k_s_fwd_l<T, 1>, gl, 256, fwdl_smem<T, 1>(), h->stream, h->d_fronts, itl, sb.P, sb.C, sb.part, n, nrhs); break;
                case 2: launch_k(k_s_fwd_l<T, 2>, gl, 256, fwdl_smem<T, 2>(), h->stream, h->d_fronts, itl, sb.P, sb.C, sb.part, n, nrhs); break;
                case 4: launch_k(k_s_fwd_l<T, 4>, gl, 256, fwdl_smem<T, 4>(), h->stream, h->d_fronts, itl, sb.P, sb.C, sb.part, n, nrhs); break;
                case 8: launch_k(k_s_fwd_l<T, 8>, gl, 256, fwdl_smem<T, 8>(), h->stream, h->d_fronts, itl, sb.P, sb.C, sb.part, n, nrhs); break;
                default: launch_k(k_s_fwd_l<T, 16>, gl, 256, fwdl_smem<T, 16>(), h->stream, h->d_fronts, itl, sb.P, sb.C, sb.part, n, nrhs); break;
            }
            MF_CUDA(cudaGetLastError());
            launch_k(k_s_fwd_red<T>, (unsigned)lv.s_fwd_red.cnt, 256, 0, h->stream, h->d_fronts, items + lv.s_fwd_red.off,
                                                                              sb.part, sb.R, nrhs);
            MF_CUDA(cudaGetLastError());
        }
    }
    if (UNIT) {
        Timer t(h, K_OTHER);
        launch_k(k_diag_div<T>, grid_stride_blocks(n * nrhs), 256, 0, h->stream, sb.C, sb.d, n, nrhs);
        MF_CUDA(cudaGetLastError());
    }
    // backward: levels descending
    for (size_t L = h->levels.size(); L-- > 0;) {
        const Level& lv = h->levels[L];
        const bool mid = h->mid_solve && lv.s_mid.cnt;
        if (mid) {
            Timer t(h, K_S_BWD);
            if (int rc = launch_mid<T, 1>(h, lv, sb, nrb, nrhs)) return rc;
        }
        if (!mid && lv.s_bwd_l.cnt) {
            Timer t(h, K_S_BWD_L);
            const unsigned gl = (unsigned)lv.s_bwd_l.cnt;
            const Item* itl = items + lv.s_bwd_l.off;
            switch (nrb) {
                case 1: launch_k(k_s_bwd_l<T, 1>, gl, 256, bwd_smem<T, 1>(), h->stream, h->d_fronts, itl, h->d_septgt, sb.P, sb.C, sb.part, n, nrhs); break;
                case 2: launch_k(k_s_bwd_l<T, 2>, gl, 256, bwd_smem<T, 2>(), h->stream, h->d_fronts, itl, h->d_septgt, sb.P, sb.C, sb.part, n, nrhs); break;
                case 4: launch_k(k_s_bwd_l<T, 4>, gl, 256, bwd_smem<T, 4>(), h->stream, h->d_fronts, itl, h->d_septgt, sb.P, sb.C, sb.part, n, nrhs); break;
                case 8: launch_k(k_s_bwd_l<T, 8>, gl, 256, bwd_smem<T, 8>(), h->stream, h->d_fronts, itl, h->d_septgt, sb.P, sb.C, sb.part, n, nrhs); break;
                default: launch_k(k_s_bwd_l<T, 16>, gl, 256, bwd_smem<T, 16>(), h->stream, h->d_fronts, itl, h->d_septgt, sb.P, sb.C, sb.part, n, nrhs); break;
            }
            MF_CUDA(cudaGetLastError());
            launch_k(k_s_bwd_red<T>, (unsigned)lv.s_bwd_red.cnt, 256, 0, h->stream, h->d_fronts, items + lv.s_bwd_red.off,
                                                                              sb.part, sb.C, sb.W, n, nrhs);
            MF_CUDA(cudaGetLastError());
        }
        const bool chain = use_chain(lv);
        if (!mid && chain && lv.s_chain_b.cnt) {
            Timer t(h, K_S_BWD);
            if (int rc = launch_chain<T, 1>(h, lv, sb, nrb, nrhs)) return rc;
        }
        for (size_t k = lv.s_steps.size(); !mid && !chain && k-- > 0;) {
            const SolveStep& st = lv.s_steps[k];
            if (!st.diag.cnt) continue;
            Timer t(h, K_S_BWD);
            const unsigned gd = (unsigned)st.diag.cnt;
            const Item* itd = items + st.diag.off;
            switch (nrb) {
                case 1: launch_kx(h->step_pdl, k_s_sdiag<T, 1, 1>, gd * kDiagSplit, 256, sdiag_smem<T, 1>(), h->stream, h->d_fronts, itd, (int)k, sb.inv2, sb.C, sb.W, n, nrhs); break;
                case 2: launch_kx(h->step_pdl, k_s_sdiag<T, 2, 1>, gd * kDiagSplit, 256, sdiag_smem<T, 2>(), h->stream, h->d_fronts, itd, (int)k, sb.inv2, sb.C, sb.W, n, nrhs); break;
                case 4: launch_kx(h->step_pdl, k_s_sdiag<T, 4, 1>, gd * kDiagSplit, 256, sdiag_smem<T, 4>(), h->stream, h->d_fronts, itd, (int)k, sb.inv2, sb.C, sb.W, n, nrhs); break;
                case 8: launch_kx(h->step_pdl, k_s_sdiag<T, 8, 1>, gd * kDiagSplit, 256, sdiag_smem<T, 8>(), h->stream, h->d_fronts, itd, (int)k, sb.inv2, sb.C, sb.W, n, nrhs); break;
                default: launch_kx(h->step_pdl, k_s_sdiag<T, 16, 1>, gd * kDiagSplit, 256, sdiag_smem<T, 16>(), h->stream, h->d_fronts, itd, (int)k, sb.inv2, sb.C, sb.W, n, nrhs); break;
            }
            MF_CUDA(cudaGetLastError());
            if (st.bwd.cnt) {
                const unsigned gb = (unsigned)st.bwd.cnt;
                const Item* itb = items + st.bwd.off;
                switch (nrb) {
                    case 1: launch_kx(h->step_pdl, k_s_btile<T, 1>, gb, 256, btile_smem<T, 1>(), h->stream, h->d_fronts, itb, (int)k, sb.P, sb.C, sb.W, n, nrhs); break;
                    case 2: launch_kx(h->step_pdl, k_s_btile<T, 2>, gb, 256, btile_smem<T, 2>(), h->stream, h->d_fronts, itb, (int)k, sb.P, sb.C, sb.W, n, nrhs); break;
                    case 4: launch_kx(h->step_pdl, k_s_btile<T, 4>, gb, 256, btile_smem<T, 4>(), h->stream, h->d_fronts, itb, (int)k, sb.P, sb.C, sb.W, n, nrhs); break;
                    case 8: launch_kx(h->step_pdl, k_s_btile<T, 8>, gb, 256, btile_smem<T, 8>(), h->stream, h->d_fronts, itb, (int)k, sb.P, sb.C, sb.W, n, nrhs); break;
                    default: launch_kx(h->step_pdl, k_s_btile<T, 16>, gb, 256, btile_smem<T, 16>(), h->stream, h->d_fronts, itb, (int)k, sb.P, sb.C, sb.W, n, nrhs); break;
                }
                MF_CUDA(cudaGetLastError());
            }
        }
        if (lv.s_small.cnt) {
            Timer t(h, K_S_SMALL);
            const unsigned g = (unsigned)((lv.s_small.cnt + kSmallWarps - 1) / kSmallWarps);
            const Item* it = items + lv.s_small.off;
            const int64_t c = lv.s_small.cnt;
            switch (nrb) {
                case 1: launch_k(k_s_small_bwd<T, UNIT, 1>, g, kSmallWarps * 32, 0, h->stream, 
                            h->d_fronts, it, c, h->d_septgt, sb.P, sb.C, n, nrhs); break;
                case 2: launch_k(k_s_small_bwd<T, UNIT, 2>, g, kSmallWarps * 32, 0, h->stream, 
                            h->d_fronts, it, c, h->d_septgt, sb.P, sb.C, n, nrhs); break;
                case 4: launch_k(k_s_small_bwd<T, UNIT, 4>, g, kSmallWarps * 32, 0, h->stream, 
                            h->d_fronts, it, c, h->d_septgt, sb.P, sb.C, n, nrhs); break;
                case 8: launch_k(k_s_small_bwd<T, UNIT, 8>, g, kSmallWarps * 32, 0, h->stream, 
                            h->d_fronts, it, c, h->d_septgt, sb.P, sb.C, n, nrhs); break;
                default: launch_k(k_s_small_bwd<T, UNIT, 16>, g, kSmallWarps * 32, 0, h->stream, 
                            h->d_fronts, it, c, h->d_septgt, sb.P, sb.C, n, nrhs); break;
            }
            MF_CUDA(cudaGetLastError());
        }
        if (lv.s_tiny.cnt)
            if (int rc = launch_tiny<T, UNIT, 1, kTinyNJ>(h, lv.s_tiny, sb, nrb, nrhs)) return rc;
        if (lv.s_tiny2.cnt)
            if (int rc = launch_tiny<T, UNIT, 1, kTinyNJ2>(h, lv.s_tiny2, sb, nrb, nrhs)) return rc;
    }
    if (h->sub_tasks.cnt) {
        // the subtrees of small fronts, backward, in one launch
        Timer t(h, K_S_SMALL);
        const unsigned g = (unsigned)h->sub_tasks.cnt;
        const int64_t t0 = h->sub_tasks.off;
        switch (nrb) {
            case 1: launch_k(k_s_sub_bwd<T, UNIT, 1>, g, kSubWarps * 32, 0, h->stream, 
                        h->d_fronts, items, t0, h->d_septgt, sb.P, sb.C, n, nrhs); break;
            case 2: launch_k(k_s_sub_bwd<T, UNIT, 2>, g, kSubWarps * 32, 0, h->stream, 
                        h->d_fronts, items, t0, h->d_septgt, sb.P, sb.C, n, nrhs); break;
            case 4: launch_k(k_s_sub_bwd<T, UNIT, 4>, g, kSubWarps * 32, 0, h->stream, 
                        h->d_fronts, items, t0, h->d_septgt, sb.P, sb.C, n, nrhs); break;
            case 8: launch_k(k_s_sub_bwd<T, UNIT, 8>, g, kSubWarps * 32, 0, h->stream, 
                        h->d_fronts, items, t0, h->d_septgt, sb.P, sb.C, n, nrhs); break;
            default: launch_k(k_s_sub_bwd<T, UNIT, 16>, g, kSubWarps * 32, 0, h->stream, 
                        h->d_fronts, items, t0, h->d_septgt, sb.P, sb.C, n, nrhs); break;
        }
        MF_CUDA(cudaGetLastError());
    }
    return 0;
}

// Solve in place on d_C (n x nrhs, ld n, elimination order); nrhs <= nrhs_cap.
int launch_solve_with(mf_handle* h, int64_t nrhs, double* R, double* W, double* C, double* part) {
    if (nrhs <= 0) return 0;
    if (h->selinv_done) {
        set_error("the FP64 panels hold the selected inverse (mf_selinv), not a factor: factorize again");
        return -1;
    }
    if (!have_fp64(h)) {
        set_error("no FP64 factor storage: a mixed handle has it only after an FP64 factorization");
        return -1;
    }
    if (h->mixed && !h->fp64_current) {
        set_error("the FP64 factor storage does not hold the current matrix: the last mixed factorization "
                  "stayed in FP32; use the refined solve");
        return -1;
    }
    if (nrhs > kMaxRhs) { set_error("launch_solve_with: nrhs chunk above 16"); return -1; }
    SolveBufs<double> sb{h->d_P, h->d_inv, h->d_d, R, W, C, part, h->d_inv2};
    return h->diag ? solve_impl<double, 1>(h, sb, (int)nrhs) : solve_impl<double, 0>(h, sb, (int)nrhs);
}
int launch_solve(mf_handle* h, int64_t nrhs) {
    if (nrhs <= 0) return 0;
    if (h->selinv_done) {
        set_error("the FP64 panels hold the selected inverse (mf_selinv), not a factor: factorize again");
        return -1;
    }
    if (!have_fp64(h)) {
        set_error("no FP64 factor storage: a mixed handle has it only after an FP64 factorization");
        return -1;
    }
    if (h->mixed && !h->fp64_current) {
        set_error("the FP64 factor storage does not hold the current matrix: the last mixed factorization "
                  "stayed in FP32; use the refined solve");
        return -1;
    }
    if (nrhs > kMaxRhs) { set_error("launch_solve: nrhs chunk above 16"); return -1; }
    SolveBufs<double> sb{h->d_P, h->d_inv, h->d_d, h->d_R, h->d_W, h->d_C, h->d_part, h->d_inv2};
    return run_captured(h, 3, nrhs, 0, 0, [&]() {
        return h->diag ? solve_impl<double, 1>(h, sb, (int)nrhs) : solve_impl<double, 0>(h, sb, (int)nrhs);
    });
}

// Same on the single-precision factor: f32.C (n x nrhs, elimination order) in place.
int launch_solve_mixed(mf_handle* h, int64_t nrhs) {
    if (nrhs <= 0) return 0;
    if (nrhs > kMaxRhs) { set_error("launch_solve: nrhs chunk above 16"); return -1; }
    SolveBufs<float> sb{h->f32.P, h->f32.inv, h->f32.d, h->f32.R, h->f32.W, h->f32.C, h->f32.part, h->f32.inv2};
    return run_captured(h, 4, nrhs, 0, 0, [&]() {
        return h->diag ? solve_impl<float, 1>(h, sb, (int)nrhs) : solve_impl<float, 0>(h, sb, (int)nrhs);
    });
}

}  // namespace mf
