// Mixed precision: FP64 refinement around the single-precision factor.
//
// The matrix is scaled symmetrically, A_hat = S A S with S = diag(|a_ii|^-1/2),
// and A_hat is factored in FP32 (the same plan and kernels as the FP64 path,
// instantiated for float).  M^-1 r = S A_hat^-1 S r is applied by an FP32
// supernodal solve.  FP64 stays in the residual b - A x (CSR of the original
// values, elimination order), the solution update and the scalars:
//   Cholesky : preconditioned conjugate gradients, one CG per right-hand side;
//   LDLt      : right-preconditioned restarted GMRES (GMRES-IR; the FP32
//               LDLt factor of an indefinite matrix is no SPD preconditioner,
//               and classical refinement stalls when kappa * eps32 is near 1),
//               classical Gram-Schmidt applied twice, one Krylov space per
//               right-hand side;
//   a Cholesky handle split into row segments (a batch of independent
//               matrices): conjugate gradients with CG scalars per segment
//               and column (segment dot products over row chunks, summed in
//               a fixed order), so every matrix follows its own recurrence;
//   an LDLt handle split into segments: GMRES with one Krylov space per
//               (segment, column), inner products per segment.
// With segments the backward error is measured per segment and the loop
// runs until the worst segment meets the tolerance.
// Every iteration measures the normwise backward error
//   eta = ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf)
// per column and stops when all columns reach the tolerance.  Reductions are
// two-pass in a fixed order (dots) or order-independent (max), so a run is
// bitwise repeatable.
#include <algorithm>
#include <cmath>
#include <vector>

#include "mf_internal.cuh"

namespace mf {

constexpr int kRedBlocks = 148 * 4;  // partial sums per reduction
// d_red layout: [0,48) residual maxima, [48] ||A||_inf, [64,144) CG scalars,
// [256, 256 + 16*kRedBlocks) dot partials
constexpr int kRedPart = 256;

__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
    // non-negative doubles order like their bit patterns
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// y = A x for nrhs columns (ld n); values read through the stored-value map
__global__ void k_spmv(const int64_t* __restrict__ ptr, const int32_t* __restrict__ col,
                       const int64_t* __restrict__ src, const double* __restrict__ nz, const double* __restrict__ x,
                       double* __restrict__ y, int64_t n, int nrhs) {
    pdl_prologue();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    double acc[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) acc[r] = 0.0;
    for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
        const double a = nz[src[p]];
        const int64_t c = col[p];
#pragma unroll
        for (int r = 0; r < 16; ++r)
            if (r < nrhs) acc[r] += a * x[c + r * n];
    }
#pragma unroll
    for (int r = 0; r < 16; ++r)
        if (r < nrhs) y[i + r * n] = acc[r];
}

// t = b - A x for row i (all columns) with the stored-value map; the
// products are added in the row's stored order
template <int NR>
__device__ __forceinline__ void resid_row(const int64_t* __restrict__ ptr, const int32_t* __restrict__ col,
                                          const int64_t* __restrict__ src, const double* __restrict__ nz,
                                          const double* __restrict__ x, int64_t i, int64_t n, int nrhs,
                                          double (&acc)[NR]) {
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = 0.0;
    const int64_t p1 = ptr[i + 1];
#pragma unroll 4
    for (int64_t p = ptr[i]; p < p1; ++p) {
        const double a = nz[src[p]];
        const int64_t c = col[p];
#pragma unroll
        for (int r = 0; r < NR; ++r)
            if (r < nrhs) acc[r] += a * x[c + r * n];
    }
}

// t = b - A x and the maxima needed by the backward error:
// red[0..nrhs) = max|t|, red[16..) = max|x|, red[32..) = max|b|
template <int NR>
__global__ void __launch_bounds__(256) k_resid(const int64_t* __restrict__ ptr, const int32_t* __restrict__ col,
                                               const int64_t* __restrict__ src, const double* __restrict__ nz,
                                               const double* __restrict__ x, const double* __restrict__ b,
                                               double* __restrict__ t, double* __restrict__ red, int64_t n,
                                               int nrhs) {
    pdl_prologue();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool live = i < n;
    if (!live) i = n - 1;  // keep the whole block in the reductions; results of this lane are ignored below
    double acc[NR];
    resid_row<NR>(ptr, col, src, nz, x, i, n, nrhs, acc);
    // block-level maxima first, then one atomic per block and quantity
    __shared__ double mx[48];
    if (threadIdx.x < 48) mx[threadIdx.x] = 0.0;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        if (r >= nrhs) break;  // uniform across the block
        const double bi = b[i + r * n];
        const double ti = bi - acc[r];
        if (t && live) t[i + r * n] = ti;
        double v0 = fabs(ti), v1 = fabs(x[i + r * n]), v2 = fabs(bi);
        for (int o = 16; o > 0; o >>= 1) {
            v0 = fmax(v0, __shfl_xor_sync(0xffffffffu, v0, o));
            v1 = fmax(v1, __shfl_xor_sync(0xffffffffu, v1, o));
            v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomic_max_nonneg(mx + r, v0);
            atomic_max_nonneg(mx + 16 + r, v1);
            atomic_max_nonneg(mx + 32 + r, v2);
        }
    }
    __syncthreads();
    if (threadIdx.x < 48 && (threadIdx.x & 15) < nrhs) atomic_max_nonneg(red + threadIdx.x, mx[threadIdx.x]);
}

// Per-segment version: one thread per row, and the maxima of every segment
// go to segred[s * kSegRed + (0|16|32) + r] (zeroed by k_seg_zero) by
// atomic max, order-independent; a warp whose rows lie in one segment
// reduces by shuffles first.
template <int NR>
__global__ void __launch_bounds__(256) k_resid_seg(const int64_t* __restrict__ ptr, const int32_t* __restrict__ col,
                                                   const int64_t* __restrict__ src, const double* __restrict__ nz,
                                                   const double* __restrict__ x, const double* __restrict__ b,
                                                   double* __restrict__ t, const int32_t* __restrict__ rowseg,
                                                   double* __restrict__ segred, int64_t n, int nrhs) {
    pdl_prologue();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool live = i < n;
    if (!live) i = n - 1;
    double acc[NR];
    resid_row<NR>(ptr, col, src, nz, x, i, n, nrhs, acc);
    const int sg = live ? rowseg[i] : -1;
    const int sg0 = __shfl_sync(0xffffffffu, sg, 0);
    const bool one = __all_sync(0xffffffffu, sg == sg0);
    if (one && sg0 < 0) return;  // a warp past the last row
    double* q = segred + (int64_t)(one ? sg0 : sg) * kSegRed;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        if (r >= nrhs) break;  // uniform across the grid
        const double bi = b[i + r * n];
        const double ti = bi - acc[r];
        if (t && live) t[i + r * n] = ti;
        double v0 = fabs(ti), v1 = fabs(x[i + r * n]), v2 = fabs(bi);
        if (one) {
            for (int o = 16; o > 0; o >>= 1) {
                v0 = fmax(v0, __shfl_xor_sync(0xffffffffu, v0, o));
                v1 = fmax(v1, __shfl_xor_sync(0xffffffffu, v1, o));
                v2 = fmax(v2, __shfl_xor_sync(0xffffffffu, v2, o));
            }
            if ((threadIdx.x & 31) != 0) continue;
        } else if (!live) {
            continue;
        }
        atomic_max_nonneg(q + r, v0);
        atomic_max_nonneg(q + 16 + r, v1);
        atomic_max_nonneg(q + 32 + r, v2);
    }
}

// segred[s * kSegRed + q] = 0 for q < 48 (entry 48, the segment's ||A||_inf, stays)
__global__ void k_seg_zero(double* __restrict__ segred, int64_t nseg) {
    pdl_prologue();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < nseg * 48) segred[(i / 48) * kSegRed + i % 48] = 0.0;
}

// per chunk and column: sum of u .* v over the chunk's rows into
// chunkred[c * kChunkRed + kSegRed + r]
__global__ void k_dot_chunk(const double* __restrict__ u, const double* __restrict__ v,
                            const int64_t* __restrict__ chunkrow, double* __restrict__ chunkred, int64_t n,
                            int nrhs) {
    pdl_prologue();
    __shared__ double sh[256];
    const int64_t c = blockIdx.x;
    const int64_t r0 = chunkrow[c], r1 = chunkrow[c + 1];
    for (int r = 0; r < nrhs; ++r) {
        double s = 0.0;
        for (int64_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) s += u[i + r * n] * v[i + r * n];
        sh[threadIdx.x] = s;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) chunkred[c * kChunkRed + kSegRed + r] = sh[0];
        __syncthreads();
    }
}

// out[s * 80 + r] = sum over the chunks of segment s (fixed order)
__global__ void k_dot_seg(const double* __restrict__ chunkred, const int64_t* __restrict__ segchunk,
                          double* __restrict__ out, int64_t nseg, int nrhs) {
    pdl_prologue();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nseg * 16) return;
    const int64_t sg = i / 16;
    const int r = (int)(i % 16);
    if (r >= nrhs) return;
    double v = 0.0;
    for (int64_t c = segchunk[sg]; c < segchunk[sg + 1]; ++c) v += chunkred[c * kChunkRed + kSegRed + r];
    out[sg * 80 + r] = v;
}

// eta of every (segment, column); segeta[s] = worst column of segment s,
// out[r] = worst segment of column r
__global__ void k_seg_eta(const double* __restrict__ segred, int64_t nseg, int nrhs, double* __restrict__ out,
                          double* __restrict__ segeta) {
    pdl_prologue();
    __shared__ double mx[16];
    if (threadIdx.x < 16) mx[threadIdx.x] = 0.0;
    __syncthreads();
    double worst[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) worst[r] = 0.0;
    for (int64_t s = threadIdx.x; s < nseg; s += blockDim.x) {
        const double* q = segred + s * kSegRed;
        double w = 0.0;
#pragma unroll
        for (int r = 0; r < 16; ++r)
            if (r < nrhs) {
                const double den = q[48] * q[16 + r] + q[32 + r];
                const double e = den > 0.0 ? q[r] / den : (q[r] > 0.0 ? INFINITY : 0.0);
                w = fmax(w, e);
                worst[r] = fmax(worst[r], e);
            }
        segeta[s] = w;
    }
#pragma unroll
    for (int r = 0; r < 16; ++r) {
        double v = worst[r];
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if ((threadIdx.x & 31) == 0 && r < nrhs) atomic_max_nonneg(mx + r, v);
    }
    __syncthreads();
    if (threadIdx.x < 16) out[threadIdx.x] = mx[threadIdx.x];
}

// ||A||_inf (max absolute row sum) into *out: one row per thread, the
// warp's maximum by shuffles, one atomic per warp (one per row serialised
// every thread of the grid on the same address)
__global__ void k_anorm(const int64_t* __restrict__ ptr, const int64_t* __restrict__ src,
                        const double* __restrict__ nz, double* __restrict__ out, int64_t n) {
    pdl_prologue();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    double s = 0.0;
    if (i < n)
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) s += fabs(nz[src[p]]);
    for (int o = 16; o > 0; o >>= 1) s = fmax(s, __shfl_xor_sync(0xffffffffu, s, o));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, s);
}

// per-column partial dot products: part[blk * 16 + r]
__global__ void k_dot_part(const double* __restrict__ u, const double* __restrict__ v, double* __restrict__ part,
                           int64_t n, int nrhs) {
    pdl_prologue();
    __shared__ double sh[256];
    for (int r = 0; r < nrhs; ++r) {
        double s = 0.0;
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            s += u[i + r * n] * v[i + r * n];
        sh[threadIdx.x] = s;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[blockIdx.x * 16 + r] = sh[0];
        __syncthreads();
    }
}

// out[r] = sum over blocks (fixed order)
// one warp per right-hand side: lane l adds blocks l, l + 32, ... in order,
// then a fixed shuffle tree (deterministic, and the loads of a lane are
// independent instead of one dependent chain over all blocks)
__global__ void k_dot_final(const double* __restrict__ part, double* __restrict__ out, int nblocks, int nrhs) {
    pdl_prologue();
    const int r = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (r >= nrhs) return;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += part[b * 16 + r];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[r] = s;
}

// CG scalars: mode 0: alpha = rz / pq; mode 1: beta = rz_new / rz, rz = rz_new
__global__ void k_cg_scalars(double* __restrict__ sc, int nrhs, int mode) {
    pdl_prologue();
    int r = threadIdx.x;
    if (r >= nrhs) return;
    double* rz = sc;           // [0..16)
    double* pq = sc + 16;      // [16..32)
    double* alpha = sc + 32;   // [32..48)
    double* rzn = sc + 48;     // [48..64)
    double* beta = sc + 64;    // [64..80)
    if (mode == 0) {
        alpha[r] = (pq[r] != 0.0 && rz[r] != 0.0) ? rz[r] / pq[r] : 0.0;
    } else {
        beta[r] = rz[r] != 0.0 ? rzn[r] / rz[r] : 0.0;
        rz[r] = rzn[r];
    }
}

// x += alpha p ; r -= alpha q
__global__ void k_cg_xr(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                        const double* __restrict__ q, const double* __restrict__ alpha, int64_t n, int nrhs) {
    pdl_prologue();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n * nrhs; i += stride) {
        const double a = alpha[i / n];
        x[i] += a * p[i];
        r[i] -= a * q[i];
    }
}

// p = z + beta p
__global__ void k_cg_p(double* __restrict__ p, const double* __restrict__ z, const double* __restrict__ beta,
                       int64_t n, int nrhs) {
    pdl_prologue();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n * nrhs; i += stride) p[i] = z[i] + beta[i / n] * p[i];
}

// the CG scalars above for every segment: sc[s * 80 + ...]
__global__ void k_cg_scalars_seg(double* __restrict__ sc, int64_t nseg, int nrhs, int mode) {
    pdl_prologue();
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= nseg * 16) return;
    const int r = (int)(i % 16);
    if (r >= nrhs) return;
    double* q = sc + (i / 16) * 80;
    if (mode == 0) {
        q[32 + r] = (q[16 + r] != 0.0 && q[r] != 0.0) ? q[r] / q[16 + r] : 0.0;
    } else {
        q[64 + r] = q[r] != 0.0 ? q[48 + r] / q[r] : 0.0;
        q[r] = q[48 + r];
    }
}

// x += alpha_s p ; r -= alpha_s q   (alpha of the row's segment)
__global__ void k_cg_xr_seg(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                            const double* __restrict__ q, const double* __restrict__ sc,
                            const int32_t* __restrict__ rowseg, int64_t n, int nrhs) {
    pdl_prologue();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n * nrhs; i += stride) {
        const double a = sc[(int64_t)rowseg[i % n] * 80 + 32 + i / n];
        x[i] += a * p[i];
        r[i] -= a * q[i];
    }
}

// p = z + beta_s p
__global__ void k_cg_p_seg(double* __restrict__ p, const double* __restrict__ z, const double* __restrict__ sc,
                           const int32_t* __restrict__ rowseg, int64_t n, int nrhs) {
    pdl_prologue();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n * nrhs; i += stride) p[i] = z[i] + sc[(int64_t)rowseg[i % n] * 80 + 64 + i / n] * p[i];
}

// c = (float)(s .* r)   and   z = s .* (double)c  (+= when ACC)
__global__ void k_to32(float* __restrict__ c, const double* __restrict__ r, const double* __restrict__ s, int64_t n,
                       int nrhs) {
    pdl_prologue();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n * nrhs; i += stride) c[i] = (float)(s[i % n] * r[i]);
}
template <bool ACC>
__global__ void k_from32(double* __restrict__ z, const float* __restrict__ c, const double* __restrict__ s, int64_t n,
                         int nrhs) {
    pdl_prologue();
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < n * nrhs; i += stride) {
        double v = s[i % n] * (double)c[i];
        if (ACC) z[i] += v; else z[i] = v;
    }
}

// ---------------------------------------------------------------------------
// GMRES kernels.  Krylov vectors V_i / Z_i are n x nrhs blocks (ld n) spaced
// `vs` doubles apart; coefficient arrays are indexed [i * 16 + r].
// ---------------------------------------------------------------------------
constexpr int kGmresM = 24;  // restart length

// part[(blk * J + i) * 16 + r] = this block's share of <V_i(:, r), w(:, r)>
__global__ void k_mdot_part(const double* __restrict__ V, int64_t vs, int J, const double* __restrict__ w,
                            double* __restrict__ part, int64_t n, int nrhs) {
    pdl_prologue();
    __shared__ double sh[256];
    for (int i = 0; i < J; ++i)
        for (int r = 0; r < nrhs; ++r) {
            const double* v = V + i * vs + (int64_t)r * n;
            const double* ww = w + (int64_t)r * n;
            double s = 0.0;
            for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
                s += v[k] * ww[k];
            sh[threadIdx.x] = s;
            __syncthreads();
            for (int o = blockDim.x / 2; o > 0; o >>= 1) {
                if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
                __syncthreads();
            }
            if (threadIdx.x == 0) part[((int64_t)blockIdx.x * J + i) * 16 + r] = sh[0];
            __syncthreads();
        }
}

// out[i * 16 + r] = sum over blocks (fixed order)
// one warp per output (i, r), as k_dot_final
__global__ void k_mdot_final(const double* __restrict__ part, double* __restrict__ out, int nblocks, int J,
                             int nrhs) {
    pdl_prologue();
    const int o = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (o >= J * 16) return;
    const int i = o / 16, r = o % 16;
    if (r >= nrhs) return;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += part[((int64_t)b * J + i) * 16 + r];
    for (int q = 16; q > 0; q >>= 1) s += __shfl_xor_sync(0xffffffffu, s, q);
    if (lane == 0) out[o] = s;
}

// w(:, r) -= sum_{i < J} c[i * 16 + r] V_i(:, r)
__global__ void k_mupd(double* __restrict__ w, const double* __restrict__ V, int64_t vs, int J,
                       const double* __restrict__ c, int64_t n, int nrhs) {
    pdl_prologue();
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n * nrhs;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(k / n);
        double s = 0.0;
        for (int i = 0; i < J; ++i) s += c[i * 16 + r] * V[i * vs + k];
        w[k] -= s;
    }
}

// dst(:, r) = src(:, r) * c[r]
__global__ void k_colscale(double* __restrict__ dst, const double* __restrict__ src, const double* __restrict__ c,
                           int64_t n, int nrhs) {
    pdl_prologue();
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n * nrhs;
         k += (int64_t)gridDim.x * blockDim.x)
        dst[k] = src[k] * c[k / n];
}

// Segmented forms of the GMRES kernels: a right-hand side of every segment
// has its own Krylov space, so coefficients are indexed (i, segment, column)
// as c[(i * G + s) * 16 + r] with G segments.
__global__ void k_mdot_chunk(const double* __restrict__ V, int64_t vs, int J, const double* __restrict__ w,
                             const int64_t* __restrict__ chunkrow, double* __restrict__ part, int64_t n, int nrhs) {
    pdl_prologue();
    __shared__ double sh[256];
    const int64_t c = blockIdx.x;
    const int64_t r0 = chunkrow[c], r1 = chunkrow[c + 1];
    for (int i = 0; i < J; ++i)
        for (int r = 0; r < nrhs; ++r) {
            const double* v = V + i * vs + (int64_t)r * n;
            const double* ww = w + (int64_t)r * n;
            double sum = 0.0;
            for (int64_t k = r0 + threadIdx.x; k < r1; k += blockDim.x) sum += v[k] * ww[k];
            sh[threadIdx.x] = sum;
            __syncthreads();
            for (int o = blockDim.x / 2; o > 0; o >>= 1) {
                if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
                __syncthreads();
            }
            if (threadIdx.x == 0) part[(c * J + i) * 16 + r] = sh[0];
            __syncthreads();
        }
}
__global__ void k_mdot_seg(const double* __restrict__ part, const int64_t* __restrict__ segchunk,
                           double* __restrict__ out, int64_t G, int J, int nrhs) {
    pdl_prologue();
    const int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (o >= (int64_t)J * G * 16) return;
    const int r = (int)(o % 16);
    const int64_t sg = (o / 16) % G;
    const int i = (int)(o / (16 * G));
    double v = 0.0;
    if (r < nrhs)
        for (int64_t c = segchunk[sg]; c < segchunk[sg + 1]; ++c) v += part[(c * J + i) * 16 + r];
    out[o] = v;
}
__global__ void k_mupd_seg(double* __restrict__ w, const double* __restrict__ V, int64_t vs, int J,
                           const double* __restrict__ c, const int32_t* __restrict__ rowseg, int64_t G, int64_t n,
                           int nrhs) {
    pdl_prologue();
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n * nrhs;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q = (int64_t)rowseg[k % n] * 16 + k / n;
        double sum = 0.0;
        for (int i = 0; i < J; ++i) sum += c[i * G * 16 + q] * V[i * vs + k];
        w[k] -= sum;
    }
}
__global__ void k_colscale_seg(double* __restrict__ dst, const double* __restrict__ src, const double* __restrict__ c,
                               const int32_t* __restrict__ rowseg, int64_t n, int nrhs) {
    pdl_prologue();
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n * nrhs;
         k += (int64_t)gridDim.x * blockDim.x)
        dst[k] = src[k] * c[(int64_t)rowseg[k % n] * 16 + k / n];
}

// ||A||_inf of every chunk into chunkred[c * kChunkRed + 48]; k_seg_anorm
// takes the maximum over a segment's chunks into segred[s * kSegRed + 48]
__global__ void k_anorm_chunk(const int64_t* __restrict__ ptr, const int64_t* __restrict__ src,
                              const double* __restrict__ nz, const int64_t* __restrict__ chunkrow,
                              double* __restrict__ chunkred) {
    pdl_prologue();
    const int64_t c = blockIdx.x;
    double v = 0.0;
    for (int64_t i = chunkrow[c] + threadIdx.x; i < chunkrow[c + 1]; i += blockDim.x) {
        double rs = 0.0;
        for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) rs += fabs(nz[src[p]]);
        v = fmax(v, rs);
    }
    __shared__ double mx;
    if (threadIdx.x == 0) mx = 0.0;
    __syncthreads();
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&mx, v);
    __syncthreads();
    if (threadIdx.x == 0) chunkred[c * kChunkRed + 48] = mx;
}
__global__ void k_seg_anorm(const double* __restrict__ chunkred, const int64_t* __restrict__ segchunk,
                            double* __restrict__ segred, int64_t nseg) {
    pdl_prologue();
    const int64_t sg = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (sg >= nseg) return;
    double v = 0.0;
    for (int64_t c = segchunk[sg]; c < segchunk[sg + 1]; ++c) v = fmax(v, chunkred[c * kChunkRed + 48]);
    segred[sg * kSegRed + 48] = v;
}

static unsigned gs_blocks(int64_t work) {
    int64_t b = (work + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    if (b < 1) b = 1;
    return (unsigned)b;
}

static inline unsigned row_blocks(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + 255) / 256); }

// z = M^-1 r (ACC: z += M^-1 r) through the FP32 factor
template <bool ACC>
static int apply_prec(mf_handle* h, const double* r, double* z, int nrhs) {
    launch_k(k_to32, gs_blocks(h->n * nrhs), 256, 0, h->stream, h->f32.C, r, h->d_scale, h->n, nrhs);
    MF_CUDA(cudaGetLastError());
    int rc = launch_solve_mixed(h, nrhs);
    if (rc) return rc;
    launch_k(k_from32<ACC>, gs_blocks(h->n * nrhs), 256, 0, h->stream, z, h->f32.C, h->d_scale, h->n, nrhs);
    MF_CUDA(cudaGetLastError());
    return 0;
}

static int dot(mf_handle* h, const double* u, const double* v, double* out, int nrhs) {
    double* part = h->d_red + kRedPart;
    launch_k(k_dot_part, kRedBlocks, 256, 0, h->stream, u, v, part, h->n, nrhs);
    MF_CUDA(cudaGetLastError());
    launch_k(k_dot_final, 1, 32 * 16, 0, h->stream, part, out, kRedBlocks, nrhs);
    MF_CUDA(cudaGetLastError());
    return 0;
}

// per-segment dot products into h->d_segsc[s * 80 + off + r]
static int dot_seg(mf_handle* h, const double* u, const double* v, int off, int nrhs) {
    if (h->nchunk > 0) {
        launch_k(k_dot_chunk, (unsigned)h->nchunk, 256, 0, h->stream, u, v, h->d_chunkrow, h->d_chunkred, h->n, nrhs);
        MF_CUDA(cudaGetLastError());
    }
    launch_k(k_dot_seg, (unsigned)((h->nseg * 16 + 255) / 256), 256, 0, h->stream, h->d_chunkred, h->d_segchunk,
                                                                             h->d_segsc + off, h->nseg, nrhs);
    MF_CUDA(cudaGetLastError());
    return 0;
}

// backward error per column into eta[] (host); t receives b - A x when non-null
static int backward_error(mf_handle* h, const double* x, const double* b, double* t, int nrhs, double* eta,
                          double* maxima = nullptr) {
    Timer tm(h, K_SPMV);
    double* red = h->d_red;  // [0..48) maxima, [48] ||A||_inf
    if (h->nseg > 0) {
        launch_k(k_seg_zero, (unsigned)((h->nseg * 48 + 255) / 256), 256, 0, h->stream, h->d_segred, h->nseg);
        MF_CUDA(cudaGetLastError());
        if (h->n > 0) {
            const unsigned g = row_blocks(h->n);
#define MF_RESID_SEG(NRV)                                                                                        \
    launch_k(k_resid_seg<NRV>, g, 256, 0, h->stream, h->d_csrptr, h->d_csrcol, h->d_csrsrc, h->cur_nz, x, b, t, \
             h->d_rowseg, h->d_segred, h->n, nrhs)
            if (nrhs <= 1) MF_RESID_SEG(1);
            else if (nrhs <= 2) MF_RESID_SEG(2);
            else if (nrhs <= 4) MF_RESID_SEG(4);
            else if (nrhs <= 8) MF_RESID_SEG(8);
            else MF_RESID_SEG(16);
#undef MF_RESID_SEG
            MF_CUDA(cudaGetLastError());
        }
        launch_k(k_seg_eta, 1, 256, 0, h->stream, h->d_segred, h->nseg, nrhs, red, h->d_segeta);
        MF_CUDA(cudaGetLastError());
        MF_CUDA(cudaMemcpyAsync(eta, red, 16 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        MF_CUDA(cudaStreamSynchronize(h->stream));
        return 0;
    }
    MF_CUDA(cudaMemsetAsync(red, 0, 48 * sizeof(double), h->stream));
    {
        const unsigned g = row_blocks(h->n);
#define MF_RESID(NRV) \
    launch_k(k_resid<NRV>, g, 256, 0, h->stream, h->d_csrptr, h->d_csrcol, h->d_csrsrc, h->cur_nz, x, b, t, red, h->n, nrhs)
        if (nrhs <= 1) MF_RESID(1);
        else if (nrhs <= 2) MF_RESID(2);
        else if (nrhs <= 4) MF_RESID(4);
        else if (nrhs <= 8) MF_RESID(8);
        else MF_RESID(16);
#undef MF_RESID
    }
    MF_CUDA(cudaGetLastError());
    double hred[49];
    MF_CUDA(cudaMemcpyAsync(hred, red, 49 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    MF_CUDA(cudaStreamSynchronize(h->stream));
    for (int r = 0; r < nrhs; ++r) {
        double den = hred[48] * hred[16 + r] + hred[32 + r];
        eta[r] = den > 0.0 ? hred[r] / den : (hred[r] > 0.0 ? INFINITY : 0.0);
    }
    if (maxima)
        for (int q = 0; q < 49; ++q) maxima[q] = hred[q];
    return 0;
}

// Right-preconditioned restarted GMRES, M^-1 = the FP32 factor solve; one
// Krylov space per right-hand side, all columns advanced together.  With G
// row segments (a batch of independent matrices) every (segment, column)
// pair q = s * 16 + r has its own Krylov space: the inner products are
// taken per segment and the coefficients applied per row's segment.
// Returns the total number of preconditioner applications in *iters.
static int gmres(mf_handle* h, const double* b, double* x, int nrhs, double tol, int maxit, int* iters,
                 double* eta_out) {
    const int64_t n = h->n;
    const int M = kGmresM;
    const int64_t vs = n * nrhs;
    const bool seg = h->nseg > 1;
    const int64_t G = seg ? h->nseg : 1;
    const int64_t Q = G * 16;  // (segment, column) slots
    const int nblk = (int)std::min<int64_t>(148 * 4, std::max<int64_t>(1, (n + 255) / 256));
    const int64_t npart = (int64_t)std::max<int64_t>(148 * 4, seg ? h->nchunk : 0) * (M + 1) * 16;
    const int64_t need = (int64_t)(2 * M + 1) * n * h->nrhs_cap + npart + (M + 1) * Q + 64 * 16;
    if (h->kry_doubles < need) {
        std::lock_guard<std::recursive_mutex> lk(device_mutex());
        if (h->d_kry) cudaFree(h->d_kry);
        h->d_kry = nullptr;
        h->kry_doubles = 0;
        MF_CUDA(cudaMalloc(&h->d_kry, sizeof(double) * need));
        h->kry_doubles = need;
        h->bytes += (int64_t)sizeof(double) * need;
    }
    double* V = h->d_kry;                                    // M + 1 blocks
    double* Z = V + (int64_t)(M + 1) * n * h->nrhs_cap;      // M blocks
    double* part = Z + (int64_t)M * n * h->nrhs_cap;         // partial sums
    double* coef = part + npart;                             // (M + 1) * Q coefficients
    double* R = h->d_iv + 2 * (int64_t)n * h->nrhs_cap;      // residual
    double eta[16], mx[49];
    std::vector<double> H((size_t)(M + 1) * M * Q), g((size_t)(M + 1) * Q), cs((size_t)M * Q), sn((size_t)M * Q);
    std::vector<double> hc((size_t)(M + 1) * Q), beta(Q), tgt(Q), inv(Q), segred;
    int rc, used = 0;
    double worst = INFINITY;
    MF_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n * nrhs, h->stream));
    auto live = [&](int64_t q) { return (int)(q % 16) < nrhs; };
    // out_host[(i * G + s) * 16 + r] = <V_i, w> over the rows of segment s
    auto mdot = [&](const double* Vb, int J, const double* w, double* out_host) -> int {
        if (seg) {
            if (h->nchunk > 0) {
                launch_k(k_mdot_chunk, (unsigned)h->nchunk, 256, 0, h->stream, Vb, vs, J, w, h->d_chunkrow, part, n, nrhs);
                MF_CUDA(cudaGetLastError());
            }
            launch_k(k_mdot_seg, (unsigned)((J * Q + 255) / 256), 256, 0, h->stream, part, h->d_segchunk, coef, G, J,
                                                                                nrhs);
        } else {
            launch_k(k_mdot_part, nblk, 256, 0, h->stream, Vb, vs, J, w, part, n, nrhs);
            MF_CUDA(cudaGetLastError());
            launch_k(k_mdot_final, (unsigned)((J * 16 + 7) / 8), 256, 0, h->stream, part, coef, nblk, J, nrhs);
        }
        MF_CUDA(cudaGetLastError());
        MF_CUDA(cudaMemcpyAsync(out_host, coef, sizeof(double) * J * Q, cudaMemcpyDeviceToHost, h->stream));
        MF_CUDA(cudaStreamSynchronize(h->stream));
        return 0;
    };
    auto colscale = [&](double* dst, const double* src, const double* c_host) -> int {
        MF_CUDA(cudaMemcpyAsync(coef, c_host, sizeof(double) * Q, cudaMemcpyHostToDevice, h->stream));
        if (seg) launch_k(k_colscale_seg, gs_blocks(vs), 256, 0, h->stream, dst, src, coef, h->d_rowseg, n, nrhs);
        else launch_k(k_colscale, gs_blocks(vs), 256, 0, h->stream, dst, src, coef, n, nrhs);
        MF_CUDA(cudaGetLastError());
        return 0;
    };
    auto mupd = [&](double* w, const double* Vb, int J, const double* c_host) -> int {
        MF_CUDA(cudaMemcpyAsync(coef, c_host, sizeof(double) * J * Q, cudaMemcpyHostToDevice, h->stream));
        if (seg) launch_k(k_mupd_seg, gs_blocks(vs), 256, 0, h->stream, w, Vb, vs, J, coef, h->d_rowseg, G, n, nrhs);
        else launch_k(k_mupd, gs_blocks(vs), 256, 0, h->stream, w, Vb, vs, J, coef, n, nrhs);
        MF_CUDA(cudaGetLastError());
        return 0;
    };
    while (true) {
        // true residual and backward error of the current x, and the inner
        // target of every slot on GMRES's ||r||_2: half the tolerance at the
        // current scale, widened by sqrt(rows) / 8 -- a residual spread over
        // m rows has ||r||_inf near a few times ||r||_2 / sqrt(m); the outer
        // loop checks the true backward error and restarts if it is missed
        if ((rc = backward_error(h, x, b, R, nrhs, eta, mx))) return rc;
        worst = 0.0;
        for (int r = 0; r < nrhs; ++r) worst = std::max(worst, eta[r]);
        if (worst <= tol || used >= maxit) break;
        if (h->nseg > 0) {
            // per-segment maxima (d_segred) of the residual, x, b and ||A||_inf
            segred.resize((size_t)h->nseg * kSegRed);
            MF_CUDA(cudaMemcpyAsync(segred.data(), h->d_segred, sizeof(double) * segred.size(),
                                    cudaMemcpyDeviceToHost, h->stream));
            MF_CUDA(cudaStreamSynchronize(h->stream));
            for (int64_t q = 0; q < Q; ++q) {
                const double* sr = segred.data() + (q / 16) * kSegRed;  // one segment when !seg
                const int r = (int)(q % 16);
                const int64_t rows = seg ? h->h_segptr[q / 16 + 1] - h->h_segptr[q / 16] : n;
                tgt[q] = 0.5 * tol * (sr[48] * sr[16 + r] + sr[32 + r]) *
                         std::max(1.0, std::sqrt((double)rows) / 8.0);
            }
        } else {
            for (int r = 0; r < 16; ++r)
                tgt[r] = 0.5 * tol * (mx[48] * mx[16 + r] + mx[32 + r]) * std::max(1.0, std::sqrt((double)n) / 8.0);
        }
        if ((rc = mdot(R, 1, R, hc.data()))) return rc;
        for (int64_t q = 0; q < Q; ++q) {
            beta[q] = live(q) ? std::sqrt(std::max(hc[q], 0.0)) : 0.0;
            inv[q] = beta[q] > 0.0 ? 1.0 / beta[q] : 0.0;
        }
        if ((rc = colscale(V, R, inv.data()))) return rc;
        std::fill(H.begin(), H.end(), 0.0);
        std::fill(g.begin(), g.end(), 0.0);
        for (int64_t q = 0; q < Q; ++q) g[q] = beta[q];
        int j = 0;
        bool stop = false;
        for (; j < M && !stop && used < maxit; ++j) {
            double* Vj = V + j * vs;
            double* Zj = Z + j * vs;
            double* w = V + (j + 1) * vs;
            if ((rc = apply_prec<false>(h, Vj, Zj, nrhs))) return rc;
            ++used;
            {
                Timer tm(h, K_SPMV);
                launch_k(k_spmv, row_blocks(n), 256, 0, h->stream, h->d_csrptr, h->d_csrcol, h->d_csrsrc, h->cur_nz, Zj, w,
                                                              n, nrhs);
                MF_CUDA(cudaGetLastError());
            }
            // classical Gram-Schmidt, twice
            for (int pass = 0; pass < 2; ++pass) {
                if ((rc = mdot(V, j + 1, w, hc.data()))) return rc;
                if ((rc = mupd(w, V, j + 1, hc.data()))) return rc;
                for (int i = 0; i <= j; ++i)
                    for (int64_t q = 0; q < Q; ++q) H[((size_t)i * M + j) * Q + q] += hc[i * Q + q];
            }
            if ((rc = mdot(w, 1, w, hc.data()))) return rc;
            stop = true;
            for (int64_t q = 0; q < Q; ++q) {
                if (!live(q)) { inv[q] = 0.0; continue; }
                const double hn = std::sqrt(std::max(hc[q], 0.0));
                H[((size_t)(j + 1) * M + j) * Q + q] = hn;
                inv[q] = hn > 0.0 ? 1.0 / hn : 0.0;
                // apply the earlier rotations to column j, then a new one
                for (int i = 0; i < j; ++i) {
                    double& a = H[((size_t)i * M + j) * Q + q];
                    double& c2 = H[((size_t)(i + 1) * M + j) * Q + q];
                    const double t0 = cs[i * Q + q] * a + sn[i * Q + q] * c2;
                    c2 = -sn[i * Q + q] * a + cs[i * Q + q] * c2;
                    a = t0;
                }
                double& a = H[((size_t)j * M + j) * Q + q];
                double& c2 = H[((size_t)(j + 1) * M + j) * Q + q];
                const double den = std::hypot(a, c2);
                const double c = den > 0.0 ? a / den : 1.0, sgn = den > 0.0 ? c2 / den : 0.0;
                cs[j * Q + q] = c;
                sn[j * Q + q] = sgn;
                a = den;
                c2 = 0.0;
                g[(j + 1) * Q + q] = -sgn * g[j * Q + q];
                g[j * Q + q] = c * g[j * Q + q];
                if (std::fabs(g[(j + 1) * Q + q]) > tgt[q] && hn > 0.0) stop = false;
            }
            if ((rc = colscale(w, w, inv.data()))) return rc;
        }
        // y = H^-1 g (upper triangular, j x j), x += Z y
        std::vector<double> y((size_t)j * Q, 0.0);
        for (int64_t q = 0; q < Q; ++q) {
            if (!live(q)) continue;
            for (int i = j - 1; i >= 0; --i) {
                double v = g[i * Q + q];
                for (int k = i + 1; k < j; ++k) v -= H[((size_t)i * M + k) * Q + q] * y[k * Q + q];
                const double d = H[((size_t)i * M + i) * Q + q];
                y[i * Q + q] = d != 0.0 ? v / d : 0.0;
            }
        }
        for (auto& v : y) v = -v;  // mupd subtracts
        if ((rc = mupd(x, Z, j, y.data()))) return rc;
    }
    if (iters) *iters = used;
    if (eta_out) *eta_out = worst;
    return 0;
}

int launch_anorm(mf_handle* h) {
    double* out = h->d_red + 48;
    MF_CUDA(cudaMemsetAsync(out, 0, sizeof(double), h->stream));
    launch_k(k_anorm, row_blocks(h->n), 256, 0, h->stream, h->d_csrptr, h->d_csrsrc, h->cur_nz, out, h->n);
    MF_CUDA(cudaGetLastError());
    if (h->nseg > 0) {
        if (h->nchunk > 0) {
            launch_k(k_anorm_chunk, (unsigned)h->nchunk, 256, 0, h->stream, h->d_csrptr, h->d_csrsrc, h->cur_nz,
                                                                       h->d_chunkrow, h->d_chunkred);
            MF_CUDA(cudaGetLastError());
        }
        launch_k(k_seg_anorm, (unsigned)((h->nseg + 255) / 256), 256, 0, h->stream, h->d_chunkred, h->d_segchunk,
                                                                               h->d_segred, h->nseg);
        MF_CUDA(cudaGetLastError());
    }
    return 0;
}

// Solve A x = b (b, x: n x nrhs, ld n, elimination order, device) to
// backward error <= tol with at most maxit refinement steps.
int refine(mf_handle* h, const double* b, double* x, int nrhs, double tol, int maxit, int* iters, double* eta_out) {
    const int64_t n = h->n;
    const int64_t cap = (int64_t)n * h->nrhs_cap;
    double* R = h->d_iv + 2 * cap;  // [0, 2cap) hold b and x of the caller
    double* Z = R + cap;
    double* Pv = Z + cap;
    double* Q = Pv + cap;
    double* sc = h->d_red + 64;  // CG scalars (80 doubles)
    double eta[16];
    int rc, it = 0;
    double worst = INFINITY;
    if (h->mixed_fallback) {
        // the FP32 factorization failed: the FP64 factor is on the device
        MF_CUDA(cudaMemcpyAsync(h->d_C, b, sizeof(double) * n * nrhs, cudaMemcpyDeviceToDevice, h->stream));
        if ((rc = launch_solve(h, nrhs))) return rc;
        MF_CUDA(cudaMemcpyAsync(x, h->d_C, sizeof(double) * n * nrhs, cudaMemcpyDeviceToDevice, h->stream));
        if ((rc = backward_error(h, x, b, nullptr, nrhs, eta))) return rc;
        worst = 0.0;
        for (int r = 0; r < nrhs; ++r) worst = std::max(worst, eta[r]);
        if (iters) *iters = 1;
        if (eta_out) *eta_out = worst;
        return 0;
    }
    if (!h->diag) {
        // preconditioned conjugate gradients; with row segments (a batch of
        // independent matrices) every segment has its own CG scalars, so each
        // matrix follows its own CG recurrence
        const bool seg = h->nseg > 1;
        const unsigned sgrid = (unsigned)((std::max<int64_t>(h->nseg, 1) * 16 + 255) / 256);
        auto dotv = [&](const double* u, const double* v, int off) -> int {
            return seg ? dot_seg(h, u, v, off, nrhs) : dot(h, u, v, sc + off, nrhs);
        };
        auto scalars = [&](int mode) -> int {
            if (seg) launch_k(k_cg_scalars_seg, sgrid, 256, 0, h->stream, h->d_segsc, h->nseg, nrhs, mode);
            else launch_k(k_cg_scalars, 1, 32, 0, h->stream, sc, nrhs, mode);
            MF_CUDA(cudaGetLastError());
            return 0;
        };
        MF_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n * nrhs, h->stream));
        MF_CUDA(cudaMemcpyAsync(R, b, sizeof(double) * n * nrhs, cudaMemcpyDeviceToDevice, h->stream));
        if ((rc = apply_prec<false>(h, R, Z, nrhs))) return rc;
        MF_CUDA(cudaMemcpyAsync(Pv, Z, sizeof(double) * n * nrhs, cudaMemcpyDeviceToDevice, h->stream));
        if ((rc = dotv(R, Z, 0))) return rc;  // rz
        for (it = 1; it <= maxit; ++it) {
            {
                Timer tm(h, K_SPMV);
                launch_k(k_spmv, row_blocks(n), 256, 0, h->stream, h->d_csrptr, h->d_csrcol, h->d_csrsrc, h->cur_nz, Pv, Q,
                                                              n, nrhs);
                MF_CUDA(cudaGetLastError());
            }
            if ((rc = dotv(Pv, Q, 16))) return rc;  // pq
            if ((rc = scalars(0))) return rc;
            if (seg)
                launch_k(k_cg_xr_seg, gs_blocks(n * nrhs), 256, 0, h->stream, x, R, Pv, Q, h->d_segsc, h->d_rowseg, n,
                                                                        nrhs);
            else
                launch_k(k_cg_xr, gs_blocks(n * nrhs), 256, 0, h->stream, x, R, Pv, Q, sc + 32, n, nrhs);
            MF_CUDA(cudaGetLastError());
            if ((rc = backward_error(h, x, b, nullptr, nrhs, eta))) return rc;
            worst = 0.0;
            for (int r = 0; r < nrhs; ++r) worst = std::max(worst, eta[r]);
            if (worst <= tol || it == maxit) break;
            if ((rc = apply_prec<false>(h, R, Z, nrhs))) return rc;
            if ((rc = dotv(R, Z, 48))) return rc;  // rz_new
            if ((rc = scalars(1))) return rc;
            if (seg)
                launch_k(k_cg_p_seg, gs_blocks(n * nrhs), 256, 0, h->stream, Pv, Z, h->d_segsc, h->d_rowseg, n, nrhs);
            else
                launch_k(k_cg_p, gs_blocks(n * nrhs), 256, 0, h->stream, Pv, Z, sc + 64, n, nrhs);
            MF_CUDA(cudaGetLastError());
        }
    } else {
        return gmres(h, b, x, nrhs, tol, maxit, iters, eta_out);
    }
    if (iters) *iters = it;
    if (eta_out) *eta_out = worst;
    return 0;
}

}  // namespace mf
