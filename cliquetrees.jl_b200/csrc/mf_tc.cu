// Tensor-core (tcgen05, sm_100a) tile GEMM for the single-precision fronts.
//
// acc(128 x 64) = A(128 x K) * B(64 x K)^T with A, B read from FP32 panels
// and multiplied on the 5th-generation tensor cores in TF32 with the
// accumulator in tensor memory (TMEM).  Each FP32 operand is split into
// hi = tf32(x) and lo = tf32(x - hi) and the product is accumulated as
// hi*hi + hi*lo + lo*hi ("3xTF32"), which keeps the factor close to FP32
// accuracy so the FP64 refinement converges in a few steps.
//
// Per CTA: 128 threads.  All threads stage K chunks of 32 into shared
// memory (register loads, split, 16-byte stores into the canonical K-major
// no-swizzle UMMA layout: 8-row x 16-byte core matrices), one thread issues
// tcgen05.mma and tcgen05.commit to an mbarrier per stage, so loading chunk
// c+1 overlaps the MMAs of chunk c.  The epilogue reads TMEM with
// tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = tile rows) and applies
// C -= acc (or C = acc * scale for the TRSM role).  Every mbarrier wait is
// bounded by %globaltimer; a timeout sets an error flag and the CTA frees
// its TMEM and returns.
#include <cstdint>

#include "mf_internal.cuh"

namespace mf {

namespace tc {

constexpr int TM = kTM;   // 128 tile rows (UMMA M)
constexpr int TN = kTile; // 64 tile columns (UMMA N)
constexpr int KC = 32;    // K per pipeline stage (4 UMMA K-slices of 8)
constexpr int A_BYTES = TM * KC * 4;
constexpr int B_BYTES = TN * KC * 4;
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;  // hi/lo of A and B
constexpr int SMEM_BYTES = 2 * STAGE_BYTES + 1024;       // 2 stages + barriers
constexpr uint32_t TMEM_COLS = 64;
constexpr unsigned long long kWaitNs = 2000000000ull;    // 2 s bound on any wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait on one mbarrier phase; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const unsigned long long t0 = globaltimer();
    while (!mbar_try_wait(bar, parity)) {
        if (globaltimer() - t0 > kWaitNs) return false;
    }
    return true;
}

__device__ __forceinline__ uint32_t f2tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// K-major, no swizzle: SBO = stride between 8-row core matrices along M/N,
// LBO = stride between the two 16-byte K cores of one K=8 slice.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    return d;                // base offset 0, layout type 0 (SWIZZLE_NONE)
}

// instruction descriptor: D F32, A/B TF32, both K-major, M = 128, N = 64
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TN >> 3) << 17) |
                            ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Stage rows [r0, r0 + ROWS) x columns [k, k + kc) of a column-major matrix
// into the hi/lo UMMA tiles (zero outside rmax / kc).  Optionally scale
// column k by dsc[k].
template <int ROWS>
__device__ __forceinline__ void stage(uint32_t* hi, uint32_t* lo, const float* G, int64_t ld, int r0, int rmax, int k,
                                      int kc, const float* dsc) {
    // (row, kcore) pairs; one 16-byte core row each
    for (int i = threadIdx.x; i < ROWS * (KC / 4); i += blockDim.x) {
        const int m = i % ROWS, kcore = i / ROWS;
        float x[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int kk = kcore * 4 + q;
            float v = 0.f;
            if (r0 + m < rmax && kk < kc) {
                v = G[(r0 + m) + (int64_t)(k + kk) * ld];
                if (dsc) v *= dsc[k + kk];
            }
            x[q] = v;
        }
        uint4 vh, vl;
        uint32_t h0 = f2tf32(x[0]), h1 = f2tf32(x[1]), h2 = f2tf32(x[2]), h3 = f2tf32(x[3]);
        vh.x = h0; vh.y = h1; vh.z = h2; vh.w = h3;
        vl.x = f2tf32(x[0] - __uint_as_float(h0));
        vl.y = f2tf32(x[1] - __uint_as_float(h1));
        vl.z = f2tf32(x[2] - __uint_as_float(h2));
        vl.w = f2tf32(x[3] - __uint_as_float(h3));
        const int off = ((kcore * (ROWS / 8) + (m >> 3)) * 128 + (m & 7) * 16) >> 2;  // in 32-bit words
        *reinterpret_cast<uint4*>(hi + off) = vh;
        *reinterpret_cast<uint4*>(lo + off) = vl;
    }
}

}  // namespace tc

enum TcRole { TC_LEFT = 0, TC_TRAIL = 1, TC_SYRK = 2, TC_TRSM = 3 };

template <int ROLE, int LDLT>
__global__ void __launch_bounds__(128) k_gemm_tc(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                 int ob, int c0, float* __restrict__ P, float* __restrict__ M,
                                                 const float* __restrict__ d, const float* __restrict__ inv,
                                                 int* __restrict__ err) {
    using namespace tc;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    uint32_t* st_base = reinterpret_cast<uint32_t*>(smem_raw);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + 2 * STAGE_BYTES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem_raw + 2 * STAGE_BYTES + 64);
    float* scl = reinterpret_cast<float*>(smem_raw + 2 * STAGE_BYTES + 128);  // 64 reciprocal pivots (TRSM, LDLt)

    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp;
    float* Pj = P + f.poff;
    const float* dj = LDLT ? d + f.col0 : nullptr;
    const int tid = threadIdx.x, warp = tid >> 5;

    // operands and target of this tile
    const float* A;
    const float* B;
    int64_t lda, ldb, ldc;
    int ra, amax, rb, bmax, kbeg, kend, rs, cs, rmax, cmax;
    float* C;
    bool diag_tile;
    if (ROLE == TC_LEFT) {
        const int w = min(kNB, nn - c0);
        rs = c0 + it.a * TM; cs = c0;
        A = Pj; lda = ld; ra = rs; amax = nj;
        B = Pj; ldb = ld; rb = c0; bmax = c0 + w;
        kbeg = ob * kOB; kend = c0;
        C = Pj; ldc = ld; rmax = nj - rs; cmax = w; diag_tile = it.a == 0;
    } else if (ROLE == TC_TRAIL) {
        const int e = min(nn, (ob + 1) * kOB);
        cs = e + it.b * TN; rs = cs + it.a * TM;
        A = Pj; lda = ld; ra = rs; amax = nj;
        B = Pj; ldb = ld; rb = cs; bmax = nn;
        kbeg = ob * kOB; kend = e;
        C = Pj; ldc = ld; rmax = nj - rs; cmax = nn - cs; diag_tile = it.a == 0;
    } else if (ROLE == TC_SYRK) {
        cs = it.b * TN; rs = cs + it.a * TM;
        A = Pj + nn; lda = ld; ra = rs; amax = na;
        B = Pj + nn; ldb = ld; rb = cs; bmax = na;
        kbeg = 0; kend = nn;
        C = M + f.moff; ldc = f.ldm; rmax = na - rs; cmax = na - cs; diag_tile = it.a == 0;
    } else {
        const int w = min(kNB, nn - c0);
        rs = c0 + w + it.a * TM; cs = 0;
        A = Pj + (int64_t)c0 * ld; lda = ld; ra = rs; amax = nj;
        B = inv + f.ioff + (int64_t)(c0 / kNB) * kNB * kNB; ldb = kNB; rb = 0; bmax = w;
        kbeg = 0; kend = w;
        C = Pj + (int64_t)c0 * ld; ldc = ld; rmax = nj - rs; cmax = w; diag_tile = false;
    }
    const float* dvec = (LDLT && ROLE != TC_TRSM) ? dj : nullptr;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (ROLE == TC_TRSM && LDLT) {
        for (int i = tid; i < TN; i += blockDim.x) scl[i] = i < cmax ? 1.f / dj[c0 + i] : 0.f;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    bool ok = true;
    const int nchunk = (kend - kbeg + KC - 1) / KC;
    for (int c = 0; c < nchunk && ok; ++c) {
        const int s = c & 1;
        if (c >= 2) ok = mbar_wait(&bar[s], (uint32_t)(((c - 2) >> 1) & 1));
        if (!ok) break;
        uint32_t* ahi = st_base + (s * STAGE_BYTES) / 4;
        uint32_t* alo = ahi + A_BYTES / 4;
        uint32_t* bhi = alo + A_BYTES / 4;
        uint32_t* blo = bhi + B_BYTES / 4;
        const int k = kbeg + c * KC;
        const int kc = min(KC, kend - k);
        stage<TM>(ahi, alo, A, lda, ra, amax, k, kc, dvec);
        stage<TN>(bhi, blo, B, ldb, rb, bmax, k, kc, nullptr);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int nslices = (kc + 7) / 8;
            for (int q = 0; q < nslices; ++q) {
                // K slice q = K cores 2q, 2q+1
                const uint32_t a_off = (uint32_t)(2 * q) * (TM / 8) * 128;
                const uint32_t b_off = (uint32_t)(2 * q) * (TN / 8) * 128;
                const uint64_t dah = make_desc(smem_u32(ahi) + a_off, (TM / 8) * 128, 128);
                const uint64_t dal = make_desc(smem_u32(alo) + a_off, (TM / 8) * 128, 128);
                const uint64_t dbh = make_desc(smem_u32(bhi) + b_off, (TN / 8) * 128, 128);
                const uint64_t dbl = make_desc(smem_u32(blo) + b_off, (TN / 8) * 128, 128);
                mma_tf32(tmem, dah, dbh, (c > 0 || q > 0) ? 1u : 0u);
                mma_tf32(tmem, dah, dbl, 1u);
                mma_tf32(tmem, dal, dbh, 1u);
            }
            mma_commit(&bar[s]);
        }
    }
    if (ok && nchunk > 0) {
        const int last = nchunk - 1;
        ok = mbar_wait(&bar[last & 1], (uint32_t)((last >> 1) & 1));
    }
    if (!ok) {
        if (tid == 0) atomicExch(err, 1);
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int row = warp * 32 + (tid & 31);
        const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
        for (int cb = 0; cb < TN; cb += 16) {
            float v[16];
            tc::tmem_ld16(lane_base + (uint32_t)cb, v);
            if (row < rmax) {
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int col = cb + q;
                    if (col < cmax && (!diag_tile || rs + row >= cs + col)) {
                        float* p = C + (rs + row) + (int64_t)(cs + col) * ldc;
                        if (ROLE == TC_TRSM) *p = LDLT ? v[q] * scl[col] : v[q];
                        else *p -= v[q];
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

template <int ROLE, int LDLT>
static int launch_one(mf_handle* h, const ItemList& l, int ob, int c0, const FactorBufs<float>& fb) {
    if (!l.cnt) return 0;
    k_gemm_tc<ROLE, LDLT><<<(unsigned)l.cnt, 128, tc::SMEM_BYTES, h->stream>>>(
        h->d_fronts, h->d_items + l.off, ob, c0, fb.P, fb.M, fb.d, fb.inv, h->d_err);
    MF_CUDA(cudaGetLastError());
    return 0;
}

template <int LDLT>
static int set_attrs() {
    MF_CUDA(cudaFuncSetAttribute(k_gemm_tc<TC_LEFT, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES));
    MF_CUDA(cudaFuncSetAttribute(k_gemm_tc<TC_TRAIL, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES));
    MF_CUDA(cudaFuncSetAttribute(k_gemm_tc<TC_SYRK, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES));
    MF_CUDA(cudaFuncSetAttribute(k_gemm_tc<TC_TRSM, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES));
    return 0;
}

int tc_prepare(mf_handle* h) { return h->diag ? set_attrs<1>() : set_attrs<0>(); }

int tc_launch(mf_handle* h, int role, const ItemList& l, int ob, int c0, const FactorBufs<float>& fb) {
    if (h->diag) {
        switch (role) {
            case TC_LEFT: return launch_one<TC_LEFT, 1>(h, l, ob, c0, fb);
            case TC_TRAIL: return launch_one<TC_TRAIL, 1>(h, l, ob, c0, fb);
            case TC_SYRK: return launch_one<TC_SYRK, 1>(h, l, ob, c0, fb);
            default: return launch_one<TC_TRSM, 1>(h, l, ob, c0, fb);
        }
    }
    switch (role) {
        case TC_LEFT: return launch_one<TC_LEFT, 0>(h, l, ob, c0, fb);
        case TC_TRAIL: return launch_one<TC_TRAIL, 0>(h, l, ob, c0, fb);
        case TC_SYRK: return launch_one<TC_SYRK, 0>(h, l, ob, c0, fb);
        default: return launch_one<TC_TRSM, 0>(h, l, ob, c0, fb);
    }
}

}  // namespace mf
