// Tensor-core (tcgen05, sm_100a) tile GEMM for the single-precision fronts.
//
// acc(128 x TN) = A(128 x K) * B(TN x K)^T with A, B read from the FP32
// panels by TMA and multiplied on the 5th-generation tensor cores in TF32
// with the accumulator in tensor memory (TMEM).  Each FP32 operand x is
// split into hi = x rounded to TF32 and lo = x - hi (rounded to TF32), and
// the product is accumulated as hi*hi + hi*lo + lo*hi ("3xTF32"), which
// keeps the factor close to FP32 accuracy so the FP64 refinement converges
// in a few steps.
//
// Data path per CTA (256 threads, one output tile):
//   * thread 0 issues cp.async.bulk.tensor 2D loads (no swizzle) of
//     32-row x KC-column boxes of the column-major panel into a ring of
//     NRAW raw stages; a box lands as [k][32 rows] (rows contiguous);
//   * all threads wait on the stage's mbarrier and convert it into one of
//     NOP operand stages: 4 consecutive k of one row are read (conflict-free
//     across a warp: consecutive rows), scaled by the LDLt pivots where the
//     role needs A*D, split into hi/lo and stored as one 16-byte row of an
//     8-row core matrix of the canonical K-major no-swizzle UMMA layout
//     (core matrices 128 B apart along M/N, (rows/8)*128 B apart along K);
//     `kind::tf32` takes K-major operands only, so this conversion is also
//     the transpose;
//   * thread 0 issues 3 tcgen05.mma per K slice of 8, commits them to the
//     operand stage's mbarrier and refills the raw stage it just released,
//     so TMA, the conversion of chunk c+1 and the MMAs of chunk c overlap.
// Tiles start on a 4-row boundary (a TMA box must start on 16 bytes): a
// tile whose first wanted row is not aligned starts at the aligned row below
// it and the epilogue drops the extra rows.  The epilogue reads TMEM with
// tcgen05.ld (warp w owns TMEM lanes 32(w%4).. and column half w/4) and
// applies C -= acc (or C = acc / d for the TRSM role).  Every mbarrier wait
// is bounded by %globaltimer; a timeout sets an error flag, waits (bounded)
// for the loads and MMAs in flight, frees the TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "mf_internal.cuh"

namespace mf {

namespace tc {

constexpr int TM = kTM;        // 128 tile rows (UMMA M)
constexpr int KC = 32;         // K per pipeline stage (4 UMMA K-slices of 8)
constexpr int NT = 256;        // threads per CTA
constexpr int BOX_BYTES = 32 * KC * 4;  // one 32-row raw box: 4 KB
constexpr unsigned long long kWaitNs = 2000000000ull;  // 2 s bound on any wait

template <int TN>
struct Cfg {
    static constexpr int A_BYTES = TM * KC * 4;  // 16 KB
    static constexpr int B_BYTES = TN * KC * 4;
    static constexpr int RAW_BYTES = A_BYTES + B_BYTES;           // one raw stage (TMA destination)
    static constexpr int OP_BYTES = 2 * A_BYTES + 2 * B_BYTES;    // one operand stage (hi + lo of A and B)
    static constexpr int NRAW = TN == 64 ? 4 : 3;
    static constexpr int NOP = 2;
    static constexpr int RING_BYTES = NRAW * RAW_BYTES + NOP * OP_BYTES;
    static constexpr int SMEM_BYTES = RING_BYTES + 512 /* barriers, pivots, TMEM slot */ + 128 /* alignment */;
    static constexpr uint32_t TX_BYTES = (uint32_t)RAW_BYTES;  // bytes the TMA writes per stage
    static constexpr uint32_t TMEM_COLS = TN;
    static constexpr uint32_t LBO_A = (TM / 8) * 128;  // K-adjacent core matrices
    static constexpr uint32_t LBO_B = (TN / 8) * 128;
    // instruction descriptor: D F32, A/B TF32, both K-major, M = 128, N = TN
    static constexpr uint32_t IDESC =
        (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
};
static_assert(Cfg<128>::SMEM_BYTES <= 232448, "tensor-core SYRK tile exceeds the shared-memory limit");
static_assert(Cfg<64>::SMEM_BYTES <= 232448, "tensor-core tile exceeds the shared-memory limit");

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
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
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer();
    while (!mbar_try_wait(bar, parity)) {
        if (globaltimer() - t0 > kWaitNs) return false;
    }
    return true;
}

// 2D tiled TMA load of one 32 x KC box (x = row, y = column) into shared memory
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// Shared-memory matrix descriptor, K-major without swizzle: LBO = stride
// between K-adjacent core matrices, SBO = stride between M/N-adjacent ones.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    return d;                // base offset 0, layout type 0 (no swizzle)
}

template <int TN>
__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(Cfg<TN>::IDESC), "r"(acc)
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

__device__ __forceinline__ uint32_t f2tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// Convert ROWS rows x KC columns of a raw stage ([row/32][k][row%32]) into
// the hi/lo K-major operand tiles.  Columns k >= kc are zero; when dsc is
// given, column k is scaled by dsc[k] first.
template <int ROWS>
__device__ __forceinline__ void convert(const float* __restrict__ raw, uint32_t* __restrict__ hi,
                                        uint32_t* __restrict__ lo, int kc, const float* __restrict__ dsc) {
#pragma unroll 2
    for (int i = threadIdx.x; i < ROWS * (KC / 4); i += NT) {
        const int m = i % ROWS, kq = i / ROWS;
        const float* src = raw + (m >> 5) * (32 * KC) + (kq * 4) * 32 + (m & 31);
        float x[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int k = kq * 4 + e;
            float v = k < kc ? src[e * 32] : 0.f;
            if (dsc && k < kc) v *= dsc[k];
            x[e] = v;
        }
        uint4 vh, vl;
        vh.x = f2tf32(x[0]);
        vh.y = f2tf32(x[1]);
        vh.z = f2tf32(x[2]);
        vh.w = f2tf32(x[3]);
        vl.x = f2tf32(x[0] - __uint_as_float(vh.x));
        vl.y = f2tf32(x[1] - __uint_as_float(vh.y));
        vl.z = f2tf32(x[2] - __uint_as_float(vh.z));
        vl.w = f2tf32(x[3] - __uint_as_float(vh.w));
        const int off = (kq * (ROWS / 8) + (m >> 3)) * 32 + (m & 7) * 4;  // 32-bit words
        *reinterpret_cast<uint4*>(hi + off) = vh;
        *reinterpret_cast<uint4*>(lo + off) = vl;
    }
}

}  // namespace tc

enum TcRole { TC_LEFT = 0, TC_TRAIL = 1, TC_SYRK = 2, TC_TRSM = 3 };

template <int ROLE>
struct TcTileN {
    static constexpr int value = ROLE == TC_SYRK ? kTcSyrkN : kTile;
};

template <int ROLE, int LDLT>
__global__ void __launch_bounds__(tc::NT) k_gemm_tc(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                    int ob, int c0, float* __restrict__ P, float* __restrict__ M,
                                                    const float* __restrict__ d,
                                                    const CUtensorMap* __restrict__ maps,
                                                    const CUtensorMap* __restrict__ inv_map, int* __restrict__ err) {
    using namespace tc;
    constexpr int TN = TcTileN<ROLE>::value;
    using C_ = Cfg<TN>;
    constexpr int NRAW = C_::NRAW, NOP = C_::NOP;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base = smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127);
    unsigned char* raw_base = base;
    unsigned char* op_base = base + NRAW * C_::RAW_BYTES;
    uint64_t* full = reinterpret_cast<uint64_t*>(base + C_::RING_BYTES);  // raw stage landed
    uint64_t* opfree = full + NRAW;                                        // MMAs done with an operand stage
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(opfree + NOP);
    float* scl = reinterpret_cast<float*>(base + C_::RING_BYTES + 256);    // 64 reciprocal pivots (TRSM, LDLt)

    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, na = f.na, nj = nn + na, ld = f.ldp;
    float* Pj = P + f.poff;
    const float* dj = LDLT ? d + f.col0 : nullptr;
    const int tid = threadIdx.x, warp = tid >> 5;
    const CUtensorMap* amap = maps + it.front;
    const CUtensorMap* bmap = amap;

    // tile geometry: TMA rows xa (A) and xb (B); K range [kbeg, kend) of
    // map columns (A at ka0 + k, B at kb0 + k); C coordinates of tile row 0
    // / column 0 are (orow, ocol); valid C range rows [rlo, rhi) x columns
    // [clo, chi); lower triangle only if tri.
    int xa, xb, kbeg, kend, ka0, kb0, orow, ocol, rlo, rhi, clo, chi;
    bool tri;
    float* C;
    int64_t ldc;
    if (ROLE == TC_LEFT) {
        const int w = min(kNB, nn - c0);
        xa = c0 + it.a * TM; xb = c0;
        kbeg = ob * kOB; kend = c0; ka0 = kb0 = 0;
        orow = xa; ocol = c0; rlo = c0; rhi = nj; clo = c0; chi = c0 + w; tri = true;
        C = Pj; ldc = ld;
    } else if (ROLE == TC_TRAIL) {
        const int e = min(nn, (ob + 1) * kOB);
        const int cs = e + it.b * TN;
        xa = cs + it.a * TM; xb = cs;
        kbeg = ob * kOB; kend = e; ka0 = kb0 = 0;
        orow = xa; ocol = cs; rlo = cs; rhi = nj; clo = cs; chi = nn; tri = true;
        C = Pj; ldc = ld;
    } else if (ROLE == TC_SYRK) {
        const int x0 = nn & ~3;            // aligned start at or before the first L21 row
        const int cs = x0 + it.b * TN;     // panel row of tile column 0
        xa = cs + it.a * TM; xb = cs;
        kbeg = 0; kend = nn; ka0 = kb0 = 0;
        orow = xa - nn; ocol = cs - nn; rlo = 0; rhi = na; clo = 0; chi = na; tri = true;
        C = M + f.moff; ldc = f.ldm;
    } else {
        const int w = min(kNB, nn - c0);
        const int r0 = c0 + w;
        xa = (r0 & ~3) + it.a * TM; xb = 0;
        kbeg = 0; kend = w; ka0 = c0;
        kb0 = (int)((f.ioff + (int64_t)(c0 / kNB) * kNB * kNB) / kNB);
        orow = xa; ocol = c0; rlo = r0; rhi = nj; clo = c0; chi = c0 + w; tri = false;
        C = Pj; ldc = ld;
        bmap = inv_map;
    }
    const float* dvec = (LDLT && ROLE != TC_TRSM) ? dj : nullptr;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(C_::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < NRAW; ++s) mbar_init(&full[s], 1);
        for (int s = 0; s < NOP; ++s) mbar_init(&opfree[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (ROLE == TC_TRSM && LDLT) {
        for (int i = tid; i < kNB; i += NT) scl[i] = ocol + i < chi ? 1.f / dj[ocol + i] : 0.f;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    // a TMA box must start on a 16-byte boundary: rows on multiples of 4
    const bool aligned = ((xa | xb) & 3) == 0;
    const int nchunk = aligned ? (kend - kbeg + KC - 1) / KC : 0;
    if (!aligned && tid == 0) atomicExch(err, 2);

    auto raw_ptr = [&](int s) { return raw_base + s * C_::RAW_BYTES; };
    auto op_ptr = [&](int s) { return op_base + s * C_::OP_BYTES; };
    auto issue = [&](int c) {  // thread 0: loads of chunk c into raw stage c % NRAW
        const int s = c % NRAW;
        unsigned char* st = raw_ptr(s);
        const int k = kbeg + c * KC;
        mbar_expect_tx(&full[s], C_::TX_BYTES);
#pragma unroll
        for (int i = 0; i < TM / 32; ++i) tma_load_2d(st + i * BOX_BYTES, amap, xa + 32 * i, ka0 + k, &full[s]);
#pragma unroll
        for (int i = 0; i < TN / 32; ++i)
            tma_load_2d(st + C_::A_BYTES + i * BOX_BYTES, bmap, xb + 32 * i, kb0 + k, &full[s]);
    };

    int issued = 0;  // chunks whose loads thread 0 has issued
    if (tid == 0)
        for (; issued < NRAW && issued < nchunk; ++issued) issue(issued);

    bool bad = false;
    int consumed = 0;   // chunks whose loads every thread has seen land
    int committed = 0;  // chunks whose MMAs thread 0 has committed
    for (int c = 0; c < nchunk; ++c) {
        const int rs = c % NRAW, os = c % NOP;
        bool ok = mbar_wait(&full[rs], (uint32_t)((c / NRAW) & 1));
        if (ok && c >= NOP) ok = mbar_wait(&opfree[os], (uint32_t)(((c - NOP) / NOP) & 1));
        if (__syncthreads_or(!ok)) { bad = true; break; }
        consumed = c + 1;
        const float* raw = reinterpret_cast<const float*>(raw_ptr(rs));
        uint32_t* op = reinterpret_cast<uint32_t*>(op_ptr(os));
        const int kc = min(KC, kend - (kbeg + c * KC));
        convert<TM>(raw, op, op + C_::A_BYTES / 4, kc, dvec ? dvec + kbeg + c * KC : nullptr);
        convert<TN>(raw + C_::A_BYTES / 4, op + 2 * C_::A_BYTES / 4, op + (2 * C_::A_BYTES + C_::B_BYTES) / 4, kc,
                    nullptr);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t ahi = smem_u32(op), alo = ahi + C_::A_BYTES;
            const uint32_t bhi = alo + C_::A_BYTES, blo = bhi + C_::B_BYTES;
            const int nslices = (kc + 7) / 8;
            for (int q = 0; q < nslices; ++q) {
                const uint32_t oa = (uint32_t)(2 * q) * C_::LBO_A, ob_ = (uint32_t)(2 * q) * C_::LBO_B;
                const uint64_t dah = make_desc(ahi + oa, C_::LBO_A, 128);
                const uint64_t dal = make_desc(alo + oa, C_::LBO_A, 128);
                const uint64_t dbh = make_desc(bhi + ob_, C_::LBO_B, 128);
                const uint64_t dbl = make_desc(blo + ob_, C_::LBO_B, 128);
                mma_tf32<TN>(tmem, dah, dbh, (c > 0 || q > 0) ? 1u : 0u);
                mma_tf32<TN>(tmem, dah, dbl, 1u);
                mma_tf32<TN>(tmem, dal, dbh, 1u);
            }
            mma_commit(&opfree[os]);
            committed = c + 1;
            // the raw stage of chunk c has been converted by every thread
            if (issued < nchunk) issue(issued++);
        }
    }
    if (!bad && nchunk > 0) {
        const int last = nchunk - 1;
        bad = !mbar_wait(&opfree[last % NOP], (uint32_t)((last / NOP) & 1));
        bad = __syncthreads_or(bad);
    }
    if (bad) {
        if (tid == 0) {
            atomicExch(err, 1);
            // let the loads and MMAs already in flight finish before the
            // shared buffers and the TMEM go away (each wait bounded)
            for (int c = consumed; c < issued; ++c) (void)mbar_wait(&full[c % NRAW], (uint32_t)((c / NRAW) & 1));
            if (committed > 0)
                (void)mbar_wait(&opfree[(committed - 1) % NOP], (uint32_t)(((committed - 1) / NOP) & 1));
        }
        __syncthreads();
    } else if (nchunk > 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int lw = warp & 3;                 // TMEM lane quarter this warp may read
        const int r = lw * 32 + (tid & 31);
        const int row = orow + r;
        const uint32_t lane_base = tmem + ((uint32_t)(lw * 32) << 16);
        const int cb0 = (warp >> 2) * (TN / 2);  // column half
#pragma unroll
        for (int cb = cb0; cb < cb0 + TN / 2; cb += 16) {
            float v[16];
            tc::tmem_ld16(lane_base + (uint32_t)cb, v);
            if (row >= rlo && row < rhi) {
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int col = ocol + cb + q;
                    if (col >= clo && col < chi && (!tri || row >= col)) {
                        float* p = C + row + (int64_t)col * ldc;
                        if (ROLE == TC_TRSM) *p = LDLT ? v[q] * scl[cb + q] : v[q];
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
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C_::TMEM_COLS)
                     : "memory");
    }
}

template <int ROLE, int LDLT>
static int launch_one(mf_handle* h, const ItemList& l, int ob, int c0, const FactorBufs<float>& fb) {
    if (!l.cnt) return 0;
    constexpr int smem = tc::Cfg<TcTileN<ROLE>::value>::SMEM_BYTES;
    k_gemm_tc<ROLE, LDLT><<<(unsigned)l.cnt, tc::NT, smem, h->stream>>>(
        h->d_fronts, h->d_items + l.off, ob, c0, fb.P, fb.M, fb.d,
        reinterpret_cast<const CUtensorMap*>(h->d_tmaps), reinterpret_cast<const CUtensorMap*>(h->d_tmap_inv),
        h->d_err);
    MF_CUDA(cudaGetLastError());
    return 0;
}

template <int LDLT>
static int set_attrs() {
    constexpr int s64 = tc::Cfg<kTile>::SMEM_BYTES, ss = tc::Cfg<kTcSyrkN>::SMEM_BYTES;
    MF_CUDA(cudaFuncSetAttribute(k_gemm_tc<TC_LEFT, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64));
    MF_CUDA(cudaFuncSetAttribute(k_gemm_tc<TC_TRAIL, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64));
    MF_CUDA(cudaFuncSetAttribute(k_gemm_tc<TC_SYRK, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss));
    MF_CUDA(cudaFuncSetAttribute(k_gemm_tc<TC_TRSM, LDLT>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64));
    return 0;
}

// One 2D tensor map per blocked front over its FP32 panel (rows = nj, the
// contiguous dimension; columns = nn; column stride ldp * 4 bytes), and one
// over the FP32 diagonal-block inverses viewed as 64 x (ninv / 64).  Boxes
// are 32 x KC without swizzle; loads past the extents read zeros.
static int build_maps(mf_handle* h) {
    using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    void* fnp = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    MF_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fnp, cudaEnableDefault, &q));
    if (!fnp || q != cudaDriverEntryPointSuccess) {
        set_error("cuTensorMapEncodeTiled not available from the driver");
        return -3;
    }
    EncodeFn encode = reinterpret_cast<EncodeFn>(fnp);
    const int64_t nex = (int64_t)h->h_fronts.size();
    std::vector<CUtensorMap> maps((size_t)std::max<int64_t>(nex, 1));
    memset(maps.data(), 0, sizeof(CUtensorMap) * maps.size());
    const cuuint32_t box[2] = {32, (cuuint32_t)tc::KC};
    const cuuint32_t estr[2] = {1, 1};
    for (int64_t j = 0; j < nex; ++j) {
        const Front& f = h->h_fronts[(size_t)j];
        if (f.nn + f.na <= kSmallMax) continue;  // small fronts never reach the tensor-core kernels
        const cuuint64_t dims[2] = {(cuuint64_t)(f.nn + f.na), (cuuint64_t)f.nn};
        const cuuint64_t strides[1] = {(cuuint64_t)f.ldp * 4};
        CUresult r = encode(&maps[(size_t)j], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, h->f32.P + f.poff, dims, strides,
                            box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            set_error("cuTensorMapEncodeTiled failed for a front panel (code " + std::to_string((int)r) + ")");
            return -3;
        }
    }
    CUtensorMap inv_map;
    memset(&inv_map, 0, sizeof(inv_map));
    {
        const int64_t cols = std::max<int64_t>(h->ninv / kNB, 1);
        const cuuint64_t dims[2] = {(cuuint64_t)kNB, (cuuint64_t)cols};
        const cuuint64_t strides[1] = {(cuuint64_t)kNB * 4};
        CUresult r = encode(&inv_map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, h->f32.inv, dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            set_error("cuTensorMapEncodeTiled failed for the inverse blocks (code " + std::to_string((int)r) + ")");
            return -3;
        }
    }
    void* dm = nullptr;
    void* di = nullptr;
    MF_CUDA(cudaMalloc(&dm, sizeof(CUtensorMap) * maps.size()));
    cudaError_t e = cudaMalloc(&di, sizeof(CUtensorMap));
    if (e == cudaSuccess) e = cudaMemcpy(dm, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(di, &inv_map, sizeof(CUtensorMap), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(dm);
        if (di) cudaFree(di);
        return cuda_fail(e, "tensor map upload");
    }
    h->d_tmaps = dm;
    h->d_tmap_inv = di;
    h->bytes += (int64_t)(sizeof(CUtensorMap) * (maps.size() + 1));
    return 0;
}

int tc_prepare(mf_handle* h) {
    if (!h->d_tmaps) {
        int rc = build_maps(h);
        if (rc) return rc;
    }
    return h->diag ? set_attrs<1>() : set_attrs<0>();
}

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
