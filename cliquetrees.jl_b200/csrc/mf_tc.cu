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
// Persistent and warp-specialised: a CTA (one per SM) walks the launch's
// tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...; its warps form a
// pipeline connected by mbarriers:
//   * warp 16 (one lane) issues cp.async.bulk.tensor 2D loads (no swizzle)
//     of 32-row x KC-column boxes of the column-major panel into a ring of
//     NRAW raw stages; a box lands as [k][32 rows] (rows contiguous);
//   * warps 8..15 convert a raw stage into one of NOP operand stages: 4
//     consecutive k of one row are read (conflict-free across a warp:
//     consecutive rows), scaled by the LDLt pivots where the role needs A*D,
//     split into hi/lo and stored as one 16-byte row of an 8-row core matrix
//     of the canonical K-major no-swizzle UMMA layout (core matrices 128 B
//     apart along M/N, (rows/8)*128 B apart along K); `kind::tf32` takes
//     K-major operands only, so this conversion is also the transpose;
//   * warp 17 (one lane) issues 3 tcgen05.mma per K slice of 8 into one of
//     two TMEM accumulators and commits each operand stage back to the
//     converters and each finished tile to the epilogue;
//   * warps 0..7 (warp w reads TMEM lanes 32(w%4).. = tile rows, column
//     half w/4) load the C tile into registers while its MMAs run, then read
//     the finished accumulator with tcgen05.ld and store C - acc (or
//     acc / d for the TRSM role) while the next tile is multiplied.
// Tiles start on a 4-row boundary (a TMA box must start on 16 bytes): a
// tile whose first wanted row is not aligned starts at the aligned row below
// it and the epilogue drops the extra rows.  Every mbarrier wait is bounded
// by %globaltimer and by a shared abort flag; a timeout sets the error flag
// and every role drains what it has in flight (each wait bounded) before the
// TMEM is freed.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "mf_internal.cuh"

namespace mf {

namespace tc {

#ifndef MF_TC_TERMS
#define MF_TC_TERMS 3  // products per K slice: hi*hi + hi*lo + lo*hi
#endif

constexpr int TM = kTM;        // 128 tile rows (UMMA M)
constexpr int KC = 32;         // K per pipeline stage (4 UMMA K-slices of 8)
constexpr int NEPI = 8;        // epilogue warps 0..7 (warp w: TMEM lane quarter w % 4, column half w / 4)
constexpr int NCONV = 8;       // converter warps 8..15
constexpr int WTMA = 16;       // TMA producer warp
constexpr int WMMA = 17;       // MMA issuer warp (also allocates the TMEM)
constexpr int NT = 18 * 32;    // threads per CTA
constexpr int CT = NCONV * 32; // converter threads
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
    static constexpr int SMEM_BYTES = RING_BYTES + 256 /* barriers, TMEM slot, abort flag */ + 128 /* alignment */;
    static constexpr uint32_t TX_BYTES = (uint32_t)RAW_BYTES;  // bytes the TMA writes per stage
    static constexpr uint32_t TMEM_COLS = 2 * TN;              // two accumulators
    static constexpr uint32_t LBO_A = (TM / 8) * 128;  // K-adjacent core matrices
    static constexpr uint32_t LBO_B = (TN / 8) * 128;
    // instruction descriptor: D F32, A/B TF32, both K-major, M = 128, N = TN
    static constexpr uint32_t IDESC =
        (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
};
// Pre-split operands (SPLIT): no raw stages, three operand stages filled by
// bulk copies of the pre-split units
template <int TN>
struct SplitCfg {
    static constexpr int NOP = 3;
    static constexpr int RING_BYTES = NOP * Cfg<TN>::OP_BYTES;
    static constexpr int SMEM_BYTES = RING_BYTES + 256 + 128;
};
static_assert(SplitCfg<128>::SMEM_BYTES <= 232448, "split tensor-core tile exceeds the shared-memory limit");
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

// try_wait that lets the hardware suspend the thread (up to `hint_ns`)
// until the phase completes, so waiting warps do not take issue slots from
// the working ones
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}

// bounded wait on one mbarrier phase; false on timeout or once *abort is set
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, const volatile int* abort) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer();
    while (!mbar_try_wait_sleep(bar, parity, 20000u)) {
        if (*abort || globaltimer() - t0 > kWaitNs) return false;
    }
    return true;
}

// bounded wait that ignores the abort flag: used to drain copies and MMAs
// still in flight before the CTA exits
__device__ __forceinline__ bool mbar_drain(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer();
    while (!mbar_try_wait_sleep(bar, parity, 20000u)) {
        if (globaltimer() - t0 > kWaitNs) return false;
    }
    return true;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 2D tiled TMA load of one 32 x KC box (x = row, y = column) into shared memory
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// non-tensor bulk copy of `bytes` contiguous bytes global -> shared (both
// 16-byte aligned, bytes a multiple of 16), completing on an mbarrier
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
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

// x rounded to TF32 (10 explicit mantissa bits, ties away from zero) with
// integer operations: adding half a TF32 unit to the magnitude bits and
// clearing the 13 dropped bits.  Finite inputs only.  Integer ALU work keeps
// the split off the conversion pipe, which would otherwise limit the MMAs.
__device__ __forceinline__ uint32_t f2tf32(float x) { return (__float_as_uint(x) + 0x1000u) & 0xFFFFE000u; }

// Convert ROWS rows x KC columns of a raw stage ([row/32][k][row%32]) into
// the hi/lo K-major operand tiles.  Columns k >= kc are zero; when dsc is
// given, column k is scaled by dsc[k] first.
template <int ROWS>
__device__ __forceinline__ void convert(int ct, const float* __restrict__ raw, uint32_t* __restrict__ hi,
                                        uint32_t* __restrict__ lo, int kc, const float* __restrict__ dsc) {
#pragma unroll 2
    for (int i = ct; i < ROWS * (KC / 4); i += CT) {
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
    static constexpr int value = ROLE == TC_SYRK ? kTcSyrkN : ROLE == TC_TRAIL ? kTcTrailN : kTile;
};

// Geometry of one tile: TMA rows xa (A) and xb (B); K range [kbeg, kend)
// of map columns (A at ka0 + k, B at kb0 + k); C coordinates of tile row 0
// / column 0 are (orow, ocol); valid C range rows [rlo, rhi) x columns
// [clo, chi); lower triangle only if tri.
struct TileGeom {
    int xa, xb, kbeg, kend, ka0, kb0, orow, ocol, rlo, rhi, clo, chi, nchunk, front;
    bool tri;
    float* C;
    int64_t ldc;
};

template <int ROLE>
__device__ __forceinline__ TileGeom tile_geom(const Front* __restrict__ fronts, const Item& it, int obs, int obw, int c0,
                                              float* P, float* M) {
    constexpr int TN = TcTileN<ROLE>::value;
    const Front f = fronts[it.front];
    const int nn = f.nn, na = f.na, nj = nn + na;
    TileGeom g;
    g.front = it.front;
    if (ROLE == TC_LEFT) {
        const int w = min(kNB, nn - c0);
        g.xa = c0 + it.a * tc::TM; g.xb = c0;
        g.kbeg = obs; g.kend = c0; g.ka0 = g.kb0 = 0;
        g.orow = g.xa; g.ocol = c0; g.rlo = c0; g.rhi = nj; g.clo = c0; g.chi = c0 + w; g.tri = true;
        g.C = P + f.poff; g.ldc = f.ldp;
    } else if (ROLE == TC_TRAIL) {
        const int e = min(nn, obs + obw);
        const int cs = e + it.b * TN;
        g.xa = cs + it.a * tc::TM; g.xb = cs;
        g.kbeg = obs; g.kend = e; g.ka0 = g.kb0 = 0;
        g.orow = g.xa; g.ocol = cs; g.rlo = cs; g.rhi = nj; g.clo = cs; g.chi = nn; g.tri = true;
        g.C = P + f.poff; g.ldc = f.ldp;
    } else if (ROLE == TC_SYRK) {
        const int x0 = nn & ~3;            // aligned start at or before the first L21 row
        const int cs = x0 + it.b * TN;     // panel row of tile column 0
        g.xa = cs + it.a * tc::TM; g.xb = cs;
        g.kbeg = 0; g.kend = nn; g.ka0 = g.kb0 = 0;
        g.orow = g.xa - nn; g.ocol = cs - nn; g.rlo = 0; g.rhi = na; g.clo = 0; g.chi = na; g.tri = true;
        g.C = M + f.moff; g.ldc = f.ldm;
    } else {
        const int w = min(kNB, nn - c0);
        const int r0 = c0 + w;
        g.xa = (r0 & ~3) + it.a * tc::TM; g.xb = 0;
        g.kbeg = 0; g.kend = w; g.ka0 = c0;
        g.kb0 = (int)((f.ioff + (int64_t)(c0 / kNB) * kNB * kNB) / kNB);
        g.orow = g.xa; g.ocol = c0; g.rlo = r0; g.rhi = nj; g.clo = c0; g.chi = c0 + w; g.tri = false;
        g.C = P + f.poff; g.ldc = f.ldp;
    }
    // a TMA box must start on a 16-byte boundary: rows on multiples of 4
    const bool aligned = ((g.xa | g.xb) & 3) == 0;
    g.nchunk = aligned ? (g.kend - g.kbeg + tc::KC - 1) / tc::KC : 0;
    return g;
}

// SPLIT: the operands come pre-split (k_tc_split) in 32 KB units of hi and
// lo tiles already in the operand layout, so the producer bulk-copies a
// unit of A and one of B into an operand stage and the converter warps idle
// (TRAIL and SYRK only: their row blocks line up with the units).
template <int ROLE, int LDLT, bool SPLIT>
__global__ void __launch_bounds__(tc::NT, 1) k_gemm_tc(const Front* __restrict__ fronts,
                                                       const Item* __restrict__ items, int64_t ntiles, int obs, int obw, int c0,
                                                       float* __restrict__ P, float* __restrict__ M,
                                                       const float* __restrict__ d,
                                                       const CUtensorMap* __restrict__ maps,
                                                       const CUtensorMap* __restrict__ inv_map,
                                                       const float* __restrict__ split, int* __restrict__ err) {
    pdl_prologue();
    using namespace tc;
    constexpr int TN = TcTileN<ROLE>::value;
    using C_ = Cfg<TN>;
    static_assert(!SPLIT || (TN == kSplitRows && TM == kSplitRows && KC == kSplitK),
                  "pre-split units are 128 rows x 32 columns");
    constexpr int NRAW = SPLIT ? 0 : C_::NRAW;
    constexpr int NRAWD = NRAW > 0 ? NRAW : 1;  // divisor in the raw-stage code, which SPLIT never runs
    constexpr int NOP = SPLIT ? SplitCfg<TN>::NOP : C_::NOP;
    constexpr int RING = SPLIT ? SplitCfg<TN>::RING_BYTES : C_::RING_BYTES;
    extern __shared__ unsigned char smem_raw[];
    unsigned char* base = smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127);
    unsigned char* raw_base = base;
    unsigned char* op_base = base + NRAW * C_::RAW_BYTES;
    uint64_t* raw_full = reinterpret_cast<uint64_t*>(base + RING);  // TMA landed
    uint64_t* raw_empty = raw_full + NRAW;    // converters done with a raw stage
    uint64_t* op_full = raw_empty + NRAW;     // converters filled an operand stage
    uint64_t* op_empty = op_full + NOP;       // MMAs done with an operand stage
    uint64_t* acc_full = op_empty + NOP;      // accumulator ready for the epilogue
    uint64_t* acc_empty = acc_full + 2;       // epilogue done with an accumulator
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == WMMA) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(C_::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < NRAW; ++s) { mbar_init(&raw_full[s], 1); mbar_init(&raw_empty[s], NCONV); }
        for (int s = 0; s < NOP; ++s) { mbar_init(&op_full[s], SPLIT ? 1 : NCONV); mbar_init(&op_empty[s], 1); }
        for (int s = 0; s < 2; ++s) { mbar_init(&acc_full[s], 1); mbar_init(&acc_empty[s], NEPI); }
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    auto fail = [&](int code) {
        *abort = 1;
        atomicExch(err, code);
    };

    if (SPLIT && warp == WTMA) {
        // ---------------- bulk-copy producer of pre-split units ----------------
        if (lane == 0) {
            int64_t g = 0;
            bool ok = true;
            constexpr int nunit = LDLT ? 2 : 1;
            for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                const Item it = items[t];
                const TileGeom tg = tile_geom<ROLE>(fronts, it, obs, obw, c0, P, M);
                const int nkc = (tg.kend - tg.kbeg + KC - 1) / KC;
                const int64_t ua = it.pad + ((int64_t)(it.a + it.b) * nkc) * nunit + (LDLT ? 1 : 0);
                const int64_t ub = it.pad + ((int64_t)it.b * nkc) * nunit;
                for (int c = 0; c < nkc; ++c, ++g) {
                    const int os = (int)(g % NOP);
                    if (g >= NOP && !mbar_wait(&op_empty[os], (uint32_t)(((g / NOP) - 1) & 1), abort)) {
                        fail(1);
                        ok = false;
                        break;
                    }
                    unsigned char* st = op_base + os * C_::OP_BYTES;
                    mbar_expect_tx(&op_full[os], (uint32_t)C_::OP_BYTES);
                    bulk_load(st, split + (ua + (int64_t)c * nunit) * kSplitUnitFloats, 2 * C_::A_BYTES, &op_full[os]);
                    bulk_load(st + 2 * C_::A_BYTES, split + (ub + (int64_t)c * nunit) * kSplitUnitFloats,
                              2 * C_::B_BYTES, &op_full[os]);
                }
            }
            // drain: the copies of the last stages must land before the CTA exits
            for (int64_t q = (g > NOP ? g - NOP : 0); q < g; ++q)
                (void)mbar_drain(&op_full[q % NOP], (uint32_t)((q / NOP) & 1));
        }
    } else if (warp == WTMA) {
        // ---------------- TMA producer ----------------
        if (lane == 0) {
            int64_t g = 0;  // chunks issued by this CTA
            bool ok = true;
            for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                const Item it = items[t];
                const TileGeom tg = tile_geom<ROLE>(fronts, it, obs, obw, c0, P, M);
                if (tg.nchunk == 0) { fail(2); ok = false; break; }
                const CUtensorMap* amap = maps + it.front;
                const CUtensorMap* bmap = ROLE == TC_TRSM ? inv_map : amap;
                for (int c = 0; c < tg.nchunk; ++c, ++g) {
                    const int s = (int)(g % NRAWD);
                    if (g >= NRAWD && !mbar_wait(&raw_empty[s], (uint32_t)(((g / NRAWD) - 1) & 1), abort)) {
                        fail(1);
                        ok = false;
                        break;
                    }
                    unsigned char* st = raw_base + s * C_::RAW_BYTES;
                    const int k = tg.kbeg + c * KC;
                    mbar_expect_tx(&raw_full[s], C_::TX_BYTES);
#pragma unroll
                    for (int i = 0; i < TM / 32; ++i)
                        tma_load_2d(st + i * BOX_BYTES, amap, tg.xa + 32 * i, tg.ka0 + k, &raw_full[s]);
#pragma unroll
                    for (int i = 0; i < TN / 32; ++i)
                        tma_load_2d(st + C_::A_BYTES + i * BOX_BYTES, bmap, tg.xb + 32 * i, tg.kb0 + k, &raw_full[s]);
                }
            }
            // drain: the last NRAW stages' loads must land before the CTA exits
            for (int64_t q = (g > NRAWD ? g - NRAWD : 0); q < g; ++q)
                (void)mbar_drain(&raw_full[q % NRAWD], (uint32_t)((q / NRAWD) & 1));
        }
    } else if (warp >= NEPI && warp < NEPI + NCONV) {
        // ---------------- converters (idle when the operands come pre-split) ----------------
        if (!SPLIT) {
        const int ct = tid - NEPI * 32;
        int64_t g = 0;
        for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const Item it = items[t];
            const TileGeom tg = tile_geom<ROLE>(fronts, it, obs, obw, c0, P, M);
            const float* dvec = (LDLT && ROLE != TC_TRSM) ? d + fronts[it.front].col0 : nullptr;
            bool ok = true;
            for (int c = 0; c < tg.nchunk; ++c, ++g) {
                const int rs = (int)(g % NRAWD), os = (int)(g % NOP);
                ok = mbar_wait(&raw_full[rs], (uint32_t)((g / NRAWD) & 1), abort);
                if (ok && g >= NOP) ok = mbar_wait(&op_empty[os], (uint32_t)(((g / NOP) - 1) & 1), abort);
                if (!__all_sync(0xffffffffu, ok)) { ok = false; break; }
                const float* raw = reinterpret_cast<const float*>(raw_base + rs * C_::RAW_BYTES);
                uint32_t* op = reinterpret_cast<uint32_t*>(op_base + os * C_::OP_BYTES);
                const int kc = min(KC, tg.kend - (tg.kbeg + c * KC));
                convert<TM>(ct, raw, op, op + C_::A_BYTES / 4, kc, dvec ? dvec + tg.kbeg + c * KC : nullptr);
                convert<TN>(ct, raw + C_::A_BYTES / 4, op + 2 * C_::A_BYTES / 4,
                            op + (2 * C_::A_BYTES + C_::B_BYTES) / 4, kc, nullptr);
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&raw_empty[rs]);
                    mbar_arrive(&op_full[os]);
                }
            }
            if (!ok) { if (lane == 0) fail(1); break; }
        }
        }
    } else if (warp == WMMA) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int64_t g = 0, i = 0;
            bool ok = true;
            for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++i) {
                const Item it = items[t];
                const TileGeom tg = tile_geom<ROLE>(fronts, it, obs, obw, c0, P, M);
                const int a = (int)(i & 1);
                if (i >= 2 && !mbar_wait(&acc_empty[a], (uint32_t)(((i / 2) - 1) & 1), abort)) {
                    fail(1);
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t dt = tmem + (uint32_t)(a * TN);
                for (int c = 0; c < tg.nchunk; ++c, ++g) {
                    const int os = (int)(g % NOP);
                    if (!mbar_wait(&op_full[os], (uint32_t)((g / NOP) & 1), abort)) { fail(1); ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t ahi = smem_u32(op_base + os * C_::OP_BYTES), alo = ahi + C_::A_BYTES;
                    const uint32_t bhi = alo + C_::A_BYTES, blo = bhi + C_::B_BYTES;
                    const int kc = min(KC, tg.kend - (tg.kbeg + c * KC));
                    const int nslices = (kc + 7) / 8;
                    for (int q = 0; q < nslices; ++q) {
                        const uint32_t oa = (uint32_t)(2 * q) * C_::LBO_A, ob_ = (uint32_t)(2 * q) * C_::LBO_B;
                        const uint64_t dah = make_desc(ahi + oa, C_::LBO_A, 128);
                        const uint64_t dal = make_desc(alo + oa, C_::LBO_A, 128);
                        const uint64_t dbh = make_desc(bhi + ob_, C_::LBO_B, 128);
                        const uint64_t dbl = make_desc(blo + ob_, C_::LBO_B, 128);
                        mma_tf32<TN>(dt, dah, dbh, (c > 0 || q > 0) ? 1u : 0u);
#if MF_TC_TERMS > 1
                        mma_tf32<TN>(dt, dah, dbl, 1u);
                        mma_tf32<TN>(dt, dal, dbh, 1u);
#endif
                    }
                    mma_commit(&op_empty[os]);
                }
                if (ok) mma_commit(&acc_full[a]);
            }
            // drain: every MMA issued must finish before the TMEM is freed
            if (g > 0) (void)mbar_drain(&op_empty[(g - 1) % NOP], (uint32_t)(((g - 1) / NOP) & 1));
        }
    } else {
        // ---------------- epilogue (warps 0..7) ----------------
        // C -= acc: the C values of the next tile are loaded into registers
        // while its MMAs run, so the read latency is hidden behind them
        constexpr int HC = TN / 2;  // columns per epilogue thread
        const int quarter = warp & 3, half = warp >> 2;
        int64_t i = 0;
        for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++i) {
            const Item it = items[t];
            const TileGeom tg = tile_geom<ROLE>(fronts, it, obs, obw, c0, P, M);
            const int a = (int)(i & 1);
            const int row = tg.orow + quarter * 32 + lane;
            const int cbase = tg.ocol + half * HC;
            const bool row_ok = row >= tg.rlo && row < tg.rhi;
            // 32-bit offsets: a front's panel and update matrix stay below 2^31 elements
            const int ldc = (int)tg.ldc;
            float* cblk = tg.C + row + (int64_t)cbase * ldc;
            float cv[HC];
            // the SYRK writes M = -L21 L21^T without reading it (the extend-add
            // of the children into M follows it); the panel roles update C
            if (ROLE != TC_TRSM && ROLE != TC_SYRK) {
#pragma unroll
                for (int q = 0; q < HC; ++q) {
                    const int col = cbase + q;
                    const bool valid = row_ok && col >= tg.clo && col < tg.chi && (!tg.tri || row >= col);
                    cv[q] = valid ? __ldcg(cblk + q * ldc) : 0.f;
                }
            }
            const bool ok = mbar_wait(&acc_full[a], (uint32_t)((i / 2) & 1), abort);
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0) fail(1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(a * TN + half * HC);
            const float* dj = (ROLE == TC_TRSM && LDLT) ? d + fronts[it.front].col0 : nullptr;
#pragma unroll
            for (int cb = 0; cb < HC; cb += 16) {
                float v[16];
                tc::tmem_ld16(lane_base + (uint32_t)cb, v);
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int col = cbase + cb + q;
                    if (row_ok && col >= tg.clo && col < tg.chi && (!tg.tri || row >= col)) {
                        float* p = cblk + (cb + q) * ldc;
                        if (ROLE == TC_TRSM) *p = LDLT ? v[q] / dj[col] : v[q];
                        else if (ROLE == TC_SYRK) *p = -v[q];
                        else *p = cv[cb + q] - v[q];
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[a]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == WMMA) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C_::TMEM_COLS)
                     : "memory");
    }
}

template <int ROLE, int LDLT>
static int launch_one(mf_handle* h, const ItemList& l, int obs, int obw, int c0, const FactorBufs<float>& fb) {
    if (!l.cnt) return 0;
    constexpr int smem = tc::Cfg<TcTileN<ROLE>::value>::SMEM_BYTES;
    const int64_t grid = std::min<int64_t>(l.cnt, h->grid_cap > 0 ? h->grid_cap : h->num_sms > 0 ? h->num_sms : 148);
    launch_kx(pdl_enabled() || (h->panel_pdl && (ROLE == 0 || ROLE == 3)), k_gemm_tc<ROLE, LDLT, false>,
              (unsigned)grid, tc::NT, smem, h->stream, 
        h->d_fronts, h->d_items + l.off, l.cnt, obs, obw, c0, fb.P, fb.M, fb.d,
        reinterpret_cast<const CUtensorMap*>(h->d_tmaps), reinterpret_cast<const CUtensorMap*>(h->d_tmap_inv),
        nullptr, h->d_err);
    MF_CUDA(cudaGetLastError());
    return 0;
}

// One CTA per unit (front, 128-row block, 32-column chunk): the panel's rows
// R0 + 128 rb .. and columns K0 + 32 kc .. (zero past the front's rows and
// the role's K range) split into TF32 hi / lo in the operand layout of the
// tensor-core kernel (convert<>'s), unit by unit; LDLt writes a second unit
// with the columns scaled by the pivots (the A operand of L D L^T).
// TRAIL: rows from the outer block's end e = min(nn, obs + obw), K = [obs, e);
// SYRK: rows from nn & ~3, K = [0, nn).
template <int LDLT, int SYRK>
__global__ void __launch_bounds__(256) k_tc_split(const Front* __restrict__ fronts, const Item* __restrict__ items,
                                                  int obs, int obw, const float* __restrict__ P,
                                                  const float* __restrict__ d, float* __restrict__ split) {
    pdl_prologue();
    const Item it = items[blockIdx.x];
    const Front f = fronts[it.front];
    const int nn = f.nn, nj = nn + f.na, ld = f.ldp;
    int R0, K0, Kend;
    if (SYRK) {
        R0 = nn & ~3; K0 = 0; Kend = nn;
    } else {
        const int e = min(nn, obs + obw);
        R0 = e; K0 = obs; Kend = e;
    }
    const int nkc = (Kend - K0 + kSplitK - 1) / kSplitK;
    const int m = threadIdx.x & (kSplitRows - 1), kh = threadIdx.x >> 7;
    const int r = R0 + it.a * kSplitRows + m;
    const int kb = K0 + it.b * kSplitK + 16 * kh;
    const float* Pj = P + f.poff;
    float x[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
        const int k = kb + u;
        x[u] = (r < nj && k < Kend) ? Pj[r + (int64_t)k * ld] : 0.f;
    }
    constexpr int nunit = LDLT ? 2 : 1;
#pragma unroll
    for (int v = 0; v < nunit; ++v) {
        uint32_t* U = reinterpret_cast<uint32_t*>(split) +
                      ((int64_t)it.pad + ((int64_t)it.a * nkc + it.b) * nunit + v) * kSplitUnitFloats;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float y[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int k = kb + 4 * q + e;
                y[e] = x[4 * q + e];
                if (v == 1 && k < Kend) y[e] *= d[f.col0 + k];
            }
            uint4 vh, vl;
            vh.x = tc::f2tf32(y[0]);
            vh.y = tc::f2tf32(y[1]);
            vh.z = tc::f2tf32(y[2]);
            vh.w = tc::f2tf32(y[3]);
            vl.x = tc::f2tf32(y[0] - __uint_as_float(vh.x));
            vl.y = tc::f2tf32(y[1] - __uint_as_float(vh.y));
            vl.z = tc::f2tf32(y[2] - __uint_as_float(vh.z));
            vl.w = tc::f2tf32(y[3] - __uint_as_float(vh.w));
            const int kq = 4 * kh + q;
            const int off = (kq * (kSplitRows / 8) + (m >> 3)) * 32 + (m & 7) * 4;  // 32-bit words
            *reinterpret_cast<uint4*>(U + off) = vh;
            *reinterpret_cast<uint4*>(U + kSplitRows * kSplitK + off) = vl;
        }
    }
}

template <int ROLE, int LDLT>
static int launch_split(mf_handle* h, const ItemList& l, const ItemList& units, int obs, int obw, int c0,
                        const FactorBufs<float>& fb) {
    if (!l.cnt) return 0;
    if (units.cnt) {
        launch_k(k_tc_split<LDLT, ROLE == TC_SYRK>, (unsigned)units.cnt, 256, 0, h->stream, 
            h->d_fronts, h->d_items + units.off, obs, obw, fb.P, fb.d, h->f32.split);
        MF_CUDA(cudaGetLastError());
    }
    constexpr int smem = tc::SplitCfg<TcTileN<ROLE>::value>::SMEM_BYTES;
    const int64_t grid = std::min<int64_t>(l.cnt, h->grid_cap > 0 ? h->grid_cap : h->num_sms > 0 ? h->num_sms : 148);
    launch_k(k_gemm_tc<ROLE, LDLT, true>, (unsigned)grid, tc::NT, smem, h->stream, 
        h->d_fronts, h->d_items + l.off, l.cnt, obs, obw, c0, fb.P, fb.M, fb.d,
        reinterpret_cast<const CUtensorMap*>(h->d_tmaps), reinterpret_cast<const CUtensorMap*>(h->d_tmap_inv),
        h->f32.split, h->d_err);
    MF_CUDA(cudaGetLastError());
    return 0;
}

template <int LDLT>
static int set_attrs() {
    constexpr int s64 = tc::Cfg<kTile>::SMEM_BYTES, ss = tc::Cfg<kTcSyrkN>::SMEM_BYTES;
    constexpr int st = tc::Cfg<kTcTrailN>::SMEM_BYTES;
    MF_CUDA(cudaFuncSetAttribute(k_gemm_tc<TC_LEFT, LDLT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64));
    MF_CUDA(cudaFuncSetAttribute(k_gemm_tc<TC_TRAIL, LDLT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, st));
    MF_CUDA(cudaFuncSetAttribute(k_gemm_tc<TC_SYRK, LDLT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss));
    MF_CUDA(cudaFuncSetAttribute(k_gemm_tc<TC_TRSM, LDLT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s64));
    constexpr int sp = tc::SplitCfg<128>::SMEM_BYTES;
    MF_CUDA(cudaFuncSetAttribute(k_gemm_tc<TC_TRAIL, LDLT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp));
    MF_CUDA(cudaFuncSetAttribute(k_gemm_tc<TC_SYRK, LDLT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sp));
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
    std::lock_guard<std::recursive_mutex> lk(device_mutex());
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

// the trailing update (role 1) or SYRK (role 2) from pre-split operands:
// k_tc_split over `units`, then the tile kernel
int tc_launch_split(mf_handle* h, int role, const ItemList& l, const ItemList& units, int obs, int obw, int c0,
                    const FactorBufs<float>& fb) {
    if (h->diag)
        return role == TC_TRAIL ? launch_split<TC_TRAIL, 1>(h, l, units, obs, obw, c0, fb)
                                : launch_split<TC_SYRK, 1>(h, l, units, obs, obw, c0, fb);
    return role == TC_TRAIL ? launch_split<TC_TRAIL, 0>(h, l, units, obs, obw, c0, fb)
                            : launch_split<TC_SYRK, 0>(h, l, units, obs, obw, c0, fb);
}

int tc_launch(mf_handle* h, int role, const ItemList& l, int obs, int obw, int c0, const FactorBufs<float>& fb) {
    if (h->diag) {
        switch (role) {
            case TC_LEFT: return launch_one<TC_LEFT, 1>(h, l, obs, obw, c0, fb);
            case TC_TRAIL: return launch_one<TC_TRAIL, 1>(h, l, obs, obw, c0, fb);
            case TC_SYRK: return launch_one<TC_SYRK, 1>(h, l, obs, obw, c0, fb);
            default: return launch_one<TC_TRSM, 1>(h, l, obs, obw, c0, fb);
        }
    }
    switch (role) {
        case TC_LEFT: return launch_one<TC_LEFT, 0>(h, l, obs, obw, c0, fb);
        case TC_TRAIL: return launch_one<TC_TRAIL, 0>(h, l, obs, obw, c0, fb);
        case TC_SYRK: return launch_one<TC_SYRK, 0>(h, l, obs, obw, c0, fb);
        default: return launch_one<TC_TRSM, 0>(h, l, obs, obw, c0, fb);
    }
}

}  // namespace mf
