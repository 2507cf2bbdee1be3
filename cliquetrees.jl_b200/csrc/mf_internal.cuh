// Internal declarations of the B200 multifrontal numeric phase.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <string>
#include <cstdlib>
#include <mutex>
#include <utility>
#include <vector>

namespace mf {

// ---------------------------------------------------------------------------
// Device layout.  Every front j (postorder, 0-based) owns
//   * a panel   P_j : nj x nn column major, leading dimension nj, at Pval+poff.
//                     Rows 0..nn-1 are the diagonal block D (lower triangle
//                     used), rows nn..nj-1 are the off-diagonal block L.
//                     This is the reference's Dval/Lval pair stacked into one
//                     matrix so that every kernel sees one leading dimension.
//   * an update matrix M_j : na x na column major (lower triangle used) at
//                     Mval+moff, alive from the factorization of j until its
//                     parent has been assembled.
// ---------------------------------------------------------------------------
struct Front {
    int64_t poff;   // panel offset in Pval (multiple of 4 elements)
    int64_t moff;   // update-matrix offset in Mval (na > 0)
    int64_t roff;   // first row of this front's solve update block in Rval (block at R + roff*nrhs)
    int64_t ioff;   // offset of its 64x64 diagonal-block inverses in the inverse scratch
    int64_t i2off;  // offset of its 256x256 diagonal super-block inverses (blocked solves), -1 if none
    int32_t nn;     // |res(j)|
    int32_t na;     // |sep(j)|
    int32_t col0;   // first (permuted) column of res(j)
    int32_t sep0;   // offset of sep(j)/rel(j) in septgt/reltgt
    int32_t chd0;   // children of j are chdtgt[chd0:chd1]
    int32_t chd1;
    int32_t parent; // -1 for roots
    int32_t level;  // height above the leaves
    int32_t ldp;    // panel leading dimension: nj rounded up to a multiple of 4
    int32_t ldm;    // update-matrix leading dimension: na rounded up to a multiple of 4
};

// A front of the reference's ChordalSymbolic and where its blocks live
// inside the execution front that contains it.
struct RefFront {
    int64_t Dptr;   // offset of its nn x nn block in the reference Dval
    int64_t Lptr;   // offset of its na x nn block in the reference Lval
    int32_t nn, na;
    int32_t res0;   // first column
    int32_t sep0;   // offset of sep(j) in septgt (and in sepmap)
    int32_t exec;   // execution front holding it
    int32_t pad;
};

// Pivot rule of the factorization: delta < 0 is NoRegularization (a pivot
// of the wrong sign, or zero, is rejected); otherwise DynamicRegularization
// (dynamic_regularization.jl:75-90): a pivot with s * d < eps becomes
// delta * s.
struct Reg {
    double delta = -1.0;
    double eps = 0.0;
};

// One unit of grouped work: front plus up to two tile coordinates.
struct Item {
    int32_t front;
    int32_t a;
    int32_t b;
    int32_t pad;
};

// A contiguous list of items inside the uploaded item buffer.
// one child update row that lands on a row of a blocked front, for the
// forward gather: the child's R block (at R + roff * nrhs, leading dimension
// ma) row a
struct GCon {
    int64_t roff;
    int32_t a;
    int32_t ma;
};

struct ItemList {
    int64_t off = 0;
    int64_t cnt = 0;
};

constexpr int kSmallMax = 96;   // fronts with nj <= kSmallMax: one fused CTA
constexpr int kWarpSmallNJ = 16; // of those, fronts with nj <= kWarpSmallNJ: one warp each (k_small_warp)
constexpr int kWarpSmallNJ2 = 32; // and kWarpSmallNJ < nj <= kWarpSmallNJ2: one warp each, 32-row variant
constexpr int kTinyNJ = 16;      // solves: fronts with nj <= kTinyNJ take 16 lanes each (k_s_tiny_*)
constexpr int kTinyNJ2 = 32;     // and kTinyNJ < nj <= kTinyNJ2 a warp each, with k_s_tiny_*'s design
constexpr int kNB = 64;         // sub-panel width of the blocked path
#ifndef MF_KOB
#define MF_KOB 256
#endif
constexpr int kOB = MF_KOB;     // outer block: trailing updates run with K = kOB
constexpr int kOBWide = 2 * kOB;  // outer block of levels whose largest front has >= kWideFrontNN columns
constexpr int kWideFrontNN = 12288;
constexpr int kTile = 64;       // tile edge of the grouped update kernels
constexpr int kTM = 128;        // rows of a tensor-core (tcgen05) tile; columns stay kTile
constexpr int kEAcols = 16;     // parent columns per extend-add work item
constexpr int kEArows = 1024;   // parent rows per extend-add work item
constexpr int kSolveRows = 256; // rows per gather work item
constexpr int kTcSyrkN = 128;   // tile columns of the tensor-core SYRK
constexpr int kTcTrailN = 128;  // tile columns of the tensor-core trailing update
constexpr int kSplitRows = 128;  // rows of a pre-split operand unit
constexpr int kSplitK = 32;      // columns (K) of a pre-split operand unit
constexpr int kSplitUnitFloats = 2 * kSplitRows * kSplitK;  // hi and lo tiles: 32 KB
constexpr int kFwdRows = 64;    // rows per forward-update work item
constexpr int kSolveNB = 256;   // columns of a solve step: a super-block of four 64-column diagonal blocks
constexpr int kBwdRows = 512;   // rows of L21 per backward partial-sum work item
constexpr int kFwdCols = 512;   // columns of L21 per forward partial-sum work item
constexpr int kChainMinSteps = 64;  // super-block steps of a level from which its solve runs as one k_s_chain launch
constexpr int kMidCluster = 8;   // CTAs of the cluster that solves one front of a single-super-block level
constexpr int64_t kMidMaxL21 = 1 << 20;  // such levels' largest nn * na (a cluster streams L21 from 8 SMs)

// One 64-wide sub-panel s of outer block b (columns b*kob + s*kNB ..., kob the level's outer-block width).
struct PanelStep {
    int b = 0, s = 0;
    ItemList left;    // (front, row tile)  : left-looking update from the outer block's earlier sub-panels
    ItemList diag;    // (front)            : diagonal block factor + inverse
    ItemList panel;   // (front, row tile)  : panel TRSM below the diagonal block (GEMM with the inverse)
    ItemList trail;   // (front, ti, tj)    : after the last sub-panel of an outer block: trailing update, K = kob
    // the first trail_ncrit (trail_tc_ncrit) items update the next outer
    // block's columns; the rest may run beside that block's sub-panels
    int64_t trail_ncrit = 0, trail_tc_ncrit = 0;
    // the same work in 128-row tiles for the tensor-core (tcgen05) kernels
    ItemList left_tc, panel_tc, trail_tc;
    // (front, 128-row block, 32-column chunk, first unit): the trailing
    // update's operands split into TF32 hi / lo tiles once (k_tc_split);
    // trail_tc items carry the front's first unit in pad
    ItemList split_tc;
};

// One 256-column super-block K of the blocked fronts' diagonal blocks.
struct SolveStep {
    ItemList diag;    // (front)            x_K = X_K b_K (forward) or X_K^T b_K (backward)
    ItemList fwd;     // (front, row tile)  rows below the super-block -= L x_K
    ItemList bwd;     // (front, col tile)  columns left of the super-block -= L^T x_K
};

struct Level {
    ItemList small_warp;     // (front)           fronts with nj <= kWarpSmallNJ: one warp each (k_small_warp)
    ItemList small_warp2;    // (front)           kWarpSmallNJ < nj <= kWarpSmallNJ2: one warp each (MF_WARP_FRONT32=0: k_small)
    ItemList small;          // (front)           other fronts with nj <= kSmallMax: one CTA each (k_small)
    int small_maxnj = 0;     // largest nj of those (sizes k_small's shared memory and CTA)
    // extend-add for blocked fronts, item (front, col tile, row chunk, first
    // segment): ea adds the children into the panel columns before the
    // panel is factored; ea_upd adds them into the update matrix after the
    // SYRK has written M = -L21 L21^T.  Each item's segments (two Items per
    // child, children in reverse order) are {child, b0, b1}, {a0, a1}: the
    // child columns b0..b1 and rows a0..a1 whose relative indices land in the
    // item's columns and rows.
    ItemList ea;
    ItemList ea_upd;
    std::vector<PanelStep> steps;
    ItemList syrk;           // (front, ti, tj)   M -= L L^T
    ItemList syrk_tc;        // 128 x 64 tiles for the tcgen05 kernel
    ItemList split_syrk;     // (front, row block, chunk, first unit) of the SYRK's split operands
    // solves
    ItemList s_small;        // (front)
    ItemList s_tiny;         // (front)           small fronts with nj <= kTinyNJ: 16 lanes each
    ItemList s_tiny2;        // (front)           small fronts with kTinyNJ < nj <= kTinyNJ2: a warp each
    ItemList s_gather;       // (front, row tile) forward gather of child updates
    std::vector<SolveStep> s_steps;
    ItemList s_fwd_l;        // (front, row tile, col chunk; pad = partial slot) R -= L21 x1
    ItemList s_fwd_red;      // (front, row tile, first partial slot, chunks)
    ItemList s_bwd_l;        // (front, col tile, row chunk; pad = partial slot) C1 -= L^T x[sep]
    ItemList s_bwd_red;      // (front, col tile, first partial slot)
    // levels whose blocked fronts all have nn <= kSolveNB and nn * na <=
    // kMidMaxL21: one cluster per front does the forward (k_s_mid_fwd) or
    // backward (k_s_mid_bwd) work of s_gather .. s_bwd_red in one launch;
    // item (front, first s_gather item, first s_bwd_l slot, gather tiles)
    ItemList s_mid;
    // the super-block chain of the blocked fronts as one launch per
    // direction (k_s_chain): items (front, a, step K, counter base), a = -1 - q
    // for diagonal part q, else the tile; d_chain[chain_tk] / [chain_tk + 1]
    // are the forward / backward ticket counters
    ItemList s_chain_f;
    ItemList s_chain_b;
    int64_t chain_tk = -1;
    int max_nn_blocked = 0;
    int kob = kOB;           // outer-block width of this level's panel steps (kOB or kOBWide)
    // FP32 kernel choice of this level, set by mf_autotune: 1 = tcgen05
    // tensor-core tiles (128 x 64 / 128 x 128), 0 = FFMA tiles (64 x 64)
    int tc_steps = 1;        // left-looking, TRSM and trailing roles of the panel steps
    int tc_syrk = 1;         // the SYRK role
};

struct KernelTimes {
    double ms[24] = {0};
    int64_t launches[24] = {0};
};

enum KernelId {
    K_ASSEMBLE = 0, K_SMALL, K_EA, K_PANEL, K_UPDATE, K_SYRK,
    K_S_SMALL, K_S_GATHER, K_S_FWD, K_S_BWD_L, K_S_BWD, K_PERM, K_OTHER,
    K_DIAG, K_LEFT, K_SPMV,
    K_SOLVE_PASS,  // not a kernel: solve passes (launches) made while profiling
    K_SOLVE_RHS,   // not a kernel: right-hand-side columns those passes solved
    K_COUNT
};

// The solves handle a front with one warp when the factorization kept it
// whole (nj <= kSmallMax) or it is narrow with a short L21 (a warp streams
// L21 row by row, so a long one serialises); otherwise it is blocked in the
// factorization too and its diagonal-block inverses exist.
constexpr int kSmallSolveNA = 256;
__host__ __device__ inline bool solve_small(const Front& f) {
    return f.nn + f.na <= kSmallMax || (f.nn <= kNB && f.na <= kSmallSolveNA);
}

// Super-block K of a blocked front: its inverse X_K (wK x wK, lower, unit
// diagonal for LDLt) is stored column major with leading dimension
// super_ld(wK) at inv2 + f.i2off + K * kSolveNB * kSolveNB.
__host__ __device__ inline int super_ld(int wK) { return wK == kSolveNB ? kSolveNB : ((wK + 3) & ~3); }

// numeric buffers of one precision
template <typename T>
struct FactorBufs {
    T* P = nullptr;    // panels
    T* M = nullptr;    // update matrices
    T* inv = nullptr;  // diagonal-block inverses
    T* d = nullptr;    // LDLt pivots (n)
    T* inv2 = nullptr; // 256x256 super-block inverses
};

template <typename T>
struct SolveBufs {
    const T* P = nullptr;
    const T* inv = nullptr;
    const T* d = nullptr;
    T* R = nullptr;
    T* W = nullptr;
    T* C = nullptr;
    T* part = nullptr;  // backward partial sums (nbwd_part * 64 * 16)
    const T* inv2 = nullptr;  // super-block inverses
};

// An instantiated CUDA graph of one fixed launch sequence of a handle (a
// factorization or a solve), keyed by what the sequence depends on.
struct GraphEntry {
    int64_t key[4];
    cudaGraphExec_t exec;
};

// single-precision copy of the factor and solve workspaces (mixed mode)
struct Mixed {
    float* split = nullptr;   // pre-split TF32 operand units of the trailing updates / SYRK (32 KB each)
    float* P = nullptr;
    float* M = nullptr;
    float* inv = nullptr;
    float* d = nullptr;
    float* R = nullptr;
    float* W = nullptr;
    float* C = nullptr;
    float* part = nullptr;
    float* inv2 = nullptr;
};

}  // namespace mf

struct mf_handle {
    int device = 0;
    int num_sms = 0;              // streaming multiprocessors of the device (persistent grids)
    int diag = 0;                 // 0 Cholesky, 1 LDLt
    int64_t n = 0, nfr = 0, nsep = 0;
    int64_t ndz = 0, nlz = 0, npanel = 0, nmval = 0, nrval_per_rhs = 0;
    int nrhs_cap = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    // host copies
    int64_t nexec = 0;              // execution fronts (after amalgamation)
    std::vector<mf::Front> h_fronts;        // execution fronts
    std::vector<mf::RefFront> h_ref;        // reference fronts
    std::vector<int32_t> h_exec_of;         // reference front -> execution front
    std::vector<int32_t> h_exec_chd;        // execution children CSR targets
    std::vector<int32_t> h_exec_rel;        // execution rel (indexed like septgt)
    std::vector<int32_t> h_sepmap;          // reference sep rows -> execution panel rows
    std::vector<int64_t> h_resptr, h_sepptr, h_septgt, h_Dptr, h_Lptr;
    std::vector<mf::Level> levels;
    mf::ItemList inv2_items;                // (front, super-block) of the super-block inverses
    std::vector<mf::Item> h_items;

    // device symbolic
    mf::Front* d_fronts = nullptr;
    int32_t* d_septgt = nullptr;
    int32_t* d_reltgt = nullptr;
    int32_t* d_chdtgt = nullptr;
    int32_t* d_colfront = nullptr;  // column -> reference front (n)
    mf::RefFront* d_ref = nullptr;  // reference fronts (nfr)
    int32_t* d_sepmap = nullptr;    // reference sep rows -> execution panel rows (nsep)
    mf::Item* d_items = nullptr;

    // device numeric
    double* d_P = nullptr;         // panels
    double* d_inv = nullptr;       // inverses of the 64x64 diagonal blocks
    int64_t ninv = 0;
    double* d_inv2 = nullptr;      // inverses of the 256x256 diagonal super-blocks (blocked solves)
    int64_t ninv2 = 0;
    double* d_M = nullptr;         // update matrices
    double* d_d = nullptr;         // LDLt pivots (n)
    double* d_signs = nullptr;     // pivot signs (n) or null
    long long* d_info = nullptr;   // first failing column (1-based), LLONG_MAX if none
    int* d_err = nullptr;          // set by a kernel whose bounded wait timed out
    int* d_rescued = nullptr;      // single-precision fronts / diagonal blocks refactored in FP64
    bool use_tc = true;            // tcgen05 tensor cores for the FP32 GEMMs
    void* d_tmaps = nullptr;       // CUtensorMap per execution front (FP32 panels)
    void* d_tmap_inv = nullptr;    // CUtensorMap over the FP32 diagonal-block inverses
    double* d_R = nullptr;         // solve updates (sum na * nrhs_cap)
    double* d_W = nullptr;         // solve work (n * nrhs_cap)
    double* d_part = nullptr;      // backward partial sums
    std::vector<int64_t> h_grow;   // forward gather: per row of every blocked front, its first GCon
    std::vector<mf::GCon> h_gcon;  // forward gather contributions, row by row
    int64_t* d_grow = nullptr;
    mf::GCon* d_gcon = nullptr;
    int64_t nbwd_part = 0;         // partial slots (max over levels)
    int64_t nsplit_units = 0;      // largest number of split operand units one launch needs
    bool tc_split = true;          // tensor-core updates read pre-split operands (MF_TC_SPLIT=0: convert per tile)
    mf::ItemList sub_tasks;        // k_s_sub_fwd / _bwd tasks (subtrees of small fronts), one CTA each
    int* d_chain = nullptr;        // k_s_chain ticket and progress counters, zeroed per solve
    int64_t nchain = 0;
    int solve_chain = 2;           // k_s_chain launches: 1 every level (MF_SOLVE_CHAIN=1), 0 none (=0),
                                   // 2 the levels of at least kChainMinSteps steps (default)
    bool tiny_solve = true;        // k_s_tiny_* for the fronts with nj <= kTinyNJ (MF_TINY_SOLVE=0: k_s_small_*)
    bool panel_pdl = false;        // the factorization's sub-panel chain (left-looking, diagonal block, TRSM)
                                   // launched for programmatic dependence (MF_PANEL_PDL=1)
    cudaStream_t side = nullptr;   // the factorization's look-ahead stream (trailing updates beside the next
                                   // outer block's sub-panels), forked from and joined into `stream`
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool lookahead = true;         // MF_LOOKAHEAD=0: every trailing update on `stream`
    int grid_cap = 0;              // while > 0: the persistent tensor-core kernels' CTA count limit
    int side_free_sms = 24;        // SMs the look-ahead trailing update leaves to the sub-panel kernels (MF_SIDE_FREE_SMS)
    bool step_pdl = true;          // solve-step kernels launched for programmatic dependence (MF_STEP_PDL=0: off)
    bool mid_solve = false;        // one cluster launch per single-super-block level and direction (MF_MID_SOLVE=1)
    double* d_C = nullptr;         // solve rhs / solution (n * nrhs_cap), permuted order
    double* d_B = nullptr;         // rhs in original order (n * nrhs_cap)
    int64_t* d_perm = nullptr;     // permutation (n)
    double* d_DL = nullptr;        // staging for reference-layout Dval|Lval (ndz+nlz)
    int64_t* d_slot = nullptr;     // assembly map into Dval|Lval (nnz)
    int64_t* d_pslot = nullptr;    // assembly map into panels (nnz)
    double* d_nz = nullptr;        // nonzero values staging (nnz)
    int32_t* d_nzrow = nullptr;    // permuted row of each stored value (nnz)
    int32_t* d_nzcol = nullptr;    // permuted column of each stored value (nnz)
    int64_t* d_dslot = nullptr;    // index of a_ii among the stored values (n), -1 if absent
    int64_t nnz = 0;

    // mixed precision (FP32 fronts + FP64 refinement)
    bool mixed = false;
    mf::Mixed f32;
    double* d_scale = nullptr;     // symmetric diagonal scaling, elimination order (n)
    // FP64 residual: CSR of the whole symmetric matrix in elimination order
    int64_t* d_csrptr = nullptr;   // n+1
    int32_t* d_csrcol = nullptr;   // nnz_full
    int64_t* d_csrsrc = nullptr;   // index of each entry among the stored values
    int64_t nnz_full = 0;
    double* d_iv = nullptr;        // refinement vectors: b, x, r, z, p, q (6 * n * nrhs_cap)
    double* d_kry = nullptr;       // GMRES bases V, Z and partial sums (allocated on first use)
    int64_t kry_doubles = 0;
    double* d_red = nullptr;       // reductions and scalars (see mf_refine.cu)
    const double* cur_nz = nullptr; // values of the current matrix (device)
    bool mixed_fallback = false;   // FP32 factorization failed; the FP64 factor is used
    // the FP64 factor storage holds the factor of the current values: set by
    // every completed FP64 factorization, cleared when a mixed factorization
    // stays in FP32 (its FP64 storage then still holds an older matrix)
    bool fp64_current = false;
    // independent row segments (a batch of matrices factored as one forest):
    // the refinement measures the backward error of every segment separately
    int64_t nseg = 0;
    int64_t* d_segptr = nullptr;   // nseg + 1 row boundaries, elimination order
    double* d_segred = nullptr;    // per segment: max|t|, max|x|, max|b| (3 x 16), ||A||_inf
    double* d_segeta = nullptr;    // per segment: worst backward error of the last refinement step
    // row chunks of at most kChunkRows rows inside one segment, so that the
    // per-segment reductions spread over many CTAs even for large segments
    std::vector<int64_t> h_segptr; // host copy of the segment boundaries
    int64_t nchunk = 0;
    int64_t* d_chunkrow = nullptr; // nchunk + 1 row boundaries
    int32_t* d_chunkseg = nullptr; // segment of every chunk
    int64_t* d_segchunk = nullptr; // chunks of segment s: [d_segchunk[s], d_segchunk[s+1])
    int32_t* d_rowseg = nullptr;   // segment of every row (n)
    double* d_chunkred = nullptr;  // per chunk: residual maxima (kSegRed) and dot partials (16)
    double* d_segsc = nullptr;     // per segment: CG scalars (80)

    double* d_logdet = nullptr;    // per-block partial results of mf_logdet (allocated on first use)
    void* cublas = nullptr;        // cuBLAS handle of the selected inversion (created on first use)
    bool selinv_done = false;      // the FP64 panels hold the selected inverse (mf_selinv), not a factor
    mf::Reg reg;                   // pivot rule of the FP64 factorization (mf_set_regularization)
    int64_t bytes = 0;             // device bytes allocated
    // optional per-kernel timing
    bool profile = false;
    mf::KernelTimes times;
    // autotuning: per-level times of the panel steps and of the SYRK
    bool tuning = false;
    std::vector<double> tune_steps_ms, tune_syrk_ms;
    // CUDA graphs of the factorization and solve launch sequences
    bool use_graphs = true;
    std::vector<mf::GraphEntry> graphs;
    std::vector<cudaEvent_t> ev_pool;
};

namespace mf {

void set_error(const std::string& msg);
// Held while a stream is being captured into a CUDA graph and around every
// device allocation, free or device-wide synchronisation of the library:
// those calls fail ("operation not permitted when stream is capturing") if
// another thread's stream is capturing at the same moment.
std::recursive_mutex& device_mutex();
int cuda_fail(cudaError_t e, const char* where);

// Programmatic dependent launch.  Every kernel of the factorization, solve
// and refinement paths starts with pdl_prologue(): it waits until the grid
// it depends on has completed and its memory is visible (a no-op for a grid
// launched without the attribute), then lets the next grid of the stream be
// launched.  launch_k() launches with the attribute, so consecutive kernels
// of a captured graph overlap the next launch's setup with the tail of the
// current one while keeping stream order for every memory access.  Opt-in
// (MF_PDL=1 in the environment): on the 80^3 workload the graph replays ran
// about 2 % slower with it (100.9 vs 98.8 ms FP64, 46.9 vs 45.9 ms mixed).
__device__ __forceinline__ void pdl_prologue() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

inline bool pdl_enabled() {
    static const bool on = [] {
        const char* e = getenv("MF_PDL");
        return e && e[0] == '1';
    }();
    return on;
}

// the launch itself: with the attribute when `pdl`
template <typename... KArgs, typename... Args>
inline cudaError_t launch_kx(bool pdl, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                             cudaStream_t st, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_k(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                            Args&&... args) {
    return launch_kx(pdl_enabled(), kern, grid, block, smem, st, std::forward<Args>(args)...);
}

// The blocked solve-step kernels (k_s_sdiag, k_s_ftile, k_s_btile) let the
// next grid launch at once and wait for the previous one only after they
// have issued their loads of the panel or the inverse, which no kernel of
// the solve writes; they are launched with the attribute unless
// MF_STEP_PDL=0, so each step's launch and those loads overlap the step
// before it.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }


#define MF_CUDA(call)                                                  \
    do {                                                               \
        cudaError_t _e = (call);                                       \
        if (_e != cudaSuccess) return mf::cuda_fail(_e, #call);        \
    } while (0)

// plan construction (mf_plan.cu)
int build_plan(mf_handle* h, const int64_t* resptr, const int64_t* sepptr, const int64_t* septgt,
               const int64_t* reltgt, const int64_t* chdptr, const int64_t* chdtgt, const int64_t* Dptr,
               const int64_t* Lptr);

// kernel launchers (mf_factor.cu / mf_solve.cu); all stream ordered
int launch_factor(mf_handle* h);
// FP64 factor storage (panels, update matrices, block inverses): a mixed
// handle releases it in mf_enable_mixed and allocates it again only when a
// factorization falls back to FP64; a non-zero return means it is absent.
int ensure_fp64(mf_handle* h);
int have_fp64(const mf_handle* h);
int launch_factor_mixed(mf_handle* h);
int tc_prepare(mf_handle* h);
int tc_launch(mf_handle* h, int role, const ItemList& l, int obs, int obw, int c0, const FactorBufs<float>& fb);
int tc_launch_split(mf_handle* h, int role, const ItemList& l, const ItemList& units, int obs, int obw, int c0,
                    const FactorBufs<float>& fb);
int launch_assemble_mixed(mf_handle* h, const double* dnz);
int launch_dl_to_panel(mf_handle* h, const double* dDval, const double* dLval);
int launch_panel_to_dl(mf_handle* h, double* dDval, double* dLval);
int launch_panel32_to_dl(mf_handle* h, double* dDval, double* dLval);
int launch_assemble(mf_handle* h, const double* dnz);
int launch_solve(mf_handle* h, int64_t nrhs);
// the FP64 solve with caller-provided work buffers in place of the handle's
// (R: nrval_per_rhs*nrhs, W and C: n*nrhs, part: nbwd_part*64*16 doubles)
int launch_solve_with(mf_handle* h, int64_t nrhs, double* R, double* W, double* C, double* part);
int launch_solve_mixed(mf_handle* h, int64_t nrhs);
int launch_permute_to(mf_handle* h, const double* B, int64_t ldb, const int64_t* perm, int64_t nrhs, double* dst);
int launch_permute_from(mf_handle* h, double* B, int64_t ldb, const int64_t* perm, int64_t nrhs, const double* src);
int launch_anorm(mf_handle* h);
// selected inversion of the FP64 Cholesky factor in place (mf_selinv)
int launch_selinv(mf_handle* h);
// log|det A| and sign(det A) from the factor on the device (mf_logdet)
int launch_logdet(mf_handle* h, double* logabsdet, double* sign);
constexpr int kSegRed = 49;  // doubles per segment in d_segred
constexpr int kChunkRows = 16384;  // rows per reduction chunk of a segment
constexpr int kChunkRed = kSegRed + 16;  // doubles per chunk in d_chunkred
int refine(mf_handle* h, const double* b, double* x, int nrhs, double tol, int maxit, int* iters, double* eta);
constexpr int kRedDoubles = 256 + 16 * 148 * 4;
int launch_permute_in(mf_handle* h, const double* B, int64_t ldb, const int64_t* perm, int64_t nrhs);
int launch_permute_out(mf_handle* h, double* B, int64_t ldb, const int64_t* perm, int64_t nrhs);
const char* last_error();

// Run `body` (stream-ordered launches on h->stream) as a CUDA graph: the
// first call with a key captures and instantiates it, later calls replay it.
// Runs `body` directly when graphs are off, per-kernel profiling is on, the
// handle's stream is the legacy default stream, or the caller is already
// capturing that stream.
int run_captured(mf_handle* h, int64_t k0, int64_t k1, int64_t k2, int64_t k3, const std::function<int()>& body);
void release_graphs(mf_handle* h);

// timing helpers
struct Timer {
    mf_handle* h;
    int k;
    cudaEvent_t a = nullptr, b = nullptr;
    Timer(mf_handle* h_, int k_);
    ~Timer();
};

}  // namespace mf
