// C ABI of the B200 multifrontal numeric phase (include/mfgpu.h).
#include <algorithm>
#include <cmath>
#include <climits>
#include <cstring>
#include <cstdlib>
#include <new>

#include <cublas_v2.h>

#include "../../include/mfgpu.h"
#include "mf_internal.cuh"

using namespace mf;

namespace {

template <typename T>
int dalloc(mf_handle* h, T** p, int64_t count, int64_t* total) {
    *p = nullptr;
    if (count <= 0) return 0;
    std::lock_guard<std::recursive_mutex> lk(device_mutex());
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * (size_t)count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(std::string("cudaMalloc of ") + std::to_string(sizeof(T) * (size_t)count) +
                  " bytes failed: " + cudaGetErrorString(e));
        *p = nullptr;
        return -4;
    }
    *total += sizeof(T) * count;
    (void)h;
    return 0;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

void free_all(mf_handle* h) {
    std::lock_guard<std::recursive_mutex> lk(device_mutex());
    void* ptrs[] = {h->d_fronts, h->d_septgt, h->d_reltgt, h->d_chdtgt, h->d_colfront, h->d_ref, h->d_sepmap,
                    h->d_items,  h->d_P,      h->d_M,      h->d_d,      h->d_signs,    h->d_info, h->d_R,
                    h->d_W,      h->d_C,      h->d_B,      h->d_perm,   h->d_DL,       h->d_slot, h->d_pslot,
                    h->d_nz,     h->d_inv,    h->d_nzrow,  h->d_nzcol,  h->d_dslot,    h->d_scale,
                    h->d_csrptr, h->d_csrcol, h->d_csrsrc, h->d_iv,     h->d_red,      h->f32.P,  h->f32.M,
                    h->f32.inv,  h->f32.d,    h->f32.R,    h->f32.W,    h->f32.C,      h->d_err,
                    h->d_part,   h->f32.part, h->d_tmaps,  h->d_tmap_inv, h->d_segptr, h->d_segred,
                    h->d_segeta, h->d_kry,    h->d_inv2,   h->f32.inv2,   h->d_chunkrow, h->d_chunkseg,
                    h->d_segchunk, h->d_rowseg, h->d_chunkred, h->d_segsc, h->d_logdet, h->d_rescued, h->d_chain, h->f32.split,
                    h->d_grow, h->d_gcon};
    release_graphs(h);
    if (h->cublas) cublasDestroy(static_cast<cublasHandle_t>(h->cublas));
    h->cublas = nullptr;
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    h->side = nullptr;
    h->ev_fork = h->ev_join = nullptr;
}

int init_info(mf_handle* h) {
    static const long long big = LLONG_MAX;
    MF_CUDA(cudaMemcpyAsync(h->d_info, &big, sizeof(long long), cudaMemcpyHostToDevice, h->stream));
    MF_CUDA(cudaMemsetAsync(h->d_rescued, 0, sizeof(int), h->stream));
    return 0;
}

int read_info(mf_handle* h, int64_t* info) {
    long long v = 0;
    MF_CUDA(cudaMemcpyAsync(&v, h->d_info, sizeof(long long), cudaMemcpyDeviceToHost, h->stream));
    MF_CUDA(cudaStreamSynchronize(h->stream));
    if (info) *info = (v == LLONG_MAX) ? 0 : (int64_t)v;
    return 0;
}

int upload_signs(mf_handle* h, const double* signs, const double** dsigns) {
    *dsigns = nullptr;
    if (!signs) return 0;
    if (!h->d_signs) {
        int64_t tot = 0;
        int rc = dalloc(h, &h->d_signs, h->n, &tot);
        if (rc) return rc;
    }
    MF_CUDA(cudaMemcpyAsync(h->d_signs, signs, sizeof(double) * h->n, cudaMemcpyHostToDevice, h->stream));
    *dsigns = h->d_signs;
    return 0;
}

int64_t g_total_bytes_last = 0;

}  // namespace

extern "C" {

const char* mf_last_error(void) { return mf::last_error(); }

int mf_create(int64_t n, int64_t nfr, const int64_t* resptr, const int64_t* sepptr, const int64_t* septgt,
              const int64_t* reltgt, const int64_t* chdptr, const int64_t* chdtgt, const int64_t* Dptr,
              const int64_t* Lptr, int diag, int nrhs_cap, int device, mf_handle** out) {
    if (!out) { set_error("mf_create: out is NULL"); return -1; }
    *out = nullptr;
    if (n < 0 || nfr < 0 || (n > 0 && nfr == 0) || !resptr || !sepptr || !chdptr || !Dptr || !Lptr ||
        (nfr > 0 && !chdtgt) || (diag != 0 && diag != 1) || nrhs_cap < 1 || nrhs_cap > 16 || device < 0) {
        set_error("mf_create: bad arguments");
        return -1;
    }
    if (n > INT32_MAX / 2) { set_error("mf_create: n too large for 32-bit row indices"); return -1; }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device >= ndev) {
        cudaGetLastError();
        set_error("mf_create: no CUDA device");
        return -3;
    }
    DeviceGuard g(device);
    mf_handle* h = new (std::nothrow) mf_handle();
    if (!h) { set_error("out of host memory"); return -4; }
    h->device = device;
    if (cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        cudaGetLastError();
        h->num_sms = 148;
    }
    h->diag = diag;
    h->n = n;
    h->nfr = nfr;
    h->nrhs_cap = nrhs_cap;
    int rc;
    try {
        rc = build_plan(h, resptr, sepptr, septgt, reltgt, chdptr, chdtgt, Dptr, Lptr);
    } catch (const std::bad_alloc&) {
        set_error("out of host memory building the plan");
        rc = -4;
    }
    if (rc) { delete h; return rc; }
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaStreamCreate / cudaEventCreate failed");
        if (h->stream) cudaStreamDestroy(h->stream);
        if (h->side) cudaStreamDestroy(h->side);
        if (h->ev_fork) cudaEventDestroy(h->ev_fork);
        delete h;
        return -3;
    }
    h->own_stream = true;

    int64_t tot = 0;
    int64_t nsep = h->nsep;
    const int64_t nex = h->nexec;
    std::vector<int32_t> sep32(nsep), colfront(n);
    for (int64_t i = 0; i < nsep; ++i) sep32[i] = (int32_t)septgt[i];
    for (int64_t j = 0; j < nfr; ++j)
        for (int64_t c = resptr[j]; c < resptr[j + 1]; ++c) colfront[c] = (int32_t)j;
    rc = 0;
    // allocations and the synchronous uploads below stay clear of other
    // threads' stream captures
    std::lock_guard<std::recursive_mutex> lk(device_mutex());
    rc = rc ? rc : dalloc(h, &h->d_fronts, nex, &tot);
    rc = rc ? rc : dalloc(h, &h->d_septgt, nsep, &tot);
    rc = rc ? rc : dalloc(h, &h->d_reltgt, (int64_t)h->h_exec_rel.size(), &tot);
    rc = rc ? rc : dalloc(h, &h->d_chdtgt, (int64_t)h->h_exec_chd.size(), &tot);
    rc = rc ? rc : dalloc(h, &h->d_colfront, n, &tot);
    rc = rc ? rc : dalloc(h, &h->d_ref, nfr, &tot);
    rc = rc ? rc : dalloc(h, &h->d_sepmap, (int64_t)h->h_sepmap.size(), &tot);
    rc = rc ? rc : dalloc(h, &h->d_items, (int64_t)h->h_items.size(), &tot);
    rc = rc ? rc : dalloc(h, &h->d_grow, std::max<int64_t>((int64_t)h->h_grow.size(), 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_gcon, std::max<int64_t>((int64_t)h->h_gcon.size(), 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_P, h->npanel, &tot);
    rc = rc ? rc : dalloc(h, &h->d_inv, std::max<int64_t>(h->ninv, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_inv2, std::max<int64_t>(h->ninv2, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_M, h->nmval, &tot);
    rc = rc ? rc : dalloc(h, &h->d_d, std::max<int64_t>(n, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_info, 1, &tot);
    rc = rc ? rc : dalloc(h, &h->d_err, 1, &tot);
    rc = rc ? rc : dalloc(h, &h->d_rescued, 1, &tot);
    rc = rc ? rc : dalloc(h, &h->d_R, std::max<int64_t>(h->nrval_per_rhs * nrhs_cap, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_W, std::max<int64_t>(n * nrhs_cap, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_part, std::max<int64_t>(h->nbwd_part * kNB * 16, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_chain, std::max<int64_t>(h->nchain, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_C, std::max<int64_t>(n * nrhs_cap, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_B, std::max<int64_t>(n * nrhs_cap, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_perm, std::max<int64_t>(n, 1), &tot);
    if (rc) { free_all(h); delete h; return rc; }
    auto up = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
        if (!bytes) return cudaSuccess;
        return cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
    };
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = up(h->d_fronts, h->h_fronts.data(), sizeof(Front) * nex);
    if (e == cudaSuccess) e = up(h->d_septgt, sep32.data(), sizeof(int32_t) * nsep);
    if (e == cudaSuccess) e = up(h->d_reltgt, h->h_exec_rel.data(), sizeof(int32_t) * h->h_exec_rel.size());
    if (e == cudaSuccess) e = up(h->d_chdtgt, h->h_exec_chd.data(), sizeof(int32_t) * h->h_exec_chd.size());
    if (e == cudaSuccess) e = up(h->d_colfront, colfront.data(), sizeof(int32_t) * n);
    if (e == cudaSuccess) e = up(h->d_ref, h->h_ref.data(), sizeof(RefFront) * nfr);
    if (e == cudaSuccess) e = up(h->d_sepmap, h->h_sepmap.data(), sizeof(int32_t) * h->h_sepmap.size());
    if (e == cudaSuccess) e = up(h->d_items, h->h_items.data(), sizeof(Item) * h->h_items.size());
    if (e == cudaSuccess) e = up(h->d_grow, h->h_grow.data(), sizeof(int64_t) * h->h_grow.size());
    if (e == cudaSuccess) e = up(h->d_gcon, h->h_gcon.data(), sizeof(GCon) * h->h_gcon.size());
    if (e == cudaSuccess) e = cudaMemset(h->d_P, 0, sizeof(double) * std::max<int64_t>(h->npanel, 0));
    if (e == cudaSuccess) e = cudaMemset(h->d_err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(h->d_rescued, 0, sizeof(int));
    if (e == cudaSuccess && n) {  // the permutation a NULL perm argument stands for, until one is passed
        std::vector<int64_t> iota((size_t)n);
        for (int64_t i = 0; i < n; ++i) iota[(size_t)i] = i;
        e = up(h->d_perm, iota.data(), sizeof(int64_t) * (size_t)n);
    }
    {
        // the one-launch chain measured slower than the per-step launches
        // on the 80^3 workload (38 steps at most: critical path per step
        // unchanged, waits added) and faster on the KKT workload's 133-step
        // root, so by default only levels of many steps use it
        const char* senv = getenv("MF_TC_SPLIT");
        h->tc_split = !(senv && senv[0] == '0');
        const char* cenv = getenv("MF_SOLVE_CHAIN");
        h->solve_chain = !cenv ? 2 : cenv[0] == '1' ? 1 : cenv[0] == '0' ? 0 : 2;
        // the sub-panel chain launched for programmatic dependence measured
        // no faster (80^3: 42.5 vs 42.2 ms; KKT: 232.6 vs 228.9 ms): opt-in
        const char* ppenv = getenv("MF_PANEL_PDL");
        h->panel_pdl = ppenv && ppenv[0] == '1';
        const char* fenv = getenv("MF_SIDE_FREE_SMS");
        if (fenv && atoi(fenv) >= 0) h->side_free_sms = atoi(fenv);
        const char* lenv = getenv("MF_LOOKAHEAD");
        h->lookahead = !(lenv && lenv[0] == '0');
        const char* penv = getenv("MF_STEP_PDL");
        h->step_pdl = !(penv && penv[0] == '0');
        const char* tenv = getenv("MF_TINY_SOLVE");
        h->tiny_solve = !(tenv && tenv[0] == '0');
        // the cluster-per-front level kernels measured slower than the
        // per-kernel launches on the 80^3 workload (a front's cluster holds
        // eight register-heavy CTAs however small the front), so opt-in
        const char* menv = getenv("MF_MID_SOLVE");
        h->mid_solve = menv && menv[0] == '1';
    }
    {
        const char* tcenv = getenv("MF_TENSOR_CORES");
        h->use_tc = !(tcenv && tcenv[0] == '0');
        const char* genv = getenv("MF_GRAPHS");
        h->use_graphs = !(genv && genv[0] == '0');
    }
    if (e != cudaSuccess) {
        cuda_fail(e, "mf_create upload");
        free_all(h);
        delete h;
        return -3;
    }
    g_total_bytes_last = tot;
    h->times = KernelTimes();
    h->bytes = tot;
    *out = h;
    return 0;
}

void mf_destroy(mf_handle* h) {
    if (!h) return;
    DeviceGuard g(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
}

int mf_plan_info(int64_t n, int64_t nfr, const int64_t* resptr, const int64_t* sepptr, const int64_t* septgt,
                 const int64_t* reltgt, const int64_t* chdptr, const int64_t* chdtgt, const int64_t* Dptr,
                 const int64_t* Lptr, int nrhs_cap, int64_t* out) {
    if (!out || n < 0 || nfr < 0 || !resptr || !sepptr || !chdptr || !Dptr || !Lptr || nrhs_cap < 1 ||
        nrhs_cap > 16) {
        set_error("mf_plan_info: bad arguments");
        return -1;
    }
    mf_handle h;
    h.n = n;
    h.nfr = nfr;
    h.nrhs_cap = nrhs_cap;
    int rc;
    try {
        rc = build_plan(&h, resptr, sepptr, septgt, reltgt, chdptr, chdtgt, Dptr, Lptr);
    } catch (const std::bad_alloc&) {
        set_error("out of host memory building the plan");
        rc = -4;
    }
    if (rc) return rc;
    int64_t launches = 0;
    for (const Level& lv : h.levels) {
        launches += (lv.small_warp.cnt > 0) + (lv.small_warp2.cnt > 0) + (lv.small.cnt > 0) + (lv.ea.cnt > 0) + (lv.ea_upd.cnt > 0) +
                    (lv.syrk.cnt > 0);
        for (const PanelStep& st : lv.steps)
            launches += (st.left.cnt > 0) + (st.diag.cnt > 0) + (st.panel.cnt > 0) + (st.trail.cnt > 0);
    }
    out[0] = h.nexec;
    out[1] = (int64_t)h.levels.size();
    out[2] = h.npanel;
    out[3] = h.nmval;
    out[4] = h.nrval_per_rhs;
    out[5] = (int64_t)h.h_items.size();
    out[6] = launches;
    return 0;
}

int mf_set_stream(mf_handle* h, void* stream) {
    if (!h) { set_error("null handle"); return -1; }
    DeviceGuard g(h->device);
    if (h->own_stream && h->stream) {
        cudaStreamSynchronize(h->stream);
        cudaStreamDestroy(h->stream);
        h->own_stream = false;
        h->stream = nullptr;
    }
    if (stream) {
        h->stream = (cudaStream_t)stream;
        h->own_stream = false;
    } else {
        MF_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->own_stream = true;
    }
    return 0;
}

int mf_chol_impl(mf_handle* h, double* Dval, double* Lval, double* d, const double* signs, int64_t* info) {
    if (!h || (!Dval && h->ndz) || (!Lval && h->nlz) || (h->diag && !d && h->n)) {
        set_error("mf_chol_impl: bad arguments");
        return -1;
    }
    DeviceGuard g(h->device);
    int rc;
    if ((rc = ensure_fp64(h))) return rc;
    if (!h->d_DL) {
        int64_t tot = 0;
        if ((rc = dalloc(h, &h->d_DL, std::max<int64_t>(h->ndz + h->nlz, 1), &tot))) return rc;
    }
    if (h->ndz)
        MF_CUDA(cudaMemcpyAsync(h->d_DL, Dval, sizeof(double) * h->ndz, cudaMemcpyHostToDevice, h->stream));
    if (h->nlz)
        MF_CUDA(cudaMemcpyAsync(h->d_DL + h->ndz, Lval, sizeof(double) * h->nlz, cudaMemcpyHostToDevice,
                                h->stream));
    if ((rc = launch_dl_to_panel(h, h->d_DL, h->d_DL + h->ndz))) return rc;
    const double* ds = nullptr;
    if ((rc = upload_signs(h, signs, &ds))) return rc;
    double* keep = h->d_signs;
    h->d_signs = const_cast<double*>(ds);
    if ((rc = init_info(h))) { h->d_signs = keep; return rc; }
    rc = launch_factor(h);
    h->d_signs = keep;
    if (rc) return rc;
    if ((rc = launch_panel_to_dl(h, h->d_DL, h->d_DL + h->ndz))) return rc;
    if (h->ndz)
        MF_CUDA(cudaMemcpyAsync(Dval, h->d_DL, sizeof(double) * h->ndz, cudaMemcpyDeviceToHost, h->stream));
    if (h->nlz)
        MF_CUDA(cudaMemcpyAsync(Lval, h->d_DL + h->ndz, sizeof(double) * h->nlz, cudaMemcpyDeviceToHost,
                                h->stream));
    if (h->diag && h->n)
        MF_CUDA(cudaMemcpyAsync(d, h->d_d, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
    return read_info(h, info);
}

static int solve_chunks(mf_handle* h, const int64_t* dperm, double* hostB, double* devB, int64_t nrhs, int64_t ldb) {
    int rc;
    for (int64_t c0 = 0; c0 < nrhs; c0 += h->nrhs_cap) {
        int64_t nc = std::min<int64_t>(h->nrhs_cap, nrhs - c0);
        if (hostB) {
            if (dperm) {
                MF_CUDA(cudaMemcpy2DAsync(h->d_B, sizeof(double) * h->n, hostB + c0 * ldb, sizeof(double) * ldb,
                                          sizeof(double) * h->n, nc, cudaMemcpyHostToDevice, h->stream));
                if ((rc = launch_permute_in(h, h->d_B, h->n, dperm, nc))) return rc;
            } else {
                MF_CUDA(cudaMemcpy2DAsync(h->d_C, sizeof(double) * h->n, hostB + c0 * ldb, sizeof(double) * ldb,
                                          sizeof(double) * h->n, nc, cudaMemcpyHostToDevice, h->stream));
            }
        } else {
            if ((rc = launch_permute_in(h, devB + c0 * ldb, ldb, dperm, nc))) return rc;
        }
        if ((rc = launch_solve(h, nc))) return rc;
        if (hostB) {
            if (dperm) {
                if ((rc = launch_permute_out(h, h->d_B, h->n, dperm, nc))) return rc;
                MF_CUDA(cudaMemcpy2DAsync(hostB + c0 * ldb, sizeof(double) * ldb, h->d_B, sizeof(double) * h->n,
                                          sizeof(double) * h->n, nc, cudaMemcpyDeviceToHost, h->stream));
            } else {
                MF_CUDA(cudaMemcpy2DAsync(hostB + c0 * ldb, sizeof(double) * ldb, h->d_C, sizeof(double) * h->n,
                                          sizeof(double) * h->n, nc, cudaMemcpyDeviceToHost, h->stream));
            }
        } else {
            if ((rc = launch_permute_out(h, devB + c0 * ldb, ldb, dperm, nc))) return rc;
        }
    }
    return 0;
}

// A bounded device wait that ran out (the tensor-core pipeline's mbarriers,
// err 1; the solve chain's progress counters, err 2) leaves *d_err set and
// the result incomplete: report it after the call's last synchronization.
static int wait_error(mf_handle* h, const char* where) {
    int err = 0;
    MF_CUDA(cudaMemcpyAsync(&err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    MF_CUDA(cudaStreamSynchronize(h->stream));
    if (!err) return 0;
    set_error(std::string(where) + (err == 2 ? ": a solve-chain wait timed out" : ": a tensor-core wait timed out"));
    return -3;
}

int mf_div_impl(mf_handle* h, double* B, int64_t nrhs, int64_t ldb) {
    if (!h || nrhs < 0 || (nrhs > 0 && (!B || ldb < h->n))) { set_error("mf_div_impl: bad arguments"); return -1; }
    DeviceGuard g(h->device);
    int rc = solve_chunks(h, nullptr, B, nullptr, nrhs, ldb);
    if (rc) return rc;
    return wait_error(h, "mf_div_impl");
}

int mf_set_assembly(mf_handle* h, int64_t nnz, const int64_t* slot) {
    if (!h || nnz < 0 || (nnz > 0 && !slot)) { set_error("mf_set_assembly: bad arguments"); return -1; }
    DeviceGuard g(h->device);
    std::vector<int64_t> pslot(nnz);
    const int64_t ndz = h->ndz, nlz = h->nlz;
    std::vector<char> seen;
    for (int64_t k = 0; k < nnz; ++k) {
        int64_t s = slot[k];
        if (s < 0 || s >= ndz + nlz) { set_error("mf_set_assembly: slot out of range"); return -2; }
        int64_t p;
        if (s < ndz) {
            int64_t j = std::upper_bound(h->h_Dptr.begin(), h->h_Dptr.end(), s) - h->h_Dptr.begin() - 1;
            const RefFront& rf = h->h_ref[j];
            const Front& f = h->h_fronts[rf.exec];
            int64_t loc = s - rf.Dptr;
            int64_t r = loc % rf.nn, c = loc / rf.nn;
            if (r < c) { set_error("mf_set_assembly: slot in the upper triangle of a diagonal block"); return -2; }
            int64_t off = rf.res0 - f.col0;
            p = f.poff + (off + r) + (off + c) * (int64_t)f.ldp;
        } else {
            int64_t s2 = s - ndz;
            int64_t j = std::upper_bound(h->h_Lptr.begin(), h->h_Lptr.end(), s2) - h->h_Lptr.begin() - 1;
            const RefFront& rf = h->h_ref[j];
            const Front& f = h->h_fronts[rf.exec];
            int64_t loc = s2 - rf.Lptr;
            int64_t a = loc % rf.na, c = loc / rf.na;
            int64_t off = rf.res0 - f.col0;
            p = f.poff + h->h_sepmap[rf.sep0 + a] + (off + c) * (int64_t)f.ldp;
        }
        pslot[k] = p;
    }
    {
        // slots must be distinct: the scatter writes each entry once
        std::vector<int64_t> tmp(pslot);
        std::sort(tmp.begin(), tmp.end());
        if (std::adjacent_find(tmp.begin(), tmp.end()) != tmp.end()) {
            set_error("mf_set_assembly: duplicate slots");
            return -2;
        }
    }
    // permuted (row, col) of every stored value, diagonal positions and the
    // CSR of the whole symmetric matrix (residuals of the mixed path)
    const int64_t n = h->n;
    std::vector<int32_t> rowi(nnz), coli(nnz);
    std::vector<int64_t> dslot(n, -1);
    for (int64_t k = 0; k < nnz; ++k) {
        int64_t s = slot[k];
        int64_t r, c;
        if (s < ndz) {
            int64_t j = std::upper_bound(h->h_Dptr.begin(), h->h_Dptr.end(), s) - h->h_Dptr.begin() - 1;
            const RefFront& rf = h->h_ref[j];
            int64_t loc = s - rf.Dptr;
            r = rf.res0 + loc % rf.nn;
            c = rf.res0 + loc / rf.nn;
        } else {
            int64_t s2 = s - ndz;
            int64_t j = std::upper_bound(h->h_Lptr.begin(), h->h_Lptr.end(), s2) - h->h_Lptr.begin() - 1;
            const RefFront& rf = h->h_ref[j];
            int64_t loc = s2 - rf.Lptr;
            r = h->h_septgt[rf.sep0 + loc % rf.na];
            c = rf.res0 + loc / rf.na;
        }
        rowi[k] = (int32_t)r;
        coli[k] = (int32_t)c;
        if (r == c) dslot[r] = k;
    }
    std::vector<int64_t> cptr(n + 1, 0);
    for (int64_t k = 0; k < nnz; ++k) {
        cptr[rowi[k] + 1]++;
        if (rowi[k] != coli[k]) cptr[coli[k] + 1]++;
    }
    for (int64_t i = 0; i < n; ++i) cptr[i + 1] += cptr[i];
    const int64_t nfull = cptr[n];
    std::vector<int32_t> ccol(nfull);
    std::vector<int64_t> csrc(nfull);
    {
        std::vector<int64_t> pos(cptr.begin(), cptr.end() - 1);
        for (int64_t k = 0; k < nnz; ++k) {
            int64_t r = rowi[k], c = coli[k];
            ccol[pos[r]] = (int32_t)c; csrc[pos[r]++] = k;
            if (r != c) { ccol[pos[c]] = (int32_t)r; csrc[pos[c]++] = k; }
        }
    }
    std::lock_guard<std::recursive_mutex> lk(device_mutex());
    void* olds[] = {h->d_pslot, h->d_nz, h->d_nzrow, h->d_nzcol, h->d_dslot, h->d_csrptr, h->d_csrcol, h->d_csrsrc};
    for (void* o : olds)
        if (o) cudaFree(o);
    h->d_pslot = nullptr; h->d_nz = nullptr; h->d_nzrow = nullptr; h->d_nzcol = nullptr; h->d_dslot = nullptr;
    h->d_csrptr = nullptr; h->d_csrcol = nullptr; h->d_csrsrc = nullptr;
    int64_t tot = 0;
    int rc;
    if ((rc = dalloc(h, &h->d_pslot, std::max<int64_t>(nnz, 1), &tot))) return rc;
    if ((rc = dalloc(h, &h->d_nz, std::max<int64_t>(nnz, 1), &tot))) return rc;
    if ((rc = dalloc(h, &h->d_nzrow, std::max<int64_t>(nnz, 1), &tot))) return rc;
    if ((rc = dalloc(h, &h->d_nzcol, std::max<int64_t>(nnz, 1), &tot))) return rc;
    if ((rc = dalloc(h, &h->d_dslot, std::max<int64_t>(n, 1), &tot))) return rc;
    if ((rc = dalloc(h, &h->d_csrptr, n + 1, &tot))) return rc;
    if ((rc = dalloc(h, &h->d_csrcol, std::max<int64_t>(nfull, 1), &tot))) return rc;
    if ((rc = dalloc(h, &h->d_csrsrc, std::max<int64_t>(nfull, 1), &tot))) return rc;
    if (nnz) {
        MF_CUDA(cudaMemcpy(h->d_pslot, pslot.data(), sizeof(int64_t) * nnz, cudaMemcpyHostToDevice));
        MF_CUDA(cudaMemcpy(h->d_nzrow, rowi.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice));
        MF_CUDA(cudaMemcpy(h->d_nzcol, coli.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice));
    }
    if (n) MF_CUDA(cudaMemcpy(h->d_dslot, dslot.data(), sizeof(int64_t) * n, cudaMemcpyHostToDevice));
    MF_CUDA(cudaMemcpy(h->d_csrptr, cptr.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice));
    if (nfull) {
        MF_CUDA(cudaMemcpy(h->d_csrcol, ccol.data(), sizeof(int32_t) * nfull, cudaMemcpyHostToDevice));
        MF_CUDA(cudaMemcpy(h->d_csrsrc, csrc.data(), sizeof(int64_t) * nfull, cudaMemcpyHostToDevice));
    }
    h->bytes += tot;
    h->nnz_full = nfull;
    h->cur_nz = nullptr;
    h->nnz = nnz;
    return 0;
}

int mf_assemble(mf_handle* h, const double* nzval) {
    if (!h || (h->nnz && !nzval)) { set_error("mf_assemble: bad arguments"); return -1; }
    if (!h->d_pslot) { set_error("mf_assemble: call mf_set_assembly first"); return -1; }
    DeviceGuard g(h->device);
    if (h->nnz)
        MF_CUDA(cudaMemcpyAsync(h->d_nz, nzval, sizeof(double) * h->nnz, cudaMemcpyHostToDevice, h->stream));
    h->cur_nz = h->d_nz;
    if (h->mixed) return 0;  // the mixed factorization assembles its own scaled FP32 panels
    return launch_assemble(h, h->d_nz);
}

int mf_assemble_device(mf_handle* h, const double* nzval_dev) {
    if (!h || (h->nnz && !nzval_dev)) { set_error("mf_assemble_device: bad arguments"); return -1; }
    if (!h->d_pslot) { set_error("mf_assemble_device: call mf_set_assembly first"); return -1; }
    DeviceGuard g(h->device);
    h->cur_nz = nzval_dev;
    if (h->mixed) return 0;
    return launch_assemble(h, nzval_dev);
}

int mf_factorize(mf_handle* h, const double* signs, int64_t* info) {
    if (!h) { set_error("null handle"); return -1; }
    DeviceGuard g(h->device);
    const double* ds = nullptr;
    int rc;
    if ((rc = ensure_fp64(h))) return rc;
    if ((rc = upload_signs(h, signs, &ds))) return rc;
    double* keep = h->d_signs;
    h->d_signs = const_cast<double*>(ds);
    if ((rc = init_info(h))) { h->d_signs = keep; return rc; }
    rc = launch_factor(h);
    h->d_signs = keep;
    if (rc) return rc;
    if (info) return read_info(h, info);
    return 0;
}

int mf_solve(mf_handle* h, double* B, int64_t nrhs, int64_t ldb, const int64_t* perm) {
    if (!h || nrhs < 0 || (nrhs > 0 && (!B || ldb < h->n))) { set_error("mf_solve: bad arguments"); return -1; }
    DeviceGuard g(h->device);
    if (perm && h->n) {
        for (int64_t i = 0; i < h->n; ++i)
            if (perm[i] < 0 || perm[i] >= h->n) { set_error("mf_solve: perm out of range"); return -2; }
        MF_CUDA(cudaMemcpyAsync(h->d_perm, perm, sizeof(int64_t) * h->n, cudaMemcpyHostToDevice, h->stream));
    }
    int rc = solve_chunks(h, h->d_perm, B, nullptr, nrhs, ldb);
    if (rc) return rc;
    return wait_error(h, "mf_solve");
}

int mf_solve_device(mf_handle* h, double* B_dev, int64_t nrhs, int64_t ldb, const int64_t* perm_dev) {
    if (!h || nrhs < 0 || (nrhs > 0 && (!B_dev || ldb < h->n))) {
        set_error("mf_solve_device: bad arguments");
        return -1;
    }
    DeviceGuard g(h->device);
    return solve_chunks(h, perm_dev ? perm_dev : h->d_perm, nullptr, B_dev, nrhs, ldb);
}

}  // extern "C"

static int64_t fp64_bytes(const mf_handle* h) {
    return (int64_t)sizeof(double) * (std::max<int64_t>(h->npanel, 0) + std::max<int64_t>(h->ninv, 1) +
                                      std::max<int64_t>(h->ninv2, 1) + std::max<int64_t>(h->nmval, 0));
}

int mf::have_fp64(const mf_handle* h) { return h->d_P != nullptr || h->npanel == 0; }

int mf::ensure_fp64(mf_handle* h) {
    std::lock_guard<std::recursive_mutex> lk(device_mutex());
    if (have_fp64(h) && (h->d_M || h->nmval <= 0)) return 0;
    int64_t tot = 0;
    int rc = 0;
    rc = rc ? rc : dalloc(h, &h->d_P, h->npanel, &tot);
    rc = rc ? rc : dalloc(h, &h->d_inv, std::max<int64_t>(h->ninv, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_inv2, std::max<int64_t>(h->ninv2, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_M, h->nmval, &tot);
    if (rc) {
        for (double** p : {&h->d_P, &h->d_inv, &h->d_inv2, &h->d_M}) {
            if (*p) cudaFree(*p);
            *p = nullptr;
        }
        return rc;
    }
    if (h->npanel) MF_CUDA(cudaMemset(h->d_P, 0, sizeof(double) * h->npanel));
    h->bytes += tot;
    release_graphs(h);  // captured launches hold the buffers' addresses
    return 0;
}

extern "C" {

int mf_enable_mixed(mf_handle* h) {
    if (!h) { set_error("null handle"); return -1; }
    if (!h->d_csrptr) { set_error("mf_enable_mixed: call mf_set_assembly first"); return -1; }
    if (h->mixed) return 0;
    DeviceGuard g(h->device);
    std::lock_guard<std::recursive_mutex> lk(device_mutex());
    // the FP64 factor storage is only needed if a factorization falls back
    // to FP64: release it first (ensure_fp64 brings it back on demand); only
    // this handle's stream can be using it
    MF_CUDA(cudaStreamSynchronize(h->stream));
    release_graphs(h);
    if (h->d_P) {
        for (double** p : {&h->d_P, &h->d_inv, &h->d_inv2, &h->d_M}) {
            if (*p) cudaFree(*p);
            *p = nullptr;
        }
        h->bytes -= fp64_bytes(h);
    }
    int64_t tot = 0;
    int rc = 0;
    const int64_t n = h->n, cap = h->nrhs_cap;
    rc = rc ? rc : dalloc(h, &h->f32.P, std::max<int64_t>(h->npanel, 1), &tot);
    if (h->tc_split)
        rc = rc ? rc : dalloc(h, &h->f32.split, std::max<int64_t>(h->nsplit_units * kSplitUnitFloats, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->f32.M, std::max<int64_t>(h->nmval, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->f32.inv, std::max<int64_t>(h->ninv, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->f32.inv2, std::max<int64_t>(h->ninv2, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->f32.d, std::max<int64_t>(n, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->f32.R, std::max<int64_t>(h->nrval_per_rhs * cap, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->f32.W, std::max<int64_t>(n * cap, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->f32.part, std::max<int64_t>(h->nbwd_part * kNB * 16, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->f32.C, std::max<int64_t>(n * cap, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_scale, std::max<int64_t>(n, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_iv, std::max<int64_t>(6 * n * cap, 1), &tot);
    rc = rc ? rc : dalloc(h, &h->d_red, kRedDoubles, &tot);
    if (rc) return rc;
    h->bytes += tot;
    h->mixed = true;
    return 0;
}

int mf_factorize_mixed(mf_handle* h, const double* signs, int64_t* info, int* used_fp64) {
    if (!h) { set_error("null handle"); return -1; }
    if (!h->mixed) { set_error("mf_factorize_mixed: call mf_enable_mixed first"); return -1; }
    if (!h->cur_nz) { set_error("mf_factorize_mixed: no values (mf_assemble)"); return -1; }
    if (h->reg.delta >= 0.0) {
        set_error("mf_factorize_mixed: dynamic regularization applies to the FP64 factorization (mf_factorize)");
        return -1;
    }
    DeviceGuard g(h->device);
    const double* ds = nullptr;
    int rc;
    if ((rc = upload_signs(h, signs, &ds))) return rc;
    double* keep = h->d_signs;
    h->d_signs = const_cast<double*>(ds);
    int64_t inf = 0;
    h->fp64_current = false;  // whatever the FP64 storage holds is an older matrix
    rc = launch_assemble_mixed(h, h->cur_nz);
    if (!rc) rc = init_info(h);
    if (!rc) rc = launch_factor_mixed(h);
    if (!rc) rc = read_info(h, &inf);
    h->mixed_fallback = false;
    if (!rc && inf != 0) {
        // FP32 rejected a pivot: factor in FP64 (the refinement then takes one
        // FP64 solve), so an FP32 breakdown is never reported as a failure
        rc = ensure_fp64(h);
        if (!rc) rc = launch_assemble(h, h->cur_nz);
        if (!rc) rc = init_info(h);
        if (!rc) rc = launch_factor(h);
        if (!rc) rc = read_info(h, &inf);
        h->mixed_fallback = true;
    }
    if (!rc) rc = launch_anorm(h);
    h->d_signs = keep;
    if (rc) return rc;
    int err = 0;
    MF_CUDA(cudaMemcpyAsync(&err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    MF_CUDA(cudaStreamSynchronize(h->stream));
    if (err) {
        set_error("mf_factorize_mixed: a tensor-core wait timed out");
        return -3;
    }
    if (info) *info = inf;
    if (used_fp64) *used_fp64 = h->mixed_fallback ? 1 : 0;
    return 0;
}

int mf_autotune(mf_handle* h, int reps, double* ms) {
    if (!h) { set_error("null handle"); return -1; }
    if (!h->mixed) { set_error("mf_autotune: call mf_enable_mixed first"); return -1; }
    if (!h->cur_nz) { set_error("mf_autotune: no values (mf_assemble)"); return -1; }
    DeviceGuard g(h->device);
    const size_t nl = h->levels.size();
    reps = std::max(1, reps);
    // best[v][L]: the fastest of `reps` timed runs (after one warm-up run) of
    // variant v (0 = FFMA tiles, 1 = tcgen05 tiles) on level L
    std::vector<double> steps_best[2], syrk_best[2];
    const bool keep_profile = h->profile;
    h->profile = false;
    h->tuning = true;
    int rc = 0;
    int64_t inf = 0;
    for (int v = 0; v < 2 && !rc; ++v) {
        for (Level& lv : h->levels) lv.tc_steps = lv.tc_syrk = v;
        steps_best[v].assign(nl, 1e30);
        syrk_best[v].assign(nl, 1e30);
        for (int r = 0; r <= reps && !rc; ++r) {
            rc = launch_assemble_mixed(h, h->cur_nz);
            if (!rc) rc = init_info(h);
            if (!rc) rc = launch_factor_mixed(h);
            if (!rc) rc = read_info(h, &inf);
            if (rc || r == 0) continue;
            for (size_t L = 0; L < nl; ++L) {
                steps_best[v][L] = std::min(steps_best[v][L], h->tune_steps_ms[L]);
                syrk_best[v][L] = std::min(syrk_best[v][L], h->tune_syrk_ms[L]);
            }
        }
    }
    h->tuning = false;
    h->profile = keep_profile;
    double tot[3] = {0.0, 0.0, 0.0};
    for (size_t L = 0; L < nl && !rc; ++L) {
        Level& lv = h->levels[L];
        lv.tc_steps = steps_best[1][L] <= steps_best[0][L];
        lv.tc_syrk = syrk_best[1][L] <= syrk_best[0][L];
        tot[0] += steps_best[1][L] + syrk_best[1][L];
        tot[1] += steps_best[0][L] + syrk_best[0][L];
        tot[2] += std::min(steps_best[0][L], steps_best[1][L]) + std::min(syrk_best[0][L], syrk_best[1][L]);
    }
    if (rc) {
        for (Level& lv : h->levels) lv.tc_steps = lv.tc_syrk = 1;
        return rc;
    }
    // captured factorizations hold the previous kernel choice
    release_graphs(h);
    if (ms) {
        int64_t n_steps = 0, n_syrk = 0;
        for (const Level& lv : h->levels) { n_steps += lv.tc_steps; n_syrk += lv.tc_syrk; }
        ms[0] = tot[0];
        ms[1] = tot[1];
        ms[2] = tot[2];
        ms[3] = (double)n_steps;
        ms[4] = (double)n_syrk;
        ms[5] = (double)nl;
    }
    return 0;
}

int mf_kernel_choice(const mf_handle* h, int32_t* tc_steps, int32_t* tc_syrk) {
    if (!h) { set_error("null handle"); return -1; }
    for (size_t L = 0; L < h->levels.size(); ++L) {
        if (tc_steps) tc_steps[L] = h->levels[L].tc_steps;
        if (tc_syrk) tc_syrk[L] = h->levels[L].tc_syrk;
    }
    return 0;
}

int mf_set_kernel_choice(mf_handle* h, const int32_t* tc_steps, const int32_t* tc_syrk) {
    if (!h) { set_error("null handle"); return -1; }
    for (size_t L = 0; L < h->levels.size(); ++L) {
        if (tc_steps) h->levels[L].tc_steps = tc_steps[L] != 0;
        if (tc_syrk) h->levels[L].tc_syrk = tc_syrk[L] != 0;
    }
    release_graphs(h);
    return 0;
}

static int refined_chunks(mf_handle* h, double* hostB, double* devB, int64_t nrhs, int64_t ldb, const int64_t* dperm,
                          double tol, int maxit, int* iters, double* eta) {
    const int64_t cap = (int64_t)h->n * h->nrhs_cap;
    double* bp = h->d_iv;
    double* xp = h->d_iv + cap;
    int worst_it = 0;
    double worst_eta = 0.0;
    int rc;
    for (int64_t c0 = 0; c0 < nrhs; c0 += h->nrhs_cap) {
        int64_t nc = std::min<int64_t>(h->nrhs_cap, nrhs - c0);
        if (hostB) {
            MF_CUDA(cudaMemcpy2DAsync(h->d_B, sizeof(double) * h->n, hostB + c0 * ldb, sizeof(double) * ldb,
                                      sizeof(double) * h->n, nc, cudaMemcpyHostToDevice, h->stream));
            if ((rc = launch_permute_to(h, h->d_B, h->n, dperm, nc, bp))) return rc;
        } else {
            if ((rc = launch_permute_to(h, devB + c0 * ldb, ldb, dperm, nc, bp))) return rc;
        }
        int it = 0;
        double e = 0.0;
        if ((rc = refine(h, bp, xp, (int)nc, tol, maxit, &it, &e))) return rc;
        worst_it = std::max(worst_it, it);
        worst_eta = std::max(worst_eta, e);
        if (hostB) {
            if ((rc = launch_permute_from(h, h->d_B, h->n, dperm, nc, xp))) return rc;
            MF_CUDA(cudaMemcpy2DAsync(hostB + c0 * ldb, sizeof(double) * ldb, h->d_B, sizeof(double) * h->n,
                                      sizeof(double) * h->n, nc, cudaMemcpyDeviceToHost, h->stream));
        } else {
            if ((rc = launch_permute_from(h, devB + c0 * ldb, ldb, dperm, nc, xp))) return rc;
        }
    }
    if (iters) *iters = worst_it;
    if (eta) *eta = worst_eta;
    return 0;
}

int mf_solve_refined(mf_handle* h, double* B, int64_t nrhs, int64_t ldb, const int64_t* perm, double tol, int maxit,
                     int* iters, double* eta) {
    if (!h || nrhs < 0 || (nrhs > 0 && (!B || ldb < h->n)) || maxit < 1) {
        set_error("mf_solve_refined: bad arguments");
        return -1;
    }
    if (!h->mixed) { set_error("mf_solve_refined: call mf_enable_mixed and mf_factorize_mixed first"); return -1; }
    DeviceGuard g(h->device);
    if (perm && h->n) {
        for (int64_t i = 0; i < h->n; ++i)
            if (perm[i] < 0 || perm[i] >= h->n) { set_error("mf_solve_refined: perm out of range"); return -2; }
        MF_CUDA(cudaMemcpyAsync(h->d_perm, perm, sizeof(int64_t) * h->n, cudaMemcpyHostToDevice, h->stream));
    }
    int rc = refined_chunks(h, B, nullptr, nrhs, ldb, h->d_perm, tol, maxit, iters, eta);
    if (rc) return rc;
    return wait_error(h, "mf_solve_refined");
}

int mf_solve_refined_device(mf_handle* h, double* B_dev, int64_t nrhs, int64_t ldb, const int64_t* perm_dev,
                            double tol, int maxit, int* iters, double* eta) {
    if (!h || nrhs < 0 || (nrhs > 0 && (!B_dev || ldb < h->n)) || maxit < 1) {
        set_error("mf_solve_refined_device: bad arguments");
        return -1;
    }
    if (!h->mixed) { set_error("mf_solve_refined_device: call mf_enable_mixed first"); return -1; }
    DeviceGuard g(h->device);
    const int rc = refined_chunks(h, nullptr, B_dev, nrhs, ldb, perm_dev ? perm_dev : h->d_perm, tol, maxit, iters, eta);
    return rc ? rc : wait_error(h, "mf_solve_refined_device");
}

int mf_set_segments(mf_handle* h, int64_t nseg, const int64_t* segptr) {
    if (!h || nseg < 0 || (nseg > 0 && !segptr)) { set_error("mf_set_segments: bad arguments"); return -1; }
    if (nseg > 0) {
        if (segptr[0] != 0 || segptr[nseg] != h->n) {
            set_error("mf_set_segments: segments must start at row 0 and end at row n");
            return -1;
        }
        for (int64_t s = 0; s < nseg; ++s)
            if (segptr[s + 1] < segptr[s]) { set_error("mf_set_segments: boundaries must not decrease"); return -1; }
    }
    DeviceGuard g(h->device);
    std::lock_guard<std::recursive_mutex> lk(device_mutex());
    // only this handle's work can use the buffers replaced below
    MF_CUDA(cudaStreamSynchronize(h->stream));
    release_graphs(h);
    for (void* p : {(void*)h->d_segptr, (void*)h->d_segred, (void*)h->d_segeta, (void*)h->d_chunkrow,
                    (void*)h->d_chunkseg, (void*)h->d_segchunk, (void*)h->d_rowseg, (void*)h->d_chunkred,
                    (void*)h->d_segsc})
        if (p) cudaFree(p);
    h->d_segptr = nullptr; h->d_segred = nullptr; h->d_segeta = nullptr;
    h->d_chunkrow = nullptr; h->d_chunkseg = nullptr; h->d_segchunk = nullptr; h->d_rowseg = nullptr;
    h->d_chunkred = nullptr; h->d_segsc = nullptr;
    h->nseg = 0;
    h->nchunk = 0;
    h->h_segptr.clear();
    if (nseg == 0) return 0;
    // chunks of at most kChunkRows rows, never across a segment boundary
    std::vector<int64_t> chunkrow{0}, segchunk{0};
    std::vector<int32_t> chunkseg, rowseg((size_t)h->n);
    for (int64_t s = 0; s < nseg; ++s) {
        for (int64_t r = segptr[s]; r < segptr[s + 1]; r += kChunkRows) {
            chunkrow.push_back(std::min<int64_t>(segptr[s + 1], r + kChunkRows));
            chunkseg.push_back((int32_t)s);
        }
        segchunk.push_back((int64_t)chunkseg.size());
        for (int64_t r = segptr[s]; r < segptr[s + 1]; ++r) rowseg[(size_t)r] = (int32_t)s;
    }
    const int64_t nch = (int64_t)chunkseg.size();
    int64_t tot = 0;
    int rc = dalloc(h, &h->d_segptr, nseg + 1, &tot);
    if (!rc) rc = dalloc(h, &h->d_segred, nseg * kSegRed, &tot);
    if (!rc) rc = dalloc(h, &h->d_segeta, nseg, &tot);
    if (!rc) rc = dalloc(h, &h->d_chunkrow, nch + 1, &tot);
    if (!rc) rc = dalloc(h, &h->d_chunkseg, std::max<int64_t>(nch, 1), &tot);
    if (!rc) rc = dalloc(h, &h->d_segchunk, nseg + 1, &tot);
    if (!rc) rc = dalloc(h, &h->d_rowseg, std::max<int64_t>(h->n, 1), &tot);
    if (!rc) rc = dalloc(h, &h->d_chunkred, std::max<int64_t>(nch, 1) * kChunkRed, &tot);
    if (!rc) rc = dalloc(h, &h->d_segsc, nseg * 80, &tot);
    if (rc) return rc;
    MF_CUDA(cudaMemcpy(h->d_segptr, segptr, sizeof(int64_t) * (nseg + 1), cudaMemcpyHostToDevice));
    MF_CUDA(cudaMemset(h->d_segeta, 0, sizeof(double) * nseg));
    MF_CUDA(cudaMemcpy(h->d_chunkrow, chunkrow.data(), sizeof(int64_t) * (nch + 1), cudaMemcpyHostToDevice));
    if (nch) MF_CUDA(cudaMemcpy(h->d_chunkseg, chunkseg.data(), sizeof(int32_t) * nch, cudaMemcpyHostToDevice));
    MF_CUDA(cudaMemcpy(h->d_segchunk, segchunk.data(), sizeof(int64_t) * (nseg + 1), cudaMemcpyHostToDevice));
    if (h->n) MF_CUDA(cudaMemcpy(h->d_rowseg, rowseg.data(), sizeof(int32_t) * h->n, cudaMemcpyHostToDevice));
    h->bytes += tot;
    h->nseg = nseg;
    h->nchunk = nch;
    h->h_segptr.assign(segptr, segptr + nseg + 1);
    return 0;
}

int mf_segment_errors(mf_handle* h, double* eta) {
    if (!h || (h->nseg > 0 && !eta)) { set_error("mf_segment_errors: bad arguments"); return -1; }
    if (h->nseg == 0) return 0;
    DeviceGuard g(h->device);
    MF_CUDA(cudaMemcpyAsync(eta, h->d_segeta, sizeof(double) * h->nseg, cudaMemcpyDeviceToHost, h->stream));
    MF_CUDA(cudaStreamSynchronize(h->stream));
    return 0;
}

int mf_get_factor_mixed(mf_handle* h, double* Dval, double* Lval, double* d, double* scale) {
    if (!h || !h->mixed) { set_error("mf_get_factor_mixed: no mixed factorization"); return -1; }
    DeviceGuard g(h->device);
    int rc;
    if (!h->d_DL) {
        int64_t tot = 0;
        if ((rc = dalloc(h, &h->d_DL, std::max<int64_t>(h->ndz + h->nlz, 1), &tot))) return rc;
    }
    if ((rc = launch_panel32_to_dl(h, h->d_DL, h->d_DL + h->ndz))) return rc;
    if (Dval && h->ndz)
        MF_CUDA(cudaMemcpyAsync(Dval, h->d_DL, sizeof(double) * h->ndz, cudaMemcpyDeviceToHost, h->stream));
    if (Lval && h->nlz)
        MF_CUDA(cudaMemcpyAsync(Lval, h->d_DL + h->ndz, sizeof(double) * h->nlz, cudaMemcpyDeviceToHost, h->stream));
    if (d && h->n) {
        std::vector<float> tmp(h->n);
        MF_CUDA(cudaMemcpyAsync(tmp.data(), h->f32.d, sizeof(float) * h->n, cudaMemcpyDeviceToHost, h->stream));
        MF_CUDA(cudaStreamSynchronize(h->stream));
        for (int64_t i = 0; i < h->n; ++i) d[i] = tmp[i];
    }
    if (scale && h->n)
        MF_CUDA(cudaMemcpyAsync(scale, h->d_scale, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
    MF_CUDA(cudaStreamSynchronize(h->stream));
    return 0;
}

int mf_get_factor(mf_handle* h, double* Dval, double* Lval, double* d) {
    if (!h) { set_error("null handle"); return -1; }
    DeviceGuard g(h->device);
    int rc;
    if (Dval || Lval) {
        if (!h->d_DL) {
            int64_t tot = 0;
            if ((rc = dalloc(h, &h->d_DL, std::max<int64_t>(h->ndz + h->nlz, 1), &tot))) return rc;
        }
        if ((rc = launch_panel_to_dl(h, h->d_DL, h->d_DL + h->ndz))) return rc;
        if (Dval && h->ndz)
            MF_CUDA(cudaMemcpyAsync(Dval, h->d_DL, sizeof(double) * h->ndz, cudaMemcpyDeviceToHost, h->stream));
        if (Lval && h->nlz)
            MF_CUDA(cudaMemcpyAsync(Lval, h->d_DL + h->ndz, sizeof(double) * h->nlz, cudaMemcpyDeviceToHost,
                                    h->stream));
    }
    if (d && h->n) MF_CUDA(cudaMemcpyAsync(d, h->d_d, sizeof(double) * h->n, cudaMemcpyDeviceToHost, h->stream));
    MF_CUDA(cudaStreamSynchronize(h->stream));
    return 0;
}

int mf_synchronize(mf_handle* h) {
    if (!h) { set_error("null handle"); return -1; }
    DeviceGuard g(h->device);
    return wait_error(h, "mf_synchronize");
}

int mf_info(const mf_handle* h, int64_t* out) {
    if (!h || !out) { set_error("mf_info: bad arguments"); return -1; }
    out[0] = h->n; out[1] = h->nfr; out[2] = h->ndz; out[3] = h->nlz;
    out[4] = h->npanel; out[5] = h->nmval; out[6] = h->bytes;
    out[7] = (int64_t)h->levels.size(); out[8] = h->nexec;
    return 0;
}

int mf_exec_sizes(const mf_handle* h, int64_t* nn, int64_t* na) {
    if (!h) { set_error("null handle"); return -1; }
    for (int64_t e = 0; e < h->nexec; ++e) {
        if (nn) nn[e] = h->h_fronts[e].nn;
        if (na) na[e] = h->h_fronts[e].na;
    }
    return 0;
}

int mf_set_regularization(mf_handle* h, int mode, double delta, double epsilon) {
    if (!h || (mode != 0 && mode != 1)) { set_error("mf_set_regularization: bad arguments"); return -1; }
    if (mode == 0) {
        h->reg = Reg();
    } else {
        // defaults of DynamicRegularization{Float64}: cbrt(eps), sqrt(eps)
        const double eps = 2.220446049250313e-16;
        h->reg.delta = delta < 0 ? std::cbrt(eps) : delta;
        h->reg.eps = epsilon < 0 ? std::sqrt(eps) : epsilon;
    }
    release_graphs(h);  // captured factorizations hold the previous rule
    return 0;
}

int mf_selinv(mf_handle* h) {
    if (!h) { set_error("null handle"); return -1; }
    DeviceGuard g(h->device);
    int rc = launch_selinv(h);
    if (rc) return rc;
    MF_CUDA(cudaStreamSynchronize(h->stream));
    return 0;
}

int mf_rescued(mf_handle* h, int64_t* count) {
    if (!h || !count) { set_error("mf_rescued: bad arguments"); return -1; }
    DeviceGuard g(h->device);
    int v = 0;
    MF_CUDA(cudaMemcpyAsync(&v, h->d_rescued, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    MF_CUDA(cudaStreamSynchronize(h->stream));
    *count = v;
    return 0;
}

int mf_logdet(mf_handle* h, double* logabsdet, double* sign) {
    if (!h || !logabsdet || !sign) { set_error("mf_logdet: bad arguments"); return -1; }
    DeviceGuard g(h->device);
    return launch_logdet(h, logabsdet, sign);
}

int mf_exec_parents(const mf_handle* h, int64_t* parent) {
    if (!h || (h->nexec && !parent)) { set_error("mf_exec_parents: bad arguments"); return -1; }
    for (int64_t e = 0; e < h->nexec; ++e) parent[e] = h->h_fronts[e].parent;
    return 0;
}

int mf_profile(mf_handle* h, int enable) {
    if (!h) { set_error("null handle"); return -1; }
    h->profile = enable != 0;
    h->times = KernelTimes();
    return 0;
}

int mf_kernel_times(const mf_handle* h, double* ms, int64_t* launches) {
    if (!h) { set_error("null handle"); return -1; }
    for (int k = 0; k < K_COUNT; ++k) {
        if (ms) ms[k] = h->times.ms[k];
        if (launches) launches[k] = h->times.launches[k];
    }
    return 0;
}

}  // extern "C"
