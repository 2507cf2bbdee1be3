// mf_solve_device_static: the FP64 device solve of mf_solve_device with its
// work buffers (child updates R, gathered right-hand sides W, solution block C,
// backward partial sums) carved out of one fixed device region instead of the
// handle's buffers.  The call makes no device allocation: the region is a
// file-scope __device__ array that exists from the moment the CUDA runtime
// loads this file's module on a device.
//
// Region size: kStaticSolveDoubles doubles (32 MiB).  A call needs, for a
// chunk of c = min(nrhs, 16) right-hand sides,
//   2*n*c + nrval_per_rhs*c + nbwd_part*64*16 doubles
// (each part rounded up to 256 bytes); larger problems are rejected with -1.
//
// Nothing in the region has to start at zero: every entry a solve reads is
// written earlier in the same call (C by the permutation, R and W by the
// forward gathers, the partial sums by the backward row chunks).
#include <cuda_runtime.h>

#include <cstdio>

#include "mf_internal.cuh"

namespace mf {

constexpr int64_t kStaticSolveDoubles = int64_t(1) << 22;  // 32 MiB
constexpr int64_t kChunkRhs = 16;  // right-hand sides per solve pass (the solve kernels' limit)

static __device__ __align__(256) double g_solve_region[kStaticSolveDoubles];

// Address of the region on the current device (the caller has made the
// handle's device current).  The lookup runs on every call rather than being
// cached, so a module reloaded after a device reset or in a new primary
// context is found at its new address; the first lookup on a device loads the
// module holding the region, which is why the first call should not run
// under stream capture.
static int region_address(double** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_solve_region);
    if (e != cudaSuccess) return cuda_fail(e, "mf_solve_device_static: cudaGetSymbolAddress");
    *out = static_cast<double*>(p);
    return 0;
}

static inline int64_t round256(int64_t doubles) { return (doubles + 31) / 32 * 32; }

struct CurrentDevice {  // makes `dev` current for the call, restores the caller's
    int prev = -1;
    explicit CurrentDevice(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~CurrentDevice() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace mf

using namespace mf;

extern "C" int mf_solve_device_static(mf_handle* h, double* B_dev, int64_t nrhs, int64_t ldb,
                                      const int64_t* perm_dev) {
    if (!h || nrhs < 0 || (nrhs > 0 && (!B_dev || ldb < h->n))) {
        set_error("mf_solve_device_static: bad arguments");
        return -1;
    }
    if (nrhs == 0 || h->n == 0) return 0;
    const int64_t n = h->n;
    const int64_t chunk = nrhs < kChunkRhs ? nrhs : kChunkRhs;
    const int64_t szC = round256(n * chunk), szW = szC;
    const int64_t szR = round256(h->nrval_per_rhs * chunk);
    const int64_t szPart = round256(h->nbwd_part * kNB * kChunkRhs);
    const int64_t need = szC + szW + szR + szPart;
    if (need > kStaticSolveDoubles) {
        char msg[256];
        snprintf(msg, sizeof(msg),
                 "mf_solve_device_static: this solve needs %lld doubles of work space (n=%lld, %lld right-hand "
                 "sides per chunk) but the static region holds %lld; use mf_solve_device",
                 (long long)need, (long long)n, (long long)chunk, (long long)kStaticSolveDoubles);
        set_error(msg);
        return -1;
    }
    CurrentDevice g(h->device);
    double* base = nullptr;
    int rc = region_address(&base);
    if (rc) return rc;
    double* C = base;
    double* W = C + szC;
    double* R = W + szW;
    double* part = R + szR;
    const int64_t* perm = perm_dev ? perm_dev : h->d_perm;
    for (int64_t c0 = 0; c0 < nrhs; c0 += chunk) {
        const int64_t nc = nrhs - c0 < chunk ? nrhs - c0 : chunk;
        if ((rc = launch_permute_to(h, B_dev + c0 * ldb, ldb, perm, nc, C))) return rc;
        if ((rc = launch_solve_with(h, nc, R, W, C, part))) return rc;
        if ((rc = launch_permute_from(h, B_dev + c0 * ldb, ldb, perm, nc, C))) return rc;
    }
    return 0;
}
