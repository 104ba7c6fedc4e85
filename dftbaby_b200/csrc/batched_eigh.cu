// dftbaby_b200: batched FP64 symmetric eigensolver for the ensemble solver
// (no counterpart in DFTBaby, which diagonalises one matrix at a time with
// LAPACK, DFTB2.py:1086, Solver.py:486, 772).
//
// The lockstep SCC and Davidson of many molecules need eigen-decompositions
// of a batch of equally sized symmetric matrices every iteration.  Issued one
// by one, each small solve is bound by launch and synchronisation latency;
// cuSOLVER's batched syev (cusolverDnXsyevBatched) runs the whole batch in one
// call.  The library is resolved at run time (dlopen / dlsym, reusing the copy
// the process has already loaded), so that a cuSOLVER without the batched
// routine makes this entry point return DFTB_ERR_UNSUPPORTED instead of
// keeping the library from loading.

#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <dlfcn.h>
#include <stdio.h>

#include <mutex>
#include <vector>

#include "dftbaby_b200.h"

namespace {

thread_local char g_eig_err[256] = "";

int eig_fail(int code, const char *what) {
    snprintf(g_eig_err, sizeof(g_eig_err), "%s", what);
    return code;
}

using create_t = cusolverStatus_t (*)(cusolverDnHandle_t *);
using setstream_t = cusolverStatus_t (*)(cusolverDnHandle_t, cudaStream_t);
using params_t = cusolverStatus_t (*)(cusolverDnParams_t *);
using bufsize_t = cusolverStatus_t (*)(cusolverDnHandle_t, cusolverDnParams_t, cusolverEigMode_t, cublasFillMode_t,
                                       int64_t, cudaDataType, const void *, int64_t, cudaDataType, const void *,
                                       cudaDataType, size_t *, size_t *, int64_t);
using syev_t = cusolverStatus_t (*)(cusolverDnHandle_t, cusolverDnParams_t, cusolverEigMode_t, cublasFillMode_t,
                                    int64_t, cudaDataType, void *, int64_t, cudaDataType, void *, cudaDataType,
                                    void *, size_t, void *, size_t, int *, int64_t);

struct Api {
    create_t create = nullptr;
    setstream_t set_stream = nullptr;
    params_t create_params = nullptr;
    bufsize_t bufsize = nullptr;
    syev_t syev = nullptr;
    bool ok = false;
};

Api &api() {
    static Api a;
    static std::once_flag once;
    std::call_once(once, [] {
        void *h = dlopen("libcusolver.so.11", RTLD_NOW | RTLD_NOLOAD);
        if (!h) h = dlopen("libcusolver.so.11", RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libcusolver.so", RTLD_NOW | RTLD_GLOBAL);
        if (!h) return;
        a.create = reinterpret_cast<create_t>(dlsym(h, "cusolverDnCreate"));
        a.set_stream = reinterpret_cast<setstream_t>(dlsym(h, "cusolverDnSetStream"));
        a.create_params = reinterpret_cast<params_t>(dlsym(h, "cusolverDnCreateParams"));
        a.bufsize = reinterpret_cast<bufsize_t>(dlsym(h, "cusolverDnXsyevBatched_bufferSize"));
        a.syev = reinterpret_cast<syev_t>(dlsym(h, "cusolverDnXsyevBatched"));
        a.ok = a.create && a.set_stream && a.create_params && a.bufsize && a.syev;
    });
    return a;
}

// One handle and parameter object per host thread and device (a handle carries a stream).
struct Ctx {
    cusolverDnHandle_t h = nullptr;
    cusolverDnParams_t p = nullptr;
    std::vector<char> host;
};

Ctx *context() {
    thread_local Ctx ctx[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    Ctx &c = ctx[dev];
    if (!c.h) {
        Api &a = api();
        if (a.create(&c.h) != CUSOLVER_STATUS_SUCCESS) return nullptr;
        if (a.create_params(&c.p) != CUSOLVER_STATUS_SUCCESS) return nullptr;
    }
    return &c;
}

}  // namespace

extern "C" {

const char *dftb_eigh_last_error(void) { return g_eig_err; }

int dftb_batched_eigh_workspace_size(int n, int batch, size_t *bytes) {
    if (n <= 0 || batch <= 0 || !bytes) return eig_fail(DFTB_ERR_BAD_SIZE, "batched_eigh: sizes");
    Api &a = api();
    if (!a.ok) return eig_fail(DFTB_ERR_UNSUPPORTED, "batched_eigh: this cuSOLVER has no cusolverDnXsyevBatched");
    Ctx *c = context();
    if (!c) return eig_fail(DFTB_ERR_CUDA, "batched_eigh: cannot create a cuSOLVER handle");
    size_t dbytes = 0, hbytes = 0;
    cusolverStatus_t s = a.bufsize(c->h, c->p, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, CUDA_R_64F,
                                   nullptr, n, CUDA_R_64F, nullptr, CUDA_R_64F, &dbytes, &hbytes, batch);
    if (s != CUSOLVER_STATUS_SUCCESS) {
        snprintf(g_eig_err, sizeof(g_eig_err), "batched_eigh: buffer-size query failed (status %d)", (int)s);
        return DFTB_ERR_UNSUPPORTED;
    }
    *bytes = dbytes;
    return DFTB_OK;
}

int dftb_batched_eigh(int n, int batch, double *A, double *W, void *work, size_t work_bytes, int *info, void *stream) {
    if (n <= 0 || batch <= 0) return eig_fail(DFTB_ERR_BAD_SIZE, "batched_eigh: sizes");
    if (!A || !W || !info) return eig_fail(DFTB_ERR_NULL, "batched_eigh: null");
    Api &a = api();
    if (!a.ok) return eig_fail(DFTB_ERR_UNSUPPORTED, "batched_eigh: this cuSOLVER has no cusolverDnXsyevBatched");
    Ctx *c = context();
    if (!c) return eig_fail(DFTB_ERR_CUDA, "batched_eigh: cannot create a cuSOLVER handle");
    if (a.set_stream(c->h, reinterpret_cast<cudaStream_t>(stream)) != CUSOLVER_STATUS_SUCCESS)
        return eig_fail(DFTB_ERR_CUDA, "batched_eigh: cannot set the stream");
    size_t dbytes = 0, hbytes = 0;
    cusolverStatus_t s = a.bufsize(c->h, c->p, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, CUDA_R_64F, A, n,
                                   CUDA_R_64F, W, CUDA_R_64F, &dbytes, &hbytes, batch);
    if (s != CUSOLVER_STATUS_SUCCESS) {
        snprintf(g_eig_err, sizeof(g_eig_err), "batched_eigh: buffer-size query failed (status %d)", (int)s);
        return DFTB_ERR_UNSUPPORTED;
    }
    if (work_bytes < dbytes || (dbytes && !work)) return eig_fail(DFTB_ERR_WORKSPACE, "batched_eigh: workspace");
    if (c->host.size() < hbytes) c->host.resize(hbytes);
    s = a.syev(c->h, c->p, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, CUDA_R_64F, A, n, CUDA_R_64F, W,
               CUDA_R_64F, work, dbytes, hbytes ? c->host.data() : nullptr, hbytes, info, batch);
    if (s != CUSOLVER_STATUS_SUCCESS) {
        snprintf(g_eig_err, sizeof(g_eig_err), "batched_eigh: cusolverDnXsyevBatched failed (status %d)", (int)s);
        return s == CUSOLVER_STATUS_INVALID_VALUE ? DFTB_ERR_UNSUPPORTED : DFTB_ERR_CUDA;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(g_eig_err, sizeof(g_eig_err), "batched_eigh: %s", cudaGetErrorString(e));
        return DFTB_ERR_CUDA;
    }
    return DFTB_OK;
}

}  // extern "C"
