// dftbaby_b200: the fused device solve behind an opaque handle.
//
// DFTBaby runs its Davidson solvers in Python over numpy (LR_TDDFTB._solve_lr_equations,
// DFTB/LR_TDDFTB.py:403-527, calling Solver.HermitianDavidson, DFTB/Solver.py:404-578).  A C caller of this
// library gets the same solve as one call: the expansion space, its products, the projected matrix and
// the previous solution (the warm start of the next call, Solver.py:461-478) live in a dftb_solver
// handle whose device memory the caller provides once, at creation.  Every step runs on the device;
// the host only reads the k residual norms per iteration to decide convergence and which correction
// vectors to add, exactly as DFTBaby does.
//
// Layout: the basis V and its products AV are column-major (nov x cap, one expansion vector per
// contiguous column), the projected matrix M is cap x cap column-major.  The product kernel
// (dftb_hermitian_rv) takes (nov, m) row-major blocks, so new columns are transposed into and out of it.
//
// The small dense eigenproblem uses cuSOLVER's dsyevd and the GEMMs cuBLAS, both resolved at run time
// from the copies the process already holds (dlopen with RTLD_NOLOAD first), like the rest of this
// library; without them dftb_solver_create returns DFTB_ERR_UNSUPPORTED.

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <dlfcn.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <numeric>
#include <vector>

#include "dftbaby_b200.h"

namespace {

thread_local char g_solver_err[256] = "";

int sfail(int code, const char *what) {
    snprintf(g_solver_err, sizeof(g_solver_err), "%s", what);
    return code;
}

int scuda(cudaError_t e, const char *where) {
    if (e == cudaSuccess) return DFTB_OK;
    snprintf(g_solver_err, sizeof(g_solver_err), "%s: %s", where, cudaGetErrorString(e));
    return DFTB_ERR_CUDA;
}

using blas_create_t = cublasStatus_t (*)(cublasHandle_t *);
using blas_destroy_t = cublasStatus_t (*)(cublasHandle_t);
using blas_stream_t = cublasStatus_t (*)(cublasHandle_t, cudaStream_t);
using blas_dgemm_t = cublasStatus_t (*)(cublasHandle_t, cublasOperation_t, cublasOperation_t, int, int, int,
                                        const double *, const double *, int, const double *, int, const double *,
                                        double *, int);
using sol_create_t = cusolverStatus_t (*)(cusolverDnHandle_t *);
using sol_destroy_t = cusolverStatus_t (*)(cusolverDnHandle_t);
using sol_stream_t = cusolverStatus_t (*)(cusolverDnHandle_t, cudaStream_t);
using syevd_buf_t = cusolverStatus_t (*)(cusolverDnHandle_t, cusolverEigMode_t, cublasFillMode_t, int,
                                         const double *, int, const double *, int *);
using syevd_t = cusolverStatus_t (*)(cusolverDnHandle_t, cusolverEigMode_t, cublasFillMode_t, int, double *, int,
                                     double *, double *, int, int *);

struct Libs {
    blas_create_t blas_create = nullptr;
    blas_destroy_t blas_destroy = nullptr;
    blas_stream_t blas_stream = nullptr;
    blas_dgemm_t dgemm = nullptr;
    sol_create_t sol_create = nullptr;
    sol_destroy_t sol_destroy = nullptr;
    sol_stream_t sol_stream = nullptr;
    syevd_buf_t syevd_buf = nullptr;
    syevd_t syevd = nullptr;
    bool ok = false;
};

void *open_lib(const char *soname, const char *fallback) {
    void *h = dlopen(soname, RTLD_NOW | RTLD_NOLOAD);
    if (!h) h = dlopen(soname, RTLD_NOW | RTLD_GLOBAL);
    if (!h) h = dlopen(fallback, RTLD_NOW | RTLD_GLOBAL);
    return h;
}

Libs &libs() {
    static Libs L;
    static std::once_flag once;
    std::call_once(once, [] {
        void *b = open_lib("libcublas.so.12", "libcublas.so");
        void *s = open_lib("libcusolver.so.11", "libcusolver.so");
        if (!b || !s) return;
        L.blas_create = reinterpret_cast<blas_create_t>(dlsym(b, "cublasCreate_v2"));
        L.blas_destroy = reinterpret_cast<blas_destroy_t>(dlsym(b, "cublasDestroy_v2"));
        L.blas_stream = reinterpret_cast<blas_stream_t>(dlsym(b, "cublasSetStream_v2"));
        L.dgemm = reinterpret_cast<blas_dgemm_t>(dlsym(b, "cublasDgemm_v2"));
        L.sol_create = reinterpret_cast<sol_create_t>(dlsym(s, "cusolverDnCreate"));
        L.sol_destroy = reinterpret_cast<sol_destroy_t>(dlsym(s, "cusolverDnDestroy"));
        L.sol_stream = reinterpret_cast<sol_stream_t>(dlsym(s, "cusolverDnSetStream"));
        L.syevd_buf = reinterpret_cast<syevd_buf_t>(dlsym(s, "cusolverDnDsyevd_bufferSize"));
        L.syevd = reinterpret_cast<syevd_t>(dlsym(s, "cusolverDnDsyevd"));
        L.ok = L.blas_create && L.blas_destroy && L.blas_stream && L.dgemm && L.sol_create && L.sol_destroy &&
               L.sol_stream && L.syevd_buf && L.syevd;
    });
    return L;
}

inline unsigned cdivu(long long a, long long b) { return (unsigned)((a + b - 1) / b); }
inline size_t a256(size_t b) { return (b + 255) / 256 * 256; }

// out = in as a row-major (rows x cols) array; in is column-major (rows x cols, leading dimension ld)
__global__ void transpose_kernel(int rows, int cols, const double *in, int ld, double *out) {
    __shared__ double tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (c < cols && r < rows) tile[k][threadIdx.x] = in[(size_t)c * ld + r];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (c < cols && r < rows) out[(size_t)r * cols + c] = tile[threadIdx.x][k];
    }
}

// M[l0:l1, 0:l0] = M[0:l0, l0:l1]^T (the projected matrix of a symmetric operator)
__global__ void mirror_kernel(int l0, int l1, double *M, int ld) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // row of the new block
    const int j = blockIdx.y;                             // old column
    if (l0 + i < l1 && j < l0) M[(size_t)j * ld + l0 + i] = M[(size_t)(l0 + i) * ld + j];
}

// W[:, j] = AT[:, j] - lam[j] X[:, j]; nrm2[j] = |W[:, j]|^2 (one block per column, column-major nov x k)
__global__ void residual_cols_kernel(int nov, const double *AT, const double *X, const double *lam, double *W,
                                     double *nrm2) {
    const int j = blockIdx.x;
    const size_t o = (size_t)j * nov;
    const double l = lam[j];
    double acc = 0.0;
    for (int i = threadIdx.x; i < nov; i += blockDim.x) {
        const double w = AT[o + i] - l * X[o + i];
        W[o + i] = w;
        acc += w * w;
    }
    __shared__ double red[32];
    for (int s = 16; s > 0; s >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int s = 16; s > 0; s >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, s);
        if (threadIdx.x == 0) nrm2[j] = acc;
    }
}

// q = W[:, src] / (w[state] - omega), with DFTBaby's guard against a vanishing denominator
// (Solver.py:530-537): |w - omega| < 1e-6 -> 1e-6 omega
__global__ void precond_col_kernel(int nov, const double *Wcol, double w, const double *omega, double *q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nov) return;
    double d = w - omega[i];
    if (fabs(d) < 1.0e-6) d = 1.0e-6 * omega[i];
    q[i] = Wcol[i] / d;
}

// |q|^2 into out[0] (one block)
__global__ void norm2_kernel(int n, const double *q, double *out) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += q[i] * q[i];
    __shared__ double red[32];
    for (int s = 16; s > 0; s >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int s = 16; s > 0; s >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, s);
        if (threadIdx.x == 0) out[0] = acc;
    }
}

__global__ void scale_kernel(int n, double a, double *q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) q[i] *= a;
}

// unit vector on index idx
__global__ void unit_kernel(int n, int idx, double *q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) q[i] = i == idx ? 1.0 : 0.0;
}

// guess column from the previous XpY (row-major k x nov): q = XpY[s, :] / sqrt(omega)
__global__ void guess_kernel(int nov, const double *XpY, int s, const double *omega, double *q) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nov) q[i] = XpY[(size_t)s * nov + i] / sqrt(omega[i]);
}

// outputs, row-major (k, nov): C = X^T, XpY = sqrt(omega)/sqrt(Omega) C, XmY = sqrt(Omega)/sqrt(omega) C
__global__ void output_kernel(int nov, int k, const double *X, const double *w2, const double *omega, double *Om,
                              double *C, double *XmY, double *XpY, double *keep) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nov * k) return;
    const int j = (int)(idx / nov), i = (int)(idx % nov);
    const double Omega = sqrt(w2[j]), so = sqrt(omega[i]);
    const double x = X[(size_t)j * nov + i];
    const double xp = so / sqrt(Omega) * x;
    if (C) C[idx] = x;
    if (XpY) XpY[idx] = xp;
    if (XmY) XmY[idx] = sqrt(Omega) / so * x;
    keep[idx] = xp;
    if (i == 0 && Om) Om[j] = Omega;
}

}  // namespace

struct dftb_solver {
    int nat, nocc, nvirt, nov, k, cap;
    double *V, *AV, *M, *Wm, *evals, *T, *X, *AT, *R, *nrm2, *h, *blk, *blkU, *keep, *syevd_work;
    int *info;
    int syevd_lwork;
    void *rv_work;
    size_t rv_bytes;
    bool have_guess;
    cublasHandle_t blas;
    cusolverDnHandle_t sol;
};

namespace {

// device memory carved from the caller's workspace, in this order
struct Carve {
    size_t off = 0;
    char *base = nullptr;
    template <class T>
    T *take(size_t count) {
        T *p = base ? reinterpret_cast<T *>(base + off) : nullptr;
        off += a256(sizeof(T) * count);
        return p;
    }
};

size_t layout(dftb_solver *s, char *base, int syevd_lwork) {
    Carve c;
    c.base = base;
    const size_t nov = s->nov, cap = s->cap, k = s->k;
    s->V = c.take<double>(nov * cap);
    s->AV = c.take<double>(nov * cap);
    s->M = c.take<double>(cap * cap);
    s->Wm = c.take<double>(cap * cap);
    s->evals = c.take<double>(cap);
    s->T = c.take<double>(cap * k);
    s->X = c.take<double>(nov * k);
    s->AT = c.take<double>(nov * k);
    s->R = c.take<double>(nov * k);
    s->nrm2 = c.take<double>(k + 1);
    s->h = c.take<double>(cap);
    s->blk = c.take<double>(nov * k);
    s->blkU = c.take<double>(nov * k);
    s->keep = c.take<double>(nov * k);
    s->syevd_work = c.take<double>((size_t)std::max(syevd_lwork, 1));
    s->info = c.take<int>(1);
    s->rv_bytes = dftb_hermitian_rv_workspace_size(s->nat, s->k);
    s->rv_work = c.take<char>(s->rv_bytes);
    return c.off;
}

int query_syevd(int cap, int *lwork) {
    Libs &L = libs();
    cusolverDnHandle_t h = nullptr;
    if (L.sol_create(&h) != CUSOLVER_STATUS_SUCCESS) return sfail(DFTB_ERR_CUDA, "solver: cusolverDnCreate");
    int lw = 0;
    cusolverStatus_t st = L.syevd_buf(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, cap, nullptr, cap, nullptr,
                                      &lw);
    L.sol_destroy(h);
    if (st != CUSOLVER_STATUS_SUCCESS) return sfail(DFTB_ERR_UNSUPPORTED, "solver: dsyevd buffer query");
    *lwork = lw;
    return DFTB_OK;
}

int check_dims(int nat, int nocc, int nvirt, int nstates, int max_iter, int *cap) {
    if (nat <= 0 || nocc <= 0 || nvirt <= 0 || nstates <= 0 || max_iter <= 0) return DFTB_ERR_BAD_SIZE;
    const long long nov = (long long)nocc * nvirt;
    if (nov > 0x7fffffffLL || nstates > nov) return DFTB_ERR_BAD_SIZE;
    const long long c = std::min<long long>(nov, (long long)nstates * (max_iter + 1));
    if (c > 46340) return DFTB_ERR_BAD_SIZE;  // cap^2 must fit an int leading-dimension product
    *cap = (int)c;
    return DFTB_OK;
}

// C = op(A) op(B), column-major
int gemm(dftb_solver *s, bool ta, bool tb, int m, int n, int kk, const double *A, int lda, const double *B, int ldb,
         double *C, int ldc, double alpha = 1.0, double beta = 0.0) {
    if (m == 0 || n == 0) return DFTB_OK;
    cublasStatus_t st = libs().dgemm(s->blas, ta ? CUBLAS_OP_T : CUBLAS_OP_N, tb ? CUBLAS_OP_T : CUBLAS_OP_N, m, n, kk,
                                     &alpha, A, lda, B, ldb, &beta, C, ldc);
    return st == CUBLAS_STATUS_SUCCESS ? DFTB_OK : sfail(DFTB_ERR_CUDA, "solver: cublasDgemm");
}

// Orthogonalise column q (nov) against V[:, 0:l] twice (classical Gram-Schmidt with re-orthogonalisation)
// and normalise it; returns its norm after projection relative to before (host), through *rel.
int orthonormalize_col(dftb_solver *s, int l, double *q, double *rel, cudaStream_t st) {
    const int nov = s->nov;
    double n0 = 0.0, n1 = 0.0;
    norm2_kernel<<<1, 512, 0, st>>>(nov, q, s->nrm2 + s->k);
    int rc = scuda(cudaMemcpyAsync(&n0, s->nrm2 + s->k, sizeof(double), cudaMemcpyDeviceToHost, st), "solver: copy");
    if (rc) return rc;
    for (int pass = 0; pass < 2 && l > 0; ++pass) {
        if ((rc = gemm(s, true, false, l, 1, nov, s->V, nov, q, nov, s->h, l))) return rc;            // h = V^T q
        if ((rc = gemm(s, false, false, nov, 1, l, s->V, nov, s->h, l, q, nov, -1.0, 1.0))) return rc;  // q -= V h
    }
    norm2_kernel<<<1, 512, 0, st>>>(nov, q, s->nrm2 + s->k);
    if ((rc = scuda(cudaMemcpyAsync(&n1, s->nrm2 + s->k, sizeof(double), cudaMemcpyDeviceToHost, st), "solver: copy")))
        return rc;
    if ((rc = scuda(cudaStreamSynchronize(st), "solver: sync"))) return rc;
    *rel = n0 > 0.0 ? sqrt(n1 / n0) : 0.0;
    if (n1 > 0.0) scale_kernel<<<cdivu(nov, 256), 256, 0, st>>>(nov, 1.0 / sqrt(n1), q);
    return scuda(cudaGetLastError(), "solver: orthonormalize");
}

// products of the columns V[:, l0:l1] into AV[:, l0:l1]
int apply(dftb_solver *s, int l0, int l1, const double *gamma, const double *q_ov, const double *omega,
          cudaStream_t st) {
    const int nov = s->nov;
    for (int c0 = l0; c0 < l1; c0 += s->k) {
        const int m = std::min(s->k, l1 - c0);
        dim3 g1(cdivu(m, 32), cdivu(nov, 32));
        transpose_kernel<<<g1, dim3(32, 8), 0, st>>>(nov, m, s->V + (size_t)c0 * nov, nov, s->blk);  // (nov, m)
        int rc = dftb_hermitian_rv(s->nat, s->nocc, s->nvirt, m, gamma, q_ov, omega, s->blk, s->blkU, s->rv_work,
                                   s->rv_bytes, st);
        if (rc) return rc;
        dim3 g2(cdivu(nov, 32), cdivu(m, 32));
        transpose_kernel<<<g2, dim3(32, 8), 0, st>>>(m, nov, s->blkU, m, s->AV + (size_t)c0 * nov);  // (nov, m) cm
    }
    return scuda(cudaGetLastError(), "solver: products");
}

// extend M by the columns l0:l1 (and their mirrored rows)
int extend_projection(dftb_solver *s, int l0, int l1, cudaStream_t st) {
    const int nov = s->nov, cap = s->cap;
    int rc = gemm(s, true, false, l1, l1 - l0, nov, s->V, nov, s->AV + (size_t)l0 * nov, nov, s->M + (size_t)l0 * cap,
                  cap);
    if (rc) return rc;
    if (l0 > 0) mirror_kernel<<<dim3(cdivu(l1 - l0, 128), l0), 128, 0, st>>>(l0, l1, s->M, cap);
    return scuda(cudaGetLastError(), "solver: projection");
}

}  // namespace

extern "C" {

const char *dftb_solver_last_error(void) { return g_solver_err; }

size_t dftb_solver_workspace_size(int nat, int nocc, int nvirt, int nstates, int max_iter) {
    int cap = 0;
    if (check_dims(nat, nocc, nvirt, nstates, max_iter, &cap)) return 0;
    if (!libs().ok) return 0;
    int lw = 0;
    if (query_syevd(cap, &lw)) return 0;
    dftb_solver s{};
    s.nat = nat;
    s.nocc = nocc;
    s.nvirt = nvirt;
    s.nov = nocc * nvirt;
    s.k = nstates;
    s.cap = cap;
    return layout(&s, nullptr, lw);
}

int dftb_solver_create(int nat, int nocc, int nvirt, int nstates, int max_iter, void *work, size_t work_bytes,
                       dftb_solver **out) {
    if (!out) return sfail(DFTB_ERR_NULL, "solver_create: out");
    *out = nullptr;
    int cap = 0;
    if (check_dims(nat, nocc, nvirt, nstates, max_iter, &cap)) return sfail(DFTB_ERR_BAD_SIZE, "solver_create: sizes");
    if (!libs().ok) return sfail(DFTB_ERR_UNSUPPORTED, "solver_create: cuBLAS / cuSOLVER not found");
    int lw = 0;
    int rc = query_syevd(cap, &lw);
    if (rc) return rc;
    dftb_solver *s = (dftb_solver *)calloc(1, sizeof(dftb_solver));
    if (!s) return sfail(DFTB_ERR_WORKSPACE, "solver_create: host allocation");
    s->nat = nat;
    s->nocc = nocc;
    s->nvirt = nvirt;
    s->nov = nocc * nvirt;
    s->k = nstates;
    s->cap = cap;
    s->syevd_lwork = lw;
    if (!work || work_bytes < layout(s, nullptr, lw)) {
        free(s);
        return sfail(DFTB_ERR_WORKSPACE, "solver_create: workspace too small");
    }
    layout(s, (char *)work, lw);
    Libs &L = libs();
    if (L.blas_create(&s->blas) != CUBLAS_STATUS_SUCCESS) {
        free(s);
        return sfail(DFTB_ERR_CUDA, "solver_create: cublasCreate");
    }
    if (L.sol_create(&s->sol) != CUSOLVER_STATUS_SUCCESS) {
        L.blas_destroy(s->blas);
        free(s);
        return sfail(DFTB_ERR_CUDA, "solver_create: cusolverDnCreate");
    }
    *out = s;
    return DFTB_OK;
}

int dftb_solver_destroy(dftb_solver *s) {
    if (!s) return DFTB_OK;
    Libs &L = libs();
    if (s->blas) L.blas_destroy(s->blas);
    if (s->sol) L.sol_destroy(s->sol);
    free(s);
    return DFTB_OK;
}

int dftb_solver_reset(dftb_solver *s) {
    if (!s) return sfail(DFTB_ERR_NULL, "solver_reset: handle");
    s->have_guess = false;
    return DFTB_OK;
}

int dftb_solver_solve_hermitian(dftb_solver *s, const double *gamma, const double *q_ov, const double *omega,
                                double conv, int maxiter, int warm_start, double *Omega, double *C, double *XmY,
                                double *XpY, int *iterations, void *stream) {
    if (!s) return sfail(DFTB_ERR_NULL, "solve_hermitian: handle");
    if (!gamma || !q_ov || !omega || !Omega) return sfail(DFTB_ERR_NULL, "solve_hermitian: null");
    if (maxiter <= 0 || !(conv > 0.0)) return sfail(DFTB_ERR_BAD_SIZE, "solve_hermitian: maxiter / conv");
    cudaStream_t st = (cudaStream_t)stream;
    Libs &L = libs();
    L.blas_stream(s->blas, st);
    L.sol_stream(s->sol, st);
    const int nov = s->nov, k = s->k, cap = s->cap;
    int rc;
    // ---- initial expansion vectors (Solver.py:232-251, 461-478)
    int l = 0;
    if (warm_start && s->have_guess) {
        for (int j = 0; j < k; ++j) {
            double *q = s->V + (size_t)l * nov;
            guess_kernel<<<cdivu(nov, 256), 256, 0, st>>>(nov, s->keep, j, omega, q);
            double rel = 0.0;
            if ((rc = orthonormalize_col(s, l, q, &rel, st))) return rc;
            if (rel > 1.0e-10) ++l;
        }
    } else {
        std::vector<double> om(nov);
        if ((rc = scuda(cudaMemcpyAsync(om.data(), omega, sizeof(double) * nov, cudaMemcpyDeviceToHost, st),
                        "solve_hermitian: omega")))
            return rc;
        if ((rc = scuda(cudaStreamSynchronize(st), "solve_hermitian: sync"))) return rc;
        std::vector<int> order(nov);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return om[a] < om[b]; });
        const int lmax = std::min(k, nov);
        for (int j = 0; j < lmax; ++j)
            unit_kernel<<<cdivu(nov, 256), 256, 0, st>>>(nov, order[j], s->V + (size_t)j * nov);
        l = lmax;
    }
    if (l < k) return sfail(DFTB_ERR_BAD_SIZE, "solve_hermitian: the guess spans fewer than nstates directions");
    if ((rc = apply(s, 0, l, gamma, q_ov, omega, st))) return rc;
    if ((rc = extend_projection(s, 0, l, st))) return rc;
    std::vector<double> nrm(k), w2(k);
    int it = 0;
    bool done = false;
    for (it = 0; it < maxiter; ++it) {
        // ---- Ritz pairs of the projected matrix (Solver.py:486)
        for (int c = 0; c < l; ++c)
            if ((rc = scuda(cudaMemcpyAsync(s->Wm + (size_t)c * l, s->M + (size_t)c * cap, sizeof(double) * l,
                                            cudaMemcpyDeviceToDevice, st),
                            "solve_hermitian: copy M")))
                return rc;
        if (L.syevd(s->sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, l, s->Wm, l, s->evals, s->syevd_work,
                    s->syevd_lwork, s->info) != CUSOLVER_STATUS_SUCCESS)
            return sfail(DFTB_ERR_CUDA, "solve_hermitian: dsyevd");
        // X = V T_k, AT = AV T_k, residuals (Solver.py:495-512)
        if ((rc = gemm(s, false, false, nov, k, l, s->V, nov, s->Wm, l, s->X, nov))) return rc;
        if ((rc = gemm(s, false, false, nov, k, l, s->AV, nov, s->Wm, l, s->AT, nov))) return rc;
        residual_cols_kernel<<<k, 256, 0, st>>>(nov, s->AT, s->X, s->evals, s->R, s->nrm2);
        int info = 0;
        if ((rc = scuda(cudaMemcpyAsync(nrm.data(), s->nrm2, sizeof(double) * k, cudaMemcpyDeviceToHost, st),
                        "solve_hermitian: norms")) ||
            (rc = scuda(cudaMemcpyAsync(w2.data(), s->evals, sizeof(double) * k, cudaMemcpyDeviceToHost, st),
                        "solve_hermitian: evals")) ||
            (rc = scuda(cudaMemcpyAsync(&info, s->info, sizeof(int), cudaMemcpyDeviceToHost, st),
                        "solve_hermitian: info")) ||
            (rc = scuda(cudaStreamSynchronize(st), "solve_hermitian: sync")))
            return rc;
        if (info != 0) return sfail(DFTB_ERR_CUDA, "solve_hermitian: dsyevd did not converge");
        bool all = true;
        for (int j = 0; j < k; ++j) {
            nrm[j] = sqrt(nrm[j]);
            if (!(nrm[j] < conv)) all = false;
        }
        if (all) {
            done = true;
            break;
        }
        // ---- correction vectors for the states whose residual exceeds 0.01 conv (Solver.py:515-551)
        const int dkmax = std::min(nov - l, k);
        const double eps = 0.01 * conv;
        int added = 0;
        for (int n = 0; n < dkmax; ++n) {
            if (!(nrm[n] > eps)) continue;
            if (l + added >= cap) break;
            double *q = s->V + (size_t)(l + added) * nov;
            precond_col_kernel<<<cdivu(nov, 256), 256, 0, st>>>(nov, s->R + (size_t)n * nov, sqrt(w2[n]), omega, q);
            double rel = 0.0;
            if ((rc = orthonormalize_col(s, l + added, q, &rel, st))) return rc;
            if (rel > 1.0e-10) ++added;
        }
        if (added == 0) break;  // no new direction: the space cannot grow
        if ((rc = apply(s, l, l + added, gamma, q_ov, omega, st))) return rc;
        if ((rc = extend_projection(s, l, l + added, st))) return rc;
        l += added;
    }
    if (iterations) *iterations = it + (done ? 1 : 0);
    if (!done) {
        snprintf(g_solver_err, sizeof(g_solver_err),
                 "Davidson (Hermitian) did not converge after %d iterations (threshold %e)", it, conv);
        return DFTB_ERR_NOT_CONVERGED;
    }
    output_kernel<<<cdivu((long long)nov * k, 256), 256, 0, st>>>(nov, k, s->X, s->evals, omega, Omega, C, XmY, XpY,
                                                                   s->keep);
    s->have_guess = true;
    return scuda(cudaGetLastError(), "solve_hermitian: outputs");
}

}  // extern "C"
