// dftbaby_b200: element-wise kernels of the small MLP behind the learned
// Davidson guess and preconditioner correction (no counterpart in DFTBaby).
//
// The network is x(64, zero-padded features) -> 256 -> 256 -> 2 with ReLU.
// Its matrix products run on the tcgen05 tensor cores (dftb_bf16x3_gemm_ex with
// one BF16 segment, FP32 accumulation); the kernels here do everything in
// between: bias + ReLU with BF16 row-major and transposed copies of the
// activations (the transposed copies are the K-major operands of the
// weight-gradient products), the weighted squared-error loss and its gradient,
// the ReLU backward pass with bias-gradient column sums, and Adam on FP32
// master weights with refreshed BF16 copies.  All matrices are row-major.

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdio.h>

#include "dftbaby_b200.h"

namespace {

thread_local char g_mlp_err[256] = "";

int mlp_fail(int code, const char *what) {
    snprintf(g_mlp_err, sizeof(g_mlp_err), "%s", what);
    return code;
}

int mlp_check(const char *where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(g_mlp_err, sizeof(g_mlp_err), "%s: %s", where, cudaGetErrorString(e));
        return DFTB_ERR_CUDA;
    }
    return DFTB_OK;
}

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr int TILE = 32;

// H = relu(Z + b) on a 32 x 32 tile (samples x units); H row-major and, when
// HT is given, H^T through a shared-memory transpose so both writes coalesce.
__global__ void bias_relu_kernel(int ns, int nh, const float *__restrict__ Z, int ldz, const float *__restrict__ b,
                                 __nv_bfloat16 *__restrict__ H, int ldh, __nv_bfloat16 *__restrict__ HT, int ldht) {
    __shared__ float tile[TILE][TILE + 1];
    const int s0 = blockIdx.x * TILE, h0 = blockIdx.y * TILE;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < TILE; r += blockDim.y) {
        const int s = s0 + r, h = h0 + tx;
        float v = 0.0f;
        if (s < ns && h < nh) {
            v = fmaxf(Z[(size_t)s * ldz + h] + b[h], 0.0f);
            H[(size_t)s * ldh + h] = __float2bfloat16(v);
        }
        tile[r][tx] = v;
    }
    if (!HT) return;
    __syncthreads();
    for (int r = ty; r < TILE; r += blockDim.y) {
        const int h = h0 + r, s = s0 + tx;
        if (h < nh && s < ns) HT[(size_t)h * ldht + s] = __float2bfloat16(tile[tx][r]);
    }
}

// dZ = G o (H > 0) with the same tiling; db[h] += sum over the tile's samples.
__global__ void relu_backward_kernel(int ns, int nh, const float *__restrict__ G, int ldg,
                                     const __nv_bfloat16 *__restrict__ H, int ldh, __nv_bfloat16 *__restrict__ dZ,
                                     int lddz, __nv_bfloat16 *__restrict__ dZT, int lddzt, float *__restrict__ db) {
    __shared__ float tile[TILE][TILE + 1];
    const int s0 = blockIdx.x * TILE, h0 = blockIdx.y * TILE;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < TILE; r += blockDim.y) {
        const int s = s0 + r, h = h0 + tx;
        float v = 0.0f;
        if (s < ns && h < nh) {
            v = __bfloat162float(H[(size_t)s * ldh + h]) > 0.0f ? G[(size_t)s * ldg + h] : 0.0f;
            if (dZ) dZ[(size_t)s * lddz + h] = __float2bfloat16(v);
        }
        tile[r][tx] = v;
    }
    __syncthreads();
    if (ty == 0 && h0 + tx < nh) {
        float acc = 0.0f;
        for (int r = 0; r < TILE; ++r) acc += tile[r][tx];
        atomicAdd(&db[h0 + tx], acc);
    }
    for (int r = ty; r < TILE; r += blockDim.y) {
        const int h = h0 + r, s = s0 + tx;
        if (h < nh && s < ns) dZT[(size_t)h * lddzt + s] = __float2bfloat16(tile[tx][r]);
    }
}

// Output layer, one thread per sample:
//   y[s][o] = Z[s][o] + b[o];
//   with targets: loss += sum_o wout[o] m[s] (y - t)^2 * inv_norm and
//   dY[s][o] = 2 wout[o] m[s] (y - t) inv_norm (BF16, row-major dYp and rows o of dYT),
//   db[o] += dY[s][o].
__global__ void output_kernel(int ns, int no, const float *__restrict__ Z, int ldz, const float *__restrict__ b,
                              const float *__restrict__ T, const float *__restrict__ m,
                              const float *__restrict__ wout, float inv_norm, float *__restrict__ Y,
                              __nv_bfloat16 *__restrict__ dYp, int lddy, __nv_bfloat16 *__restrict__ dYT, int lddyt,
                              float *__restrict__ db, double *__restrict__ loss) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (s < ns) {
        for (int o = 0; o < no; ++o) {
            const float y = Z[(size_t)s * ldz + o] + b[o];
            Y[(size_t)s * no + o] = y;
            if (T) {
                const float d = y - T[(size_t)s * no + o];
                const float w = wout[o] * m[s];
                l += (double)w * d * d * inv_norm;
                const float g = 2.0f * w * d * inv_norm;
                dYp[(size_t)s * lddy + o] = __float2bfloat16(g);
                dYT[(size_t)o * lddyt + s] = __float2bfloat16(g);
                atomicAdd(&db[o], g);
            }
        }
    }
    if (!T) return;
    for (int off = 16; off > 0; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// Adam (with decoupled weight decay) on FP32 master weights W (rows x cols),
// followed by the BF16 copies Wb (row-major, ldwb) and optionally WbT (transposed, ldwbt).
__global__ void adam_kernel(int rows, int cols, float *__restrict__ W, const float *__restrict__ G,
                            float *__restrict__ mom1, float *__restrict__ mom2, float lr, float beta1, float beta2,
                            float eps, float bc1, float bc2, float wd, __nv_bfloat16 *__restrict__ Wb, int ldwb,
                            __nv_bfloat16 *__restrict__ WbT, int ldwbt) {
    const long long n = (long long)rows * cols;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float g = G[i];
        const float m1 = beta1 * mom1[i] + (1.0f - beta1) * g;
        const float m2 = beta2 * mom2[i] + (1.0f - beta2) * g * g;
        mom1[i] = m1;
        mom2[i] = m2;
        float w = W[i];
        w -= lr * ((m1 / bc1) / (sqrtf(m2 / bc2) + eps) + wd * w);
        W[i] = w;
        const int r = (int)(i / cols), c = (int)(i % cols);
        if (Wb) Wb[(size_t)r * ldwb + c] = __float2bfloat16(w);
        if (WbT) WbT[(size_t)c * ldwbt + r] = __float2bfloat16(w);
    }
}

}  // namespace

extern "C" {

const char *dftb_mlp_last_error(void) { return g_mlp_err; }

int dftb_mlp_bias_relu(int ns, int nh, const float *Z, int ldz, const float *b, void *H, int ldh, void *HT, int ldht,
                       void *stream) {
    if (ns <= 0 || nh <= 0 || ldz < nh || ldh < nh || (HT && ldht < ns)) return mlp_fail(DFTB_ERR_BAD_SIZE, "mlp_bias_relu: sizes");
    if (!Z || !b || !H) return mlp_fail(DFTB_ERR_NULL, "mlp_bias_relu: null");
    dim3 grid((ns + TILE - 1) / TILE, (nh + TILE - 1) / TILE);
    bias_relu_kernel<<<grid, dim3(TILE, 8), 0, S(stream)>>>(ns, nh, Z, ldz, b, reinterpret_cast<__nv_bfloat16 *>(H),
                                                           ldh, reinterpret_cast<__nv_bfloat16 *>(HT), ldht);
    return mlp_check("bias_relu_kernel");
}

int dftb_mlp_relu_backward(int ns, int nh, const float *G, int ldg, const void *H, int ldh, void *dZ, int lddz,
                           void *dZT, int lddzt, float *db, void *stream) {
    if (ns <= 0 || nh <= 0 || ldg < nh || ldh < nh || (dZ && lddz < nh) || lddzt < ns)
        return mlp_fail(DFTB_ERR_BAD_SIZE, "mlp_relu_backward: sizes");
    if (!G || !H || !dZT || !db) return mlp_fail(DFTB_ERR_NULL, "mlp_relu_backward: null");
    dim3 grid((ns + TILE - 1) / TILE, (nh + TILE - 1) / TILE);
    relu_backward_kernel<<<grid, dim3(TILE, 8), 0, S(stream)>>>(
        ns, nh, G, ldg, reinterpret_cast<const __nv_bfloat16 *>(H), ldh, reinterpret_cast<__nv_bfloat16 *>(dZ), lddz,
        reinterpret_cast<__nv_bfloat16 *>(dZT), lddzt, db);
    return mlp_check("relu_backward_kernel");
}

int dftb_mlp_output(int ns, int no, const float *Z, int ldz, const float *b, const float *T, const float *m,
                    const float *wout, float inv_norm, float *Y, void *dYp, int lddy, void *dYT, int lddyt, float *db,
                    double *loss, void *stream) {
    if (ns <= 0 || no <= 0 || no > 8 || ldz < no) return mlp_fail(DFTB_ERR_BAD_SIZE, "mlp_output: sizes");
    if (!Z || !b || !Y) return mlp_fail(DFTB_ERR_NULL, "mlp_output: null");
    if (T && (!m || !wout || !dYp || !dYT || !db || !loss || lddy < no || lddyt < ns))
        return mlp_fail(DFTB_ERR_NULL, "mlp_output: training outputs");
    output_kernel<<<(ns + 255) / 256, 256, 0, S(stream)>>>(ns, no, Z, ldz, b, T, m, wout, inv_norm, Y,
                                                           reinterpret_cast<__nv_bfloat16 *>(dYp), lddy,
                                                           reinterpret_cast<__nv_bfloat16 *>(dYT), lddyt, db, loss);
    return mlp_check("output_kernel");
}

int dftb_mlp_adam(int rows, int cols, float *W, const float *G, float *m1, float *m2, float lr, float beta1,
                  float beta2, float eps, int step, float weight_decay, void *Wb, int ldwb, void *WbT, int ldwbt,
                  void *stream) {
    if (rows <= 0 || cols <= 0 || step < 1 || (Wb && ldwb < cols) || (WbT && ldwbt < rows))
        return mlp_fail(DFTB_ERR_BAD_SIZE, "mlp_adam: sizes");
    if (!W || !G || !m1 || !m2) return mlp_fail(DFTB_ERR_NULL, "mlp_adam: null");
    const float bc1 = 1.0f - powf(beta1, (float)step), bc2 = 1.0f - powf(beta2, (float)step);
    const long long n = (long long)rows * cols;
    const int blocks = (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096);
    adam_kernel<<<blocks, 256, 0, S(stream)>>>(rows, cols, W, G, m1, m2, lr, beta1, beta2, eps, bc1, bc2, weight_decay,
                                               reinterpret_cast<__nv_bfloat16 *>(Wb), ldwb,
                                               reinterpret_cast<__nv_bfloat16 *>(WbT), ldwbt);
    return mlp_check("adam_kernel");
}

}  // extern "C"
