// dftbaby_b200: FP64 CUDA kernels for the LR-TD-DFTB path on B200 (sm_100a).
//
// Every extern "C" entry point is declared in include/dftbaby_b200.h, which
// also documents argument shapes and the DFTBaby interface each one replaces.
// All matrices are row-major FP64 in device memory.  Nothing here allocates:
// scratch space comes from caller-provided workspaces.

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "dftbaby_b200.h"

namespace {

thread_local char g_last_error[256] = "";

int fail(int code, const char *what) {
    snprintf(g_last_error, sizeof(g_last_error), "%s", what);
    return code;
}

int check_launch(const char *where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(g_last_error, sizeof(g_last_error), "%s: %s", where, cudaGetErrorString(e));
        return DFTB_ERR_CUDA;
    }
    return DFTB_OK;
}

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }
inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

#include "sk_device.cuh"

// One thread per matrix element (mu, nu); the value is the reference's
// lower-triangle element for (max, min), so both triangles are written
// directly and coalesced.  slako.f90:77-231.
__global__ void h0_and_s_kernel(int norb, int nat, OrbTables O, const double *r, const double *x, const double *y,
                                const double *z, const int *mprox, const double *orben, SkTables TS, SkTables TH,
                                double *S, double *H0) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y;
    if (col >= norb || row >= norb) return;
    const int mu = row > col ? row : col, nu = row > col ? col : row;
    const size_t o = (size_t)row * norb + col;
    const int i = O.ind[mu], j = O.ind[nu];
    double s = 0.0, h = 0.0;
    if (mprox[(size_t)i * nat + j] != 0) {
        if (mu == nu) {
            s = 1.0;
            h = orben[mu];
        } else if (i != j) {
            const int l1 = O.ls[mu], m1 = O.ms[mu], l2 = O.ls[nu], m2 = O.ms[nu];
            if (l1 > 1 || l2 > 1) {
                s = h = __longlong_as_double(0x7ff8000000000000ULL);
            } else {
                const int typi = O.typ[mu], typj = O.typ[nu];
                const int tmin = min(typi, typj), tmax = max(typi, typj);
                const int ipair = tmax * (tmax + 1) / 2 + tmin;
                double rij, e[3];
                pair_dir(nat, r, x, y, z, i, j, rij, e);
                if (typi <= typj) {
                    s = sk_rule(TS, ipair, rij, e, l1, m1, l2, m2);
                    h = sk_rule(TH, ipair, rij, e, l1, m1, l2, m2);
                } else {
                    const double me[3] = {-e[0], -e[1], -e[2]};
                    s = sk_rule(TS, ipair, rij, me, l2, m2, l1, m1);
                    h = sk_rule(TH, ipair, rij, me, l2, m2, l1, m1);
                }
            }
        }
    }
    S[o] = s;
    H0[o] = h;
}

// slako.f90:238-394; D planes (3, norb, norb).
__global__ void dipole_kernel(int norb, int nat, OrbTables O, const double *r, const double *x, const double *y,
                              const double *z, const double *pos, const int *mprox, const double *Smat,
                              SkTables TD, double *D) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = blockIdx.y;
    if (col >= norb || row >= norb) return;
    const int mu = row > col ? row : col, nu = row > col ? col : row;
    const size_t o = (size_t)row * norb + col, plane = (size_t)norb * norb;
    const int i = O.ind[mu], j = O.ind[nu];
    double d[3] = {0.0, 0.0, 0.0};
    if (mprox[(size_t)i * nat + j] != 0) {
        const int l1 = O.ls[mu], m1 = O.ms[mu], l2 = O.ls[nu], m2 = O.ms[nu];
        if (l1 > 1 || l2 > 1) {
            d[0] = d[1] = d[2] = __longlong_as_double(0x7ff8000000000000ULL);
        } else {
            const int typi = O.typ[mu], typj = O.typ[nu];
            const int tmin = min(typi, typj), tmax = max(typi, typj);
            const int ipair = tmax * (tmax + 1) / 2 + tmin;
            double rij, e[3];
            pair_dir(nat, r, x, y, z, i, j, rij, e);
            const double s = Smat[(size_t)mu * norb + nu];
            if (typi <= typj) {
                sk_dipole_rule(TD, ipair, rij, e, l1, m1, l2, m2, d);
#pragma unroll
                for (int c = 0; c < 3; ++c) d[c] += pos[3 * j + c] * s;
            } else {
                const double me[3] = {-e[0], -e[1], -e[2]};
                sk_dipole_rule(TD, ipair, rij, me, l2, m2, l1, m1, d);
#pragma unroll
                for (int c = 0; c < 3; ++c) d[c] += pos[3 * i + c] * s;
            }
        }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) D[c * plane + o] = d[c];
}

__global__ void dircos_kernel(int nat, const double *pos, double *r, double *x, double *y, double *z) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j >= nat || i >= nat) return;
    const double xc = pos[3 * i] - pos[3 * j], yc = pos[3 * i + 1] - pos[3 * j + 1],
                 zc = pos[3 * i + 2] - pos[3 * j + 2];
    const double rr = sqrt(xc * xc + yc * yc + zc * zc);
    const size_t o = (size_t)i * nat + j;
    r[o] = rr;
    if (rr > 0.0) {
        x[o] = xc / rr;
        y[o] = yc / rr;
        z[o] = zc / rr;
    } else {
        x[o] = 0.0;
        y[o] = 0.0;
        z[o] = 1.0;
    }
}

__global__ void gamma_kernel(int nat, const double *r, const double *sigma, double r_lr, double *g, double *glr) {
    const int B = blockIdx.x * blockDim.x + threadIdx.x;
    const int A = blockIdx.y;
    if (A >= nat || B >= nat) return;
    const size_t o = (size_t)A * nat + B;
    const double sa = sigma[A], sb = sigma[B];
    const double s2 = sa * sa + sb * sb;
    if (A == B) {
        g[o] = 1.0 / (sqrt(M_PI) * sa);
        if (glr) glr[o] = 1.0 / sqrt(M_PI * (sa * sa + 0.25 * r_lr * r_lr));
    } else {
        const double R = r[o];
        const double C = 1.0 / sqrt(2.0 * s2);
        g[o] = erf(C * R) / R;
        if (glr) {
            const double Clr = 1.0 / sqrt(2.0 * (s2 + 0.5 * r_lr * r_lr));
            glr[o] = erf(Clr * R) / R;
        }
    }
}

__global__ void ao_expand_kernel(int norb, int nat, const int *ind, const double *g, double *G) {
    const int nu = blockIdx.x * blockDim.x + threadIdx.x;
    const int mu = blockIdx.y;
    if (nu >= norb || mu >= norb) return;
    G[(size_t)mu * norb + nu] = g[(size_t)ind[mu] * nat + ind[nu]];
}

// estat[A] = sum_B gamma[A][B] dq[B]; one warp per atom
__global__ void estat_kernel(int nat, const double *gamma, const double *dq, double *estat) {
    const int A = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    if (A >= nat) return;
    double acc = 0.0;
    for (int B = lane; B < nat; B += 32) acc += gamma[(size_t)A * nat + B] * dq[B];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) estat[A] = acc;
}

__global__ void scc_h_kernel(int norb, const int *ind, const double *H0, const double *Smat, const double *estat,
                             double *H) {
    const int nu = blockIdx.x * blockDim.x + threadIdx.x;
    const int mu = blockIdx.y;
    if (nu >= norb || mu >= norb) return;
    const size_t o = (size_t)mu * norb + nu;
    const double h1 = 0.5 * (estat[ind[mu]] + estat[ind[nu]]);
    H[o] = H0[o] + h1 * Smat[o];
}

// Mulliken monopoles: one block per atom, reduction over its rows.
__global__ void monopoles_kernel(int norb, int nat, const double *P, const double *P0, const double *Smat,
                                 const int *opa, double *q, double *dq) {
    const int A = blockIdx.x;
    __shared__ int first_s;
    __shared__ double red_q[32], red_d[32];
    if (threadIdx.x == 0) {
        int f = 0;
        for (int B = 0; B < A; ++B) f += opa[B];
        first_s = f;
    }
    __syncthreads();
    const int first = first_s, n = opa[A];
    double aq = 0.0, ad = 0.0;
    for (int k = 0; k < n; ++k) {
        const size_t row = (size_t)(first + k) * norb;
        for (int nu = threadIdx.x; nu < norb; nu += blockDim.x) {
            const double s = Smat[row + nu], p = P[row + nu];
            aq += p * s;
            ad += (p - P0[row + nu]) * s;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        aq += __shfl_down_sync(0xffffffffu, aq, off);
        ad += __shfl_down_sync(0xffffffffu, ad, off);
    }
    const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (lane == 0) {
        red_q[w] = aq;
        red_d[w] = ad;
    }
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x / 32;
        aq = lane < nw ? red_q[lane] : 0.0;
        ad = lane < nw ? red_d[lane] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            aq += __shfl_down_sync(0xffffffffu, aq, off);
            ad += __shfl_down_sync(0xffffffffu, ad, off);
        }
        if (lane == 0) {
            q[A] = aq;
            dq[A] = ad;
        }
    }
}

// ----------------------------------------------------------------------------
// FP64 tiled GEMM engine.  C(m,n) = alpha * sum_k A(m,k) B(k,n) [+ beta C]
// with arbitrary element strides, a two-level batch index and optional split-K
// (atomic accumulation).  64x64x16 tiles, 256 threads, 4x4 outputs per thread.
// ----------------------------------------------------------------------------
enum { EPI_STORE = 0, EPI_ATOMIC = 1, EPI_RV = 2 };

struct GemmP {
    int M, N, K;
    const double *A;
    long long sam, sak, sa1, sa2;
    const double *B;
    long long sbk, sbn, sb1, sb2;
    double *C;
    long long scm, scn, sc1, sc2;
    double alpha, beta;
    int nb2;     // batch index z_b -> (z_b / nb2, z_b % nb2)
    int ksplit;  // gridDim.z = nbatch * ksplit
    int bscale_sqrt_omega;  // multiply B(k, n) by sqrt(omega[k])
    const double *omega;
    // EPI_RV: C(m,n) = omega[m]^p * v(m,n) + fac * sqrt(omega[m])^s * alpha * acc
    const double *v;
    long long ldv;
    double fac;
    int rv_square;  // 1: omega^2 v + fac sqrt(omega) acc (Hermitian), 0: omega v + fac acc
};

constexpr int BM = 64, BN = 64, BK = 16;

template <int EPI>
__global__ void __launch_bounds__(256) dgemm_kernel(GemmP p) {
    __shared__ double As[BK][BM + 1];
    __shared__ double Bs[BK][BN + 1];
    const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
    const int bm = blockIdx.y * BM, bn = blockIdx.x * BN;
    const int zb = blockIdx.z / p.ksplit, zk = blockIdx.z % p.ksplit;
    const int z1 = zb / p.nb2, z2 = zb % p.nb2;
    const double *A = p.A + z1 * p.sa1 + z2 * p.sa2;
    const double *B = p.B + z1 * p.sb1 + z2 * p.sb2;
    double *C = p.C + z1 * p.sc1 + z2 * p.sc2;
    const int kchunk = ((p.K + p.ksplit - 1) / p.ksplit + BK - 1) / BK * BK;
    const int k0 = zk * kchunk, k1 = min(p.K, k0 + kchunk);
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    const bool a_k_contig = (p.sak == 1);
    const bool b_n_contig = (p.sbn == 1);
    for (int kt = k0; kt < k1; kt += BK) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int e = tid + 256 * r;
            int mm, kk;
            if (a_k_contig) {
                kk = e % BK;
                mm = e / BK;
            } else {
                mm = e % BM;
                kk = e / BM;
            }
            const int gm = bm + mm, gk = kt + kk;
            As[kk][mm] = (gm < p.M && gk < k1) ? A[gm * p.sam + (long long)gk * p.sak] : 0.0;
            int nn, kb;
            if (b_n_contig) {
                nn = e % BN;
                kb = e / BN;
            } else {
                kb = e % BK;
                nn = e / BK;
            }
            const int gn = bn + nn, gkb = kt + kb;
            double bv = 0.0;
            if (gn < p.N && gkb < k1) {
                bv = B[(long long)gkb * p.sbk + gn * p.sbn];
                if (p.bscale_sqrt_omega) bv *= sqrt(p.omega[gkb]);
            }
            Bs[kb][nn] = bv;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = bm + ty + 16 * i;
        if (m >= p.M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = bn + tx + 16 * j;
            if (n >= p.N) continue;
            double *c = C + m * p.scm + n * p.scn;
            const double val = p.alpha * acc[i][j];
            if (EPI == EPI_STORE) {
                *c = (p.beta == 0.0) ? val : val + p.beta * (*c);
            } else if (EPI == EPI_ATOMIC) {
                atomicAdd(c, val);
            } else {
                const double om = p.omega[m];
                const double vv = p.v[m * p.ldv + n];
                *c = p.rv_square ? om * om * vv + p.fac * sqrt(om) * val : om * vv + p.fac * val;
            }
        }
    }
}

GemmP gemm_defaults() {
    GemmP p;
    memset(&p, 0, sizeof(p));
    p.alpha = 1.0;
    p.nb2 = 1;
    p.ksplit = 1;
    return p;
}

int launch_gemm(GemmP p, int epi, int nbatch, cudaStream_t st) {
    if (p.M <= 0 || p.N <= 0 || nbatch <= 0) return DFTB_OK;
    if (p.K <= 0) return fail(DFTB_ERR_BAD_SIZE, "gemm: K <= 0");
    dim3 grid(cdiv(p.N, BN), cdiv(p.M, BM), (unsigned)(nbatch * p.ksplit));
    if (grid.y > 65535u || grid.z > 65535u) return fail(DFTB_ERR_BAD_SIZE, "gemm: grid too large");
    if (epi == EPI_STORE)
        dgemm_kernel<EPI_STORE><<<grid, 256, 0, st>>>(p);
    else if (epi == EPI_ATOMIC)
        dgemm_kernel<EPI_ATOMIC><<<grid, 256, 0, st>>>(p);
    else
        dgemm_kernel<EPI_RV><<<grid, 256, 0, st>>>(p);
    return check_launch("dgemm_kernel");
}

// choose a K split so that about 4 CTAs per SM are in flight
int pick_ksplit(int M, int N, int K, int nbatch) {
    const long long tiles = (long long)cdiv(M, BM) * cdiv(N, BN) * nbatch;
    long long want = (148LL * 4 + tiles - 1) / tiles;
    const long long maxs = (K + 4 * BK - 1) / (4 * BK);  // at least 4 k-tiles per split
    if (want > maxs) want = maxs;
    if (want < 1) want = 1;
    if (want * nbatch > 65535) want = 65535 / nbatch;
    return (int)(want < 1 ? 1 : want);
}

// ----------------------------------------------------------------------------
// transition charges
// ----------------------------------------------------------------------------
__global__ void prefix_kernel(int nat, const int *opa, int *first) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        int f = 0;
        for (int A = 0; A < nat; ++A) {
            first[A] = f;
            f += opa[A];
        }
        first[nat] = f;
    }
}

// q[A][p][q] = 1/2 sum_{mu in A} (C1[mu][p] Sc2[mu][q] + C2[mu][q] Sc1[mu][p]).
// The output (nat x n1 x n2 doubles) is the only large stream, so the kernel is built around writing it at
// HBM speed: a CTA owns a TC_TP x TC_TQ tile of (p, q) for a run of TC_ATOMS atoms.  Per atom the rows mu of
// C1, Sc1 (TC_TP wide) and C2, Sc2 (TC_TQ wide) are staged in shared memory by cp.async, one atom ahead
// (three buffers, so one barrier per atom suffices), and the next atom's rows arrive while the current
// atom's outputs are stored; every thread writes
// adjacent pairs of q with 16-byte stores (each warp stores 512 contiguous bytes of one row p).  Atoms with up
// to TC_MAXO orbitals (s and p shells) take the staged path; larger ones read their rows from global memory.
constexpr int TC_TP = 64, TC_TQ = 128, TC_THREADS = 256, TC_MAXO = 4, TC_ATOMS = 8, TC_ROWS = 4;

__device__ __forceinline__ void cp_async8(void *dst, const double *src, bool valid) {
    // 8-byte asynchronous copy; with src-size 0 the destination is zero-filled and nothing is read
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(valid ? 8 : 0)
                 : "memory");
}

struct TcStage {
    double c1[TC_MAXO][TC_TP], s1[TC_MAXO][TC_TP], c2[TC_MAXO][TC_TQ], s2[TC_MAXO][TC_TQ];
};

__device__ __forceinline__ void tc_stage(TcStage &b, int f0, int nA, int n1, int n2, int p0, int q0,
                                         const double *C1, const double *Sc1, const double *C2,
                                         const double *Sc2) {
    for (int i = threadIdx.x; i < nA * TC_TP; i += TC_THREADS) {
        const int j = i / TC_TP, pp = i % TC_TP, p = p0 + pp;
        const bool v = p < n1;
        const size_t o = v ? (size_t)(f0 + j) * n1 + p : 0;
        cp_async8(&b.c1[j][pp], C1 + o, v);
        cp_async8(&b.s1[j][pp], Sc1 + o, v);
    }
    for (int i = threadIdx.x; i < nA * TC_TQ; i += TC_THREADS) {
        const int j = i / TC_TQ, qq = i % TC_TQ, qi = q0 + qq;
        const bool v = qi < n2;
        const size_t o = v ? (size_t)(f0 + j) * n2 + qi : 0;
        cp_async8(&b.c2[j][qq], C2 + o, v);
        cp_async8(&b.s2[j][qq], Sc2 + o, v);
    }
}

template <bool VEC>
__global__ void __launch_bounds__(TC_THREADS) tc_tile_kernel(int nat, int n1, int n2, const int *first,
                                                             const double *__restrict__ C1,
                                                             const double *__restrict__ Sc1,
                                                             const double *__restrict__ C2,
                                                             const double *__restrict__ Sc2, double *q) {
    __shared__ __align__(16) TcStage buf[3];
    const int tid = threadIdx.x;
    const int qp = tid & 63, pg = tid >> 6;  // q pair within the tile; row group
    const int q0 = blockIdx.x * TC_TQ, p0 = blockIdx.y * TC_TP;
    const int qg = q0 + 2 * qp;
    const int A0 = blockIdx.z * TC_ATOMS;
    const int A1 = min(nat, A0 + TC_ATOMS);
    // prologue: stage the first atom
    {
        const int f0 = first[A0], nA = first[A0 + 1] - f0;
        if (nA <= TC_MAXO) tc_stage(buf[0], f0, nA, n1, n2, p0, q0, C1, Sc1, C2, Sc2);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int A = A0; A < A1; ++A) {
        const int k = A - A0;
        const int f0 = first[A], nA = first[A + 1] - f0;
        const bool staged = nA <= TC_MAXO;
        if (A + 1 < A1) {
            // next atom's rows into buffer (k + 1) % 3, last read in iteration k - 2: every thread has
            // passed the barrier of iteration k - 1 since, so those reads are finished
            const int g0 = first[A + 1], nB = first[A + 2] - g0;
            if (nB <= TC_MAXO) tc_stage(buf[(k + 1) % 3], g0, nB, n1, n2, p0, q0, C1, Sc1, C2, Sc2);
            asm volatile("cp.async.commit_group;" ::: "memory");
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        const TcStage &sb = buf[k % 3];
        for (int batch = 0; batch < TC_TP / (4 * TC_ROWS); ++batch) {
            double acc0[TC_ROWS], acc1[TC_ROWS];
#pragma unroll
            for (int r = 0; r < TC_ROWS; ++r) acc0[r] = acc1[r] = 0.0;
            // this thread's rows: TC_ROWS consecutive ones, so that the staged C1 / Sc1 values of two rows
            // come in one 16-byte shared-memory read (the same address for the whole warp: a broadcast)
            const int pl0 = (batch * 4 + pg) * TC_ROWS;
            if (staged) {
                for (int j = 0; j < nA; ++j) {
                    const double2 c2 = *reinterpret_cast<const double2 *>(&sb.c2[j][2 * qp]);
                    const double2 s2 = *reinterpret_cast<const double2 *>(&sb.s2[j][2 * qp]);
#pragma unroll
                    for (int r = 0; r < TC_ROWS; r += 2) {
                        const double2 a1 = *reinterpret_cast<const double2 *>(&sb.c1[j][pl0 + r]);
                        const double2 b1 = *reinterpret_cast<const double2 *>(&sb.s1[j][pl0 + r]);
                        acc0[r] += a1.x * s2.x + c2.x * b1.x;
                        acc1[r] += a1.x * s2.y + c2.y * b1.x;
                        acc0[r + 1] += a1.y * s2.x + c2.x * b1.y;
                        acc1[r + 1] += a1.y * s2.y + c2.y * b1.y;
                    }
                }
            } else {
                for (int j = 0; j < nA; ++j) {
                    const size_t r2 = (size_t)(f0 + j) * n2;
                    const double c2a = qg < n2 ? C2[r2 + qg] : 0.0, s2a = qg < n2 ? Sc2[r2 + qg] : 0.0;
                    const double c2b = qg + 1 < n2 ? C2[r2 + qg + 1] : 0.0;
                    const double s2b = qg + 1 < n2 ? Sc2[r2 + qg + 1] : 0.0;
#pragma unroll
                    for (int r = 0; r < TC_ROWS; ++r) {
                        const int p = p0 + pl0 + r;
                        const size_t r1 = (size_t)(f0 + j) * n1 + p;
                        const double a1 = p < n1 ? C1[r1] : 0.0, b1 = p < n1 ? Sc1[r1] : 0.0;
                        acc0[r] += a1 * s2a + c2a * b1;
                        acc1[r] += a1 * s2b + c2b * b1;
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < TC_ROWS; ++r) {
                const int p = p0 + pl0 + r;  // the same for the whole warp
                if (p >= n1) continue;
                double *row = q + ((size_t)A * n1 + p) * n2;
                if (VEC) {
                    // 16-byte stores on every row: a row whose tile segment starts on an odd element (odd n2)
                    // stores the pairs (qg + 1, qg + 2), the second value taken from the next lane; lane 0
                    // stores its first column and lane 31 its second as single elements
                    const int lane = tid & 31;
                    const double nxt = __shfl_down_sync(0xffffffffu, acc0[r], 1);
                    const bool odd = (reinterpret_cast<uintptr_t>(row + q0) & 15) != 0;  // warp-uniform
                    if (!odd) {
                        if (qg + 1 < n2)
                            *reinterpret_cast<double2 *>(row + qg) = make_double2(0.5 * acc0[r], 0.5 * acc1[r]);
                        else if (qg < n2)
                            row[qg] = 0.5 * acc0[r];
                    } else {
                        if (lane == 0 && qg < n2) row[qg] = 0.5 * acc0[r];
                        if (lane < 31 && qg + 2 < n2)
                            *reinterpret_cast<double2 *>(row + qg + 1) = make_double2(0.5 * acc1[r], 0.5 * nxt);
                        else if (qg + 1 < n2)
                            row[qg + 1] = 0.5 * acc1[r];
                    }
                } else {
                    if (qg >= n2) continue;
                    row[qg] = 0.5 * acc0[r];
                    if (qg + 1 < n2) row[qg + 1] = 0.5 * acc1[r];
                }
            }
        }
    }
}

// one (n1 x n2) block of transition charges for all atoms
int launch_tc(int nat, int n1, int n2, const int *first, const double *C1, const double *Sc1, const double *C2,
              const double *Sc2, double *out, cudaStream_t st, const char *where) {
    dim3 grid(cdiv(n2, TC_TQ), cdiv(n1, TC_TP), cdiv(nat, TC_ATOMS));
    if (grid.y > 65535u || grid.z > 65535u) return fail(DFTB_ERR_BAD_SIZE, "trans_charges: grid too large");
    // 16-byte stores need an aligned base; rows that start on an odd element shift their pairs by one
    if (((uintptr_t)out & 15) == 0)
        tc_tile_kernel<true><<<grid, TC_THREADS, 0, st>>>(nat, n1, n2, first, C1, Sc1, C2, Sc2, out);
    else
        tc_tile_kernel<false><<<grid, TC_THREADS, 0, st>>>(nat, n1, n2, first, C1, Sc1, C2, Sc2, out);
    return check_launch(where);
}

// diagonal q^{pp}_A
__global__ void tc_diag_kernel(int n, const int *first, const double *C, const double *Sc, double *q) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int A = blockIdx.y;
    if (p >= n) return;
    double acc = 0.0;
    for (int mu = first[A]; mu < first[A + 1]; ++mu)
        acc += C[(size_t)mu * n + p] * Sc[(size_t)mu * n + p] + C[(size_t)mu * n + p] * Sc[(size_t)mu * n + p];
    q[(size_t)A * n + p] = 0.5 * acc;
}

// cuBLAS for plain FP64 GEMMs (the Coulomb product's two, the transition charges' S.C).  The library is resolved at run
// time (dlopen / dlsym, reusing the copy the process has already loaded), so the shared library
// loads without it and the product falls back to dgemm_kernel.
using blas_create_t = cublasStatus_t (*)(cublasHandle_t *);
using blas_stream_t = cublasStatus_t (*)(cublasHandle_t, cudaStream_t);
using blas_dgemm_t = cublasStatus_t (*)(cublasHandle_t, cublasOperation_t, cublasOperation_t, int, int, int,
                                        const double *, const double *, int, const double *, int, const double *,
                                        double *, int);
struct Blas {
    blas_create_t create = nullptr;
    blas_stream_t set_stream = nullptr;
    blas_dgemm_t dgemm = nullptr;
    bool ok = false;
};

Blas &blas() {
    static Blas b;
    static std::once_flag once;
    std::call_once(once, [] {
        void *h = dlopen("libcublas.so.12", RTLD_NOW | RTLD_NOLOAD);
        if (!h) h = dlopen("libcublas.so.12", RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libcublas.so", RTLD_NOW | RTLD_GLOBAL);
        if (!h) return;
        b.create = reinterpret_cast<blas_create_t>(dlsym(h, "cublasCreate_v2"));
        b.set_stream = reinterpret_cast<blas_stream_t>(dlsym(h, "cublasSetStream_v2"));
        b.dgemm = reinterpret_cast<blas_dgemm_t>(dlsym(h, "cublasDgemm_v2"));
        b.ok = b.create && b.set_stream && b.dgemm;
    });
    return b;
}

// one handle per host thread and device, bound to the caller's stream; nullptr if unavailable
cublasHandle_t blas_handle(cudaStream_t st) {
    Blas &b = blas();
    if (!b.ok) return nullptr;
    thread_local cublasHandle_t handles[64] = {nullptr};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    if (!handles[dev] && b.create(&handles[dev]) != CUBLAS_STATUS_SUCCESS) {
        handles[dev] = nullptr;
        return nullptr;
    }
    if (b.set_stream(handles[dev], st) != CUBLAS_STATUS_SUCCESS) return nullptr;
    return handles[dev];
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// use_blas: S.C by cuBLAS when it resolves (the entry points that may allocate; the allocation-free one
// keeps the library's own dgemm_kernel)
int trans_charges_common(int norb, int nat, int nocc, int nvirt, const double *co, const double *cv,
                         const double *Smat, const int *opa, void *work, size_t work_bytes, cudaStream_t st,
                         double **sco, double **scv, int **first, bool use_blas = true) {
    if (norb <= 0 || nat <= 0 || nocc < 0 || nvirt < 0) return fail(DFTB_ERR_BAD_SIZE, "trans_charges: sizes");
    if (!Smat || !opa || (nocc > 0 && !co) || (nvirt > 0 && !cv)) return fail(DFTB_ERR_NULL, "trans_charges: null");
    if (!work || work_bytes < dftb_trans_charges_workspace_size(norb, nocc, nvirt))
        return fail(DFTB_ERR_WORKSPACE, "trans_charges: workspace too small");
    char *w = (char *)work;
    *sco = (double *)w;
    w += align256(sizeof(double) * (size_t)norb * nocc);
    *scv = (double *)w;
    w += align256(sizeof(double) * (size_t)norb * nvirt);
    *first = (int *)w;
    prefix_kernel<<<1, 1, 0, st>>>(nat, opa, *first);
    int rc = check_launch("prefix_kernel");
    if (rc) return rc;
    // Sc = S . C (S is symmetric)
    cublasHandle_t bh = use_blas ? blas_handle(st) : nullptr;
    for (int b = 0; b < 2; ++b) {
        const int n = b == 0 ? nocc : nvirt;
        if (n == 0) continue;
        if (bh) {
            // row-major Sc (norb x n) is the column-major Sc^T = C^T S^T = C^T S
            const double one = 1.0, zero = 0.0;
            if (blas().dgemm(bh, CUBLAS_OP_N, CUBLAS_OP_N, n, norb, norb, &one, b == 0 ? co : cv, n, Smat, norb, &zero,
                             b == 0 ? *sco : *scv, n) != CUBLAS_STATUS_SUCCESS)
                return fail(DFTB_ERR_CUDA, "trans_charges: cublasDgemm (S C) failed");
            continue;
        }
        GemmP p = gemm_defaults();
        p.M = norb;
        p.N = n;
        p.K = norb;
        p.A = Smat;
        p.sam = norb;
        p.sak = 1;
        p.B = b == 0 ? co : cv;
        p.sbk = n;
        p.sbn = 1;
        p.C = b == 0 ? *sco : *scv;
        p.scm = n;
        p.scn = 1;
        rc = launch_gemm(p, EPI_STORE, 1, st);
        if (rc) return rc;
    }
    return DFTB_OK;
}

// ----------------------------------------------------------------------------
// Davidson helpers
// ----------------------------------------------------------------------------
__global__ void precondition_kernel(int nov, int nnew, const double *W, int ldw, const int *src, const int *state,
                                    const double *w, const double *omega, double *Q, int ldq) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nov * nnew) return;
    const int ia = (int)(idx / nnew), c = (int)(idx % nnew);
    const double om = omega[ia];
    double wd = w[state[c]] - om;
    if (fabs(wd) < 1.0e-6) wd = 1.0e-6 * om;
    Q[(size_t)ia * ldq + c] = W[(size_t)ia * ldw + src[c]] / wd;
}

__global__ void residual_kernel(int nov, int ncol, const double *AV, int ldav, const double *X, int ldx,
                                const double *lam, double *W, int ldw, double *nrm2) {
    const int c = blockIdx.y;
    double acc = 0.0;
    for (int ia = blockIdx.x * blockDim.x + threadIdx.x; ia < nov; ia += gridDim.x * blockDim.x) {
        const double r = AV[(size_t)ia * ldav + c] - lam[c] * X[(size_t)ia * ldx + c];
        W[(size_t)ia * ldw + c] = r;
        acc += r * r;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    __shared__ double red[32];
    const int wi = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (lane == 0) red[wi] = acc;
    __syncthreads();
    if (wi == 0) {
        acc = lane < (int)(blockDim.x / 32) ? red[lane] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
        if (lane == 0) atomicAdd(&nrm2[c], acc);
    }
}

// Row-blocked form for ncol <= 256: a block of 256 threads covers R = 256 / ncol rows x all columns
// per step (consecutive threads read consecutive elements of a row), so each thread keeps one
// column and its squared norm in a register; the R partial sums of a column meet in shared memory.
__global__ void residual_rows_kernel(int nov, int ncol, const double *AV, int ldav, const double *X, int ldx,
                                     const double *lam, double *W, int ldw, double *nrm2) {
    __shared__ double red[256];
    const int R = blockDim.x / ncol;
    const int tc = threadIdx.x % ncol, tr = threadIdx.x / ncol;
    double acc = 0.0;
    if (tr < R) {
        const double l = lam[tc];
        for (long long ia = (long long)blockIdx.x * R + tr; ia < nov; ia += (long long)gridDim.x * R) {
            const double r = AV[ia * ldav + tc] - l * X[ia * ldx + tc];
            W[ia * ldw + tc] = r;
            acc += r * r;
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x < ncol) {
        double sum = 0.0;
        for (int j = 0; j < R; ++j) sum += red[threadIdx.x + j * ncol];
        atomicAdd(&nrm2[threadIdx.x], sum);
    }
}

__global__ void sqrt_kernel(int n, double *x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = sqrt(x[i]);
}

// us = omega o vs (the first term of (A-B).v without Coulomb)
__global__ void omega_scale_kernel(long long nov, int nvec, const double *omega, const double *vs, double *us) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nov * nvec) return;
    us[idx] = omega[idx / nvec] * vs[idx];
}

// Coulomb part shared by the Hermitian and (A+B) products (cuBLAS handle: blas() above).
// us(ia, n) = omega_ia v(ia, n) + fac us(ia, n)   (in place; the non-Hermitian Coulomb epilogue)
__global__ void rv_inplace_kernel(long long total, int nvec, const double *omega, const double *vs, double *us,
                                  double fac) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    us[i] = omega[i / nvec] * vs[i] + fac * us[i];
}

//   T = q_ov . (s o V)   (split-K, atomic), G = gamma . T,  us = epilogue(q_ov^T G)
// The non-Hermitian form (s = 1) runs its two large GEMMs in cuBLAS when it is available:
// row-major X (r x c) is the column-major X^T, so T^T = V^T q_ov^T and us^T = G^T q_ov.
int coulomb_product(int nat, int nov, int nvec, const double *gamma, const double *q_ov, const double *omega,
                    const double *vs, double *us, double *T, double *G, int hermitian, cudaStream_t st) {
    cublasHandle_t bh = hermitian ? nullptr : blas_handle(st);
    if (bh) {
        const double one = 1.0, zero = 0.0;
        if (blas().dgemm(bh, CUBLAS_OP_N, CUBLAS_OP_N, nvec, nat, nov, &one, vs, nvec, q_ov, nov, &zero, T, nvec) !=
            CUBLAS_STATUS_SUCCESS)
            return fail(DFTB_ERR_CUDA, "coulomb: cublasDgemm (q_ov V) failed");
        GemmP g = gemm_defaults();
        g.M = nat;
        g.N = nvec;
        g.K = nat;
        g.A = gamma;
        g.sam = nat;
        g.sak = 1;
        g.B = T;
        g.sbk = nvec;
        g.sbn = 1;
        g.C = G;
        g.scm = nvec;
        g.scn = 1;
        int rc = launch_gemm(g, EPI_STORE, 1, st);
        if (rc) return rc;
        if (blas().dgemm(bh, CUBLAS_OP_N, CUBLAS_OP_T, nvec, nov, nat, &one, G, nvec, q_ov, nov, &zero, us, nvec) !=
            CUBLAS_STATUS_SUCCESS)
            return fail(DFTB_ERR_CUDA, "coulomb: cublasDgemm (q_ov^T G) failed");
        const long long total = (long long)nov * nvec;
        rv_inplace_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(total, nvec, omega, vs, us, 4.0);
        return check_launch("rv_inplace_kernel");
    }
    cudaError_t e = cudaMemsetAsync(T, 0, sizeof(double) * (size_t)nat * nvec, st);
    if (e != cudaSuccess) return fail(DFTB_ERR_CUDA, "memset T");
    GemmP p = gemm_defaults();
    p.M = nat;
    p.N = nvec;
    p.K = nov;
    p.A = q_ov;
    p.sam = nov;
    p.sak = 1;
    p.B = vs;
    p.sbk = nvec;
    p.sbn = 1;
    p.C = T;
    p.scm = nvec;
    p.scn = 1;
    p.bscale_sqrt_omega = hermitian;
    p.omega = omega;
    p.ksplit = pick_ksplit(nat, nvec, nov, 1);
    int rc = launch_gemm(p, EPI_ATOMIC, 1, st);
    if (rc) return rc;
    GemmP g = gemm_defaults();
    g.M = nat;
    g.N = nvec;
    g.K = nat;
    g.A = gamma;
    g.sam = nat;
    g.sak = 1;
    g.B = T;
    g.sbk = nvec;
    g.sbn = 1;
    g.C = G;
    g.scm = nvec;
    g.scn = 1;
    rc = launch_gemm(g, EPI_STORE, 1, st);
    if (rc) return rc;
    GemmP u = gemm_defaults();
    u.M = nov;
    u.N = nvec;
    u.K = nat;
    u.A = q_ov;  // (q_ov)^T: element (ia, A) at A*nov + ia
    u.sam = 1;
    u.sak = nov;
    u.B = G;
    u.sbk = nvec;
    u.sbn = 1;
    u.C = us;
    u.scm = nvec;
    u.scn = 1;
    u.omega = omega;
    u.v = vs;
    u.ldv = nvec;
    u.fac = 4.0;
    u.rv_square = hermitian;
    return launch_gemm(u, EPI_RV, 1, st);
}

// Exchange terms in the transition-charge form, accumulated into us:
//   us += sK1 * K1 v + sK2 * K2 v
int exchange_products(int nat, int nocc, int nvirt, int nvec, const double *g_lr, const double *q_oo,
                      const double *q_ov, const double *q_vv, const double *vs, double *us, double sK1, double sK2,
                      double *work, cudaStream_t st) {
    const long long no = nocc, nv = nvirt, m = nvec;
    int rc;
    // ---- K1: us[i][a][c] += sK1 * sum_B sum_b (sum_j Z[B][i][j] v[j][b][c]) q_vv[B][a][b],
    //          Z[B][i][j] = sum_A g_lr[A][B] q_oo[A][i][j]
    double *Z = work, *T = work + nat * no * no;
    GemmP p = gemm_defaults();
    p.M = nat;
    p.N = (int)(no * no);
    p.K = nat;
    p.A = g_lr;
    p.sam = 1;
    p.sak = nat;
    p.B = q_oo;
    p.sbk = no * no;
    p.sbn = 1;
    p.C = Z;
    p.scm = no * no;
    p.scn = 1;
    if ((rc = launch_gemm(p, EPI_STORE, 1, st))) return rc;
    p = gemm_defaults();
    p.M = (int)no;
    p.N = (int)(nv * m);
    p.K = (int)no;
    p.A = Z;
    p.sam = no;
    p.sak = 1;
    p.sa1 = no * no;
    p.B = vs;
    p.sbk = nv * m;
    p.sbn = 1;
    p.C = T;
    p.scm = nv * m;
    p.scn = 1;
    p.sc1 = no * nv * m;
    if ((rc = launch_gemm(p, EPI_STORE, nat, st))) return rc;
    p = gemm_defaults();
    p.M = (int)no;
    p.N = (int)nv;
    p.K = (int)nv;
    p.A = T;  // (i, b) of batch (B, c): T[B][i][b][c]
    p.sam = nv * m;
    p.sak = m;
    p.sa1 = no * nv * m;
    p.sa2 = 1;
    p.B = q_vv;  // (b, a) = q_vv[B][a][b]
    p.sbk = 1;
    p.sbn = nv;
    p.sb1 = nv * nv;
    p.sb2 = 0;
    p.C = us;  // (i, a) of column c
    p.scm = nv * m;
    p.scn = m;
    p.sc1 = 0;
    p.sc2 = 1;
    p.nb2 = (int)m;
    p.alpha = sK1;
    if ((rc = launch_gemm(p, EPI_ATOMIC, (int)(nat * m), st))) return rc;
    // ---- K2: us[i][a][c] += sK2 * sum_A sum_b q_ov[A][i][b] W[A][a][b][c],
    //          W[A][a][b][c] = sum_j Z2[A][j][a] v[j][b][c],  Z2 = g_lr . q_ov
    double *Z2 = work, *W = work + nat * no * nv;
    p = gemm_defaults();
    p.M = nat;
    p.N = (int)(no * nv);
    p.K = nat;
    p.A = g_lr;
    p.sam = nat;
    p.sak = 1;
    p.B = q_ov;
    p.sbk = no * nv;
    p.sbn = 1;
    p.C = Z2;
    p.scm = no * nv;
    p.scn = 1;
    if ((rc = launch_gemm(p, EPI_STORE, 1, st))) return rc;
    p = gemm_defaults();
    p.M = (int)nv;
    p.N = (int)(nv * m);
    p.K = (int)no;
    p.A = Z2;  // (a, j) = Z2[A][j][a]
    p.sam = 1;
    p.sak = nv;
    p.sa1 = no * nv;
    p.B = vs;
    p.sbk = nv * m;
    p.sbn = 1;
    p.C = W;
    p.scm = nv * m;
    p.scn = 1;
    p.sc1 = nv * nv * m;
    if ((rc = launch_gemm(p, EPI_STORE, nat, st))) return rc;
    p = gemm_defaults();
    p.M = (int)no;
    p.N = (int)nv;
    p.K = (int)nv;
    p.A = q_ov;  // (i, b) = q_ov[A][i][b]
    p.sam = nv;
    p.sak = 1;
    p.sa1 = no * nv;
    p.B = W;  // (b, a) = W[A][a][b][c]
    p.sbk = m;
    p.sbn = nv * m;
    p.sb1 = nv * nv * m;
    p.sb2 = 1;
    p.C = us;
    p.scm = nv * m;
    p.scn = m;
    p.sc2 = 1;
    p.nb2 = (int)m;
    p.alpha = sK2;
    return launch_gemm(p, EPI_ATOMIC, (int)(nat * m), st);
}

int check_products(int nat, int nocc, int nvirt, int nvec, int lc, const double *g, const double *g_lr,
                   const double *q_oo, const double *q_ov, const double *q_vv, const double *omega, const double *vs,
                   double *us, void *work, size_t work_bytes) {
    if (nat <= 0 || nocc <= 0 || nvirt <= 0 || nvec <= 0) return fail(DFTB_ERR_BAD_SIZE, "apbv: sizes");
    if (!g || !q_ov || !omega || !vs || !us) return fail(DFTB_ERR_NULL, "apbv: null");
    if (lc && (!g_lr || !q_oo || !q_vv)) return fail(DFTB_ERR_NULL, "apbv: lc needs g_lr, q_oo, q_vv");
    const size_t need = lc ? dftb_apbv_workspace_size(nat, nocc, nvirt, nvec)
                           : dftb_hermitian_rv_workspace_size(nat, nvec);
    if (!work || work_bytes < need) return fail(DFTB_ERR_WORKSPACE, "apbv: workspace too small");
    return DFTB_OK;
}

// ---------------------------------------------------------------------------- layout changes of column blocks

// Y (cols x rows) = X^T through a 32 x 32 shared-memory tile: reads and writes run along rows of 256 bytes
// (a strided element copy moves a whole 32-byte sector per 8-byte element on one side)
__global__ void __launch_bounds__(256) transpose_f64_kernel(int rows, int cols, const double *__restrict__ X,
                                                            long long ldx, double *__restrict__ Y, long long ldy) {
    __shared__ double t[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int k = ty; k < 32; k += 8) {
        const int r = r0 + k, c = c0 + tx;
        if (r < rows && c < cols) t[k][tx] = X[(long long)r * ldx + c];
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int c = c0 + k, r = r0 + tx;
        if (c < cols && r < rows) Y[(long long)c * ldy + r] = t[tx][k];
    }
}

// K_y[(i nvirt + a) m + c] = Kall[c][2a + y][i] (FP32 -> FP64): the exchange's last launch writes, for each
// product column c, K1^T and K2^T with their rows interleaved.  A CTA takes one a and a run of 32 i for
// every c: it reads 128-byte pieces of Kall rows and writes whole m-long rows of K1 and K2.
__global__ void __launch_bounds__(256) exchange_unpack_kernel(int m, int nv, int no, const float *__restrict__ Kall,
                                                              double *__restrict__ K1, double *__restrict__ K2) {
    __shared__ float t[2][64][33];
    const int a = blockIdx.y, i0 = blockIdx.x * 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int c0 = 0; c0 < m; c0 += 64) {
        const int mc = min(64, m - c0);
        for (int row = wid; row < 2 * mc; row += 8) {
            const int c = row >> 1, y = row & 1, i = i0 + lane;
            t[y][c][lane] = i < no ? Kall[((long long)(c0 + c) * 2 * nv + 2 * a + y) * no + i] : 0.0f;
        }
        __syncthreads();
        for (int row = wid; row < 64; row += 8) {
            const int il = row >> 1, y = row & 1, i = i0 + il;
            if (i < no) {
                double *dst = (y ? K2 : K1) + ((long long)i * nv + a) * m + c0;
                for (int c = lane; c < mc; c += 32) dst[c] = (double)t[y][c][il];
            }
        }
        __syncthreads();
    }
}

}  // namespace

// ============================================================================
// extern "C" entry points
// ============================================================================
extern "C" {

const char *dftb_version(void) { return "dftbaby_b200 0.1 (sm_100a, fp64)"; }
const char *dftb_last_error(void) { return g_last_error; }

int dftb_directional_cosines(int nat, const double *pos, double *r, double *x, double *y, double *z, void *stream) {
    if (nat <= 0) return fail(DFTB_ERR_BAD_SIZE, "directional_cosines: nat");
    if (!pos || !r || !x || !y || !z) return fail(DFTB_ERR_NULL, "directional_cosines: null");
    dim3 grid(cdiv(nat, 128), nat);
    dircos_kernel<<<grid, 128, 0, S(stream)>>>(nat, pos, r, x, y, z);
    return check_launch("dircos_kernel");
}

int dftb_h0_and_s(int norb, int nat, const int *ind, const int *typ, const int *ls, const int *ms, const double *r,
                  const double *x, const double *y, const double *z, const int *mprox, const double *orben, int deg,
                  const int *tab_filled, const double *S_knots, const double *S_coefs, const double *H_knots,
                  const double *H_coefs, int npair, int nsk, int npts, double *Sm, double *H0, void *stream) {
    if (norb <= 0 || nat <= 0 || npair <= 0 || nsk <= 0 || npts < 8) return fail(DFTB_ERR_BAD_SIZE, "h0_and_s: sizes");
    if (deg != 3) return fail(DFTB_ERR_UNSUPPORTED, "h0_and_s: only cubic splines");
    if (!ind || !typ || !ls || !ms || !r || !x || !y || !z || !mprox || !orben || !tab_filled || !S_knots ||
        !S_coefs || !H_knots || !H_coefs || !Sm || !H0)
        return fail(DFTB_ERR_NULL, "h0_and_s: null");
    OrbTables O{ind, typ, ls, ms};
    SkTables TS{tab_filled, S_knots, S_coefs, nsk, npts};
    SkTables TH{tab_filled, H_knots, H_coefs, nsk, npts};
    dim3 grid(cdiv(norb, 128), norb);
    h0_and_s_kernel<<<grid, 128, 0, S(stream)>>>(norb, nat, O, r, x, y, z, mprox, orben, TS, TH, Sm, H0);
    return check_launch("h0_and_s_kernel");
}

int dftb_dipole_matrix(int norb, int nat, const int *ind, const int *typ, const int *ls, const int *ms,
                       const double *r, const double *x, const double *y, const double *z, const double *pos,
                       const int *mprox, const double *Sm, int deg, const int *tab_filled_D, const double *D_knots,
                       const double *D_coefs, int npair, int nskd, int npts, double *D, void *stream) {
    if (norb <= 0 || nat <= 0 || npair <= 0 || nskd <= 0 || npts < 8)
        return fail(DFTB_ERR_BAD_SIZE, "dipole_matrix: sizes");
    if (deg != 3) return fail(DFTB_ERR_UNSUPPORTED, "dipole_matrix: only cubic splines");
    if (!ind || !typ || !ls || !ms || !r || !x || !y || !z || !pos || !mprox || !Sm || !tab_filled_D ||
        !D_knots || !D_coefs || !D)
        return fail(DFTB_ERR_NULL, "dipole_matrix: null");
    OrbTables O{ind, typ, ls, ms};
    SkTables TD{tab_filled_D, D_knots, D_coefs, nskd, npts};
    dim3 grid(cdiv(norb, 128), norb);
    dipole_kernel<<<grid, 128, 0, S(stream)>>>(norb, nat, O, r, x, y, z, pos, mprox, Sm, TD, D);
    return check_launch("dipole_kernel");
}

int dftb_gamma_matrices(int nat, const double *r, const double *sigma, double r_lr, double *gamma, double *gamma_lr,
                        void *stream) {
    if (nat <= 0) return fail(DFTB_ERR_BAD_SIZE, "gamma: nat");
    if (!r || !sigma || !gamma) return fail(DFTB_ERR_NULL, "gamma: null");
    dim3 grid(cdiv(nat, 128), nat);
    gamma_kernel<<<grid, 128, 0, S(stream)>>>(nat, r, sigma, r_lr, gamma, gamma_lr);
    return check_launch("gamma_kernel");
}

int dftb_ao_expand(int norb, int nat, const int *ind, const double *g, double *G, void *stream) {
    if (norb <= 0 || nat <= 0) return fail(DFTB_ERR_BAD_SIZE, "ao_expand: sizes");
    if (!ind || !g || !G) return fail(DFTB_ERR_NULL, "ao_expand: null");
    dim3 grid(cdiv(norb, 128), norb);
    ao_expand_kernel<<<grid, 128, 0, S(stream)>>>(norb, nat, ind, g, G);
    return check_launch("ao_expand_kernel");
}

int dftb_scc_hamiltonian(int norb, int nat, const int *ind, const double *H0, const double *Sm, const double *gamma,
                         const double *dq, double *estat, double *H, void *stream) {
    if (norb <= 0 || nat <= 0) return fail(DFTB_ERR_BAD_SIZE, "scc_hamiltonian: sizes");
    if (!ind || !H0 || !Sm || !gamma || !dq || !estat || !H) return fail(DFTB_ERR_NULL, "scc_hamiltonian: null");
    estat_kernel<<<cdiv(nat, 8), 256, 0, S(stream)>>>(nat, gamma, dq, estat);
    int rc = check_launch("estat_kernel");
    if (rc) return rc;
    dim3 grid(cdiv(norb, 128), norb);
    scc_h_kernel<<<grid, 128, 0, S(stream)>>>(norb, ind, H0, Sm, estat, H);
    return check_launch("scc_h_kernel");
}

int dftb_monopoles(int norb, int nat, const double *P, const double *P0, const double *Sm, const int *opa, double *q,
                   double *dq, void *stream) {
    if (norb <= 0 || nat <= 0) return fail(DFTB_ERR_BAD_SIZE, "monopoles: sizes");
    if (!P || !P0 || !Sm || !opa || !q || !dq) return fail(DFTB_ERR_NULL, "monopoles: null");
    monopoles_kernel<<<nat, 256, 0, S(stream)>>>(norb, nat, P, P0, Sm, opa, q, dq);
    return check_launch("monopoles_kernel");
}

size_t dftb_trans_charges_workspace_size(int norb, int nocc, int nvirt) {
    if (norb <= 0 || nocc < 0 || nvirt < 0) return 0;
    return align256(sizeof(double) * (size_t)norb * nocc) + align256(sizeof(double) * (size_t)norb * nvirt) +
           align256(sizeof(int) * ((size_t)norb + 1));
}

int dftb_trans_charges(int norb, int nat, int nocc, int nvirt, const double *co, const double *cv, const double *Sm,
                       const int *opa, double *q_oo, double *q_ov, double *q_vv, void *work, size_t work_bytes,
                       void *stream) {
    cudaStream_t st = S(stream);
    double *sco, *scv;
    int *first;
    if (nat > norb) return fail(DFTB_ERR_BAD_SIZE, "trans_charges: nat > norb");
    if (nat > 65535) return fail(DFTB_ERR_BAD_SIZE, "trans_charges: nat > 65535");
    int rc = trans_charges_common(norb, nat, nocc, nvirt, co, cv, Sm, opa, work, work_bytes, st, &sco, &scv, &first);
    if (rc) return rc;
    struct Blk {
        double *out;
        const double *c1, *s1, *c2, *s2;
        int n1, n2;
    } blks[3] = {{q_oo, co, sco, co, sco, nocc, nocc},
                 {q_ov, co, sco, cv, scv, nocc, nvirt},
                 {q_vv, cv, scv, cv, scv, nvirt, nvirt}};
    for (auto &b : blks) {
        if (!b.out || b.n1 == 0 || b.n2 == 0) continue;
        if ((rc = launch_tc(nat, b.n1, b.n2, first, b.c1, b.s1, b.c2, b.s2, b.out, st, "tc_tile_kernel")))
            return rc;
    }
    return DFTB_OK;
}

int dftb_trans_charges_diag(int norb, int nat, int nocc, int nvirt, const double *co, const double *cv,
                            const double *Sm, const int *opa, double *q_ii, double *q_aa, void *work,
                            size_t work_bytes, void *stream) {
    cudaStream_t st = S(stream);
    double *sco, *scv;
    int *first;
    if (nat > norb) return fail(DFTB_ERR_BAD_SIZE, "trans_charges_diag: nat > norb");
    int rc = trans_charges_common(norb, nat, nocc, nvirt, co, cv, Sm, opa, work, work_bytes, st, &sco, &scv, &first);
    if (rc) return rc;
    if (q_ii && nocc > 0) {
        tc_diag_kernel<<<dim3(cdiv(nocc, 128), nat), 128, 0, st>>>(nocc, first, co, sco, q_ii);
        if ((rc = check_launch("tc_diag_kernel"))) return rc;
    }
    if (q_aa && nvirt > 0) {
        tc_diag_kernel<<<dim3(cdiv(nvirt, 128), nat), 128, 0, st>>>(nvirt, first, cv, scv, q_aa);
        if ((rc = check_launch("tc_diag_kernel"))) return rc;
    }
    return DFTB_OK;
}

size_t dftb_hermitian_rv_workspace_size(int nat, int nvec) {
    if (nat <= 0 || nvec <= 0) return 0;
    return 2 * align256(sizeof(double) * (size_t)nat * nvec);
}

int dftb_hermitian_rv(int nat, int nocc, int nvirt, int nvec, const double *gamma, const double *q_ov,
                      const double *omega, const double *vs, double *us, void *work, size_t work_bytes,
                      void *stream) {
    if (nat <= 0 || nocc <= 0 || nvirt <= 0 || nvec <= 0) return fail(DFTB_ERR_BAD_SIZE, "hermitian_rv: sizes");
    if (!gamma || !q_ov || !omega || !vs || !us) return fail(DFTB_ERR_NULL, "hermitian_rv: null");
    if (!work || work_bytes < dftb_hermitian_rv_workspace_size(nat, nvec))
        return fail(DFTB_ERR_WORKSPACE, "hermitian_rv: workspace too small");
    double *T = (double *)work;
    double *G = (double *)((char *)work + align256(sizeof(double) * (size_t)nat * nvec));
    return coulomb_product(nat, nocc * nvirt, nvec, gamma, q_ov, omega, vs, us, T, G, 1, S(stream));
}

size_t dftb_apbv_workspace_size(int nat, int nocc, int nvirt, int nvec) {
    if (nat <= 0 || nocc <= 0 || nvirt <= 0 || nvec <= 0) return 0;
    const size_t no = nocc, nv = nvirt, m = nvec, na = nat;
    const size_t k1 = na * no * no + na * no * nv * m;
    const size_t k2 = na * no * nv + na * nv * nv * m;
    return align256(sizeof(double) * (k1 > k2 ? k1 : k2)) + dftb_hermitian_rv_workspace_size(nat, nvec);
}

int dftb_apbv(int nat, int nocc, int nvirt, int nvec, int lc, const double *g, const double *g_lr,
              const double *q_oo, const double *q_ov, const double *q_vv, const double *omega, const double *vs,
              double *us, void *work, size_t work_bytes, void *stream) {
    int rc = check_products(nat, nocc, nvirt, nvec, lc, g, g_lr, q_oo, q_ov, q_vv, omega, vs, us, work, work_bytes);
    if (rc) return rc;
    cudaStream_t st = S(stream);
    // workspace: [T | G] for the Coulomb term, then the exchange scratch
    const size_t coul = dftb_hermitian_rv_workspace_size(nat, nvec);
    double *T = (double *)work;
    double *G = (double *)((char *)work + align256(sizeof(double) * (size_t)nat * nvec));
    rc = coulomb_product(nat, nocc * nvirt, nvec, g, q_ov, omega, vs, us, T, G, 0, st);
    if (rc || !lc) return rc;
    return exchange_products(nat, nocc, nvirt, nvec, g_lr, q_oo, q_ov, q_vv, vs, us, -1.0, -1.0,
                             (double *)((char *)work + coul), st);
}

int dftb_ambv(int nat, int nocc, int nvirt, int nvec, int lc, const double *g, const double *g_lr,
              const double *q_oo, const double *q_ov, const double *q_vv, const double *omega, const double *vs,
              double *us, void *work, size_t work_bytes, void *stream) {
    int rc = check_products(nat, nocc, nvirt, nvec, lc, g, g_lr, q_oo, q_ov, q_vv, omega, vs, us, work, work_bytes);
    if (rc) return rc;
    cudaStream_t st = S(stream);
    const long long n = (long long)nocc * nvirt * nvec;
    omega_scale_kernel<<<cdiv(n, 256), 256, 0, st>>>((long long)nocc * nvirt, nvec, omega, vs, us);
    if ((rc = check_launch("omega_scale_kernel"))) return rc;
    if (!lc) return DFTB_OK;
    const size_t coul = dftb_hermitian_rv_workspace_size(nat, nvec);
    return exchange_products(nat, nocc, nvirt, nvec, g_lr, q_oo, q_ov, q_vv, vs, us, -1.0, +1.0,
                             (double *)((char *)work + coul), st);
}

int dftb_davidson_precondition(int nov, int nnew, const double *W, int ldw, const int *src, const int *state,
                               const double *w, const double *omega, double *Q, int ldq, void *stream) {
    if (nov <= 0 || nnew < 0 || ldw <= 0 || ldq < nnew) return fail(DFTB_ERR_BAD_SIZE, "precondition: sizes");
    if (nnew == 0) return DFTB_OK;
    if (!W || !src || !state || !w || !omega || !Q) return fail(DFTB_ERR_NULL, "precondition: null");
    const long long n = (long long)nov * nnew;
    precondition_kernel<<<cdiv(n, 256), 256, 0, S(stream)>>>(nov, nnew, W, ldw, src, state, w, omega, Q, ldq);
    return check_launch("precondition_kernel");
}

int dftb_davidson_residual(int nov, int ncol, const double *AV, int ldav, const double *X, int ldx, const double *lam,
                           double *W, int ldw, double *norms, void *stream) {
    if (nov <= 0 || ncol <= 0 || ldav < ncol || ldx < ncol || ldw < ncol)
        return fail(DFTB_ERR_BAD_SIZE, "residual: sizes");
    if (!AV || !X || !lam || !W || !norms) return fail(DFTB_ERR_NULL, "residual: null");
    cudaStream_t st = S(stream);
    if (cudaMemsetAsync(norms, 0, sizeof(double) * ncol, st) != cudaSuccess)
        return fail(DFTB_ERR_CUDA, "residual: memset");
    int rc;
    if (ncol <= 256) {
        const int R = 256 / ncol;
        unsigned gx = cdiv(nov, R);
        if (gx > 148 * 8) gx = 148 * 8;
        residual_rows_kernel<<<gx, 256, 0, st>>>(nov, ncol, AV, ldav, X, ldx, lam, W, ldw, norms);
        rc = check_launch("residual_rows_kernel");
    } else {
        unsigned gx = cdiv(nov, 256);
        if (gx > 592) gx = 592;
        residual_kernel<<<dim3(gx, ncol), 256, 0, st>>>(nov, ncol, AV, ldav, X, ldx, lam, W, ldw, norms);
        rc = check_launch("residual_kernel");
    }
    if (rc) return rc;
    sqrt_kernel<<<cdiv(ncol, 128), 128, 0, st>>>(ncol, norms);
    return check_launch("sqrt_kernel");
}

int dftb_transpose_f64(int rows, int cols, const double *X, int ldx, double *Y, int ldy, void *stream) {
    if (rows < 0 || cols < 0 || ldx < cols || ldy < rows) return fail(DFTB_ERR_BAD_SIZE, "transpose_f64: sizes");
    if (rows == 0 || cols == 0) return DFTB_OK;
    if (!X || !Y) return fail(DFTB_ERR_NULL, "transpose_f64: null");
    if (cdiv(cols, 32) > 65535) return fail(DFTB_ERR_BAD_SIZE, "transpose_f64: more than 2097120 columns");
    transpose_f64_kernel<<<dim3(cdiv(rows, 32), cdiv(cols, 32)), 256, 0, S(stream)>>>(rows, cols, X, ldx, Y, ldy);
    return check_launch("transpose_f64_kernel");
}

int dftb_exchange_unpack(int m, int nvirt, int nocc, const float *Kall, double *K1, double *K2, void *stream) {
    if (m < 0 || nvirt < 0 || nocc < 0) return fail(DFTB_ERR_BAD_SIZE, "exchange_unpack: sizes");
    if (m == 0 || nvirt == 0 || nocc == 0) return DFTB_OK;
    if (!Kall || !K1 || !K2) return fail(DFTB_ERR_NULL, "exchange_unpack: null");
    if (nvirt > 65535) return fail(DFTB_ERR_BAD_SIZE, "exchange_unpack: more than 65535 virtual orbitals");
    exchange_unpack_kernel<<<dim3(cdiv(nocc, 32), nvirt), 256, 0, S(stream)>>>(m, nvirt, nocc, Kall, K1, K2);
    return check_launch("exchange_unpack_kernel");
}

int dftb_dgemm(int transa, int transb, int m, int n, int k, double alpha, const double *A, int lda, const double *B,
               int ldb, double beta, double *C, int ldc, void *stream) {
    if (m < 0 || n < 0 || k < 0) return fail(DFTB_ERR_BAD_SIZE, "dgemm: sizes");
    if (m == 0 || n == 0) return DFTB_OK;
    if (!A || !B || !C) return fail(DFTB_ERR_NULL, "dgemm: null");
    GemmP p = gemm_defaults();
    p.M = m;
    p.N = n;
    p.K = k;
    p.A = A;
    p.sam = transa ? 1 : lda;
    p.sak = transa ? lda : 1;
    p.B = B;
    p.sbk = transb ? 1 : ldb;
    p.sbn = transb ? ldb : 1;
    p.C = C;
    p.scm = ldc;
    p.scn = 1;
    p.alpha = alpha;
    p.beta = beta;
    return launch_gemm(p, EPI_STORE, 1, S(stream));
}

}  // extern "C"

// ============================================================================
// Allocation-free variant of dftb_trans_charges.
//
// Some callers cannot allocate device memory at the point where they need the
// transition charges: applications that reserve the GPU's memory up front in
// their own pool and forbid any further cudaMalloc, or language bindings that
// only receive device pointers from their host program and have no allocator
// of their own.  dftb_trans_charges wants a caller-provided workspace; this
// variant instead keeps its scratch (S.C for both orbital blocks and the
// per-atom orbital offsets) in a fixed file-scope device array.
//
// The array exists once per GPU that loads this library and stays resident
// until the process exits.  On the host its name is only a stand-in symbol,
// so its device address is looked up with cudaGetSymbolAddress, once per
// device, the first time the entry point runs with that device current (the
// first call should therefore come before any stream capture).  Under lazy
// module loading the array is committed when this module is first used on a
// device, possibly by that first call.  The cached address belongs to the
// device's primary context; it is not looked up again after cudaDeviceReset.
// All calls on one device share the array: calls that can run at the same time on the GPU
// (unordered streams, concurrent host threads) race on it and must be
// serialised by the caller.  Every call rewrites the parts of the scratch it
// reads, so nothing has to be cleared between calls.
// ============================================================================
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;  // 8 MiB per device
static __device__ __align__(256) unsigned char g_tc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
void *g_tc_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_tc_scratch_mutex;

int tc_scratch_address(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        snprintf(g_last_error, sizeof(g_last_error), "trans_charges_noalloc: cudaGetDevice: %s",
                 cudaGetErrorString(e));
        return DFTB_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) return fail(DFTB_ERR_BAD_SIZE, "trans_charges_noalloc: device index");
    std::lock_guard<std::mutex> lock(g_tc_scratch_mutex);
    if (!g_tc_scratch_addr[dev]) {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_tc_scratch);
        if (e != cudaSuccess || !ptr) {
            snprintf(g_last_error, sizeof(g_last_error), "trans_charges_noalloc: cudaGetSymbolAddress: %s",
                     cudaGetErrorString(e));
            return DFTB_ERR_CUDA;
        }
        g_tc_scratch_addr[dev] = ptr;
    }
    *out = g_tc_scratch_addr[dev];
    return DFTB_OK;
}

}  // namespace

extern "C" size_t dftb_trans_charges_noalloc_max_bytes(void) { return kNoAllocScratchBytes; }

extern "C" int dftb_trans_charges_noalloc(int norb, int nat, int nocc, int nvirt, const double *co, const double *cv,
                                          const double *Sm, const int *opa, double *q_oo, double *q_ov,
                                          double *q_vv, void *stream) {
    if (norb <= 0 || nat <= 0 || nocc < 0 || nvirt < 0 || nat > norb)
        return fail(DFTB_ERR_BAD_SIZE, "trans_charges_noalloc: sizes");
    // the atom index is the grid's z extent; refuse before anything is launched
    if (nat > 65535) return fail(DFTB_ERR_BAD_SIZE, "trans_charges_noalloc: nat > 65535");
    const size_t need = dftb_trans_charges_workspace_size(norb, nocc, nvirt);
    if (need > kNoAllocScratchBytes) {
        snprintf(g_last_error, sizeof(g_last_error),
                 "trans_charges_noalloc: needs %zu bytes of scratch, the static array holds %zu "
                 "(use dftb_trans_charges with a workspace)",
                 need, kNoAllocScratchBytes);
        return DFTB_ERR_WORKSPACE;
    }
    void *scratch = nullptr;
    int rc = tc_scratch_address(&scratch);
    if (rc) return rc;
    cudaStream_t st = S(stream);
    double *sco, *scv;
    int *first;
    rc = trans_charges_common(norb, nat, nocc, nvirt, co, cv, Sm, opa, scratch, kNoAllocScratchBytes, st, &sco, &scv,
                              &first, false);
    if (rc) return rc;
    struct Blk {
        double *out;
        const double *c1, *s1, *c2, *s2;
        int n1, n2;
    } blks[3] = {{q_oo, co, sco, co, sco, nocc, nocc},
                 {q_ov, co, sco, cv, scv, nocc, nvirt},
                 {q_vv, cv, scv, cv, scv, nvirt, nvirt}};
    for (auto &b : blks) {
        if (!b.out || b.n1 == 0 || b.n2 == 0) continue;
        if ((rc = launch_tc(nat, b.n1, b.n2, first, b.c1, b.s1, b.c2, b.s2, b.out, st, "tc_tile_kernel (noalloc)")))
            return rc;
    }
    return DFTB_OK;
}
