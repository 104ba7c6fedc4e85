// FP64 matrix products emulated exactly on the int8 tensor cores of B200 (tcgen05 kind::i8), after the
// "Ozaki scheme II" of Ozaki, Uchino and Imamura (integer modular GEMMs plus the Chinese remainder theorem):
//
//   C = alpha * op(A) op(B) + beta * C            (row-major FP64; op = transpose when trans != 0)
//
// 1. Row m of op(A) is scaled by 2^sa[m] and column n of op(B) by 2^sb[n] and rounded to integers A', B'
//    of at most `bits` bits, chosen so that every entry of A'B' (K terms) stays below P/2 in magnitude,
//    P = p_1 ... p_N the product of N pairwise coprime moduli p_i <= 256.
// 2. For each modulus the symmetric residues A' mod p_i and B' mod p_i (|r| <= 128, int8) are multiplied on
//    the tensor cores with exact int32 accumulation (K < 2^17), and the epilogue keeps the product's residue
//    mod p_i as int8.
// 3. Per element, Garner's algorithm turns the N residues into mixed-radix digits (int32 arithmetic), whose
//    Horner sum in FP64 is A'B' to within FP64 rounding, and C = 2^-(sa[m] + sb[n]) A'B'.
//
// The only approximation is step 1: each entry of op(A) (op(B)) is carried with `bits` bits relative to
// the largest entry of its row (column); with N = 16 moduli and K <= 2^17 that is the full 53-bit FP64
// mantissa.  The tensor-core work is N int8 GEMMs (B200: 4.5 dense int8 POPS against ~35 TFLOP/s of FP64
// DGEMM).
//
// Kernels: ozaki_rowscale_kernel (exponents), ozaki_residue_kernel (int8 residue planes, K-major,
// zero-padded), ozaki_mma_kernel (persistent tcgen05 GEMM over (M tile, N tile, modulus), TMA operand ring,
// double-buffered TMEM accumulators, residue epilogue), ozaki_crt_kernel (Garner + Horner + scaling).

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "dftbaby_b200.h"
#include "tcgen05.cuh"

namespace ozk {

using namespace tc5;

constexpr int MAXMOD = 16;
// pairwise coprime: 2^8, 3*5*17, 11*23, 13*19 and primes
constexpr int kModuli[MAXMOD] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 211, 199, 197, 193, 191};
constexpr int KMAX = 131071;                // 128 * 128 * K < 2^31: exact int32 accumulation
constexpr int SCALE_NONFINITE = -(1 << 20);  // row/column exponent marking an Inf or NaN entry

struct Tables {
    int p[MAXMOD];
    double invp[MAXMOD];
    int D[MAXMOD][MAXMOD];  // D[j][i] = (p_0 ... p_{i-1}) mod p_j, i < j
    int Binv[MAXMOD];       // (p_0 ... p_{j-1})^-1 mod p_j
    uint32_t mb[MAXMOD];    // Barrett multiplier floor(2^32 / p) + 1
    int bias[MAXMOD];       // p 2^20, a multiple of p above 2^27
    double q3[MAXMOD / 3 + 1];  // p_3k p_3k+1 p_3k+2, the radix of digit triple k
    int c18[MAXMOD], c36[MAXMOD];  // 2^18 and 2^36 modulo p
};

// symmetric residue of t (|t| < 2^27) modulo p without float conversions: u = t + p 2^20 is in
// [0, 2^29), floor(u mb / 2^32) is floor(u / p) or one more (the multiplier's excess over 2^32 / p is
// below 1, so u mb / 2^32 exceeds u / p by less than 1/8), and the remainder is corrected once.
__device__ __forceinline__ int symmod_b(int t, int p, uint32_t mb, int bias) {
    const uint32_t u = (uint32_t)(t + bias);
    const uint32_t q = __umulhi(u, mb);
    int r = (int)(u - q * (uint32_t)p);
    if (r < 0) r += p;
    if (r > ((p - 1) >> 1)) r -= p;
    return r;
}

// ---------------------------------------------------------------------------- scaling and residues

// Y(r, k) = trans ? X[k * ldx + r] : X[r * ldx + k]; s[r] = bits - 1 - ilogb(max_k |Y(r, k)|) so that
// |Y(r, k)| 2^s[r] < 2^bits (0 for a zero row, SCALE_NONFINITE for a row holding Inf or NaN); rows in
// [rows, rpad) get 0.
__global__ void ozaki_rowscale_kernel(int rows, int rpad, int K, const double *X, long long ldx, int trans, int bits,
                                      int *s) {
    if (!trans) {
        const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
        if (warp >= rpad) return;
        double m = 0.0;
        bool bad = false;
        if (warp < rows) {
            const double *x = X + (long long)warp * ldx;
            int k = lane;
            for (; k + 96 < K; k += 128) {
                // four independent loads in flight per lane
                const double a0 = fabs(x[k]), a1 = fabs(x[k + 32]), a2 = fabs(x[k + 64]), a3 = fabs(x[k + 96]);
                bad |= !(a0 <= 1.7976931348623157e308 && a1 <= 1.7976931348623157e308 &&
                         a2 <= 1.7976931348623157e308 && a3 <= 1.7976931348623157e308);
                m = fmax(fmax(m, fmax(a0, a1)), fmax(a2, a3));
            }
            for (; k < K; k += 32) {
                const double a = fabs(x[k]);
                bad |= !(a <= 1.7976931348623157e308);
                m = fmax(m, a);
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
            bad |= __shfl_xor_sync(0xffffffffu, (int)bad, o) != 0;
        }
        if (lane == 0) s[warp] = bad ? SCALE_NONFINITE : (m > 0.0 ? bits - 1 - ilogb(m) : 0);
    } else {
        // 32 rows per block (threadIdx.x, consecutive in memory), 32 phases of k (threadIdx.y)
        __shared__ double sm[32][32];
        __shared__ int sbad[32][32];
        const int r = blockIdx.x * 32 + threadIdx.x;
        double m = 0.0;
        int bad = 0;
        if (r < rows) {
            for (int k = threadIdx.y; k < K; k += 32) {
                const double a = fabs(X[(long long)k * ldx + r]);
                bad |= !(a <= 1.7976931348623157e308);
                m = fmax(m, a);
            }
        }
        sm[threadIdx.y][threadIdx.x] = m;
        sbad[threadIdx.y][threadIdx.x] = bad;
        __syncthreads();
        if (threadIdx.y == 0 && r < rpad) {
            for (int y = 1; y < 32; ++y) {
                m = fmax(m, sm[y][threadIdx.x]);
                bad |= sbad[y][threadIdx.x];
            }
            s[r] = bad ? SCALE_NONFINITE : (m > 0.0 ? bits - 1 - ilogb(m) : 0);
        }
    }
}

constexpr int RT_ROWS = 32, RT_K = 128;

// Residue planes R[i][r][k] (i < nmod, r < rows_write, k < kpad; zero outside rows x K) of the scaled,
// rounded Y(r, k) 2^s[r].  One block per 32 x 128 tile of Y, staged through shared memory so that both the
// FP64 reads (along k, or along r when transposed) and the int8 writes (4 consecutive k per thread) coalesce.
template <int NM>
__global__ void __launch_bounds__(256) ozaki_residue_kernel(int rows, int rows_write, int K, const double *X,
                                                            long long ldx, int trans, const int *s,
                                                            const __grid_constant__ Tables tb, int8_t *R,
                                                            long long plane, int kpad) {
    __shared__ double tile[RT_ROWS][RT_K + 1];
    const int r0 = blockIdx.y * RT_ROWS, k0 = blockIdx.x * RT_K;
    for (int idx = threadIdx.x; idx < RT_ROWS * RT_K; idx += blockDim.x) {
        int rr, kk;
        if (trans) {
            rr = idx % RT_ROWS;
            kk = idx / RT_ROWS;
        } else {
            rr = idx / RT_K;
            kk = idx % RT_K;
        }
        const int r = r0 + rr, k = k0 + kk;
        double v = 0.0;
        if (r < rows && k < K) v = trans ? X[(long long)k * ldx + r] : X[(long long)r * ldx + k];
        tile[rr][kk] = v;
    }
    __syncthreads();
    for (int item = threadIdx.x; item < RT_ROWS * (RT_K / 4); item += blockDim.x) {
        const int rr = item / (RT_K / 4), kq = (item % (RT_K / 4)) * 4;
        const int r = r0 + rr, k = k0 + kq;
        if (k >= kpad || r >= rows_write) continue;
        const int sr = (r < rows) ? s[r] : 0;
        // the scaled, rounded entries (at most 53 bits) as h 2^36 + m 2^18 + l, |h| <= 2^17, 0 <= m, l < 2^18
        int h[4], md[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const long long ai =
                (sr == SCALE_NONFINITE || r >= rows) ? 0ll : __double2ll_rn(ldexp(tile[rr][kq + e], sr));
            h[e] = (int)(ai >> 36);
            md[e] = (int)((ai >> 18) & 0x3FFFF);
            l[e] = (int)(ai & 0x3FFFF);
        }
#pragma unroll
        for (int i = 0; i < NM; ++i) {
            uint32_t w = 0;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                // |h c36 + m c18 + l| < 2^25 + 2^26 + 2^18 < 2^27
                const int t = h[e] * tb.c36[i] + md[e] * tb.c18[i] + l[e];
                const int rd = symmod_b(t, tb.p[i], tb.mb[i], tb.bias[i]);
                w |= ((uint32_t)(uint8_t)(int8_t)rd) << (8 * e);
            }
            *reinterpret_cast<uint32_t *>(R + i * plane + (long long)r * kpad + k) = w;
        }
    }
}

// ---------------------------------------------------------------------------- int8 tensor-core GEMM

// 128 x 256 output tiles: per 128-byte K block a stage holds 16 KiB of A and 32 KiB of B for four
// 128 x 256 x 32 MMAs, a third fewer operand bytes per MMA than 128 x 128 tiles
constexpr int BM = 128, BN = 256, BKB = 128;  // tile rows, tile columns, K bytes (= int8 elements) per stage
constexpr int TILE_BYTES = BM * BKB;          // 16 KiB (A)
constexpr int TILE_B_BYTES = BN * BKB;        // 32 KiB (B)
constexpr int STAGES = 4;
constexpr int STAGE_BYTES = TILE_BYTES + TILE_B_BYTES;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /* alignment slack */ + 256 /* barriers */;
constexpr int EPI_THREADS = 128;
// instruction descriptor: D = S32 (bits 4-5 = 2), A = B = signed int8 (bits 7-9, 10-12 = 1), both K-major,
// N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t kIdescI8 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                              ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void umma_i8(uint32_t tmem_c, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_c),
        "l"(da), "l"(db), "r"(kIdescI8), "r"(accumulate));
}

struct Maps {
    CUtensorMap a;  // residue planes of the A operand: nmod * arows rows x kpad int8
    CUtensorMap b;  // residue planes of the B operand: nmod * brows rows x kpad int8
};

struct MmaParams {
    int M, N, kpad, nmod;
    int arows, brows;  // rows per residue plane of the A and B operands (multiples of 256)
    int8_t *RC;  // product residues: plane i at RC + i * planeC, row-major with ldr (multiple of 32)
    long long planeC;
    int ldr;
    int *err;
};

// Persistent kernel, one CTA per SM over the tiles t = (m tile, n tile, modulus), M fastest:
//   warp 0 lane 0 : TMA producer over a 4-stage ring of 128-byte-wide A (128 rows) and B (256 rows) tiles
//                   (128-byte swizzle);
//   warp 1 lane 0 : tcgen05.mma kind::i8 issuer (M = 128, N = 256, K = 32 per instruction) into one of two
//                   256-column int32 TMEM accumulators (tile j uses accumulator j % 2);
//   warps 2..5    : epilogue of tile j under the MMAs of tile j + 1: int32 -> residue mod p -> int8.
// Every wait is bounded; on timeout the kernel records an error code, stops issuing, drains its copies
// and releases TMEM.
__global__ void __launch_bounds__(192, 1) ozaki_mma_kernel(const __grid_constant__ Maps maps, const MmaParams p,
                                                           const __grid_constant__ Tables tb) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *tfull = empty + STAGES;
    uint64_t *tempty = tfull + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tempty + 2);
    int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int mt = (p.M + BM - 1) / BM, nt = (p.N + BN - 1) / BN;
    const int ntiles = mt * nt * p.nmod;
    const int kblocks = p.kpad / BKB;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&tfull[a], 1);
            mbar_init(&tempty[a], EPI_THREADS);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(2 * BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer
            int it = 0;
            bool stop = false;
            for (int t = blockIdx.x; t < ntiles && !stop; t += gridDim.x) {
                const int mi = t % mt, ni = (t / mt) % nt, mod = t / (mt * nt);
                const int ya = mod * p.arows + mi * BM, yb = mod * p.brows + ni * BN;
                for (int kb = 0; kb < kblocks; ++kb) {
                    const int s = it % STAGES;
                    if (it >= STAGES && !mbar_wait(&empty[s], ((it / STAGES) - 1) & 1)) {
                        atomicExch(p.err, 1);
                        *(volatile int *)abort_flag = 1;
                        stop = true;
                        break;
                    }
                    if (*(volatile int *)abort_flag) {
                        stop = true;
                        break;
                    }
                    uint8_t *sa = smem + s * STAGE_BYTES;
                    mbar_expect_tx(&full[s], STAGE_BYTES);
                    tma_load_2d(sa, &maps.a, &full[s], kb * BKB, ya);
                    tma_load_2d(sa + TILE_BYTES, &maps.b, &full[s], kb * BKB, yb);
                    ++it;
                }
            }
            // drain: wait (bounded) until every copy that was started has landed
            for (int j = max(0, it - STAGES); j < it; ++j) mbar_wait(&full[j % STAGES], (j / STAGES) & 1);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---------------- MMA issuer
            int it = 0, j = 0;
            bool stop = false;
            for (int t = blockIdx.x; t < ntiles && !stop; t += gridDim.x, ++j) {
                const int acc = j & 1;
                const uint32_t tacc = tmem + (uint32_t)(acc * BN);
                if (j >= 2 && !mbar_wait(&tempty[acc], ((j >> 1) - 1) & 1)) {
                    atomicExch(p.err, 4);
                    *(volatile int *)abort_flag = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                for (int kb = 0; kb < kblocks; ++kb) {
                    const int s = it % STAGES;
                    if (!mbar_wait(&full[s], (it / STAGES) & 1)) {
                        atomicExch(p.err, 2);
                        *(volatile int *)abort_flag = 1;
                        stop = true;
                        break;
                    }
                    if (*(volatile int *)abort_flag) {
                        stop = true;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sa = smem_u32(smem + s * STAGE_BYTES), sb = sa + TILE_BYTES;
#pragma unroll
                    for (int k = 0; k < BKB / 32; ++k) {
                        // 32 int8 = 32 bytes along K per instruction, inside the 128-byte swizzle atom
                        umma_i8(tacc, smem_desc_k128(sa + k * 32), smem_desc_k128(sb + k * 32),
                                (kb > 0 || k > 0) ? 1u : 0u);
                    }
                    umma_commit(&empty[s]);
                    ++it;
                }
                umma_commit(&tfull[acc]);
            }
        }
    } else {
        // ---------------- epilogue (warps 2..5): TMEM lanes 32 (warp % 4) .. + 31 are this warp's rows
        const int rq = warp & 3;
        const int rloc = rq * 32 + lane;
        int j = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++j) {
            const int mi = t % mt, ni = (t / mt) % nt, mod = t / (mt * nt);
            const int acc = j & 1;
            const int row = mi * BM + rloc, n0 = ni * BN;
            const int pm = tb.p[mod];
            const double invpd = tb.invp[mod];
            const bool ok = __all_sync(0xffffffffu, mbar_wait(&tfull[acc], (j >> 1) & 1) ? 1 : 0) != 0;
            if (!ok && lane == 0) atomicExch(p.err, 3);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const bool live = ok && !*(volatile int *)abort_flag && kblocks > 0;  // warp-uniform
            for (int c0 = 0; c0 < BN; c0 += 32) {
                uint32_t v[32];
                tmem_ld32_raw(tmem + ((uint32_t)(rq * 32) << 16) + (uint32_t)(acc * BN + c0), v);
                const int col0 = n0 + c0;
                if (live && row < p.M && col0 < p.N) {
                    uint32_t w[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        uint32_t word = 0;
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            // |a| < 2^31 is exact in FP64, so q is round(a / p) or one off near a tie
                            const int a = (int)v[4 * q + e];
                            const long long qq = (long long)rint((double)a * invpd);
                            int r = (int)((long long)a - qq * pm);
                            if (r > ((pm - 1) >> 1)) r -= pm;
                            if (r < -(pm >> 1)) r += pm;
                            word |= ((uint32_t)(uint8_t)(int8_t)r) << (8 * e);
                        }
                        w[q] = word;
                    }
                    uint4 *dst = reinterpret_cast<uint4 *>(p.RC + mod * p.planeC + (long long)row * p.ldr + col0);
                    dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
                    dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            mbar_arrive(&tempty[acc]);
            if (!ok) break;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN));
    }
}

// ---------------------------------------------------------------------------- reconstruction

// C[m][n] = alpha G[m][n] 2^-(sa[m] + sb[n]) X + beta C[m][n] (G optional), X the integer with residues RC[i][m][n] (Garner's
// mixed-radix digits v_j, symmetric, X = v_0 + p_0 (v_1 + p_1 (v_2 + ...)) evaluated in FP64).  Four
// consecutive columns per thread (one 32-bit word per residue plane); NM moduli.
template <int NM>
__global__ void __launch_bounds__(256) ozaki_crt_kernel(int M, int N, const int8_t *RC, long long planeC, int ldr,
                                                        const int *sa, const int *sb, double alpha, const double *G,
                                                        long long ldg, double beta, double *C, long long ldc,
                                                        const __grid_constant__ Tables tb) {
    const int nq = (N + 3) / 4;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)M * nq) return;
    const int m = (int)(idx / nq), n0 = (int)(idx % nq) * 4;
    uint32_t wd[NM];
#pragma unroll
    for (int i = 0; i < NM; ++i)
        wd[i] = *reinterpret_cast<const uint32_t *>(RC + i * planeC + (long long)m * ldr + n0);
    const int sm = sa[m];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int n = n0 + e;
        if (n >= N) break;
        int v[NM];
        v[0] = (int)(int8_t)(uint8_t)(wd[0] >> (8 * e));
#pragma unroll
        for (int jj = 1; jj < NM; ++jj) {
            // |r - sum_i v_i D| <= 128 + 15 * 128 * 255 < 2^19 and Binv <= 255: the product stays below 2^27
            int acc = (int)(int8_t)(uint8_t)(wd[jj] >> (8 * e));
#pragma unroll
            for (int i = 0; i < jj; ++i) acc -= v[i] * tb.D[jj][i];
            v[jj] = symmod_b(acc * tb.Binv[jj], tb.p[jj], tb.mb[jj], tb.bias[jj]);
        }
        // Horner over digit triples: each triple v_a + p_a (v_b + p_b v_c) is an exact int32 (< 2^24)
        constexpr int NG = (NM + 2) / 3;
        double x = 0.0;
#pragma unroll
        for (int g = NG - 1; g >= 0; --g) {
            const int a = 3 * g;
            int t = v[a];
            if (a + 2 < NM)
                t += tb.p[a] * (v[a + 1] + tb.p[a + 1] * v[a + 2]);
            else if (a + 1 < NM)
                t += tb.p[a] * v[a + 1];
            x = (g == NG - 1) ? (double)t : fma(x, tb.q3[g], (double)t);
        }
        const int sn = sb[n];
        double out;
        if (sm == SCALE_NONFINITE || sn == SCALE_NONFINITE)
            out = __longlong_as_double(0x7ff8000000000000ll);  // NaN
        else
            out = alpha * ldexp(x, -(sm + sn));
        if (G) out *= G[(long long)m * ldg + n];
        double *c = C + (long long)m * ldc + n;
        *c = beta == 0.0 ? out : out + beta * *c;
    }
}

template <int NM>
void launch_crt(int M, int N, const int8_t *RC, long long planeC, int ldr, const int *sa, const int *sb, double alpha,
                const double *G, long long ldg, double beta, double *C, long long ldc, const Tables &tb,
                cudaStream_t st) {
    const long long nthreads = (long long)M * ((N + 3) / 4);
    ozaki_crt_kernel<NM><<<(unsigned)((nthreads + 255) / 256), 256, 0, st>>>(M, N, RC, planeC, ldr, sa, sb, alpha,
                                                                             G, ldg, beta, C, ldc, tb);
}

// ---------------------------------------------------------------------------- host side
thread_local char g_err[256] = "";
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::mutex g_mutex;
Tables g_tables;
bool g_tables_ready = false;

int init_host() {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_encode) {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            snprintf(g_err, sizeof(g_err), "cuTensorMapEncodeTiled unavailable");
            return -1;
        }
        g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    if (!g_tables_ready) {
        Tables &t = g_tables;
        for (int i = 0; i < MAXMOD; ++i) {
            t.p[i] = kModuli[i];
            t.invp[i] = 1.0 / (double)kModuli[i];
        }
        for (int j = 0; j < MAXMOD; ++j) {
            const int pj = kModuli[j];
            long long prod = 1;  // p_0 ... p_{i-1} mod p_j
            for (int i = 0; i < MAXMOD; ++i) {
                t.D[j][i] = (i < j) ? (int)prod : 0;
                if (i < j) prod = (prod * kModuli[i]) % pj;
            }
            // prod = p_0 ... p_{j-1} mod p_j; its inverse by search (p_j <= 256)
            int inv = 0;
            for (int x = 1; x < pj && j > 0; ++x)
                if ((prod * x) % pj == 1) {
                    inv = x;
                    break;
                }
            t.Binv[j] = (j == 0) ? 1 : inv;
            t.mb[j] = (uint32_t)((1ull << 32) / (unsigned long long)pj + 1ull);
            t.bias[j] = pj << 20;
            t.c18[j] = (int)((1ull << 18) % (unsigned long long)pj);
            t.c36[j] = (int)((1ull << 36) % (unsigned long long)pj);
        }
        for (int g = 0; 3 * g < MAXMOD; ++g) {
            double q = 1.0;
            for (int i = 3 * g; i < 3 * g + 3 && i < MAXMOD; ++i) q *= (double)kModuli[i];
            t.q3[g] = q;
        }
        g_tables_ready = true;
    }
    return 0;
}

int make_map_i8(CUtensorMap *map, const void *base, long long rows, int kpad, int box_rows) {
    cuuint64_t dims[2] = {(cuuint64_t)kpad, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)kpad};
    cuuint32_t box[2] = {(cuuint32_t)BKB, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        snprintf(g_err, sizeof(g_err), "cuTensorMapEncodeTiled (int8) failed (%d): rows %lld kpad %d", (int)r, rows,
                 kpad);
        return -1;
    }
    return 0;
}

inline long long up(long long x, long long q) { return (x + q - 1) / q * q; }

// An operand in residue form: rows_total rows (padded to 256) of a K-major matrix, k columns (padded to 128):
//   int32 exponent per row | nmod int8 residue planes of rpad x kpad
struct OperandLayout {
    long long rpad, kpad, plane;
    size_t off_res, total;
};

OperandLayout operand_layout(int rows_total, int k, int nmod) {
    OperandLayout L;
    L.rpad = up(rows_total, 256);
    L.kpad = up(k, BKB);
    L.plane = L.rpad * L.kpad;
    L.off_res = (size_t)up(4 * L.rpad, 256);
    L.total = L.off_res + (size_t)nmod * L.plane;
    return L;
}

// product residues: nmod planes of m x ldr int8
inline long long product_ldr(int n) { return up(n, 32); }
inline size_t product_bytes(int m, int n, int nmod) { return (size_t)up((long long)nmod * m * product_ldr(n), 256); }

// largest bit count b with K 2^(2b) < P/2 (P the product of the first nmod moduli), at most 53
int scale_bits(int k, int nmod) {
    double log2P = 0.0;
    for (int i = 0; i < nmod; ++i) log2P += log2((double)kModuli[i]);
    const int b = (int)floor((log2P - 1.0 - log2((double)k) - 1e-6) / 2.0);
    return b < 53 ? b : 53;
}

int check_shape(int k, int nmod) {
    if (k <= 0 || k > KMAX || nmod < 8 || nmod > MAXMOD) {
        snprintf(g_err, sizeof(g_err), "ozaki: 0 < k <= %d and 8 <= nmod <= %d required", KMAX, MAXMOD);
        return DFTB_ERR_BAD_SIZE;
    }
    if (scale_bits(k, nmod) < 16) {
        snprintf(g_err, sizeof(g_err), "ozaki: %d moduli leave too few bits at k = %d", nmod, k);
        return DFTB_ERR_BAD_SIZE;
    }
    return DFTB_OK;
}

// rows [row0, row0 + rows) of the operand from Y(r, k) = trans ? X[k][r] : X[r][k]; when they are the last
// rows (row0 + rows == rows_total) the padding rows up to 256 are written as zeros too
int prepare(int trans, int rows, int k, const double *X, long long ldx, int nmod, uint8_t *op, int rows_total,
            int row0, cudaStream_t st) {
    const OperandLayout L = operand_layout(rows_total, k, nmod);
    const int bits = scale_bits(k, nmod);
    const int rows_write = (row0 + rows == rows_total) ? (int)(L.rpad - row0) : rows;
    int *s = reinterpret_cast<int *>(op) + row0;
    int8_t *R = reinterpret_cast<int8_t *>(op + L.off_res) + (long long)row0 * L.kpad;
    if (!trans) {
        const long long threads = (long long)rows_write * 32;
        ozaki_rowscale_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(rows, rows_write, k, X, ldx, 0, bits,
                                                                                 s);
    } else {
        ozaki_rowscale_kernel<<<(unsigned)((rows_write + 31) / 32), dim3(32, 32), 0, st>>>(rows, rows_write, k, X, ldx,
                                                                                         1, bits, s);
    }
    dim3 g((unsigned)(L.kpad / RT_K), (unsigned)((rows_write + RT_ROWS - 1) / RT_ROWS));
    switch (nmod) {
#define OZK_RES(NMV)                                                                                            \
    case NMV:                                                                                                   \
        ozaki_residue_kernel<NMV><<<g, 256, 0, st>>>(rows, rows_write, k, X, ldx, trans, s, g_tables, R, L.plane, \
                                                     (int)L.kpad);                                              \
        break;
        OZK_RES(8)
        OZK_RES(9)
        OZK_RES(10)
        OZK_RES(11)
        OZK_RES(12)
        OZK_RES(13)
        OZK_RES(14)
        OZK_RES(15)
        OZK_RES(16)
#undef OZK_RES
    }
    return cudaGetLastError() == cudaSuccess ? DFTB_OK : DFTB_ERR_CUDA;
}

int product(int m, int n, int k, int nmod, const uint8_t *A, int rows_a, const uint8_t *B, int rows_b, double alpha,
            const double *G, long long ldg, double beta, double *C, long long ldc, int8_t *RC, int *err,
            cudaStream_t st) {
    const OperandLayout LA = operand_layout(rows_a, k, nmod), LB = operand_layout(rows_b, k, nmod);
    Maps maps;
    memset(&maps, 0, sizeof(maps));
    if (make_map_i8(&maps.a, A + LA.off_res, (long long)nmod * LA.rpad, (int)LA.kpad, BM) ||
        make_map_i8(&maps.b, B + LB.off_res, (long long)nmod * LB.rpad, (int)LB.kpad, BN))
        return DFTB_ERR_CUDA;
    MmaParams p;
    p.M = m;
    p.N = n;
    p.kpad = (int)LA.kpad;
    p.nmod = nmod;
    p.arows = (int)LA.rpad;
    p.brows = (int)LB.rpad;
    p.RC = RC;
    p.ldr = (int)product_ldr(n);
    p.planeC = (long long)m * p.ldr;
    p.err = err;
    static bool attr_set[64] = {false};
    static int sm_count[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
        if (cudaFuncSetAttribute(ozaki_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES) !=
            cudaSuccess) {
            snprintf(g_err, sizeof(g_err), "ozaki: cannot reserve %d bytes of shared memory", SMEM_BYTES);
            return DFTB_ERR_CUDA;
        }
        int nsm = 0;
        if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm <= 0) nsm = 148;
        sm_count[dev] = nsm;
        attr_set[dev] = true;
    }
    const int sms = (dev >= 0 && dev < 64) ? sm_count[dev] : 148;
    const long long ntiles = (long long)((m + BM - 1) / BM) * ((n + BN - 1) / BN) * nmod;
    if (ntiles > (1LL << 30)) return DFTB_ERR_BAD_SIZE;
    ozaki_mma_kernel<<<(unsigned)(ntiles < sms ? ntiles : sms), 192, SMEM_BYTES, st>>>(maps, p, g_tables);
    const int *sa = reinterpret_cast<const int *>(A), *sb = reinterpret_cast<const int *>(B);
    switch (nmod) {
#define OZK_CRT(NMV)                                                                                              \
    case NMV:                                                                                                     \
        launch_crt<NMV>(m, n, RC, p.planeC, p.ldr, sa, sb, alpha, G, ldg, beta, C, ldc, g_tables, st); \
        break;
        OZK_CRT(8)
        OZK_CRT(9)
        OZK_CRT(10)
        OZK_CRT(11)
        OZK_CRT(12)
        OZK_CRT(13)
        OZK_CRT(14)
        OZK_CRT(15)
        OZK_CRT(16)
#undef OZK_CRT
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(g_err, sizeof(g_err), "ozaki: %s", cudaGetErrorString(e));
        return DFTB_ERR_CUDA;
    }
    return DFTB_OK;
}

}  // namespace ozk

extern "C" {

const char *dftb_ozaki_last_error(void) { return ozk::g_err; }

size_t dftb_ozaki_operand_size(int rows, int k, int nmod) {
    if (rows <= 0 || ozk::check_shape(k, nmod) != DFTB_OK) return 0;
    return ozk::operand_layout(rows, k, nmod).total;
}

int dftb_ozaki_prepare(int trans, int rows, int k, const double *X, int ldx, int nmod, void *operand, int rows_total,
                       int row0, void *stream) {
    using namespace ozk;
    if (int rc = check_shape(k, nmod)) return rc;
    if (rows <= 0 || row0 < 0 || row0 + rows > rows_total || ldx < (trans ? rows : k)) {
        snprintf(g_err, sizeof(g_err), "ozaki_prepare: rows %d at %d of %d, ldx %d", rows, row0, rows_total, ldx);
        return DFTB_ERR_BAD_SIZE;
    }
    if (!X || !operand) return DFTB_ERR_NULL;
    if (reinterpret_cast<uintptr_t>(operand) & 255) {
        snprintf(g_err, sizeof(g_err), "ozaki_prepare: the operand must be 256-byte aligned");
        return DFTB_ERR_BAD_SIZE;
    }
    if (init_host()) return DFTB_ERR_CUDA;
    return prepare(trans, rows, k, X, ldx, nmod, reinterpret_cast<uint8_t *>(operand), rows_total, row0,
                   reinterpret_cast<cudaStream_t>(stream));
}

size_t dftb_ozaki_product_workspace_size(int m, int n, int nmod) {
    if (m <= 0 || n <= 0 || nmod < 1 || nmod > ozk::MAXMOD) return 0;
    return ozk::product_bytes(m, n, nmod);
}

int dftb_ozaki_product(int m, int n, int k, int nmod, const void *A, int rows_a, const void *B, int rows_b,
                       double alpha, const double *G, int ldg, double beta, double *C, int ldc, void *work,
                       size_t work_bytes, int *err, void *stream) {
    using namespace ozk;
    if (int rc = check_shape(k, nmod)) return rc;
    if (m <= 0 || n <= 0 || m > rows_a || n > rows_b || ldc < n || (G && ldg < n)) {
        snprintf(g_err, sizeof(g_err), "ozaki_product: m %d of %d rows, n %d of %d rows, ldc %d", m, rows_a, n, rows_b,
                 ldc);
        return DFTB_ERR_BAD_SIZE;
    }
    if (!A || !B || !C || !work || !err) return DFTB_ERR_NULL;
    if (work_bytes < product_bytes(m, n, nmod) || ((reinterpret_cast<uintptr_t>(work) |
                                                    reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) &
                                                   255)) {
        snprintf(g_err, sizeof(g_err), "ozaki_product: workspace of %zu bytes and 256-byte aligned operands needed",
                 product_bytes(m, n, nmod));
        return DFTB_ERR_WORKSPACE;
    }
    if (init_host()) return DFTB_ERR_CUDA;
    return product(m, n, k, nmod, reinterpret_cast<const uint8_t *>(A), rows_a, reinterpret_cast<const uint8_t *>(B),
                   rows_b, alpha, G, ldg, beta, C, ldc, reinterpret_cast<int8_t *>(work), err,
                   reinterpret_cast<cudaStream_t>(stream));
}

size_t dftb_ozaki_workspace_size(int m, int n, int k, int nmod) {
    if (m <= 0 || n <= 0 || ozk::check_shape(k, nmod) != DFTB_OK) return 0;
    return ozk::operand_layout(m, k, nmod).total + ozk::operand_layout(n, k, nmod).total +
           ozk::product_bytes(m, n, nmod);
}

int dftb_ozaki_dgemm(int transa, int transb, int m, int n, int k, double alpha, const double *A, int lda,
                     const double *B, int ldb, double beta, double *C, int ldc, int nmod, void *work,
                     size_t work_bytes, int *err, void *stream) {
    using namespace ozk;
    if (int rc = check_shape(k, nmod)) return rc;
    if (m <= 0 || n <= 0) return DFTB_ERR_BAD_SIZE;
    if (!A || !B || !C || !work || !err) return DFTB_ERR_NULL;
    if (lda < (transa ? m : k) || ldb < (transb ? k : n) || ldc < n) {
        snprintf(g_err, sizeof(g_err), "ozaki_dgemm: leading dimension too small");
        return DFTB_ERR_BAD_SIZE;
    }
    const size_t need = dftb_ozaki_workspace_size(m, n, k, nmod);
    if (work_bytes < need || (reinterpret_cast<uintptr_t>(work) & 255)) {
        snprintf(g_err, sizeof(g_err), "ozaki_dgemm: workspace of %zu bytes (256-byte aligned) needed", need);
        return DFTB_ERR_WORKSPACE;
    }
    if (init_host()) return DFTB_ERR_CUDA;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    uint8_t *w = reinterpret_cast<uint8_t *>(work);
    uint8_t *opA = w, *opB = w + operand_layout(m, k, nmod).total;
    int8_t *RC = reinterpret_cast<int8_t *>(opB + operand_layout(n, k, nmod).total);
    // op(A)(r, k) = transa ? A[k][r] : A[r][k];  op(B)^T(r, k) = op(B)(k, r) = transb ? B[r][k] : B[k][r]
    int rc = prepare(transa ? 1 : 0, m, k, A, lda, nmod, opA, m, 0, st);
    if (rc == DFTB_OK) rc = prepare(transb ? 0 : 1, n, k, B, ldb, nmod, opB, n, 0, st);
    if (rc == DFTB_OK) rc = product(m, n, k, nmod, opA, m, opB, n, alpha, nullptr, 0, beta, C, ldc, RC, err, st);
    return rc;
}

}  // extern "C"
