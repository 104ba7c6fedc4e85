// Split-precision BF16 GEMM on the 5th-generation tensor cores (tcgen05) of B200.
//
//   C(m, n) = alpha * sum_s sum_k A_s(m, k) B_s(n, k)          (FP32 accumulation in TMEM)
//
// with up to three (A_s, B_s) operand pairs ("segments") that share M, N, K.
// Splitting an FP32 operand X into BF16 parts X = X_hi + X_lo and summing the
// segments (A_hi,B_hi), (A_hi,B_lo), (A_lo,B_hi) reproduces the FP32 product to
// ~2^-16 relative error at three BF16 tensor-core passes.
//
// Operands are K-major row-major BF16 matrices (A: M x K, B: N x K, leading
// dimensions multiples of 8 elements, 16-byte aligned base).  The epilogue can
//   * multiply elementwise by an FP32 matrix G (the AO-expanded gamma^lr),
//   * store FP32 C,
//   * store the result as a BF16 hi/lo pair, row-major and/or transposed
//     (the transposed store is coalesced across a warp).
//
// Structure per CTA (128 threads, one 128x128 output tile):
//   warp 0 lane 0 : TMA producer, 4-stage ring of 128x64 A and B tiles
//                   (128-byte swizzle), mbarrier::complete_tx completion;
//   warp 1 lane 0 : issues tcgen05.mma (M=128, N=128, K=16 per instruction)
//                   into a 128-column TMEM accumulator; tcgen05.commit frees
//                   ring slots and finally signals the epilogue;
//   warps 0..3    : epilogue, tcgen05.ld 32x32b of their 32 TMEM lanes.
// Every mbarrier wait is bounded; on timeout the kernel records an error
// code, stops issuing work, drains the copies it started and releases TMEM.

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "dftbaby_b200.h"
#include "tcgen05.cuh"

namespace tcg {

using namespace tc5;

constexpr int BM = 128, BN = 128, BK = 64;
// segment mode: one (A, B) tile pair per stage, 4 stages;
// shared-split mode: A_hi, A_lo, B_hi, B_lo per stage (three MMAs reuse them), 3 stages
// Row-chunk moves of the epilogue: 16 consecutive elements of one row, as 16- or 8-byte words
// when the address is aligned and the chunk is whole, element by element otherwise.
__device__ __forceinline__ void load_row16(const float *src, int n, float out[16]) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(src);
    if (n == 16 && (a & 15) == 0) {
        const float4 *s4 = reinterpret_cast<const float4 *>(src);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float4 t = s4[q];
            out[4 * q] = t.x;
            out[4 * q + 1] = t.y;
            out[4 * q + 2] = t.z;
            out[4 * q + 3] = t.w;
        }
    } else if (n == 16 && (a & 7) == 0) {
        const float2 *s2 = reinterpret_cast<const float2 *>(src);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float2 t = s2[q];
            out[2 * q] = t.x;
            out[2 * q + 1] = t.y;
        }
    } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) out[j] = j < n ? src[j] : 0.0f;
    }
}

__device__ __forceinline__ void store_row16(float *dst, int n, const float v[16]) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(dst);
    if (n == 16 && (a & 15) == 0) {
        float4 *d4 = reinterpret_cast<float4 *>(dst);
#pragma unroll
        for (int q = 0; q < 4; ++q) d4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    } else if (n == 16 && (a & 7) == 0) {
        float2 *d2 = reinterpret_cast<float2 *>(dst);
#pragma unroll
        for (int q = 0; q < 8; ++q) d2[q] = make_float2(v[2 * q], v[2 * q + 1]);
    } else {
#pragma unroll
        for (int j = 0; j < 16; ++j)
            if (j < n) dst[j] = v[j];
    }
}

__device__ __forceinline__ void store_row16_bf16(__nv_bfloat16 *dst, int n, const __nv_bfloat16 v[16]) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(dst);
    uint32_t w[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const __nv_bfloat162 pr = __halves2bfloat162(v[2 * q], v[2 * q + 1]);
        w[q] = *reinterpret_cast<const uint32_t *>(&pr);
    }
    if (n == 16 && (a & 15) == 0) {
        uint4 *d4 = reinterpret_cast<uint4 *>(dst);
        d4[0] = make_uint4(w[0], w[1], w[2], w[3]);
        d4[1] = make_uint4(w[4], w[5], w[6], w[7]);
    } else if (n == 16 && (a & 3) == 0) {
        uint32_t *d = reinterpret_cast<uint32_t *>(dst);
#pragma unroll
        for (int q = 0; q < 8; ++q) d[q] = w[q];
    } else {
#pragma unroll
        for (int j = 0; j < 16; ++j)
            if (j < n) dst[j] = v[j];
    }
}

// Transposed-output staging: per epilogue warp a [32 tile columns][32 tile rows] BF16 block for hi
// and for lo, rows padded to 40 elements (80 B, a multiple of 16 B for the 16-byte reads).
constexpr int EPI_THREADS = 128;
constexpr int TPITCH = 40;
constexpr int TSTAGE_BYTES = 4 * 2 * 32 * TPITCH * 2;

template <bool SPLIT, bool WIDE = false> struct Cfg {
    // 128 x 128 output tiles with 64-element K blocks (128-byte swizzle); WIDE (split mode only): 128 x 256
    // tiles with 32-element K blocks (64-byte swizzle), so four stages of A_hi, A_lo, B_hi, B_lo fit and a
    // stage carries the same MMA work with a quarter fewer operand bytes.  (128 x 256 tiles with 64-element
    // blocks leave room for two stages only, which measured slower.)
    static constexpr int BNX = WIDE ? 256 : 128;
    static constexpr int BKX = WIDE ? 32 : BK;
    static constexpr int TILE_AX = BM * BKX * 2;
    static constexpr int TILE_BX = BNX * BKX * 2;
    static constexpr int STAGES = WIDE ? 4 : (SPLIT ? 3 : 4);
    static constexpr int STAGE_BYTES = SPLIT ? 2 * (TILE_AX + TILE_BX) : TILE_AX + TILE_BX;
    static constexpr int SMEM_BYTES =
        STAGES * STAGE_BYTES + TSTAGE_BYTES + 1024 /* alignment slack */ + 256 /* barriers */;
    static constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BNX >> 3) << 17) |
                                      ((uint32_t)(BM >> 4) << 24);
};

struct Maps {
    CUtensorMap a[3];
    CUtensorMap b[3];
};

struct Params {
    int M, N, K, nseg;
    int ksplit;  // K ranges per output tile (gridDim.z); > 1 accumulates C with atomics
    float alpha;
    const float *G;
    long long ldg;
    float *C;
    long long ldc;
    __nv_bfloat16 *Ohi, *Olo;  // row-major hi/lo output (ld = ldo)
    long long ldo;
    __nv_bfloat16 *Thi, *Tlo;  // transposed hi/lo output: T(n, m) (ld = ldt)
    long long ldt;
    int *err;  // device error word (0 = ok)
};

// UMMA shared-memory descriptor for K-major rows of 64 B with 64-byte swizzle: 8-row groups 512 B apart
__device__ __forceinline__ uint64_t smem_desc_k64(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);  // start address
    d |= (uint64_t)1 << 16;                    // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(512 >> 4) << 32;           // stride byte offset
    d |= (uint64_t)1 << 46;                    // descriptor version
    d |= (uint64_t)4 << 61;                    // SWIZZLE_64B
    return d;
}

template <bool WIDE>
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    return WIDE ? smem_desc_k64(saddr) : smem_desc_k128(saddr);
}

// instruction descriptor: D = F32, A = B = BF16, both K-major, M = 128, N = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                            ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_c, uint64_t da, uint64_t db, uint32_t accumulate,
                                          uint32_t idesc = kIdesc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_c),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 consecutive FP32 accumulator columns of this warp's 32 TMEM lanes
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    tmem_ld32_raw(taddr, r);
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Output tile t of a launch: tiles run M-fastest, then N, then the K range (split-K index), so the
// CTAs working at one time share B tiles and the A operand stays in L2.
struct TileCoords {
    int m0, n0, kb0, kblocks;
};

__device__ __forceinline__ TileCoords tile_coords(int t, int mt, int nt, int bnx, int kblocks_all, int kper) {
    TileCoords c;
    const int mi = t % mt, rest = t / mt;
    c.m0 = mi * BM;
    c.n0 = (rest % nt) * bnx;
    c.kb0 = (rest / nt) * kper;
    c.kblocks = max(0, min(kblocks_all, c.kb0 + kper) - c.kb0);
    return c;
}

// Persistent kernel: one CTA per SM walks the tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...
//   warp 0 lane 0 : TMA producer over the operand ring (continues across tiles);
//   warp 1 lane 0 : tcgen05.mma issuer into one of two 128-column TMEM accumulators
//                   (tile j uses accumulator j % 2);
//   warps 2..5    : epilogue of tile j while the MMAs of tile j + 1 run; warp w reads TMEM
//                   lanes 32 (w % 4) .. 32 (w % 4) + 31.
// Barriers: full/empty per ring slot, tfull (MMA -> epilogue, tcgen05.commit) and tempty
// (epilogue -> MMA, 128 arrivals) per accumulator.  Every wait is bounded.
template <bool SPLIT, bool WIDE>
__global__ void __launch_bounds__(192, 1) gemm_kernel(const __grid_constant__ Maps maps, const Params p) {
    using C = Cfg<SPLIT, WIDE>;
    constexpr int STAGES = C::STAGES, STAGE_BYTES = C::STAGE_BYTES;
    constexpr int BNX = C::BNX, TILE_BX = C::TILE_BX, TILE_AX = C::TILE_AX, BKX = C::BKX;
    constexpr uint32_t IDESC = C::IDESC;
    static_assert(BNX % 32 == 0 && (!WIDE || SPLIT), "tile columns come in 32-column chunks; WIDE is split-only");
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __nv_bfloat16 *tstage = reinterpret_cast<__nv_bfloat16 *>(smem + STAGES * STAGE_BYTES);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES + TSTAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *tfull = empty + STAGES;
    uint64_t *tempty = tfull + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tempty + 2);
    int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);

    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int mt = (p.M + BM - 1) / BM, nt = (p.N + BNX - 1) / BNX;
    const int ntiles = mt * nt * p.ksplit;
    const int kblocks_all = (p.K + BKX - 1) / BKX;
    const int kper = (kblocks_all + p.ksplit - 1) / p.ksplit;

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
        // two accumulators of BNX columns (128 lanes x 2 BNX FP32)
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(2 * BNX));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // ---------------- TMA producer
            int it = 0;  // copies issued (ring position)
            bool stop = false;
            for (int t = blockIdx.x; t < ntiles && !stop; t += gridDim.x) {
                const TileCoords tc = tile_coords(t, mt, nt, BNX, kblocks_all, kper);
                const int total = SPLIT ? tc.kblocks : tc.kblocks * p.nseg;
                for (int i = 0; i < total; ++i) {
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
                    if (SPLIT) {
                        // stage layout: A_hi | A_lo | B_hi | B_lo
                        const int kx = (tc.kb0 + i) * BKX;
                        tma_load_2d(sa, &maps.a[0], &full[s], kx, tc.m0);
                        tma_load_2d(sa + TILE_AX, &maps.a[1], &full[s], kx, tc.m0);
                        tma_load_2d(sa + 2 * TILE_AX, &maps.b[0], &full[s], kx, tc.n0);
                        tma_load_2d(sa + 2 * TILE_AX + TILE_BX, &maps.b[1], &full[s], kx, tc.n0);
                    } else {
                        const int seg = i / tc.kblocks, kb = tc.kb0 + i % tc.kblocks;
                        tma_load_2d(sa, &maps.a[seg], &full[s], kb * BKX, tc.m0);
                        tma_load_2d(sa + TILE_AX, &maps.b[seg], &full[s], kb * BKX, tc.n0);
                    }
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
                const TileCoords tc = tile_coords(t, mt, nt, BNX, kblocks_all, kper);
                const int total = SPLIT ? tc.kblocks : tc.kblocks * p.nseg;
                const int acc = j & 1;
                const uint32_t tacc = tmem + (uint32_t)(acc * BNX);
                if (j >= 2 && !mbar_wait(&tempty[acc], ((j >> 1) - 1) & 1)) {
                    atomicExch(p.err, 4);
                    *(volatile int *)abort_flag = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                for (int i = 0; i < total; ++i) {
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
                    const uint32_t sa = smem_u32(smem + s * STAGE_BYTES);
                    if (SPLIT) {
                        const uint32_t sal = sa + TILE_AX, sb = sa + 2 * TILE_AX, sbl = sb + TILE_BX;
#pragma unroll
                        for (int k = 0; k < BKX / 16; ++k) {
                            // 16 BF16 = 32 bytes along K per instruction, inside the swizzle atom
                            const uint32_t o = k * 32;
                            umma_bf16(tacc, smem_desc<WIDE>(sa + o), smem_desc<WIDE>(sb + o),
                                      (i > 0 || k > 0) ? 1u : 0u, IDESC);
                            umma_bf16(tacc, smem_desc<WIDE>(sa + o), smem_desc<WIDE>(sbl + o), 1u, IDESC);
                            umma_bf16(tacc, smem_desc<WIDE>(sal + o), smem_desc<WIDE>(sb + o), 1u, IDESC);
                        }
                    } else {
                        const uint32_t sb = sa + TILE_AX;
#pragma unroll
                        for (int k = 0; k < BKX / 16; ++k) {
                            // advance 16 BF16 = 32 bytes along K inside the 128-byte swizzle atom
                            umma_bf16(tacc, smem_desc_k128(sa + k * 32), smem_desc_k128(sb + k * 32),
                                      (i > 0 || k > 0) ? 1u : 0u);
                        }
                    }
                    umma_commit(&empty[s]);  // slot s may be refilled once these MMAs have read it
                    ++it;
                }
                umma_commit(&tfull[acc]);  // accumulator complete (or abandoned) -> epilogue
            }
        }
    } else {
        // ---------------- epilogue (warps 2..5, 128 threads)
        const int rq = warp & 3;  // TMEM lane quarter this warp may access
        const int rloc = rq * 32 + lane;
        const bool stage_t = p.Thi != nullptr && p.ksplit == 1;
        __nv_bfloat16 *sh = tstage + (warp - 2) * (2 * 32 * TPITCH);
        __nv_bfloat16 *sl = sh + 32 * TPITCH;
        int j = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++j) {
            const TileCoords tc = tile_coords(t, mt, nt, BNX, kblocks_all, kper);
            const int total = SPLIT ? tc.kblocks : tc.kblocks * p.nseg;
            const int acc = j & 1;
            const int m0 = tc.m0, n0 = tc.n0;
            const int row = m0 + rloc;
            if (p.G && p.ksplit == 1 && row < p.M) {
                // pull this tile's G row into L2 while its MMAs run (128-byte lines, inside the matrix)
                const float *g = p.G + (long long)row * p.ldg + n0;
                const int ncols = min(BNX, p.N - n0);
                for (int c = 0; c < ncols; c += 32) asm volatile("prefetch.global.L2 [%0];" ::"l"(g + c));
            }
            const bool ok = __all_sync(0xffffffffu, mbar_wait(&tfull[acc], (j >> 1) & 1) ? 1 : 0) != 0;
            if (!ok && lane == 0) atomicExch(p.err, 3);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const bool live = ok && !*(volatile int *)abort_flag && total > 0;  // warp-uniform
            for (int c0 = 0; c0 < BNX; c0 += 32) {
                float v[32];
                tmem_ld32(tmem + ((uint32_t)(rq * 32) << 16) + (uint32_t)(acc * BNX + c0), v);
                const int col0 = n0 + c0;
                if (live && row < p.M && col0 < p.N) {
                    const int ncol = min(32, p.N - col0);
                    if (p.ksplit > 1) {  // partial sums over this tile's K range
#pragma unroll
                        for (int q = 0; q < 32; ++q)
                            if (q < ncol) atomicAdd(&p.C[(long long)row * p.ldc + col0 + q], p.alpha * v[q]);
                    } else {
                        const int n1 = min(16, ncol), n2 = ncol - 16;  // the two 16-column halves (n2 <= 0: none)
#pragma unroll
                        for (int q = 0; q < 32; ++q) v[q] *= p.alpha;
                        if (p.G) {
                            float g[32];
                            const float *gr = p.G + (long long)row * p.ldg + col0;
                            load_row16(gr, n1, g);
                            if (n2 > 0) load_row16(gr + 16, n2, g + 16);
#pragma unroll
                            for (int q = 0; q < 32; ++q) v[q] *= g[q];
                        }
                        if (p.C) {
                            store_row16(p.C + (long long)row * p.ldc + col0, n1, v);
                            if (n2 > 0) store_row16(p.C + (long long)row * p.ldc + col0 + 16, n2, v + 16);
                        }
                        if (p.Ohi || stage_t) {
                            __nv_bfloat16 hi[32], lo[32];
#pragma unroll
                            for (int q = 0; q < 32; ++q) {
                                hi[q] = __float2bfloat16_rn(v[q]);
                                lo[q] = __float2bfloat16_rn(v[q] - __bfloat162float(hi[q]));
                            }
                            if (p.Ohi) {
                                __nv_bfloat16 *oh = p.Ohi + (long long)row * p.ldo + col0;
                                __nv_bfloat16 *ol = p.Olo + (long long)row * p.ldo + col0;
                                store_row16_bf16(oh, n1, hi);
                                store_row16_bf16(ol, n1, lo);
                                if (n2 > 0) {
                                    store_row16_bf16(oh + 16, n2, hi + 16);
                                    store_row16_bf16(ol + 16, n2, lo + 16);
                                }
                            }
                            if (stage_t) {
                                // column c0+q of the tile: the warp's 32 lanes write 32 consecutive rows
#pragma unroll
                                for (int q = 0; q < 32; ++q) {
                                    sh[q * TPITCH + lane] = hi[q];
                                    sl[q * TPITCH + lane] = lo[q];
                                }
                            }
                        }
                    }
                }
                if (stage_t) {
                    __syncwarp();
                    if (live && col0 < p.N) {
                        // this warp's 32 x 32 block of T: T-rows col0 .. col0+31, T-columns m0+32rq .. +31
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const int c = q * 8 + (lane >> 2), part = lane & 3;
                            const int trow = col0 + c, tcol0 = m0 + rq * 32 + part * 8;
                            const int nv = min(8, p.M - tcol0);
                            if (trow < p.N && nv > 0) {
                                const long long off = (long long)trow * p.ldt + tcol0;
                                const __nv_bfloat16 *srh = sh + c * TPITCH + part * 8, *srl = sl + c * TPITCH + part * 8;
                                __nv_bfloat16 *dh = p.Thi + off, *dl = p.Tlo + off;
                                if (nv == 8 &&
                                    ((reinterpret_cast<uintptr_t>(dh) | reinterpret_cast<uintptr_t>(dl)) & 15) == 0) {
                                    *reinterpret_cast<uint4 *>(dh) = *reinterpret_cast<const uint4 *>(srh);
                                    *reinterpret_cast<uint4 *>(dl) = *reinterpret_cast<const uint4 *>(srl);
                                } else {
                                    for (int e = 0; e < nv; ++e) {
                                        dh[e] = srh[e];
                                        dl[e] = srl[e];
                                    }
                                }
                            }
                        }
                    }
                    __syncwarp();
                }
            }
            // the accumulator has been read: hand it back to the MMA issuer
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            mbar_arrive(&tempty[acc]);
            if (!ok) break;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BNX));
    }
}

// FP32 -> BF16 hi/lo split, with zero padding of the columns [cols, ld)
__global__ void split_kernel(int rows, int cols, const float *X, long long ldx, int transpose, __nv_bfloat16 *hi,
                             __nv_bfloat16 *lo, long long ld) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long outr = transpose ? cols : rows;
    if (idx >= outr * ld) return;
    const long long r = idx / ld, c = idx % ld;
    float x = 0.0f;
    const long long inr = transpose ? c : r, inc = transpose ? r : c;
    if (c < (transpose ? rows : cols)) x = X[inr * ldx + inc];
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    hi[idx] = h;
    lo[idx] = __float2bfloat16_rn(x - __bfloat162float(h));
}

__global__ void split64_kernel(int rows, int cols, const double *X, long long ldx, int transpose, __nv_bfloat16 *hi,
                               __nv_bfloat16 *lo, long long ld, double scale) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long outr = transpose ? cols : rows;
    if (idx >= outr * ld) return;
    const long long r = idx / ld, c = idx % ld;
    double x = 0.0;
    const long long inr = transpose ? c : r, inc = transpose ? r : c;
    if (c < (transpose ? rows : cols)) x = scale * X[inr * ldx + inc];
    const float xf = (float)x;
    const __nv_bfloat16 h = __float2bfloat16_rn(xf);
    hi[idx] = h;
    lo[idx] = __float2bfloat16_rn((float)(x - (double)__bfloat162float(h)));
}

// ---------------------------------------------------------------------------- host side
thread_local char g_err[256] = "";
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::mutex g_mutex;
int *g_errword[64] = {nullptr};

int get_encode() {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (g_encode) return 0;
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
        snprintf(g_err, sizeof(g_err), "cuTensorMapEncodeTiled unavailable");
        return -1;
    }
    g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    return 0;
}

int make_map(CUtensorMap *map, const void *base, int rows, int cols, long long ld, int box_rows = BM,
             int box_cols = BK) {
    // 2D BF16 tensor: innermost dimension = columns (K), box box_cols x box_rows, zero fill; rows of 64
    // elements (128 B) use the 128-byte swizzle, rows of 32 elements the 64-byte swizzle
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * 2)};
    cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    const CUtensorMapSwizzle sw = box_cols == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B;
    CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        snprintf(g_err, sizeof(g_err), "cuTensorMapEncodeTiled failed (%d): rows %d cols %d ld %lld", (int)r, rows,
                 cols, ld);
        return -1;
    }
    return 0;
}

}  // namespace tcg

extern "C" {

const char *dftb_tc_last_error(void) { return tcg::g_err; }

int dftb_bf16x3_gemm_ex(int M, int N, int K, int nseg, int shared_split, int ksplit, const void *const *A, int lda,
                        const void *const *B, int ldb, float alpha, const float *G, int ldg, float *C, int ldc,
                        void *Ohi, void *Olo, int ldo, void *Thi, void *Tlo, int ldt, int *err, void *stream);

int dftb_bf16x3_gemm(int M, int N, int K, int nseg, const void *const *A, int lda, const void *const *B, int ldb,
                     float alpha, const float *G, int ldg, float *C, int ldc, void *Ohi, void *Olo, int ldo, void *Thi,
                     void *Tlo, int ldt, int *err, void *stream) {
    return dftb_bf16x3_gemm_ex(M, N, K, nseg, 0, 1, A, lda, B, ldb, alpha, G, ldg, C, ldc, Ohi, Olo, ldo, Thi, Tlo,
                               ldt, err, stream);
}

int dftb_bf16x3_gemm_ex(int M, int N, int K, int nseg, int shared_split, int ksplit, const void *const *A, int lda,
                        const void *const *B, int ldb, float alpha, const float *G, int ldg, float *C, int ldc,
                        void *Ohi, void *Olo, int ldo, void *Thi, void *Tlo, int ldt, int *err, void *stream) {
    using namespace tcg;
    if (M <= 0 || N <= 0 || K <= 0 || nseg < 1 || nseg > 3 || ksplit < 1 || ksplit > 64) return DFTB_ERR_BAD_SIZE;
    if (shared_split < 0 || shared_split > 2 || (shared_split && nseg != 2)) {
        snprintf(g_err, sizeof(g_err), "bf16x3_gemm: shared-split mode (1, or 2 for 128 x 256 tiles) takes the pairs "
                 "(A_hi, A_lo), (B_hi, B_lo)");
        return DFTB_ERR_BAD_SIZE;
    }
    if (ksplit > 1 && (!C || G || Ohi || Thi)) {
        snprintf(g_err, sizeof(g_err), "bf16x3_gemm: split-K accumulates into C only (zeroed by the caller)");
        return DFTB_ERR_BAD_SIZE;
    }
    if (lda % 8 || ldb % 8 || lda < K || ldb < K) {
        snprintf(g_err, sizeof(g_err), "bf16x3_gemm: lda/ldb must be multiples of 8 and >= K");
        return DFTB_ERR_BAD_SIZE;
    }
    if (!A || !B || !err) return DFTB_ERR_NULL;
    if ((Ohi && (!Olo || ldo < N)) || (Thi && (!Tlo || ldt < M)) || (C && ldc < N) || (G && ldg < N))
        return DFTB_ERR_BAD_SIZE;
    if (get_encode()) return DFTB_ERR_CUDA;
    Maps maps;
    memset(&maps, 0, sizeof(maps));
    for (int s = 0; s < nseg; ++s) {
        if (!A[s] || !B[s]) return DFTB_ERR_NULL;
        if ((reinterpret_cast<uintptr_t>(A[s]) & 15) || (reinterpret_cast<uintptr_t>(B[s]) & 15)) {
            snprintf(g_err, sizeof(g_err), "bf16x3_gemm: operands must be 16-byte aligned");
            return DFTB_ERR_BAD_SIZE;
        }
        const bool wide = shared_split == 2;
        const int bkx = wide ? Cfg<true, true>::BKX : BK;
        const int bnx = wide ? Cfg<true, true>::BNX : (shared_split ? Cfg<true>::BNX : Cfg<false>::BNX);
        if (make_map(&maps.a[s], A[s], M, K, lda, BM, bkx) || make_map(&maps.b[s], B[s], N, K, ldb, bnx, bkx))
            return DFTB_ERR_CUDA;
    }
    Params p;
    p.M = M;
    p.N = N;
    p.K = K;
    p.nseg = nseg;
    p.ksplit = ksplit;
    p.alpha = alpha;
    p.G = G;
    p.ldg = ldg;
    p.C = C;
    p.ldc = ldc;
    p.Ohi = reinterpret_cast<__nv_bfloat16 *>(Ohi);
    p.Olo = reinterpret_cast<__nv_bfloat16 *>(Olo);
    p.ldo = ldo;
    p.Thi = reinterpret_cast<__nv_bfloat16 *>(Thi);
    p.Tlo = reinterpret_cast<__nv_bfloat16 *>(Tlo);
    p.ldt = ldt;
    p.err = err;
    static bool attr_set[3][64] = {{false}};
    int dev = 0;
    cudaGetDevice(&dev);
    const int mode = shared_split;  // 0 segments, 1 split, 2 split with 128 x 256 tiles
    const int smem = mode == 2 ? Cfg<true, true>::SMEM_BYTES : (mode ? Cfg<true>::SMEM_BYTES : Cfg<false>::SMEM_BYTES);
    if (dev >= 0 && dev < 64 && !attr_set[mode][dev]) {
        cudaError_t e =
            mode == 2 ? cudaFuncSetAttribute(gemm_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)
            : mode    ? cudaFuncSetAttribute(gemm_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)
                      : cudaFuncSetAttribute(gemm_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             smem);
        if (e != cudaSuccess) {
            snprintf(g_err, sizeof(g_err), "bf16x3_gemm: cannot reserve %d bytes of shared memory", smem);
            return DFTB_ERR_CUDA;
        }
        attr_set[mode][dev] = true;
    }
    const int bnx = mode == 2 ? Cfg<true, true>::BNX : (mode ? Cfg<true>::BNX : Cfg<false>::BNX);
    // persistent launch: one CTA per SM (the shared-memory footprint admits one), each walking tiles
    const long long ntiles = (long long)((M + BM - 1) / BM) * ((N + bnx - 1) / bnx) * ksplit;
    if (ntiles > (1LL << 30)) return DFTB_ERR_BAD_SIZE;
    static int sm_count[64] = {0};
    if (dev >= 0 && dev < 64 && sm_count[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        sm_count[dev] = n;
    }
    const int sms = (dev >= 0 && dev < 64) ? sm_count[dev] : 148;
    dim3 grid((unsigned)(ntiles < sms ? ntiles : sms));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (mode == 2)
        gemm_kernel<true, true><<<grid, 192, smem, st>>>(maps, p);
    else if (mode == 1)
        gemm_kernel<true, false><<<grid, 192, smem, st>>>(maps, p);
    else
        gemm_kernel<false, false><<<grid, 192, smem, st>>>(maps, p);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        snprintf(g_err, sizeof(g_err), "gemm_kernel: %s", cudaGetErrorString(e));
        return DFTB_ERR_CUDA;
    }
    return DFTB_OK;
}

int dftb_split_bf16(int rows, int cols, const float *X, int ldx, int transpose, void *hi, void *lo, int ld,
                    void *stream) {
    using namespace tcg;
    if (rows <= 0 || cols <= 0 || ld < (transpose ? rows : cols)) return DFTB_ERR_BAD_SIZE;
    if (!X || !hi || !lo) return DFTB_ERR_NULL;
    const long long n = (long long)(transpose ? cols : rows) * ld;
    split_kernel<<<(unsigned)((n + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        rows, cols, X, ldx, transpose, reinterpret_cast<__nv_bfloat16 *>(hi), reinterpret_cast<__nv_bfloat16 *>(lo),
        ld);
    return cudaGetLastError() == cudaSuccess ? DFTB_OK : DFTB_ERR_CUDA;
}

int dftb_split_bf16_f64(int rows, int cols, const double *X, int ldx, int transpose, double scale, void *hi, void *lo,
                        int ld, void *stream) {
    using namespace tcg;
    if (rows <= 0 || cols <= 0 || ld < (transpose ? rows : cols)) return DFTB_ERR_BAD_SIZE;
    if (!X || !hi || !lo) return DFTB_ERR_NULL;
    const long long n = (long long)(transpose ? cols : rows) * ld;
    split64_kernel<<<(unsigned)((n + 255) / 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        rows, cols, X, ldx, transpose, reinterpret_cast<__nv_bfloat16 *>(hi), reinterpret_cast<__nv_bfloat16 *>(lo),
        ld, scale);
    return cudaGetLastError() == cudaSuccess ? DFTB_OK : DFTB_ERR_CUDA;
}

}  // extern "C"
