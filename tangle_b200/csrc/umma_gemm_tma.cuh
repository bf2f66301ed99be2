// umma_gemm_tma.cuh -- persistent BF16 products for K-major operands:
// TMA-fed, pipelined, two tensor-memory accumulators.
//
// D[M x N] = A[M x K] B[N x K]^T (+ the epilogue of umma_gemm.cuh), both
// operands K-major (a[m * lda + k], b[n * ldb + k]), N % 16 == 0, N <= 256,
// K % 8 == 0. Each CTA walks the 128-row tiles blockIdx.x, + gridDim.x, ...
// with three roles:
//   warp 0 (one lane): the producer. For each 64-wide contraction chunk it
//     waits for a free pipeline stage, announces the stage's bytes on its
//     "full" mbarrier and issues two 2-D TMA loads: A (box 64 x 128 rows)
//     and B (box 64 x N rows), both with the 128-byte swizzle. A box row is
//     the chunk's 64 bf16 of one operand row (128 bytes, one request), and
//     the box lands in the canonical K-major SWIZZLE_128B layout: row r at
//     r * 128 bytes, its 16-byte piece j at piece j ^ (r % 8), 8-row atoms
//     of 1024 bytes (the stride byte offset). The MMA for contraction step
//     s (16 elements, 32 bytes) starts its descriptors 32 s bytes into the
//     atom; the tensor core applies the same XOR to the address bits, so
//     every stage starts on a 1024-byte boundary. Rows past M and k past K
//     read as zero.
//   warp 1 (one lane): the MMA issuer. It waits for a stage, issues its
//     tcgen05.mma instructions (K = 16 each) into the tile's accumulator and
//     commits them to the stage's "empty" mbarrier, which frees the stage
//     for the producer once the tensor core has read it; after a tile's last
//     chunk it commits to the accumulator's "full" mbarrier. Tiles alternate
//     between two accumulators, so the next tile accumulates while the
//     previous one is being drained.
//   warps 2-5: the epilogue. Each reads its 32 tensor-memory lanes of the
//     finished accumulator (warp w may access lanes 32 (w % 4) .. + 31) 16
//     columns at a time, one row per lane, and turns the slice around in
//     shared memory so that four lanes share a row: bias / ReLU / mask /
//     residual are applied and the results stored as 64-byte row pieces
//     (f32) or 32-byte ones (bf16) instead of one 16-byte piece per row and
//     lane. Then it arrives on the accumulator's "empty" mbarrier.
// Every mbarrier wait is bounded: one that gives up records an error and
// the CTA stops issuing work; before it exits, the producer waits (bounded)
// for its loads still in flight and the MMA issuer for its last commit, and
// the tensor memory is freed.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cstdint>

#include "umma_gemm.cuh"

namespace tgl {

constexpr int TMA_GEMM_STAGES = 4;
constexpr int TMA_GEMM_THREADS = 192;  // producer, MMA, four epilogue warps

// Shared memory of one pipeline stage: A chunk (128 x 64 bf16) and B chunk
// (N x 64 bf16), each 1 KiB aligned.
__host__ __device__ inline uint32_t tma_stage_bytes(int n) {
    return (uint32_t)(GEMM_BM * GEMM_KC * 2) + (((uint32_t)n * GEMM_KC * 2 + 1023u) & ~1023u);
}

// Epilogue slices: 32 rows x 16 columns per warp, rows 20 floats apart (the
// 4-float pad keeps both the row-per-lane writes and the row-piece reads
// free of bank conflicts).
constexpr int TMA_EPI_STRIDE = 20;
constexpr uint32_t TMA_EPI_BYTES = 4u * 32u * TMA_EPI_STRIDE * 4u;

// Dynamic shared memory of the kernel: the stages, the epilogue slices and
// the slack that lets the first stage start on a 1024-byte boundary.
__host__ __device__ inline uint32_t tma_smem_bytes(int n) {
    return (uint32_t)TMA_GEMM_STAGES * tma_stage_bytes(n) + TMA_EPI_BYTES + 1024u;
}

// tcgen05 shared-memory descriptor of a K-major operand in the 128-byte
// swizzle layout: start address, leading byte offset 16 (unused by this
// layout, the value the canonical form carries), stride byte offset 1024
// (one 8-row atom), version 1 at bit 46, base offset 0, layout type 2
// (SWIZZLE_128B) at bits 61-63.
__device__ inline uint64_t smem_desc_sw128(uint32_t addr) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)(16u >> 4) << 16;
    d |= (uint64_t)(1024u >> 4) << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)2u << 61;
    return d;
}

__device__ inline void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count));
}

__device__ inline void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ inline void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// 2-D TMA load of one box into shared memory, completing on `bar`. No
// multicast: the box goes to this CTA only.
__device__ inline void tma_load_2d(uint32_t dst, const CUtensorMap *map, int32_t x, int32_t y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__global__ void __launch_bounds__(TMA_GEMM_THREADS, 1)
    umma_gemm_tma_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                         GemmArgs g) {
    extern __shared__ __align__(1024) uint8_t tma_smem[];
    __shared__ __align__(8) uint64_t full_bar[TMA_GEMM_STAGES], empty_bar[TMA_GEMM_STAGES];
    __shared__ __align__(8) uint64_t acc_full_bar[2], acc_empty_bar[2];
    __shared__ uint32_t tmem_base_slot;
    __shared__ volatile int failed;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n = g.n;
    const uint32_t stage_bytes = tma_stage_bytes(n);
    const uint32_t smem0 = (smem_u32(tma_smem) + 1023u) & ~1023u;
    const int64_t tiles = ((int64_t)g.m + GEMM_BM - 1) / GEMM_BM;
    const int64_t chunks = (g.k + GEMM_KC - 1) / GEMM_KC;
    int cols = 32;
    while (cols < n) cols <<= 1;  // one accumulator: n f32 columns, a power of two >= 32
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_slot)),
                     "r"(2 * cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < TMA_GEMM_STAGES; ++s) {
            mbar_init(smem_u32(&full_bar[s]), 1);
            mbar_init(smem_u32(&empty_bar[s]), 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(smem_u32(&acc_full_bar[a]), 1);
            mbar_init(smem_u32(&acc_empty_bar[a]), 4);
        }
        asm volatile("fence.mbarrier_init.release.cluster;");
        failed = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base_slot;

    if (warp == 0) {
        if (lane == 0) {
            // Producer.
            uint32_t stage = 0, phase = 1;  // a fresh "empty" barrier counts as free
            uint32_t issued[TMA_GEMM_STAGES] = {};  // loads issued per stage
            for (int64_t t = blockIdx.x; t < tiles && !failed; t += gridDim.x) {
                for (int64_t c = 0; c < chunks && !failed; ++c) {
                    if (!mbar_wait(smem_u32(&empty_bar[stage]), phase, g.error)) {
                        failed = 1;
                        break;
                    }
                    // Whole boxes: the part past K (and past M) is filled
                    // with zeros and counts toward the stage's bytes.
                    const int32_t x = (int32_t)(c * GEMM_KC);
                    const uint32_t full = smem_u32(&full_bar[stage]);
                    mbar_expect_tx(full, (uint32_t)(GEMM_KC * 2) * (uint32_t)(GEMM_BM + n));
                    const uint32_t sa = smem0 + stage * stage_bytes;
                    const uint32_t sb = sa + GEMM_BM * GEMM_KC * 2;
                    tma_load_2d(sa, &map_a, x, (int32_t)(t * GEMM_BM), full);
                    tma_load_2d(sb, &map_b, x, 0, full);
                    ++issued[stage];
                    if (++stage == TMA_GEMM_STAGES) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
            }
            // Loads still in flight (only after a failure): wait, bounded, for
            // the stages issued but not consumed, so none lands after exit.
            if (failed) {
                for (int s = 0; s < TMA_GEMM_STAGES; ++s)
                    if (issued[s]) mbar_wait(smem_u32(&full_bar[s]), (issued[s] - 1u) & 1u, nullptr);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer.
            uint32_t stage = 0, phase = 0;
            uint32_t acc = 0, acc_phase[2] = {1u, 1u};  // fresh accumulators count as drained
            const uint32_t idesc = instr_desc_bf16(GEMM_BM, n, 0, 0);
            uint32_t last_commit_bar = 0, last_commit_phase = 0;
            bool committed = false;
            for (int64_t t = blockIdx.x; t < tiles && !failed; t += gridDim.x) {
                if (!mbar_wait(smem_u32(&acc_empty_bar[acc]), acc_phase[acc], g.error)) {
                    failed = 1;
                    break;
                }
                acc_phase[acc] ^= 1u;
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t d_tmem = tmem + acc * (uint32_t)cols;
                for (int64_t c = 0; c < chunks; ++c) {
                    if (!mbar_wait(smem_u32(&full_bar[stage]), phase, g.error)) {
                        failed = 1;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    const int64_t k0 = c * GEMM_KC;
                    const int kk = (int)(g.k - k0 < GEMM_KC ? g.k - k0 : GEMM_KC);
                    const int steps = (kk + 15) / 16;
                    const uint32_t sa = smem0 + stage * stage_bytes;
                    const uint32_t sb = sa + GEMM_BM * GEMM_KC * 2;
                    for (int s = 0; s < steps; ++s) {
                        const uint64_t da = smem_desc_sw128(sa + 32u * (uint32_t)s);
                        const uint64_t db = smem_desc_sw128(sb + 32u * (uint32_t)s);
                        const uint32_t accumulate = (c > 0 || s > 0) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
                            "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
                    }
                    // The stage is free once these MMAs have read it.
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_u32(&empty_bar[stage]))
                                 : "memory");
                    last_commit_bar = smem_u32(&empty_bar[stage]);
                    last_commit_phase = phase;
                    committed = true;
                    if (++stage == TMA_GEMM_STAGES) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (failed) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&acc_full_bar[acc]))
                             : "memory");
                acc ^= 1u;
            }
            // After a failure: let the last MMAs finish before the tensor
            // memory is freed (bounded).
            if (failed && committed) mbar_wait(last_commit_bar, last_commit_phase, nullptr);
        }
    } else {
        // Epilogue: warps 2-5; this warp's tensor-memory lanes and tile rows.
        const int quarter = warp & 3;
        float *slice = reinterpret_cast<float *>(tma_smem + (smem0 - smem_u32(tma_smem)) +
                                                 TMA_GEMM_STAGES * stage_bytes) +
                       quarter * 32 * TMA_EPI_STRIDE;
        const int cq = 4 * (lane & 3);  // this lane's 4 columns of a slice
        uint32_t acc = 0, acc_phase[2] = {0u, 0u};
        for (int64_t t = blockIdx.x; t < tiles && !failed; t += gridDim.x) {
            // The whole warp agrees on the wait before its collective loads.
            const bool ready = __all_sync(0xFFFFFFFFu, mbar_wait(smem_u32(&acc_full_bar[acc]), acc_phase[acc], g.error));
            if (!ready) {
                failed = 1;
                break;
            }
            acc_phase[acc] ^= 1u;
            asm volatile("tcgen05.fence::after_thread_sync;");
            const int64_t row0 = t * GEMM_BM + 32 * quarter;
            const uint32_t d_tmem = tmem + acc * (uint32_t)cols;
            for (int c0 = 0; c0 < n; c0 += 16) {
                uint32_t r[16];
                const uint32_t taddr = d_tmem + ((uint32_t)(32 * quarter) << 16) + (uint32_t)c0;
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15}, [%16];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                      "=r"(r[15])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                // Row per lane in.
                float4 *mine = reinterpret_cast<float4 *>(slice + lane * TMA_EPI_STRIDE);
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    mine[j] = make_float4(__uint_as_float(r[4 * j]), __uint_as_float(r[4 * j + 1]),
                                          __uint_as_float(r[4 * j + 2]), __uint_as_float(r[4 * j + 3]));
                __syncwarp();
                // Four lanes per row out: rows lane / 4 + 8 i, columns c0 + cq .. + 3.
                const int col = c0 + cq;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int rr = (lane >> 2) + 8 * i;
                    const int64_t row = row0 + rr;
                    const float4 a4 = *reinterpret_cast<const float4 *>(slice + rr * TMA_EPI_STRIDE + cq);
                    if (row < g.m) {
                        float v[4] = {a4.x, a4.y, a4.z, a4.w};
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            float x = v[j];
                            if (g.bias) x += g.bias[col + j];
                            if (g.relu) x = fmaxf(x, 0.0f);
                            if (g.mask && !(__bfloat162float(g.mask[row * g.ld_mask + col + j]) > 0.0f)) x = 0.0f;
                            if (g.residual) x += g.residual[row * g.ld_res + col + j];
                            v[j] = x;
                        }
                        if (g.out_f32)
                            *reinterpret_cast<float4 *>(g.out_f32 + row * g.ldo + col) = make_float4(v[0], v[1], v[2], v[3]);
                        if (g.out_bf16) {
                            __nv_bfloat162 h[2] = {__floats2bfloat162_rn(v[0], v[1]), __floats2bfloat162_rn(v[2], v[3])};
                            *reinterpret_cast<uint2 *>(g.out_bf16 + row * g.ldo_bf16 + col) = *reinterpret_cast<uint2 *>(h);
                        }
                    }
                }
                __syncwarp();
            }
            // This warp's lanes are read: the accumulator may be reused.
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(&acc_empty_bar[acc]));
            acc ^= 1u;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (warp == 1) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * cols));
}

}  // namespace tgl
