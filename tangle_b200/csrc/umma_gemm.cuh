// umma_gemm.cuh -- BF16 matrix products on the 5th-generation tensor cores
// (tcgen05.mma, accumulators in tensor memory) for the warm-start network.
//
// D[M x N] = sum_k A[m, k] B[n, k] over k in [k_begin, k_end), f32 accumulate.
// Each operand is K-major (A[m * ld + k]) or MN-major (A[k * ld + m]) in
// global memory; a CTA of 128 threads owns one 128-row tile of D and loops
// over K in chunks of up to 64, staging each chunk into shared memory in
// the canonical no-swizzle layout the MMA descriptors describe:
//
//   8 x 16-byte "core matrices"; element (r, k) of an R-row operand lives at
//   ((k / 8) * (R / 8) + r / 8) * 128 bytes, plus, within the core matrix,
//   (r % 8) * 16 + (k % 8) * 2 for K-major or (k % 8) * 16 + (r % 8) * 2
//   for MN-major. Row groups are 128 bytes apart (stride byte offset) and
//   k groups (R / 8) * 128 bytes apart (leading byte offset), in both cases.
//
// One elected thread issues the chunk's MMAs (K = 16 each) and commits them
// to an mbarrier that every thread waits on (a bounded wait that records a
// timeout instead of spinning forever). Then each warp reads its 32 rows of
// the accumulator with tcgen05.ld and runs the epilogue. Descriptor bit
// layouts follow the PTX ISA's tcgen05 shared-memory and instruction
// descriptors.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace tgl {

struct GemmArgs {
    const __nv_bfloat16 *a;  // K-major: a[m * lda + k]; MN-major: a[k * lda + m]
    const __nv_bfloat16 *b;  // K-major: b[n * ldb + k]; MN-major: b[k * ldb + n]
    int64_t lda, ldb;
    int m, n;                // D is m x n; n % 16 == 0, 16 <= n <= 256
    int64_t k;               // contraction length (% 8 == 0 when an operand is K-major)
    int a_mn, b_mn;          // operand majors (0 = K-major, 1 = MN-major)
    int64_t k_split;         // contraction per CTA along grid.y (split K), % 64 == 0
    // Epilogue: v = acc (+ bias[n]) (relu) -> out_f32[m * ldo + n] and/or
    // out_bf16[m * ldo_bf16 + n]; with split K, out_f32 + blockIdx.y * m * ldo.
    const float *bias;
    int relu;
    // Optional: v *= (mask[m * ld_mask + n] > 0) (the ReLU derivative of a
    // stored activation), then v += residual[m * ld_res + n].
    const __nv_bfloat16 *mask;
    int64_t ld_mask;
    const float *residual;
    int64_t ld_res;
    float *out_f32;
    int64_t ldo;
    __nv_bfloat16 *out_bf16;
    int64_t ldo_bf16;
    unsigned int *error;     // set to 1 when a wait gave up
};

constexpr int GEMM_BM = 128;
constexpr int GEMM_KC = 64;   // contraction elements staged per chunk
constexpr int GEMM_THREADS = 128;

__device__ inline uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// tcgen05 shared-memory matrix descriptor, no swizzle: start address, leading
// and stride byte offsets (all >> 4), the fixed version field (1) at bit 46,
// base offset 0, layout type 0.
__device__ inline uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;
    return d;
}

// Instruction descriptor of kind::f16: D f32 (bits 4-5 = 1), A and B bf16
// (bits 7-9 = 1, 10-12 = 1), majors at bits 15 / 16, N >> 3 at bit 17,
// M >> 4 at bit 24.
__host__ __device__ inline uint32_t instr_desc_bf16(int m, int n, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

// Stage rows [r0, r0 + R) x contraction [k0, k0 + kc) of one operand into
// the canonical layout at `dst`; out-of-range elements become zero. Every
// 16-byte global vector is one row of one core matrix.
template <int R>
__device__ inline void stage_operand(uint8_t *dst, const __nv_bfloat16 *src, int64_t ld, int mn, int rows,
                                     int64_t r0, int64_t k0, int kc, int64_t k_end) {
    const int kgroups = kc / 8;
    if (!mn) {
        // K-major: vector (r, kg) holds k = k0 + 8 kg .. +7 of row r.
        for (int v = threadIdx.x; v < R * kgroups; v += blockDim.x) {
            const int r = v / kgroups, kg = v % kgroups;
            const int64_t row = r0 + r, kk = k0 + 8 * kg;
            uint4 val = make_uint4(0u, 0u, 0u, 0u);
            if (row < rows && kk < k_end) val = *reinterpret_cast<const uint4 *>(src + row * ld + kk);
            *reinterpret_cast<uint4 *>(dst + (kg * (R / 8) + r / 8) * 128 + (r % 8) * 16) = val;
        }
    } else {
        // MN-major: vector (k, rg) holds r = r0 + 8 rg .. +7 of contraction row k.
        const int rgroups = R / 8;
        for (int v = threadIdx.x; v < kc * rgroups; v += blockDim.x) {
            const int k = v / rgroups, rg = v % rgroups;
            const int64_t kk = k0 + k, row = r0 + 8 * rg;
            uint4 val = make_uint4(0u, 0u, 0u, 0u);
            if (kk < k_end && row < rows) val = *reinterpret_cast<const uint4 *>(src + kk * ld + row);
            *reinterpret_cast<uint4 *>(dst + ((k / 8) * rgroups + rg) * 128 + (k % 8) * 16) = val;
        }
    }
}

__device__ inline bool mbar_wait(uint32_t bar, uint32_t phase, unsigned int *error) {
    for (uint32_t spin = 0; spin < (1u << 26); ++spin) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
        if (done) return true;
    }
    if (error) atomicExch(error, 1u);
    return false;
}

// One 128 x N tile of D per CTA (blockIdx.x over M tiles, blockIdx.y over
// K splits). N columns of f32 accumulator in tensor memory.
__global__ void __launch_bounds__(GEMM_THREADS, 1) umma_gemm_kernel(GemmArgs g) {
    extern __shared__ __align__(1024) uint8_t gemm_smem[];
    __shared__ __align__(8) uint64_t mma_bar;
    __shared__ uint32_t tmem_base_slot;
    __shared__ int failed;
    uint8_t *sa = gemm_smem;                                    // 128 x KC
    uint8_t *sb = gemm_smem + GEMM_BM * GEMM_KC * 2;            // N x KC
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t m0 = (int64_t)blockIdx.x * GEMM_BM;
    const int64_t k_begin = (int64_t)blockIdx.y * g.k_split;
    const int64_t k_end = k_begin + g.k_split < g.k ? k_begin + g.k_split : g.k;
    int cols = 32;
    while (cols < g.n) cols <<= 1;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_slot)),
                     "r"(cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mma_bar)));
        asm volatile("fence.mbarrier_init.release.cluster;");
        failed = 0;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base_slot;
    const uint32_t idesc = instr_desc_bf16(GEMM_BM, g.n, g.a_mn, g.b_mn);
    const uint32_t lbo_a = (GEMM_BM / 8) * 128, lbo_b = (uint32_t)(g.n / 8) * 128;
    uint32_t phase = 0;
    bool any = false;
    for (int64_t k0 = k_begin; k0 < k_end; k0 += GEMM_KC) {
        // The chunk, rounded up to the MMA's K of 16 (the staging zero-fills
        // contraction indices at or past k_end).
        const int kc_raw = (int)((k_end - k0) < GEMM_KC ? (k_end - k0) : GEMM_KC);
        const int kc = (kc_raw + 15) & ~15;
        stage_operand<GEMM_BM>(sa, g.a, g.lda, g.a_mn, g.m, m0, k0, kc, k_end);
        // B has n rows; stage with R = 256 bound but n-row layout.
        {
            const int kgroups = kc / 8, rgroups = g.n / 8;
            if (!g.b_mn) {
                for (int v = threadIdx.x; v < g.n * kgroups; v += blockDim.x) {
                    const int r = v / kgroups, kg = v % kgroups;
                    const int64_t kk = k0 + 8 * kg;
                    uint4 val = make_uint4(0u, 0u, 0u, 0u);
                    if (kk < k_end) val = *reinterpret_cast<const uint4 *>(g.b + (int64_t)r * g.ldb + kk);
                    *reinterpret_cast<uint4 *>(sb + (kg * rgroups + r / 8) * 128 + (r % 8) * 16) = val;
                }
            } else {
                for (int v = threadIdx.x; v < kc * rgroups; v += blockDim.x) {
                    const int k = v / rgroups, rg = v % rgroups;
                    const int64_t kk = k0 + k;
                    uint4 val = make_uint4(0u, 0u, 0u, 0u);
                    if (kk < k_end) val = *reinterpret_cast<const uint4 *>(g.b + kk * g.ldb + 8 * rg);
                    *reinterpret_cast<uint4 *>(sb + ((k / 8) * rgroups + rg) * 128 + (k % 8) * 16) = val;
                }
            }
        }
        // Generic-proxy stores must be visible to the tensor core's reads.
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0 && !failed) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a_addr = smem_u32(sa), b_addr = smem_u32(sb);
            for (int s = 0; s < kc / 16; ++s) {
                const uint64_t da = smem_desc(a_addr + 2 * s * lbo_a, lbo_a, 128);
                const uint64_t db = smem_desc(b_addr + 2 * s * lbo_b, lbo_b, 128);
                const uint32_t accumulate = (any || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&mma_bar))
                         : "memory");
        }
        any = true;
        // Everyone waits for the chunk's MMAs before the buffers are reused.
        if (!mbar_wait(smem_u32(&mma_bar), phase, g.error)) failed = 1;
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        __syncthreads();
    }
    // Epilogue: warp w owns rows 32 w .. 32 w + 31 (tensor-memory lanes).
    const int64_t row = m0 + 32 * warp + lane;
    float *out_f32 = g.out_f32 ? g.out_f32 + (int64_t)blockIdx.y * g.m * g.ldo : nullptr;
    if (any && !failed) {
        for (int c0 = 0; c0 < g.n; c0 += 16) {
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < g.m) {
                float v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    float x = __uint_as_float(r[j]);
                    if (g.bias) x += g.bias[c0 + j];
                    if (g.relu) x = fmaxf(x, 0.0f);
                    if (g.mask && !(__bfloat162float(g.mask[row * g.ld_mask + c0 + j]) > 0.0f)) x = 0.0f;
                    if (g.residual) x += g.residual[row * g.ld_res + c0 + j];
                    v[j] = x;
                }
                if (out_f32) {
                    float4 *o = reinterpret_cast<float4 *>(out_f32 + row * g.ldo + c0);
#pragma unroll
                    for (int j = 0; j < 4; ++j) o[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
                }
                if (g.out_bf16) {
                    __nv_bfloat162 h[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) h[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
                    uint4 *o = reinterpret_cast<uint4 *>(g.out_bf16 + row * g.ldo_bf16 + c0);
                    o[0] = *reinterpret_cast<uint4 *>(&h[0]);
                    o[1] = *reinterpret_cast<uint4 *>(&h[4]);
                }
            }
        }
    } else if (!any && row < g.m) {
        // Empty contraction range: zeros (plus bias).
        for (int c = 0; c < g.n; ++c) {
            float x = g.bias ? g.bias[c] : 0.0f;
            if (g.relu) x = fmaxf(x, 0.0f);
            if (out_f32) out_f32[row * g.ldo + c] = x;
            if (g.out_bf16) g.out_bf16[row * g.ldo_bf16 + c] = __float2bfloat16_rn(x);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols));
}

}  // namespace tgl
