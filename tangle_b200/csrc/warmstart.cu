// warmstart.cu -- kernels of the learned warm start: the tensor-core matrix
// product (umma_gemm.cuh) behind a C ABI entry.
#include <cuda_runtime.h>

#include <string>

#include <cuda.h>

#include <algorithm>
#include <cstdlib>
#include <mutex>

#include "../../include/tangle_cuda.h"
#include "umma_gemm.cuh"
#include "umma_gemm_tma.cuh"

namespace tgl {
void set_last_error(const std::string &message);
}

namespace {

int gemm_error(int code, const std::string &message) {
    tgl::set_last_error(message);
    return code;
}

// cuTensorMapEncodeTiled through the runtime's driver entry points (the
// library does not link libcuda itself); null when the driver lacks it.
using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_tiled() {
    static std::once_flag once;
    static EncodeTiled fn = nullptr;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    return fn;
}

// A K-major bf16 operand of `rows` rows and `k` columns (leading dimension
// `ld` elements) as a 2-D tensor map with boxes of 64 contraction elements
// (128 bytes) by `box_rows` rows in the 128-byte swizzle: each box is one
// contraction chunk in the canonical K-major SWIZZLE_128B layout.
// Out-of-range elements read as zero.
bool kmajor_map(CUtensorMap *map, const void *base, int64_t rows, int64_t k, int64_t ld, int box_rows) {
    EncodeTiled encode = encode_tiled();
    if (!encode) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * 2u};
    const cuuint32_t box[2] = {(cuuint32_t)tgl::GEMM_KC, (cuuint32_t)box_rows};
    const cuuint32_t element_strides[2] = {1u, 1u};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box,
                  element_strides, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The persistent TMA kernel for products whose operands are both K-major and
// whose contraction is not split; 0 when it ran, 1 when this product or the
// driver calls for the staged kernel instead, or an error code.
int gemm_tma(const tgl_gemm *p, const tgl::GemmArgs &g, cudaStream_t stream) {
    if (p->a_mn || p->b_mn || p->k_split > 0 || p->k <= 0 || std::getenv("TGL_GEMM_STAGED")) return 1;
    if (p->m > 0x7FFFFF80 || p->k > 0x7FFFFFF0) return 1;  // TMA coordinates are 32-bit
    CUtensorMap map_a, map_b;
    if (!kmajor_map(&map_a, p->a, p->m, p->k, p->lda, tgl::GEMM_BM) ||
        !kmajor_map(&map_b, p->b, p->n, p->k, p->ldb, p->n))
        return 1;
    const size_t smem = tgl::tma_smem_bytes(p->n);
    static std::once_flag once;
    static int sms = 0;
    std::call_once(once, [] {
        int device = 0;
        cudaGetDevice(&device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cudaFuncSetAttribute(tgl::umma_gemm_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tgl::tma_smem_bytes(256));
    });
    int cols = 32;
    while (cols < p->n) cols <<= 1;
    const int by_smem = (int)((220u * 1024u) / smem), by_tmem = 512 / (2 * cols);
    const int per_sm = std::max(1, std::min(by_smem, by_tmem));
    const int64_t tiles = ((int64_t)p->m + tgl::GEMM_BM - 1) / tgl::GEMM_BM;
    const int blocks = (int)std::min<int64_t>(tiles, (int64_t)std::max(sms, 1) * per_sm);
    tgl::umma_gemm_tma_kernel<<<blocks, tgl::TMA_GEMM_THREADS, smem, stream>>>(map_a, map_b, g);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return gemm_error(TGL_ERR_CUDA, std::string("tgl_gemm_bf16: ") + cudaGetErrorString(e));
    return 0;
}

}  // namespace

extern "C" int tgl_gemm_bf16(const tgl_gemm *p, void *stream) {
    if (!p || !p->a || !p->b || (!p->out_f32 && !p->out_bf16))
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: null argument");
    if (p->n < 16 || p->n > 256 || p->n % 16 || p->m < 0 || p->k < 0)
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: n must be a multiple of 16 in [16, 256]");
    if (((!p->a_mn || !p->b_mn) && p->k % 8) || (p->a_mn && p->lda % 8) || (p->b_mn && p->ldb % 8) ||
        (!p->a_mn && p->lda % 8) || (!p->b_mn && p->ldb % 8))
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: leading dimensions (and K with a K-major operand) "
                                           "must be multiples of 8 elements");
    if ((p->a_mn ? p->lda < p->m : p->lda < p->k) || (p->b_mn ? p->ldb < p->n : p->ldb < p->k) ||
        (p->out_f32 && p->ldo < p->n) || (p->out_bf16 && p->ldo_bf16 < p->n))
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: a leading dimension is shorter than its rows");
    if ((reinterpret_cast<uintptr_t>(p->a) | reinterpret_cast<uintptr_t>(p->b)) & 15)
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: operands must be 16-byte aligned");
    if (p->out_f32 && (p->ldo % 4 || (reinterpret_cast<uintptr_t>(p->out_f32) & 15)))
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: f32 output must be 16-byte aligned with ldo % 4 == 0");
    if (p->out_bf16 && (p->ldo_bf16 % 8 || (reinterpret_cast<uintptr_t>(p->out_bf16) & 15)))
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: bf16 output must be 16-byte aligned with ldo % 8 == 0");
    const int64_t k_split = p->k_split > 0 ? p->k_split : (p->k > 0 ? p->k : 1);
    if ((p->mask && p->ld_mask < p->n) || (p->residual && p->ld_res < p->n))
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: mask or residual rows are shorter than n");
    if (p->k_split > 0 && (p->k_split % 64 || p->bias || p->relu || p->out_bf16 || p->mask || p->residual))
        return gemm_error(TGL_ERR_INVALID, "tgl_gemm_bf16: split K needs k_split % 64 == 0 and a plain f32 output");
    if (p->m == 0) return 0;
    tgl::GemmArgs g{};
    g.a = reinterpret_cast<const __nv_bfloat16 *>(p->a);
    g.b = reinterpret_cast<const __nv_bfloat16 *>(p->b);
    g.lda = p->lda;
    g.ldb = p->ldb;
    g.m = p->m;
    g.n = p->n;
    g.k = p->k;
    g.a_mn = p->a_mn ? 1 : 0;
    g.b_mn = p->b_mn ? 1 : 0;
    g.k_split = k_split;
    g.bias = p->bias;
    g.relu = p->relu ? 1 : 0;
    g.mask = reinterpret_cast<const __nv_bfloat16 *>(p->mask);
    g.ld_mask = p->ld_mask;
    g.residual = p->residual;
    g.ld_res = p->ld_res;
    g.out_f32 = p->out_f32;
    g.ldo = p->ldo;
    g.out_bf16 = reinterpret_cast<__nv_bfloat16 *>(p->out_bf16);
    g.ldo_bf16 = p->ldo_bf16;
    g.error = p->error;
    const int64_t splits = p->k > 0 ? (p->k + k_split - 1) / k_split : 1;
    if (splits > 65535) return gemm_error(TGL_ERR_UNSUPPORTED, "tgl_gemm_bf16: too many K splits");
    if (splits == 1) {
        const int rc = gemm_tma(p, g, static_cast<cudaStream_t>(stream));
        if (rc != 1) return rc;
    }
    const size_t smem = (size_t)tgl::GEMM_BM * tgl::GEMM_KC * 2 + (size_t)p->n * tgl::GEMM_KC * 2;
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(tgl::umma_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)((size_t)tgl::GEMM_BM * tgl::GEMM_KC * 2 + 256 * tgl::GEMM_KC * 2));
        configured = true;
    }
    dim3 grid((unsigned)((p->m + tgl::GEMM_BM - 1) / tgl::GEMM_BM), (unsigned)splits);
    tgl::umma_gemm_kernel<<<grid, tgl::GEMM_THREADS, smem, static_cast<cudaStream_t>(stream)>>>(g);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return gemm_error(TGL_ERR_CUDA, std::string("tgl_gemm_bf16: ") + cudaGetErrorString(e));
    return 0;
}

// ---------------------------------------------------------------- contact graph

#include "common.cuh"
#include "warmstart.cuh"

namespace tgl {
namespace {

constexpr uint32_t WFULL = 0xFFFFFFFFu;

// Closest points of segments a and b (b shifted to its minimum image):
// parameters s on a, t on b, the distance, and the offset from a's point to
// b's. The closed form of find_segment_corrections' solve, without its
// parallel-axis end-point refinement (features need no bit parity).
__device__ inline void pair_geometry(const WorldDev &w, uint32_t a, uint32_t b, float &s, float &t, float &distance,
                                     float3 &offset) {
    const float4 a0 = w.geom[2 * (size_t)a], a1 = w.geom[2 * (size_t)a + 1];
    const float4 b0 = w.geom[2 * (size_t)b], b1 = w.geom[2 * (size_t)b + 1];
    float p2x = b0.x, p2y = b0.y, p2z = b0.z, q2x = b1.x, q2y = b1.y, q2z = b1.z;
    minimum_image(a0.x, a0.y, a0.z, a1.x, a1.y, a1.z, p2x, p2y, p2z, q2x, q2y, q2z, w.grid);
    const float d1x = a1.x - a0.x, d1y = a1.y - a0.y, d1z = a1.z - a0.z;
    const float d2x = q2x - p2x, d2y = q2y - p2y, d2z = q2z - p2z;
    const float rx = a0.x - p2x, ry = a0.y - p2y, rz = a0.z - p2z;
    const float A = d1x * d1x + d1y * d1y + d1z * d1z, Eq = d2x * d2x + d2y * d2y + d2z * d2z;
    const float F = d2x * rx + d2y * ry + d2z * rz;
    s = 0.0f;
    t = 0.0f;
    if (A <= 1.0e-20f && Eq > 1.0e-20f) {
        t = clampf(F / Eq, 0.0f, 1.0f);
    } else if (A > 1.0e-20f) {
        const float C = d1x * rx + d1y * ry + d1z * rz;
        if (Eq <= 1.0e-20f) {
            s = clampf(-C / A, 0.0f, 1.0f);
        } else {
            const float B = d1x * d2x + d1y * d2y + d1z * d2z;
            const float den = A * Eq - B * B;
            if (fabsf(den) > 1.0e-6f * A * Eq) s = clampf((B * F - C * Eq) / den, 0.0f, 1.0f);
            const float proj = (B * s + F) / Eq;
            if (proj < 0.0f) {
                s = clampf(-C / A, 0.0f, 1.0f);
            } else if (proj > 1.0f) {
                t = 1.0f;
                s = clampf((B - C) / A, 0.0f, 1.0f);
            } else {
                t = proj;
            }
        }
    }
    offset = make_float3((p2x + d2x * t) - (a0.x + d1x * s), (p2y + d2y * t) - (a0.y + d1y * s),
                         (p2z + d2z * t) - (a0.z + d1z * s));
    distance = sqrtf(offset.x * offset.x + offset.y * offset.y + offset.z * offset.z);
}

// One warp per segment a walks its Verlet list; pairs (a, b) with b > a and
// a gap below `cutoff` become edges.
__device__ inline bool keep_pair(const WorldDev &w, uint32_t a, uint32_t b, float cutoff, float &s, float &t,
                                 float &distance, float3 &offset) {
    pair_geometry(w, a, b, s, t, distance, offset);
    const float gap = distance - w.geom[2 * (size_t)a].w - w.geom[2 * (size_t)b].w;
    return gap <= cutoff;
}

__global__ void graph_count_kernel(WorldDev w, GraphBuffers g, float cutoff) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t a = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); a < w.S; a += warps) {
        const uint32_t count = segment_on(w, a) ? w.nbr_count[a] : 0u;
        uint32_t kept = 0;
        if (count <= w.block) {
            for (uint32_t i0 = 0; i0 < count; i0 += 32) {
                bool keep = false;
                if (i0 + lane < count) {
                    const uint32_t b = w.nbr_list[(size_t)a * w.block + i0 + lane];
                    float s, t, dist;
                    float3 off;
                    if (b > a && in_focus(w, g, a, b) && keep_pair(w, a, b, cutoff, s, t, dist, off)) {
                        keep = true;
                        atomicAdd(&g.in_count[b], 1u);
                    }
                }
                kept += __popc(__ballot_sync(WFULL, keep));
            }
        }
        if (lane == 0) {
            g.fwd_count[a] = kept;
            g.fill[a] = 0;
        }
    }
}

// Exclusive scan of fwd_count + in_count into offsets[0..S], S + 1 entries;
// three phases over blocks of 1024.
__global__ void __launch_bounds__(1024) graph_scan_blocks_kernel(WorldDev w, GraphBuffers g) {
    __shared__ int32_t warp_sums[32];
    const uint32_t i = blockIdx.x * 1024 + threadIdx.x;
    int32_t v = i < w.S ? (int32_t)(g.fwd_count[i] + g.in_count[i]) : 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int32_t t = __shfl_up_sync(WFULL, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int32_t x = warp_sums[lane], xi = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int32_t t = __shfl_up_sync(WFULL, xi, o);
            if (lane >= o) xi += t;
        }
        warp_sums[lane] = xi - x;
        if (lane == 31) g.block_sums[blockIdx.x] = xi;
    }
    __syncthreads();
    if (i < w.S) g.offsets[i] = incl - v + warp_sums[warp];
}

__global__ void graph_scan_sums_kernel(GraphBuffers g, int blocks) {
    if (threadIdx.x != 0) return;
    int32_t total = 0;
    for (int b = 0; b < blocks; ++b) {
        const int32_t x = g.block_sums[b];
        g.block_sums[b] = total;
        total += x;
    }
    g.block_sums[blocks] = total;
}

__global__ void graph_scan_add_kernel(WorldDev w, GraphBuffers g, int blocks) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < w.S) g.offsets[i] += g.block_sums[i / 1024];
    if (i == 0) g.offsets[w.S] = g.block_sums[blocks];
}

__device__ inline void write_edge(const GraphBuffers &g, int64_t e, int32_t dst, int32_t src, float s, float t,
                                  float depth, float3 off, float diameter) {
    g.dst[e] = dst;
    g.src[e] = src;
    g.s[e] = s;
    g.t[e] = t;
    g.depth[e] = depth;
    const float inv = 1.0f / diameter;
    __nv_bfloat16 *f = g.edge_features + e * MP_EDGE_FEATURES;
    f[0] = __float2bfloat16_rn(off.x * inv);
    f[1] = __float2bfloat16_rn(off.y * inv);
    f[2] = __float2bfloat16_rn(off.z * inv);
    f[3] = __float2bfloat16_rn(depth * inv);
    f[4] = __float2bfloat16_rn(s);
    f[5] = __float2bfloat16_rn(t);
#pragma unroll
    for (int j = 6; j < MP_EDGE_FEATURES; ++j) f[j] = __float2bfloat16_rn(0.0f);
}

// Edges of pair (a, b), a < b: the forward edge (dst a, src b) at a's
// forward slot (ascending b), the reverse edge (dst b, src a) at the next
// free incoming slot of b (sorted by source afterwards).
__global__ void graph_fill_kernel(WorldDev w, GraphBuffers g, float cutoff) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t a = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); a < w.S; a += warps) {
        const uint32_t count = segment_on(w, a) ? w.nbr_count[a] : 0u;
        if (count > w.block) continue;
        const int64_t base = (int64_t)g.offsets[a] + g.in_count[a];
        uint32_t rank = 0;
        for (uint32_t i0 = 0; i0 < count; i0 += 32) {
            bool keep = false;
            uint32_t b = 0;
            float s = 0.0f, t = 0.0f, dist = 0.0f;
            float3 off = make_float3(0.0f, 0.0f, 0.0f);
            if (i0 + lane < count) {
                b = w.nbr_list[(size_t)a * w.block + i0 + lane];
                keep = b > a && in_focus(w, g, a, b) && keep_pair(w, a, b, cutoff, s, t, dist, off);
            }
            const uint32_t ballot = __ballot_sync(WFULL, keep);
            if (keep) {
                const int64_t e = base + rank + __popc(ballot & ((1u << lane) - 1u));
                const int64_t r = (int64_t)g.offsets[b] + atomicAdd(&g.fill[b], 1u);
                const float ra = w.geom[2 * (size_t)a].w, rb = w.geom[2 * (size_t)b].w;
                const float depth = fmaxf(ra + rb - dist, 0.0f);
                write_edge(g, e, (int32_t)a, (int32_t)b, s, t, depth, off, 2.0f * ra);
                write_edge(g, r, (int32_t)b, (int32_t)a, t, s, depth, make_float3(-off.x, -off.y, -off.z), 2.0f * rb);
                g.twin[e] = (int32_t)r;
                g.twin[r] = (int32_t)e;
            }
            rank += __popc(ballot);
        }
    }
}

// Sort each segment's incoming edges (sources below it) by source, carrying
// every per-edge record; the twins of moved edges are fixed afterwards.
__global__ void graph_sort_kernel(WorldDev w, GraphBuffers g) {
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < w.S; b += gridDim.x * blockDim.x) {
        const int64_t lo = g.offsets[b], n = g.in_count[b];
        for (int64_t i = 1; i < n; ++i) {
            for (int64_t j = i; j > 0 && g.src[lo + j] < g.src[lo + j - 1]; --j) {
                const int64_t x = lo + j, y = lo + j - 1;
                int32_t ti = g.src[x]; g.src[x] = g.src[y]; g.src[y] = ti;
                ti = g.twin[x]; g.twin[x] = g.twin[y]; g.twin[y] = ti;
                float tf = g.s[x]; g.s[x] = g.s[y]; g.s[y] = tf;
                tf = g.t[x]; g.t[x] = g.t[y]; g.t[y] = tf;
                tf = g.depth[x]; g.depth[x] = g.depth[y]; g.depth[y] = tf;
                uint4 *fx = reinterpret_cast<uint4 *>(g.edge_features + x * MP_EDGE_FEATURES);
                uint4 *fy = reinterpret_cast<uint4 *>(g.edge_features + y * MP_EDGE_FEATURES);
                const uint4 a0 = fx[0], a1 = fx[1];
                fx[0] = fy[0];
                fx[1] = fy[1];
                fy[0] = a0;
                fy[1] = a1;
            }
        }
    }
}

__global__ void graph_twin_kernel(WorldDev w, GraphBuffers g) {
    const int64_t E = g.offsets[w.S];
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x)
        if (g.src[e] < g.dst[e]) g.twin[g.twin[e]] = (int32_t)e;
}

// Node features (16 per vertex, 7 used): unit tangent (3), discrete
// curvature x d, rest curvature x d, d / 10 um, and the overlap depth / d of
// the vertex's segments, split by the closest-point parameters.
__global__ void node_features_kernel(WorldDev w, GraphBuffers g, MpGraph graph) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < w.V; v += gridDim.x * blockDim.x) {
        const int4 l = w.links[v];
        const float4 x = w.pos[v];
        const float4 p = l.x >= 0 ? w.pos[l.x] : x, q = l.y >= 0 ? w.pos[l.y] : x;
        float tx = q.x - p.x, ty = q.y - p.y, tz = q.z - p.z;
        const float tl = sqrtf(tx * tx + ty * ty + tz * tz);
        if (tl > 0.0f) {
            tx /= tl;
            ty /= tl;
            tz /= tl;
        }
        const float diameter = 2.0f * w.vtx_static[v].w;
        float curvature = 0.0f;
        if (l.x >= 0 && l.y >= 0) {
            const float ux = x.x - p.x, uy = x.y - p.y, uz = x.z - p.z;
            const float vx = q.x - x.x, vy = q.y - x.y, vz = q.z - x.z;
            const float lu = sqrtf(ux * ux + uy * uy + uz * uz), lv = sqrtf(vx * vx + vy * vy + vz * vz);
            if (lu > 1.0e-12f && lv > 1.0e-12f) {
                const float c = clampf((ux * vx + uy * vy + uz * vz) / (lu * lv), -1.0f, 1.0f);
                curvature = 2.0f * sqrtf(0.5f * (1.0f - c)) / (0.5f * (lu + lv));
            }
        }
        // Overlap depth, and the push: the depth-weighted unit normals away
        // from the contacts of the vertex's two segments, by its share.
        float overlap = 0.0f, px = 0.0f, py = 0.0f, pz = 0.0f;
        for (int side = 0; side < 2; ++side) {
            const int32_t seg = side == 0 ? l.z : l.w;
            if (seg < 0) continue;
            for (int32_t e = graph.offsets[seg]; e < graph.offsets[seg + 1]; ++e) {
                const float share = side == 0 ? g.s[e] : 1.0f - g.s[e];
                const float depth = g.depth[e];
                overlap += depth * share;
                if (depth > 0.0f) {
                    const __nv_bfloat16 *f = g.edge_features + (int64_t)e * MP_EDGE_FEATURES;
                    const float ox = __bfloat162float(f[0]), oy = __bfloat162float(f[1]), oz = __bfloat162float(f[2]);
                    const float on = sqrtf(ox * ox + oy * oy + oz * oz);
                    if (on > 0.0f) {
                        const float k = share * depth / (on * diameter);
                        px -= k * ox;
                        py -= k * oy;
                        pz -= k * oz;
                    }
                }
            }
        }
        __nv_bfloat16 *f = g.node_features + (size_t)v * MP_NODE_FEATURES;
        f[0] = __float2bfloat16_rn(tx);
        f[1] = __float2bfloat16_rn(ty);
        f[2] = __float2bfloat16_rn(tz);
        f[3] = __float2bfloat16_rn(curvature * diameter);
        f[4] = __float2bfloat16_rn(w.rest_curvature[v] * diameter);
        f[5] = __float2bfloat16_rn(diameter / 10.0e-6f);
        f[6] = __float2bfloat16_rn(overlap / diameter);
        f[7] = __float2bfloat16_rn(px);
        f[8] = __float2bfloat16_rn(py);
        f[9] = __float2bfloat16_rn(pz);
#pragma unroll
        for (int j = 10; j < MP_NODE_FEATURES; ++j) f[j] = __float2bfloat16_rn(0.0f);
    }
}

__global__ void displace_kernel(WorldDev w, const float *dx, int64_t ld, float scale, int in_diameters,
                                float max_step) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < w.V; v += gridDim.x * blockDim.x) {
        if (w.pinned[v] || !vertex_on(w, v)) continue;  // frozen (inactive) fibers stay put
        const float k0 = in_diameters ? scale * 2.0f * w.vtx_static[v].w : scale;
        float mx = k0 * dx[v * ld], my = k0 * dx[v * ld + 1], mz = k0 * dx[v * ld + 2];
        const float m = sqrtf(mx * mx + my * my + mz * mz);
        if (m > max_step && m > 0.0f) {
            const float k = max_step / m;
            mx *= k;
            my *= k;
            mz *= k;
        }
        float4 p = w.pos[v];
        const float extent = w.vtx_static[v].w;
        p.x = p.x + mx;
        if (!w.grid.periodic[0]) p.x = clampf(p.x, w.grid.lower[0] + extent, w.grid.upper[0] - extent);
        p.y = p.y + my;
        if (!w.grid.periodic[1]) p.y = clampf(p.y, w.grid.lower[1] + extent, w.grid.upper[1] - extent);
        p.z = p.z + mz;
        if (!w.grid.periodic[2]) p.z = clampf(p.z, w.grid.lower[2] + extent, w.grid.upper[2] - extent);
        w.pos[v] = p;
    }
}

__global__ void geometry_kernel(WorldDev w) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < w.S; s += gridDim.x * blockDim.x) {
        const uint32_t v0 = w.seg_v0[s];
        const float4 a = w.pos[v0], b = w.pos[v0 + 1];
        const float dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
        w.geom[2 * (size_t)s] = make_float4(a.x, a.y, a.z, w.seg_static[s].x);
        w.geom[2 * (size_t)s + 1] = make_float4(b.x, b.y, b.z, 0.5f * sqrtf(dx * dx + dy * dy + dz * dz));
    }
}

// Max of corr[].w (the last contact pass's per-segment penetration) and of
// the curvature ratio, as u32 bits of non-negative floats.
__global__ void residual_kernel(WorldDev w, unsigned int *out2, float *block_sums) {
    __shared__ float warp_sums[8];
    unsigned int pen = 0, ratio = 0;
    float sum = 0.0f;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < w.S; s += gridDim.x * blockDim.x) {
        const float p = segment_on(w, s) ? fmaxf(w.corr[2 * (size_t)s].w, 0.0f) : 0.0f;
        pen = max(pen, __float_as_uint(p));
        sum += p / (2.0f * w.seg_static[s].x);
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(WFULL, sum, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        float b = 0.0f;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) b += warp_sums[k];
        block_sums[blockIdx.x] = b;
    }
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < w.V; v += gridDim.x * blockDim.x) {
        const int4 l = w.links[v];
        const float maximum = w.vtx_static[v].x;
        if (l.x < 0 || l.y < 0 || !(maximum > 0.0f)) continue;
        const float4 a = w.pos[l.x], c = w.pos[v], b = w.pos[l.y];
        const float ax = c.x - a.x, ay = c.y - a.y, az = c.z - a.z;
        const float bx = b.x - c.x, by = b.y - c.y, bz = b.z - c.z;
        const float la = sqrtf(ax * ax + ay * ay + az * az), lb = sqrtf(bx * bx + by * by + bz * bz);
        if (la > 1.0e-7f && lb > 1.0e-7f) {
            const float cosine = clampf((ax * bx + ay * by + az * bz) / (la * lb), -1.0f, 1.0f);
            const float curvature = 2.0f * sqrtf(0.5f * (1.0f - cosine)) / (0.5f * (la + lb));
            ratio = max(ratio, __float_as_uint(fmaxf(curvature / maximum, 0.0f)));
        }
    }
    pen = __reduce_max_sync(WFULL, pen);
    ratio = __reduce_max_sync(WFULL, ratio);
    if ((threadIdx.x & 31) == 0) {
        if (pen) atomicMax(&out2[0], pen);
        if (ratio) atomicMax(&out2[1], ratio);
    }
}

int blocks_for(int64_t n, int threads, int cap) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (int)b;
}

}  // namespace

void launch_graph_count(const WorldDev &w, const GraphBuffers &g, float cutoff, cudaStream_t st) {
    cudaMemsetAsync(g.in_count, 0, (size_t)w.S * sizeof(uint32_t), st);
    graph_count_kernel<<<blocks_for(w.S, 8, 148 * 32), 256, 0, st>>>(w, g, cutoff);
}

int launch_graph_offsets(const WorldDev &w, const GraphBuffers &g, cudaStream_t st) {
    const int blocks = (int)((w.S + 1023) / 1024);
    graph_scan_blocks_kernel<<<blocks, 1024, 0, st>>>(w, g);
    graph_scan_sums_kernel<<<1, 32, 0, st>>>(g, blocks);
    graph_scan_add_kernel<<<blocks_for(w.S, 256, 1 << 20), 256, 0, st>>>(w, g, blocks);
    return 3;
}

void launch_graph_fill(const WorldDev &w, const GraphBuffers &g, float cutoff, cudaStream_t st) {
    graph_fill_kernel<<<blocks_for(w.S, 8, 148 * 32), 256, 0, st>>>(w, g, cutoff);
    graph_sort_kernel<<<blocks_for(w.S, 256, 1 << 20), 256, 0, st>>>(w, g);
    graph_twin_kernel<<<148 * 8, 256, 0, st>>>(w, g);
}

void launch_node_features(const WorldDev &w, const GraphBuffers &g, const MpGraph &graph, cudaStream_t st) {
    node_features_kernel<<<blocks_for(w.V, 256, 1 << 20), 256, 0, st>>>(w, g, graph);
}

void launch_displace(const WorldDev &w, const float *dx, int64_t ld, float scale, int in_diameters, float max_step,
                     cudaStream_t st) {
    displace_kernel<<<blocks_for(w.V, 256, 1 << 20), 256, 0, st>>>(w, dx, ld, scale, in_diameters, max_step);
    geometry_kernel<<<blocks_for(w.S, 256, 1 << 20), 256, 0, st>>>(w);
}

// Sums the per-block partials in block order (a fixed order: repeatable).
__global__ void residual_finish_kernel(const float *block_sums, int blocks, float *total) {
    if (threadIdx.x != 0) return;
    float sum = 0.0f;
    for (int b = 0; b < blocks; ++b) sum += block_sums[b];
    *total = sum;
}

void launch_residual(const WorldDev &w, float *out3, cudaStream_t st) {
    cudaMemsetAsync(out3, 0, 3 * sizeof(float), st);
    residual_kernel<<<RESIDUAL_BLOCKS, 256, 0, st>>>(w, reinterpret_cast<unsigned int *>(out3), out3 + 3);
    residual_finish_kernel<<<1, 32, 0, st>>>(out3 + 3, RESIDUAL_BLOCKS, out3 + 2);
}

}  // namespace tgl

// ---------------------------------------------------------------- message passing

namespace tgl {
namespace {

constexpr int MP_ROWS_PER_CHUNK = 4096;  // rows per partial in column sums

// One warp per edge: lanes cover the 64 embedding columns two at a time.
__global__ void edge_inputs_kernel(MpGraph g, const float *h, __nv_bfloat16 *x, int64_t ld) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t e = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); e < g.E; e += warps) {
        const int32_t v0 = g.seg_v0[g.src[e]];
        const float t = g.t[e];
        const float2 a = reinterpret_cast<const float2 *>(h + (int64_t)v0 * MP_HIDDEN)[lane];
        const float2 b = reinterpret_cast<const float2 *>(h + (int64_t)(v0 + 1) * MP_HIDDEN)[lane];
        reinterpret_cast<__nv_bfloat162 *>(x + e * ld)[lane] =
            __floats2bfloat162_rn((1.0f - t) * a.x + t * b.x, (1.0f - t) * a.y + t * b.y);
    }
}

// Total share of vertex v in the edges into its two segments (the messages'
// weights), at least 1 when used as a divisor.
__device__ inline float vertex_weight(const MpGraph &g, int4 l) {
    float w = 0.0f;
    if (l.z >= 0)
        for (int32_t e = g.offsets[l.z]; e < g.offsets[l.z + 1]; ++e) w += g.s[e];
    if (l.w >= 0)
        for (int32_t e = g.offsets[l.w]; e < g.offsets[l.w + 1]; ++e) w += 1.0f - g.s[e];
    return w;
}

// One warp per vertex: [h, the weighted mean of the messages into its two
// segments (weights: its share, s or 1 - s), mean of the fiber neighbors' h].
__global__ void node_inputs_kernel(MpGraph g, const float *h, const float *m, __nv_bfloat16 *x) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t v = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); v < g.V; v += warps) {
        const int4 l = g.links[v];
        const float2 hv = reinterpret_cast<const float2 *>(h + v * MP_HIDDEN)[lane];
        float2 agg = make_float2(0.0f, 0.0f);
        if (l.z >= 0)
            for (int32_t e = g.offsets[l.z]; e < g.offsets[l.z + 1]; ++e) {
                const float w = g.s[e];
                const float2 me = reinterpret_cast<const float2 *>(m + (int64_t)e * MP_HIDDEN)[lane];
                agg.x += w * me.x;
                agg.y += w * me.y;
            }
        if (l.w >= 0)
            for (int32_t e = g.offsets[l.w]; e < g.offsets[l.w + 1]; ++e) {
                const float w = 1.0f - g.s[e];
                const float2 me = reinterpret_cast<const float2 *>(m + (int64_t)e * MP_HIDDEN)[lane];
                agg.x += w * me.x;
                agg.y += w * me.y;
            }
        const float norm = 1.0f / fmaxf(vertex_weight(g, l), 1.0f);
        agg.x *= norm;
        agg.y *= norm;
        float2 nb = make_float2(0.0f, 0.0f);
        const int count = (l.x >= 0) + (l.y >= 0);
        if (l.x >= 0) {
            const float2 p = reinterpret_cast<const float2 *>(h + (int64_t)l.x * MP_HIDDEN)[lane];
            nb.x += p.x;
            nb.y += p.y;
        }
        if (l.y >= 0) {
            const float2 q = reinterpret_cast<const float2 *>(h + (int64_t)l.y * MP_HIDDEN)[lane];
            nb.x += q.x;
            nb.y += q.y;
        }
        if (count) {
            nb.x /= (float)count;
            nb.y /= (float)count;
        }
        __nv_bfloat162 *row = reinterpret_cast<__nv_bfloat162 *>(x + v * 3 * MP_HIDDEN);
        row[lane] = __floats2bfloat162_rn(hv.x, hv.y);
        row[32 + lane] = __floats2bfloat162_rn(agg.x, agg.y);
        row[64 + lane] = __floats2bfloat162_rn(nb.x, nb.y);
    }
}

// dH[v] += dX[v, 0:64] + sum over fiber neighbors u of dX[u, 128:192] / count(u);
// dM[e] = (1 - s_e) dX[first vertex of dst, 64:128] + s_e dX[second vertex, 64:128].
__global__ void node_inputs_backward_kernel(MpGraph g, const float *dx, float *dh, __nv_bfloat16 *dm, float *dm32) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t v = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); v < g.V; v += warps) {
        const int4 l = g.links[v];
        float2 acc = reinterpret_cast<const float2 *>(dx + v * 3 * MP_HIDDEN)[lane];
        for (int side = 0; side < 2; ++side) {
            const int32_t u = side == 0 ? l.x : l.y;
            if (u < 0) continue;
            const int4 lu = g.links[u];
            const float count = (float)((lu.x >= 0) + (lu.y >= 0));
            const float2 d = reinterpret_cast<const float2 *>(dx + (int64_t)u * 3 * MP_HIDDEN + 2 * MP_HIDDEN)[lane];
            acc.x += d.x / count;
            acc.y += d.y / count;
        }
        float2 *out = reinterpret_cast<float2 *>(dh + v * MP_HIDDEN) + lane;
        const float2 old = *out;
        *out = make_float2(old.x + acc.x, old.y + acc.y);
    }
    for (int64_t e = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); e < g.E; e += warps) {
        const int32_t v0 = g.seg_v0[g.dst[e]];
        const float s = g.s[e];
        const float wa = (1.0f - s) / fmaxf(vertex_weight(g, g.links[v0]), 1.0f);
        const float wb = s / fmaxf(vertex_weight(g, g.links[v0 + 1]), 1.0f);
        const float2 a = reinterpret_cast<const float2 *>(dx + (int64_t)v0 * 3 * MP_HIDDEN + MP_HIDDEN)[lane];
        const float2 b = reinterpret_cast<const float2 *>(dx + (int64_t)(v0 + 1) * 3 * MP_HIDDEN + MP_HIDDEN)[lane];
        const float2 d = make_float2(wa * a.x + wb * b.x, wa * a.y + wb * b.y);
        reinterpret_cast<__nv_bfloat162 *>(dm + e * MP_HIDDEN)[lane] = __floats2bfloat162_rn(d.x, d.y);
        if (dm32) reinterpret_cast<float2 *>(dm32 + e * MP_HIDDEN)[lane] = d;
    }
}

__global__ void convert_kernel(int64_t n, const float *src, __nv_bfloat16 *dst) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = __float2bfloat16_rn(src[i]);
}

// dH[u] += sum over edges e whose source segment holds u of its share
// ((1 - t_e) for the first vertex, t_e for the second) of dX_edge[e, 0:64];
// the edges with source c are the twins of the edges into c.
__global__ void edge_inputs_backward_kernel(MpGraph g, const float *dx, int64_t ld, float *dh) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t u = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); u < g.V; u += warps) {
        const int4 l = g.links[u];
        float2 acc = make_float2(0.0f, 0.0f);
        if (l.z >= 0)  // u is the second vertex of segment l.z
            for (int32_t f = g.offsets[l.z]; f < g.offsets[l.z + 1]; ++f) {
                const int32_t e = g.twin[f];
                const float w = g.t[e];
                const float2 d = reinterpret_cast<const float2 *>(dx + (int64_t)e * ld)[lane];
                acc.x += w * d.x;
                acc.y += w * d.y;
            }
        if (l.w >= 0)  // u is the first vertex of segment l.w
            for (int32_t f = g.offsets[l.w]; f < g.offsets[l.w + 1]; ++f) {
                const int32_t e = g.twin[f];
                const float w = 1.0f - g.t[e];
                const float2 d = reinterpret_cast<const float2 *>(dx + (int64_t)e * ld)[lane];
                acc.x += w * d.x;
                acc.y += w * d.y;
            }
        float2 *out = reinterpret_cast<float2 *>(dh + u * MP_HIDDEN) + lane;
        const float2 old = *out;
        *out = make_float2(old.x + acc.x, old.y + acc.y);
    }
}

// Column sums in two passes: partial[chunk][j] over MP_ROWS_PER_CHUNK rows,
// then the chunks in order.
__global__ void column_partials_kernel(const float *x, int64_t rows, int32_t n, int64_t ld, float *partial) {
    const int64_t chunk = blockIdx.y;
    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const int64_t r0 = chunk * MP_ROWS_PER_CHUNK;
        const int64_t r1 = r0 + MP_ROWS_PER_CHUNK < rows ? r0 + MP_ROWS_PER_CHUNK : rows;
        float sum = 0.0f;
        for (int64_t r = r0; r < r1; ++r) sum += x[r * ld + j];
        partial[chunk * n + j] = sum;
    }
}

__global__ void column_finish_kernel(const float *partial, int64_t chunks, int32_t n, float *out, int accumulate) {
    for (int32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        float sum = accumulate ? out[j] : 0.0f;
        for (int64_t c = 0; c < chunks; ++c) sum += partial[c * n + j];
        out[j] = sum;
    }
}

// Adam (Kingma & Ba 2015) with bias correction; also refreshes the bf16 copy.
__global__ void adam_kernel(int64_t n, float *w, const float *g, float *m, float *v, __nv_bfloat16 *wb, float lr,
                            float beta1, float beta2, float eps, float c1, float c2) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = beta1 * m[i] + (1.0f - beta1) * gi;
        const float vi = beta2 * v[i] + (1.0f - beta2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16_rn(wi);
    }
}

// Mean squared error over rows x cols; dy = 2 (y - target) / (rows cols),
// zero in the padding columns; the loss as per-block partials summed in order.
__global__ void mse_kernel(int64_t rows, const float *y, int64_t ld_y, const float *target, int32_t cols,
                           float *dy, int64_t ld_dy, __nv_bfloat16 *dyb, float *partial) {
    __shared__ float warp_sums[8];
    const float scale = 2.0f / ((float)rows * (float)cols);
    float sum = 0.0f;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < rows; r += (int64_t)gridDim.x * blockDim.x) {
        for (int64_t j = 0; j < ld_dy; ++j) {
            float d = 0.0f;
            if (j < cols) {
                const float diff = y[r * ld_y + j] - target[r * cols + j];
                sum += diff * diff;
                d = scale * diff;
            }
            if (dy) dy[r * ld_dy + j] = d;
            if (dyb) dyb[r * ld_dy + j] = __float2bfloat16_rn(d);
        }
    }
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(WFULL, sum, o);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
        float total = 0.0f;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) total += warp_sums[k];
        partial[blockIdx.x] = total;
    }
}

__global__ void mse_finish_kernel(const float *partial, int blocks, float inv_count, float *loss) {
    if (threadIdx.x != 0) return;
    float total = 0.0f;
    for (int b = 0; b < blocks; ++b) total += partial[b];
    *loss = total * inv_count;
}

int warps_grid(int64_t items) {
    int64_t b = (items + 7) / 8;
    if (b < 1) b = 1;
    if (b > 148 * 64) b = 148 * 64;
    return (int)b;
}

MpGraph view(const tgl_mp_graph *p) {
    MpGraph g;
    g.V = p->vertex_count;
    g.S = p->segment_count;
    g.E = p->edge_count;
    g.seg_v0 = p->seg_v0;
    g.links = reinterpret_cast<const int4 *>(p->links);
    g.offsets = p->offsets;
    g.dst = p->dst;
    g.src = p->src;
    g.twin = p->twin;
    g.s = p->s;
    g.t = p->t;
    return g;
}

int launched(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        tgl::set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
        return TGL_ERR_CUDA;
    }
    return 0;
}

bool bad_graph(const tgl_mp_graph *p) {
    return !p || !p->seg_v0 || !p->links || !p->offsets || (p->edge_count > 0 && (!p->dst || !p->src || !p->twin ||
                                                                                   !p->s || !p->t)) ||
           p->vertex_count < 0 || p->segment_count < 0 || p->edge_count < 0;
}

}  // namespace
}  // namespace tgl

using tgl::MP_HIDDEN;

extern "C" int tgl_mp_edge_inputs(const tgl_mp_graph *graph, const float *h, void *x_edge, int64_t ld_x, void *stream) {
    if (tgl::bad_graph(graph) || !h || !x_edge || ld_x < MP_HIDDEN || ld_x % 8)
        return gemm_error(TGL_ERR_INVALID, "tgl_mp_edge_inputs: bad arguments");
    if (graph->edge_count == 0) return 0;
    tgl::edge_inputs_kernel<<<tgl::warps_grid(graph->edge_count), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        tgl::view(graph), h, static_cast<__nv_bfloat16 *>(x_edge), ld_x);
    return tgl::launched("tgl_mp_edge_inputs");
}

extern "C" int tgl_mp_node_inputs(const tgl_mp_graph *graph, const float *h, const float *m, void *x_node,
                                  void *stream) {
    if (tgl::bad_graph(graph) || !h || !x_node || (graph->edge_count > 0 && !m))
        return gemm_error(TGL_ERR_INVALID, "tgl_mp_node_inputs: bad arguments");
    if (graph->vertex_count == 0) return 0;
    tgl::node_inputs_kernel<<<tgl::warps_grid(graph->vertex_count), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        tgl::view(graph), h, m, static_cast<__nv_bfloat16 *>(x_node));
    return tgl::launched("tgl_mp_node_inputs");
}

extern "C" int tgl_convert_bf16(int64_t n, const float *src, void *dst, void *stream) {
    if (n < 0 || !src || !dst) return gemm_error(TGL_ERR_INVALID, "tgl_convert_bf16: bad arguments");
    if (n == 0) return 0;
    tgl::convert_kernel<<<(int)((n + 255) / 256 < 8192 ? (n + 255) / 256 : 8192), 256, 0,
                          static_cast<cudaStream_t>(stream)>>>(n, src, static_cast<__nv_bfloat16 *>(dst));
    return tgl::launched("tgl_convert_bf16");
}

extern "C" int tgl_mp_node_inputs_backward(const tgl_mp_graph *graph, const float *dx_node, float *dh, void *dm,
                                           float *dm_f32, void *stream) {
    if (tgl::bad_graph(graph) || !dx_node || !dh || (graph->edge_count > 0 && !dm))
        return gemm_error(TGL_ERR_INVALID, "tgl_mp_node_inputs_backward: bad arguments");
    const int64_t items = graph->vertex_count > graph->edge_count ? graph->vertex_count : graph->edge_count;
    if (items == 0) return 0;
    tgl::node_inputs_backward_kernel<<<tgl::warps_grid(items), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        tgl::view(graph), dx_node, dh, static_cast<__nv_bfloat16 *>(dm), dm_f32);
    return tgl::launched("tgl_mp_node_inputs_backward");
}

extern "C" int tgl_mp_edge_inputs_backward(const tgl_mp_graph *graph, const float *dx_edge, int64_t ld_dx, float *dh,
                                           void *stream) {
    if (tgl::bad_graph(graph) || !dh || (graph->edge_count > 0 && !dx_edge) || ld_dx < MP_HIDDEN || ld_dx % 2)
        return gemm_error(TGL_ERR_INVALID, "tgl_mp_edge_inputs_backward: bad arguments");
    if (graph->vertex_count == 0) return 0;
    tgl::edge_inputs_backward_kernel<<<tgl::warps_grid(graph->vertex_count), 256, 0,
                                       static_cast<cudaStream_t>(stream)>>>(tgl::view(graph), dx_edge, ld_dx, dh);
    return tgl::launched("tgl_mp_edge_inputs_backward");
}

extern "C" int64_t tgl_column_sums_scratch(int64_t rows, int32_t n) {
    return ((rows + tgl::MP_ROWS_PER_CHUNK - 1) / tgl::MP_ROWS_PER_CHUNK) * (int64_t)n;
}

extern "C" int tgl_column_sums(const float *x, int64_t rows, int32_t n, int64_t ld, float *out, int32_t accumulate,
                               float *scratch, void *stream) {
    if (!x || !out || !scratch || rows < 0 || n <= 0 || ld < n)
        return gemm_error(TGL_ERR_INVALID, "tgl_column_sums: bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t chunks = (rows + tgl::MP_ROWS_PER_CHUNK - 1) / tgl::MP_ROWS_PER_CHUNK;
    if (chunks > 65535) return gemm_error(TGL_ERR_UNSUPPORTED, "tgl_column_sums: too many rows");
    if (chunks > 0) {
        dim3 grid((unsigned)((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024), (unsigned)chunks);
        tgl::column_partials_kernel<<<grid, 256, 0, st>>>(x, rows, n, ld, scratch);
    }
    tgl::column_finish_kernel<<<(n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024, 256, 0, st>>>(scratch, chunks, n, out,
                                                                                                accumulate);
    return tgl::launched("tgl_column_sums");
}

extern "C" int tgl_adam_step(int64_t n, float *w, const float *g, float *m, float *v, void *w_bf16, float lr,
                             float beta1, float beta2, float eps, int32_t step, void *stream) {
    if (n < 0 || !w || !g || !m || !v || step < 1) return gemm_error(TGL_ERR_INVALID, "tgl_adam_step: bad arguments");
    if (n == 0) return 0;
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    tgl::adam_kernel<<<(int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096), 256, 0,
                       static_cast<cudaStream_t>(stream)>>>(n, w, g, m, v, static_cast<__nv_bfloat16 *>(w_bf16), lr,
                                                            beta1, beta2, eps, c1, c2);
    return tgl::launched("tgl_adam_step");
}

extern "C" int tgl_mse(int64_t rows, const float *y, int64_t ld_y, const float *target, int32_t cols, float *loss,
                       float *dy, int64_t ld_dy, void *dy_bf16, float *scratch, void *stream) {
    if (rows <= 0 || !y || !target || !loss || !scratch || cols <= 0 || ld_y < cols || ld_dy < cols)
        return gemm_error(TGL_ERR_INVALID, "tgl_mse: bad arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int blocks = (int)((rows + 255) / 256 < 1024 ? (rows + 255) / 256 : 1024);
    tgl::mse_kernel<<<blocks, 256, 0, st>>>(rows, y, ld_y, target, cols, dy, ld_dy,
                                            static_cast<__nv_bfloat16 *>(dy_bf16), scratch);
    tgl::mse_finish_kernel<<<1, 32, 0, st>>>(scratch, blocks, 1.0f / ((float)rows * (float)cols), loss);
    return tgl::launched("tgl_mse");
}
