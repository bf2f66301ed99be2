// noalloc.cu -- a contact pass that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host application that hands this
// library its own device buffers from a fixed memory pool it manages (a
// simulation embedding the contact step in a larger solver, or a service
// with a pre-reserved memory budget that forbids allocation after start-up),
// and code running where allocation is unavailable or would stall, such as
// a real-time loop that must never wait on the allocator. For them,
// tgl_contact_pass_noalloc computes one contact pass from device arrays the
// caller already owns, using only a scratch array that is part of this
// library's image: `noalloc_scratch` below, a fixed 5 MiB (plus alignment)
// that every GPU which loads the library holds until the process exits.
//
// The result is the reference's find_segment_corrections
// (crates/tangle_contact/src/device/contact.rs:232-902) with every segment
// taking the exact 27-cell scan (contact.rs:365-437): the contacts a world
// of neighbor_capacity 1 finds, summed in the same cell order.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/tangle_cuda.h"
#include "common.cuh"
#include "contact.cuh"

namespace tgl {
void set_last_error(const std::string &message);  // world.cu
}

namespace {

constexpr uint32_t NOALLOC_MAX_SEGMENTS = 1u << 18;  // 262,144
constexpr uint32_t NOALLOC_MAX_CELLS = 1u << 18;
constexpr int NOALLOC_MAX_DEVICES = 64;
constexpr uint32_t FULL = 0xFFFFFFFFu;

// Layout: cell counts [MAX_CELLS], cell offsets [MAX_CELLS], then per
// segment its cell, its arrival ticket and the slot order [MAX_SEGMENTS]
// each, all u32.
constexpr size_t NOALLOC_WORDS = 2ull * NOALLOC_MAX_CELLS + 3ull * NOALLOC_MAX_SEGMENTS;
static __device__ __align__(256) uint32_t noalloc_scratch[NOALLOC_WORDS];

// The array's address per device, with the id of the CUDA context it was
// looked up in: a context that is destroyed and created again (after
// cudaDeviceReset, say) reloads the library's module, and the array may move.
struct ScratchSlot {
    unsigned long long context_id;
    uint32_t *address;
};
std::mutex g_scratch_mutex;
ScratchSlot g_scratch[NOALLOC_MAX_DEVICES] = {};

// Messages go where tgl_last_error() reads them.
int noalloc_error(int code, const std::string &message) {
    tgl::set_last_error(message);
    return code;
}

struct NoallocArgs {
    const float *positions;
    const uint32_t *segment_vertices;
    const uint32_t *segment_fibers;
    const float *segment_radii;
    const float *arc;
    uint32_t S;
    uint32_t C;
    tgl::Grid grid;
    float correction_fraction;
    uint32_t aggregation;
    uint32_t *counts, *offsets, *cell_of, *ticket, *segments;
    float *corrections;
    float *penetrations;
};

__device__ inline void segment_records(const NoallocArgs &a, uint32_t s, float4 &oa, float4 &ob) {
    const uint32_t v0 = a.segment_vertices[2 * s], v1 = a.segment_vertices[2 * s + 1];
    const float px = a.positions[3 * v0], py = a.positions[3 * v0 + 1], pz = a.positions[3 * v0 + 2];
    const float qx = a.positions[3 * v1], qy = a.positions[3 * v1 + 1], qz = a.positions[3 * v1 + 2];
    const float dx = qx - px, dy = qy - py, dz = qz - pz;
    oa = make_float4(px, py, pz, a.segment_radii[s]);
    ob = make_float4(qx, qy, qz, 0.5f * sqrtf(dx * dx + dy * dy + dz * dz));
}

// count_cell_segments with the arrival ticket (cell_list.rs:116-164).
__global__ void noalloc_count(NoallocArgs a) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < a.S; s += gridDim.x * blockDim.x) {
        float4 oa, ob;
        segment_records(a, s, oa, ob);
        const uint32_t cell = tgl::proxy_cell(oa.x, oa.y, oa.z, ob.x, ob.y, ob.z, a.grid);
        a.cell_of[s] = cell;
        a.ticket[s] = atomicAdd(&a.counts[cell], 1u);
    }
}

// Exclusive scan of the counts, one block.
__global__ void __launch_bounds__(1024) noalloc_scan(NoallocArgs a) {
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < a.C; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < a.C ? a.counts[i] : 0u;
        uint32_t incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const uint32_t ws = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0u;
            uint32_t wi = ws;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(FULL, wi, o);
                if (lane >= o) wi += t;
            }
            if (lane < (int)(blockDim.x >> 5)) warp_sums[lane] = wi - ws;
        }
        __syncthreads();
        const uint32_t exclusive = carry + warp_sums[warp] + incl - v;
        if (i < a.C) a.offsets[i] = exclusive;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = exclusive + v;
        __syncthreads();
    }
}

__global__ void noalloc_scatter(NoallocArgs a) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < a.S; s += gridDim.x * blockDim.x)
        a.segments[a.offsets[a.cell_of[s]] + a.ticket[s]] = s;
}

// rank_cell_segments (cell_list.rs:346-378): ascending segments per cell,
// ranked over the global slot range into the free ticket array, then copied.
__global__ void noalloc_rank(NoallocArgs a) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < a.C; c += warps) {
        const uint32_t n = a.counts[c];
        if (n < 2) continue;
        const uint32_t off = a.offsets[c];
        for (uint32_t i = lane; i < n; i += 32) {
            const uint32_t key = a.segments[off + i];
            uint32_t rank = 0;
            for (uint32_t j = 0; j < n; ++j) rank += a.segments[off + j] < key ? 1u : 0u;
            a.ticket[off + rank] = key;
        }
        __syncwarp();
        for (uint32_t i = lane; i < n; i += 32) a.segments[off + i] = a.ticket[off + i];
        __syncwarp();
    }
}

// The exact 27-cell scan of contact.rs:365-437 for every segment, one warp
// per segment, hits summed in scan order.
__global__ void noalloc_contact(NoallocArgs a) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t segment = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; segment < a.S; segment += warps) {
        float4 ha, hb;
        segment_records(a, segment, ha, hb);
        const tgl::Home h = tgl::make_home(ha, hb, segment);
        const uint32_t owner = a.segment_fibers[segment];
        const float own_arc0 = a.arc[a.segment_vertices[2 * segment]];
        const float own_arc1 = a.arc[a.segment_vertices[2 * segment + 1]];
        const uint32_t home = a.cell_of[segment];
        tgl::ContactAcc acc = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        for (uint32_t n = 0; n < 27; ++n) {
            const uint32_t cell = tgl::stencil_cell(home, n, a.grid);
            if (cell == TGL_NONE) continue;
            const uint32_t count = a.counts[cell], start = a.offsets[cell];
            for (uint32_t k0 = 0; k0 < count; k0 += 32) {
                const uint32_t k = k0 + lane;
                tgl::PairTerms pt;
                bool hit = false;
                if (k < count) {
                    const uint32_t other = a.segments[start + k];
                    const float arc0 = a.arc[a.segment_vertices[2 * other]];
                    const float arc1 = a.arc[a.segment_vertices[2 * other + 1]];
                    const float gap = fmaxf(arc0 - own_arc1, own_arc0 - arc1);  // along_fiber_gap
                    const float other_radius = a.segment_radii[other];
                    const bool near_along_fiber = a.segment_fibers[other] == owner && gap < h.radius + other_radius;
                    if (other != segment && !near_along_fiber) {
                        float4 oa, ob;
                        segment_records(a, other, oa, ob);
                        float p2x, p2y, p2z, q2x, q2y, q2z;
                        if (tgl::contact_reach(h, oa, ob, a.grid, p2x, p2y, p2z, q2x, q2y, q2z))
                            hit = tgl::contact_solve(h, other, oa.w, p2x, p2y, p2z, q2x, q2y, q2z,
                                                     a.correction_fraction, a.aggregation, pt);
                    }
                }
                uint32_t bits = __ballot_sync(FULL, hit);
                while (bits) {
                    const int j = __ffs(bits) - 1;
                    bits &= bits - 1u;
                    tgl::add_hit(acc, a.aggregation, __shfl_sync(FULL, pt.pen, j), __shfl_sync(FULL, pt.t0x, j),
                                 __shfl_sync(FULL, pt.t0y, j), __shfl_sync(FULL, pt.t0z, j),
                                 __shfl_sync(FULL, pt.t1x, j), __shfl_sync(FULL, pt.t1y, j),
                                 __shfl_sync(FULL, pt.t1z, j), __shfl_sync(FULL, pt.aggw, j));
                }
            }
        }
        if (lane == 0) {
            if (a.aggregation != 2 && acc.weight > 1.0e-20f) {
                acc.c0x /= acc.weight;
                acc.c0y /= acc.weight;
                acc.c0z /= acc.weight;
                acc.c1x /= acc.weight;
                acc.c1y /= acc.weight;
                acc.c1z /= acc.weight;
            }
            float *out = a.corrections + 6 * (size_t)segment;
            out[0] = acc.c0x;
            out[1] = acc.c0y;
            out[2] = acc.c0z;
            out[3] = acc.c1x;
            out[4] = acc.c1y;
            out[5] = acc.c1z;
            a.penetrations[segment] = acc.maxpen;
        }
    }
}

// The unique id (cuCtxGetId, CUDA 12.0+) of the calling thread's current
// context, through the runtime's driver entry points so the library does not
// link libcuda itself. Ids are never reused within a process, unlike context
// handles. False when no context is current yet or the driver lacks either
// call.
bool current_context_id(unsigned long long *id) {
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    if (!get_current || !get_id) {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa = cudaDriverEntryPointSymbolNotFound, qb = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
            qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b)
            return false;
        get_current = reinterpret_cast<GetCurrent>(a);
        get_id = reinterpret_cast<GetId>(b);
    }
    CUcontext ctx = nullptr;
    return get_current(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, id) == CUDA_SUCCESS;
}

// The scratch array's device address in the current device's context. The
// host-side name of a __device__ array is not a device address, so it is
// looked up with cudaGetSymbolAddress: on the first call on each device, and
// again whenever that device's current context is a new one.
int scratch_address(uint32_t **out) {
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= NOALLOC_MAX_DEVICES)
        return noalloc_error(TGL_ERR_NO_DEVICE, "no usable current CUDA device");
    unsigned long long context = 0;
    bool known = current_context_id(&context);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    ScratchSlot &slot = g_scratch[device];
    if (!known || !slot.address || slot.context_id != context) {
        void *ptr = nullptr;
        // With no context current yet, this lookup makes the runtime create
        // the device's primary context; its id is read afterwards.
        cudaError_t e = cudaGetSymbolAddress(&ptr, noalloc_scratch);
        if (e != cudaSuccess)
            return noalloc_error(TGL_ERR_CUDA, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
        if (!known && !current_context_id(&context))
            return noalloc_error(TGL_ERR_CUDA, "cannot identify the current CUDA context");
        slot.address = static_cast<uint32_t *>(ptr);
        slot.context_id = context;
    }
    *out = slot.address;
    return 0;
}

}  // namespace

extern "C" int tgl_contact_pass_noalloc(const tgl_noalloc_inputs *in, float *corrections, float *segment_max_penetration,
                                         void *stream) {
    if (!in || !corrections || !segment_max_penetration)
        return noalloc_error(TGL_ERR_INVALID, "null argument");
    if (!in->positions || !in->segment_vertices || !in->segment_fibers || !in->segment_radii || !in->vertex_arc_lengths)
        return noalloc_error(TGL_ERR_INVALID, "a required device array is null");
    if (in->segment_count == 0) return noalloc_error(TGL_ERR_INVALID, "no segments");
    if (in->segment_count > NOALLOC_MAX_SEGMENTS)
        return noalloc_error(TGL_ERR_UNSUPPORTED, "tgl_contact_pass_noalloc takes at most 262144 segments, got " +
                                                      std::to_string(in->segment_count));
    if (in->cells[0] == 0 || in->cells[1] == 0 || in->cells[2] == 0)
        return noalloc_error(TGL_ERR_INVALID, "every axis needs at least one cell");
    // Each axis is bounded before it is multiplied, and the running product
    // after every factor, so the count cannot wrap: a factor is at most
    // 2^18 and the product before it at most 2^18.
    uint64_t cells = 1;
    for (int ax = 0; ax < 3; ++ax) {
        if (in->cells[ax] > NOALLOC_MAX_CELLS)
            return noalloc_error(TGL_ERR_UNSUPPORTED, "tgl_contact_pass_noalloc takes at most 262144 cells, got " +
                                                          std::to_string(in->cells[ax]) + " on one axis");
        cells *= in->cells[ax];
        if (cells > NOALLOC_MAX_CELLS)
            return noalloc_error(TGL_ERR_UNSUPPORTED, "tgl_contact_pass_noalloc takes at most 262144 cells, got " +
                                                          std::to_string(in->cells[0]) + " x " + std::to_string(in->cells[1]) +
                                                          " x " + std::to_string(in->cells[2]));
    }
    if (!(in->correction_fraction > 0.0f && in->correction_fraction <= 1.0f) || in->contact_aggregation > 2)
        return noalloc_error(TGL_ERR_INVALID, "correction_fraction must be in (0, 1], contact_aggregation 0-2");
    uint32_t *scratch = nullptr;
    if (int rc = scratch_address(&scratch)) return rc;
    NoallocArgs a{};
    a.positions = in->positions;
    a.segment_vertices = in->segment_vertices;
    a.segment_fibers = in->segment_fibers;
    a.segment_radii = in->segment_radii;
    a.arc = in->vertex_arc_lengths;
    a.S = in->segment_count;
    a.C = (uint32_t)cells;
    for (int ax = 0; ax < 3; ++ax) {
        a.grid.lower[ax] = in->cell_lower[ax];
        a.grid.upper[ax] = in->cell_upper[ax];
        a.grid.periodic[ax] = in->cell_periodic[ax] ? 1u : 0u;
        a.grid.cells[ax] = in->cells[ax];
        a.grid.length[ax] = in->cell_upper[ax] - in->cell_lower[ax];
        a.grid.width[ax] = a.grid.length[ax] / (float)in->cells[ax];
        a.grid.inv_length[ax] = 1.0f / a.grid.length[ax];
        if (!(a.grid.length[ax] > 0.0f)) return noalloc_error(TGL_ERR_INVALID, "cell bounds must have upper > lower");
    }
    a.correction_fraction = in->correction_fraction;
    a.aggregation = in->contact_aggregation;
    a.counts = scratch;
    a.offsets = scratch + NOALLOC_MAX_CELLS;
    a.cell_of = scratch + 2 * NOALLOC_MAX_CELLS;
    a.ticket = a.cell_of + NOALLOC_MAX_SEGMENTS;
    a.segments = a.ticket + NOALLOC_MAX_SEGMENTS;
    a.corrections = corrections;
    a.penetrations = segment_max_penetration;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The counts are the only scratch that must start at zero; the rest is
    // fully written before it is read.
    if (cudaMemsetAsync(a.counts, 0, (size_t)a.C * sizeof(uint32_t), st) != cudaSuccess)
        return noalloc_error(TGL_ERR_CUDA, "cudaMemsetAsync of the scratch counts failed");
    int blocks = (int)std::min<uint32_t>((a.S + 255) / 256, 4096);
    noalloc_count<<<blocks, 256, 0, st>>>(a);
    noalloc_scan<<<1, 1024, 0, st>>>(a);
    noalloc_scatter<<<blocks, 256, 0, st>>>(a);
    noalloc_rank<<<(int)std::min<uint32_t>((a.C + 7) / 8, 4096), 256, 0, st>>>(a);
    noalloc_contact<<<(int)std::min<uint32_t>((a.S + 7) / 8, 8192), 256, 0, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_error(TGL_ERR_CUDA, std::string("kernel launch failed: ") + cudaGetErrorString(e));
    return 0;
}
