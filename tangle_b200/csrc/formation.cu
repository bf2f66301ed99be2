// formation.cu -- the formation hooks that run outside the update step:
// the immediate application of a layer target, vertex-target capture, the
// target residuals, cell compaction and its metrics, and per-fiber curvature
// limits (crates/tangle_relax/src/device/kernels.rs:538-923,
// world.rs:1723-2194). The targets' per-step application lives in the
// update kernels (formation.cuh).
//
// Every kernel works on the active fibers (the first FA entries of
// fiber_order), one warp per fiber. Sums the reference forms serially per
// fiber (a fiber's centre) are serial here too, on lane 0, so that they round
// alike; the compaction metrics, which the reference sums serially over the
// whole world in f32, are summed in f64 in a fixed order (per-thread, then
// per block, then over the blocks in block order): every term is the
// reference's f32 term, only the accumulation is more precise.
#include "formation.cuh"

#include <algorithm>

namespace tgl {

namespace {

constexpr uint32_t ALL_LANES = 0xFFFFFFFFu;

int blocks_of(uint32_t warps_needed, int warps_per_block, int cap) {
    long long b = ((long long)warps_needed + warps_per_block - 1) / warps_per_block;
    return (int)std::max(1LL, std::min<long long>(b, cap));
}

// apply_layer_target_range's immediate launch (world.rs:1758-1800).
__global__ void layer_targets_now_kernel(WorldDev w) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < w.FA; k += warps) {
        const uint32_t f = w.fiber_order[k];
        const uint2 span = w.fiber_vspan[f];
        layer_target_staged(w, f, w.pos + span.x, (int)span.y, lane);
    }
}

// initialize_vertex_displacement_targets (kernels.rs:583-602).
__global__ void init_vertex_targets_kernel(WorldDev w, const uint32_t *vertices, uint32_t count, float displacement,
                                           float *target, float *command) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        float4 p = w.pos[vertices[k]];
        const float coordinate = coordinate_of(p, w.target_axis);
        target[k] = coordinate + displacement;
        command[k] = coordinate;
    }
}

// measure_layer_target_error (kernels.rs:636-680): the largest distance of
// an active targeted fiber's centre from its layer's target.
__global__ void layer_error_kernel(WorldDev w, unsigned int *bits) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < w.FA; k += warps) {
        if (lane != 0) continue;
        const uint32_t f = w.fiber_order[k];
        uint32_t layer;
        const uint2 span = w.fiber_vspan[f];
        if (!layer_targeted(w, f, layer) || span.y == 0) continue;
        const float error = fabsf(w.layer_target[layer] - layer_center(w.pos + span.x, (int)span.y, w.layer_axis));
        if (error > 0.0f) atomicMax(bits, __float_as_uint(error));  // the serial `error > maximum` from 0
    }
}

// measure_vertex_target_error (kernels.rs:682-711) over the targets whose
// vertex is active.
__global__ void vertex_error_kernel(WorldDev w, const uint32_t *vertices, const uint32_t *fibers, uint32_t count,
                                    unsigned int *bits) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        if (w.fiber_on != nullptr && w.fiber_on[fibers[k]] == 0u) continue;
        float4 p = w.pos[vertices[k]];
        const float error = fabsf(w.target_coord[k] - coordinate_of(p, w.target_axis));
        if (error > 0.0f) atomicMax(bits, __float_as_uint(error));
    }
}

struct Box {
    float lower[3], upper[3];
};

// compact_rigid_fiber_centers (kernels.rs:712-764): each active fiber's
// centre keeps its fractional position in the cell; the fiber translates
// rigidly and its wall reactions clear.
__global__ void compact_rigid_kernel(WorldDev w, Box nb) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const Grid &g = w.grid;
    for (uint32_t k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < w.FA; k += warps) {
        const uint32_t f = w.fiber_order[k];
        const uint2 span = w.fiber_vspan[f];
        float4 *P = w.pos + span.x;
        const int n = (int)span.y;
        float d[3] = {0.0f, 0.0f, 0.0f};
        if (lane == 0 && n > 0) {
            float c[3] = {0.0f, 0.0f, 0.0f};
            for (int i = 0; i < n; ++i) {
                const float4 p = P[i];
                c[0] += p.x;
                c[1] += p.y;
                c[2] += p.z;
            }
            for (int a = 0; a < 3; ++a) {
                c[a] /= (float)n;
                const float fraction = (c[a] - g.lower[a]) / (g.upper[a] - g.lower[a]);
                d[a] = nb.lower[a] + fraction * (nb.upper[a] - nb.lower[a]) - c[a];
            }
        }
        for (int a = 0; a < 3; ++a) d[a] = __shfl_sync(ALL_LANES, d[a], 0);
        for (int i = lane; i < n; i += 32) {
            float4 p = P[i];
            p.x += d[0];
            p.y += d[1];
            p.z += d[2];
            P[i] = p;
            if (w.reaction) w.reaction[span.x + i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    }
}

// compact_moving_walls (kernels.rs:789-818, kinematics 1): active vertices
// projected inside the new walls, the projection recorded as the wall
// reaction; compact_affine_vertices (kernels.rs:766-787, kinematics 2): the
// cell's deformation gradient applied to every active vertex.
__global__ void compact_vertices_kernel(WorldDev w, Box nb, uint32_t kinematics) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const Grid &g = w.grid;
    for (uint32_t k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < w.FA; k += warps) {
        const uint32_t f = w.fiber_order[k];
        const uint2 span = w.fiber_vspan[f];
        for (uint32_t i = lane; i < span.y; i += 32) {
            const uint32_t v = span.x + i;
            float4 p = w.pos[v];
            float r[3] = {0.0f, 0.0f, 0.0f};
            for (int a = 0; a < 3; ++a) {
                float &x = coordinate_of(p, (uint32_t)a);
                if (kinematics == 2) {
                    const float fraction = (x - g.lower[a]) / (g.upper[a] - g.lower[a]);
                    x = nb.lower[a] + fraction * (nb.upper[a] - nb.lower[a]);
                } else if (!g.periodic[a]) {
                    const float radius = w.vtx_static[v].w;
                    const float previous = x;
                    x = clampf(previous, nb.lower[a] + radius, nb.upper[a] - radius);
                    r[a] = previous - x;  // negative: the lower face, positive: the upper face
                }
            }
            w.pos[v] = p;
            if (w.reaction) w.reaction[v] = make_float4(r[0], r[1], r[2], 0.0f);
        }
    }
}

// The compaction metrics' sums (kernels.rs:842-891): load per axis (|end
// corrections|), contact energy, stretch energy, bending energy, and the
// six face loads; each term is the reference's f32 term.
constexpr int SUMS = 12;

__global__ void __launch_bounds__(256) metrics_partial_kernel(WorldDev w, float contact_stiffness,
                                                              float stretch_stiffness, float bending_stiffness,
                                                              double *partials) {
    __shared__ double warp_sums[8][SUMS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    double acc[SUMS];
    for (int q = 0; q < SUMS; ++q) acc[q] = 0.0;
    for (uint32_t k = blockIdx.x * (blockDim.x >> 5) + warp; k < w.FA; k += warps) {
        const uint32_t f = w.fiber_order[k];
        const uint2 span = w.fiber_vspan[f];
        const uint32_t s0 = w.fiber_s0[f];
        const int n = (int)span.y;
        const float4 *P = w.pos + span.x;
        for (int i = lane; i + 1 < n; i += 32) {
            const uint32_t s = s0 + (uint32_t)i;
            const float4 c0 = w.corr[2 * (size_t)s], c1 = w.corr[2 * (size_t)s + 1];
            acc[0] += (double)(fabsf(c0.x) + fabsf(c1.x));
            acc[1] += (double)(fabsf(c0.y) + fabsf(c1.y));
            acc[2] += (double)(fabsf(c0.z) + fabsf(c1.z));
            const float penetration = c0.w;
            acc[3] += (double)(0.5f * contact_stiffness * penetration * penetration);
            const float4 a = P[i], b = P[i + 1];
            const float dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
            const float length = sqrtf(dx * dx + dy * dy + dz * dz);
            const float rest = w.rest[s];
            if (rest > 1.0e-7f) {
                const float extension = length - rest;
                acc[4] += (double)(0.5f * stretch_stiffness * extension * extension / rest);
            }
        }
        for (int i = lane; i < n; i += 32) {
            if (i > 0 && i + 1 < n) {
                const float maximum = w.vtx_static[span.x + i].x;
                if (maximum > 0.0f) {
                    const float excess = fmaxf(curvature_ratio_at([&](int q) { return P[q]; }, i, maximum) - 1.0f, 0.0f);
                    acc[5] += (double)(0.5f * bending_stiffness * excess * excess);
                }
            }
            if (w.reaction) {
                const float4 r = w.reaction[span.x + i];
                acc[6] += (double)fmaxf(-r.x, 0.0f);
                acc[7] += (double)fmaxf(r.x, 0.0f);
                acc[8] += (double)fmaxf(-r.y, 0.0f);
                acc[9] += (double)fmaxf(r.y, 0.0f);
                acc[10] += (double)fmaxf(-r.z, 0.0f);
                acc[11] += (double)fmaxf(r.z, 0.0f);
            }
        }
    }
    for (int q = 0; q < SUMS; ++q) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(ALL_LANES, v, o);
        if (lane == 0) warp_sums[warp][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < SUMS) {
        double v = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v += warp_sums[k][threadIdx.x];
        partials[(size_t)blockIdx.x * SUMS + threadIdx.x] = v;
    }
}

// kernels.rs:892-922: the pressures per axis (face loads on walled axes,
// correction loads on periodic ones) over the face areas, the energies, and
// the six face pressures.
__global__ void metrics_final_kernel(const double *partials, int blocks, Grid g, float correction_fraction,
                                     float contact_stiffness, float *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double total[SUMS];
    for (int q = 0; q < SUMS; ++q) total[q] = 0.0;
    for (int b = 0; b < blocks; ++b)
        for (int q = 0; q < SUMS; ++q) total[q] += partials[(size_t)b * SUMS + q];
    float s[SUMS];
    for (int q = 0; q < SUMS; ++q) s[q] = (float)total[q];
    const float length_x = g.upper[0] - g.lower[0], length_y = g.upper[1] - g.lower[1],
                length_z = g.upper[2] - g.lower[2];
    const float inverse_projection = 1.0f / fmaxf(correction_fraction, 1.0e-7f);
    const float load_x = g.periodic[0] ? s[0] : s[6] + s[7];
    const float load_y = g.periodic[1] ? s[1] : s[8] + s[9];
    const float load_z = g.periodic[2] ? s[2] : s[10] + s[11];
    out[0] = contact_stiffness * load_x * inverse_projection / (length_y * length_z);
    out[1] = contact_stiffness * load_y * inverse_projection / (length_x * length_z);
    out[2] = contact_stiffness * load_z * inverse_projection / (length_x * length_y);
    out[3] = s[3];
    out[4] = s[4];
    out[5] = s[5];
    out[6] = s[3] + s[4] + s[5];
    out[7] = contact_stiffness * s[6] * inverse_projection / (length_y * length_z);
    out[8] = contact_stiffness * s[7] * inverse_projection / (length_y * length_z);
    out[9] = contact_stiffness * s[8] * inverse_projection / (length_x * length_z);
    out[10] = contact_stiffness * s[9] * inverse_projection / (length_x * length_z);
    out[11] = contact_stiffness * s[10] * inverse_projection / (length_x * length_y);
    out[12] = contact_stiffness * s[11] * inverse_projection / (length_x * length_y);
}

// set_fiber_maximum_curvatures (world.rs:2185-2194): every vertex of fiber f
// (its ends included) takes values[f].
__global__ void fiber_curvatures_kernel(WorldDev w, float4 *vtx_static, const float *values) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t f = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); f < w.F; f += warps) {
        const uint2 span = w.fiber_vspan[f];
        const float value = values[f];
        for (uint32_t i = lane; i < span.y; i += 32) vtx_static[span.x + i].x = value;
    }
}

// The reactions of inactive fibers' vertices cleared (the reference clears
// every vertex's reaction at the start of each update step).
__global__ void clear_inactive_reactions_kernel(WorldDev w) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t f = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); f < w.F; f += warps) {
        if (w.fiber_on == nullptr || w.fiber_on[f] != 0u) continue;
        const uint2 span = w.fiber_vspan[f];
        for (uint32_t i = lane; i < span.y; i += 32) w.reaction[span.x + i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

}  // namespace

void launch_layer_targets_now(const WorldDev &w, cudaStream_t st) {
    layer_targets_now_kernel<<<blocks_of(w.FA, 8, 148 * 64), 256, 0, st>>>(w);
}

void launch_init_vertex_targets(const WorldDev &w, const uint32_t *vertices, uint32_t count, float displacement,
                                float *target, float *command, cudaStream_t st) {
    init_vertex_targets_kernel<<<blocks_of(count, 256, 4096), 256, 0, st>>>(w, vertices, count, displacement, target,
                                                                             command);
}

void launch_target_errors(const WorldDev &w, const uint32_t *vertices, const uint32_t *fibers, uint32_t count,
                          unsigned int *bits2, cudaStream_t st) {
    cudaMemsetAsync(bits2, 0, 2 * sizeof(unsigned int), st);
    if (w.layer_target) layer_error_kernel<<<blocks_of(w.FA, 8, 148 * 64), 256, 0, st>>>(w, bits2);
    if (w.vertex_target && count)
        vertex_error_kernel<<<blocks_of(count, 256, 4096), 256, 0, st>>>(w, vertices, fibers, count, bits2 + 1);
}

void launch_compaction(const WorldDev &w, const float new_lower[3], const float new_upper[3], uint32_t kinematics,
                       cudaStream_t st) {
    Box nb;
    for (int a = 0; a < 3; ++a) {
        nb.lower[a] = new_lower[a];
        nb.upper[a] = new_upper[a];
    }
    if (kinematics == 0)
        compact_rigid_kernel<<<blocks_of(w.FA, 8, 148 * 64), 256, 0, st>>>(w, nb);
    else
        compact_vertices_kernel<<<blocks_of(w.FA, 8, 148 * 64), 256, 0, st>>>(w, nb, kinematics);
}

void launch_compaction_metrics(const WorldDev &w, float correction_fraction, float contact_stiffness,
                               float stretch_stiffness, float bending_stiffness, double *partials, float *out13,
                               cudaStream_t st) {
    metrics_partial_kernel<<<METRIC_BLOCKS, 256, 0, st>>>(w, contact_stiffness, stretch_stiffness, bending_stiffness,
                                                          partials);
    metrics_final_kernel<<<1, 32, 0, st>>>(partials, METRIC_BLOCKS, w.grid, correction_fraction, contact_stiffness,
                                           out13);
}

void launch_set_fiber_curvatures(const WorldDev &w, float4 *vtx_static, const float *values, cudaStream_t st) {
    fiber_curvatures_kernel<<<blocks_of(w.F, 8, 148 * 64), 256, 0, st>>>(w, vtx_static, values);
}

void launch_clear_inactive_reactions(const WorldDev &w, cudaStream_t st) {
    if (w.reaction && w.fiber_on)
        clear_inactive_reactions_kernel<<<blocks_of(w.F, 8, 148 * 64), 256, 0, st>>>(w);
}

}  // namespace tgl
