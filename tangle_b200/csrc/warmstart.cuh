// warmstart.cuh -- device structures of the learned warm start: the contact
// graph a world extracts (world.cu) and the message-passing kernels over it
// (warmstart.cu).
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

#include "kernels.cuh"

namespace tgl {

constexpr int MP_HIDDEN = 64;        // embedding width
constexpr int MP_NODE_FEATURES = 16; // node feature row (7 used)
constexpr int MP_EDGE_FEATURES = 16; // edge feature row (6 used)

// The contact graph of one world: nodes are vertices, edges are directed
// segment pairs (dst <- src) within a gap cutoff, both directions of every
// pair present, stored by destination segment (CSR) and, within one, by
// ascending source segment.
struct MpGraph {
    int32_t V, S, E;
    const int32_t *seg_v0;     // [S] first vertex of each segment (second = first + 1)
    const int4 *links;         // [V] previous vertex, next vertex, segment before, segment after (-1 = none)
    const int32_t *offsets;    // [S + 1]
    const int32_t *dst;        // [E]
    const int32_t *src;        // [E]
    const int32_t *twin;       // [E] the reverse edge
    const float *s;            // [E] closest-point parameter on the destination segment
    const float *t;            // [E] closest-point parameter on the source segment
};

// World-owned buffers the graph is built into.
struct GraphBuffers {
    uint32_t *fwd_count, *in_count, *fill;  // [S]
    int32_t *offsets;                        // [S + 1]
    int32_t *dst, *src, *twin;               // [E]
    float *s, *t, *depth;                    // [E]
    __nv_bfloat16 *edge_features;            // [E * 16]
    __nv_bfloat16 *node_features;            // [V * 16]
    int32_t *block_sums;                     // scan scratch
    int64_t edge_capacity;
    // Focus fibers (nullptr: all): only pairs with a segment on one of them
    // become edges (a new ply's contacts on a relaxed stack).
    const uint32_t *fiber_focus;             // [F] nonzero = in focus
};

// Whether pair (a, b) may enter the graph under the focus set.
__device__ inline bool in_focus(const WorldDev &w, const GraphBuffers &g, uint32_t a, uint32_t b) {
    return g.fiber_focus == nullptr || g.fiber_focus[__float_as_uint(w.seg_static[a].w)] != 0u ||
           g.fiber_focus[__float_as_uint(w.seg_static[b].w)] != 0u;
}

// Graph extraction from the world's Verlet lists (built from the current
// positions): counts, offsets and edge records.
void launch_graph_count(const WorldDev &w, const GraphBuffers &g, float cutoff, cudaStream_t st);
int launch_graph_offsets(const WorldDev &w, const GraphBuffers &g, cudaStream_t st);  // kernels launched
void launch_graph_fill(const WorldDev &w, const GraphBuffers &g, float cutoff, cudaStream_t st);
void launch_node_features(const WorldDev &w, const GraphBuffers &g, const MpGraph &graph, cudaStream_t st);
// Positions += scale * dx (rows of ld floats; times the vertex's diameter
// when in_diameters), each vertex's move capped at max_step, pinned vertices
// kept; geometry records refreshed.
void launch_displace(const WorldDev &w, const float *dx, int64_t ld, float scale, int in_diameters, float max_step,
                     cudaStream_t st);
// Residual of the current positions without moving them, from the last
// contact pass (corr[].w): max penetration, max curvature ratio, and the sum
// over segments of penetration / diameter (out[0..2]); out holds
// 3 + RESIDUAL_BLOCKS floats (per-block partial sums after the three).
constexpr int RESIDUAL_BLOCKS = 148 * 8;
void launch_residual(const WorldDev &w, float *out, cudaStream_t st);

}  // namespace tgl
