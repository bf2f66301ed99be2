// formation.cuh -- device helpers of the formation hooks, shared by the
// update kernels (kernels.cu), which apply the targets at the end of every
// update step, and the standalone formation kernels (formation.cu).
#pragma once

#include "kernels.cuh"

namespace tgl {

__device__ inline float &coordinate_of(float4 &p, uint32_t axis) { return axis == 0 ? p.x : (axis == 1 ? p.y : p.z); }

// Mean coordinate of n vertices along an axis: a serial f32 sum in vertex
// order over the count, as apply_formation_layer_targets and
// measure_layer_target_error compute it (kernels.rs:569-573, :664-668).
__device__ inline float layer_center(const float4 *P, int n, uint32_t axis) {
    float center = 0.0f;
    for (int i = 0; i < n; ++i) {
        float4 p = P[i];
        center += coordinate_of(p, axis);
    }
    return center / (float)n;
}

// Does fiber f carry a layer that the installed target range covers
// (kernels.rs:556-563)?
__device__ inline bool layer_targeted(const WorldDev &w, uint32_t f, uint32_t &layer) {
    layer = w.fiber_layer[f];
    return layer != TGL_NONE && layer < w.layer_count && layer >= w.layer_first && layer <= w.layer_last;
}

// apply_formation_layer_targets (kernels.rs:538-581) for fiber f, whose n
// vertices are at P, the whole warp on the fiber: the fiber's mean
// coordinate moves toward its layer's target by stiffness, capped at
// max_translation; every vertex (pinned ones too) translates alike.
__device__ inline void layer_target_staged(const WorldDev &w, uint32_t f, float4 *P, int n, int lane) {
    uint32_t layer;
    if (!layer_targeted(w, f, layer) || n <= 0) return;
    float translation = 0.0f;
    if (lane == 0)
        translation = clampf((w.layer_target[layer] - layer_center(P, n, w.layer_axis)) * w.layer_stiffness,
                             -w.layer_max_translation, w.layer_max_translation);
    translation = __shfl_sync(0xFFFFFFFFu, translation, 0);
    for (int i = lane; i < n; i += 32) coordinate_of(P[i], w.layer_axis) += translation;
    __syncwarp();
}

// apply_vertex_targets (kernels.rs:604-634) for the targeted vertices among
// the n vertices at P (first vertex v0): each is set to its commanded
// coordinate advanced toward its target by stiffness, capped at
// max_translation.
__device__ inline void vertex_targets_staged(const WorldDev &w, float4 *P, int n, uint32_t v0, int lane) {
    for (int i = lane; i < n; i += 32) {
        const int32_t k = w.vertex_target[v0 + i];
        if (k < 0) continue;
        const float command = w.command_coord[k];
        const float translation = clampf((w.target_coord[k] - command) * w.target_stiffness,
                                         -w.target_max_translation, w.target_max_translation);
        w.command_coord[k] = command + translation;
        coordinate_of(P[i], w.target_axis) = command + translation;
    }
    __syncwarp();
}

// The targets at the end of an update step (world.rs:1420-1447): the layer
// target, then the vertex targets.
__device__ inline void formation_targets_staged(const WorldDev &w, uint32_t f, float4 *P, int n, uint32_t v0,
                                                int lane) {
    if (w.layer_target != nullptr) layer_target_staged(w, f, P, n, lane);
    if (w.vertex_target != nullptr) vertex_targets_staged(w, P, n, v0, lane);
}

}  // namespace tgl
