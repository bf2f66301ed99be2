// kernels.cuh -- device buffers of one relaxation world and the launch
// entry points of its kernels (kernels.cu).
#pragma once

#include "common.cuh"

namespace tgl {

// One specimen of an arena: its box, neighbor skin and cell range.
struct SpecimenDev {
    Grid grid;
    float skin;
    uint32_t cell_base;       // first cell of the specimen in the arena's cell numbering
    uint32_t build_prefilter; // sphere pre-test on (>= 3 cells on every periodic axis)
    float build_sphere_eps;
    float line_eps;
    uint32_t cell_count;      // cells of the specimen
    uint32_t seg_base;        // first segment (= first cell-list slot) of the specimen
    uint32_t pad;
};

// Every device pointer and size a kernel needs, passed by value.
// Bounding box of a cell's segment spheres (radii x 1.0003) in the cell's
// own frame: centre minus the cell's lower corner, wrapped to the nearest
// image on periodic axes; as order-preserving int keys (float_key), and the
// largest |x| + |y| + |z| of a centre (f32 bits). Empty cells keep
// [+inf, -inf].
struct CellBox {
    int lo[3], hi[3];
    uint32_t mag, pad;
};

struct WorldDev {
    uint32_t V, S, F, C;
    uint32_t block;      // neighbor slots per segment list
    uint32_t max_fiber;  // most vertices in one fiber
    float skin;          // neighbor skin
    // Contact lists: per cell-list slot, the Verlet-list entries that lie
    // within contact_skin of touching at the contact_ref snapshot (0 = off).
    float contact_skin;
    uint32_t contact_block;  // entries per slot
    // Longest half length for which a pair within reach + contact_skin has
    // one minimum image (L/2 > 2 H + 2 r_max + contact_skin on every periodic
    // axis); a longer segment makes every pass refresh (read the Verlet list).
    float contact_half_limit;
    Grid grid;
    // Static, uploaded once.
    const float4 *seg_static;   // [S] radius, arc(first vertex), arc(second vertex), fiber bits
    const uint32_t *seg_v0;     // [S] first vertex (second = first + 1)
    const uint2 *fiber_vspan;   // [F] first vertex, vertex count
    const uint32_t *fiber_s0;   // [F] first segment
    const uint32_t *fiber_order; // [F] fibers by descending vertex count
    // The grouped-lane update's order of the first FA fibers: fiber_order
    // itself, or its fibers ranked by their curvature-sweep rounds, whichever
    // order_by_rounds_kernel timed as faster. The rounds of each fiber's last
    // sweeps, and their moving average over the order epochs.
    uint32_t *update_order;     // [F]
    uint32_t *fiber_rounds;     // [F]
    uint32_t *rounds_avg;       // [F] 16 x rounds
    const float4 *vtx_static;   // [V] max curvature, rest chord to v-2, rest chord to v+2, wall extent
    const uint32_t *pinned;     // [V]
    const float *rest;          // [S] rest lengths
    const int4 *links;          // [V] previous vertex, next vertex, segment before, segment after (-1 = none)
    const float *rest_curvature; // [V] discrete curvature of the intrinsic shape (0 at fiber ends)
    // Resident state.
    float4 *pos;      // [V] xyz, w = 0
    float4 *ref_pos;  // [V] positions the lists were built from
    float4 *geom;     // [2S] {first xyz, radius}, {second xyz, half length}
    float4 *corr;     // [2S] {end-0 correction, max penetration}, {end-1 correction, 0}
    float *vertex_step; // [V]
    // Cell list.
    uint32_t *cell_counts;   // [C]
    uint32_t *cell_offsets;  // [C]
    uint32_t *cell_segments; // [S] segment per slot, cell order
    uint32_t *cell_of;       // [S] cell of each segment
    uint32_t *ticket;        // [S] scatter position inside its cell; sort scratch
    float4 *slot_geom;       // [2S] geometry records in slot order
    float4 *slot_sphere;     // [S] midpoint and half length + radius, slot order
    CellBox *cell_box;       // [C] box of each cell's bounding spheres, cell frame (build culling)
    // Verlet lists.
    uint32_t *nbr_count; // [S] true neighbor count
    uint32_t *nbr_list;  // [S * block]
    // Contact lists (allocated only when contact_skin > 0). The 32 slots of
    // a contact-pass batch (slots 32b .. 32b + 31) share one chunk of
    // 32 * contact_block entries, their lists back to back in slot order,
    // each in ascending segment order.
    uint32_t *contact_count; // [S] per slot: list length, CONTACT_USE_VERLET or CONTACT_USE_SCAN
    uint32_t *contact_list;  // [S * contact_block] the chunks
    float4 *contact_ref;     // [V] positions the contact lists were filtered at
    Control *ctl;
    float *xyz_stage;    // [3V] interleaved staging for host copies
    // Arena (several specimens relaxed together; the kernels' ARENA
    // instantiations only): specimen tables, the specimen of every segment,
    // fiber, vertex and cell, and a control word per specimen at ctl + 1 + p
    // (ctl[0] then holds the any-specimen flags: active, rebuild pending).
    uint32_t P;
    const SpecimenDev *specs;  // [P]
    const uint32_t *seg_spec;  // [S]
    const uint32_t *fiber_spec; // [F]
    const uint32_t *vtx_spec;  // [V]
    const uint32_t *cell_spec; // [C]
    // Staged activation (activate_formation_step, kernels.rs:164-221): the
    // cell list holds the NS segments of active fibers, the update kernels
    // run the first FA entries of fiber_order (the active fibers), and
    // fiber_on flags each fiber (nullptr: all active, NS = S, FA = F).
    uint32_t NS, FA;
    const uint32_t *fiber_on;  // [F]
    // Wall reactions of the last update step (kernels.rs:1421-1453 and the
    // curvature cleanup): xyz per vertex, w unused; nullptr when no axis has
    // walls (every reaction is then zero).
    float4 *reaction;          // [V]
    // Formation layer target (kernels.rs:538-581), applied at the end of
    // every update step while layer_target is set.
    const uint32_t *fiber_layer; // [F] layer of each fiber, TGL_NONE = none
    const float *layer_target;   // [layer_count] target centre coordinates
    uint32_t layer_count, layer_first, layer_last, layer_axis;
    float layer_stiffness, layer_max_translation;
    // Vertex displacement targets (kernels.rs:583-634), applied after the
    // layer target: target index of each vertex (-1 = none).
    const int32_t *vertex_target; // [V]
    const float *target_coord;    // [targets] absolute target coordinates
    float *command_coord;         // [targets] commanded coordinates so far
    uint32_t target_axis;
    float target_stiffness, target_max_translation;
};

// Contact-list states of a slot besides its list length: the list ran past
// its batch's chunk (walk the Verlet list), or the Verlet list itself
// overflowed (the exact cell scan).
constexpr uint32_t CONTACT_USE_VERLET = 0xFFFFFFFEu;
constexpr uint32_t CONTACT_USE_SCAN = 0xFFFFFFFFu;

// Is segment s on a fiber that takes part (staged activation)?
__device__ inline bool segment_on(const WorldDev &w, uint32_t s) {
    return w.fiber_on == nullptr || w.fiber_on[__float_as_uint(w.seg_static[s].w)] != 0u;
}

// Is vertex v on an active fiber (through either of its segments)?
__device__ inline bool vertex_on(const WorldDev &w, uint32_t v) {
    if (w.fiber_on == nullptr) return true;
    const int4 l = w.links[v];
    return segment_on(w, (uint32_t)(l.z >= 0 ? l.z : l.w));
}

// kernels.rs:925-980 at one interior vertex of a fiber whose positions are
// p(local index).
template <typename Fetch>
__device__ inline float curvature_ratio_at(Fetch p, int i, float maximum) {
    float4 a0 = p(i - 1), c = p(i), b1 = p(i + 1);
    float ax = c.x - a0.x, ay = c.y - a0.y, az = c.z - a0.z;
    float bx = b1.x - c.x, by = b1.y - c.y, bz = b1.z - c.z;
    float first_length = sqrtf(ax * ax + ay * ay + az * az);
    float second_length = sqrtf(bx * bx + by * by + bz * bz);
    float ratio = 0.0f;
    if (first_length > 1.0e-7f && second_length > 1.0e-7f) {
        float cosine = (ax * bx + ay * by + az * bz) / (first_length * second_length);
        cosine = clampf(cosine, -1.0f, 1.0f);
        float dual_length = 0.5f * (first_length + second_length);
        float curvature = 2.0f * sqrtf(0.5f * (1.0f - cosine)) / dual_length;
        ratio = curvature / maximum;
    }
    return ratio;
}

// Formation launchers (formation.cu).
// apply_formation_layer_targets once, outside a batch (world.rs:1758-1800).
void launch_layer_targets_now(const WorldDev &w, cudaStream_t st);
// initialize_vertex_displacement_targets (kernels.rs:583-602) into target
// and command.
void launch_init_vertex_targets(const WorldDev &w, const uint32_t *vertices, uint32_t count, float displacement,
                                float *target, float *command, cudaStream_t st);
// measure_layer_target_error / measure_vertex_target_error (kernels.rs:
// 636-711) as u32 bits of the non-negative maxima: bits2[0] layer, bits2[1]
// vertex (fibers[k]: the fiber of target k's vertex).
void launch_target_errors(const WorldDev &w, const uint32_t *vertices, const uint32_t *fibers, uint32_t count,
                          unsigned int *bits2, cudaStream_t st);
// compact_rigid_fiber_centers (kinematics 0), compact_moving_walls (1),
// compact_affine_vertices (2) (kernels.rs:712-818), from the box in w.grid.
void launch_compaction(const WorldDev &w, const float new_lower[3], const float new_upper[3], uint32_t kinematics,
                       cudaStream_t st);
// measure_compaction_metrics (kernels.rs:820-923) into out13 (device),
// through METRIC_BLOCKS * 12 doubles of partial sums.
constexpr int METRIC_BLOCKS = 296;
void launch_compaction_metrics(const WorldDev &w, float correction_fraction, float contact_stiffness,
                               float stretch_stiffness, float bending_stiffness, double *partials, float *out13,
                               cudaStream_t st);
// set_fiber_maximum_curvatures (world.rs:2185-2194): every vertex of fiber f
// takes values[f] (device array of F).
void launch_set_fiber_curvatures(const WorldDev &w, float4 *vtx_static, const float *values, cudaStream_t st);
// Zeroes the wall reactions of inactive fibers' vertices.
void launch_clear_inactive_reactions(const WorldDev &w, cudaStream_t st);
// Segment geometry records from the positions.
int launch_refresh_geometry(const WorldDev &w, cudaStream_t st);

struct StepParams {
    float penetration_tolerance;
    float correction_fraction;
    float stretch_stiffness;
    float bend_stiffness;
    float curvature_limit_stiffness;
    float curvature_limit_safety_margin;
    float curvature_ratio_tolerance;
    float max_step;
    uint32_t constraint_iterations;
    uint32_t curvature_cleanup_sweeps;
    uint32_t contact_aggregation;
    uint32_t force_full_iterations;
    uint32_t max_iterations;  // the batch size: the gate stops at this many
    uint32_t motion_model;    // 0 flexible, 1 rigid translation
};

// Launch plans, fixed per world. The tune_* fields, when nonzero, override
// the planner's own choice (tgl_world_set_launch_params and the autotuner
// set them; no choice changes a result).
struct LaunchPlan {
    int tune_lanes = 0;           // lanes per fiber
    int tune_contact_per_sm = 0;  // contact-pass blocks per SM
    int tune_build_ch = 0;        // build chunk
    bool arena;             // the kernels' arena instantiations (several specimens)
    int num_sms;
    int contact_group;      // lanes per segment in the contact pass (8, 16 or 32)
    int contact_blocks;
    float line_eps;         // absolute margin of the contact pass's line-distance bound
    int fiber_warps;        // fibers per block of the update kernel
    int fiber_blocks;
    size_t fiber_smem;
    bool fiber_lanes;       // grouped-lane update (fibers of at most 256 vertices)
    int lanes_per_fiber;    // lanes per fiber in its curvature sweeps (2, 4, 8 or 32)
    int lanes_stride;
    size_t lanes_smem;      // staged fibers of one warp
    int lanes_wpb;          // warps per block (1, 2 or 4)
    int tune_wpb = 0;       // requested warps per block (0: the default, 4)
    int lanes_blocks;
    int order_period;       // update launches per fiber-order epoch (0: creation order, no order kernel)
    int order_ranked;       // always the ranked order (1) instead of timing it against the creation order (0)
    bool contact_lists;     // contact lists on (contact_skin > 0)
    int build_ch;           // candidate slots staged per build chunk
    size_t build_smem;
    int build_prefilter;    // sphere pre-test on (needs >= 3 cells per periodic axis)
    float build_sphere_eps; // its absolute margin
    int sort_warps;
    size_t sort_smem;
};

// Each launcher returns the number of kernels it enqueued.
int launch_begin_batch(const WorldDev &w, const LaunchPlan &lp, cudaStream_t st);
int launch_flag_displacement(const WorldDev &w, const LaunchPlan &lp, cudaStream_t st);
int launch_measure_start(const WorldDev &w, const LaunchPlan &lp, cudaStream_t st);
// Kernels in one rebuild pipeline (launch_rebuild's launches).
constexpr int REBUILD_KERNELS = 11;
int launch_rebuild(const WorldDev &w, const LaunchPlan &lp, cudaStream_t st);
// The cell list alone (clear, count, scan, scatter, rank) on w's grid and
// cell buffers, gated on the rebuild flag like the full rebuild.
int launch_cell_list(const WorldDev &w, const LaunchPlan &lp, cudaStream_t st);
// capture_segment_contacts (contact.rs:9-230) on the cell list of w's grid:
// pairs of different fibers within max_gap of touching, appended to the
// output arrays (count[0]; count[1] set on overflow).
void launch_capture(const WorldDev &w, float max_gap, uint32_t capacity, uint32_t *count, uint32_t *pairs,
                    float *coordinates, float *gaps, float *angles, cudaStream_t st);
int launch_request_rebuild(const WorldDev &w, const LaunchPlan &lp, cudaStream_t st);
// With the gate and contact lists on, enqueues the listed pass and the
// refresh pass, each of which returns at once unless the device-side refresh
// flag picks it; otherwise the full-list pass.
int launch_contact(const WorldDev &w, const LaunchPlan &lp, const StepParams &sp, bool gate, cudaStream_t st);
// Sets a batch graph's rebuild condition for one step from the pending
// rebuild flag, and counts the rebuild pipelines it lets run.
int launch_rebuild_condition(const WorldDev &w, cudaGraphConditionalHandle rebuild, cudaStream_t st);
// One step of a looped batch graph: the rebuild condition and the loop's
// condition (another step while active and fewer than `steps` begun).
int launch_step_condition(const WorldDev &w, cudaGraphConditionalHandle rebuild, cudaGraphConditionalHandle loop,
                          uint32_t steps, cudaStream_t st);
int launch_fiber_update(const WorldDev &w, const LaunchPlan &lp, const StepParams &sp, cudaStream_t st);
// Sets *flag (device) when a staged coordinate is not finite.
int launch_stage_nonfinite(const WorldDev &w, unsigned int *flag, cudaStream_t st);
int launch_positions_from_stage(const WorldDev &w, cudaStream_t st);
int launch_positions_to_stage(const WorldDev &w, cudaStream_t st);
int launch_corrections_to_stage(const WorldDev &w, float *corr6, float *pen, cudaStream_t st);

void plan_launches(const WorldDev &w, LaunchPlan &lp);

}  // namespace tgl
