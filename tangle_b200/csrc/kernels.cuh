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
    // Verlet lists.
    uint32_t *nbr_count; // [S] true neighbor count
    uint32_t *nbr_list;  // [S * block]
    // Contact lists (allocated only when contact_skin > 0).
    uint32_t *contact_count; // [S] per slot; above contact_block = use the Verlet list
    uint32_t *contact_list;  // [S * contact_block] per slot, ascending segment order
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
};

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

// Launch plans, fixed per world.
struct LaunchPlan {
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
    size_t lanes_smem;
    int lanes_blocks;
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
int launch_fiber_update(const WorldDev &w, const LaunchPlan &lp, const StepParams &sp, cudaStream_t st);
int launch_positions_from_stage(const WorldDev &w, cudaStream_t st);
int launch_positions_to_stage(const WorldDev &w, cudaStream_t st);
int launch_corrections_to_stage(const WorldDev &w, float *corr6, float *pen, cudaStream_t st);

void plan_launches(const WorldDev &w, LaunchPlan &lp);

}  // namespace tgl
