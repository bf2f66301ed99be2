/*
 * relax_oracle.h -- CPU restatement of TANGLE's plain relaxation path.
 *
 * TEST INFRASTRUCTURE ONLY. This oracle is the checker for the CUDA path in
 * tangle_b200/ and the timed CPU baseline of bench.py. Nothing in the product
 * library links, imports or calls it.
 *
 * It restates, operation by operation and in f32 with no FMA contraction,
 * the CubeCL kernels of the reference (SueHeir/tangle):
 *   crates/tangle_contact/src/device/cell_list.rs   (proxy_cell, cell list)
 *   crates/tangle_contact/src/device/neighbor.rs    (Verlet lists)
 *   crates/tangle_contact/src/device/contact.rs     (find_segment_corrections)
 *   crates/tangle_relax/src/device/kernels.rs       (internal, apply, curvature,
 *                                                    reductions and the gate)
 *   crates/tangle_relax/src/device/world.rs         (upload sizing, run_batch
 *                                                    order, read_status)
 * restricted to round, non-adaptive, flexible-motion fibers.
 *
 * Pinning: the reference cannot be built here (Rust is absent and its CubeCL
 * dependency is not vendored), so bit-level agreement with the reference's
 * own CPU backend is unpinned. The oracle is pinned instead against every
 * known-answer test the reference holds for this path
 * (crates/tangle_relax/src/device/world_tests.rs and
 * crates/tangle_python/python/tests/test_api.py), restated in tests/.
 */
#ifndef TANGLE_RELAX_ORACLE_H
#define TANGLE_RELAX_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Non-adaptive PackedAssembly subset (packed.rs:49-112). Arrays are
 * borrowed and copied; interleaved xyz for positions. */
typedef struct {
    uint32_t vertex_count;
    uint32_t segment_count;
    uint32_t fiber_count;
    uint32_t reserved;
    const float *positions;            /* 3V */
    const float *intrinsic_positions;  /* 3V */
    const uint32_t *segment_vertices;  /* 2S */
    const uint32_t *segment_fibers;    /* S */
    const float *segment_radii;        /* S */
    const float *segment_rest_lengths; /* S */
    const uint32_t *fiber_vertex_spans;  /* 2F: start, count */
    const uint32_t *fiber_segment_spans; /* 2F: start, count */
    const uint32_t *vertex_segments;   /* 2V: previous, next (UINT32_MAX) */
    const float *vertex_max_curvature; /* V */
    const uint32_t *vertex_pinned;     /* V, may be NULL */
    float cell_lower[3];
    float cell_upper[3];
    uint32_t cell_periodic[3];
    uint32_t reserved2;
} orc_packed;

/* CellListConfig (tangle_contact/src/lib.rs:15-40) plus the neighbor-list
 * byte cap (world.rs:36, 120 MiB in the reference). */
typedef struct {
    float cell_size_scale;
    float neighbor_skin_scale;
    uint32_t neighbor_capacity;
    uint32_t reserved;
    uint64_t max_list_bytes;
} orc_cell_list_config;

/* RelaxationConfig fields the plain path reads (plugin.rs:77-175). */
typedef struct {
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
    uint32_t contact_aggregation; /* 0 average, 1 penetration weighted, 2 deepest */
    uint32_t force_full_iterations;
    uint32_t motion_model;        /* FiberMotion (plugin.rs:30-44): 0 flexible, 1 rigid translation */
    uint32_t reserved;
} orc_relax_config;

/* BatchStatus (world.rs:91-114). */
typedef struct {
    uint64_t total_iterations;
    uint64_t batch_iterations;
    float max_penetration;
    float max_displacement;
    float max_curvature_ratio;
    uint32_t converged;
    uint32_t cell_list_overflow;
    uint32_t reserved;
} orc_batch_status;

typedef struct orc_world orc_world;

int orc_world_create(const orc_packed *packed, const orc_cell_list_config *cell_list,
                     float max_step, orc_world **out);
void orc_world_destroy(orc_world *world);
int orc_run_batch(orc_world *world, const orc_relax_config *config, uint32_t iterations,
                  orc_batch_status *status);
int orc_download_positions(const orc_world *world, float *xyz, size_t len);
int orc_upload_positions(orc_world *world, const float *xyz, size_t len);
float orc_cell_size(const orc_world *world);
uint64_t orc_cell_count(const orc_world *world);
void orc_cell_dims(const orc_world *world, uint32_t dims[3]);
float orc_neighbor_skin(const orc_world *world);
uint32_t orc_neighbor_block(const orc_world *world);
uint32_t orc_neighbor_list_rebuilds(const orc_world *world);
/* Curvature triplet projections that moved a vertex, since creation. */
uint64_t orc_curvature_projections(const orc_world *world);
void orc_set_threads(int threads);

/* Parity taps. Each rebuilds nothing; they copy the current state out. */
int orc_debug_cell_list(const orc_world *world, uint32_t *cell_counts, uint32_t *cell_offsets,
                        uint32_t *cell_segments);
/* counts[S] (true counts) and lists[S*block] (first min(count, block) entries,
 * sorted for non-overflowed lists). */
int orc_debug_neighbor_lists(const orc_world *world, uint32_t *counts, uint32_t *lists);
/* One contact pass on the current positions and lists, without moving
 * anything: corrections[6S], segment_max_penetration[S]. */
int orc_debug_corrections(orc_world *world, const orc_relax_config *config,
                          float *corrections, float *segment_max_penetration);
/* Forces a neighbor-list rebuild from the current positions now. */
int orc_debug_rebuild(orc_world *world);
/* Formation hooks (world.rs:1723-2194; kernels.rs:164-221, 538-923); the
 * same meanings as the tgl_world_* functions of include/tangle_cuda.h. */
int orc_set_active_fibers(orc_world *world, const uint8_t *active, uint64_t fiber_count,
                          uint32_t *active_segments, uint32_t *active_vertices);
int orc_set_layer_targets(orc_world *world, uint32_t axis, const float *targets, uint32_t count,
                          const uint32_t *fiber_layers, uint32_t first_layer, uint32_t last_layer,
                          float stiffness, float max_translation, int apply_now);
int orc_set_vertex_targets(orc_world *world, uint32_t axis, const uint32_t *vertices, uint32_t count,
                           float displacement, float stiffness, float max_translation);
int orc_vertex_target_state(const orc_world *world, float *coordinates, float *command_coordinates,
                            uint32_t count);
int orc_target_errors(const orc_world *world, float *layer_error, uint32_t *has_layer,
                      float *vertex_error, uint32_t *has_vertex);
int orc_compact_cell(orc_world *world, const float new_lower[3], const float new_upper[3],
                     uint32_t kinematics);
int orc_cell_bounds(const orc_world *world, float lower[3], float upper[3]);
int orc_compaction_metrics(const orc_world *world, float correction_fraction, const float stiffness[3],
                           float out[13]);
int orc_wall_reactions(const orc_world *world, float *xyz, size_t len);
int orc_set_fiber_max_curvatures(orc_world *world, const float *values, size_t count);
/* The f32 arc cosine the curvature projection uses (see relax_oracle.cpp). */
float orc_acos_f32(float x);
const char *orc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
