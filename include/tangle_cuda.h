/*
 * tangle_cuda.h -- C ABI of the B200 (sm_100a) relaxation backend.
 *
 * This library is the "cuda" implementation of TANGLE's relaxation seam: the
 * `RelaxationBackend` / `DeviceWorld` enum of the reference
 * (crates/tangle_relax/src/device/plugin.rs:15-28, :309-893), whose every
 * method forwards to `DeviceFiberWorld<R>`
 * (crates/tangle_relax/src/device/world.rs). Each entry point below names the
 * reference method it replaces. A Rust host binds these with `extern "C"`
 * declarations; Python binds them with ctypes (tangle_b200/device.py).
 *
 * Conventions (all entry points):
 *   - return 0 on success, a nonzero TGL_ERR_* code on failure, never throw;
 *     tgl_last_error() gives the calling thread's last message;
 *   - host arrays are borrowed for the duration of the call and copied;
 *   - a world handle is driven from one thread at a time (one handle per
 *     thread is fine); kernels of one call are asynchronous and the call
 *     returns after its single status readback, like the reference's
 *     run_batch + read_status.
 * Scope: round sections, non-adaptive layouts, flexible motion -- the plain
 * relaxation path. Positions are f32 in metres, interleaved xyz.
 */
#ifndef TANGLE_CUDA_H
#define TANGLE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TGL_OK 0
#define TGL_ERR_INVALID 1     /* bad argument or assembly */
#define TGL_ERR_CUDA 2        /* a CUDA runtime call failed */
#define TGL_ERR_NO_DEVICE 3   /* no usable sm_100 device */
#define TGL_ERR_MEMORY 4      /* device allocation failed */
#define TGL_ERR_UNSUPPORTED 5 /* a setting outside the plain path */

/* Non-adaptive PackedAssembly subset
 * (crates/tangle_relax/src/device/packed.rs:49-112, packing :150-320).
 * Fibers must be packed as the reference packs them: a fiber's vertices are
 * consecutive, its segments are consecutive, and its k-th segment joins its
 * k-th and (k+1)-th vertices. */
typedef struct {
    uint32_t vertex_count;
    uint32_t segment_count;
    uint32_t fiber_count;
    uint32_t reserved;
    const float *positions;              /* 3V placed xyz */
    const float *intrinsic_positions;    /* 3V rest-shape xyz */
    const uint32_t *segment_vertices;    /* 2S */
    const uint32_t *segment_fibers;      /* S */
    const float *segment_radii;          /* S */
    const float *segment_rest_lengths;   /* S */
    const uint32_t *fiber_vertex_spans;  /* 2F: first vertex, count */
    const uint32_t *fiber_segment_spans; /* 2F: first segment, count */
    const uint32_t *vertex_segments;     /* 2V: previous, next (UINT32_MAX) */
    const float *vertex_max_curvature;   /* V: 0 = unrestricted */
    const uint32_t *vertex_pinned;       /* V: nonzero = pinned; NULL = none */
    float cell_lower[3];
    float cell_upper[3];
    uint32_t cell_periodic[3];
    uint32_t reserved2;
} tgl_packed;

/* CellListConfig (crates/tangle_contact/src/lib.rs:15-40) plus the cap on the
 * neighbor-list buffer: 0 keeps the reference's 120 MiB
 * (crates/tangle_relax/src/device/world.rs:35-36). The cap only chooses
 * which segments use the exact cell-scan fallback, never which contacts
 * are found. */
typedef struct {
    float cell_size_scale;     /* >= 1, default 1 */
    float neighbor_skin_scale; /* >= 0, default 2 (x largest radius) */
    uint32_t neighbor_capacity;/* > 0, default 48 slots per segment */
    uint32_t reserved;
    uint64_t max_list_bytes;   /* 0 = 120 MiB */
} tgl_cell_list_config;

/* RelaxationConfig fields the plain path reads
 * (crates/tangle_relax/src/device/plugin.rs:77-175, defaults :145-175). */
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
    uint32_t contact_aggregation;   /* 0 uniform average, 1 penetration weighted, 2 deepest only */
    uint32_t force_full_iterations; /* nonzero: ignore the tolerances */
    uint32_t motion_model;          /* FiberMotion (plugin.rs:30-44): 0 flexible, 1 rigid translation */
    uint32_t reserved;
} tgl_relax_config;

/* BatchStatus (crates/tangle_relax/src/device/world.rs:91-114). */
typedef struct {
    uint64_t total_iterations;
    uint64_t batch_iterations;
    float max_penetration;
    float max_displacement;
    float max_curvature_ratio;
    uint32_t converged;
    uint32_t cell_list_overflow;
    uint32_t reserved;
} tgl_batch_status;

typedef struct tgl_world tgl_world;

/* DeviceFiberWorld::upload (world.rs:308-690; DeviceWorld::upload,
 * plugin.rs:325-356). Copies every array to the current CUDA device, sizes
 * the cell grid and neighbor lists exactly as the reference does, and marks
 * the lists stale so the first contact pass builds them. */
int tgl_world_create(const tgl_packed *packed, const tgl_cell_list_config *cell_list, float max_step,
                     tgl_world **out);

/* Drop of the world (frees every device buffer and captured graph). */
void tgl_world_destroy(tgl_world *world);

/* Batched relaxation (no reference counterpart: the reference relaxes one
 * world at a time). Packs `count` specimens into one arena: their vertices,
 * segments, fibers and cells concatenated in order (specimen i's vertex v
 * is arena vertex v + the vertex counts of specimens 0..i-1), each with its
 * own box, cell grid, neighbor skin, lists and control word, sized exactly
 * as tgl_world_create sizes it alone. tgl_run_batch then advances every
 * specimen in one captured graph; each specimen's gate stops it on its own
 * (its convergence mask), as a batch of its own world would, and the batch
 * status covers all of them (largest counts and metrics; converged when all
 * are). One neighbor-list block serves every specimen: the capacity within
 * max_list_bytes (8 GiB when 0). Contact lists are on as in a single world
 * (TGL_CONTACT_SKIN), one contact skin for all specimens (a tenth of the
 * smallest neighbor skin) and a refresh flag per specimen; fibers of at
 * most 256 vertices. Checkpoints, residuals and the warm start take single
 * worlds. */
int tgl_arena_create(const tgl_packed *specimens, uint32_t count, const tgl_cell_list_config *cell_list,
                     float max_step, tgl_world **out);
/* Each specimen's status after the last batch (statuses[count]). */
int tgl_arena_status(tgl_world *world, const tgl_relax_config *config, tgl_batch_status *statuses, uint32_t count);

/* DeviceFiberWorld::checkpoint (world.rs:758-823; plugin.rs:393-404) for the
 * plain path: the persistent state a restart needs, which is the current
 * positions (interleaved xyz, len = 3 * vertex_count) and the lifetime
 * iteration count. Scratch (cell and neighbor lists, corrections, gate
 * metrics) is rebuilt by the first batch after a restore, as in the
 * reference. */
int tgl_world_checkpoint(tgl_world *world, float *xyz, size_t len, uint64_t *total_iterations);

/* DeviceFiberWorld::restore (world.rs:693-756; plugin.rs:358-391): uploads
 * `packed` (whose positions are the checkpoint's) as tgl_world_create does,
 * and continues the lifetime iteration count from `total_iterations`, which
 * must fit in 32 bits as the reference's control word requires. */
int tgl_world_restore(const tgl_packed *packed, const tgl_cell_list_config *cell_list, float max_step,
                      uint64_t total_iterations, tgl_world **out);

/* DeviceFiberWorld::run_batch + read_status (world.rs:1020-1505,
 * :2337-2369; DeviceWorld::run_batch, plugin.rs:407-418): up to `iterations`
 * corrections plus one measure-only pass, stopping on the device as soon as
 * the tolerances are met, then one status readback. */
int tgl_run_batch(tgl_world *world, const tgl_relax_config *config, uint32_t iterations,
                  tgl_batch_status *status);

/* DeviceFiberWorld::download_positions (world.rs:2384-2390;
 * plugin.rs:519-530): interleaved xyz, len == 3V floats. */
int tgl_download_positions(tgl_world *world, float *xyz, size_t len);

/* Replaces the resident positions (host -> device), as the reference's
 * host-side operations between batches do (layer targets, needling); the
 * next batch's displacement check requests a list rebuild if needed. */
int tgl_upload_positions(tgl_world *world, const float *xyz, size_t len);

/* DeviceWorld::cell_size / cell_count (plugin.rs:597-636). */
float tgl_cell_size(const tgl_world *world);
uint64_t tgl_cell_count(const tgl_world *world);
/* Cells per axis (world.rs:412-414). */
void tgl_cell_dims(const tgl_world *world, uint32_t dims[3]);
/* Neighbor skin = skin scale x largest radius (world.rs:356). */
float tgl_neighbor_skin(const tgl_world *world);
/* Slots per segment list after the byte cap (world.rs:914-916). */
uint32_t tgl_neighbor_block(const tgl_world *world);
/* DeviceFiberWorld::neighbor_list_rebuilds (world/neighbor_list.rs:167-176). */
int tgl_neighbor_list_rebuilds(tgl_world *world, uint32_t *rebuilds);

/* Contact lists (no reference counterpart: an internal second level under
 * the Verlet lists that changes no result). Each cell-list slot keeps the
 * entries of its segment's Verlet list that lie within `contact_skin` of
 * touching at a snapshot of the positions, in the Verlet list's order; the
 * contact pass reads them instead of the Verlet list until some vertex moves
 * more than contact_skin / 2 from the snapshot or the Verlet lists are
 * rebuilt. The skin is 0.1 of the neighbor skin unless the environment
 * variable TGL_CONTACT_SKIN, read when a world is created, gives another
 * fraction in (0, 1] (0 turns them off); they are also off when a periodic
 * box edge is under about four segment lengths plus four radii, and every
 * pass reads the Verlet lists while some segment is stretched that far.
 * Reports the skin (0 when off), the entries per slot, and the refreshes
 * done so far. */
int tgl_contact_list_info(tgl_world *world, float *contact_skin, uint32_t *block, uint32_t *refreshes);

/* DeviceFiberWorld::capture_contacts (world.rs:2195-2335) with
 * capture_segment_contacts (crates/tangle_contact/src/device/contact.rs:9-230):
 * every pair of segments of different fibers whose surfaces are at most
 * `maximum_surface_gap` apart (negative gaps are overlaps), found on a
 * whole-segment cell grid of cell size + gap. Writes up to `capacity` pairs
 * (segments[2 i], segments[2 i + 1], first < second), their closest-point
 * parameters (coordinates[2 i] on the first, [2 i + 1] on the second), the
 * surface gaps and the crossing angles (radians, in [0, pi / 2]), sorted by
 * (first, second, s, t); *count is the number written and *overflow is 1
 * when more pairs existed. The next batch rebuilds the neighbor lists, as
 * in the reference (the capture reuses their cell buffers). */
int tgl_capture_contacts(tgl_world *world, float maximum_surface_gap, uint32_t capacity, uint32_t *segments,
                         float *coordinates, float *surface_gaps, float *crossing_angles, uint32_t *count,
                         uint32_t *overflow);

/* ---- Formation hooks (single worlds; an arena returns TGL_ERR_UNSUPPORTED). */

/* DeviceFiberWorld::activate_formation_step (world.rs:2139-2183;
 * kernels.rs:164-221; plugin.rs:783-795) with the step comparison done by
 * the caller: active[f] != 0 makes fiber f take part in every later kernel
 * (cell list, contact pass, update, measurements), 0 freezes it where it is.
 * A world starts with every fiber active. Requests a neighbor-list rebuild;
 * writes the active segment and vertex counts. */
int tgl_world_set_active_fibers(tgl_world *world, const uint8_t *active, uint64_t fiber_count,
                                uint32_t *active_segments, uint32_t *active_vertices);

/* A persistent formation layer target (apply_layer_targets /
 * apply_single_layer_target, world.rs:1723-1804; kernels.rs:538-581): each
 * active fiber whose layer lies in [first_layer, last_layer] and below
 * `count` moves along `axis` so that its mean coordinate approaches
 * targets[layer] by `stiffness` (in (0, 1]), at most `max_translation`
 * (> 0) per application; applied once at once when `apply_now` is 1, and at
 * the end of every update step until cleared. fiber_layers[f] is fiber f's
 * layer, 0xFFFFFFFF for none. */
typedef struct {
    uint32_t axis;
    uint32_t count;
    const float *targets;
    const uint32_t *fiber_layers;
    uint32_t first_layer;
    uint32_t last_layer;
    float stiffness;
    float max_translation;
    uint32_t apply_now;
    uint32_t reserved;
} tgl_layer_targets;

/* Installs (targets != NULL) or clears (NULL; clear_layer_targets,
 * world.rs:1806-1810) the layer target. */
int tgl_world_set_layer_targets(tgl_world *world, const tgl_layer_targets *targets);

/* Persistent vertex displacement targets (apply_vertex_displacement_targets,
 * world.rs:1811-1859; kernels.rs:583-634): each listed vertex (distinct
 * indices) gets the target coordinate = its current coordinate along `axis`
 * + `displacement` (finite, non-zero), and at the end of every update step
 * its coordinate is set to a commanded value that advances toward the target
 * by `stiffness` (in (0, 1]), at most `max_translation` (> 0) per step. With
 * `coordinates` and `command_coordinates` given (a restore), those are the
 * targets and commands instead. */
typedef struct {
    uint32_t axis;
    uint32_t count;
    const uint32_t *vertices;
    float displacement;
    float stiffness;
    float max_translation;
    uint32_t reserved;
    const float *coordinates;
    const float *command_coordinates;
} tgl_vertex_targets;

/* Installs (targets != NULL) or clears (NULL; clear_vertex_targets,
 * world.rs:1861-1863) the vertex targets. */
int tgl_world_set_vertex_targets(tgl_world *world, const tgl_vertex_targets *targets);

/* The installed vertex targets' target and commanded coordinates (count ==
 * the installed count), for a checkpoint (world.rs:260-279). */
int tgl_world_vertex_target_state(tgl_world *world, float *coordinates, float *command_coordinates, uint32_t count);

/* formation_target_error (world.rs:1865-1929): the largest distance of an
 * active targeted fiber's centre from its layer target, and of an active
 * targeted vertex from its target; has_layer / has_vertex say which targets
 * are installed (the error is 0 when not). */
int tgl_world_target_errors(tgl_world *world, float *layer_error, uint32_t *has_layer, float *vertex_error,
                            uint32_t *has_vertex);

/* compact_cell (world.rs:1931-2054; kernels.rs:712-818): the cell shrinks
 * to [new_lower, new_upper] (inside the current cell, every edge above two
 * largest radii) and the active fibers follow by `kinematics`: 0 rigid fiber
 * centres (each fiber keeps its centre's fractional position), 1 moving
 * walls (vertices projected inside the new walls, the projection recorded
 * as wall reactions), 2 affine (every vertex scaled with the cell). The grid
 * keeps its cell size with fewer cells; a list rebuild is requested. */
int tgl_world_compact_cell(tgl_world *world, const float new_lower[3], const float new_upper[3],
                           uint32_t kinematics);

/* cell_bounds (world.rs:2133-2137). */
int tgl_world_cell_bounds(tgl_world *world, float lower[3], float upper[3]);

/* compaction_metrics + wall_face_pressures (world.rs:2056-2131;
 * kernels.rs:820-923) for the last batch's state: out[0..3] pressure per
 * axis, out[3] contact, out[4] stretch, out[5] bending, out[6] total penalty
 * energy, out[7..13] lower/upper face pressure per axis. stiffness = {contact,
 * stretch, bending} (each >= 0); correction_fraction > 0. The sums run in
 * f64 in a fixed order over the reference's f32 terms. */
int tgl_world_compaction_metrics(tgl_world *world, float correction_fraction, const float stiffness[3],
                                 float out[13]);

/* The wall reactions of the last update step (interleaved xyz, len == 3V),
 * and their replacement (a restore, world.rs:693-712). */
int tgl_world_wall_reactions(tgl_world *world, float *xyz, size_t len);
int tgl_world_set_wall_reactions(tgl_world *world, const float *xyz, size_t len);

/* set_fiber_maximum_curvatures (world.rs:2185-2194): every vertex of fiber f
 * (its ends included) takes the limit values[f] (1 / length; 0 = none). */
int tgl_world_set_fiber_max_curvatures(tgl_world *world, const float *values, size_t count);

/* Parity taps (no reference counterpart beyond its tests' readbacks,
 * world_tests.rs:1342-1363). Forces a neighbor-list rebuild from the current
 * positions now. */
int tgl_debug_rebuild(tgl_world *world);
/* Cell list in cell order: counts and exclusive offsets [cell_count], and the
 * segment in every slot [S] (ascending segment within each cell). */
int tgl_debug_cell_list(tgl_world *world, uint32_t *cell_counts, uint32_t *cell_offsets,
                        uint32_t *cell_segments);
/* True neighbor counts [S] and lists [S * block], segment-major; lists of
 * segments whose count exceeds the block are not meaningful. */
int tgl_debug_neighbor_lists(tgl_world *world, uint32_t *counts, uint32_t *lists);
/* Contact lists as the contact pass stores them: a state per cell-list slot
 * [S] -- the slot's list length, 0xFFFFFFFE where its list ran past its
 * batch's chunk (the pass reads the Verlet list) or 0xFFFFFFFF where the
 * Verlet list overflowed (the pass scans the cells) -- and the chunks
 * [ceil(S / 32) * 32 * block]: the 32 slots of batch b (slots 32b to
 * 32b + 31) keep their lists back to back, in slot order, from entry
 * 32b * block on; `chunks` may be null (the states alone).
 * TGL_ERR_UNSUPPORTED when contact lists are off. */
int tgl_debug_contact_lists(tgl_world *world, uint32_t *states, uint32_t *chunks);
/* One contact pass (find_segment_corrections, contact.rs:232-902) on the
 * current positions and lists, moving nothing: corrections [6S] and
 * per-segment maximum penetration [S]. */
int tgl_debug_corrections(tgl_world *world, const tgl_relax_config *config, float *corrections,
                          float *segment_max_penetration);

/* Number of kernels this world has launched since creation (graph-replayed
 * launches included); used to report the bench's launch count. */
uint64_t tgl_kernel_launches(const tgl_world *world);

/* Per-kernel device time of the last batch, from CUDA events recorded
 * around every step's kernels when timing is enabled (measurement support;
 * no reference counterpart). Steps whose kernels returned at once (after
 * convergence) are excluded. */
typedef struct {
    double contact_ms;      /* summed over contact passes that ran */
    double update_ms;       /* summed over fiber updates that ran */
    double rebuild_ms;      /* summed over neighbor-list rebuilds that ran */
    uint32_t contact_passes;
    uint32_t updates;
    uint32_t rebuilds;
    uint32_t reserved;
} tgl_kernel_times;

/* ---- Launch parameters and their autotuner (no reference counterpart: the
 * reference's CubeCL kernels take fixed launch shapes). None of these
 * parameters changes a result: every choice gives the same positions, bit
 * for bit, and the same gate decisions; they only move time between
 * kernels. */
typedef struct {
    uint32_t lanes_per_fiber;       /* lanes per fiber in the curvature sweeps: 2, 4, 8 or 32 */
    uint32_t contact_blocks_per_sm; /* contact-pass blocks per SM (256 threads each): 1, 2 or 3 */
    uint32_t build_chunk;           /* candidate slots a Verlet-build block stages at once: 512 to 4096 */
    float contact_skin_fraction;    /* contact-list skin over the neighbor skin: 0 (lists off) or (0, 1];
                                       above 0 only where the world allocated contact lists */
    uint32_t update_warps_per_block; /* warps per fiber-update block: 1, 2 or 4 (fewer where one warp's
                                        staged fibers times this exceed 200 KB of shared memory) */
    uint32_t reserved[3];
} tgl_launch_params;

int tgl_world_get_launch_params(tgl_world *world, tgl_launch_params *params);
/* Applies `params` (validated first); the next batch recaptures its graph
 * and refreshes the contact lists. */
int tgl_world_set_launch_params(tgl_world *world, const tgl_launch_params *params);

typedef struct {
    uint32_t trials;            /* timed trial batches run */
    uint32_t trial_iterations;  /* iterations per trial batch */
    float default_ms;           /* the parameters the world had, per trial batch */
    float best_ms;              /* the chosen parameters, per trial batch */
} tgl_autotune_report;

/* Searches the launch parameters one at a time (coordinate descent over the
 * candidate sets above, starting from the world's current ones), timing
 * each candidate with CUDA events on a batch of `trial_iterations`
 * iterations of `config` (force_full_iterations implied), best of two after
 * one untimed batch that captures its graph. Every trial starts from the
 * world's state at the call: positions, last steps, formation commands and
 * control words are saved first and restored after each trial and at the
 * end, and the next batch rebuilds the neighbor lists, so the positions
 * that follow are those the world would have given without the search (its
 * rebuild count is one higher). The best parameters are applied and
 * returned. */
int tgl_autotune(tgl_world *world, const tgl_relax_config *config, uint32_t trial_iterations,
                 tgl_launch_params *best, tgl_autotune_report *report);

int tgl_set_kernel_timing(tgl_world *world, int enable);
/* The cudaStream_t every kernel of this world runs on (as void*), so a
 * caller can order its own work or record CUDA events against it. */
void *tgl_world_stream(const tgl_world *world);
int tgl_last_kernel_times(tgl_world *world, tgl_kernel_times *times);

/* Inputs of tgl_contact_pass_noalloc: device pointers the caller owns. */
typedef struct {
    const float *positions;          /* device, 3V interleaved xyz */
    const uint32_t *segment_vertices;/* device, 2S */
    const uint32_t *segment_fibers;  /* device, S */
    const float *segment_radii;      /* device, S */
    const float *vertex_arc_lengths; /* device, V: rest arc length from the fiber start */
    uint32_t segment_count;          /* at most 262144 */
    uint32_t cells[3];               /* cells per axis; product at most 262144 */
    float cell_lower[3];
    float cell_upper[3];
    uint32_t cell_periodic[3];
    float correction_fraction;
    uint32_t contact_aggregation;
    uint32_t reserved;
} tgl_noalloc_inputs;

/* One contact pass for callers that cannot allocate device memory: a host
 * that manages a fixed device memory pool itself and hands this library
 * only its own buffers, or a loop that must never wait on the allocator.
 * It has no counterpart in the reference. Every candidate is found by the
 * exact 27-cell scan of the reference's cell list (the result a world of
 * neighbor_capacity 1 gives), from device arrays the caller owns, writing
 * corrections [6S] and per-segment maximum penetration [S] to device
 * buffers the caller owns. Its only working memory is a fixed 5 MiB array
 * compiled into this library (so every GPU that loads it holds that array
 * until the process exits); it calls no allocator. Limits: 262144 segments
 * and 262144 cells; larger inputs are rejected with TGL_ERR_UNSUPPORTED.
 * The kernels are queued on `stream` (a cudaStream_t, NULL = default) and
 * the call returns without waiting. The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) with that device current,
 * and so does the first call after that device's context was replaced (a
 * cudaDeviceReset, say); make those calls before any stream capture. Each
 * axis of `cells` and their product must be at most 262144; the check runs
 * before anything is queued. All calls share the one
 * array: two calls whose kernels overlap on the GPU (different streams, or
 * different host threads) race and corrupt each other's results. */
int tgl_contact_pass_noalloc(const tgl_noalloc_inputs *inputs, float *corrections, float *segment_max_penetration,
                             void *stream);

/* ---- Learned warm start (no reference counterpart: an addition on top of
 * the plain method, which stays the drop-in and runs after it to the same
 * gates). */

/* One BF16 matrix product on the tensor cores (tcgen05.mma, f32 accumulate
 * in tensor memory): D[m x n] = sum_k A[m, k] B[n, k], then + bias[n],
 * then max(0, .) when relu, stored as f32 (out_f32[i * ldo + j]) and/or
 * bf16 (out_bf16[i * ldo_bf16 + j]). A and B are device bf16 arrays, each
 * K-major (A[i * lda + k]) or MN-major (A[k * lda + i]); n is a multiple of
 * 16 in [16, 256]; leading dimensions are multiples of 8, and so is k when
 * an operand is K-major; pointers are 16-byte aligned. With k_split > 0
 * (a multiple of 64) the contraction is split over CTAs and split s writes
 * its partial product to out_f32 + s * m * ldo (no bias, relu or bf16).
 * `error` (device u32, may be null) is set to 1 if a wait for the tensor
 * cores gave up. Queued on `stream`; returns without waiting. */
typedef struct tgl_gemm {
    const void *a;
    const void *b;
    int64_t lda, ldb;
    int32_t m, n;
    int64_t k;
    int32_t a_mn, b_mn;
    int64_t k_split;
    const float *bias;
    int32_t relu, reserved;
    const void *mask;         /* bf16 [m x ld_mask]: zero the result where mask <= 0 (after relu) */
    int64_t ld_mask;
    const float *residual;    /* f32 [m x ld_res]: added last */
    int64_t ld_res;
    float *out_f32;
    int64_t ldo;
    void *out_bf16;
    int64_t ldo_bf16;
    unsigned int *error;
} tgl_gemm;
int tgl_gemm_bf16(const tgl_gemm *gemm, void *stream);

/* The contact graph of a world for message passing: nodes are vertices;
 * edges are directed segment pairs (dst <- src) whose gap is within a
 * cutoff, both directions of every pair present, grouped by destination
 * segment (CSR `offsets`) and by ascending source within one. All pointers
 * are device memory owned by the world (valid until its next graph build). */
typedef struct tgl_mp_graph {
    int32_t vertex_count, segment_count, edge_count, reserved;
    const int32_t *seg_v0;   /* [S] first vertex of each segment (the second is the next) */
    const int32_t *links;    /* [4 V] previous vertex, next vertex, segment before, segment after; -1 = none */
    const int32_t *offsets;  /* [S + 1] */
    const int32_t *dst, *src, *twin;  /* [E]; twin = the reverse edge */
    const float *s, *t;      /* [E] closest-point parameters on dst / src */
} tgl_mp_graph;

/* Device buffers a contact graph is written into (sizes: V vertices, S
 * segments, E edges). */
typedef struct tgl_mp_graph_out {
    int32_t *seg_v0;       /* [S] */
    int32_t *links;        /* [4 V] */
    int32_t *offsets;      /* [S + 1] */
    int32_t *dst, *src, *twin;  /* [E] */
    float *s, *t;          /* [E] */
    void *node_features;   /* bf16 [V x 16] */
    void *edge_features;   /* bf16 [E x 16] */
} tgl_mp_graph_out;

/* The contact graph of the world's current positions, in two calls: the
 * first rebuilds the neighbor lists from the positions and counts the
 * edges (pairs of the Verlet lists whose closest-point gap is at most
 * `cutoff`, both directions); the second, with the same world and nothing
 * run in between, writes the graph and its features into `out`:
 * node features (unit tangent, curvature x d, rest curvature x d,
 * d / 10 um, overlap depth / d, and the push: the depth-weighted unit
 * normals away from the vertex's contacts / d) and edge features
 * (closest-point offset / d,
 * overlap depth / d, s, t), each padded with zeros to 16. Both wait for
 * completion. */
int tgl_warmstart_graph_count(tgl_world *world, float cutoff, int64_t *edge_count);
/* Restricts the next contact graphs to pairs with a segment on a focus fiber
 * (fiber_focus[f] nonzero; one flag per fiber), as for a ply deposited on a
 * relaxed stack, whose proposal moves only its own fibers; NULL restores
 * every pair. Nodes stay every vertex. */
int tgl_warmstart_set_focus(tgl_world *world, const uint8_t *fiber_focus, size_t fibers);
int tgl_warmstart_graph_fill(tgl_world *world, const tgl_mp_graph_out *out);

/* Moves every unpinned vertex by scale * dx[v * ld .. v * ld + 2] (device
 * f32; times the vertex's fiber diameter when in_diameters), each move
 * capped at max_step, walls respected; queued on the world's stream. The
 * next batch's displacement checks see the move. */
int tgl_world_displace(tgl_world *world, const float *dx, int64_t ld, float scale, int32_t in_diameters,
                       float max_step);

/* The residual of the current positions without moving them (one contact
 * pass on lists valid for them): maximum penetration, maximum curvature
 * ratio, and the sum over segments of their deepest penetration divided by
 * their diameter. */
int tgl_world_residual(tgl_world *world, const tgl_relax_config *config, float *max_penetration,
                       float *max_curvature_ratio, float *total_penetration);

/* Message-passing steps over a graph, hidden width 64, queued on `stream`.
 * x_edge[e, 0:64] = bf16((1 - t_e) h[first vertex of src] + t_e h[second]). */
int tgl_mp_edge_inputs(const tgl_mp_graph *graph, const float *h, void *x_edge, int64_t ld_x, void *stream);
/* x_node[v] (bf16, 192 wide) = [h_v, the mean of the messages m (f32
 * [E x 64]) into the vertex's two segments weighted by the vertex's share
 * (1 - s or s; divided by the total share, at least 1), mean of the fiber
 * neighbors' h]. */
int tgl_mp_node_inputs(const tgl_mp_graph *graph, const float *h, const float *m, void *x_node, void *stream);
/* Backward of tgl_mp_node_inputs: dh (f32 [V x 64]) += the h and
 * neighbor-mean parts of dx_node (f32 [V x 192]); dm (bf16 [E x 64], and
 * f32 when dm_f32 is not null) = the message gradient. */
int tgl_mp_node_inputs_backward(const tgl_mp_graph *graph, const float *dx_node, float *dh, void *dm, float *dm_f32,
                                void *stream);
/* dst (bf16) = src (f32), n elements. */
int tgl_convert_bf16(int64_t n, const float *src, void *dst, void *stream);
/* Backward of tgl_mp_edge_inputs: dh += the shares of dx_edge[:, 0:64]. */
int tgl_mp_edge_inputs_backward(const tgl_mp_graph *graph, const float *dx_edge, int64_t ld_dx, float *dh,
                                void *stream);
/* out[j] (+)= sum_i x[i * ld + j] for j < n, in a fixed order; scratch holds
 * tgl_column_sums_scratch(rows, n) floats. */
int64_t tgl_column_sums_scratch(int64_t rows, int32_t n);
int tgl_column_sums(const float *x, int64_t rows, int32_t n, int64_t ld, float *out, int32_t accumulate,
                    float *scratch, void *stream);
/* One Adam step (bias-corrected; step counts from 1) on n f32 weights, and
 * their bf16 copy when w_bf16 is not null. */
int tgl_adam_step(int64_t n, float *w, const float *g, float *m, float *v, void *w_bf16, float lr, float beta1,
                  float beta2, float eps, int32_t step, void *stream);
/* Mean squared error of y[:, 0:cols] against target [rows x cols] into
 * *loss, and dy = its gradient (f32 and/or bf16, zero past cols); scratch
 * holds 1024 floats. */
int tgl_mse(int64_t rows, const float *y, int64_t ld_y, const float *target, int32_t cols, float *loss, float *dy,
            int64_t ld_dy, void *dy_bf16, float *scratch, void *stream);

/* Thread-local message of the last failed call on this thread. */
const char *tgl_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
