// world.cu -- the resident relaxation world behind the C ABI of
// include/tangle_cuda.h: upload and grid sizing
// (crates/tangle_relax/src/device/world.rs:308-690, :874-917), batches
// (run_batch, world.rs:1020-1505) replayed from captured CUDA graphs, and
// the single status readback (read_status, world.rs:2337-2369).
#include <cuda_runtime.h>

#include <cmath>
#include <algorithm>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/tangle_cuda.h"
#include "kernels.cuh"
#include "warmstart.cuh"

using namespace tgl;

namespace {

thread_local std::string g_error;
constexpr uint64_t REFERENCE_MAX_LIST_BYTES = 120ull << 20;  // world.rs:36
constexpr uint32_t CONTACT_BLOCK = 32;  // contact-list entries per slot

int set_error(int code, const std::string &message) {
    g_error = message;
    return code;
}

#define TGL_CUDA(call)                                                                               \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess)                                                                       \
            return set_error(TGL_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));       \
    } while (0)

uint32_t f32_to_u32_host(float x) {
    if (x != x || x <= 0.0f) return 0;
    if (x >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)x;
}

// The cell count of a grid, or 0 when the grid is unusable: an axis with no
// cell or more than 2^30 cells (proxy_cell and stencil_cell wrap periodic
// axes in i32 as (raw % n + n) % n, which stays below 2^31 only then), or a
// product above `limit`. The product is checked after every factor, so it
// cannot wrap (a factor is at most 2^30 and the running product at most
// `limit` <= 2^32 before it).
uint64_t checked_cell_count(const uint32_t cells[3], uint64_t limit) {
    uint64_t C = 1;
    for (int a = 0; a < 3; ++a) {
        if (cells[a] == 0 || cells[a] > (1u << 30)) return 0;
        C *= cells[a];
        if (C > limit) return 0;
    }
    return C;
}

struct GraphKey {
    uint32_t iterations;
    StepParams sp;
    bool operator<(const GraphKey &o) const {
        if (iterations != o.iterations) return iterations < o.iterations;
        return std::memcmp(&sp, &o.sp, sizeof(StepParams)) < 0;
    }
};

struct GraphEntry {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;      // kernels per replay (a looped graph: those before its loop)
    bool looped = false;  // one WHILE node over a step (4 kernels per step that ran)
    uint32_t iterations = 0;
    // With kernel timing on: four events per step (before the rebuild,
    // before the contact pass, before the fiber update, after it).
    std::vector<cudaEvent_t> events;
};

void destroy_entry(GraphEntry &e) {
    if (e.exec) cudaGraphExecDestroy(e.exec);
    if (e.graph) cudaGraphDestroy(e.graph);
    for (cudaEvent_t ev : e.events) cudaEventDestroy(ev);
    e.exec = nullptr;
    e.graph = nullptr;
    e.events.clear();
}

}  // namespace

namespace tgl {
// Sets the calling thread's tgl_last_error() message (used by noalloc.cu).
void set_last_error(const std::string &message) { g_error = message; }
}  // namespace tgl

// Scratch of the warm-start contact graph (counts, offsets, overlap depths),
// grown on demand; the graph itself goes to the caller's buffers.
struct WarmGraph {
    GraphBuffers b{};
    int32_t *offsets = nullptr;  // [S + 1]
    float *depth = nullptr;      // [depth_capacity]
    int64_t depth_capacity = 0;
    float *residual = nullptr;   // [2]
    uint32_t *focus = nullptr;   // [F] focus flags (b.fiber_focus points here while a focus is set)
    int64_t edges = 0;
    float cutoff = 0.0f;
    bool ready = false, counted = false;

    ~WarmGraph() {
        cudaFree(focus);
        cudaFree(b.fwd_count);
        cudaFree(b.in_count);
        cudaFree(b.fill);
        cudaFree(b.block_sums);
        cudaFree(offsets);
        cudaFree(depth);
        cudaFree(residual);
    }
};

struct tgl_world {
    int device = 0;
    cudaStream_t stream = nullptr;
    // Batch graphs skip gated-off steps with conditional nodes (driver and
    // runtime 12.8 or later), their bodies captured on body_stream.
    cudaStream_t body_stream = nullptr;
    bool conditional = false;
    // Batch graphs loop on the device (a WHILE node over one step) unless
    // kernel timing, which needs events per step, is on.
    cudaStream_t loop_stream = nullptr;
    bool loop = false;
    uint32_t rebuild_bodies_seen = 0;
    WorldDev dev{};
    LaunchPlan lp{};
    float cell_size = 0.0f;
    uint64_t neighbor_slots = 0;
    Control *host_ctl = nullptr;  // pinned
    std::vector<void *> allocations;
    std::map<GraphKey, GraphEntry> graphs;
    uint64_t launches = 0;
    bool timing = false;
    bool arena = false;
    uint32_t specimens = 1;
    const GraphEntry *last = nullptr;  // graph of the last batch
    uint64_t last_batch_iterations = 0;
    WarmGraph warm;
    // Formation state (single worlds): the host's copy of the fiber layout,
    // the active flags, and the device buffers of the targets, the
    // compaction metrics and the target errors.
    std::vector<uint2> h_vspan;
    std::vector<uint32_t> h_s0;
    std::vector<uint32_t> h_active;
    uint32_t *fiber_order_d = nullptr;
    uint32_t *fiber_on_d = nullptr;
    float4 *vtx_static_d = nullptr;
    uint32_t *fiber_layer_d = nullptr;
    float *layer_target_d = nullptr;
    uint32_t layer_capacity = 0;
    int32_t *vertex_target_d = nullptr;
    uint32_t *target_vertices_d = nullptr, *target_fibers_d = nullptr;
    float *target_coord_d = nullptr, *command_coord_d = nullptr;
    uint32_t target_capacity = 0, target_count = 0;
    std::vector<uint32_t> h_target_vertices;
    unsigned int *error_bits_d = nullptr;
    unsigned int *nonfinite_d = nullptr;  // upload check flag
    double *metric_partials_d = nullptr;
    float *metric_out_d = nullptr;
    uint64_t allocated_cells = 0;
    float maximum_radius = 0.0f, maximum_length = 0.0f;  // over every specimen
    float contact_fraction = 0.0f;  // contact-list skin over the neighbor skin (0: lists off)
    // What sizes the contact skin: the smallest neighbor skin and every
    // specimen's grid (one of each for a single world).
    float contact_skin_base = 0.0f;
    std::vector<Grid> contact_grids;

    ~tgl_world() {
        for (auto &kv : graphs) destroy_entry(kv.second);
        for (void *p : allocations) cudaFree(p);
        if (host_ctl) cudaFreeHost(host_ctl);
        if (stream) cudaStreamDestroy(stream);
        if (body_stream) cudaStreamDestroy(body_stream);
        if (loop_stream) cudaStreamDestroy(loop_stream);
    }

    template <typename T>
    int alloc(T **out, size_t count) {
        void *p = nullptr;
        size_t bytes = count * sizeof(T);
        if (bytes == 0) bytes = sizeof(T);
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess)
            return set_error(TGL_ERR_MEMORY, std::string("cudaMalloc of ") + std::to_string(bytes) +
                                                 " bytes failed: " + cudaGetErrorString(e));
        allocations.push_back(p);
        *out = (T *)p;
        return 0;
    }

    template <typename T>
    int upload(T **out, const std::vector<T> &host) {
        if (int rc = alloc(out, host.size())) return rc;
        if (!host.empty()) TGL_CUDA(cudaMemcpy(*out, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice));
        return 0;
    }
};

namespace {

StepParams step_params(const tgl_relax_config &c, uint32_t iterations) {
    StepParams sp{};
    sp.penetration_tolerance = c.penetration_tolerance;
    sp.correction_fraction = c.correction_fraction;
    sp.stretch_stiffness = c.stretch_stiffness;
    sp.bend_stiffness = c.bend_stiffness;
    sp.curvature_limit_stiffness = c.curvature_limit_stiffness;
    sp.curvature_limit_safety_margin = c.curvature_limit_safety_margin;
    sp.curvature_ratio_tolerance = c.curvature_ratio_tolerance;
    sp.max_step = c.max_step;
    sp.constraint_iterations = c.constraint_iterations;
    sp.curvature_cleanup_sweeps = c.curvature_cleanup_sweeps;
    sp.contact_aggregation = c.contact_aggregation;
    sp.force_full_iterations = c.force_full_iterations ? 1u : 0u;
    sp.motion_model = c.motion_model;
    sp.max_iterations = iterations;
    return sp;
}

// plugin.rs:951-983 assertions on the solver configuration.
int validate_config(const tgl_relax_config &c) {
    if (!(c.penetration_tolerance >= 0.0f)) return set_error(TGL_ERR_INVALID, "penetration_tolerance must be non-negative");
    if (!(c.correction_fraction > 0.0f && c.correction_fraction <= 1.0f))
        return set_error(TGL_ERR_INVALID, "correction_fraction must be in (0, 1]");
    if (!(c.stretch_stiffness >= 0.0f && c.stretch_stiffness <= 1.0f))
        return set_error(TGL_ERR_INVALID, "stretch_stiffness must be in [0, 1]");
    if (!(c.bend_stiffness >= 0.0f && c.bend_stiffness <= 1.0f))
        return set_error(TGL_ERR_INVALID, "bend_stiffness must be in [0, 1]");
    if (!(c.curvature_limit_stiffness >= 0.0f && c.curvature_limit_stiffness <= 1.0f))
        return set_error(TGL_ERR_INVALID, "curvature_limit_stiffness must be in [0, 1]");
    if (!(c.curvature_limit_safety_margin >= 0.0f && c.curvature_limit_safety_margin < 0.1f))
        return set_error(TGL_ERR_INVALID, "curvature_limit_safety_margin must be in [0, 0.1)");
    if (!(c.curvature_ratio_tolerance >= 0.0f)) return set_error(TGL_ERR_INVALID, "curvature_ratio_tolerance must be non-negative");
    if (c.constraint_iterations == 0) return set_error(TGL_ERR_INVALID, "constraint_iterations must be positive");
    if (c.curvature_cleanup_sweeps == 0) return set_error(TGL_ERR_INVALID, "curvature_cleanup_sweeps must be positive");
    if (c.motion_model > 1) return set_error(TGL_ERR_INVALID, "motion_model must be 0 (flexible) or 1 (rigid translation)");
    if (!(c.max_step > 0.0f)) return set_error(TGL_ERR_INVALID, "max_step must be positive");
    if (c.contact_aggregation > 2) return set_error(TGL_ERR_INVALID, "contact_aggregation must be 0, 1 or 2");
    return 0;
}

// The graph a stream is capturing into.
static cudaError_t capture_graph(cudaStream_t st, cudaGraph_t *graph) {
    cudaStreamCaptureStatus status;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &status, nullptr, graph, nullptr, nullptr);
    if (e != cudaSuccess) return e;
    return status == cudaStreamCaptureStatusActive ? cudaSuccess : cudaErrorStreamCaptureInvalidated;
}

// Appends an IF node on `handle` (with an ELSE body when `size` is 2) after
// the capture's current dependencies and makes it the capture's only
// dependency; its bodies come back in `bodies`.
static cudaError_t append_conditional(cudaStream_t st, cudaGraphConditionalHandle handle, cudaGraphConditionalNodeType type,
                                      unsigned size, cudaGraph_t *bodies) {
    cudaStreamCaptureStatus status;
    cudaGraph_t graph = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(st, &status, nullptr, &graph, &deps, &ndeps);
    if (e != cudaSuccess) return e;
    cudaGraphNodeParams params{};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = type;
    params.conditional.size = size;
    cudaGraphNode_t node;
    if ((e = cudaGraphAddNode(&node, graph, deps, ndeps, &params)) != cudaSuccess) return e;
    for (unsigned i = 0; i < size; ++i) bodies[i] = params.conditional.phGraph_out[i];
    return cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
}

static cudaError_t append_if(cudaStream_t st, cudaGraphConditionalHandle handle, unsigned size, cudaGraph_t *bodies) {
    return append_conditional(st, handle, cudaGraphCondTypeIf, size, bodies);
}

// Captures `enqueue(stream)` into a conditional body on `st`.
template <typename F>
static cudaError_t capture_body_on(cudaStream_t st, cudaGraph_t body, F enqueue) {
    cudaError_t e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    cudaError_t inner = enqueue(st);
    cudaGraph_t out = nullptr;
    e = cudaStreamEndCapture(st, &out);
    return inner != cudaSuccess ? inner : e;
}

template <typename F>
static cudaError_t capture_body(tgl_world *w, cudaGraph_t body, F enqueue) {
    return capture_body_on(w->body_stream, body, [&](cudaStream_t st) {
        enqueue(st);
        return cudaSuccess;
    });
}

// One step's rebuild as a conditional node: a kernel sets the condition
// from the pending-rebuild flag and an IF node runs the rebuild pipeline
// only then, so the eleven gated-off launches are not made at all (every
// kernel keeps its own test). The contact pass stays two gated launches:
// an IF/ELSE node between them measured slower than the launch it saves.
static cudaError_t enqueue_conditional_rebuild(tgl_world *w, int *kernels) {
    cudaGraph_t graph = nullptr;
    cudaError_t e = capture_graph(w->stream, &graph);
    if (e != cudaSuccess) return e;
    cudaGraphConditionalHandle rebuild = 0;
    if ((e = cudaGraphConditionalHandleCreate(&rebuild, graph, 0, 0)) != cudaSuccess) return e;
    *kernels += launch_rebuild_condition(w->dev, rebuild, w->stream);
    cudaGraph_t body = nullptr;
    if ((e = append_if(w->stream, rebuild, 1, &body)) != cudaSuccess) return e;
    return capture_body(w, body, [&](cudaStream_t st) { launch_rebuild(w->dev, w->lp, st); });
}

// run_batch's launch sequence (world.rs:1020-1505): begin, displacement
// check, then iterations + 1 steps of [rebuild if flagged, contact pass with
// the gate, fiber update]; kernels after the gate return at once once it
// has stopped the batch. Returns the kernels launched every time the graph
// runs, or -1 with the error set.
int enqueue_batch(tgl_world *w, const StepParams &sp, uint32_t iterations, std::vector<cudaEvent_t> *events) {
    int kernels = 0;
    kernels += launch_begin_batch(w->dev, w->lp, w->stream);
    kernels += launch_flag_displacement(w->dev, w->lp, w->stream);
    kernels += launch_measure_start(w->dev, w->lp, w->stream);
    for (uint32_t step = 0; step <= iterations; ++step) {
        if (events) cudaEventRecordWithFlags((*events)[4 * step], w->stream, cudaEventRecordExternal);
        if (w->conditional) {
            cudaError_t e = enqueue_conditional_rebuild(w, &kernels);
            if (e != cudaSuccess) {
                set_error(TGL_ERR_CUDA, std::string("conditional graph node: ") + cudaGetErrorString(e));
                return -1;
            }
        } else {
            kernels += launch_rebuild(w->dev, w->lp, w->stream);
        }
        if (events) cudaEventRecordWithFlags((*events)[4 * step + 1], w->stream, cudaEventRecordExternal);
        kernels += launch_contact(w->dev, w->lp, sp, true, w->stream);
        if (events) cudaEventRecordWithFlags((*events)[4 * step + 2], w->stream, cudaEventRecordExternal);
        kernels += launch_fiber_update(w->dev, w->lp, sp, w->stream);
        if (events) cudaEventRecordWithFlags((*events)[4 * step + 3], w->stream, cudaEventRecordExternal);
    }
    return kernels;
}

// run_batch's loop on the device: begin, displacement check and start
// metrics, then one WHILE node whose body is one step -- the step condition
// (rebuild flag, and whether another step follows), an IF node holding the
// rebuild pipeline, the contact pass with the gate and the fiber update. The
// gate in the contact pass ends the loop (the residual check); at most
// iterations + 1 steps run, as in the unrolled graph, whose steps after the
// gate stops are launches that return at once. Returns the kernels launched
// before the loop, or -1 with the error set.
int enqueue_batch_loop(tgl_world *w, const StepParams &sp, uint32_t iterations) {
    int kernels = 0;
    kernels += launch_begin_batch(w->dev, w->lp, w->stream);
    kernels += launch_flag_displacement(w->dev, w->lp, w->stream);
    kernels += launch_measure_start(w->dev, w->lp, w->stream);
    cudaGraph_t graph = nullptr;
    cudaError_t e = capture_graph(w->stream, &graph);
    cudaGraphConditionalHandle loop = 0;
    cudaGraph_t body = nullptr;
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&loop, graph, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) e = append_conditional(w->stream, loop, cudaGraphCondTypeWhile, 1, &body);
    if (e == cudaSuccess)
        e = capture_body_on(w->loop_stream, body, [&](cudaStream_t st) -> cudaError_t {
            cudaGraph_t step_graph = nullptr;
            cudaError_t f = capture_graph(st, &step_graph);
            cudaGraphConditionalHandle rebuild = 0;
            if (f == cudaSuccess) f = cudaGraphConditionalHandleCreate(&rebuild, step_graph, 0, 0);
            if (f != cudaSuccess) return f;
            launch_step_condition(w->dev, rebuild, loop, iterations + 1, st);
            cudaGraph_t rebuild_body = nullptr;
            if ((f = append_if(st, rebuild, 1, &rebuild_body)) != cudaSuccess) return f;
            if ((f = capture_body(w, rebuild_body, [&](cudaStream_t bs) { launch_rebuild(w->dev, w->lp, bs); })) !=
                cudaSuccess)
                return f;
            launch_contact(w->dev, w->lp, sp, true, st);
            launch_fiber_update(w->dev, w->lp, sp, st);
            return cudaGetLastError();
        });
    if (e != cudaSuccess) {
        set_error(TGL_ERR_CUDA, std::string("looped batch graph: ") + cudaGetErrorString(e));
        return -1;
    }
    return kernels;
}

// world.rs:2337-2369 for one control word.
void status_of(const Control &h, const tgl_relax_config &c, tgl_batch_status *status) {
    bool overflow = h.cell_overflow != 0 || h.control[3] != 0;
    status->total_iterations = h.control[1];
    status->batch_iterations = h.control[2];
    status->max_penetration = h.metrics[0];
    status->max_displacement = h.metrics[1];
    status->max_curvature_ratio = h.metrics[2];
    status->converged = (!c.force_full_iterations && h.metrics[0] <= c.penetration_tolerance &&
                         h.metrics[2] <= 1.0f + c.curvature_ratio_tolerance && !overflow)
                            ? 1u
                            : 0u;
    status->cell_list_overflow = overflow ? 1u : 0u;
    status->reserved = 0;
}

// The batch status; for an arena, over all specimens: the largest
// iteration counts and metrics, converged when every specimen is.
int read_status(tgl_world *w, const tgl_relax_config &c, tgl_batch_status *status) {
    const size_t words = w->arena ? (size_t)w->specimens + 1 : 1;
    TGL_CUDA(cudaMemcpyAsync(w->host_ctl, w->dev.ctl, words * sizeof(Control), cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    if (!w->arena) {
        status_of(*w->host_ctl, c, status);
        return 0;
    }
    tgl_batch_status total{};
    total.converged = 1;
    for (uint32_t p = 0; p < w->specimens; ++p) {
        tgl_batch_status one{};
        status_of(w->host_ctl[1 + p], c, &one);
        total.total_iterations = std::max(total.total_iterations, one.total_iterations);
        total.batch_iterations = std::max(total.batch_iterations, one.batch_iterations);
        total.max_penetration = std::fmax(total.max_penetration, one.max_penetration);
        total.max_displacement = std::fmax(total.max_displacement, one.max_displacement);
        total.max_curvature_ratio = std::fmax(total.max_curvature_ratio, one.max_curvature_ratio);
        total.converged &= one.converged;
        total.cell_list_overflow |= one.cell_list_overflow;
    }
    *status = total;
    return 0;
}

}  // namespace

extern "C" {

const char *tgl_last_error(void) { return g_error.c_str(); }

namespace {

// One specimen prepared on the host: sizing and static data, its indices
// local to the specimen.
struct HostSpecimen {
    uint32_t V = 0, S = 0, F = 0, max_fiber = 0;
    float cell_size = 0.0f, skin = 0.0f, maximum_radius = 0.0f, maximum_length = 0.0f;
    Grid grid{};
    uint64_t C = 0, neighbor_slots = 0;
    uint32_t block = 0;
    std::vector<float4> vtx_static, seg_static, geom, pos;
    std::vector<uint32_t> pinned, seg_v0, fiber_s0;
    std::vector<uint2> fiber_vspan;
    std::vector<float> rest, rest_curvature;
    std::vector<int4> links;
};

// Upload validation (world.rs:314-319) and the layout the reference's
// packing produces (packed.rs:200-248).
int validate_packed(const tgl_packed *pk, const tgl_cell_list_config *cl, float max_step, HostSpecimen &h) {
    const uint32_t V = pk->vertex_count, S = pk->segment_count, F = pk->fiber_count;
    // world.rs:314-319 upload assertions.
    if (S == 0 || F == 0) return set_error(TGL_ERR_INVALID, "assembly has no segments or fibers");
    if (!(cl->cell_size_scale >= 1.0f)) return set_error(TGL_ERR_INVALID, "cell_size_scale must be at least 1");
    if (!(std::isfinite(cl->neighbor_skin_scale) && cl->neighbor_skin_scale >= 0.0f))
        return set_error(TGL_ERR_INVALID, "neighbor_skin_scale must be finite and non-negative");
    if (cl->neighbor_capacity == 0) return set_error(TGL_ERR_INVALID, "neighbor_capacity must be positive");
    if (!(max_step > 0.0f)) return set_error(TGL_ERR_INVALID, "max_step must be positive");
    if (!pk->positions || !pk->intrinsic_positions || !pk->segment_vertices || !pk->segment_fibers ||
        !pk->segment_radii || !pk->segment_rest_lengths || !pk->fiber_vertex_spans || !pk->fiber_segment_spans ||
        !pk->vertex_segments || !pk->vertex_max_curvature)
        return set_error(TGL_ERR_INVALID, "a required packed array is null");
    for (int a = 0; a < 3; ++a)
        if (!(std::isfinite(pk->cell_lower[a]) && std::isfinite(pk->cell_upper[a]) && pk->cell_upper[a] > pk->cell_lower[a]))
            return set_error(TGL_ERR_INVALID, "cell bounds must be finite with upper > lower");
    // The layout the reference's packing produces (packed.rs:200-248).
    uint64_t vsum = 0, ssum = 0;
    uint32_t &max_fiber = h.max_fiber;
    max_fiber = 0;
    for (uint32_t f = 0; f < F; ++f) {
        uint32_t v0 = pk->fiber_vertex_spans[2 * f], n = pk->fiber_vertex_spans[2 * f + 1];
        uint32_t s0 = pk->fiber_segment_spans[2 * f], m = pk->fiber_segment_spans[2 * f + 1];
        if (n < 2 || m != n - 1 || (uint64_t)v0 + n > V || (uint64_t)s0 + m > S)
            return set_error(TGL_ERR_INVALID, "fiber " + std::to_string(f) + " has an invalid vertex or segment span");
        for (uint32_t k = 0; k < m; ++k) {
            uint32_t s = s0 + k;
            if (pk->segment_vertices[2 * s] != v0 + k || pk->segment_vertices[2 * s + 1] != v0 + k + 1 ||
                pk->segment_fibers[s] != f)
                return set_error(TGL_ERR_INVALID, "segment " + std::to_string(s) +
                                                      " is not packed as its fiber's consecutive vertex pair");
        }
        for (uint32_t k = 0; k < n; ++k) {
            uint32_t v = v0 + k;
            uint32_t prev = k > 0 ? s0 + k - 1 : TGL_NONE, next = k + 1 < n ? s0 + k : TGL_NONE;
            if (pk->vertex_segments[2 * v] != prev || pk->vertex_segments[2 * v + 1] != next)
                return set_error(TGL_ERR_INVALID, "vertex_segments disagrees with the fiber packing at vertex " +
                                                      std::to_string(v));
        }
        vsum += n;
        ssum += m;
        if (n > max_fiber) max_fiber = n;
    }
    if (vsum != V || ssum != S) return set_error(TGL_ERR_INVALID, "fiber spans do not cover every vertex and segment once");
    for (uint64_t i = 0; i < 3ull * V; ++i)
        if (!std::isfinite(pk->positions[i]) || !std::isfinite(pk->intrinsic_positions[i]))
            return set_error(TGL_ERR_INVALID, "positions must be finite");
    for (uint32_t s = 0; s < S; ++s)
        if (!(pk->segment_radii[s] > 0.0f) || !std::isfinite(pk->segment_radii[s]) || !std::isfinite(pk->segment_rest_lengths[s]))
            return set_error(TGL_ERR_INVALID, "segment radii must be positive and finite");
    if ((size_t)max_fiber * 3 * sizeof(float4) > 200 * 1024)
        return set_error(TGL_ERR_UNSUPPORTED, "a fiber has more vertices than one warp can stage in shared memory");

    return 0;
}

// world.rs:321-417 sizing and the static per-segment / per-vertex records.
int prepare_specimen(const tgl_packed *pk, const tgl_cell_list_config *cl, float max_step, HostSpecimen &h) {
    const uint32_t V = pk->vertex_count, S = pk->segment_count, F = pk->fiber_count;
    h.V = V;
    h.S = S;
    h.F = F;
    // ---- world.rs:321-417: grid sizing for a uniform layout, in f32.
    const float *P = pk->positions;
    float maximum_rest_length = 0.0f, maximum_initial_length = 0.0f, maximum_radius = 0.0f;
    for (uint32_t s = 0; s < S; ++s) {
        maximum_rest_length = std::fmax(maximum_rest_length, pk->segment_rest_lengths[s]);
        uint32_t a = pk->segment_vertices[2 * s], b = pk->segment_vertices[2 * s + 1];
        float dx = P[3 * b] - P[3 * a], dy = P[3 * b + 1] - P[3 * a + 1], dz = P[3 * b + 2] - P[3 * a + 2];
        maximum_initial_length = std::fmax(maximum_initial_length, std::sqrt(dx * dx + dy * dy + dz * dz));
        maximum_radius = std::fmax(maximum_radius, pk->segment_radii[s]);
    }
    float maximum_length = std::fmax(maximum_rest_length, maximum_initial_length);
    float skin = cl->neighbor_skin_scale * maximum_radius;
    float interaction_margin = 2.0f * maximum_radius + std::fmax(2.0f * max_step, skin);
    // Every segment is a leaf: one proxy piece and list weight 1 each.
    float piece_length = std::fmin(maximum_length, std::fmax(maximum_length, 2.0f * interaction_margin));
    h.cell_size = (piece_length + interaction_margin) * cl->cell_size_scale;
    Grid grid{};
    for (int a = 0; a < 3; ++a) {
        grid.lower[a] = pk->cell_lower[a];
        grid.upper[a] = pk->cell_upper[a];
        grid.periodic[a] = pk->cell_periodic[a] ? 1u : 0u;
        float extent = pk->cell_upper[a] - pk->cell_lower[a];
        grid.cells[a] = f32_to_u32_host(std::fmax(std::floor(extent / h.cell_size), 1.0f));
        grid.length[a] = extent;
        grid.width[a] = extent / (float)grid.cells[a];
        grid.inv_length[a] = 1.0f / extent;
    }
    const uint64_t C = checked_cell_count(grid.cells, 1ull << 31);
    if (C == 0 || !(h.cell_size > 0.0f))
        return set_error(TGL_ERR_UNSUPPORTED, "cell grid too large: the cell size is tiny against the box");
    // world.rs:476-509 and :874-917: list room and the byte cap.
    uint64_t max_bytes = cl->max_list_bytes ? cl->max_list_bytes : REFERENCE_MAX_LIST_BYTES;
    uint64_t slots = std::min<uint64_t>((uint64_t)cl->neighbor_capacity * S, max_bytes / 4);
    h.neighbor_slots = std::max<uint64_t>(slots, 1);
    uint32_t block = (uint32_t)std::min<uint64_t>(cl->neighbor_capacity, std::min<uint64_t>(h.neighbor_slots / S, 0xFFFFFFFFull));

    // ---- static per-segment and per-vertex data.
    std::vector<float> arc(V, 0.0f);  // packed.rs:561-580
    std::vector<float4> &vtx_static = h.vtx_static;
    vtx_static.resize(V);
    std::vector<uint32_t> &pinned = h.pinned;
    pinned.assign(V, 0);
    std::vector<uint2> &fiber_vspan = h.fiber_vspan;
    fiber_vspan.resize(F);
    std::vector<uint32_t> &fiber_s0 = h.fiber_s0;
    fiber_s0.resize(F);
    const float *X = pk->intrinsic_positions;
    for (uint32_t f = 0; f < F; ++f) {
        uint32_t v0 = pk->fiber_vertex_spans[2 * f], n = pk->fiber_vertex_spans[2 * f + 1];
        fiber_vspan[f] = make_uint2(v0, n);
        fiber_s0[f] = pk->fiber_segment_spans[2 * f];
        double total = 0.0;
        for (uint32_t v = v0 + 1; v < v0 + n; ++v) {
            double sum = 0.0;
            for (int a = 0; a < 3; ++a) {
                double delta = (double)X[3 * (size_t)v + a] - (double)X[3 * (size_t)(v - 1) + a];
                sum += delta * delta;
            }
            total += std::sqrt(sum);
            arc[v] = (float)total;
        }
        float radius = pk->segment_radii[fiber_s0[f]];  // packed.rs:527-546
        for (uint32_t k = 0; k < n; ++k) {
            uint32_t v = v0 + k;
            // Rest chords to the second neighbors (kernels.rs:1118-1121,
            // :1149-1152), rounded exactly as the kernel computes them.
            float chord_prev = 0.0f, chord_next = 0.0f;
            if (k >= 2) {
                uint32_t o = v - 2;
                float rx = X[3 * o] - X[3 * v], ry = X[3 * o + 1] - X[3 * v + 1], rz = X[3 * o + 2] - X[3 * v + 2];
                chord_prev = std::sqrt(rx * rx + ry * ry + rz * rz);
            }
            if (k + 2 < n) {
                uint32_t o = v + 2;
                float rx = X[3 * o] - X[3 * v], ry = X[3 * o + 1] - X[3 * v + 1], rz = X[3 * o + 2] - X[3 * v + 2];
                chord_next = std::sqrt(rx * rx + ry * ry + rz * rz);
            }
            vtx_static[v] = make_float4(pk->vertex_max_curvature[v], chord_prev, chord_next, radius);
            pinned[v] = pk->vertex_pinned && pk->vertex_pinned[v] ? 1u : 0u;
        }
    }
    std::vector<float4> &seg_static = h.seg_static;
    seg_static.resize(S);
    std::vector<uint32_t> &seg_v0 = h.seg_v0;
    seg_v0.resize(S);
    h.rest.assign(pk->segment_rest_lengths, pk->segment_rest_lengths + S);
    std::vector<float4> &geom = h.geom;
    geom.resize(2 * (size_t)S);
    for (uint32_t s = 0; s < S; ++s) {
        uint32_t a = pk->segment_vertices[2 * s], b = pk->segment_vertices[2 * s + 1];
        uint32_t fiber = pk->segment_fibers[s];
        float fb;
        std::memcpy(&fb, &fiber, 4);
        seg_static[s] = make_float4(pk->segment_radii[s], arc[a], arc[b], fb);
        seg_v0[s] = a;
        float dx = P[3 * b] - P[3 * a], dy = P[3 * b + 1] - P[3 * a + 1], dz = P[3 * b + 2] - P[3 * a + 2];
        geom[2 * (size_t)s] = make_float4(P[3 * a], P[3 * a + 1], P[3 * a + 2], pk->segment_radii[s]);
        geom[2 * (size_t)s + 1] = make_float4(P[3 * b], P[3 * b + 1], P[3 * b + 2], 0.5f * std::sqrt(dx * dx + dy * dy + dz * dz));
    }
    std::vector<float4> &pos = h.pos;
    pos.resize(V);
    for (uint32_t v = 0; v < V; ++v) pos[v] = make_float4(P[3 * v], P[3 * v + 1], P[3 * v + 2], 0.0f);
    // Fiber links and the rest shape's discrete curvature (warm-start
    // features; curvature.rs:21-55 form, f64 on the host).
    std::vector<int4> &links = h.links;
    links.resize(V);
    std::vector<float> &rest_curvature = h.rest_curvature;
    rest_curvature.assign(V, 0.0f);
    for (uint32_t f = 0; f < F; ++f) {
        const uint32_t v0 = fiber_vspan[f].x, n = fiber_vspan[f].y, s0 = fiber_s0[f];
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t v = v0 + k;
            links[v] = make_int4(k > 0 ? (int)(v - 1) : -1, k + 1 < n ? (int)(v + 1) : -1,
                                 k > 0 ? (int)(s0 + k - 1) : -1, k + 1 < n ? (int)(s0 + k) : -1);
            if (k > 0 && k + 1 < n) {
                double u[3], w3[3], lu = 0.0, lw = 0.0, dot = 0.0;
                for (int a = 0; a < 3; ++a) {
                    u[a] = (double)X[3 * (size_t)v + a] - (double)X[3 * (size_t)(v - 1) + a];
                    w3[a] = (double)X[3 * (size_t)(v + 1) + a] - (double)X[3 * (size_t)v + a];
                    lu += u[a] * u[a];
                    lw += w3[a] * w3[a];
                    dot += u[a] * w3[a];
                }
                lu = std::sqrt(lu);
                lw = std::sqrt(lw);
                if (lu > 0.0 && lw > 0.0) {
                    double c = std::fmax(-1.0, std::fmin(1.0, dot / (lu * lw)));
                    rest_curvature[v] = (float)(2.0 * std::sqrt(0.5 * (1.0 - c)) / (0.5 * (lu + lw)));
                }
            }
        }
    }

    h.skin = skin;
    h.maximum_radius = maximum_radius;
    h.maximum_length = maximum_length;
    h.grid = grid;
    h.C = C;
    h.block = block;
    return 0;
}

}  // namespace

namespace {

void set_contact_skin(tgl_world *w, float fraction);

// Device world from prepared specimens: one (a single world) or several (an
// arena, relaxed together with a gate per specimen).
int build_world(std::vector<HostSpecimen> &hosts, const tgl_cell_list_config *cl, bool arena, tgl_world **out) {
    int device_count = 0;
    if (cudaGetDeviceCount(&device_count) != cudaSuccess || device_count == 0)
        return set_error(TGL_ERR_NO_DEVICE, "no CUDA device");

    tgl_world *w = new tgl_world();
    auto fail = [&](int rc) {
        delete w;
        return rc;
    };
    cudaGetDevice(&w->device);
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, w->device);
    if (prop.major < 10) return fail(set_error(TGL_ERR_NO_DEVICE, "the relaxation kernels are built for sm_100a"));
    if (cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&w->body_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&w->loop_stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(set_error(TGL_ERR_CUDA, "cudaStreamCreate failed"));
    {
        int driver = 0, runtime = 0;
        w->conditional = cudaDriverGetVersion(&driver) == cudaSuccess && cudaRuntimeGetVersion(&runtime) == cudaSuccess &&
                         driver >= 12080 && runtime >= 12080 && std::getenv("TGL_NO_CONDITIONAL_GRAPHS") == nullptr;
        w->loop = w->conditional && std::getenv("TGL_NO_LOOP_GRAPHS") == nullptr;
    }
    if (cudaMallocHost(&w->host_ctl, (hosts.size() > 1 || arena ? hosts.size() + 1 : 1) * sizeof(Control)) != cudaSuccess)
        return fail(set_error(TGL_ERR_MEMORY, "cudaMallocHost failed"));

    // ---- concatenate the specimens (a single world is one specimen).
    const uint32_t count = (uint32_t)hosts.size();
    uint64_t V64 = 0, S64 = 0, F64 = 0, C64 = 0;
    uint32_t max_fiber = 0;
    for (const HostSpecimen &h : hosts) {
        V64 += h.V;
        S64 += h.S;
        F64 += h.F;
        C64 += h.C;
        max_fiber = std::max(max_fiber, h.max_fiber);
    }
    if (V64 >= 0xFFFFFFFFull || S64 >= 0xFFFFFFFFull || C64 > (1ull << 31))
        return fail(set_error(TGL_ERR_UNSUPPORTED, "arena too large for 32-bit indices"));
    const uint32_t V = (uint32_t)V64, S = (uint32_t)S64, F = (uint32_t)F64;
    const uint64_t C = C64;
    std::vector<float4> vtx_static, seg_static, geom, pos;
    std::vector<uint32_t> pinned, seg_v0, fiber_s0, seg_spec, fiber_spec, vtx_spec, cell_spec;
    std::vector<uint2> fiber_vspan;
    std::vector<float> rest, rest_curvature;
    std::vector<int4> links;
    std::vector<SpecimenDev> specs(count);
    vtx_static.reserve(V);
    uint32_t vbase = 0, sbase = 0, fbase = 0, cbase = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const HostSpecimen &h = hosts[i];
        for (uint32_t v = 0; v < h.V; ++v) {
            vtx_static.push_back(h.vtx_static[v]);
            pinned.push_back(h.pinned[v]);
            pos.push_back(h.pos[v]);
            rest_curvature.push_back(h.rest_curvature[v]);
            int4 l = h.links[v];
            links.push_back(make_int4(l.x >= 0 ? l.x + (int)vbase : -1, l.y >= 0 ? l.y + (int)vbase : -1,
                                      l.z >= 0 ? l.z + (int)sbase : -1, l.w >= 0 ? l.w + (int)sbase : -1));
            vtx_spec.push_back(i);
        }
        for (uint32_t s = 0; s < h.S; ++s) {
            float4 st = h.seg_static[s];
            uint32_t fiber;
            std::memcpy(&fiber, &st.w, 4);
            fiber += fbase;
            std::memcpy(&st.w, &fiber, 4);
            seg_static.push_back(st);
            seg_v0.push_back(h.seg_v0[s] + vbase);
            rest.push_back(h.rest[s]);
            geom.push_back(h.geom[2 * (size_t)s]);
            geom.push_back(h.geom[2 * (size_t)s + 1]);
            seg_spec.push_back(i);
        }
        for (uint32_t f = 0; f < h.F; ++f) {
            fiber_vspan.push_back(make_uint2(h.fiber_vspan[f].x + vbase, h.fiber_vspan[f].y));
            fiber_s0.push_back(h.fiber_s0[f] + sbase);
            fiber_spec.push_back(i);
        }
        for (uint64_t c = 0; c < h.C; ++c) cell_spec.push_back(i);
        SpecimenDev &sd = specs[i];
        sd.grid = h.grid;
        sd.skin = h.skin;
        sd.cell_base = cbase;
        sd.cell_count = (uint32_t)h.C;
        sd.seg_base = sbase;
        float edge = 0.0f;
        sd.build_prefilter = 1;
        for (int a = 0; a < 3; ++a) {
            if (h.grid.periodic[a] && h.grid.cells[a] < 3) sd.build_prefilter = 0;
            edge = std::max(edge, h.grid.length[a]);
        }
        sd.build_sphere_eps = 1.0e-6f * edge;
        sd.line_eps = 4.0e-6f * edge;
        vbase += h.V;
        sbase += h.S;
        fbase += h.F;
        cbase += (uint32_t)h.C;
    }
    // Fibers by descending vertex count, so a warp's fibers finish together.
    std::vector<uint32_t> fiber_order(F);
    for (uint32_t f = 0; f < F; ++f) fiber_order[f] = f;
    std::stable_sort(fiber_order.begin(), fiber_order.end(),
                     [&](uint32_t a, uint32_t b) { return fiber_vspan[a].y > fiber_vspan[b].y; });
    const HostSpecimen &h0 = hosts[0];
    w->cell_size = h0.cell_size;
    w->neighbor_slots = h0.neighbor_slots;
    uint32_t block = h0.block;
    if (arena) {
        // One list block for every specimen: the capacity, within the byte
        // cap (8 GiB unless one is given).
        uint64_t max_bytes = cl->max_list_bytes ? cl->max_list_bytes : (8ull << 30);
        uint64_t slots = std::min<uint64_t>((uint64_t)cl->neighbor_capacity * S, max_bytes / 4);
        w->neighbor_slots = std::max<uint64_t>(slots, 1);
        block = (uint32_t)std::min<uint64_t>(cl->neighbor_capacity, std::max<uint64_t>(w->neighbor_slots / S, 1));
    }
    const float skin = h0.skin;
    const Grid grid = h0.grid;
    WorldDev &d = w->dev;
    d.V = V;
    d.S = S;
    d.F = F;
    d.C = (uint32_t)C;
    d.NS = S;  // every fiber starts active
    d.FA = F;
    w->allocated_cells = C;
    w->maximum_radius = h0.maximum_radius;
    w->maximum_length = h0.maximum_length;
    w->contact_skin_base = h0.skin;
    w->contact_grids.clear();
    for (const HostSpecimen &h : hosts) {
        w->maximum_radius = std::max(w->maximum_radius, h.maximum_radius);
        w->maximum_length = std::max(w->maximum_length, h.maximum_length);
        w->contact_skin_base = std::min(w->contact_skin_base, h.skin);
        w->contact_grids.push_back(h.grid);
    }
    d.block = block;
    d.max_fiber = max_fiber;
    d.skin = skin;
    d.grid = grid;
    // Contact lists: on by default at a tenth of the skin (TGL_CONTACT_SKIN
    // sets the fraction, 0 turns them off); in an arena one contact skin
    // serves every specimen (a tenth of the smallest neighbor skin) and one
    // refresh flag covers them all.
    float contact_fraction = 0.1f;
    if (const char *env = std::getenv("TGL_CONTACT_SKIN")) contact_fraction = std::strtof(env, nullptr);
    if (!(contact_fraction > 0.0f && contact_fraction <= 1.0f) || !(w->contact_skin_base > 0.0f))
        contact_fraction = 0.0f;
    set_contact_skin(w, contact_fraction);
    d.contact_block = d.contact_skin > 0.0f ? CONTACT_BLOCK : 0u;
    int rc = 0;
    float4 *seg_static_d, *vtx_static_d;
    uint32_t *seg_v0_d, *fiber_s0_d, *pinned_d, *fiber_order_d;
    uint2 *fiber_vspan_d;
    float *rest_d, *rest_curvature_d;
    int4 *links_d;
    if ((rc = w->upload(&links_d, links)) || (rc = w->upload(&rest_curvature_d, rest_curvature)))
        return fail(rc);
    d.links = links_d;
    d.rest_curvature = rest_curvature_d;
    if ((rc = w->upload(&seg_static_d, seg_static)) || (rc = w->upload(&seg_v0_d, seg_v0)) ||
        (rc = w->upload(&fiber_vspan_d, fiber_vspan)) || (rc = w->upload(&fiber_s0_d, fiber_s0)) ||
        (rc = w->upload(&fiber_order_d, fiber_order)) ||
        (rc = w->upload(&vtx_static_d, vtx_static)) || (rc = w->upload(&pinned_d, pinned)) ||
        (rc = w->upload(&rest_d, rest)) || (rc = w->upload(&d.pos, pos)) || (rc = w->upload(&d.ref_pos, pos)) ||
        (rc = w->upload(&d.geom, geom)) || (rc = w->alloc(&d.corr, 2 * (size_t)S)) ||
        (rc = w->alloc(&d.vertex_step, V)) || (rc = w->alloc(&d.cell_counts, C)) ||
        (rc = w->alloc(&d.cell_offsets, C)) || (rc = w->alloc(&d.cell_segments, S)) ||
        (rc = w->alloc(&d.cell_box, C)) ||
        (rc = w->alloc(&d.cell_of, S)) || (rc = w->alloc(&d.ticket, S)) ||
        (rc = w->alloc(&d.slot_geom, 2 * (size_t)S)) || (rc = w->alloc(&d.slot_sphere, S)) || (rc = w->alloc(&d.nbr_count, S)) ||
        (rc = w->alloc(&d.nbr_list, std::max<uint64_t>((uint64_t)S * block, 1))) ||
        (rc = w->alloc(&d.ctl, arena ? (size_t)count + 1 : 1)) ||
        (rc = w->alloc(&d.xyz_stage, 3 * (size_t)V)))
        return fail(rc);
    if (d.contact_block &&
        ((rc = w->alloc(&d.contact_count, S)) ||
         (rc = w->alloc(&d.contact_list, (size_t)(S + 31) / 32 * 32 * d.contact_block)) ||  // whole chunks
         (rc = w->upload(&d.contact_ref, pos))))
        return fail(rc);
    d.seg_static = seg_static_d;
    d.seg_v0 = seg_v0_d;
    d.fiber_vspan = fiber_vspan_d;
    d.fiber_s0 = fiber_s0_d;
    d.fiber_order = fiber_order_d;
    d.vtx_static = vtx_static_d;
    w->fiber_order_d = fiber_order_d;
    w->vtx_static_d = vtx_static_d;
    // The update's own fiber order (chosen on the device) starts as
    // fiber_order, every fiber at zero rounds.
    if ((rc = w->upload(&d.update_order, fiber_order)) || (rc = w->alloc(&d.fiber_rounds, F)) ||
        (rc = w->alloc(&d.rounds_avg, F)))
        return fail(rc);
    if (cudaMemset(d.fiber_rounds, 0, F * sizeof(uint32_t)) != cudaSuccess ||
        cudaMemset(d.rounds_avg, 0, F * sizeof(uint32_t)) != cudaSuccess)
        return fail(set_error(TGL_ERR_CUDA, "device initialisation failed"));
    if (!arena) {
        w->h_vspan = fiber_vspan;
        w->h_s0 = fiber_s0;
        w->h_active.assign(F, 1u);
        // Wall reactions are kept when some axis has walls (on periodic
        // axes every reaction is zero).
        if (!grid.periodic[0] || !grid.periodic[1] || !grid.periodic[2]) {
            if ((rc = w->alloc(&d.reaction, V))) return fail(rc);
            if (cudaMemset(d.reaction, 0, V * sizeof(float4)) != cudaSuccess)
                return fail(set_error(TGL_ERR_CUDA, "device initialisation failed"));
        }
    }
    d.pinned = pinned_d;
    d.rest = rest_d;
    d.P = count;
    w->arena = arena;
    w->specimens = count;
    if (arena) {
        SpecimenDev *specs_d;
        uint32_t *seg_spec_d, *fiber_spec_d, *vtx_spec_d, *cell_spec_d;
        if ((rc = w->upload(&specs_d, specs)) || (rc = w->upload(&seg_spec_d, seg_spec)) ||
            (rc = w->upload(&fiber_spec_d, fiber_spec)) || (rc = w->upload(&vtx_spec_d, vtx_spec)) ||
            (rc = w->upload(&cell_spec_d, cell_spec)))
            return fail(rc);
        d.specs = specs_d;
        d.seg_spec = seg_spec_d;
        d.fiber_spec = fiber_spec_d;
        d.vtx_spec = vtx_spec_d;
        d.cell_spec = cell_spec_d;
    }
    Control ctl{};
    ctl.metrics[0] = INFINITY;  // world.rs:470
    ctl.metrics[1] = 0.0f;
    ctl.metrics[2] = INFINITY;
    ctl.neighbor_state[0] = 1;  // lists start stale (world.rs:516-517)
    ctl.contact_state[0] = 1;
    std::vector<Control> controls(arena ? count + 1 : 1, ctl);
    if (cudaMemcpy(d.ctl, controls.data(), controls.size() * sizeof(Control), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(d.corr, 0, 2 * (size_t)S * sizeof(float4)) != cudaSuccess ||
        cudaMemset(d.vertex_step, 0, V * sizeof(float)) != cudaSuccess ||
        cudaMemset(d.cell_counts, 0, C * sizeof(uint32_t)) != cudaSuccess ||
        cudaMemset(d.cell_offsets, 0, C * sizeof(uint32_t)) != cudaSuccess ||
        cudaMemset(d.nbr_count, 0, S * sizeof(uint32_t)) != cudaSuccess)
        return fail(set_error(TGL_ERR_CUDA, "device initialisation failed"));
    {  // Any permutation works before the first rebuild replaces it.
        std::vector<uint32_t> iota(S);
        for (uint32_t s = 0; s < S; ++s) iota[s] = s;
        if (cudaMemcpy(d.cell_segments, iota.data(), S * sizeof(uint32_t), cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(set_error(TGL_ERR_CUDA, "device initialisation failed"));
    }
    w->lp.arena = arena;
    plan_launches(d, w->lp);
    if (arena && !w->lp.fiber_lanes)
        return fail(set_error(TGL_ERR_UNSUPPORTED, "an arena needs fibers of at most 256 vertices"));
    *out = w;
    return 0;
}

}  // namespace

int tgl_world_create(const tgl_packed *pk, const tgl_cell_list_config *cl, float max_step, tgl_world **out) {
    if (!pk || !cl || !out) return set_error(TGL_ERR_INVALID, "null argument");
    *out = nullptr;
    std::vector<HostSpecimen> hosts(1);
    if (int rc = validate_packed(pk, cl, max_step, hosts[0])) return rc;
    if (int rc = prepare_specimen(pk, cl, max_step, hosts[0])) return rc;
    return build_world(hosts, cl, false, out);
}

int tgl_arena_create(const tgl_packed *specimens, uint32_t count, const tgl_cell_list_config *cl, float max_step,
                     tgl_world **out) {
    if (!specimens || !cl || !out || count == 0) return set_error(TGL_ERR_INVALID, "null argument or no specimens");
    *out = nullptr;
    std::vector<HostSpecimen> hosts(count);
    for (uint32_t i = 0; i < count; ++i) {
        int rc = validate_packed(&specimens[i], cl, max_step, hosts[i]);
        if (!rc) rc = prepare_specimen(&specimens[i], cl, max_step, hosts[i]);
        if (rc) return set_error(rc, "specimen " + std::to_string(i) + ": " + g_error);
    }
    return build_world(hosts, cl, true, out);
}

void tgl_world_destroy(tgl_world *w) { delete w; }

int tgl_arena_status(tgl_world *w, const tgl_relax_config *config, tgl_batch_status *statuses, uint32_t count) {
    if (!w || !config || !statuses) return set_error(TGL_ERR_INVALID, "null argument");
    if (!w->arena) return set_error(TGL_ERR_INVALID, "not an arena");
    if (count != w->specimens) return set_error(TGL_ERR_INVALID, "status array length differs from the specimen count");
    TGL_CUDA(cudaMemcpyAsync(w->host_ctl, w->dev.ctl, (count + 1) * sizeof(Control), cudaMemcpyDeviceToHost,
                             w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    for (uint32_t p = 0; p < count; ++p) status_of(w->host_ctl[1 + p], *config, &statuses[p]);
    return 0;
}

int tgl_world_checkpoint(tgl_world *w, float *xyz, size_t len, uint64_t *total_iterations) {
    if (!w || !xyz || !total_iterations) return set_error(TGL_ERR_INVALID, "null argument");
    if (w->arena) return set_error(TGL_ERR_UNSUPPORTED, "checkpoints are per specimen; an arena has several");
    if (int rc = tgl_download_positions(w, xyz, len)) return rc;
    TGL_CUDA(cudaMemcpyAsync(w->host_ctl, w->dev.ctl, sizeof(Control), cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    *total_iterations = w->host_ctl->control[1];
    return 0;
}

int tgl_world_restore(const tgl_packed *pk, const tgl_cell_list_config *cl, float max_step,
                      uint64_t total_iterations, tgl_world **out) {
    if (!out) return set_error(TGL_ERR_INVALID, "null argument");
    *out = nullptr;
    if (total_iterations > 0xFFFFFFFFull)  // world.rs:707
        return set_error(TGL_ERR_INVALID, "checkpoint iteration count exceeds u32");
    tgl_world *w = nullptr;
    if (int rc = tgl_world_create(pk, cl, max_step, &w)) return rc;
    const uint32_t lifetime = (uint32_t)total_iterations;
    cudaError_t e = cudaMemcpy(reinterpret_cast<char *>(w->dev.ctl) + offsetof(Control, control) + sizeof(uint32_t),
                               &lifetime, sizeof(uint32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        tgl_world_destroy(w);
        return set_error(TGL_ERR_CUDA, std::string("restore failed: ") + cudaGetErrorString(e));
    }
    *out = w;
    return 0;
}

int tgl_run_batch(tgl_world *w, const tgl_relax_config *config, uint32_t iterations, tgl_batch_status *status) {
    if (!w || !config || !status) return set_error(TGL_ERR_INVALID, "null argument");
    w->warm.counted = false;
    if (iterations == 0) return set_error(TGL_ERR_INVALID, "iterations must be positive");  // world.rs:1021
    if (int rc = validate_config(*config)) return rc;
    StepParams sp = step_params(*config, iterations);
    GraphKey key{iterations, sp};
    auto it = w->graphs.find(key);
    if (it == w->graphs.end()) {
        GraphEntry entry;
        entry.iterations = iterations;
        if (w->timing) {
            entry.events.resize(4 * ((size_t)iterations + 1));
            for (cudaEvent_t &ev : entry.events)
                if (cudaEventCreate(&ev) != cudaSuccess) {
                    destroy_entry(entry);
                    return set_error(TGL_ERR_CUDA, "cudaEventCreate failed");
                }
        }
        entry.looped = w->loop && !w->timing;
        TGL_CUDA(cudaStreamBeginCapture(w->stream, cudaStreamCaptureModeThreadLocal));
        entry.kernels = entry.looped ? enqueue_batch_loop(w, sp, iterations)
                                     : enqueue_batch(w, sp, iterations, w->timing ? &entry.events : nullptr);
        cudaError_t e = cudaStreamEndCapture(w->stream, &entry.graph);
        if (entry.kernels < 0) {  // the error is set
            destroy_entry(entry);
            return TGL_ERR_CUDA;
        }
        if (e != cudaSuccess) return set_error(TGL_ERR_CUDA, std::string("graph capture failed: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&entry.exec, entry.graph, 0);
        if (e != cudaSuccess) {
            destroy_entry(entry);
            return set_error(TGL_ERR_CUDA, std::string("graph instantiation failed: ") + cudaGetErrorString(e));
        }
        if (w->graphs.size() >= 16) {  // keep the cache small
            auto old = w->graphs.begin();
            if (&old->second == w->last) w->last = nullptr;
            destroy_entry(old->second);
            w->graphs.erase(old);
        }
        it = w->graphs.emplace(key, entry).first;
    }
    TGL_CUDA(cudaGraphLaunch(it->second.exec, w->stream));
    w->launches += (uint64_t)it->second.kernels;
    if (int rc = read_status(w, *config, status)) return rc;
    if (it->second.looped)  // the step condition, two contact passes, the order kernel and the update per step that ran
        w->launches += (w->lp.order_period > 0 ? 5ull : 4ull) * w->host_ctl[0].loop_step;
    if (w->conditional) {  // rebuild pipelines the graph ran (REBUILD_KERNELS each)
        const uint32_t bodies = w->host_ctl[0].rebuild_bodies;
        w->launches += (uint64_t)REBUILD_KERNELS * (bodies >= w->rebuild_bodies_seen ? bodies - w->rebuild_bodies_seen : bodies);
        w->rebuild_bodies_seen = bodies;
    }
    TGL_CUDA(cudaGetLastError());
    w->last = &it->second;
    w->last_batch_iterations = status->batch_iterations;
    return 0;
}

void *tgl_world_stream(const tgl_world *w) { return w ? (void *)w->stream : nullptr; }

int tgl_set_kernel_timing(tgl_world *w, int enable) {
    if (!w) return set_error(TGL_ERR_INVALID, "null argument");
    if ((enable != 0) != w->timing) {
        for (auto &kv : w->graphs) destroy_entry(kv.second);
        w->graphs.clear();
        w->last = nullptr;
        w->timing = enable != 0;
    }
    return 0;
}

int tgl_last_kernel_times(tgl_world *w, tgl_kernel_times *times) {
    if (!w || !times) return set_error(TGL_ERR_INVALID, "null argument");
    std::memset(times, 0, sizeof(*times));
    if (!w->last || w->last->events.empty()) return set_error(TGL_ERR_INVALID, "no timed batch: enable timing first");
    const GraphEntry &e = *w->last;
    uint32_t steps = e.iterations + 1;
    uint32_t contact_passes = (uint32_t)std::min<uint64_t>(w->last_batch_iterations + 1, steps);
    uint32_t updates = (uint32_t)std::min<uint64_t>(w->last_batch_iterations, steps);
    for (uint32_t k = 0; k < steps; ++k) {
        float rebuild = 0.0f, contact = 0.0f, update = 0.0f;
        TGL_CUDA(cudaEventElapsedTime(&rebuild, e.events[4 * k], e.events[4 * k + 1]));
        TGL_CUDA(cudaEventElapsedTime(&contact, e.events[4 * k + 1], e.events[4 * k + 2]));
        TGL_CUDA(cudaEventElapsedTime(&update, e.events[4 * k + 2], e.events[4 * k + 3]));
        times->rebuild_ms += rebuild;
        if (k < contact_passes) times->contact_ms += contact;
        if (k < updates) times->update_ms += update;
    }
    times->contact_passes = contact_passes;
    times->updates = updates;
    times->rebuilds = steps;
    return 0;
}

int tgl_download_positions(tgl_world *w, float *xyz, size_t len) {
    if (!w || !xyz) return set_error(TGL_ERR_INVALID, "null argument");
    if (len != 3 * (size_t)w->dev.V) return set_error(TGL_ERR_INVALID, "position buffer has the wrong length");
    w->launches += launch_positions_to_stage(w->dev, w->stream);
    TGL_CUDA(cudaMemcpyAsync(xyz, w->dev.xyz_stage, len * sizeof(float), cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    return 0;
}

int tgl_upload_positions(tgl_world *w, const float *xyz, size_t len) {
    if (!w || !xyz) return set_error(TGL_ERR_INVALID, "null argument");
    w->warm.counted = false;
    if (len != 3 * (size_t)w->dev.V) return set_error(TGL_ERR_INVALID, "position buffer has the wrong length");
    if (!w->nonfinite_d && w->alloc(&w->nonfinite_d, 1)) return TGL_ERR_MEMORY;
    // The coordinates are checked where they land, in the staging buffer,
    // before anything the world holds changes (no host pass over them).
    TGL_CUDA(cudaMemcpyAsync(w->dev.xyz_stage, xyz, len * sizeof(float), cudaMemcpyHostToDevice, w->stream));
    TGL_CUDA(cudaMemsetAsync(w->nonfinite_d, 0, sizeof(unsigned int), w->stream));
    w->launches += launch_stage_nonfinite(w->dev, w->nonfinite_d, w->stream);
    unsigned int nonfinite = 0;
    TGL_CUDA(cudaMemcpyAsync(&nonfinite, w->nonfinite_d, sizeof(unsigned int), cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    if (nonfinite) return set_error(TGL_ERR_INVALID, "positions must be finite");
    w->launches += launch_positions_from_stage(w->dev, w->stream);
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    return 0;
}

float tgl_cell_size(const tgl_world *w) { return w ? w->cell_size : 0.0f; }
uint64_t tgl_cell_count(const tgl_world *w) { return w ? w->dev.C : 0; }
void tgl_cell_dims(const tgl_world *w, uint32_t dims[3]) {
    for (int a = 0; a < 3; ++a) dims[a] = w ? w->dev.grid.cells[a] : 0;
}
float tgl_neighbor_skin(const tgl_world *w) { return w ? w->dev.skin : 0.0f; }
uint32_t tgl_neighbor_block(const tgl_world *w) { return w ? w->dev.block : 0; }
uint64_t tgl_kernel_launches(const tgl_world *w) { return w ? w->launches : 0; }

int tgl_neighbor_list_rebuilds(tgl_world *w, uint32_t *rebuilds) {
    if (!w || !rebuilds) return set_error(TGL_ERR_INVALID, "null argument");
    TGL_CUDA(cudaMemcpyAsync(w->host_ctl, w->dev.ctl, sizeof(Control), cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    if (!w->arena) {
        *rebuilds = w->host_ctl->neighbor_state[1];
        return 0;
    }
    TGL_CUDA(cudaMemcpyAsync(w->host_ctl, w->dev.ctl, (w->specimens + 1) * sizeof(Control), cudaMemcpyDeviceToHost,
                             w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    uint32_t total = 0;  // an arena: the specimens' rebuilds together
    for (uint32_t p = 0; p < w->specimens; ++p) total += w->host_ctl[1 + p].neighbor_state[1];
    *rebuilds = total;
    return 0;
}

int tgl_contact_list_info(tgl_world *w, float *contact_skin, uint32_t *block, uint32_t *refreshes) {
    if (!w || !contact_skin || !block || !refreshes) return set_error(TGL_ERR_INVALID, "null argument");
    TGL_CUDA(cudaMemcpyAsync(w->host_ctl, w->dev.ctl, sizeof(Control), cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    *contact_skin = w->dev.contact_skin;
    *block = w->dev.contact_block;
    *refreshes = w->host_ctl->contact_state[1];
    return 0;
}

int tgl_debug_contact_lists(tgl_world *w, uint32_t *counts, uint32_t *lists) {
    if (!w || !counts) return set_error(TGL_ERR_INVALID, "null argument");
    if (!w->dev.contact_block) return set_error(TGL_ERR_UNSUPPORTED, "contact lists are off for this world");
    const size_t S = w->dev.S, padded = (S + 31) / 32 * 32;
    TGL_CUDA(cudaMemcpyAsync(counts, w->dev.contact_count, S * 4ull, cudaMemcpyDeviceToHost, w->stream));
    if (lists)
        TGL_CUDA(cudaMemcpyAsync(lists, w->dev.contact_list, padded * w->dev.contact_block * 4ull,
                                 cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    return 0;
}

int tgl_warmstart_graph_count(tgl_world *w, float cutoff, int64_t *edge_count) {
    if (!w || !edge_count) return set_error(TGL_ERR_INVALID, "null argument");
    if (w->arena) return set_error(TGL_ERR_UNSUPPORTED, "the warm start takes one specimen");
    if (!(cutoff >= 0.0f) || !std::isfinite(cutoff)) return set_error(TGL_ERR_INVALID, "cutoff must be finite and >= 0");
    const WorldDev &d = w->dev;
    GraphBuffers &b = w->warm.b;
    if (!w->warm.ready) {
        const size_t S = d.S;
        if (cudaMalloc(&b.fwd_count, S * 4) != cudaSuccess || cudaMalloc(&b.in_count, S * 4) != cudaSuccess ||
            cudaMalloc(&b.fill, S * 4) != cudaSuccess || cudaMalloc(&w->warm.offsets, (S + 1) * 4) != cudaSuccess ||
            cudaMalloc(&b.block_sums, (S / 1024 + 2) * 4) != cudaSuccess)
            return set_error(TGL_ERR_MEMORY, "warm-start graph allocation failed");
        w->warm.ready = true;
    }
    b.offsets = w->warm.offsets;
    // Lists from the current positions, then counts and offsets.
    w->launches += launch_request_rebuild(d, w->lp, w->stream);
    w->launches += launch_rebuild(d, w->lp, w->stream);
    launch_graph_count(d, b, cutoff, w->stream);
    w->launches += 1 + launch_graph_offsets(d, b, w->stream);
    int32_t edges = 0;
    TGL_CUDA(cudaMemcpyAsync(&edges, b.offsets + d.S, sizeof(int32_t), cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    TGL_CUDA(cudaGetLastError());
    if (edges < 0) return set_error(TGL_ERR_UNSUPPORTED, "contact graph too large for 32-bit edge indices");
    if (edges > w->warm.depth_capacity) {
        cudaFree(w->warm.depth);
        w->warm.depth = nullptr;
        w->warm.depth_capacity = 0;
        const size_t cap = (size_t)edges + edges / 4 + 1024;
        if (cudaMalloc(&w->warm.depth, cap * sizeof(float)) != cudaSuccess)
            return set_error(TGL_ERR_MEMORY, "warm-start edge allocation failed");
        w->warm.depth_capacity = (int64_t)cap;
    }
    w->warm.edges = edges;
    w->warm.cutoff = cutoff;
    w->warm.counted = true;
    *edge_count = edges;
    return 0;
}

int tgl_warmstart_set_focus(tgl_world *w, const uint8_t *fiber_focus, size_t fibers) {
    if (!w) return set_error(TGL_ERR_INVALID, "null argument");
    if (w->arena) return set_error(TGL_ERR_UNSUPPORTED, "the warm start takes one specimen");
    w->warm.counted = false;
    if (!fiber_focus) {
        w->warm.b.fiber_focus = nullptr;
        return 0;
    }
    if (fibers != w->dev.F) return set_error(TGL_ERR_INVALID, "one focus flag per fiber");
    if (!w->warm.focus && cudaMalloc(&w->warm.focus, (size_t)w->dev.F * sizeof(uint32_t)) != cudaSuccess)
        return set_error(TGL_ERR_MEMORY, "cudaMalloc of the focus flags failed");
    std::vector<uint32_t> flags(fibers);
    for (size_t f = 0; f < fibers; ++f) flags[f] = fiber_focus[f] ? 1u : 0u;
    TGL_CUDA(cudaMemcpyAsync(w->warm.focus, flags.data(), fibers * sizeof(uint32_t), cudaMemcpyHostToDevice, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    w->warm.b.fiber_focus = w->warm.focus;
    return 0;
}

int tgl_warmstart_graph_fill(tgl_world *w, const tgl_mp_graph_out *out) {
    if (!w || !out || !out->seg_v0 || !out->links || !out->offsets || !out->node_features)
        return set_error(TGL_ERR_INVALID, "null argument");
    if (!w->warm.counted) return set_error(TGL_ERR_INVALID, "tgl_warmstart_graph_count must come first");
    const int64_t E = w->warm.edges;
    if (E > 0 && (!out->dst || !out->src || !out->twin || !out->s || !out->t || !out->edge_features))
        return set_error(TGL_ERR_INVALID, "null edge buffer");
    w->warm.counted = false;
    const WorldDev &d = w->dev;
    GraphBuffers b = w->warm.b;
    b.offsets = w->warm.offsets;
    b.dst = out->dst;
    b.src = out->src;
    b.twin = out->twin;
    b.s = out->s;
    b.t = out->t;
    b.depth = w->warm.depth;
    b.edge_features = static_cast<__nv_bfloat16 *>(out->edge_features);
    b.node_features = static_cast<__nv_bfloat16 *>(out->node_features);
    launch_graph_fill(d, b, w->warm.cutoff, w->stream);
    MpGraph g{};
    g.V = (int32_t)d.V;
    g.S = (int32_t)d.S;
    g.E = (int32_t)E;
    g.seg_v0 = reinterpret_cast<const int32_t *>(d.seg_v0);
    g.links = d.links;
    g.offsets = b.offsets;
    g.dst = b.dst;
    g.src = b.src;
    g.twin = b.twin;
    g.s = b.s;
    g.t = b.t;
    launch_node_features(d, b, g, w->stream);
    w->launches += 4;
    TGL_CUDA(cudaMemcpyAsync(out->seg_v0, d.seg_v0, (size_t)d.S * 4, cudaMemcpyDeviceToDevice, w->stream));
    TGL_CUDA(cudaMemcpyAsync(out->links, d.links, (size_t)d.V * 16, cudaMemcpyDeviceToDevice, w->stream));
    TGL_CUDA(cudaMemcpyAsync(out->offsets, b.offsets, ((size_t)d.S + 1) * 4, cudaMemcpyDeviceToDevice, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    TGL_CUDA(cudaGetLastError());
    return 0;
}

int tgl_world_displace(tgl_world *w, const float *dx, int64_t ld, float scale, int32_t in_diameters, float max_step) {
    if (!w || !dx) return set_error(TGL_ERR_INVALID, "null argument");
    w->warm.counted = false;
    if (ld < 3 || !std::isfinite(scale) || !(max_step > 0.0f)) return set_error(TGL_ERR_INVALID, "bad displacement arguments");
    launch_displace(w->dev, dx, ld, scale, in_diameters, max_step, w->stream);
    w->launches += 2;
    TGL_CUDA(cudaGetLastError());
    return 0;
}

int tgl_world_residual(tgl_world *w, const tgl_relax_config *config, float *max_penetration,
                       float *max_curvature_ratio, float *total_penetration) {
    if (!w || !config || !max_penetration || !max_curvature_ratio || !total_penetration)
        return set_error(TGL_ERR_INVALID, "null argument");
    if (w->arena) return set_error(TGL_ERR_UNSUPPORTED, "the residual is per specimen; use tgl_arena_status");
    if (int rc = validate_config(*config)) return rc;
    if (!w->warm.residual && cudaMalloc(&w->warm.residual, (3 + RESIDUAL_BLOCKS) * sizeof(float)) != cudaSuccess)
        return set_error(TGL_ERR_MEMORY, "cudaMalloc failed");
    StepParams sp = step_params(*config, 1);
    w->launches += launch_flag_displacement(w->dev, w->lp, w->stream);
    w->launches += launch_rebuild(w->dev, w->lp, w->stream);
    w->launches += launch_contact(w->dev, w->lp, sp, false, w->stream);
    launch_residual(w->dev, w->warm.residual, w->stream);
    w->launches += 1;
    float out[3];
    TGL_CUDA(cudaMemcpyAsync(out, w->warm.residual, sizeof(out), cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    TGL_CUDA(cudaGetLastError());
    *max_penetration = out[0];
    *max_curvature_ratio = out[1];
    *total_penetration = out[2];
    return 0;
}

int tgl_capture_contacts(tgl_world *w, float maximum_surface_gap, uint32_t capacity, uint32_t *segments,
                         float *coordinates, float *surface_gaps, float *crossing_angles, uint32_t *count,
                         uint32_t *overflow) {
    if (!w || !segments || !coordinates || !surface_gaps || !crossing_angles || !count || !overflow)
        return set_error(TGL_ERR_INVALID, "null argument");
    if (!(std::isfinite(maximum_surface_gap) && maximum_surface_gap >= 0.0f))  // world.rs:2203
        return set_error(TGL_ERR_INVALID, "maximum_surface_gap must be finite and non-negative");
    if (capacity == 0) return set_error(TGL_ERR_INVALID, "capacity must be positive");
    if (w->arena) return set_error(TGL_ERR_UNSUPPORTED, "contact capture takes one specimen");
    w->warm.counted = false;
    // world.rs:2209-2218: whole-segment cells grown by the gap (never finer
    // than the neighbor grid, whose cell buffers the capture reuses).
    WorldDev cap = w->dev;
    const float cell = w->cell_size + maximum_surface_gap;
    for (int a = 0; a < 3; ++a) {
        const float extent = cap.grid.length[a];
        cap.grid.cells[a] = f32_to_u32_host(std::fmax(std::floor(extent / cell), 1.0f));
        cap.grid.width[a] = extent / (float)cap.grid.cells[a];
    }
    const uint64_t C = checked_cell_count(cap.grid.cells, w->dev.C);
    if (C == 0) return set_error(TGL_ERR_UNSUPPORTED, "capture grid finer than the neighbor grid");
    cap.C = (uint32_t)C;
    uint32_t *count_d = nullptr, *pairs_d = nullptr;
    float *coords_d = nullptr, *gaps_d = nullptr, *angles_d = nullptr;
    auto release = [&]() {
        cudaFree(count_d);
        cudaFree(pairs_d);
        cudaFree(coords_d);
        cudaFree(gaps_d);
        cudaFree(angles_d);
    };
    if (cudaMalloc(&count_d, 2 * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&pairs_d, 2ull * capacity * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&coords_d, 2ull * capacity * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&gaps_d, (size_t)capacity * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&angles_d, (size_t)capacity * sizeof(float)) != cudaSuccess) {
        release();
        return set_error(TGL_ERR_MEMORY, "contact capture allocation failed");
    }
    // The shared cell buffers take the capture layout, so the next contact
    // pass must rebuild its lists first: the rebuild flag stays raised.
    w->launches += launch_request_rebuild(w->dev, w->lp, w->stream);
    w->launches += launch_cell_list(cap, w->lp, w->stream);
    cudaMemsetAsync(count_d, 0, 2 * sizeof(uint32_t), w->stream);
    launch_capture(cap, maximum_surface_gap, capacity, count_d, pairs_d, coords_d, gaps_d, angles_d, w->stream);
    w->launches += 1;
    uint32_t counts[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(counts, count_d, sizeof(counts), cudaMemcpyDeviceToHost, w->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(w->stream);
    const uint32_t n = std::min(counts[0], capacity);
    std::vector<uint32_t> pr(2 * (size_t)n);
    std::vector<float> co(2 * (size_t)n), ga(n), an(n);
    if (e == cudaSuccess && n) {
        cudaMemcpy(pr.data(), pairs_d, pr.size() * 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(co.data(), coords_d, co.size() * 4, cudaMemcpyDeviceToHost);
        cudaMemcpy(ga.data(), gaps_d, ga.size() * 4, cudaMemcpyDeviceToHost);
        e = cudaMemcpy(an.data(), angles_d, an.size() * 4, cudaMemcpyDeviceToHost);
    }
    release();
    if (e != cudaSuccess) return set_error(TGL_ERR_CUDA, std::string("contact capture: ") + cudaGetErrorString(e));
    // world.rs:2314-2321: the device appends in a run-dependent order; sort by
    // (first, second, s, t) so every run sees the same sequence.
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](uint32_t l, uint32_t r) {
        if (pr[2 * l] != pr[2 * r]) return pr[2 * l] < pr[2 * r];
        if (pr[2 * l + 1] != pr[2 * r + 1]) return pr[2 * l + 1] < pr[2 * r + 1];
        if (co[2 * l] != co[2 * r]) return co[2 * l] < co[2 * r];
        return co[2 * l + 1] < co[2 * r + 1];
    });
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t k = order[i];
        segments[2 * i] = pr[2 * k];
        segments[2 * i + 1] = pr[2 * k + 1];
        coordinates[2 * i] = co[2 * k];
        coordinates[2 * i + 1] = co[2 * k + 1];
        surface_gaps[i] = ga[k];
        crossing_angles[i] = an[k];
    }
    *count = n;
    *overflow = counts[1] != 0 ? 1u : 0u;
    return 0;
}

int tgl_debug_rebuild(tgl_world *w) {
    if (!w) return set_error(TGL_ERR_INVALID, "null argument");
    w->warm.counted = false;
    w->launches += launch_request_rebuild(w->dev, w->lp, w->stream);
    w->launches += launch_rebuild(w->dev, w->lp, w->stream);
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    TGL_CUDA(cudaGetLastError());
    return 0;
}

int tgl_debug_cell_list(tgl_world *w, uint32_t *cell_counts, uint32_t *cell_offsets, uint32_t *cell_segments) {
    if (!w || !cell_counts || !cell_offsets || !cell_segments) return set_error(TGL_ERR_INVALID, "null argument");
    TGL_CUDA(cudaMemcpyAsync(cell_counts, w->dev.cell_counts, w->dev.C * 4ull, cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaMemcpyAsync(cell_offsets, w->dev.cell_offsets, w->dev.C * 4ull, cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaMemcpyAsync(cell_segments, w->dev.cell_segments, w->dev.S * 4ull, cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    return 0;
}

int tgl_debug_neighbor_lists(tgl_world *w, uint32_t *counts, uint32_t *lists) {
    if (!w || !counts || !lists) return set_error(TGL_ERR_INVALID, "null argument");
    TGL_CUDA(cudaMemcpyAsync(counts, w->dev.nbr_count, w->dev.S * 4ull, cudaMemcpyDeviceToHost, w->stream));
    size_t n = (size_t)w->dev.S * w->dev.block;
    if (n) TGL_CUDA(cudaMemcpyAsync(lists, w->dev.nbr_list, n * 4, cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    return 0;
}

int tgl_debug_corrections(tgl_world *w, const tgl_relax_config *config, float *corrections, float *segment_max) {
    if (!w || !config || !corrections || !segment_max) return set_error(TGL_ERR_INVALID, "null argument");
    if (int rc = validate_config(*config)) return rc;
    StepParams sp = step_params(*config, 1);
    float *corr6 = nullptr, *pen = nullptr;
    TGL_CUDA(cudaMalloc(&corr6, 6ull * w->dev.S * sizeof(float)));
    if (cudaMalloc(&pen, (size_t)w->dev.S * sizeof(float)) != cudaSuccess) {
        cudaFree(corr6);
        return set_error(TGL_ERR_MEMORY, "cudaMalloc failed");
    }
    w->launches += launch_rebuild(w->dev, w->lp, w->stream);
    w->launches += launch_contact(w->dev, w->lp, sp, false, w->stream);
    w->launches += launch_corrections_to_stage(w->dev, corr6, pen, w->stream);
    cudaMemcpyAsync(corrections, corr6, 6ull * w->dev.S * sizeof(float), cudaMemcpyDeviceToHost, w->stream);
    cudaMemcpyAsync(segment_max, pen, (size_t)w->dev.S * sizeof(float), cudaMemcpyDeviceToHost, w->stream);
    cudaError_t e = cudaStreamSynchronize(w->stream);
    cudaFree(corr6);
    cudaFree(pen);
    if (e != cudaSuccess) return set_error(TGL_ERR_CUDA, cudaGetErrorString(e));
    TGL_CUDA(cudaGetLastError());
    return 0;
}

}  // extern "C"

// ------------------------------------------------------------- formation hooks

namespace {

// A change to the world's by-value kernel parameters (counts, targets,
// grid) retires every captured batch graph.
void invalidate_graphs(tgl_world *w) {
    for (auto &kv : w->graphs) destroy_entry(kv.second);
    w->graphs.clear();
    w->last = nullptr;
    w->warm.counted = false;
}

int formation_world(tgl_world *w) {
    if (!w) return set_error(TGL_ERR_INVALID, "null argument");
    if (w->arena) return set_error(TGL_ERR_UNSUPPORTED, "formation hooks take a single world, not an arena");
    return 0;
}

// The fiber of vertex v (binary search over the fiber spans).
uint32_t fiber_of_vertex(const tgl_world *w, uint32_t v) {
    size_t lo = 0, hi = w->h_vspan.size();
    while (hi - lo > 1) {
        const size_t mid = (lo + hi) / 2;
        if (w->h_vspan[mid].x <= v)
            lo = mid;
        else
            hi = mid;
    }
    return (uint32_t)lo;
}

}  // namespace

extern "C" {

int tgl_world_set_active_fibers(tgl_world *w, const uint8_t *active, uint64_t fiber_count, uint32_t *active_segments,
                                uint32_t *active_vertices) {
    if (int rc = formation_world(w)) return rc;
    if (!active || !active_segments || !active_vertices) return set_error(TGL_ERR_INVALID, "null argument");
    WorldDev &d = w->dev;
    if (fiber_count != d.F) return set_error(TGL_ERR_INVALID, "active flags need one entry per fiber");
    uint64_t segments = 0, vertices = 0;
    std::vector<uint32_t> order;
    order.reserve(d.F);
    for (uint32_t f = 0; f < d.F; ++f) {
        w->h_active[f] = active[f] ? 1u : 0u;
        if (!active[f]) continue;
        order.push_back(f);
        segments += w->h_vspan[f].y - 1;
        vertices += w->h_vspan[f].y;
    }
    // Active fibers by descending vertex count, as at creation.
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return w->h_vspan[a].y > w->h_vspan[b].y; });
    if (!order.empty()) {
        TGL_CUDA(cudaMemcpyAsync(w->fiber_order_d, order.data(), order.size() * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, w->stream));
        TGL_CUDA(cudaMemcpyAsync(d.update_order, order.data(), order.size() * sizeof(uint32_t),
                                 cudaMemcpyHostToDevice, w->stream));
    }
    const bool all = order.size() == d.F;
    if (!all) {
        if (!w->fiber_on_d && w->alloc(&w->fiber_on_d, d.F)) return TGL_ERR_MEMORY;
        TGL_CUDA(cudaMemcpyAsync(w->fiber_on_d, w->h_active.data(), d.F * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                 w->stream));
    }
    d.fiber_on = all ? nullptr : w->fiber_on_d;
    d.FA = (uint32_t)order.size();
    d.NS = (uint32_t)segments;
    plan_launches(d, w->lp);
    launch_clear_inactive_reactions(d, w->stream);
    // world.rs:2179-2181: newly active fibers are missing from the lists.
    w->launches += launch_request_rebuild(d, w->lp, w->stream);
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    TGL_CUDA(cudaGetLastError());
    invalidate_graphs(w);
    *active_segments = (uint32_t)segments;
    *active_vertices = (uint32_t)vertices;
    return 0;
}

int tgl_world_set_layer_targets(tgl_world *w, const tgl_layer_targets *t) {
    if (int rc = formation_world(w)) return rc;
    WorldDev &d = w->dev;
    invalidate_graphs(w);
    if (!t) {  // world.rs:1806-1810
        d.layer_target = nullptr;
        return 0;
    }
    // world.rs:1774-1777 and :1750.
    if (t->axis >= 3) return set_error(TGL_ERR_INVALID, "layer axis must be 0, 1 or 2");
    if (t->count == 0 || !t->targets || !t->fiber_layers) return set_error(TGL_ERR_INVALID, "layer targets are empty");
    if (!(t->stiffness > 0.0f && t->stiffness <= 1.0f)) return set_error(TGL_ERR_INVALID, "stiffness must be in (0, 1]");
    if (!(t->max_translation > 0.0f)) return set_error(TGL_ERR_INVALID, "max_translation must be positive");
    if (t->first_layer > t->last_layer) return set_error(TGL_ERR_INVALID, "first_layer exceeds last_layer");
    if (!w->fiber_layer_d && w->alloc(&w->fiber_layer_d, d.F)) return TGL_ERR_MEMORY;
    if (t->count > w->layer_capacity) {
        if (w->alloc(&w->layer_target_d, t->count)) return TGL_ERR_MEMORY;
        w->layer_capacity = t->count;
    }
    TGL_CUDA(cudaMemcpyAsync(w->fiber_layer_d, t->fiber_layers, d.F * sizeof(uint32_t), cudaMemcpyHostToDevice,
                             w->stream));
    TGL_CUDA(cudaMemcpyAsync(w->layer_target_d, t->targets, t->count * sizeof(float), cudaMemcpyHostToDevice,
                             w->stream));
    d.fiber_layer = w->fiber_layer_d;
    d.layer_target = w->layer_target_d;
    d.layer_count = t->count;
    d.layer_first = t->first_layer;
    d.layer_last = t->last_layer;
    d.layer_axis = t->axis;
    d.layer_stiffness = t->stiffness;
    d.layer_max_translation = t->max_translation;
    if (t->apply_now) {  // the first correction at once (world.rs:1778-1799)
        launch_layer_targets_now(d, w->stream);
        w->launches += 1 + launch_refresh_geometry(d, w->stream);
    }
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    TGL_CUDA(cudaGetLastError());
    return 0;
}

int tgl_world_set_vertex_targets(tgl_world *w, const tgl_vertex_targets *t) {
    if (int rc = formation_world(w)) return rc;
    WorldDev &d = w->dev;
    invalidate_graphs(w);
    if (!t) {  // world.rs:1861-1863
        d.vertex_target = nullptr;
        w->target_count = 0;
        w->h_target_vertices.clear();
        return 0;
    }
    // world.rs:1819-1828.
    if (t->axis >= 3) return set_error(TGL_ERR_INVALID, "target axis must be 0, 1 or 2");
    if (t->count == 0 || !t->vertices) return set_error(TGL_ERR_INVALID, "vertex targets are empty");
    if (!(t->stiffness > 0.0f && t->stiffness <= 1.0f)) return set_error(TGL_ERR_INVALID, "stiffness must be in (0, 1]");
    if (!(t->max_translation > 0.0f)) return set_error(TGL_ERR_INVALID, "max_translation must be positive");
    const bool restoring = t->coordinates != nullptr;
    if (restoring != (t->command_coordinates != nullptr))
        return set_error(TGL_ERR_INVALID, "coordinates and command_coordinates come together");
    if (!restoring && !(std::isfinite(t->displacement) && t->displacement != 0.0f))
        return set_error(TGL_ERR_INVALID, "displacement must be finite and non-zero");
    std::vector<int32_t> map(d.V, -1);
    std::vector<uint32_t> fibers(t->count);
    for (uint32_t k = 0; k < t->count; ++k) {
        const uint32_t v = t->vertices[k];
        if (v >= d.V) return set_error(TGL_ERR_INVALID, "vertex target index out of range");
        if (map[v] >= 0) return set_error(TGL_ERR_INVALID, "vertex target indices must be distinct");
        map[v] = (int32_t)k;
        fibers[k] = fiber_of_vertex(w, v);
    }
    if (!w->vertex_target_d && w->alloc(&w->vertex_target_d, d.V)) return TGL_ERR_MEMORY;
    if (t->count > w->target_capacity) {  // the four per-target buffers grow together
        if (w->alloc(&w->target_vertices_d, t->count) || w->alloc(&w->target_fibers_d, t->count) ||
            w->alloc(&w->target_coord_d, t->count) || w->alloc(&w->command_coord_d, t->count))
            return TGL_ERR_MEMORY;
        w->target_capacity = t->count;
    }
    TGL_CUDA(cudaMemcpyAsync(w->vertex_target_d, map.data(), d.V * sizeof(int32_t), cudaMemcpyHostToDevice, w->stream));
    TGL_CUDA(cudaMemcpyAsync(w->target_vertices_d, t->vertices, t->count * sizeof(uint32_t), cudaMemcpyHostToDevice,
                             w->stream));
    TGL_CUDA(cudaMemcpyAsync(w->target_fibers_d, fibers.data(), t->count * sizeof(uint32_t), cudaMemcpyHostToDevice,
                             w->stream));
    d.target_axis = t->axis;
    d.target_stiffness = t->stiffness;
    d.target_max_translation = t->max_translation;
    d.target_coord = w->target_coord_d;
    d.command_coord = w->command_coord_d;
    d.vertex_target = w->vertex_target_d;
    if (restoring) {
        TGL_CUDA(cudaMemcpyAsync(w->target_coord_d, t->coordinates, t->count * sizeof(float), cudaMemcpyHostToDevice,
                                 w->stream));
        TGL_CUDA(cudaMemcpyAsync(w->command_coord_d, t->command_coordinates, t->count * sizeof(float),
                                 cudaMemcpyHostToDevice, w->stream));
    } else {
        launch_init_vertex_targets(d, w->target_vertices_d, t->count, t->displacement, w->target_coord_d,
                                   w->command_coord_d, w->stream);
        w->launches += 1;
    }
    w->target_count = t->count;
    w->h_target_vertices.assign(t->vertices, t->vertices + t->count);
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    TGL_CUDA(cudaGetLastError());
    return 0;
}

int tgl_world_vertex_target_state(tgl_world *w, float *coordinates, float *command_coordinates, uint32_t count) {
    if (int rc = formation_world(w)) return rc;
    if (!coordinates || !command_coordinates) return set_error(TGL_ERR_INVALID, "null argument");
    if (!w->dev.vertex_target) return set_error(TGL_ERR_INVALID, "no vertex targets are installed");
    if (count != w->target_count) return set_error(TGL_ERR_INVALID, "count differs from the installed target count");
    TGL_CUDA(cudaMemcpyAsync(coordinates, w->target_coord_d, count * sizeof(float), cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaMemcpyAsync(command_coordinates, w->command_coord_d, count * sizeof(float), cudaMemcpyDeviceToHost,
                             w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    return 0;
}

int tgl_world_target_errors(tgl_world *w, float *layer_error, uint32_t *has_layer, float *vertex_error,
                            uint32_t *has_vertex) {
    if (int rc = formation_world(w)) return rc;
    if (!layer_error || !has_layer || !vertex_error || !has_vertex) return set_error(TGL_ERR_INVALID, "null argument");
    const WorldDev &d = w->dev;
    *has_layer = d.layer_target ? 1u : 0u;
    *has_vertex = d.vertex_target ? 1u : 0u;
    *layer_error = 0.0f;
    *vertex_error = 0.0f;
    if (!d.layer_target && !d.vertex_target) return 0;
    if (!w->error_bits_d && w->alloc(&w->error_bits_d, 2)) return TGL_ERR_MEMORY;
    launch_target_errors(d, w->target_vertices_d, w->target_fibers_d, w->target_count, w->error_bits_d, w->stream);
    w->launches += (d.layer_target ? 1 : 0) + (d.vertex_target ? 1 : 0);
    unsigned int bits[2] = {0, 0};
    TGL_CUDA(cudaMemcpyAsync(bits, w->error_bits_d, sizeof(bits), cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    TGL_CUDA(cudaGetLastError());
    std::memcpy(layer_error, &bits[0], 4);
    std::memcpy(vertex_error, &bits[1], 4);
    return 0;
}

int tgl_world_compact_cell(tgl_world *w, const float new_lower[3], const float new_upper[3], uint32_t kinematics) {
    if (int rc = formation_world(w)) return rc;
    if (!new_lower || !new_upper) return set_error(TGL_ERR_INVALID, "null argument");
    if (kinematics > 2) return set_error(TGL_ERR_INVALID, "kinematics must be 0 (rigid centres), 1 (walls) or 2 (affine)");
    WorldDev &d = w->dev;
    // world.rs:1937-1950.
    uint32_t cells[3];
    for (int a = 0; a < 3; ++a) {
        if (!std::isfinite(new_lower[a]) || !std::isfinite(new_upper[a]))
            return set_error(TGL_ERR_INVALID, "the new cell bounds must be finite");
        if (!(new_upper[a] - new_lower[a] > 2.0f * w->maximum_radius))
            return set_error(TGL_ERR_INVALID, "the new cell must be wider than two largest radii on every axis");
        if (!(new_lower[a] >= d.grid.lower[a]) || !(new_upper[a] <= d.grid.upper[a]))
            return set_error(TGL_ERR_INVALID, "compaction cannot grow the cell");
        cells[a] = f32_to_u32_host(std::fmax(std::floor((new_upper[a] - new_lower[a]) / w->cell_size), 1.0f));
    }
    const uint64_t C = checked_cell_count(cells, w->allocated_cells);
    if (C == 0) return set_error(TGL_ERR_INVALID, "the compacted grid needs more cells than allocated");
    launch_compaction(d, new_lower, new_upper, kinematics, w->stream);
    w->launches += 1;
    // world.rs:2035-2053: the resident cell and the grid follow; the cell
    // size stays.
    for (int a = 0; a < 3; ++a) {
        const float extent = new_upper[a] - new_lower[a];
        d.grid.lower[a] = new_lower[a];
        d.grid.upper[a] = new_upper[a];
        d.grid.cells[a] = cells[a];
        d.grid.length[a] = extent;
        d.grid.width[a] = extent / (float)cells[a];
        d.grid.inv_length[a] = 1.0f / extent;
    }
    d.C = (uint32_t)C;
    w->contact_grids.assign(1, d.grid);
    // The contact lists' single-image bound follows the new box edges.
    if (d.contact_skin > 0.0f) {
        d.contact_half_limit = INFINITY;
        for (int a = 0; a < 3; ++a)
            if (d.grid.periodic[a])
                d.contact_half_limit =
                    std::fmin(d.contact_half_limit,
                              0.999f * 0.5f * (0.5f * d.grid.length[a] - 2.0f * w->maximum_radius - d.contact_skin));
    }
    plan_launches(d, w->lp);
    w->launches += launch_refresh_geometry(d, w->stream);
    w->launches += launch_request_rebuild(d, w->lp, w->stream);  // world.rs:2052
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    TGL_CUDA(cudaGetLastError());
    invalidate_graphs(w);
    return 0;
}

int tgl_world_cell_bounds(tgl_world *w, float lower[3], float upper[3]) {
    if (!w || !lower || !upper) return set_error(TGL_ERR_INVALID, "null argument");
    for (int a = 0; a < 3; ++a) {
        lower[a] = w->dev.grid.lower[a];
        upper[a] = w->dev.grid.upper[a];
    }
    return 0;
}

int tgl_world_compaction_metrics(tgl_world *w, float correction_fraction, const float stiffness[3], float out[13]) {
    if (int rc = formation_world(w)) return rc;
    if (!stiffness || !out) return set_error(TGL_ERR_INVALID, "null argument");
    // world.rs:2061-2064.
    if (!(correction_fraction > 0.0f)) return set_error(TGL_ERR_INVALID, "correction_fraction must be positive");
    for (int k = 0; k < 3; ++k)
        if (!(stiffness[k] >= 0.0f)) return set_error(TGL_ERR_INVALID, "energy stiffnesses must be non-negative");
    if (!w->metric_partials_d && w->alloc(&w->metric_partials_d, (size_t)METRIC_BLOCKS * 12)) return TGL_ERR_MEMORY;
    if (!w->metric_out_d && w->alloc(&w->metric_out_d, 13)) return TGL_ERR_MEMORY;
    launch_compaction_metrics(w->dev, correction_fraction, stiffness[0], stiffness[1], stiffness[2],
                              w->metric_partials_d, w->metric_out_d, w->stream);
    w->launches += 2;
    TGL_CUDA(cudaMemcpyAsync(out, w->metric_out_d, 13 * sizeof(float), cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    TGL_CUDA(cudaGetLastError());
    return 0;
}

int tgl_world_wall_reactions(tgl_world *w, float *xyz, size_t len) {
    if (int rc = formation_world(w)) return rc;
    if (!xyz) return set_error(TGL_ERR_INVALID, "null argument");
    const WorldDev &d = w->dev;
    if (len != 3 * (size_t)d.V) return set_error(TGL_ERR_INVALID, "reaction buffer has the wrong length");
    if (!d.reaction) {  // no walls: every reaction is zero
        std::memset(xyz, 0, len * sizeof(float));
        return 0;
    }
    std::vector<float4> r(d.V);
    TGL_CUDA(cudaMemcpyAsync(r.data(), d.reaction, d.V * sizeof(float4), cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    for (uint32_t v = 0; v < d.V; ++v) {
        xyz[3 * (size_t)v] = r[v].x;
        xyz[3 * (size_t)v + 1] = r[v].y;
        xyz[3 * (size_t)v + 2] = r[v].z;
    }
    return 0;
}

int tgl_world_set_wall_reactions(tgl_world *w, const float *xyz, size_t len) {
    if (int rc = formation_world(w)) return rc;
    if (!xyz) return set_error(TGL_ERR_INVALID, "null argument");
    const WorldDev &d = w->dev;
    if (len != 3 * (size_t)d.V) return set_error(TGL_ERR_INVALID, "reaction buffer has the wrong length");
    if (!d.reaction) return 0;  // no walls: reactions stay zero
    std::vector<float4> r(d.V);
    for (uint32_t v = 0; v < d.V; ++v)
        r[v] = make_float4(xyz[3 * (size_t)v], xyz[3 * (size_t)v + 1], xyz[3 * (size_t)v + 2], 0.0f);
    TGL_CUDA(cudaMemcpyAsync(d.reaction, r.data(), d.V * sizeof(float4), cudaMemcpyHostToDevice, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    return 0;
}

int tgl_world_set_fiber_max_curvatures(tgl_world *w, const float *values, size_t count) {
    if (int rc = formation_world(w)) return rc;
    if (!values) return set_error(TGL_ERR_INVALID, "null argument");
    const WorldDev &d = w->dev;
    if (count != d.F) return set_error(TGL_ERR_INVALID, "one curvature limit per fiber");  // world.rs:2186
    for (size_t f = 0; f < count; ++f)
        if (!(values[f] >= 0.0f) || !std::isfinite(values[f]))
            return set_error(TGL_ERR_INVALID, "curvature limits must be finite and non-negative");
    float *values_d = nullptr;
    if (cudaMalloc(&values_d, count * sizeof(float)) != cudaSuccess) return set_error(TGL_ERR_MEMORY, "cudaMalloc failed");
    cudaError_t e = cudaMemcpyAsync(values_d, values, count * sizeof(float), cudaMemcpyHostToDevice, w->stream);
    if (e == cudaSuccess) {
        launch_set_fiber_curvatures(d, w->vtx_static_d, values_d, w->stream);
        w->launches += 1;
        e = cudaStreamSynchronize(w->stream);
    }
    cudaFree(values_d);
    if (e != cudaSuccess) return set_error(TGL_ERR_CUDA, std::string("curvature limits: ") + cudaGetErrorString(e));
    TGL_CUDA(cudaGetLastError());
    return 0;
}

}  // extern "C"

namespace {

// The contact skin and its single-image bound for a fraction of the
// neighbor skin (as build_world sets them); a fraction the bound leaves no
// room for turns the lists off.
void set_contact_skin(tgl_world *w, float fraction) {
    WorldDev &d = w->dev;
    d.contact_skin = fraction > 0.0f ? fraction * w->contact_skin_base : 0.0f;
    // A pair's minimum image must stay fixed while its vertices move less
    // than the contact skin: with every half length below H, pairs within
    // reach + contact skin are closer than half a box length on every
    // periodic axis, so H = (L/2 - 2 r_max - contact_skin) / 2, less 0.1 %,
    // over every specimen's box.
    d.contact_half_limit = INFINITY;
    for (const Grid &g : w->contact_grids)
        for (int a = 0; a < 3; ++a)
            if (g.periodic[a])
                d.contact_half_limit = std::fmin(
                    d.contact_half_limit, 0.999f * 0.5f * (0.5f * g.length[a] - 2.0f * w->maximum_radius - d.contact_skin));
    if (!(d.contact_half_limit > 0.5f * w->maximum_length)) d.contact_skin = 0.0f;  // no room: full lists every pass
    w->contact_fraction = d.contact_skin > 0.0f ? fraction : 0.0f;
}

void drop_graphs(tgl_world *w) {
    for (auto &kv : w->graphs) destroy_entry(kv.second);
    w->graphs.clear();
    w->last = nullptr;
}

int check_launch_params(const tgl_world *w, const tgl_launch_params &p) {
    if (p.lanes_per_fiber != 2 && p.lanes_per_fiber != 4 && p.lanes_per_fiber != 8 && p.lanes_per_fiber != 32)
        return set_error(TGL_ERR_INVALID, "lanes_per_fiber must be 2, 4, 8 or 32");
    if (p.contact_blocks_per_sm < 1 || p.contact_blocks_per_sm > 3)
        return set_error(TGL_ERR_INVALID, "contact_blocks_per_sm must be 1, 2 or 3");
    if (p.build_chunk < 512 || p.build_chunk > 4096)
        return set_error(TGL_ERR_INVALID, "build_chunk must be between 512 and 4096");
    if (!(p.contact_skin_fraction >= 0.0f && p.contact_skin_fraction <= 1.0f))
        return set_error(TGL_ERR_INVALID, "contact_skin_fraction must be in [0, 1]");
    if (p.contact_skin_fraction > 0.0f && w->dev.contact_block == 0)
        return set_error(TGL_ERR_UNSUPPORTED, "this world has no contact lists to size");
    if (p.update_warps_per_block != 1 && p.update_warps_per_block != 2 && p.update_warps_per_block != 4)
        return set_error(TGL_ERR_INVALID, "update_warps_per_block must be 1, 2 or 4");
    return 0;
}

void current_launch_params(const tgl_world *w, tgl_launch_params *p) {
    std::memset(p, 0, sizeof(*p));
    p->lanes_per_fiber = (uint32_t)w->lp.lanes_per_fiber;
    const int per_sm = (w->lp.contact_blocks + w->lp.num_sms - 1) / std::max(w->lp.num_sms, 1);
    p->contact_blocks_per_sm = (uint32_t)(w->lp.tune_contact_per_sm ? w->lp.tune_contact_per_sm : std::min(3, std::max(per_sm, 1)));
    p->build_chunk = (uint32_t)w->lp.build_ch;
    p->contact_skin_fraction = w->contact_fraction;
    p->update_warps_per_block = (uint32_t)(w->lp.tune_wpb ? w->lp.tune_wpb : 4);
}

int apply_launch_params(tgl_world *w, const tgl_launch_params &p) {
    if (int rc = check_launch_params(w, p)) return rc;
    w->lp.tune_lanes = (int)p.lanes_per_fiber;
    w->lp.tune_contact_per_sm = (int)p.contact_blocks_per_sm;
    w->lp.tune_build_ch = (int)p.build_chunk;
    w->lp.tune_wpb = (int)p.update_warps_per_block;
    if (w->dev.contact_block) set_contact_skin(w, p.contact_skin_fraction);
    plan_launches(w->dev, w->lp);
    drop_graphs(w);
    // The contact lists were filtered at the old skin: refresh them first.
    if (w->dev.contact_block) {
        const uint32_t one = 1;
        TGL_CUDA(cudaMemcpyAsync(reinterpret_cast<char *>(w->dev.ctl) + offsetof(Control, contact_state), &one,
                                 sizeof(uint32_t), cudaMemcpyHostToDevice, w->stream));
        TGL_CUDA(cudaStreamSynchronize(w->stream));
    }
    return 0;
}

// The state a trial batch changes and the search restores: positions, the
// last applied steps, the formation commands and the control words (the
// lists, snapshots and corrections are rebuilt from these).
struct SavedState {
    float4 *pos = nullptr;
    float *step = nullptr;
    float *command = nullptr;
    std::vector<Control> ctl;
    ~SavedState() {
        cudaFree(pos);
        cudaFree(step);
        cudaFree(command);
    }
};

int save_state(tgl_world *w, SavedState &s) {
    const WorldDev &d = w->dev;
    if (cudaMalloc(&s.pos, d.V * sizeof(float4)) != cudaSuccess || cudaMalloc(&s.step, d.V * sizeof(float)) != cudaSuccess)
        return set_error(TGL_ERR_MEMORY, "cudaMalloc of the autotuner's saved state failed");
    if (w->target_count && cudaMalloc(&s.command, w->target_count * sizeof(float)) != cudaSuccess)
        return set_error(TGL_ERR_MEMORY, "cudaMalloc of the autotuner's saved state failed");
    const size_t words = w->arena ? (size_t)w->specimens + 1 : 1;
    s.ctl.resize(words);
    TGL_CUDA(cudaMemcpyAsync(s.pos, d.pos, d.V * sizeof(float4), cudaMemcpyDeviceToDevice, w->stream));
    TGL_CUDA(cudaMemcpyAsync(s.step, d.vertex_step, d.V * sizeof(float), cudaMemcpyDeviceToDevice, w->stream));
    if (s.command)
        TGL_CUDA(cudaMemcpyAsync(s.command, d.command_coord, w->target_count * sizeof(float), cudaMemcpyDeviceToDevice,
                                 w->stream));
    TGL_CUDA(cudaMemcpyAsync(s.ctl.data(), d.ctl, words * sizeof(Control), cudaMemcpyDeviceToHost, w->stream));
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    return 0;
}

// Puts the saved state back and requests a neighbor-list rebuild and a
// contact-list refresh for the next batch.
int restore_state(tgl_world *w, const SavedState &s) {
    const WorldDev &d = w->dev;
    TGL_CUDA(cudaMemcpyAsync(d.pos, s.pos, d.V * sizeof(float4), cudaMemcpyDeviceToDevice, w->stream));
    TGL_CUDA(cudaMemcpyAsync(d.vertex_step, s.step, d.V * sizeof(float), cudaMemcpyDeviceToDevice, w->stream));
    if (s.command)
        TGL_CUDA(cudaMemcpyAsync(d.command_coord, s.command, w->target_count * sizeof(float), cudaMemcpyDeviceToDevice,
                                 w->stream));
    std::vector<Control> ctl = s.ctl;
    for (Control &c : ctl) {
        c.neighbor_state[0] = 1;
        c.contact_state[0] = 1;
    }
    TGL_CUDA(cudaMemcpyAsync(d.ctl, ctl.data(), ctl.size() * sizeof(Control), cudaMemcpyHostToDevice, w->stream));
    w->launches += launch_refresh_geometry(d, w->stream);
    TGL_CUDA(cudaStreamSynchronize(w->stream));
    return 0;
}

// One trial: the saved state, an untimed batch (graph capture), then the
// better of two timed batches.
int trial(tgl_world *w, const SavedState &s, const tgl_relax_config &config, uint32_t iterations, float *ms) {
    tgl_batch_status st{};
    cudaEvent_t start = nullptr, end = nullptr;
    if (cudaEventCreate(&start) != cudaSuccess || cudaEventCreate(&end) != cudaSuccess) {
        cudaEventDestroy(start);
        return set_error(TGL_ERR_CUDA, "cudaEventCreate failed");
    }
    float best = INFINITY;
    int rc = 0;
    for (int run = 0; run < 3 && rc == 0; ++run) {
        if ((rc = restore_state(w, s))) break;
        cudaEventRecord(start, w->stream);
        if ((rc = tgl_run_batch(w, &config, iterations, &st))) break;
        cudaEventRecord(end, w->stream);
        if (cudaEventSynchronize(end) != cudaSuccess) {
            rc = set_error(TGL_ERR_CUDA, "trial batch failed");
            break;
        }
        float t = 0.0f;
        cudaEventElapsedTime(&t, start, end);
        if (run > 0) best = std::fmin(best, t);
    }
    cudaEventDestroy(start);
    cudaEventDestroy(end);
    *ms = best;
    return rc;
}

}  // namespace

extern "C" {

int tgl_world_get_launch_params(tgl_world *w, tgl_launch_params *params) {
    if (!w || !params) return set_error(TGL_ERR_INVALID, "null argument");
    current_launch_params(w, params);
    return 0;
}

int tgl_world_set_launch_params(tgl_world *w, const tgl_launch_params *params) {
    if (!w || !params) return set_error(TGL_ERR_INVALID, "null argument");
    return apply_launch_params(w, *params);
}

int tgl_autotune(tgl_world *w, const tgl_relax_config *config, uint32_t trial_iterations, tgl_launch_params *best,
                 tgl_autotune_report *report) {
    if (!w || !config || !best) return set_error(TGL_ERR_INVALID, "null argument");
    if (trial_iterations == 0 || trial_iterations > 4096)
        return set_error(TGL_ERR_INVALID, "trial_iterations must be between 1 and 4096");
    if (int rc = validate_config(*config)) return rc;
    tgl_relax_config trial_config = *config;
    trial_config.force_full_iterations = 1;
    const bool was_timing = w->timing;
    if (was_timing) tgl_set_kernel_timing(w, 0);
    SavedState saved;
    if (int rc = save_state(w, saved)) return rc;
    tgl_launch_params current{};
    current_launch_params(w, &current);
    const tgl_launch_params original = current;
    float current_ms = INFINITY;
    uint32_t trials = 0;
    auto fail = [&](int rc) {
        apply_launch_params(w, original);
        restore_state(w, saved);
        if (was_timing) tgl_set_kernel_timing(w, 1);
        return rc;
    };
    if (int rc = apply_launch_params(w, current)) return fail(rc);
    if (int rc = trial(w, saved, trial_config, trial_iterations, &current_ms)) return fail(rc);
    ++trials;
    const float default_ms = current_ms;
    const bool lanes = w->lp.fiber_lanes && config->motion_model == 0;
    const uint32_t lane_choices[] = {2, 4, 8, 32};
    const uint32_t block_choices[] = {1, 2, 3};
    const uint32_t chunk_choices[] = {1024, 1536, 2048, 3072, 4096};
    const float skin_choices[] = {0.05f, 0.1f, 0.15f, 0.25f};
    const uint32_t wpb_choices[] = {1, 2, 4};
    // Coordinate descent: each parameter in turn over its candidates, the
    // others held at the best so far.
    for (int parameter = 0; parameter < 5; ++parameter) {
        std::vector<tgl_launch_params> candidates;
        tgl_launch_params c = current;
        if (parameter == 0 && lanes)
            for (uint32_t v : lane_choices) c.lanes_per_fiber = v, candidates.push_back(c);
        if (parameter == 1)
            for (uint32_t v : block_choices) c.contact_blocks_per_sm = v, candidates.push_back(c);
        if (parameter == 2)
            for (uint32_t v : chunk_choices) c.build_chunk = v, candidates.push_back(c);
        if (parameter == 3 && w->dev.contact_block)
            for (float v : skin_choices) c.contact_skin_fraction = v, candidates.push_back(c);
        if (parameter == 4 && lanes)
            for (uint32_t v : wpb_choices) c.update_warps_per_block = v, candidates.push_back(c);
        for (const tgl_launch_params &candidate : candidates) {
            if (std::memcmp(&candidate, &current, sizeof(candidate)) == 0) continue;
            if (int rc = apply_launch_params(w, candidate)) return fail(rc);
            float ms = INFINITY;
            if (int rc = trial(w, saved, trial_config, trial_iterations, &ms)) return fail(rc);
            ++trials;
            if (ms < current_ms) {
                current_ms = ms;
                current = candidate;
            }
        }
    }
    if (int rc = apply_launch_params(w, current)) return fail(rc);
    if (int rc = restore_state(w, saved)) return fail(rc);
    if (was_timing) tgl_set_kernel_timing(w, 1);
    *best = current;
    if (report) {
        report->trials = trials;
        report->trial_iterations = trial_iterations;
        report->default_ms = default_ms;
        report->best_ms = current_ms;
    }
    return 0;
}

}  // extern "C"
