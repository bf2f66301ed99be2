/*
 * relax_oracle.cpp -- CPU restatement of TANGLE's plain relaxation path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
 * baseline. Built with -O2 -ffp-contract=off (no FMA contraction, SSE f32),
 * so every expression below rounds exactly as written, left to right, like
 * the reference's Rust/CubeCL source it restates. Each function cites the
 * reference file:line it follows (paths relative to the reference project).
 *
 * Scope: round sections (segment_lane_offsets == 0, so the lane loop of
 * contact.rs:641-652 is one lane at zero offset and every director/turn term
 * vanishes), non-adaptive layouts (every segment one proxy piece, list
 * weight 1), flexible and rigid-translation motion.
 */
#include "relax_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr uint32_t NONE = 0xFFFFFFFFu;
/* world.rs:36 -- the reference's neighbor-list buffer cap. */
constexpr uint64_t REFERENCE_MAX_LIST_BYTES = 120ull << 20;

thread_local std::string g_error;

int fail(const std::string &message) {
    g_error = message;
    return 1;
}

/* Rust f32::clamp: if x < lo then lo; if x > hi then hi. */
inline float clampf(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

/* Rust `f32 as i32`: saturating, NaN -> 0. */
inline int32_t f32_to_i32(float x) {
    if (std::isnan(x)) return 0;
    if (x >= 2147483648.0f) return std::numeric_limits<int32_t>::max();
    if (x < -2147483648.0f) return std::numeric_limits<int32_t>::min();
    return (int32_t)x;
}

/* Rust `f32 as u32`: saturating, NaN -> 0. */
inline uint32_t f32_to_u32(float x) {
    if (std::isnan(x) || x <= 0.0f) return 0;
    if (x >= 4294967296.0f) return NONE;
    return (uint32_t)x;
}

/* The cell count of a grid, or 0 when it is unusable: an axis with no cell
 * or more than 2^30 cells (proxy_cell's periodic wrap (raw % n + n) % n is
 * done in i32 and stays below 2^31 only then), or a product above `limit`,
 * checked after every factor so it cannot wrap. world.rs:410-415 sizes each
 * axis as `floor(extent / cell).max(1) as u32`. */
inline uint64_t checked_cell_count(const uint32_t cells[3], uint64_t limit) {
    uint64_t C = 1;
    for (int a = 0; a < 3; ++a) {
        if (cells[a] == 0 || cells[a] > (1u << 30)) return 0;
        C *= cells[a];
        if (C > limit) return 0;
    }
    return C;
}

inline uint32_t f32_bits(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    return u;
}

inline float bits_f32(uint32_t u) {
    float x;
    std::memcpy(&x, &u, 4);
    return x;
}

struct Grid {
    float lower[3], upper[3];
    uint32_t periodic[3];
    uint32_t cx, cy, cz;
};

/* f32 arc cosine with one fixed rounding sequence, so that every build of
the relaxation (these kernels and the CPU oracle) rounds it identically.
The reference calls the backend's acos (kernels.rs:1211), whose last bits
differ between libm and GPU runtimes. Method: the usual reduction to asin
on [0, 1/2] -- acos x = pi/2 - asin x for |x| <= 1/2, and
acos x = 2 asin(sqrt((1 - x)/2)) (or pi minus that for x < 0) otherwise --
with asin s = s + s z P(z), z = s^2 <= 1/4, where P is a degree-5
polynomial least-squares fitted in f64 to (asin(sqrt z) - sqrt z)/(z sqrt z)
on Chebyshev nodes of [0, 1/4]. Maximum error 1.01 ulp against f64 acos
over 440k samples of [-1, 1]. */
inline float acos_f32(float x) {
    const float pio2_hi = 1.57079637050628662109375f;
    const float pio2_lo = -4.371138828673793e-08f;
    float ax = std::fabs(x);
    if (ax <= 0.5f) {
        float z = x * x;
        float p = ((((0.03381037712097168f * z + 0.01707467809319496f) * z + 0.031116951256990433f) * z +
                    0.04459794610738754f) * z + 0.07500099390745163f) * z + 0.1666666567325592f;
        float r = x + x * z * p;
        return pio2_hi - (r - pio2_lo);
    }
    float z = 0.5f * (1.0f - ax);
    float s = std::sqrt(z);
    float p = ((((0.03381037712097168f * z + 0.01707467809319496f) * z + 0.031116951256990433f) * z +
                0.04459794610738754f) * z + 0.07500099390745163f) * z + 0.1666666567325592f;
    float r = s + s * z * p;
    if (x > 0.0f) return 2.0f * r;
    return 2.0f * (pio2_hi - (r - pio2_lo));
}

/* proxy_cell, cell_list.rs:34-79 (proxies == 1: the segment midpoint). */
inline uint32_t proxy_cell(float px, float py, float pz, float qx, float qy, float qz,
                           const Grid &g) {
    float midpoint_x = 0.5f * (px + qx);
    float midpoint_y = 0.5f * (py + qy);
    float midpoint_z = 0.5f * (pz + qz);
    float width_x = (g.upper[0] - g.lower[0]) / (float)g.cx;
    float width_y = (g.upper[1] - g.lower[1]) / (float)g.cy;
    float width_z = (g.upper[2] - g.lower[2]) / (float)g.cz;
    int32_t raw_x = f32_to_i32(std::floor((midpoint_x - g.lower[0]) / width_x));
    int32_t raw_y = f32_to_i32(std::floor((midpoint_y - g.lower[1]) / width_y));
    int32_t raw_z = f32_to_i32(std::floor((midpoint_z - g.lower[2]) / width_z));
    int32_t cx = (int32_t)g.cx, cy = (int32_t)g.cy, cz = (int32_t)g.cz;
    uint32_t x = (uint32_t)std::min(std::max(raw_x, 0), cx - 1);
    uint32_t y = (uint32_t)std::min(std::max(raw_y, 0), cy - 1);
    uint32_t z = (uint32_t)std::min(std::max(raw_z, 0), cz - 1);
    if (g.periodic[0]) x = (uint32_t)((raw_x % cx + cx) % cx);
    if (g.periodic[1]) y = (uint32_t)((raw_y % cy + cy) % cy);
    if (g.periodic[2]) z = (uint32_t)((raw_z % cz + cz) % cz);
    return (z * g.cy + y) * g.cx + x;
}

/* along_fiber_gap, cell_list.rs:100-112. */
inline float along_fiber_gap(const float *arc, uint32_t a0, uint32_t a1, uint32_t b0,
                             uint32_t b1) {
    float after = arc[b0] - arc[a1];
    float before = arc[a0] - arc[b1];
    return std::fmax(after, before);
}

/* The 27-cell stencil with periodic uniqueness (neighbor.rs:242-274,
 * contact.rs:390-427). Returns the neighbor cell or NONE. */
inline uint32_t stencil_cell(uint32_t home, uint32_t neighbor, const Grid &g) {
    uint32_t home_x = home % g.cx;
    uint32_t home_y = (home / g.cx) % g.cy;
    uint32_t home_z = home / (g.cx * g.cy);
    int32_t offset_x = (int32_t)(neighbor % 3) - 1;
    int32_t offset_y = (int32_t)((neighbor / 3) % 3) - 1;
    int32_t offset_z = (int32_t)(neighbor / 9) - 1;
    int32_t rx = (int32_t)home_x + offset_x;
    int32_t ry = (int32_t)home_y + offset_y;
    int32_t rz = (int32_t)home_z + offset_z;
    int32_t cx = (int32_t)g.cx, cy = (int32_t)g.cy, cz = (int32_t)g.cz;
    bool valid_x = g.periodic[0] != 0 || (rx >= 0 && rx < cx);
    bool valid_y = g.periodic[1] != 0 || (ry >= 0 && ry < cy);
    bool valid_z = g.periodic[2] != 0 || (rz >= 0 && rz < cz);
    bool unique_x = g.periodic[0] == 0 ||
                    !((g.cx == 1 && offset_x != 0) ||
                      (g.cx == 2 && ((home_x == 0 && offset_x > 0) || (home_x == 1 && offset_x < 0))));
    bool unique_y = g.periodic[1] == 0 ||
                    !((g.cy == 1 && offset_y != 0) ||
                      (g.cy == 2 && ((home_y == 0 && offset_y > 0) || (home_y == 1 && offset_y < 0))));
    bool unique_z = g.periodic[2] == 0 ||
                    !((g.cz == 1 && offset_z != 0) ||
                      (g.cz == 2 && ((home_z == 0 && offset_z > 0) || (home_z == 1 && offset_z < 0))));
    if (!(valid_x && valid_y && valid_z && unique_x && unique_y && unique_z)) return NONE;
    uint32_t nx = (uint32_t)((rx % cx + cx) % cx);
    uint32_t ny = (uint32_t)((ry % cy + cy) % cy);
    uint32_t nz = (uint32_t)((rz % cz + cz) % cz);
    return (nz * g.cy + ny) * g.cx + nx;
}

/* neighbor.rs:27-86 (proxies == 1, so the canonical test always passes:
 * proxy_of(x, 1) == 0 for every x). */
inline float proxy_pair_axis_distance(float p1x, float p1y, float p1z, float d1x, float d1y,
                                      float d1z, float p2x, float p2y, float p2z, float d2x,
                                      float d2y, float d2z) {
    const float length_epsilon = 1.0e-20f;
    const float parallel_relative_epsilon = 1.0e-6f;
    float rx = p1x - p2x;
    float ry = p1y - p2y;
    float rz = p1z - p2z;
    float a = d1x * d1x + d1y * d1y + d1z * d1z;
    float e = d2x * d2x + d2y * d2y + d2z * d2z;
    float f = d2x * rx + d2y * ry + d2z * rz;
    float s = 0.0f;
    float t = 0.0f;
    if (a <= length_epsilon && e > length_epsilon) {
        t = clampf(f / e, 0.0f, 1.0f);
    } else if (a > length_epsilon) {
        float c = d1x * rx + d1y * ry + d1z * rz;
        if (e <= length_epsilon) {
            s = clampf(-c / a, 0.0f, 1.0f);
        } else {
            float b = d1x * d2x + d1y * d2y + d1z * d2z;
            float denominator = a * e - b * b;
            if (std::fabs(denominator) > parallel_relative_epsilon * a * e) {
                s = clampf((b * f - c * e) / denominator, 0.0f, 1.0f);
            }
            float projected = (b * s + f) / e;
            if (projected < 0.0f) {
                s = clampf(-c / a, 0.0f, 1.0f);
            } else if (projected > 1.0f) {
                t = 1.0f;
                s = clampf((b - c) / a, 0.0f, 1.0f);
            } else {
                t = projected;
            }
        }
    }
    float delta_x = (p2x + d2x * t) - (p1x + d1x * s);
    float delta_y = (p2y + d2y * t) - (p1y + d1y * s);
    float delta_z = (p2z + d2z * t) - (p1z + d1z * s);
    return std::sqrt(delta_x * delta_x + delta_y * delta_y + delta_z * delta_z);
}

}  // namespace

struct orc_world {
    uint32_t V = 0, S = 0, F = 0;
    std::vector<float> positions, intrinsic;
    std::vector<uint32_t> segment_vertices, segment_fibers;
    std::vector<float> radii, rest_lengths;
    std::vector<uint32_t> fiber_vertex_spans, fiber_segment_spans;
    std::vector<uint32_t> vertex_segments;
    std::vector<float> max_curvature;
    std::vector<uint32_t> pinned;
    std::vector<float> arc;          /* packed.rs:561-580 */
    std::vector<float> wall_extents; /* packed.rs:527-546 */
    Grid grid{};
    float cell_size = 0.0f;
    float neighbor_skin = 0.0f;
    uint32_t neighbor_capacity = 0;
    uint64_t neighbor_slots = 0;
    uint32_t neighbor_block = 0;
    /* world.rs:466-468: active, lifetime iterations, batch iterations, failure */
    uint32_t control[4] = {0, 0, 0, 0};
    float metrics[3];
    uint32_t neighbor_state[2] = {1, 0};
    uint32_t cell_overflow = 0;
    std::vector<uint32_t> cell_counts, cell_offsets, cell_segments;
    std::vector<uint32_t> neighbor_counts, neighbor_segments;
    std::vector<float> reference_positions;
    std::vector<float> corrections, segment_max, curvature_ratio, internal, vertex_step,
        wall_reactions;
    /* Curvature triplets that moved a vertex (a diagnostic count). */
    uint64_t projections = 0;
    /* Staged activation (kernels.rs:164-221; world.rs:2139-2183): the
     * segment_active / vertex_active masks, derived per fiber, and the
     * active segment count (the cell list's slots). */
    std::vector<uint8_t> fiber_on, segment_on, vertex_on;
    std::vector<uint32_t> vertex_fiber;
    uint32_t slots = 0;
    uint64_t allocated_cells = 0;
    float maximum_radius = 0.0f;
    /* Formation layer target (world.rs:1723-1810) and vertex targets
     * (world.rs:1811-1863). */
    bool layer_on = false;
    uint32_t layer_axis = 0, layer_first = 0, layer_last = 0;
    float layer_stiffness = 0.0f, layer_max_translation = 0.0f;
    std::vector<float> layer_targets;
    std::vector<uint32_t> fiber_layers;
    bool targets_on = false;
    uint32_t target_axis = 0;
    float target_stiffness = 0.0f, target_max_translation = 0.0f;
    std::vector<uint32_t> target_vertices;
    std::vector<float> target_coordinates, command_coordinates;
};

namespace {

/* world.rs:308-417 and :874-917 for a uniform layout. */
int size_world(orc_world &w, const orc_cell_list_config &cl, float max_step) {
    float maximum_rest_length = 0.0f;
    for (uint32_t s = 0; s < w.S; ++s) maximum_rest_length = std::fmax(maximum_rest_length, w.rest_lengths[s]);
    float maximum_initial_length = 0.0f;
    for (uint32_t s = 0; s < w.S; ++s) {
        uint32_t first = w.segment_vertices[2 * s], second = w.segment_vertices[2 * s + 1];
        float dx = w.positions[3 * second] - w.positions[3 * first];
        float dy = w.positions[3 * second + 1] - w.positions[3 * first + 1];
        float dz = w.positions[3 * second + 2] - w.positions[3 * first + 2];
        maximum_initial_length = std::fmax(maximum_initial_length, std::sqrt(dx * dx + dy * dy + dz * dz));
    }
    float maximum_length = std::fmax(maximum_rest_length, maximum_initial_length);
    float maximum_radius = 0.0f;
    for (uint32_t s = 0; s < w.S; ++s) maximum_radius = std::fmax(maximum_radius, w.radii[s]);
    w.neighbor_skin = cl.neighbor_skin_scale * maximum_radius;
    float interaction_margin = 2.0f * maximum_radius + std::fmax(2.0f * max_step, w.neighbor_skin);
    /* Every segment is a leaf, so list_block_length == maximum_length and
     * every list weight and proxy count is ceil(len / max_len).max(1) == 1. */
    float list_block_length = std::fmin(maximum_length, std::fmax(maximum_length, 2.0f * interaction_margin));
    for (uint32_t s = 0; s < w.S; ++s) {
        uint32_t first = w.segment_vertices[2 * s], second = w.segment_vertices[2 * s + 1];
        float dx = w.positions[3 * second] - w.positions[3 * first];
        float dy = w.positions[3 * second + 1] - w.positions[3 * first + 1];
        float dz = w.positions[3 * second + 2] - w.positions[3 * first + 2];
        float length = std::fmax(w.rest_lengths[s], std::sqrt(dx * dx + dy * dy + dz * dz));
        uint32_t weight = std::max(f32_to_u32(std::ceil(length / list_block_length)), 1u);
        if (weight != 1) return fail("internal: a uniform layout produced a list weight above one");
    }
    float piece_length = list_block_length;
    w.cell_size = (piece_length + interaction_margin) * cl.cell_size_scale;
    float extent[3];
    for (int a = 0; a < 3; ++a) extent[a] = w.grid.upper[a] - w.grid.lower[a];
    uint32_t dims[3];
    for (int a = 0; a < 3; ++a) {
        float cells = std::fmax(std::floor(extent[a] / w.cell_size), 1.0f);
        dims[a] = f32_to_u32(cells);
    }
    uint64_t cell_count = checked_cell_count(dims, 1ull << 31);
    if (cell_count == 0 || !(w.cell_size > 0.0f)) return fail("cell grid too large: the cell size is tiny against the box");
    w.grid.cx = dims[0];
    w.grid.cy = dims[1];
    w.grid.cz = dims[2];
    uint64_t max_bytes = cl.max_list_bytes ? cl.max_list_bytes : REFERENCE_MAX_LIST_BYTES;
    w.neighbor_capacity = cl.neighbor_capacity;
    uint64_t slots = std::min<uint64_t>((uint64_t)cl.neighbor_capacity * w.S, max_bytes / 4);
    w.neighbor_slots = std::max<uint64_t>(slots, 1);
    uint64_t total = std::max<uint64_t>(w.S, 1);
    w.neighbor_block = (uint32_t)std::min<uint64_t>(cl.neighbor_capacity,
                                                    std::min<uint64_t>(w.neighbor_slots / total, 0xFFFFFFFFull));
    w.allocated_cells = cell_count;
    w.maximum_radius = maximum_radius;
    w.cell_counts.assign(cell_count, 0);
    w.cell_offsets.assign(cell_count, 0);
    w.cell_segments.assign(w.S, 0);
    w.neighbor_counts.assign(w.S, 0);
    w.neighbor_segments.assign((size_t)w.neighbor_block * w.S, 0);
    return 0;
}

/* Cell-list build: cell_list.rs:8-378, world/cell_list.rs:94-209. A stable
 * counting sort over ascending segment index gives the ranked order
 * rank_cell_segments produces (ascending segment within each cell). */
void build_cell_list(orc_world &w) {
    std::fill(w.cell_counts.begin(), w.cell_counts.end(), 0u);
    w.cell_overflow = 0;
    std::vector<uint32_t> cell_of(w.S);
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < (int64_t)w.S; ++s) {
        if (!w.segment_on[s]) continue; /* inactive segments stay out of the cell list */
        uint32_t first = w.segment_vertices[2 * s], second = w.segment_vertices[2 * s + 1];
        const float *p = &w.positions[3 * first];
        const float *q = &w.positions[3 * second];
        cell_of[s] = proxy_cell(p[0], p[1], p[2], q[0], q[1], q[2], w.grid);
    }
    for (uint32_t s = 0; s < w.S; ++s)
        if (w.segment_on[s]) w.cell_counts[cell_of[s]] += 1;
    uint32_t running = 0;
    for (size_t c = 0; c < w.cell_counts.size(); ++c) {
        w.cell_offsets[c] = running;
        running += w.cell_counts[c];
    }
    w.slots = running;
    std::vector<uint32_t> cursor(w.cell_counts.size(), 0);
    for (uint32_t s = 0; s < w.S; ++s) {
        if (!w.segment_on[s]) continue;
        uint32_t c = cell_of[s];
        w.cell_segments[w.cell_offsets[c] + cursor[c]++] = s;
    }
}

/* neighbor.rs:109-411 and world/neighbor_list.rs:19-114: one slot (one
 * segment here) at a time; each list sorted ascending by segment. */
void build_neighbor_lists(orc_world &w) {
    build_cell_list(w);
    const float length_x = w.grid.upper[0] - w.grid.lower[0];
    const float length_y = w.grid.upper[1] - w.grid.lower[1];
    const float length_z = w.grid.upper[2] - w.grid.lower[2];
    const uint32_t block = w.neighbor_block;
    const float skin = w.neighbor_skin;
#pragma omp parallel
    {
        std::vector<uint32_t> found;
#pragma omp for schedule(dynamic, 256)
        for (int64_t slot = 0; slot < (int64_t)w.slots; ++slot) {
            uint32_t segment = w.cell_segments[slot];
            uint32_t first_vertex = w.segment_vertices[2 * segment];
            uint32_t second_vertex = w.segment_vertices[2 * segment + 1];
            float p1x = w.positions[3 * first_vertex], p1y = w.positions[3 * first_vertex + 1],
                  p1z = w.positions[3 * first_vertex + 2];
            float q1x = w.positions[3 * second_vertex], q1y = w.positions[3 * second_vertex + 1],
                  q1z = w.positions[3 * second_vertex + 2];
            float d1x = q1x - p1x, d1y = q1y - p1y, d1z = q1z - p1z;
            uint32_t owner = w.segment_fibers[segment];
            float radius = w.radii[segment];
            float half_length = 0.5f * std::sqrt(d1x * d1x + d1y * d1y + d1z * d1z);
            uint32_t home = proxy_cell(p1x, p1y, p1z, q1x, q1y, q1z, w.grid);
            found.clear();
            for (uint32_t neighbor = 0; neighbor < 27; ++neighbor) {
                uint32_t cell = stencil_cell(home, neighbor, w.grid);
                if (cell == NONE) continue;
                uint32_t candidates = w.cell_counts[cell];
                uint32_t start = w.cell_offsets[cell];
                for (uint32_t local = 0; local < candidates; ++local) {
                    uint32_t other = w.cell_segments[start + local];
                    uint32_t third_vertex = w.segment_vertices[2 * other];
                    uint32_t fourth_vertex = w.segment_vertices[2 * other + 1];
                    float gap = along_fiber_gap(w.arc.data(), first_vertex, second_vertex, third_vertex, fourth_vertex);
                    float other_radius = w.radii[other];
                    bool near_along_fiber = w.segment_fibers[other] == owner && gap < radius + other_radius;
                    if (other == segment || near_along_fiber) continue;
                    float p2x = w.positions[3 * third_vertex], p2y = w.positions[3 * third_vertex + 1],
                          p2z = w.positions[3 * third_vertex + 2];
                    float q2x = w.positions[3 * fourth_vertex], q2y = w.positions[3 * fourth_vertex + 1],
                          q2z = w.positions[3 * fourth_vertex + 2];
                    if (w.grid.periodic[0]) {
                        float image_shift = std::round(0.5f * (p2x + q2x - p1x - q1x) / length_x) * length_x;
                        p2x -= image_shift;
                        q2x -= image_shift;
                    }
                    if (w.grid.periodic[1]) {
                        float image_shift = std::round(0.5f * (p2y + q2y - p1y - q1y) / length_y) * length_y;
                        p2y -= image_shift;
                        q2y -= image_shift;
                    }
                    if (w.grid.periodic[2]) {
                        float image_shift = std::round(0.5f * (p2z + q2z - p1z - q1z) / length_z) * length_z;
                        p2z -= image_shift;
                        q2z -= image_shift;
                    }
                    float d2x = q2x - p2x, d2y = q2y - p2y, d2z = q2z - p2z;
                    float interaction = (radius + other_radius + skin) * (1.0f + 1.0e-4f);
                    float midpoint_dx = 0.5f * (p2x + q2x - p1x - q1x);
                    float midpoint_dy = 0.5f * (p2y + q2y - p1y - q1y);
                    float midpoint_dz = 0.5f * (p2z + q2z - p1z - q1z);
                    float reach = half_length + 0.5f * std::sqrt(d2x * d2x + d2y * d2y + d2z * d2z) + interaction;
                    if (midpoint_dx * midpoint_dx + midpoint_dy * midpoint_dy + midpoint_dz * midpoint_dz <=
                            reach * reach &&
                        proxy_pair_axis_distance(p1x, p1y, p1z, d1x, d1y, d1z, p2x, p2y, p2z, d2x, d2y, d2z) <=
                            interaction) {
                        found.push_back(other);
                    }
                }
            }
            uint32_t count = (uint32_t)found.size();
            w.neighbor_counts[segment] = count;
            /* sort_neighbor_lists only orders lists that fit; an overflowed
             * list is never read (contact.rs:357-363). */
            if (count <= block) std::sort(found.begin(), found.end());
            uint32_t keep = std::min(count, block);
            std::copy(found.begin(), found.begin() + keep,
                      w.neighbor_segments.begin() + (size_t)block * segment);
        }
    }
    w.reference_positions = w.positions; /* neighbor.rs:411-422 */
}

/* world/neighbor_list.rs:19-114 gated on neighbor_state[0]. */
void rebuild_neighbor_lists_if_requested(orc_world &w) {
    if (w.neighbor_state[0] == 0) return;
    build_neighbor_lists(w);
    w.neighbor_state[0] = 0; /* neighbor.rs:426-432 */
    w.neighbor_state[1] += 1;
}

/* neighbor.rs:446-465. */
void flag_neighbor_list_displacement(orc_world &w) {
    float maximum_displacement = 0.5f * w.neighbor_skin;
    uint32_t flag = 0;
#pragma omp parallel for schedule(static) reduction(| : flag)
    for (int64_t v = 0; v < (int64_t)w.V; ++v) {
        if (!w.vertex_on[v]) continue;
        float dx = w.positions[3 * v] - w.reference_positions[3 * v];
        float dy = w.positions[3 * v + 1] - w.reference_positions[3 * v + 1];
        float dz = w.positions[3 * v + 2] - w.reference_positions[3 * v + 2];
        if (dx * dx + dy * dy + dz * dz > maximum_displacement * maximum_displacement) flag = 1;
    }
    if (flag) w.neighbor_state[0] = 1;
}

/* contact.rs:232-902, one round lane per segment. */
void find_segment_corrections(orc_world &w, float correction_fraction, uint32_t aggregation) {
    const float length_x = w.grid.upper[0] - w.grid.lower[0];
    const float length_y = w.grid.upper[1] - w.grid.lower[1];
    const float length_z = w.grid.upper[2] - w.grid.lower[2];
    const uint32_t block = w.neighbor_block;
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t si = 0; si < (int64_t)w.S; ++si) {
        const uint32_t segment = (uint32_t)si;
        if (!w.segment_on[segment]) continue; /* active_segments only (contact.rs:268-272) */
        uint32_t first_vertex = w.segment_vertices[2 * segment];
        uint32_t second_vertex = w.segment_vertices[2 * segment + 1];
        float p1x = w.positions[3 * first_vertex], p1y = w.positions[3 * first_vertex + 1],
              p1z = w.positions[3 * first_vertex + 2];
        float q1x = w.positions[3 * second_vertex], q1y = w.positions[3 * second_vertex + 1],
              q1z = w.positions[3 * second_vertex + 2];
        float d1x = q1x - p1x, d1y = q1y - p1y, d1z = q1z - p1z;
        uint32_t owner = w.segment_fibers[segment];
        float radius = w.radii[segment];
        float half_length = 0.5f * std::sqrt(d1x * d1x + d1y * d1y + d1z * d1z);
        const float length_epsilon = 1.0e-20f;
        const float parallel_relative_epsilon = 1.0e-6f;
        float c0x = 0.0f, c0y = 0.0f, c0z = 0.0f, c1x = 0.0f, c1y = 0.0f, c1z = 0.0f;
        float maximum_penetration = 0.0f;
        float correction_weight = 0.0f;
        uint32_t listed_count = w.neighbor_counts[segment];
        bool listed = listed_count <= block;
        uint32_t ranges = listed ? 1u : 27u;
        uint32_t home_cell = 0;
        if (!listed) {
            const float *rp = &w.reference_positions[3 * first_vertex];
            const float *rq = &w.reference_positions[3 * second_vertex];
            home_cell = proxy_cell(rp[0], rp[1], rp[2], rq[0], rq[1], rq[2], w.grid);
        }
        for (uint32_t range = 0; range < ranges; ++range) {
            uint32_t count = 0;
            size_t start = 0;
            if (listed) {
                count = listed_count;
                start = (size_t)block * segment;
            } else {
                uint32_t cell = stencil_cell(home_cell, range, w.grid);
                if (cell != NONE) {
                    count = w.cell_counts[cell];
                    start = w.cell_offsets[cell];
                }
            }
            for (uint32_t slot = 0; slot < count; ++slot) {
                uint32_t other = listed ? w.neighbor_segments[start + slot] : w.cell_segments[start + slot];
                uint32_t third_vertex = w.segment_vertices[2 * other];
                uint32_t fourth_vertex = w.segment_vertices[2 * other + 1];
                float gap = along_fiber_gap(w.arc.data(), first_vertex, second_vertex, third_vertex, fourth_vertex);
                float other_radius = w.radii[other];
                bool near_along_fiber = w.segment_fibers[other] == owner && gap < radius + other_radius;
                if (other == segment || near_along_fiber) continue;
                float p2x = w.positions[3 * third_vertex], p2y = w.positions[3 * third_vertex + 1],
                      p2z = w.positions[3 * third_vertex + 2];
                float q2x = w.positions[3 * fourth_vertex], q2y = w.positions[3 * fourth_vertex + 1],
                      q2z = w.positions[3 * fourth_vertex + 2];
                float image_dx = 0.5f * (p2x + q2x - p1x - q1x);
                float image_dy = 0.5f * (p2y + q2y - p1y - q1y);
                float image_dz = 0.5f * (p2z + q2z - p1z - q1z);
                if (w.grid.periodic[0]) {
                    float image_shift = std::round(image_dx / length_x) * length_x;
                    p2x -= image_shift;
                    q2x -= image_shift;
                }
                if (w.grid.periodic[1]) {
                    float image_shift = std::round(image_dy / length_y) * length_y;
                    p2y -= image_shift;
                    q2y -= image_shift;
                }
                if (w.grid.periodic[2]) {
                    float image_shift = std::round(image_dz / length_z) * length_z;
                    p2z -= image_shift;
                    q2z -= image_shift;
                }
                float d2x = q2x - p2x, d2y = q2y - p2y, d2z = q2z - p2z;
                float midpoint_dx = 0.5f * (p2x + q2x - p1x - q1x);
                float midpoint_dy = 0.5f * (p2y + q2y - p1y - q1y);
                float midpoint_dz = 0.5f * (p2z + q2z - p1z - q1z);
                float reach = (half_length + 0.5f * std::sqrt(d2x * d2x + d2y * d2y + d2z * d2z) + radius +
                               other_radius) *
                              (1.0f + 1.0e-4f);
                if (!(midpoint_dx * midpoint_dx + midpoint_dy * midpoint_dy + midpoint_dz * midpoint_dz <=
                      reach * reach))
                    continue;
                /* contact.rs:663-728: lane offsets are zero, so the lane
                 * segment is the segment itself. */
                float rx = p1x - p2x, ry = p1y - p2y, rz = p1z - p2z;
                float a = d1x * d1x + d1y * d1y + d1z * d1z;
                float e = d2x * d2x + d2y * d2y + d2z * d2z;
                float f = d2x * rx + d2y * ry + d2z * rz;
                float s = 0.0f, t = 0.0f;
                if (a <= length_epsilon && e > length_epsilon) {
                    t = clampf(f / e, 0.0f, 1.0f);
                } else if (a > length_epsilon) {
                    float c = d1x * rx + d1y * ry + d1z * rz;
                    if (e <= length_epsilon) {
                        s = clampf(-c / a, 0.0f, 1.0f);
                    } else {
                        float b = d1x * d2x + d1y * d2y + d1z * d2z;
                        float denominator = a * e - b * b;
                        bool parallel = std::fabs(denominator) <= parallel_relative_epsilon * a * e;
                        if (!parallel) s = clampf((b * f - c * e) / denominator, 0.0f, 1.0f);
                        float projected = (b * s + f) / e;
                        if (projected < 0.0f) {
                            s = clampf(-c / a, 0.0f, 1.0f);
                        } else if (projected > 1.0f) {
                            t = 1.0f;
                            s = clampf((b - c) / a, 0.0f, 1.0f);
                        } else {
                            t = projected;
                        }
                        if (parallel) {
                            float end_s = 1.0f, end_t = 0.0f;
                            float end_projected = (b + f) / e;
                            if (end_projected < 0.0f) {
                                end_s = clampf(-c / a, 0.0f, 1.0f);
                            } else if (end_projected > 1.0f) {
                                end_t = 1.0f;
                                end_s = clampf((b - c) / a, 0.0f, 1.0f);
                            } else {
                                end_t = end_projected;
                            }
                            float gap_x = rx + d1x * s - d2x * t;
                            float gap_y = ry + d1y * s - d2y * t;
                            float gap_z = rz + d1z * s - d2z * t;
                            float end_gap_x = rx + d1x * end_s - d2x * end_t;
                            float end_gap_y = ry + d1y * end_s - d2y * end_t;
                            float end_gap_z = rz + d1z * end_s - d2z * end_t;
                            if (end_gap_x * end_gap_x + end_gap_y * end_gap_y + end_gap_z * end_gap_z <
                                gap_x * gap_x + gap_y * gap_y + gap_z * gap_z) {
                                s = end_s;
                                t = end_t;
                            }
                        }
                    }
                }
                float point1x = p1x + d1x * s, point1y = p1y + d1y * s, point1z = p1z + d1z * s;
                float point2x = p2x + d2x * t, point2y = p2y + d2y * t, point2z = p2z + d2z * t;
                float delta_x = point2x - point1x, delta_y = point2y - point1y, delta_z = point2z - point1z;
                float distance = std::sqrt(delta_x * delta_x + delta_y * delta_y + delta_z * delta_z);
                float penetration = radius + other_radius - distance;
                if (!(penetration > 0.0f)) continue;
                bool deepest = penetration > maximum_penetration;
                if (deepest) maximum_penetration = penetration;
                float nx, ny, nz;
                if (distance > 1.0e-7f) {
                    float inverse_distance = 1.0f / distance;
                    nx = delta_x * inverse_distance;
                    ny = delta_y * inverse_distance;
                    nz = delta_z * inverse_distance;
                } else {
                    /* contact.rs:768-812 */
                    nx = d1y * d2z - d1z * d2y;
                    ny = d1z * d2x - d1x * d2z;
                    nz = d1x * d2y - d1y * d2x;
                    float normal_length = std::sqrt(nx * nx + ny * ny + nz * nz);
                    if (normal_length <= 1.0e-7f) {
                        if (std::fabs(d1x) <= std::fabs(d1y) && std::fabs(d1x) <= std::fabs(d1z)) {
                            nx = 0.0f;
                            ny = d1z;
                            nz = -d1y;
                        } else if (std::fabs(d1y) <= std::fabs(d1z)) {
                            nx = -d1z;
                            ny = 0.0f;
                            nz = d1x;
                        } else {
                            nx = d1y;
                            ny = -d1x;
                            nz = 0.0f;
                        }
                        normal_length = std::sqrt(nx * nx + ny * ny + nz * nz);
                    }
                    if (normal_length > 1.0e-7f) {
                        nx /= normal_length;
                        ny /= normal_length;
                        nz /= normal_length;
                    } else {
                        nx = 1.0f;
                    }
                    float dominant;
                    if (std::fabs(nx) >= std::fabs(ny) && std::fabs(nx) >= std::fabs(nz))
                        dominant = nx;
                    else if (std::fabs(ny) >= std::fabs(nz))
                        dominant = ny;
                    else
                        dominant = nz;
                    if (dominant < 0.0f) {
                        nx = -nx;
                        ny = -ny;
                        nz = -nz;
                    }
                    if (segment > other) {
                        nx = -nx;
                        ny = -ny;
                        nz = -nz;
                    }
                }
                /* contact.rs:814-870 with every turn term zero. */
                float weight_0 = 1.0f - s;
                float weight_1 = s;
                float other_weight_0 = 1.0f - t;
                float denominator = weight_0 * weight_0 + weight_1 * weight_1 + other_weight_0 * other_weight_0 + t * t;
                float magnitude = -correction_fraction * penetration / denominator;
                float aggregate_weight = 1.0f;
                if (aggregation == 1) aggregate_weight = penetration;
                if (aggregation == 2) {
                    if (deepest) {
                        c0x = nx * magnitude * weight_0;
                        c0y = ny * magnitude * weight_0;
                        c0z = nz * magnitude * weight_0;
                        c1x = nx * magnitude * weight_1;
                        c1y = ny * magnitude * weight_1;
                        c1z = nz * magnitude * weight_1;
                        correction_weight = 1.0f;
                    }
                } else {
                    c0x += nx * magnitude * weight_0 * aggregate_weight;
                    c0y += ny * magnitude * weight_0 * aggregate_weight;
                    c0z += nz * magnitude * weight_0 * aggregate_weight;
                    c1x += nx * magnitude * weight_1 * aggregate_weight;
                    c1y += ny * magnitude * weight_1 * aggregate_weight;
                    c1z += nz * magnitude * weight_1 * aggregate_weight;
                    correction_weight += aggregate_weight;
                }
            }
        }
        if (aggregation != 2 && correction_weight > 1.0e-20f) {
            c0x /= correction_weight;
            c0y /= correction_weight;
            c0z /= correction_weight;
            c1x /= correction_weight;
            c1y /= correction_weight;
            c1z /= correction_weight;
        }
        float *out = &w.corrections[6 * (size_t)segment];
        out[0] = c0x;
        out[1] = c0y;
        out[2] = c0z;
        out[3] = c1x;
        out[4] = c1y;
        out[5] = c1z;
        w.segment_max[segment] = maximum_penetration;
    }
}

/* kernels.rs:925-980. */
void measure_curvature_ratio(orc_world &w) {
#pragma omp parallel for schedule(static)
    for (int64_t vi = 0; vi < (int64_t)w.V; ++vi) {
        uint32_t index = (uint32_t)vi;
        if (!w.vertex_on[index]) continue; /* inactive vertices keep their last ratio */
        float maximum = w.max_curvature[index];
        float ratio = 0.0f;
        uint32_t previous_segment = w.vertex_segments[2 * index];
        uint32_t next_segment = w.vertex_segments[2 * index + 1];
        if (maximum > 0.0f && previous_segment != NONE && next_segment != NONE) {
            uint32_t pa = w.segment_vertices[2 * previous_segment], pb = w.segment_vertices[2 * previous_segment + 1];
            uint32_t previous = pa == index ? pb : pa;
            uint32_t na = w.segment_vertices[2 * next_segment], nb = w.segment_vertices[2 * next_segment + 1];
            uint32_t next = na == index ? nb : na;
            const float *P = w.positions.data();
            float ax = P[3 * index] - P[3 * previous];
            float ay = P[3 * index + 1] - P[3 * previous + 1];
            float az = P[3 * index + 2] - P[3 * previous + 2];
            float bx = P[3 * next] - P[3 * index];
            float by = P[3 * next + 1] - P[3 * index + 1];
            float bz = P[3 * next + 2] - P[3 * index + 2];
            float first_length = std::sqrt(ax * ax + ay * ay + az * az);
            float second_length = std::sqrt(bx * bx + by * by + bz * bz);
            if (first_length > 1.0e-7f && second_length > 1.0e-7f) {
                float cosine = (ax * bx + ay * by + az * bz) / (first_length * second_length);
                cosine = clampf(cosine, -1.0f, 1.0f);
                float dual_length = 0.5f * (first_length + second_length);
                float curvature = 2.0f * std::sqrt(0.5f * (1.0f - cosine)) / dual_length;
                ratio = curvature / maximum;
            }
        }
        w.curvature_ratio[index] = ratio;
    }
}

/* kernels.rs:95-162: atomic u32 max of non-negative f32 bits, then the gate. */
void reduce_and_assess(orc_world &w, const orc_relax_config &config, uint32_t max_iterations) {
    uint32_t reduced[3] = {0, 0, 0};
    for (uint32_t s = 0; s < w.S; ++s)
        if (w.segment_on[s]) reduced[0] = std::max(reduced[0], f32_bits(std::fmax(w.segment_max[s], 0.0f)));
    for (uint32_t v = 0; v < w.V; ++v) {
        if (!w.vertex_on[v]) continue;
        reduced[1] = std::max(reduced[1], f32_bits(std::fmax(w.vertex_step[v], 0.0f)));
        reduced[2] = std::max(reduced[2], f32_bits(std::fmax(w.curvature_ratio[v], 0.0f)));
    }
    float maximum_penetration = bits_f32(reduced[0]);
    float maximum_curvature_ratio = bits_f32(reduced[2]);
    w.metrics[0] = maximum_penetration;
    w.metrics[1] = bits_f32(reduced[1]);
    w.metrics[2] = maximum_curvature_ratio;
    if (w.cell_overflow != 0 ||
        (config.force_full_iterations == 0 && maximum_penetration <= config.penetration_tolerance &&
         maximum_curvature_ratio <= 1.0f + config.curvature_ratio_tolerance) ||
        w.control[2] >= max_iterations) {
        if (w.cell_overflow != 0) w.control[3] = 1;
        w.control[0] = 0;
    } else {
        w.control[1] += 1;
        w.control[2] += 1;
    }
}

/* kernels.rs:1027-1163 (Jacobi) then :1417-1453. */
void internal_pass(orc_world &w, float stretch_stiffness, float bend_stiffness) {
    const float *P = w.positions.data();
    const float *X = w.intrinsic.data();
#pragma omp parallel for schedule(static)
    for (int64_t vi = 0; vi < (int64_t)w.V; ++vi) {
        uint32_t index = (uint32_t)vi;
        float *out = &w.internal[3 * (size_t)index];
        if (!w.vertex_on[index]) continue;
        if (w.pinned[index]) {
            out[0] = out[1] = out[2] = 0.0f;
            continue;
        }
        float x = P[3 * index], y = P[3 * index + 1], z = P[3 * index + 2];
        float cx = 0.0f, cy = 0.0f, cz = 0.0f;
        uint32_t previous_segment = w.vertex_segments[2 * index];
        uint32_t next_segment = w.vertex_segments[2 * index + 1];
        for (int side = 0; side < 2; ++side) {
            uint32_t segment = side == 0 ? previous_segment : next_segment;
            if (segment == NONE) continue;
            uint32_t first = w.segment_vertices[2 * segment], second = w.segment_vertices[2 * segment + 1];
            uint32_t other = first == index ? second : first;
            float dx = P[3 * other] - x, dy = P[3 * other + 1] - y, dz = P[3 * other + 2] - z;
            float length = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (length > 1.0e-7f) {
                float magnitude = 0.5f * stretch_stiffness * (length - w.rest_lengths[segment]) / length;
                cx += dx * magnitude;
                cy += dy * magnitude;
                cz += dz * magnitude;
            }
        }
        for (int side = 0; side < 2; ++side) {
            uint32_t adjacent = side == 0 ? previous_segment : next_segment;
            if (adjacent == NONE) continue;
            uint32_t first = w.segment_vertices[2 * adjacent], second = w.segment_vertices[2 * adjacent + 1];
            uint32_t middle = first == index ? second : first;
            uint32_t outer_segment = w.vertex_segments[2 * middle + (side == 0 ? 0 : 1)];
            if (outer_segment == NONE) continue;
            uint32_t outer_first = w.segment_vertices[2 * outer_segment];
            uint32_t outer_second = w.segment_vertices[2 * outer_segment + 1];
            uint32_t other = outer_first == middle ? outer_second : outer_first;
            float dx = P[3 * other] - x, dy = P[3 * other + 1] - y, dz = P[3 * other + 2] - z;
            float length = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (length > 1.0e-7f) {
                float rx = X[3 * other] - X[3 * index];
                float ry = X[3 * other + 1] - X[3 * index + 1];
                float rz = X[3 * other + 2] - X[3 * index + 2];
                float rest_chord = std::sqrt(rx * rx + ry * ry + rz * rz);
                float magnitude = 0.5f * bend_stiffness * (length - rest_chord) / length;
                cx += dx * magnitude;
                cy += dy * magnitude;
                cz += dz * magnitude;
            }
        }
        out[0] = cx;
        out[1] = cy;
        out[2] = cz;
    }
#pragma omp parallel for schedule(static)
    for (int64_t vi = 0; vi < (int64_t)w.V; ++vi) {
        uint32_t index = (uint32_t)vi;
        if (!w.vertex_on[index] || w.pinned[index]) continue;
        for (int axis = 0; axis < 3; ++axis) {
            size_t coordinate = 3 * (size_t)index + axis;
            float radius = w.wall_extents[coordinate];
            float moved = w.positions[coordinate] + w.internal[coordinate];
            w.positions[coordinate] = w.grid.periodic[axis]
                                          ? moved
                                          : clampf(moved, w.grid.lower[axis] + radius, w.grid.upper[axis] - radius);
            if (!w.grid.periodic[axis]) w.wall_reactions[coordinate] += moved - w.positions[coordinate];
        }
    }
}

/* kernels.rs:1455-1537. */
void apply_contact_corrections(orc_world &w, float max_step) {
#pragma omp parallel for schedule(static)
    for (int64_t vi = 0; vi < (int64_t)w.V; ++vi) {
        uint32_t index = (uint32_t)vi;
        if (!w.vertex_on[index]) continue;
        if (w.pinned[index]) {
            w.vertex_step[index] = 0.0f;
            continue;
        }
        uint32_t previous = w.vertex_segments[2 * index];
        uint32_t next = w.vertex_segments[2 * index + 1];
        float cx = 0.0f, cy = 0.0f, cz = 0.0f;
        if (previous != NONE) {
            cx += w.corrections[6 * (size_t)previous + 3];
            cy += w.corrections[6 * (size_t)previous + 4];
            cz += w.corrections[6 * (size_t)previous + 5];
        }
        if (next != NONE) {
            cx += w.corrections[6 * (size_t)next];
            cy += w.corrections[6 * (size_t)next + 1];
            cz += w.corrections[6 * (size_t)next + 2];
        }
        float length = std::sqrt(cx * cx + cy * cy + cz * cz);
        if (length > max_step) {
            float scale = max_step / length;
            cx *= scale;
            cy *= scale;
            cz *= scale;
        }
        float c[3] = {cx, cy, cz};
        for (int axis = 0; axis < 3; ++axis) {
            size_t coordinate = 3 * (size_t)index + axis;
            float radius = w.wall_extents[coordinate];
            float moved = w.positions[coordinate] + c[axis];
            w.positions[coordinate] = w.grid.periodic[axis]
                                          ? moved
                                          : clampf(moved, w.grid.lower[axis] + radius, w.grid.upper[axis] - radius);
            if (!w.grid.periodic[axis]) w.wall_reactions[coordinate] += moved - w.positions[coordinate];
        }
        w.vertex_step[index] = std::sqrt(cx * cx + cy * cy + cz * cz);
    }
}

/* kernels.rs:1165-1322. */
void project_curvature_triplet(orc_world &w, uint32_t previous, uint32_t center, uint32_t next, float stiffness,
                               float safety_margin) {
    float maximum_curvature = w.max_curvature[center] * (1.0f - safety_margin);
    if (!(maximum_curvature > 0.0f)) return;
    float *P = w.positions.data();
    float ux = P[3 * center] - P[3 * previous];
    float uy = P[3 * center + 1] - P[3 * previous + 1];
    float uz = P[3 * center + 2] - P[3 * previous + 2];
    float vx = P[3 * next] - P[3 * center];
    float vy = P[3 * next + 1] - P[3 * center + 1];
    float vz = P[3 * next + 2] - P[3 * center + 2];
    float first_length = std::sqrt(ux * ux + uy * uy + uz * uz);
    float second_length = std::sqrt(vx * vx + vy * vy + vz * vz);
    if (!(first_length > 1.0e-7f && second_length > 1.0e-7f)) return;
    float unx = ux / first_length, uny = uy / first_length, unz = uz / first_length;
    float vnx = vx / second_length, vny = vy / second_length, vnz = vz / second_length;
    float cosine = clampf(unx * vnx + uny * vny + unz * vnz, -1.0f, 1.0f);
    float sine_half = 0.25f * maximum_curvature * (first_length + second_length);
    if (!(sine_half < 1.0f)) return;
    float minimum_cosine = 1.0f - 2.0f * sine_half * sine_half;
    float violation = minimum_cosine - cosine;
    float sine = std::sqrt(std::fmax(1.0f - cosine * cosine, 0.0f));
    if (violation > 0.0f && sine > 1.0e-3f) violation = (acos_f32(cosine) - acos_f32(minimum_cosine)) * sine;
    if (!(violation > 0.0f)) return;
    float gux = (vnx - cosine * unx) / first_length;
    float guy = (vny - cosine * uny) / first_length;
    float guz = (vnz - cosine * unz) / first_length;
    float gvx = (unx - cosine * vnx) / second_length;
    float gvy = (uny - cosine * vny) / second_length;
    float gvz = (unz - cosine * vnz) / second_length;
    float cgx = gux - gvx, cgy = guy - gvy, cgz = guz - gvz;
    float previous_weight = w.pinned[previous] ? 0.0f : 1.0f;
    float center_weight = w.pinned[center] ? 0.0f : 1.0f;
    float next_weight = w.pinned[next] ? 0.0f : 1.0f;
    float denominator = previous_weight * (gux * gux + guy * guy + guz * guz) +
                        center_weight * (cgx * cgx + cgy * cgy + cgz * cgz) +
                        next_weight * (gvx * gvx + gvy * gvy + gvz * gvz);
    if (!(denominator > 1.0e-12f)) return;
    if (previous_weight > 0.0f || center_weight > 0.0f || next_weight > 0.0f)
        __atomic_fetch_add(&w.projections, 1, __ATOMIC_RELAXED);
    float scale = stiffness * violation / denominator;
    const float pg[3] = {gux, guy, guz};
    const float cg[3] = {cgx, cgy, cgz};
    const float ng[3] = {gvx, gvy, gvz};
    for (int axis = 0; axis < 3; ++axis) {
        size_t pc = 3 * (size_t)previous + axis, cc = 3 * (size_t)center + axis, nc = 3 * (size_t)next + axis;
        float moved_previous = P[pc] - previous_weight * scale * pg[axis];
        float moved_center = P[cc] + center_weight * scale * cg[axis];
        float moved_next = P[nc] + next_weight * scale * ng[axis];
        float previous_value = moved_previous, center_value = moved_center, next_value = moved_next;
        if (!w.grid.periodic[axis]) {
            float lo = w.grid.lower[axis], hi = w.grid.upper[axis];
            previous_value = clampf(moved_previous, lo + w.wall_extents[pc], hi - w.wall_extents[pc]);
            center_value = clampf(moved_center, lo + w.wall_extents[cc], hi - w.wall_extents[cc]);
            next_value = clampf(moved_next, lo + w.wall_extents[nc], hi - w.wall_extents[nc]);
            if (previous_weight > 0.0f) w.wall_reactions[pc] += moved_previous - previous_value;
            if (center_weight > 0.0f) w.wall_reactions[cc] += moved_center - center_value;
            if (next_weight > 0.0f) w.wall_reactions[nc] += moved_next - next_value;
        }
        if (previous_weight > 0.0f) P[pc] = previous_value;
        if (center_weight > 0.0f) P[cc] = center_value;
        if (next_weight > 0.0f) P[nc] = next_value;
    }
}

/* kernels.rs:1324-1415: forward then backward Gauss-Seidel per fiber. */
void project_fiber_curvature(orc_world &w, uint32_t sweeps, float stiffness, float safety_margin) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t fi = 0; fi < (int64_t)w.F; ++fi) {
        uint32_t start = w.fiber_vertex_spans[2 * fi];
        uint32_t count = w.fiber_vertex_spans[2 * fi + 1];
        if (count < 3 || !w.fiber_on[fi]) continue;
        for (uint32_t sweep = 0; sweep < sweeps; ++sweep) {
            for (uint32_t local = 2; local < count; ++local) {
                uint32_t vertex = start + local;
                project_curvature_triplet(w, vertex - 2, vertex - 1, vertex, stiffness, safety_margin);
            }
            for (uint32_t local = 2; local < count; ++local) {
                uint32_t vertex = start + count - 1 - local;
                project_curvature_triplet(w, vertex, vertex + 1, vertex + 2, stiffness, safety_margin);
            }
        }
    }
}

}  // namespace

extern "C" {

const char *orc_last_error(void) { return g_error.c_str(); }

float orc_acos_f32(float x) { return acos_f32(x); }

void orc_set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

int orc_world_create(const orc_packed *pk, const orc_cell_list_config *cl, float max_step, orc_world **out) {
    if (!pk || !cl || !out) return fail("null argument");
    if (pk->segment_count == 0 || pk->fiber_count == 0) return fail("assembly has no segments or fibers");
    if (!(cl->cell_size_scale >= 1.0f)) return fail("cell_size_scale must be at least 1");
    if (!(std::isfinite(cl->neighbor_skin_scale) && cl->neighbor_skin_scale >= 0.0f))
        return fail("neighbor_skin_scale must be finite and non-negative");
    if (cl->neighbor_capacity == 0) return fail("neighbor_capacity must be positive");
    if (!(max_step > 0.0f)) return fail("max_step must be positive");
    orc_world *w = new orc_world();
    w->V = pk->vertex_count;
    w->S = pk->segment_count;
    w->F = pk->fiber_count;
    w->positions.assign(pk->positions, pk->positions + 3 * (size_t)w->V);
    w->intrinsic.assign(pk->intrinsic_positions, pk->intrinsic_positions + 3 * (size_t)w->V);
    w->segment_vertices.assign(pk->segment_vertices, pk->segment_vertices + 2 * (size_t)w->S);
    w->segment_fibers.assign(pk->segment_fibers, pk->segment_fibers + w->S);
    w->radii.assign(pk->segment_radii, pk->segment_radii + w->S);
    w->rest_lengths.assign(pk->segment_rest_lengths, pk->segment_rest_lengths + w->S);
    w->fiber_vertex_spans.assign(pk->fiber_vertex_spans, pk->fiber_vertex_spans + 2 * (size_t)w->F);
    w->fiber_segment_spans.assign(pk->fiber_segment_spans, pk->fiber_segment_spans + 2 * (size_t)w->F);
    w->vertex_segments.assign(pk->vertex_segments, pk->vertex_segments + 2 * (size_t)w->V);
    w->max_curvature.assign(pk->vertex_max_curvature, pk->vertex_max_curvature + w->V);
    if (pk->vertex_pinned)
        w->pinned.assign(pk->vertex_pinned, pk->vertex_pinned + w->V);
    else
        w->pinned.assign(w->V, 0);
    for (int a = 0; a < 3; ++a) {
        w->grid.lower[a] = pk->cell_lower[a];
        w->grid.upper[a] = pk->cell_upper[a];
        w->grid.periodic[a] = pk->cell_periodic[a] ? 1 : 0;
    }
    for (uint32_t s = 0; s < w->S; ++s) {
        if (w->segment_vertices[2 * s] >= w->V || w->segment_vertices[2 * s + 1] >= w->V || w->segment_fibers[s] >= w->F) {
            delete w;
            return fail("segment refers to a vertex or fiber out of range");
        }
    }
    /* packed.rs:561-580: rest arc length, f64 accumulate of f32 intrinsics. */
    w->arc.assign(w->V, 0.0f);
    w->wall_extents.assign(3 * (size_t)w->V, 0.0f);
    for (uint32_t f = 0; f < w->F; ++f) {
        uint32_t start = w->fiber_vertex_spans[2 * f], count = w->fiber_vertex_spans[2 * f + 1];
        if ((uint64_t)start + count > w->V || count < 2) {
            delete w;
            return fail("fiber vertex span out of range or shorter than two vertices");
        }
        double total = 0.0;
        for (uint32_t v = start + 1; v < start + count; ++v) {
            double sum = 0.0;
            for (int a = 0; a < 3; ++a) {
                double delta = (double)w->intrinsic[3 * (size_t)v + a] - (double)w->intrinsic[3 * (size_t)(v - 1) + a];
                sum += delta * delta;
            }
            total += std::sqrt(sum);
            w->arc[v] = (float)total;
        }
        float radius = w->radii[w->fiber_segment_spans[2 * f]];
        for (uint32_t v = start; v < start + count; ++v)
            for (int a = 0; a < 3; ++a) w->wall_extents[3 * (size_t)v + a] = radius;
    }
    if (size_world(*w, *cl, max_step)) {
        delete w;
        return 1;
    }
    /* packed.rs:289-303: every segment and vertex starts active. */
    w->fiber_on.assign(w->F, 1);
    w->segment_on.assign(w->S, 1);
    w->vertex_on.assign(w->V, 1);
    w->vertex_fiber.assign(w->V, 0);
    for (uint32_t f = 0; f < w->F; ++f)
        for (uint32_t k = 0; k < w->fiber_vertex_spans[2 * f + 1]; ++k) w->vertex_fiber[w->fiber_vertex_spans[2 * f] + k] = f;
    w->slots = w->S;
    w->metrics[0] = std::numeric_limits<float>::infinity();
    w->metrics[1] = 0.0f;
    w->metrics[2] = std::numeric_limits<float>::infinity();
    w->reference_positions = w->positions;
    w->corrections.assign(6 * (size_t)w->S, 0.0f);
    w->segment_max.assign(w->S, 0.0f);
    w->curvature_ratio.assign(w->V, 0.0f);
    w->internal.assign(3 * (size_t)w->V, 0.0f);
    w->vertex_step.assign(w->V, 0.0f);
    w->wall_reactions.assign(3 * (size_t)w->V, 0.0f);
    *out = w;
    return 0;
}

void orc_world_destroy(orc_world *w) { delete w; }

/* world.rs:1020-1505 for the plain flexible path, then read_status
 * (world.rs:2337-2369). */
/* kernels.rs:1539-1646 apply_rigid_contact_corrections: each fiber moves as
 * a whole by its deepest segment's mean end correction (the first segment
 * with the largest squared length wins ties), capped at max_step, clamped
 * on walled axes so that every vertex stays inside. */
void apply_rigid_contact_corrections(orc_world &w, float max_step) {
    const int64_t F = (int64_t)w.fiber_vertex_spans.size() / 2;
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < F; ++f) {
        if (!w.fiber_on[f]) continue;
        const uint32_t s0 = w.fiber_segment_spans[2 * f], m = w.fiber_segment_spans[2 * f + 1];
        const uint32_t v0 = w.fiber_vertex_spans[2 * f], n = w.fiber_vertex_spans[2 * f + 1];
        float tx = 0.0f, ty = 0.0f, tz = 0.0f, deepest_squared = 0.0f;
        for (uint32_t local = 0; local < m; ++local) {
            const size_t seg = s0 + local;
            const float cx = 0.5f * (w.corrections[6 * seg] + w.corrections[6 * seg + 3]);
            const float cy = 0.5f * (w.corrections[6 * seg + 1] + w.corrections[6 * seg + 4]);
            const float cz = 0.5f * (w.corrections[6 * seg + 2] + w.corrections[6 * seg + 5]);
            const float squared = cx * cx + cy * cy + cz * cz;
            if (squared > deepest_squared) {
                deepest_squared = squared;
                tx = cx;
                ty = cy;
                tz = cz;
            }
        }
        const float length = std::sqrt(tx * tx + ty * ty + tz * tz);
        if (length > max_step) {
            const float scale = max_step / length;
            tx *= scale;
            ty *= scale;
            tz *= scale;
        }
        const float rx = tx, ry = ty, rz = tz;
        float lower[3], upper[3];
        for (int a = 0; a < 3; ++a) {
            const size_t c = 3 * (size_t)v0 + a;
            lower[a] = w.grid.lower[a] + w.wall_extents[c] - w.positions[c];
            upper[a] = w.grid.upper[a] - w.wall_extents[c] - w.positions[c];
        }
        for (uint32_t local = 1; local < n; ++local)
            for (int a = 0; a < 3; ++a) {
                const size_t c = 3 * (size_t)(v0 + local) + a;
                lower[a] = std::max(lower[a], w.grid.lower[a] + w.wall_extents[c] - w.positions[c]);
                upper[a] = std::min(upper[a], w.grid.upper[a] - w.wall_extents[c] - w.positions[c]);
            }
        float t[3] = {tx, ty, tz};
        for (int a = 0; a < 3; ++a)
            if (!w.grid.periodic[a]) t[a] = t[a] < lower[a] ? lower[a] : (t[a] > upper[a] ? upper[a] : t[a]);
        const float applied = std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        const float reaction[3] = {(rx - t[0]) / (float)n, (ry - t[1]) / (float)n, (rz - t[2]) / (float)n};
        for (uint32_t local = 0; local < n; ++local) {
            const size_t v = v0 + local;
            for (int a = 0; a < 3; ++a) {
                w.positions[3 * v + a] += t[a];
                w.wall_reactions[3 * v + a] += reaction[a];
            }
            w.vertex_step[v] = applied;
        }
    }
}

/* apply_formation_layer_targets (kernels.rs:538-581): every active fiber
 * whose layer the target range covers moves along the axis by its centre's
 * capped, stiffness-scaled distance to the layer target. */
static void apply_layer_targets(orc_world &w) {
    if (!w.layer_on) return;
    for (uint32_t f = 0; f < w.F; ++f) {
        const uint32_t layer = w.fiber_layers[f];
        if (layer == NONE || layer >= w.layer_targets.size() || layer < w.layer_first || layer > w.layer_last) continue;
        const uint32_t start = w.fiber_vertex_spans[2 * f], count = w.fiber_vertex_spans[2 * f + 1];
        if (count == 0 || !w.vertex_on[start]) continue;
        float center = 0.0f;
        for (uint32_t local = 0; local < count; ++local) center += w.positions[3 * (size_t)(start + local) + w.layer_axis];
        center /= (float)count;
        const float translation = clampf((w.layer_targets[layer] - center) * w.layer_stiffness,
                                         -w.layer_max_translation, w.layer_max_translation);
        for (uint32_t local = 0; local < count; ++local)
            w.positions[3 * (size_t)(start + local) + w.layer_axis] += translation;
    }
}

/* apply_vertex_targets (kernels.rs:604-634). */
static void apply_vertex_targets(orc_world &w) {
    if (!w.targets_on) return;
    for (size_t k = 0; k < w.target_vertices.size(); ++k) {
        const uint32_t vertex = w.target_vertices[k];
        if (!w.vertex_on[vertex]) continue;
        const float command = w.command_coordinates[k];
        const float translation = clampf((w.target_coordinates[k] - command) * w.target_stiffness,
                                         -w.target_max_translation, w.target_max_translation);
        w.command_coordinates[k] = command + translation;
        w.positions[3 * (size_t)vertex + w.target_axis] = command + translation;
    }
}

int orc_run_batch(orc_world *w, const orc_relax_config *config, uint32_t iterations, orc_batch_status *status) {
    if (!w || !config || !status) return fail("null argument");
    if (iterations == 0) return fail("iterations must be positive");
    w->control[2] = 0; /* kernels.rs:3-12 */
    if (w->control[3] == 0) w->control[0] = 1;
    flag_neighbor_list_displacement(*w);
    for (uint32_t step = 0; step <= iterations; ++step) {
        rebuild_neighbor_lists_if_requested(*w);
        if (w->control[0]) {
            find_segment_corrections(*w, config->correction_fraction, config->contact_aggregation);
            measure_curvature_ratio(*w);
            reduce_and_assess(*w, *config, iterations);
        }
        if (w->control[0]) {
            std::fill(w->wall_reactions.begin(), w->wall_reactions.end(), 0.0f);
            if (config->motion_model == 1) {  // world.rs:1369-1404
                apply_rigid_contact_corrections(*w, config->max_step);
            } else {
                for (uint32_t c = 0; c < config->constraint_iterations; ++c)
                    internal_pass(*w, config->stretch_stiffness, config->bend_stiffness);
                apply_contact_corrections(*w, config->max_step);
                project_fiber_curvature(*w, config->curvature_cleanup_sweeps, config->curvature_limit_stiffness,
                                        config->curvature_limit_safety_margin);
            }
            /* world.rs:1420-1447: the manufacturing targets after the mechanics. */
            apply_layer_targets(*w);
            apply_vertex_targets(*w);
        }
        flag_neighbor_list_displacement(*w);
    }
    bool overflow = w->cell_overflow != 0 || w->control[3] != 0;
    status->total_iterations = w->control[1];
    status->batch_iterations = w->control[2];
    status->max_penetration = w->metrics[0];
    status->max_displacement = w->metrics[1];
    status->max_curvature_ratio = w->metrics[2];
    status->converged = (!config->force_full_iterations && w->metrics[0] <= config->penetration_tolerance &&
                         w->metrics[2] <= 1.0f + config->curvature_ratio_tolerance && !overflow)
                            ? 1
                            : 0;
    status->cell_list_overflow = overflow ? 1 : 0;
    status->reserved = 0;
    return 0;
}

int orc_download_positions(const orc_world *w, float *xyz, size_t len) {
    if (!w || !xyz) return fail("null argument");
    if (len != w->positions.size()) return fail("position buffer has the wrong length");
    std::memcpy(xyz, w->positions.data(), len * sizeof(float));
    return 0;
}

int orc_upload_positions(orc_world *w, const float *xyz, size_t len) {
    if (!w || !xyz) return fail("null argument");
    if (len != w->positions.size()) return fail("position buffer has the wrong length");
    std::memcpy(w->positions.data(), xyz, len * sizeof(float));
    return 0;
}

float orc_cell_size(const orc_world *w) { return w->cell_size; }
uint64_t orc_cell_count(const orc_world *w) { return w->cell_counts.size(); }
void orc_cell_dims(const orc_world *w, uint32_t dims[3]) {
    dims[0] = w->grid.cx;
    dims[1] = w->grid.cy;
    dims[2] = w->grid.cz;
}
float orc_neighbor_skin(const orc_world *w) { return w->neighbor_skin; }
uint32_t orc_neighbor_block(const orc_world *w) { return w->neighbor_block; }
uint32_t orc_neighbor_list_rebuilds(const orc_world *w) { return w->neighbor_state[1]; }
uint64_t orc_curvature_projections(const orc_world *w) { return w->projections; }

int orc_debug_cell_list(const orc_world *w, uint32_t *cell_counts, uint32_t *cell_offsets, uint32_t *cell_segments) {
    std::memcpy(cell_counts, w->cell_counts.data(), w->cell_counts.size() * 4);
    std::memcpy(cell_offsets, w->cell_offsets.data(), w->cell_offsets.size() * 4);
    std::memcpy(cell_segments, w->cell_segments.data(), w->cell_segments.size() * 4);
    return 0;
}

int orc_debug_neighbor_lists(const orc_world *w, uint32_t *counts, uint32_t *lists) {
    std::memcpy(counts, w->neighbor_counts.data(), w->neighbor_counts.size() * 4);
    std::memcpy(lists, w->neighbor_segments.data(), w->neighbor_segments.size() * 4);
    return 0;
}

int orc_debug_corrections(orc_world *w, const orc_relax_config *config, float *corrections, float *segment_max) {
    rebuild_neighbor_lists_if_requested(*w);
    find_segment_corrections(*w, config->correction_fraction, config->contact_aggregation);
    std::memcpy(corrections, w->corrections.data(), w->corrections.size() * 4);
    std::memcpy(segment_max, w->segment_max.data(), w->segment_max.size() * 4);
    return 0;
}

int orc_debug_rebuild(orc_world *w) {
    w->neighbor_state[0] = 1;
    rebuild_neighbor_lists_if_requested(*w);
    return 0;
}

/* ---- Formation hooks (world.rs:1723-2194; kernels.rs:164-221, 538-923). */

/* activate_formation_step (world.rs:2139-2183) with the step comparison done
 * by the caller: the masks follow the fiber flags, and the lists are
 * rebuilt before the next contact pass. */
int orc_set_active_fibers(orc_world *w, const uint8_t *active, uint64_t fiber_count, uint32_t *active_segments,
                          uint32_t *active_vertices) {
    if (!w || !active || !active_segments || !active_vertices) return fail("null argument");
    if (fiber_count != w->F) return fail("active flags need one entry per fiber");
    for (uint32_t f = 0; f < w->F; ++f) w->fiber_on[f] = active[f] ? 1 : 0;
    uint32_t segments = 0, vertices = 0;
    for (uint32_t s = 0; s < w->S; ++s) segments += (w->segment_on[s] = w->fiber_on[w->segment_fibers[s]]);
    for (uint32_t v = 0; v < w->V; ++v) vertices += (w->vertex_on[v] = w->fiber_on[w->vertex_fiber[v]]);
    w->neighbor_state[0] = 1;
    *active_segments = segments;
    *active_vertices = vertices;
    return 0;
}

/* apply_layer_target_range (world.rs:1758-1804), clear_layer_targets
 * (:1806-1810) when targets is NULL. */
int orc_set_layer_targets(orc_world *w, uint32_t axis, const float *targets, uint32_t count,
                          const uint32_t *fiber_layers, uint32_t first_layer, uint32_t last_layer, float stiffness,
                          float max_translation, int apply_now) {
    if (!w) return fail("null argument");
    if (!targets) {
        w->layer_on = false;
        return 0;
    }
    if (axis >= 3 || count == 0 || !fiber_layers) return fail("bad layer target");
    if (!(stiffness > 0.0f && stiffness <= 1.0f) || !(max_translation > 0.0f)) return fail("bad layer target gains");
    w->layer_on = true;
    w->layer_axis = axis;
    w->layer_targets.assign(targets, targets + count);
    w->fiber_layers.assign(fiber_layers, fiber_layers + w->F);
    w->layer_first = first_layer;
    w->layer_last = last_layer;
    w->layer_stiffness = stiffness;
    w->layer_max_translation = max_translation;
    if (apply_now) apply_layer_targets(*w); /* the immediate launch ignores the gate */
    return 0;
}

/* apply_vertex_displacement_targets (world.rs:1811-1859) with
 * initialize_vertex_displacement_targets (kernels.rs:583-602);
 * clear_vertex_targets (:1861-1863) when vertices is NULL. */
int orc_set_vertex_targets(orc_world *w, uint32_t axis, const uint32_t *vertices, uint32_t count, float displacement,
                           float stiffness, float max_translation) {
    if (!w) return fail("null argument");
    if (!vertices) {
        w->targets_on = false;
        w->target_vertices.clear();
        return 0;
    }
    if (axis >= 3 || count == 0) return fail("bad vertex target");
    if (!(std::isfinite(displacement) && displacement != 0.0f)) return fail("displacement must be finite and non-zero");
    if (!(stiffness > 0.0f && stiffness <= 1.0f) || !(max_translation > 0.0f)) return fail("bad vertex target gains");
    for (uint32_t k = 0; k < count; ++k)
        if (vertices[k] >= w->V) return fail("vertex target index out of range");
    w->targets_on = true;
    w->target_axis = axis;
    w->target_stiffness = stiffness;
    w->target_max_translation = max_translation;
    w->target_vertices.assign(vertices, vertices + count);
    w->target_coordinates.resize(count);
    w->command_coordinates.resize(count);
    for (uint32_t k = 0; k < count; ++k) {
        const float coordinate = w->positions[3 * (size_t)vertices[k] + axis];
        w->target_coordinates[k] = coordinate + displacement;
        w->command_coordinates[k] = coordinate;
    }
    return 0;
}

int orc_vertex_target_state(const orc_world *w, float *coordinates, float *command_coordinates, uint32_t count) {
    if (!w || !coordinates || !command_coordinates) return fail("null argument");
    if (!w->targets_on || count != w->target_vertices.size()) return fail("count differs from the installed targets");
    std::memcpy(coordinates, w->target_coordinates.data(), count * sizeof(float));
    std::memcpy(command_coordinates, w->command_coordinates.data(), count * sizeof(float));
    return 0;
}

/* measure_layer_target_error / measure_vertex_target_error (kernels.rs:
 * 636-711): serial maxima from zero. */
int orc_target_errors(const orc_world *w, float *layer_error, uint32_t *has_layer, float *vertex_error,
                      uint32_t *has_vertex) {
    if (!w || !layer_error || !has_layer || !vertex_error || !has_vertex) return fail("null argument");
    *has_layer = w->layer_on ? 1 : 0;
    *has_vertex = w->targets_on ? 1 : 0;
    float maximum = 0.0f;
    if (w->layer_on)
        for (uint32_t f = 0; f < w->F; ++f) {
            const uint32_t layer = w->fiber_layers[f];
            if (layer == NONE || layer >= w->layer_targets.size() || layer < w->layer_first || layer > w->layer_last)
                continue;
            const uint32_t start = w->fiber_vertex_spans[2 * f], count = w->fiber_vertex_spans[2 * f + 1];
            if (count == 0 || !w->vertex_on[start]) continue;
            float center = 0.0f;
            for (uint32_t local = 0; local < count; ++local)
                center += w->positions[3 * (size_t)(start + local) + w->layer_axis];
            center /= (float)count;
            const float error = std::fabs(w->layer_targets[layer] - center);
            if (error > maximum) maximum = error;
        }
    *layer_error = maximum;
    maximum = 0.0f;
    if (w->targets_on)
        for (size_t k = 0; k < w->target_vertices.size(); ++k) {
            const uint32_t vertex = w->target_vertices[k];
            if (!w->vertex_on[vertex]) continue;
            const float error = std::fabs(w->target_coordinates[k] - w->positions[3 * (size_t)vertex + w->target_axis]);
            if (error > maximum) maximum = error;
        }
    *vertex_error = maximum;
    return 0;
}

/* compact_cell (world.rs:1931-2054) with compact_rigid_fiber_centers,
 * compact_moving_walls and compact_affine_vertices (kernels.rs:712-818):
 * kinematics 0, 1, 2. */
int orc_compact_cell(orc_world *w, const float new_lower[3], const float new_upper[3], uint32_t kinematics) {
    if (!w || !new_lower || !new_upper) return fail("null argument");
    if (kinematics > 2) return fail("kinematics must be 0, 1 or 2");
    uint32_t cells[3];
    for (int a = 0; a < 3; ++a) {
        if (!std::isfinite(new_lower[a]) || !std::isfinite(new_upper[a])) return fail("bounds must be finite");
        if (!(new_upper[a] - new_lower[a] > 2.0f * w->maximum_radius)) return fail("cell narrower than two radii");
        if (!(new_lower[a] >= w->grid.lower[a]) || !(new_upper[a] <= w->grid.upper[a]))
            return fail("compaction cannot grow the cell");
        cells[a] = f32_to_u32(std::fmax(std::floor((new_upper[a] - new_lower[a]) / w->cell_size), 1.0f));
    }
    const uint64_t C = checked_cell_count(cells, w->allocated_cells);
    if (C == 0) return fail("the compacted grid needs more cells than allocated");
    const float *ol = w->grid.lower, *ou = w->grid.upper;
    if (kinematics == 0) {
        for (uint32_t f = 0; f < w->F; ++f) {
            const uint32_t start = w->fiber_vertex_spans[2 * f], count = w->fiber_vertex_spans[2 * f + 1];
            if (count == 0 || !w->vertex_on[start]) continue;
            float c[3] = {0.0f, 0.0f, 0.0f};
            for (uint32_t local = 0; local < count; ++local)
                for (int a = 0; a < 3; ++a) c[a] += w->positions[3 * (size_t)(start + local) + a];
            float d[3];
            for (int a = 0; a < 3; ++a) {
                c[a] /= (float)count;
                const float fraction = (c[a] - ol[a]) / (ou[a] - ol[a]);
                d[a] = new_lower[a] + fraction * (new_upper[a] - new_lower[a]) - c[a];
            }
            for (uint32_t local = 0; local < count; ++local)
                for (int a = 0; a < 3; ++a) {
                    w->positions[3 * (size_t)(start + local) + a] += d[a];
                    w->wall_reactions[3 * (size_t)(start + local) + a] = 0.0f;
                }
        }
    } else {
        for (uint32_t v = 0; v < w->V; ++v) {
            if (!w->vertex_on[v]) continue;
            for (int a = 0; a < 3; ++a) {
                const size_t c = 3 * (size_t)v + a;
                if (kinematics == 2) {
                    const float fraction = (w->positions[c] - ol[a]) / (ou[a] - ol[a]);
                    w->positions[c] = new_lower[a] + fraction * (new_upper[a] - new_lower[a]);
                    w->wall_reactions[c] = 0.0f;
                } else if (!w->grid.periodic[a]) {
                    const float previous = w->positions[c];
                    const float projected =
                        clampf(previous, new_lower[a] + w->wall_extents[c], new_upper[a] - w->wall_extents[c]);
                    w->positions[c] = projected;
                    w->wall_reactions[c] = previous - projected;
                } else {
                    w->wall_reactions[c] = 0.0f;
                }
            }
        }
    }
    for (int a = 0; a < 3; ++a) {
        w->grid.lower[a] = new_lower[a];
        w->grid.upper[a] = new_upper[a];
    }
    w->grid.cx = cells[0];
    w->grid.cy = cells[1];
    w->grid.cz = cells[2];
    w->cell_counts.assign(C, 0);
    w->cell_offsets.assign(C, 0);
    w->neighbor_state[0] = 1;
    return 0;
}

int orc_cell_bounds(const orc_world *w, float lower[3], float upper[3]) {
    if (!w || !lower || !upper) return fail("null argument");
    for (int a = 0; a < 3; ++a) {
        lower[a] = w->grid.lower[a];
        upper[a] = w->grid.upper[a];
    }
    return 0;
}

/* measure_compaction_metrics (kernels.rs:820-923), serial f32 as the
 * reference sums; curvature ratios from the last gate's measurement. */
int orc_compaction_metrics(const orc_world *w, float correction_fraction, const float stiffness[3], float out[13]) {
    if (!w || !stiffness || !out) return fail("null argument");
    if (!(correction_fraction > 0.0f)) return fail("correction_fraction must be positive");
    const float contact_stiffness = stiffness[0], stretch_stiffness = stiffness[1], bending_stiffness = stiffness[2];
    float load_x = 0.0f, load_y = 0.0f, load_z = 0.0f, contact_energy = 0.0f, stretch_energy = 0.0f;
    for (uint32_t segment = 0; segment < w->S; ++segment) {
        if (!w->segment_on[segment]) continue;
        const float *c = &w->corrections[6 * (size_t)segment];
        load_x += std::fabs(c[0]) + std::fabs(c[3]);
        load_y += std::fabs(c[1]) + std::fabs(c[4]);
        load_z += std::fabs(c[2]) + std::fabs(c[5]);
        const float penetration = w->segment_max[segment];
        contact_energy += 0.5f * contact_stiffness * penetration * penetration;
        const uint32_t first = w->segment_vertices[2 * segment], second = w->segment_vertices[2 * segment + 1];
        const float dx = w->positions[3 * second] - w->positions[3 * first];
        const float dy = w->positions[3 * second + 1] - w->positions[3 * first + 1];
        const float dz = w->positions[3 * second + 2] - w->positions[3 * first + 2];
        const float length = std::sqrt(dx * dx + dy * dy + dz * dz);
        const float rest = w->rest_lengths[segment];
        if (rest > 1.0e-7f) {
            const float extension = length - rest;
            stretch_energy += 0.5f * stretch_stiffness * extension * extension / rest;
        }
    }
    float bending_energy = 0.0f;
    for (uint32_t v = 0; v < w->V; ++v) {
        const float excess = std::fmax(w->curvature_ratio[v] - 1.0f, 0.0f);
        bending_energy += 0.5f * bending_stiffness * excess * excess;
    }
    const float lx = w->grid.upper[0] - w->grid.lower[0], ly = w->grid.upper[1] - w->grid.lower[1],
                lz = w->grid.upper[2] - w->grid.lower[2];
    float face[6] = {0, 0, 0, 0, 0, 0};
    for (uint32_t v = 0; v < w->V; ++v)
        for (int a = 0; a < 3; ++a) {
            const float r = w->wall_reactions[3 * (size_t)v + a];
            face[2 * a] += std::fmax(-r, 0.0f);
            face[2 * a + 1] += std::fmax(r, 0.0f);
        }
    const float inverse_projection = 1.0f / std::fmax(correction_fraction, 1.0e-7f);
    const float px = w->grid.periodic[0] ? load_x : face[0] + face[1];
    const float py = w->grid.periodic[1] ? load_y : face[2] + face[3];
    const float pz = w->grid.periodic[2] ? load_z : face[4] + face[5];
    out[0] = contact_stiffness * px * inverse_projection / (ly * lz);
    out[1] = contact_stiffness * py * inverse_projection / (lx * lz);
    out[2] = contact_stiffness * pz * inverse_projection / (lx * ly);
    out[3] = contact_energy;
    out[4] = stretch_energy;
    out[5] = bending_energy;
    out[6] = contact_energy + stretch_energy + bending_energy;
    out[7] = contact_stiffness * face[0] * inverse_projection / (ly * lz);
    out[8] = contact_stiffness * face[1] * inverse_projection / (ly * lz);
    out[9] = contact_stiffness * face[2] * inverse_projection / (lx * lz);
    out[10] = contact_stiffness * face[3] * inverse_projection / (lx * lz);
    out[11] = contact_stiffness * face[4] * inverse_projection / (lx * ly);
    out[12] = contact_stiffness * face[5] * inverse_projection / (lx * ly);
    return 0;
}

int orc_wall_reactions(const orc_world *w, float *xyz, size_t len) {
    if (!w || !xyz) return fail("null argument");
    if (len != w->wall_reactions.size()) return fail("reaction buffer has the wrong length");
    std::memcpy(xyz, w->wall_reactions.data(), len * sizeof(float));
    return 0;
}

/* set_fiber_maximum_curvatures (world.rs:2185-2194). */
int orc_set_fiber_max_curvatures(orc_world *w, const float *values, size_t count) {
    if (!w || !values) return fail("null argument");
    if (count != w->F) return fail("one curvature limit per fiber");
    for (uint32_t v = 0; v < w->V; ++v) w->max_curvature[v] = values[w->vertex_fiber[v]];
    return 0;
}

}  // extern "C"
