// common.cuh -- device data layout and the f32 geometry shared by the
// relaxation kernels.
//
// Every expression is written in the reference's operand order and the
// library is compiled with -fmad=false (no FMA contraction), IEEE division
// and square root, so each value rounds exactly as in the reference's
// CubeCL source (crates/tangle_contact/src/device/*.rs,
// crates/tangle_relax/src/device/kernels.rs) evaluated left to right.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define TGL_NONE 0xFFFFFFFFu

namespace tgl {

// Orthorhombic cell and its uniform grid. `length` is upper - lower and
// `width` is length / cells, both rounded in f32 exactly as proxy_cell
// computes them (cell_list.rs:60-62).
struct Grid {
    float lower[3];
    float upper[3];
    float length[3];
    float width[3];
    float inv_length[3];  // 1 / length in f32, for image_round's fast path
    uint32_t periodic[3];
    uint32_t cells[3];
};

// Rust `f32 as i32`: saturating, NaN -> 0.
__host__ __device__ inline int32_t f32_to_i32(float x) {
    if (x != x) return 0;
    if (x >= 2147483648.0f) return 2147483647;
    if (x < -2147483648.0f) return (-2147483647 - 1);
    return (int32_t)x;
}

// Rust f32::clamp.
__host__ __device__ inline float clampf(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

// f32 arc cosine with one fixed rounding sequence, so that every build of
// the relaxation (these kernels and the CPU oracle) rounds it identically.
// The reference calls the backend's acos (kernels.rs:1211), whose last bits
// differ between libm and GPU runtimes. Method: the usual reduction to asin
// on [0, 1/2] -- acos x = pi/2 - asin x for |x| <= 1/2, and
// acos x = 2 asin(sqrt((1 - x)/2)) (or pi minus that for x < 0) otherwise --
// with asin s = s + s z P(z), z = s^2 <= 1/4, where P is a degree-5
// polynomial least-squares fitted in f64 to (asin(sqrt z) - sqrt z)/(z sqrt z)
// on Chebyshev nodes of [0, 1/4]. Maximum error 1.01 ulp against f64 acos
// over 440k samples of [-1, 1].
__host__ __device__ inline float acos_f32(float x) {
    const float pio2_hi = 1.57079637050628662109375f;
    const float pio2_lo = -4.371138828673793e-08f;
    float ax = fabsf(x);
    if (ax <= 0.5f) {
        float z = x * x;
        float p = ((((0.03381037712097168f * z + 0.01707467809319496f) * z + 0.031116951256990433f) * z +
                    0.04459794610738754f) * z + 0.07500099390745163f) * z + 0.1666666567325592f;
        float r = x + x * z * p;
        return pio2_hi - (r - pio2_lo);
    }
    float z = 0.5f * (1.0f - ax);
    float s = sqrtf(z);
    float p = ((((0.03381037712097168f * z + 0.01707467809319496f) * z + 0.031116951256990433f) * z +
                0.04459794610738754f) * z + 0.07500099390745163f) * z + 0.1666666567325592f;
    float r = s + s * z * p;
    if (x > 0.0f) return 2.0f * r;
    return 2.0f * (pio2_hi - (r - pio2_lo));
}

// proxy_cell (cell_list.rs:34-79) for a one-piece segment: the cell of its midpoint.
__device__ inline uint32_t proxy_cell(float px, float py, float pz, float qx, float qy, float qz,
                                      const Grid &g) {
    float mx = 0.5f * (px + qx);
    float my = 0.5f * (py + qy);
    float mz = 0.5f * (pz + qz);
    int32_t rx = f32_to_i32(floorf((mx - g.lower[0]) / g.width[0]));
    int32_t ry = f32_to_i32(floorf((my - g.lower[1]) / g.width[1]));
    int32_t rz = f32_to_i32(floorf((mz - g.lower[2]) / g.width[2]));
    int32_t cx = (int32_t)g.cells[0], cy = (int32_t)g.cells[1], cz = (int32_t)g.cells[2];
    uint32_t x = (uint32_t)min(max(rx, 0), cx - 1);
    uint32_t y = (uint32_t)min(max(ry, 0), cy - 1);
    uint32_t z = (uint32_t)min(max(rz, 0), cz - 1);
    if (g.periodic[0]) x = (uint32_t)((rx % cx + cx) % cx);
    if (g.periodic[1]) y = (uint32_t)((ry % cy + cy) % cy);
    if (g.periodic[2]) z = (uint32_t)((rz % cz + cz) % cz);
    return (z * g.cells[1] + y) * g.cells[0] + x;
}

// The 27-cell stencil with periodic uniqueness (neighbor.rs:242-274,
// contact.rs:390-427): the neighbor cell, or TGL_NONE when it is outside a
// wall or repeats another stencil entry of a 1- or 2-cell periodic axis.
__device__ inline uint32_t stencil_cell(uint32_t home, uint32_t neighbor, const Grid &g) {
    uint32_t hx = home % g.cells[0];
    uint32_t hy = (home / g.cells[0]) % g.cells[1];
    uint32_t hz = home / (g.cells[0] * g.cells[1]);
    int32_t ox = (int32_t)(neighbor % 3) - 1;
    int32_t oy = (int32_t)((neighbor / 3) % 3) - 1;
    int32_t oz = (int32_t)(neighbor / 9) - 1;
    int32_t rx = (int32_t)hx + ox, ry = (int32_t)hy + oy, rz = (int32_t)hz + oz;
    int32_t cx = (int32_t)g.cells[0], cy = (int32_t)g.cells[1], cz = (int32_t)g.cells[2];
    bool valid = (g.periodic[0] || (rx >= 0 && rx < cx)) && (g.periodic[1] || (ry >= 0 && ry < cy)) &&
                 (g.periodic[2] || (rz >= 0 && rz < cz));
    bool unique_x = !g.periodic[0] ||
                    !((cx == 1 && ox != 0) || (cx == 2 && ((hx == 0 && ox > 0) || (hx == 1 && ox < 0))));
    bool unique_y = !g.periodic[1] ||
                    !((cy == 1 && oy != 0) || (cy == 2 && ((hy == 0 && oy > 0) || (hy == 1 && oy < 0))));
    bool unique_z = !g.periodic[2] ||
                    !((cz == 1 && oz != 0) || (cz == 2 && ((hz == 0 && oz > 0) || (hz == 1 && oz < 0))));
    if (!(valid && unique_x && unique_y && unique_z)) return TGL_NONE;
    uint32_t nx = (uint32_t)((rx % cx + cx) % cx);
    uint32_t ny = (uint32_t)((ry % cy + cy) % cy);
    uint32_t nz = (uint32_t)((rz % cz + cz) % cz);
    return (nz * g.cells[1] + ny) * g.cells[0] + nx;
}

// roundf(x / length[a]) -- the image count of a periodic axis -- without the
// IEEE division in all but a vanishing set of cases. With q = x * (1/length)
// rounded twice in f32, |q - x/length| <= |q| 2^-22 and the correctly
// rounded quotient is within |q| 2^-24 of x/length; for |q| < 4096 both lie
// within 7.4e-4 of q. Rounding to the nearest integer only changes at
// half-integers, so when q is more than 1e-3 from one, roundf(q) is exactly
// roundf(x / length) (same integer, same sign of zero). Otherwise the
// division is done.
__device__ inline float image_round(float x, int a, const Grid &g) {
    float q = x * g.inv_length[a];
    float aq = fabsf(q);
    if (aq < 0.499f) return copysignf(0.0f, q);  // the common case: same cell image
    float fraction = aq - floorf(aq);
    if (aq < 4096.0f && fabsf(fraction - 0.5f) > 1.0e-3f) return roundf(q);
    return roundf(x / g.length[a]);
}

// Minimum-image shift of the second segment against the first, per periodic
// axis (neighbor.rs:301-318, contact.rs:456-473). Returns true when some axis
// shifted by a nonzero number of box lengths.
__device__ inline bool minimum_image(float p1x, float p1y, float p1z, float q1x, float q1y, float q1z,
                                     float &p2x, float &p2y, float &p2z, float &q2x, float &q2y, float &q2z,
                                     const Grid &g) {
    float image_dx = 0.5f * (p2x + q2x - p1x - q1x);
    float image_dy = 0.5f * (p2y + q2y - p1y - q1y);
    float image_dz = 0.5f * (p2z + q2z - p1z - q1z);
    bool moved = false;
    if (g.periodic[0]) {
        float images = image_round(image_dx, 0, g);
        float shift = images * g.length[0];
        p2x -= shift;
        q2x -= shift;
        moved |= images != 0.0f;
    }
    if (g.periodic[1]) {
        float images = image_round(image_dy, 1, g);
        float shift = images * g.length[1];
        p2y -= shift;
        q2y -= shift;
        moved |= images != 0.0f;
    }
    if (g.periodic[2]) {
        float images = image_round(image_dz, 2, g);
        float shift = images * g.length[2];
        p2z -= shift;
        q2z -= shift;
        moved |= images != 0.0f;
    }
    return moved;
}

// neighbor.rs:27-86 with one proxy piece per segment (the canonical-pair
// test always passes): distance between the two segment axes.
__device__ inline float axis_distance(float p1x, float p1y, float p1z, float d1x, float d1y, float d1z,
                                      float p2x, float p2y, float p2z, float d2x, float d2y, float d2z) {
    const float length_epsilon = 1.0e-20f;
    const float parallel_relative_epsilon = 1.0e-6f;
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
            if (fabsf(denominator) > parallel_relative_epsilon * a * e)
                s = clampf((b * f - c * e) / denominator, 0.0f, 1.0f);
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
    float dx = (p2x + d2x * t) - (p1x + d1x * s);
    float dy = (p2y + d2y * t) - (p1y + d1y * s);
    float dz = (p2z + d2z * t) - (p1z + d1z * s);
    return sqrtf(dx * dx + dy * dy + dz * dz);
}

// Device-side state shared by the kernels of one world.
struct Control {
    // crates/tangle_relax/src/device/world.rs:466-468: active, lifetime
    // iterations, batch iterations, terminal failure.
    uint32_t control[4];
    // metrics (world.rs:470): max penetration, max step, max curvature ratio.
    float metrics[3];
    // neighbor_state (neighbor.rs:1-9): rebuild pending, rebuilds done.
    uint32_t neighbor_state[2];
    // Running maxima (as u32 bits of non-negative floats) for the next gate:
    // penetration, vertex step, curvature ratio.
    uint32_t acc[3];
    // Blocks of the contact kernel finished this pass (last-block gate and
    // the reset of next_batch).
    uint32_t done_blocks;
    // Next 32-slot batch a warp of the running contact pass takes; the last
    // block to finish puts it back to 0.
    uint32_t next_batch;
    uint32_t cell_overflow;
    // Contact lists: refresh pending, refreshes done.
    uint32_t contact_state[2];
    // Rebuild pipelines a batch graph's conditional node has run.
    uint32_t rebuild_bodies;
    // Steps a looped batch graph has begun (its WHILE node's counter).
    uint32_t loop_step;
    // The update's fiber order: launches of the ranking kernel, the order
    // the last update ran in (0 creation, 1 ranked), the one chosen for the
    // cycle's last epochs, update time and launches per order this cycle, and
    // the last update's start and end (%globaltimer ns).
    uint32_t order_tick;
    uint32_t order_mode;
    uint32_t order_best;
    uint32_t order_runs[2];
    unsigned long long order_ns[2];
    unsigned long long order_begin;
    unsigned long long order_end;
};

}  // namespace tgl
