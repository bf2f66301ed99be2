// contact.cuh -- the per-pair arithmetic of find_segment_corrections
// (crates/tangle_contact/src/device/contact.rs:450-870) for round lanes at
// zero offset, shared by the contact kernels.
#pragma once

#include "common.cuh"

namespace tgl {

struct PairTerms {
    float pen, t0x, t0y, t0z, t1x, t1y, t1z, aggw;
};

// Home segment of a candidate pair, as the contact pass reads it.
struct Home {
    float p1x, p1y, p1z, q1x, q1y, q1z, d1x, d1y, d1z, radius, half_length;
    uint32_t segment;
};

__device__ inline Home make_home(float4 a, float4 b, uint32_t segment) {
    Home h;
    h.p1x = a.x;
    h.p1y = a.y;
    h.p1z = a.z;
    h.radius = a.w;
    h.q1x = b.x;
    h.q1y = b.y;
    h.q1z = b.z;
    h.half_length = b.w;  // 0.5 |q1 - p1|
    h.d1x = h.q1x - h.p1x;
    h.d1y = h.q1y - h.p1y;
    h.d1z = h.q1z - h.p1z;
    h.segment = segment;
    return h;
}

// The midpoint reject of find_segment_corrections (contact.rs:456-493):
// shifts the candidate to its minimum image and returns whether the
// capsules can touch.
__device__ inline bool contact_reach(const Home &h, float4 oa, float4 ob, const Grid &g, float &p2x, float &p2y,
                                     float &p2z, float &q2x, float &q2y, float &q2z) {
    p2x = oa.x, p2y = oa.y, p2z = oa.z, q2x = ob.x, q2y = ob.y, q2z = ob.z;
    bool moved = minimum_image(h.p1x, h.p1y, h.p1z, h.q1x, h.q1y, h.q1z, p2x, p2y, p2z, q2x, q2y, q2z, g);
    float d2x = q2x - p2x, d2y = q2y - p2y, d2z = q2z - p2z;
    float mdx = 0.5f * (p2x + q2x - h.p1x - h.q1x);
    float mdy = 0.5f * (p2y + q2y - h.p1y - h.q1y);
    float mdz = 0.5f * (p2z + q2z - h.p1z - h.q1z);
    // Without a periodic shift d2 equals the unshifted q2 - p2, whose half
    // length the geometry record carries; after a shift it is recomputed.
    float other_half = moved ? 0.5f * sqrtf(d2x * d2x + d2y * d2y + d2z * d2z) : ob.w;
    float reach = (h.half_length + other_half + h.radius + oa.w) * (1.0f + 1.0e-4f);
    return mdx * mdx + mdy * mdy + mdz * mdz <= reach * reach;
}

// contact_reach and, in `wide`, the same test with `extra` added to the
// reach (the sum is formed as contact_reach forms it, then `extra` added, so
// a pair that passes the exact test always passes the wide one).
__device__ inline bool contact_reach_wide(const Home &h, float4 oa, float4 ob, const Grid &g, float extra,
                                          float &p2x, float &p2y, float &p2z, float &q2x, float &q2y, float &q2z,
                                          bool &exact) {
    p2x = oa.x, p2y = oa.y, p2z = oa.z, q2x = ob.x, q2y = ob.y, q2z = ob.z;
    bool moved = minimum_image(h.p1x, h.p1y, h.p1z, h.q1x, h.q1y, h.q1z, p2x, p2y, p2z, q2x, q2y, q2z, g);
    float d2x = q2x - p2x, d2y = q2y - p2y, d2z = q2z - p2z;
    float mdx = 0.5f * (p2x + q2x - h.p1x - h.q1x);
    float mdy = 0.5f * (p2y + q2y - h.p1y - h.q1y);
    float mdz = 0.5f * (p2z + q2z - h.p1z - h.q1z);
    float other_half = moved ? 0.5f * sqrtf(d2x * d2x + d2y * d2y + d2z * d2z) : ob.w;
    float base = h.half_length + other_half + h.radius + oa.w;
    float reach = base * (1.0f + 1.0e-4f);
    float wide = (base + extra) * (1.0f + 1.0e-4f);
    float m2 = mdx * mdx + mdy * mdy + mdz * mdz;
    exact = m2 <= reach * reach;
    return m2 <= wide * wide;
}

// Whether two segments (the second already at its minimum image) may come
// within `extra` of touching: their f32 closest-point distance against
// r1 + r2 + extra with margins for its rounding. The closest-point solve
// returns a distance between two points of the segments, so it can only
// overestimate the true distance, by rounding, or, for axes within 1e-3 rad
// of parallel (where it takes an end point without solving), by at most
// 1e-3 of a segment length; the margins (1 % relative, 2e-3 of the summed
// half lengths, and `eps`) cover both.
__device__ inline bool within_contact_skin(const Home &h, float p2x, float p2y, float p2z, float q2x, float q2y,
                                           float q2z, float other_radius, float extra, float eps) {
    const float d2x = q2x - p2x, d2y = q2y - p2y, d2z = q2z - p2z;
    const float distance = axis_distance(h.p1x, h.p1y, h.p1z, h.d1x, h.d1y, h.d1z, p2x, p2y, p2z, d2x, d2y, d2z);
    const float other_half = 0.5f * sqrtf(d2x * d2x + d2y * d2y + d2z * d2z);
    const float threshold =
        (h.radius + other_radius + extra) * 1.01f + 2.0e-3f * (h.half_length + other_half) + eps;
    return distance <= threshold;
}

// A lower bound test on the capsules' overlap: the segments lie on their
// axis lines, so their distance is at least the lines' distance
// |(p2 - p1) . (d1 x d2)| / |d1 x d2|. When that exceeds r1 + r2 by a margin
// (1e-3 relative plus `eps`, above every f32 rounding in this bound and in
// the closest-point solve), the solve's penetration is certainly negative.
// Axes closer to parallel than 0.01 rad (where d1 x d2 loses relative
// accuracy) give no bound.
__device__ inline bool lines_may_touch(const Home &h, float p2x, float p2y, float p2z, float q2x, float q2y,
                                       float q2z, float other_radius, float eps) {
    const float d2x = q2x - p2x, d2y = q2y - p2y, d2z = q2z - p2z;
    const float nx = h.d1y * d2z - h.d1z * d2y;
    const float ny = h.d1z * d2x - h.d1x * d2z;
    const float nz = h.d1x * d2y - h.d1y * d2x;
    const float nn = nx * nx + ny * ny + nz * nz;
    const float aa = h.d1x * h.d1x + h.d1y * h.d1y + h.d1z * h.d1z;
    const float ee = d2x * d2x + d2y * d2y + d2z * d2z;
    if (!(nn > 1.0e-4f * aa * ee)) return true;
    const float rn = (p2x - h.p1x) * nx + (p2y - h.p1y) * ny + (p2z - h.p1z) * nz;
    const float threshold = (h.radius + other_radius) * 1.001f + eps;
    return rn * rn <= threshold * threshold * nn;
}

// One candidate of find_segment_corrections past the midpoint reject
// (contact.rs:663-870) for a round lane at zero offset: returns true with
// the pair's terms when the capsules overlap.
__device__ inline bool contact_solve(const Home &h, uint32_t other, float other_radius, float p2x, float p2y,
                                     float p2z, float q2x, float q2y, float q2z, float correction_fraction,
                                     uint32_t aggregation, PairTerms &out) {
    const float length_epsilon = 1.0e-20f;
    const float parallel_relative_epsilon = 1.0e-6f;
    const float p1x = h.p1x, p1y = h.p1y, p1z = h.p1z, d1x = h.d1x, d1y = h.d1y, d1z = h.d1z;
    const float radius = h.radius;
    float d2x = q2x - p2x, d2y = q2y - p2y, d2z = q2z - p2z;
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
            bool parallel = fabsf(denominator) <= parallel_relative_epsilon * a * e;
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
            if (parallel) {  // contact.rs:695-726
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
                float gx = rx + d1x * s - d2x * t, gy = ry + d1y * s - d2y * t, gz = rz + d1z * s - d2z * t;
                float ex = rx + d1x * end_s - d2x * end_t, ey = ry + d1y * end_s - d2y * end_t,
                      ez = rz + d1z * end_s - d2z * end_t;
                if (ex * ex + ey * ey + ez * ez < gx * gx + gy * gy + gz * gz) {
                    s = end_s;
                    t = end_t;
                }
            }
        }
    }
    float point1x = p1x + d1x * s, point1y = p1y + d1y * s, point1z = p1z + d1z * s;
    float point2x = p2x + d2x * t, point2y = p2y + d2y * t, point2z = p2z + d2z * t;
    float delta_x = point2x - point1x, delta_y = point2y - point1y, delta_z = point2z - point1z;
    float distance = sqrtf(delta_x * delta_x + delta_y * delta_y + delta_z * delta_z);
    float penetration = radius + other_radius - distance;
    if (!(penetration > 0.0f)) return false;
    float nx, ny, nz;
    if (distance > 1.0e-7f) {
        float inverse_distance = 1.0f / distance;
        nx = delta_x * inverse_distance;
        ny = delta_y * inverse_distance;
        nz = delta_z * inverse_distance;
    } else {  // contact.rs:768-812
        nx = d1y * d2z - d1z * d2y;
        ny = d1z * d2x - d1x * d2z;
        nz = d1x * d2y - d1y * d2x;
        float normal_length = sqrtf(nx * nx + ny * ny + nz * nz);
        if (normal_length <= 1.0e-7f) {
            if (fabsf(d1x) <= fabsf(d1y) && fabsf(d1x) <= fabsf(d1z)) {
                nx = 0.0f;
                ny = d1z;
                nz = -d1y;
            } else if (fabsf(d1y) <= fabsf(d1z)) {
                nx = -d1z;
                ny = 0.0f;
                nz = d1x;
            } else {
                nx = d1y;
                ny = -d1x;
                nz = 0.0f;
            }
            normal_length = sqrtf(nx * nx + ny * ny + nz * nz);
        }
        if (normal_length > 1.0e-7f) {
            nx /= normal_length;
            ny /= normal_length;
            nz /= normal_length;
        } else {
            nx = 1.0f;
        }
        float dominant;
        if (fabsf(nx) >= fabsf(ny) && fabsf(nx) >= fabsf(nz))
            dominant = nx;
        else if (fabsf(ny) >= fabsf(nz))
            dominant = ny;
        else
            dominant = nz;
        if (dominant < 0.0f) {
            nx = -nx;
            ny = -ny;
            nz = -nz;
        }
        if (h.segment > other) {
            nx = -nx;
            ny = -ny;
            nz = -nz;
        }
    }
    float weight_0 = 1.0f - s;
    float weight_1 = s;
    float other_weight_0 = 1.0f - t;
    float denominator = weight_0 * weight_0 + weight_1 * weight_1 + other_weight_0 * other_weight_0 + t * t;
    float magnitude = -correction_fraction * penetration / denominator;
    float aggregate_weight = aggregation == 1 ? penetration : 1.0f;
    out.pen = penetration;
    out.t0x = nx * magnitude * weight_0 * aggregate_weight;
    out.t0y = ny * magnitude * weight_0 * aggregate_weight;
    out.t0z = nz * magnitude * weight_0 * aggregate_weight;
    out.t1x = nx * magnitude * weight_1 * aggregate_weight;
    out.t1y = ny * magnitude * weight_1 * aggregate_weight;
    out.t1z = nz * magnitude * weight_1 * aggregate_weight;
    out.aggw = aggregate_weight;
    return true;
}

struct ContactAcc {
    float c0x, c0y, c0z, c1x, c1y, c1z, weight, maxpen;
};

// contact.rs:750-870 for one hit: the running sums in the reference's order.
__device__ inline void add_hit(ContactAcc &acc, uint32_t aggregation, float pen, float t0x, float t0y, float t0z,
                               float t1x, float t1y, float t1z, float aggw) {
    bool deepest = pen > acc.maxpen;
    if (deepest) acc.maxpen = pen;
    if (aggregation == 2) {
        if (deepest) {
            acc.c0x = t0x;
            acc.c0y = t0y;
            acc.c0z = t0z;
            acc.c1x = t1x;
            acc.c1y = t1y;
            acc.c1z = t1z;
            acc.weight = 1.0f;
        }
    } else {
        acc.c0x += t0x;
        acc.c0y += t0y;
        acc.c0z += t0z;
        acc.c1x += t1x;
        acc.c1y += t1y;
        acc.c1z += t1z;
        acc.weight += aggw;
    }
}

}  // namespace tgl
