// capture.cu -- capture_segment_contacts (crates/tangle_contact/src/device/
// contact.rs:9-230): every pair of segments of different fibers whose
// surfaces are within a gap of each other, with its closest-point
// coordinates, surface gap and crossing angle, on a whole-segment cell grid.
#include "kernels.cuh"

namespace tgl {
namespace {

// One thread per segment walks the 27 cells around its midpoint's cell; a
// stencil cell past a periodic face shifts the other segment by a box length
// before the minimum-image rounding, as the reference does (contact.rs:82-130).
__global__ void capture_kernel(WorldDev w, float max_gap, uint32_t capacity, uint32_t *count, uint32_t *pairs,
                               float *coordinates, float *gaps, float *angles) {
    const Grid &g = w.grid;
    const float length_epsilon = 1.0e-20f, parallel_relative_epsilon = 1.0e-6f;
    for (uint32_t segment = blockIdx.x * blockDim.x + threadIdx.x; segment < w.S;
         segment += gridDim.x * blockDim.x) {
        if (!segment_on(w, segment)) continue;
        const uint32_t v0 = w.seg_v0[segment];
        const float4 P1 = w.pos[v0], Q1 = w.pos[v0 + 1];
        const float p1x = P1.x, p1y = P1.y, p1z = P1.z, q1x = Q1.x, q1y = Q1.y, q1z = Q1.z;
        const float d1x = q1x - p1x, d1y = q1y - p1y, d1z = q1z - p1z;
        const float4 own = w.seg_static[segment];
        const uint32_t owner = __float_as_uint(own.w);
        const float radius = own.x;
        const float mx = 0.5f * (p1x + q1x), my = 0.5f * (p1y + q1y), mz = 0.5f * (p1z + q1z);
        const int32_t cx = (int32_t)g.cells[0], cy = (int32_t)g.cells[1], cz = (int32_t)g.cells[2];
        const int32_t rx = f32_to_i32(floorf((mx - g.lower[0]) / g.width[0]));
        const int32_t ry = f32_to_i32(floorf((my - g.lower[1]) / g.width[1]));
        const int32_t rz = f32_to_i32(floorf((mz - g.lower[2]) / g.width[2]));
        int32_t hx = min(max(rx, 0), cx - 1), hy = min(max(ry, 0), cy - 1), hz = min(max(rz, 0), cz - 1);
        if (g.periodic[0]) hx = (rx % cx + cx) % cx;
        if (g.periodic[1]) hy = (ry % cy + cy) % cy;
        if (g.periodic[2]) hz = (rz % cz + cz) % cz;
        const uint32_t home = ((uint32_t)hz * g.cells[1] + (uint32_t)hy) * g.cells[0] + (uint32_t)hx;
        for (uint32_t n = 0; n < 27; ++n) {
            const uint32_t cell = stencil_cell(home, n, g);
            if (cell == TGL_NONE) continue;
            const int32_t ox = (int32_t)(n % 3) - 1, oy = (int32_t)((n / 3) % 3) - 1, oz = (int32_t)(n / 9) - 1;
            const int32_t nx = hx + ox, ny = hy + oy, nz = hz + oz;
            const float sx = nx < 0 ? -g.length[0] : (nx >= cx ? g.length[0] : 0.0f);
            const float sy = ny < 0 ? -g.length[1] : (ny >= cy ? g.length[1] : 0.0f);
            const float sz = nz < 0 ? -g.length[2] : (nz >= cz ? g.length[2] : 0.0f);
            const uint32_t start = w.cell_offsets[cell], cnt = w.cell_counts[cell];
            for (uint32_t k = 0; k < cnt; ++k) {
                const uint32_t other = w.cell_segments[start + k];
                if (other <= segment || __float_as_uint(w.seg_static[other].w) == owner) continue;
                const uint32_t u0 = w.seg_v0[other];
                const float4 P2 = w.pos[u0], Q2 = w.pos[u0 + 1];
                float p2x = P2.x + sx, p2y = P2.y + sy, p2z = P2.z + sz;
                float q2x = Q2.x + sx, q2y = Q2.y + sy, q2z = Q2.z + sz;
                const float idx = 0.5f * (p2x + q2x - p1x - q1x);
                const float idy = 0.5f * (p2y + q2y - p1y - q1y);
                const float idz = 0.5f * (p2z + q2z - p1z - q1z);
                if (g.periodic[0]) {
                    const float shift = roundf(idx / g.length[0]) * g.length[0];
                    p2x -= shift;
                    q2x -= shift;
                }
                if (g.periodic[1]) {
                    const float shift = roundf(idy / g.length[1]) * g.length[1];
                    p2y -= shift;
                    q2y -= shift;
                }
                if (g.periodic[2]) {
                    const float shift = roundf(idz / g.length[2]) * g.length[2];
                    p2z -= shift;
                    q2z -= shift;
                }
                const float d2x = q2x - p2x, d2y = q2y - p2y, d2z = q2z - p2z;
                const float r0x = p1x - p2x, r0y = p1y - p2y, r0z = p1z - p2z;
                const float a = d1x * d1x + d1y * d1y + d1z * d1z;
                const float e = d2x * d2x + d2y * d2y + d2z * d2z;
                const float f = d2x * r0x + d2y * r0y + d2z * r0z;
                float s = 0.0f, t = 0.0f;
                if (a <= length_epsilon && e > length_epsilon) {
                    t = clampf(f / e, 0.0f, 1.0f);
                } else if (a > length_epsilon) {
                    const float c = d1x * r0x + d1y * r0y + d1z * r0z;
                    if (e <= length_epsilon) {
                        s = clampf(-c / a, 0.0f, 1.0f);
                    } else {
                        const float b = d1x * d2x + d1y * d2y + d1z * d2z;
                        const float denominator = a * e - b * b;
                        if (fabsf(denominator) > parallel_relative_epsilon * a * e)
                            s = clampf((b * f - c * e) / denominator, 0.0f, 1.0f);
                        const float projected = (b * s + f) / e;
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
                const float dx = (p2x + d2x * t) - (p1x + d1x * s);
                const float dy = (p2y + d2y * t) - (p1y + d1y * s);
                const float dz = (p2z + d2z * t) - (p1z + d1z * s);
                const float gap = sqrtf(dx * dx + dy * dy + dz * dz) - radius - w.seg_static[other].x;
                if (!(gap <= max_gap)) continue;
                const uint32_t at = atomicAdd(&count[0], 1u);
                if (at >= capacity) {
                    count[1] = 1u;
                    continue;
                }
                pairs[2 * (size_t)at] = segment;
                pairs[2 * (size_t)at + 1] = other;
                coordinates[2 * (size_t)at] = s;
                coordinates[2 * (size_t)at + 1] = t;
                gaps[at] = gap;
                const float product = sqrtf(a * e);
                float angle = 0.0f;
                if (product > length_epsilon)
                    angle = acos_f32(clampf(fabsf((d1x * d2x + d1y * d2y + d1z * d2z) / product), 0.0f, 1.0f));
                angles[at] = angle;
            }
        }
    }
}

}  // namespace

void launch_capture(const WorldDev &w, float max_gap, uint32_t capacity, uint32_t *count, uint32_t *pairs,
                    float *coordinates, float *gaps, float *angles, cudaStream_t st) {
    int blocks = (int)((w.S + 127) / 128);
    if (blocks < 1) blocks = 1;
    if (blocks > 148 * 32) blocks = 148 * 32;
    capture_kernel<<<blocks, 128, 0, st>>>(w, max_gap, capacity, count, pairs, coordinates, gaps, angles);
}

}  // namespace tgl
