// kernels.cu -- sm_100a kernels of the plain relaxation path.
//
// One relaxation step is three launches, fused from the reference's ~13:
//   [rebuild, gated on neighbor_state[0]]  cell list + Verlet lists (in a
//                     batch graph, the body of a conditional node that runs
//                     it only when a rebuild is pending)
//   contact_kernel    find_segment_corrections (contact.rs:232-902); the
//                     last block to finish reduces the gate metrics and runs
//                     assess_reduced_metrics (kernels.rs:129-162)
//   fiber_kernel      everything after the gate, which only ever touches one
//                     fiber: internal stretch/bend x constraint_iterations
//                     (kernels.rs:1027-1163, :1417-1453), apply contact
//                     (:1455-1537), curvature Gauss-Seidel (:1165-1415), the
//                     displacement check (neighbor.rs:446-465) and the next
//                     gate's curvature and step measurements (:925-980,
//                     :95-127). One warp owns one fiber, staged in shared
//                     memory.
// Float reductions that feed positions are done in the reference's order
// (contacts summed in ascending list order); only maxima, which are exact in
// any order, use atomics (on u32 bits of non-negative floats).
#include "kernels.cuh"
#include "formation.cuh"
#include "contact.cuh"

#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>

namespace tgl {

namespace {

constexpr uint32_t FULL = 0xFFFFFFFFu;
constexpr int CELL_SORT_CAP = 512;  // slots sorted in shared memory per cell

__device__ inline uint32_t warp_max_u32(uint32_t v) { return __reduce_max_sync(FULL, v); }

// Specimen accessors. A single world is specimen 0 with the world's own
// grid, skin and control word (the ARENA = false instantiations compile to
// exactly that); an arena looks each element's specimen up.
template <bool A> __device__ inline uint32_t spec_of_seg(const WorldDev &w, uint32_t s) { return A ? w.seg_spec[s] : 0u; }
template <bool A> __device__ inline uint32_t spec_of_fiber(const WorldDev &w, uint32_t f) {
    return A ? w.fiber_spec[f] : 0u;
}
template <bool A> __device__ inline uint32_t spec_of_vtx(const WorldDev &w, uint32_t v) { return A ? w.vtx_spec[v] : 0u; }
template <bool A> __device__ inline uint32_t spec_of_cell(const WorldDev &w, uint32_t c) {
    return A ? w.cell_spec[c] : 0u;
}
template <bool A> __device__ inline const Grid &grid_of(const WorldDev &w, uint32_t p) {
    return A ? w.specs[p].grid : w.grid;
}
template <bool A> __device__ inline float skin_of(const WorldDev &w, uint32_t p) { return A ? w.specs[p].skin : w.skin; }
template <bool A> __device__ inline uint32_t cell_base_of(const WorldDev &w, uint32_t p) {
    return A ? w.specs[p].cell_base : 0u;
}
template <bool A> __device__ inline Control *ctl_of(const WorldDev &w, uint32_t p) { return A ? w.ctl + 1 + p : w.ctl; }
// Whether specimen p's rebuild is pending (an arena rebuilds per specimen).
template <bool A> __device__ inline bool rebuilding(const WorldDev &w, uint32_t p) {
    return ctl_of<A>(w, p)->neighbor_state[0] != 0;
}
// Raises specimen p's rebuild flag (and, in an arena, the any-specimen one).
template <bool A> __device__ inline void flag_rebuild(const WorldDev &w, uint32_t p) {
    ctl_of<A>(w, p)->neighbor_state[0] = 1;
    if (A) w.ctl->neighbor_state[0] = 1;
}
// Raises specimen p's contact-list refresh flag (and, in an arena, the
// any-specimen one, which lets the refresh pass run).
template <bool A> __device__ inline void flag_refresh(const WorldDev &w, uint32_t p) {
    ctl_of<A>(w, p)->contact_state[0] = 1;
    if (A) w.ctl->contact_state[0] = 1;
}

// ---------------------------------------------------------------- batch control

// kernels.rs:3-12 begin_relaxation_batch; also clears the gate accumulators.
__device__ inline void begin_batch(Control *ctl) {
    ctl->control[2] = 0;
    if (ctl->control[3] == 0) ctl->control[0] = 1;
    ctl->acc[0] = 0;
    ctl->acc[1] = 0;
    ctl->acc[2] = 0;
    ctl->done_blocks = 0;
    ctl->next_batch = 0;
}

template <bool A>
__global__ void begin_batch_kernel(WorldDev w) {
    if (threadIdx.x == 0) w.ctl->loop_step = 0;
    if constexpr (!A) {
        if (threadIdx.x == 0) begin_batch(w.ctl);
    } else {
        for (uint32_t p = threadIdx.x; p < w.P; p += blockDim.x) {
            begin_batch(w.ctl + 1 + p);
            // A specimen resumed with a refresh still pending (it stopped
            // first) gets it in this batch.
            if (w.ctl[1 + p].contact_state[0]) w.ctl->contact_state[0] = 1;
        }
        if (threadIdx.x == 0) {
            w.ctl->control[0] = 1;  // some specimen may run; the first gate refines it
            w.ctl->done_blocks = 0;
            w.ctl->next_batch = 0;
        }
    }
}

// Whether vertex v at (x, y, z) has moved more than half the contact skin
// (less 0.1 %, a margin for rounding) from the contact lists' snapshot.
__device__ inline bool contact_moved(const WorldDev &w, uint32_t v, float x, float y, float z) {
    const float limit = 0.4995f * w.contact_skin;
    const float4 c = w.contact_ref[v];
    const float dx = x - c.x, dy = y - c.y, dz = z - c.z;
    return dx * dx + dy * dy + dz * dz > limit * limit;
}

// neighbor.rs:446-465, over the active vertices, and the same check
// against the contact lists' snapshot.
template <bool A>
__global__ void flag_displacement_kernel(WorldDev w) {
    uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    bool far = false, contact_far = false;
    if (v < w.V && (A || vertex_on(w, v))) {
        const uint32_t spec = spec_of_vtx<A>(w, v);
        float md = 0.5f * skin_of<A>(w, spec);
        float4 p = w.pos[v], r = w.ref_pos[v];
        float dx = p.x - r.x, dy = p.y - r.y, dz = p.z - r.z;
        far = dx * dx + dy * dy + dz * dz > md * md;
        if (A && far) flag_rebuild<A>(w, spec);
        if (w.contact_skin > 0.0f && contact_moved(w, v, p.x, p.y, p.z)) {
            contact_far = true;
            if (A) flag_refresh<A>(w, spec);
        }
    }
    if (w.contact_skin > 0.0f && v < w.S && w.geom[2 * (size_t)v + 1].w > w.contact_half_limit) {
        contact_far = true;
        if (A) flag_refresh<A>(w, spec_of_seg<A>(w, v));
    }
    if (A) return;
    if (__any_sync(FULL, far) && (threadIdx.x & 31) == 0) w.ctl->neighbor_state[0] = 1;
    if (__any_sync(FULL, contact_far) && (threadIdx.x & 31) == 0) w.ctl->contact_state[0] = 1;
}

// neighbor.rs:436-441 (every specimen of an arena).
template <bool A>
__global__ void request_rebuild_kernel(WorldDev w) {
    if (A)
        for (uint32_t p = threadIdx.x; p < w.P; p += blockDim.x) w.ctl[1 + p].neighbor_state[0] = 1;
    if (threadIdx.x == 0) w.ctl->neighbor_state[0] = 1;
}

// Gate inputs for the first step of a batch: curvature ratio of the current
// positions and the last applied step (kernels.rs:112-127).
template <bool A>
__global__ void measure_start_kernel(WorldDev w) {
    if (w.ctl->control[0] == 0) return;
    const int lane = threadIdx.x & 31;
    const int warps = blockDim.x >> 5;
    uint32_t cmax = 0, smax = 0;
    for (uint32_t k = blockIdx.x * warps + (threadIdx.x >> 5); k < w.FA; k += gridDim.x * warps) {
        const uint32_t f = w.fiber_order[k];
        const uint32_t spec = spec_of_fiber<A>(w, f);
        if (A && ctl_of<A>(w, spec)->control[0] == 0) continue;
        uint2 span = w.fiber_vspan[f];
        const float4 *P = w.pos + span.x;
        for (uint32_t i = lane; i < span.y; i += 32) {
            float step = w.vertex_step[span.x + i];
            smax = max(smax, __float_as_uint(fmaxf(step, 0.0f)));
            if (i > 0 && i + 1 < span.y) {
                float maximum = w.vtx_static[span.x + i].x;
                if (maximum > 0.0f) {
                    float r = curvature_ratio_at([&](int k) { return P[k]; }, (int)i, maximum);
                    cmax = max(cmax, __float_as_uint(fmaxf(r, 0.0f)));
                }
            }
        }
        if (A) {  // per fiber: its specimen's maxima
            cmax = warp_max_u32(cmax);
            smax = warp_max_u32(smax);
            if (lane == 0) {
                if (smax) atomicMax(&ctl_of<A>(w, spec)->acc[1], smax);
                if (cmax) atomicMax(&ctl_of<A>(w, spec)->acc[2], cmax);
            }
            cmax = smax = 0;
        }
    }
    if (A) return;
    cmax = warp_max_u32(cmax);
    smax = warp_max_u32(smax);
    if (lane == 0) {
        if (smax) atomicMax(&w.ctl->acc[1], smax);
        if (cmax) atomicMax(&w.ctl->acc[2], cmax);
    }
}

// ---------------------------------------------------------------- cell list
// cell_list.rs:8-378 / world/cell_list.rs:94-209, gated on the rebuild flag.

// (In an arena, only the cells, segments and vertices of specimens whose
// rebuild is pending are touched: each specimen owns a contiguous cell range
// and the slot range of its own segment ids, so the other specimens' lists
// stay as they are.)
template <bool A>
__global__ void rb_clear_kernel(WorldDev w) {
    if (w.ctl->neighbor_state[0] == 0) return;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < w.C; c += gridDim.x * blockDim.x)
        if (!A || rebuilding<A>(w, spec_of_cell<A>(w, c))) w.cell_counts[c] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) w.ctl->cell_overflow = 0;
}

// count_cell_segments: each segment's midpoint cell, and its arrival ticket;
// the segments of inactive fibers stay out of the cell list.
template <bool A>
__global__ void rb_count_kernel(WorldDev w) {
    if (w.ctl->neighbor_state[0] == 0) return;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < w.S; s += gridDim.x * blockDim.x) {
        const uint32_t spec = spec_of_seg<A>(w, s);
        if (A && !rebuilding<A>(w, spec)) continue;
        if (!A && !segment_on(w, s)) continue;
        float4 a = w.geom[2 * (size_t)s], b = w.geom[2 * (size_t)s + 1];
        uint32_t cell = cell_base_of<A>(w, spec) + proxy_cell(a.x, a.y, a.z, b.x, b.y, b.z, grid_of<A>(w, spec));
        w.cell_of[s] = cell;
        w.ticket[s] = atomicAdd(&w.cell_counts[cell], 1u);
    }
}

// Exclusive scan of the cell counts in one block (4096 cells per round).
// In an arena, block p scans specimen p's cell range alone, starting at its
// first slot (its first segment id), and only when its rebuild is pending.
template <bool A>
__global__ void __launch_bounds__(1024) rb_scan_kernel(WorldDev w) {
    if (w.ctl->neighbor_state[0] == 0) return;
    const uint32_t spec = A ? blockIdx.x : 0u;
    if (A && !rebuilding<A>(w, spec)) return;
    const uint32_t first = A ? w.specs[spec].cell_base : 0u;
    const uint32_t end = A ? first + w.specs[spec].cell_count : w.C;
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t carry_s;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry_s = A ? w.specs[spec].seg_base : 0u;
    __syncthreads();
    for (uint32_t base = first; base < end; base += 4096) {
        uint32_t idx = base + threadIdx.x * 4;
        uint32_t v[4];
        uint32_t local = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            v[k] = (idx + k < end) ? w.cell_counts[idx + k] : 0u;
            local += v[k];
        }
        uint32_t incl = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t ws = warp_sums[lane];
            uint32_t wi = ws;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t t = __shfl_up_sync(FULL, wi, o);
                if (lane >= o) wi += t;
            }
            warp_sums[lane] = wi - ws;  // exclusive warp offsets
        }
        __syncthreads();
        uint32_t run = carry_s + warp_sums[warp] + incl - local;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (idx + k < end) w.cell_offsets[idx + k] = run;
            run += v[k];
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry_s = run;
        __syncthreads();
    }
}

// scatter_cell_segments.
template <bool A>
__global__ void rb_scatter_kernel(WorldDev w) {
    if (w.ctl->neighbor_state[0] == 0) return;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < w.S; s += gridDim.x * blockDim.x)
        if (A ? rebuilding<A>(w, spec_of_seg<A>(w, s)) : segment_on(w, s))
            w.cell_segments[w.cell_offsets[w.cell_of[s]] + w.ticket[s]] = s;
}

// rank_cell_segments (cell_list.rs:346-378): ascending segment order inside
// every cell. One warp per cell; a rank sort in shared memory, or over the
// global range (into the free ticket array) for very crowded cells.
template <bool A>
__global__ void rb_sort_cells_kernel(WorldDev w) {
    if (w.ctl->neighbor_state[0] == 0) return;
    extern __shared__ uint32_t sort_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    uint32_t *buf = sort_smem + warp * CELL_SORT_CAP;
    for (uint32_t c = blockIdx.x * warps + warp; c < w.C; c += gridDim.x * warps) {
        if (A && !rebuilding<A>(w, spec_of_cell<A>(w, c))) continue;
        uint32_t n = w.cell_counts[c];
        if (n < 2) continue;
        uint32_t off = w.cell_offsets[c];
        uint32_t *seg = w.cell_segments + off;
        if (n <= CELL_SORT_CAP) {
            for (uint32_t i = lane; i < n; i += 32) buf[i] = seg[i];
            __syncwarp();
            for (uint32_t i = lane; i < n; i += 32) {
                uint32_t key = buf[i], rank = 0;
                for (uint32_t j = 0; j < n; ++j) rank += buf[j] < key ? 1u : 0u;
                seg[rank] = key;
            }
            __syncwarp();
        } else {
            uint32_t *tmp = w.ticket + off;
            for (uint32_t i = lane; i < n; i += 32) {
                uint32_t key = seg[i], rank = 0;
                for (uint32_t j = 0; j < n; ++j) rank += seg[j] < key ? 1u : 0u;
                tmp[rank] = key;
            }
            __syncwarp();
            for (uint32_t i = lane; i < n; i += 32) seg[i] = tmp[i];
            __syncwarp();
        }
    }
}

// gather_cell_slot_geometry (neighbor.rs:109-170): geometry in slot order,
// plus each slot's bounding sphere (midpoint, half length + radius) for the
// build's pre-test.
template <bool A>
__global__ void rb_gather_kernel(WorldDev w) {
    if (w.ctl->neighbor_state[0] == 0) return;
    for (uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < w.NS; slot += gridDim.x * blockDim.x) {
        uint32_t s = w.cell_segments[slot];
        if (A && !rebuilding<A>(w, spec_of_seg<A>(w, s))) continue;
        float4 a = w.geom[2 * (size_t)s], b = w.geom[2 * (size_t)s + 1];
        w.slot_geom[2 * (size_t)slot] = a;
        w.slot_geom[2 * (size_t)slot + 1] = b;
        w.slot_sphere[slot] = make_float4(0.5f * (a.x + b.x), 0.5f * (a.y + b.y), 0.5f * (a.z + b.z), b.w + a.w);
    }
}

// The exact pair test of build_segment_neighbor_lists (neighbor.rs:282-359)
// for home segment 1 against the segment in `slot`.
__device__ inline bool build_pair(const WorldDev &w, const Grid &grid, float skin, float p1x, float p1y, float p1z,
                                  float q1x, float q1y, float q1z, float d1x, float d1y, float d1z, float radius,
                                  float half_length, uint32_t segment, float4 own, uint32_t slot, uint32_t &other) {
    const float4 oa = w.slot_geom[2 * (size_t)slot], ob = w.slot_geom[2 * (size_t)slot + 1];
    other = w.cell_segments[slot];
    float p2x = oa.x, p2y = oa.y, p2z = oa.z, q2x = ob.x, q2y = ob.y, q2z = ob.z;
    const float other_radius = oa.w;
    bool moved = minimum_image(p1x, p1y, p1z, q1x, q1y, q1z, p2x, p2y, p2z, q2x, q2y, q2z, grid);
    float d2x = q2x - p2x, d2y = q2y - p2y, d2z = q2z - p2z;
    float interaction = (radius + other_radius + skin) * (1.0f + 1.0e-4f);
    float mdx = 0.5f * (p2x + q2x - p1x - q1x);
    float mdy = 0.5f * (p2y + q2y - p1y - q1y);
    float mdz = 0.5f * (p2z + q2z - p1z - q1z);
    float other_half = moved ? 0.5f * sqrtf(d2x * d2x + d2y * d2y + d2z * d2z) : ob.w;
    float reach = half_length + other_half + interaction;
    if (!(mdx * mdx + mdy * mdy + mdz * mdz <= reach * reach)) return false;
    if (!(axis_distance(p1x, p1y, p1z, d1x, d1y, d1z, p2x, p2y, p2z, d2x, d2y, d2z) <= interaction)) return false;
    // The pair-independent exclusions (neighbor.rs:282-294).
    float4 os = w.seg_static[other];
    float gap = fmaxf(os.y - own.z, own.y - os.z);  // along_fiber_gap
    bool near_along_fiber = __float_as_uint(os.w) == __float_as_uint(own.w) && gap < radius + os.x;
    return other != segment && !near_along_fiber;
}

// Order-preserving int key of an f32, for shared-memory atomic min / max.
__device__ inline int float_key(float x) {
    const int b = __float_as_int(x);
    return b >= 0 ? b : b ^ 0x7fffffff;
}
__device__ inline float key_float(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7fffffff); }

// Distance along one axis from 0 to the interval [lo, hi].
__device__ inline float interval_gap(float lo, float hi) { return fmaxf(0.0f, fmaxf(lo, -hi)); }

// Each cell's CellBox, once per rebuild: one warp per cell reduces the
// bounding spheres in its slot range. The build's culling reads the 27
// boxes around a home cell from here instead of every home block
// recomputing the boxes of its stencil cells.
template <bool A>
__global__ void rb_boxes_kernel(WorldDev w) {
    if (w.ctl->neighbor_state[0] == 0) return;
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < w.C; c += warps) {
        const uint32_t spec = spec_of_cell<A>(w, c);
        if (A && !rebuilding<A>(w, spec)) continue;
        const Grid &g = grid_of<A>(w, spec);
        const uint32_t local = c - cell_base_of<A>(w, spec);
        const float face[3] = {g.lower[0] + (float)(local % g.cells[0]) * g.width[0],
                               g.lower[1] + (float)((local / g.cells[0]) % g.cells[1]) * g.width[1],
                               g.lower[2] + (float)(local / (g.cells[0] * g.cells[1])) * g.width[2]};
        int lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = float_key(INFINITY);
            hi[a] = float_key(-INFINITY);
        }
        uint32_t mag = 0u;
        const uint32_t n = w.cell_counts[c], off = w.cell_offsets[c];
        for (uint32_t i = lane; i < n; i += 32) {
            const float4 sp = w.slot_sphere[off + i];
            const float r = sp.w * 1.0003f;
            const float centre[3] = {sp.x, sp.y, sp.z};
            for (int a = 0; a < 3; ++a) {
                float p = centre[a] - face[a];
                if (g.periodic[a]) p -= rintf(p * g.inv_length[a]) * g.length[a];
                float l = p - r, h = p + r;
                if (!(isfinite(l) && isfinite(h))) {
                    l = -INFINITY;
                    h = INFINITY;
                }
                lo[a] = min(lo[a], float_key(l));
                hi[a] = max(hi[a], float_key(h));
            }
            mag = max(mag, __float_as_uint(fabsf(sp.x) + fabsf(sp.y) + fabsf(sp.z)));
        }
        CellBox box;
        for (int a = 0; a < 3; ++a) {
            box.lo[a] = __reduce_min_sync(FULL, lo[a]);
            box.hi[a] = __reduce_max_sync(FULL, hi[a]);
        }
        box.mag = __reduce_max_sync(FULL, mag);
        box.pad = 0u;
        if (lane == 0) w.cell_box[c] = box;
    }
}

// build_segment_neighbor_lists (neighbor.rs:171-364). One block per home cell.
// The 27 stencil cells' bounding spheres are staged in shared memory; each
// warp takes one home segment and tests 32 candidates at a time with a
// conservative sphere test. A pair the exact test accepts always passes it:
// the sphere threshold exceeds the exact reach by 2e-4 relative plus an
// absolute margin far above f32 rounding, and the sphere test's image
// (nearest integer of the separation in box lengths, ties to even) can only
// differ from the exact test's near a half-box separation, which with at
// least 3 cells on every periodic axis is beyond any reach. (Coordinates are
// unwrapped, so a segment's cell says nothing about its image.) Survivors
// queue up and get the exact test 32 at a time; hits append in scan order
// and are sorted later.
//
// Stencil-cell culling (with the sphere test on). rb_boxes_kernel bounds each
// cell's spheres, radii scaled by 1.0003, by a box in that cell's own frame
// (centre minus the cell's lower corner, wrapped into the nearest image on
// periodic axes, so the frame is right whichever image the unwrapped
// coordinates sit in), once per rebuild; the block reads the boxes of its 27
// stencil cells (a stencil staged in several chunks tests each chunk against
// its cells' whole boxes, a superset). A home warp then skips every cell
// whose box is farther from its own sphere centre (in the home cell's frame,
// shifted by the stencil offset, nearest of the three images on periodic
// axes) than (home radius + skin) * 1.0002 + the sphere test's margin + a
// rounding margin. The distance to a box of balls is at most the distance to
// any of the balls, so no candidate of a skipped cell can pass the sphere
// test: the lists are the same, the scan is shorter. A non-finite sphere
// makes its cell's box unbounded (never skipped).
// Arena specimens are small (a few hundred cells each, with short lists), so
// their build is bound by the blocks in flight: five per SM at 48 registers
// and a 1,536-candidate chunk (rebuild stage of 512 specimens 91.9 -> 71.9
// ms). The single world sets no occupancy floor (0): at 80 registers three
// blocks with 3,072-candidate chunks fit, and a floor of three (69
// registers) measured 5 % slower on its longer per-cell scans.
template <bool A>
__global__ void __launch_bounds__(256, A ? 5 : 0) rb_build_kernel(WorldDev w, int ch, int prefilter_world, float sphere_eps_world) {
    if (w.ctl->neighbor_state[0] == 0) return;
    extern __shared__ float4 build_smem[];
    uint32_t *slot_of = reinterpret_cast<uint32_t *>(build_smem + ch);
    __shared__ uint32_t st_count[27], st_off[27], st_prefix[28];
    __shared__ float st_face[27][3];      // lower corner of each stencil cell
    __shared__ int box_lo[27][3], box_hi[27][3];  // float_key of the staged spheres' box, cell frame
    __shared__ uint32_t box_mag[27];      // largest |x| + |y| + |z| of a staged centre (f32 bits)
    __shared__ uint32_t queue[8][64];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    const uint32_t block = w.block;
    uint32_t *q = queue[warp];
    for (uint32_t h = blockIdx.x; h < w.C; h += gridDim.x) {
        const uint32_t spec = spec_of_cell<A>(w, h);
        if (A && !rebuilding<A>(w, spec)) continue;
        const Grid &g = grid_of<A>(w, spec);
        const float skin = skin_of<A>(w, spec);
        const uint32_t cell_base = cell_base_of<A>(w, spec);
        const int prefilter = A ? (int)w.specs[spec].build_prefilter : prefilter_world;
        const float sphere_eps = A ? w.specs[spec].build_sphere_eps : sphere_eps_world;
        uint32_t nh = w.cell_counts[h];
        if (nh == 0) continue;
        uint32_t hoff = w.cell_offsets[h];
        if (threadIdx.x < 27) {
            uint32_t cell = stencil_cell(h - cell_base, threadIdx.x, g);
            if (cell != TGL_NONE) {
                st_face[threadIdx.x][0] = g.lower[0] + (float)(cell % g.cells[0]) * g.width[0];
                st_face[threadIdx.x][1] = g.lower[1] + (float)((cell / g.cells[0]) % g.cells[1]) * g.width[1];
                st_face[threadIdx.x][2] = g.lower[2] + (float)(cell / (g.cells[0] * g.cells[1])) * g.width[2];
                cell += cell_base;
            }
            st_count[threadIdx.x] = cell == TGL_NONE ? 0u : w.cell_counts[cell];
            st_off[threadIdx.x] = cell == TGL_NONE ? 0u : w.cell_offsets[cell];
            if (prefilter && cell != TGL_NONE) {
                const CellBox box = w.cell_box[cell];
                for (int a = 0; a < 3; ++a) {
                    box_lo[threadIdx.x][a] = box.lo[a];
                    box_hi[threadIdx.x][a] = box.hi[a];
                }
                box_mag[threadIdx.x] = box.mag;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t run = 0;
            for (int k = 0; k < 27; ++k) {
                st_prefix[k] = run;
                run += st_count[k];
            }
            st_prefix[27] = run;
        }
        __syncthreads();
        const uint32_t total = st_prefix[27];
        // Rounding margin of the culling test: coordinates, corners and box
        // lengths are all within f32 rounding of their true values.
        float grid_scale = 0.0f, wmax = 0.0f;
        for (int a = 0; a < 3; ++a) {
            grid_scale += fabsf(g.lower[a]) + 2.0f * g.length[a];
            wmax = fmaxf(wmax, g.width[a]);
        }
        for (uint32_t base = 0; base < total; base += (uint32_t)ch) {
            uint32_t len = min((uint32_t)ch, total - base);
            for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
                uint32_t flat = base + i;
                int k = 0;
                while (k < 26 && st_prefix[k + 1] <= flat) ++k;
                uint32_t slot = st_off[k] + (flat - st_prefix[k]);
                slot_of[i] = slot;
                build_smem[i] = w.slot_sphere[slot];
            }
            __syncthreads();
            for (uint32_t hi = warp; hi < nh; hi += warps) {
                const uint32_t home = hoff + hi;
                const float4 a = w.slot_geom[2 * (size_t)home], b = w.slot_geom[2 * (size_t)home + 1];
                const float4 hs = w.slot_sphere[home];
                const uint32_t segment = w.cell_segments[home];
                const float p1x = a.x, p1y = a.y, p1z = a.z, radius = a.w;
                const float q1x = b.x, q1y = b.y, q1z = b.z;
                const float d1x = q1x - p1x, d1y = q1y - p1y, d1z = q1z - p1z;
                const float half_length = b.w;
                const float4 own = w.seg_static[segment];
                uint32_t count = base == 0 ? 0u : w.nbr_count[segment];
                uint32_t *list = w.nbr_list + (size_t)segment * block;
                // Lane k < 27 decides whether stencil cell k is scanned.
                bool scan = false;
                if (lane < 27) {
                    scan = max(st_prefix[lane], base) < min(st_prefix[lane + 1], base + len);
                    if (scan && prefilter) {
                        const float hc[3] = {hs.x, hs.y, hs.z};
                        const int off[3] = {lane % 3 - 1, (lane / 3) % 3 - 1, lane / 9 - 1};
                        float far2 = 0.0f;
                        for (int ax = 0; ax < 3; ++ax) {
                            float qh = hc[ax] - st_face[13][ax];
                            if (g.periodic[ax]) qh -= rintf(qh * g.inv_length[ax]) * g.length[ax];
                            const float shift = (float)off[ax] * g.width[ax] - qh;
                            const float lo = key_float(box_lo[lane][ax]) + shift;
                            const float hi_edge = key_float(box_hi[lane][ax]) + shift;
                            float gap = interval_gap(lo, hi_edge);
                            if (g.periodic[ax]) {
                                gap = g.cells[ax] < 3 ? 0.0f
                                                      : fminf(gap, fminf(interval_gap(lo + g.length[ax], hi_edge + g.length[ax]),
                                                                         interval_gap(lo - g.length[ax], hi_edge - g.length[ax])));
                            }
                            far2 += gap * gap;
                        }
                        const float margin =
                            1.0e-3f * wmax +
                            8.0e-6f * (__uint_as_float(box_mag[lane]) + fabsf(hs.x) + fabsf(hs.y) + fabsf(hs.z) + grid_scale);
                        const float reach = (hs.w + skin) * 1.0002f + sphere_eps + margin;
                        scan = !(far2 > reach * reach);
                    }
                }
                uint32_t cells_left = __ballot_sync(FULL, scan);
                uint32_t queued = 0;
                uint32_t c = 0, c_end = 0;  // the current cell's staged range
                for (;;) {
                    if (c >= c_end && cells_left) {
                        const int k = __ffs(cells_left) - 1;
                        cells_left &= cells_left - 1u;
                        c = max(st_prefix[k], base) - base;
                        c_end = min(st_prefix[k + 1], base + len) - base;
                    }
                    const bool more = c < c_end;
                    if (more) {
                        const uint32_t cc = c + lane;
                        bool pass = false;
                        if (cc < c_end) {
                            pass = true;
                            if (prefilter) {
                                float4 sp = build_smem[cc];
                                float dx = sp.x - hs.x, dy = sp.y - hs.y, dz = sp.z - hs.z;
                                if (g.periodic[0]) dx -= rintf(dx * g.inv_length[0]) * g.length[0];
                                if (g.periodic[1]) dy -= rintf(dy * g.inv_length[1]) * g.length[1];
                                if (g.periodic[2]) dz -= rintf(dz * g.inv_length[2]) * g.length[2];
                                float limit = (hs.w + sp.w + skin) * 1.0002f + sphere_eps;
                                pass = dx * dx + dy * dy + dz * dz <= limit * limit;
                            }
                        }
                        uint32_t ballot = __ballot_sync(FULL, pass);
                        if (pass) q[queued + __popc(ballot & ((1u << lane) - 1u))] = cc;
                        queued += __popc(ballot);
                        c += 32;
                        __syncwarp();
                    }
                    // Exact tests, 32 at a time, or the remainder at the end.
                    if (queued >= 32 || (!more && queued)) {
                        uint32_t n = min(queued, 32u);
                        bool hit = false;
                        uint32_t other = 0;
                        if ((uint32_t)lane < n)
                            hit = build_pair(w, g, skin, p1x, p1y, p1z, q1x, q1y, q1z, d1x, d1y, d1z, radius,
                                             half_length, segment, own, slot_of[q[lane]], other);
                        uint32_t ballot = __ballot_sync(FULL, hit);
                        uint32_t rank = __popc(ballot & ((1u << lane) - 1u));
                        if (hit && count + rank < block) list[count + rank] = other;
                        count += __popc(ballot);
                        __syncwarp();
                        uint32_t rest = queued - n;
                        uint32_t moved_entry = (uint32_t)lane < rest ? q[n + lane] : 0u;
                        __syncwarp();
                        if ((uint32_t)lane < rest) q[lane] = moved_entry;
                        __syncwarp();
                        queued = rest;
                    } else if (!more) {
                        break;
                    }
                }
                if (lane == 0) w.nbr_count[segment] = count;
            }
            __syncthreads();
        }
    }
}

// sort_neighbor_lists (neighbor.rs:373-411): ascending segment order for
// every list that fits its block; overflowed lists are never read.
template <bool A>
__global__ void rb_sort_lists_kernel(WorldDev w) {
    if (w.ctl->neighbor_state[0] == 0) return;
    extern __shared__ uint32_t list_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    uint32_t *buf = list_smem + (size_t)warp * w.block;
    for (uint32_t s = blockIdx.x * warps + warp; s < w.S; s += gridDim.x * warps) {
        if (A && !rebuilding<A>(w, spec_of_seg<A>(w, s))) continue;
        uint32_t n = w.nbr_count[s];
        if (n < 2 || n > w.block) continue;
        uint32_t *list = w.nbr_list + (size_t)s * w.block;
        for (uint32_t i = lane; i < n; i += 32) buf[i] = list[i];
        __syncwarp();
        for (uint32_t i = lane; i < n; i += 32) {
            uint32_t key = buf[i], rank = 0;
            for (uint32_t j = 0; j < n; ++j) rank += buf[j] < key ? 1u : 0u;
            list[rank] = key;
        }
        __syncwarp();
    }
}

// snapshot_neighbor_reference_positions (neighbor.rs:412-425).
template <bool A>
__global__ void rb_snapshot_kernel(WorldDev w) {
    if (w.ctl->neighbor_state[0] == 0) return;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < w.V; v += gridDim.x * blockDim.x)
        if (!A || rebuilding<A>(w, spec_of_vtx<A>(w, v))) w.ref_pos[v] = w.pos[v];
}

// finish_neighbor_list_rebuild (neighbor.rs:426-435).
// New Verlet lists (and slots) also call for new contact lists.
__device__ inline void finish_rebuild(Control *ctl) {
    if (ctl->neighbor_state[0] == 0) return;
    ctl->neighbor_state[0] = 0;
    ctl->neighbor_state[1] += 1;
    ctl->contact_state[0] = 1;
}

template <bool A>
__global__ void rb_finish_kernel(WorldDev w) {
    if (!A) {
        if (threadIdx.x == 0) finish_rebuild(w.ctl);
        return;
    }
    if (w.ctl->neighbor_state[0] == 0) return;
    for (uint32_t p = threadIdx.x; p < w.P; p += blockDim.x) finish_rebuild(w.ctl + 1 + p);
    __syncthreads();
    if (threadIdx.x == 0) {
        w.ctl->neighbor_state[0] = 0;
        w.ctl->contact_state[0] = 1;  // the arena's one refresh flag: new lists somewhere
    }
}

// ---------------------------------------------------------------- contact pass

// contact.rs:879-901: average (unless deepest-only) and store.
__device__ inline void finish_segment(const WorldDev &w, uint32_t segment, ContactAcc acc, uint32_t aggregation) {
    if (aggregation != 2 && acc.weight > 1.0e-20f) {
        acc.c0x /= acc.weight;
        acc.c0y /= acc.weight;
        acc.c0z /= acc.weight;
        acc.c1x /= acc.weight;
        acc.c1y /= acc.weight;
        acc.c1z /= acc.weight;
    }
    w.corr[2 * (size_t)segment] = make_float4(acc.c0x, acc.c0y, acc.c0z, acc.maxpen);
    w.corr[2 * (size_t)segment + 1] = make_float4(acc.c1x, acc.c1y, acc.c1z, 0.0f);
}

// A segment whose list overflowed: the whole warp scans the 27 cells around
// the home cell of the positions the lists were built from
// (contact.rs:365-437), 32 candidates at a time, summing hits in scan order.
template <bool A>
__device__ ContactAcc overflow_segment(const WorldDev &w, const StepParams &sp, uint32_t segment, int lane) {
    const uint32_t spec = spec_of_seg<A>(w, segment);
    const Grid &g = grid_of<A>(w, spec);
    const uint32_t cell_base = cell_base_of<A>(w, spec);
    const Home h = make_home(w.geom[2 * (size_t)segment], w.geom[2 * (size_t)segment + 1], segment);
    const float4 own = w.seg_static[segment];
    const uint32_t owner = __float_as_uint(own.w);
    const uint32_t v0 = w.seg_v0[segment];
    const float4 r0 = w.ref_pos[v0], r1 = w.ref_pos[v0 + 1];
    const uint32_t home = proxy_cell(r0.x, r0.y, r0.z, r1.x, r1.y, r1.z, g);
    ContactAcc acc = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    for (uint32_t n = 0; n < 27; ++n) {
        uint32_t cell = stencil_cell(home, n, g);
        if (cell == TGL_NONE) continue;
        cell += cell_base;
        const uint32_t count = w.cell_counts[cell];
        const uint32_t start = w.cell_offsets[cell];
        for (uint32_t k0 = 0; k0 < count; k0 += 32) {
            uint32_t k = k0 + lane;
            PairTerms pt;
            bool hit = false;
            if (k < count) {
                uint32_t other = w.cell_segments[start + k];
                float4 os = w.seg_static[other];
                float gap = fmaxf(os.y - own.z, own.y - os.z);
                bool near_along_fiber = __float_as_uint(os.w) == owner && gap < h.radius + os.x;
                if (other != segment && !near_along_fiber) {
                    float4 oa = w.geom[2 * (size_t)other], ob = w.geom[2 * (size_t)other + 1];
                    float p2x, p2y, p2z, q2x, q2y, q2z;
                    if (contact_reach(h, oa, ob, g, p2x, p2y, p2z, q2x, q2y, q2z))
                        hit = contact_solve(h, other, oa.w, p2x, p2y, p2z, q2x, q2y, q2z, sp.correction_fraction,
                                            sp.contact_aggregation, pt);
                }
            }
            uint32_t bits = __ballot_sync(FULL, hit);
            while (bits) {
                int j = __ffs(bits) - 1;
                bits &= bits - 1u;
                add_hit(acc, sp.contact_aggregation, __shfl_sync(FULL, pt.pen, j), __shfl_sync(FULL, pt.t0x, j),
                        __shfl_sync(FULL, pt.t0y, j), __shfl_sync(FULL, pt.t0z, j), __shfl_sync(FULL, pt.t1x, j),
                        __shfl_sync(FULL, pt.t1y, j), __shfl_sync(FULL, pt.t1z, j), __shfl_sync(FULL, pt.aggw, j));
            }
        }
    }
    return acc;
}

// Owner segment (batch lane) of flat candidate index f: the last h with
// pre[h] <= f (segments without candidates share their successor's start).
__device__ inline int owner_of(const uint32_t *pre, uint32_t f) {
    int h = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1)
        if (pre[h + step] <= f) h += step;
    return h;
}

// Neighbor-list entries are read once per pass: stream them past L2.
__device__ inline uint32_t load_stream(const uint32_t *p) { return __ldcs(p); }

// Geometry records are gathered many times per pass: keep them in L2 ahead
// of the streamed lists (a per-load cache-eviction hint, no cache state kept).
__device__ inline uint64_t make_keep_policy() {
    uint64_t policy;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(policy));
    return policy;
}

__device__ inline float4 load_keep(const float4 *p, uint64_t policy) {
    float4 v;
    asm volatile("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p), "l"(policy));
    return v;
}

constexpr int CONTACT_WARPS = 8;

// kernels.rs:129-162 assess_reduced_metrics on one control word: publish the
// gate metrics, stop or count the iteration, clear the accumulators.
__device__ inline void assess_reduced_metrics(Control *c, const StepParams &sp, uint32_t overflow) {
    float maximum_penetration = __uint_as_float(atomicAdd(&c->acc[0], 0u));
    float maximum_step = __uint_as_float(atomicAdd(&c->acc[1], 0u));
    float maximum_curvature_ratio = __uint_as_float(atomicAdd(&c->acc[2], 0u));
    c->metrics[0] = maximum_penetration;
    c->metrics[1] = maximum_step;
    c->metrics[2] = maximum_curvature_ratio;
    if (overflow != 0 ||
        (sp.force_full_iterations == 0 && maximum_penetration <= sp.penetration_tolerance &&
         maximum_curvature_ratio <= 1.0f + sp.curvature_ratio_tolerance) ||
        c->control[2] >= sp.max_iterations) {
        if (overflow != 0) c->control[3] = 1;
        c->control[0] = 0;
    } else {
        c->control[1] += 1;
        c->control[2] += 1;
    }
    c->acc[0] = 0;
    c->acc[1] = 0;
    c->acc[2] = 0;
}

// Contact pass modes: the Verlet lists as they are (CONTACT_FULL); the
// Verlet lists plus a refresh of the contact lists and their snapshot
// (CONTACT_REFRESH, run when the refresh flag is set); the contact lists
// (CONTACT_LISTED, run when it is clear).
enum { CONTACT_FULL = 0, CONTACT_REFRESH = 1, CONTACT_LISTED = 2 };

// find_segment_corrections (contact.rs:232-902) over warp-owned batches of 32
// segments taken in cell-list order: lane i owns the i-th segment's sums. The batch's listed
// candidates are walked as one flat sequence, 32 at a time, through the
// exact midpoint reject; the survivors queue up in that order and get the
// closed-form closest-point solve 32 at a time, and every hit is added to
// its segment's sums in list order, as the reference's serial loop adds it.
// Overflowed segments then take the exact cell scan. With `gate`, the last
// block to finish runs assess_reduced_metrics (kernels.rs:129-162).
//
// Contact lists. A candidate can only produce a hit while its segments'
// distance is below r1 + r2, and while no vertex has moved more than
// contact_skin / 2 from a snapshot, no segment distance has shrunk by more
// than contact_skin since it. So the Verlet-list entries whose distance at
// the snapshot is within contact_skin of touching (within_contact_skin, a
// conservative test) hold every hit of every pass until a vertex moves
// farther; the update kernel flags that, as it flags Verlet rebuilds, and a
// Verlet rebuild forces a refresh. Hits are summed in ascending segment
// order from a sub-sequence of the same sorted list, so the sums are bit for
// bit those of the full list. (The minimum image cannot change within the
// window while every half length stays below contact_half_limit, which the
// update kernel checks with the displacements.)
// In an arena (A) every lane looks up its segment's
// specimen: grid and line margin for its candidates, whether the specimen is
// still active, and the specimen whose gate its penetration feeds.
template <int MODE, bool A = false>
__global__ void __launch_bounds__(256, 3) contact_kernel(WorldDev w, StepParams sp, int gate, float line_eps_world) {
    __shared__ float4 home_geom[CONTACT_WARPS][64];
    __shared__ uint32_t prefix[CONTACT_WARPS][33];
    __shared__ float4 queue_geom[CONTACT_WARPS][128];  // 64 entries: {p2, r2}, {q2, other}
    __shared__ uint8_t queue_owner[CONTACT_WARPS][64]; // owner lane; bit 7: passed the exact tests (refresh)
    __shared__ uint32_t segments[CONTACT_WARPS][32];
    __shared__ const uint32_t *sources[CONTACT_WARPS][32];
    __shared__ uint32_t kept_count[CONTACT_WARPS][32];
    __shared__ uint32_t hit_mask[CONTACT_WARPS][32];   // queue lanes holding each owner's hits; zero between rounds
    __shared__ uint32_t lane_spec[A ? CONTACT_WARPS : 1][32];
    __shared__ uint32_t warp_max[CONTACT_WARPS];
    __shared__ int is_last;
    if (gate && w.ctl->control[0] == 0) return;
    // One world refreshes everything or nothing. In an arena a listed pass
    // always runs (for the specimens whose lists hold) and a refresh pass
    // when some specimen's flag is up (for those specimens).
    if (MODE == CONTACT_REFRESH && w.ctl->contact_state[0] == 0) return;
    if (!A && MODE == CONTACT_LISTED && w.ctl->contact_state[0] != 0) return;
    const bool refresh_follows = A && MODE == CONTACT_LISTED && w.ctl->contact_state[0] != 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t block = w.block;
    const uint32_t cblock = w.contact_block;
    const float cskin = w.contact_skin;
    float4 *hg = home_geom[warp];
    uint32_t *pre = prefix[warp];
    float4 *qg = queue_geom[warp];
    uint8_t *qo = queue_owner[warp];
    uint32_t *seg_of = segments[warp];
    const uint32_t **src = sources[warp];
    uint32_t *kept = kept_count[warp];
    uint32_t *hm = hit_mask[warp];
    hm[lane] = 0u;
    uint32_t thread_max = 0;
    const uint64_t geom_policy = make_keep_policy();
    if (MODE == CONTACT_REFRESH) {
        // The snapshot the next passes measure displacement against (in an
        // arena, of the specimens this pass refreshes).
        for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < w.V; v += gridDim.x * blockDim.x) {
            if (A) {
                const Control *c = ctl_of<A>(w, spec_of_vtx<A>(w, v));
                if (c->control[0] == 0 || c->contact_state[0] == 0) continue;
            }
            w.contact_ref[v] = w.pos[v];
        }
    }
    // One world: warps take the batches in slot order from one counter, so
    // the batches in flight at any moment are a narrow band of neighboring
    // cells whose candidates' records stay in L2 (a fixed stride lets the
    // warps drift apart over the pass and widen that band). An arena keeps
    // the fixed stride: its hundreds of thousands of batches per pass would
    // queue on the counter's one address (measured on 512 specimens: 4.26 ms
    // per pass with the counter against 2.47 ms with the stride, while one
    // mid-size world's 62 k batches run 0.283 ms against 0.309 ms).
    const auto take_batch = [&]() {
        uint32_t b = 0;
        if (lane == 0) b = atomicAdd(&w.ctl->next_batch, 1u);
        return __shfl_sync(FULL, b, 0) * 32u;
    };
    const uint32_t stride = gridDim.x * CONTACT_WARPS * 32u;
    for (uint32_t base = A ? (blockIdx.x * CONTACT_WARPS + warp) * 32u : take_batch(); base < w.NS;
         base = A ? base + stride : take_batch()) {
        // Batches follow the cell list's slot order, so the 32 segments of a
        // batch are spatial neighbors and share most of their candidates.
        const bool in_range = base + lane < w.NS;
        const uint32_t segment = in_range ? w.cell_segments[base + lane] : 0u;
        const uint32_t my_spec = A && in_range ? spec_of_seg<A>(w, segment) : 0u;
        // Segments of an arena specimen whose gate has stopped it are
        // skipped; of the others, a listed pass takes those whose specimen's
        // lists hold and a refresh pass those whose specimen's flag is up.
        const bool alive = in_range && (!A || ctl_of<A>(w, my_spec)->control[0] != 0);
        const bool flagged = A && MODE != CONTACT_FULL && alive && ctl_of<A>(w, my_spec)->contact_state[0] != 0;
        const bool valid = MODE == CONTACT_LISTED ? alive && !flagged : MODE == CONTACT_REFRESH && A ? flagged : alive;
        // A listed pass reads the slot's contact-list state (coalesced), and
        // the segment's Verlet count only where its contact list did not fit
        // the batch's chunk; the other passes walk the Verlet lists. Every
        // slot with a list in the chunk counts toward the others' offsets,
        // whoever takes it in this pass.
        const uint32_t cstate = MODE == CONTACT_LISTED && in_range ? w.contact_count[base + lane] : 0u;
        uint32_t count = 0u;
        if (MODE != CONTACT_LISTED) count = valid ? w.nbr_count[segment] : 0u;
        else if (valid && cstate == CONTACT_USE_VERLET) count = w.nbr_count[segment];
        const bool listed = MODE == CONTACT_LISTED ? valid && cstate != CONTACT_USE_SCAN : valid && count <= block;
        if (A) lane_spec[A ? warp : 0][lane] = my_spec;
        uint32_t k = listed ? count : 0u;
        const uint32_t *source = w.nbr_list + (size_t)segment * block;
        if (MODE == CONTACT_LISTED) {
            // The batch's contact lists lie back to back in its chunk, in
            // lane order: a lane's list starts after the lists of the lanes
            // before it that read the chunk.
            const bool chunked = listed && cstate != CONTACT_USE_VERLET;  // cstate <= 32 * cblock
            uint32_t before = in_range && cstate < CONTACT_USE_VERLET ? cstate : 0u;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(FULL, before, o);
                if (lane >= o) before += t;
            }
            if (chunked) {
                k = cstate;
                source = w.contact_list + (size_t)base * cblock + (before - cstate);
            }
        }
        uint32_t incl = k;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t t = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += t;
        }
        pre[lane + 1] = incl;
        if (lane == 0) pre[0] = 0;
        if (valid) {
            hg[2 * lane] = w.geom[2 * (size_t)segment];
            hg[2 * lane + 1] = w.geom[2 * (size_t)segment + 1];
        }
        seg_of[lane] = segment;
        src[lane] = source;
        kept[lane] = 0;
        __syncwarp();
        const uint32_t total = pre[32];
        ContactAcc acc = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        uint32_t queued = 0;
        // Refresh: entries kept so far in this batch (the chunk's fill level;
        // owners' lists are emitted in lane order) and the owners whose list
        // ran past the chunk's end.
        uint32_t emitted = 0, spilled_owners = 0;
        // Software pipeline over the flat candidate sequence: the list entry
        // of round r + 2 and the geometry of round r + 1 are in flight while
        // round r is tested.
        int h_next = 0, h_next2 = 0;
        uint32_t other_next = 0, other_next2 = 0;
        float4 oa_next = make_float4(0.0f, 0.0f, 0.0f, 0.0f), ob_next = oa_next;
        if (lane < (int)total) {
            h_next = owner_of(pre, lane);
            other_next = load_stream(src[h_next] + (lane - pre[h_next]));
        }
        if (32u + lane < total) {
            h_next2 = owner_of(pre, 32u + lane);
            other_next2 = load_stream(src[h_next2] + (32u + lane - pre[h_next2]));
        }
        if (lane < (int)total) {
            oa_next = load_keep(w.geom + 2 * (size_t)other_next, geom_policy);
            ob_next = load_keep(w.geom + 2 * (size_t)other_next + 1, geom_policy);
        }
        for (uint32_t f0 = 0; f0 < total || queued; f0 += 32) {
            if (f0 < total) {
                const uint32_t f = f0 + lane;
                const int h = h_next;
                const uint32_t other = other_next;
                const float4 oa = oa_next, ob = ob_next;
                // Advance the pipeline.
                h_next = h_next2;
                other_next = other_next2;
                if (f + 32 < total) {
                    oa_next = load_keep(w.geom + 2 * (size_t)other_next, geom_policy);
                    ob_next = load_keep(w.geom + 2 * (size_t)other_next + 1, geom_policy);
                }
                if (f + 64 < total) {
                    h_next2 = owner_of(pre, f + 64);
                    other_next2 = load_stream(src[h_next2] + (f + 64 - pre[h_next2]));
                }
                bool pass = false, exact = false;
                float p2x = 0.0f, p2y = 0.0f, p2z = 0.0f, q2x = 0.0f, q2y = 0.0f, q2z = 0.0f, r2 = 0.0f;
                uint32_t other_id = 0;
                int owner = 0;
                if (f < total) {
                    const Home home = make_home(hg[2 * h], hg[2 * h + 1], seg_of[h]);
                    const uint32_t hspec = A ? lane_spec[A ? warp : 0][h] : 0u;
                    const Grid &g = grid_of<A>(w, hspec);
                    const float line_eps = A ? w.specs[hspec].line_eps : line_eps_world;
                    if (MODE == CONTACT_REFRESH) {
                        // Queue what may come within the contact skin; mark
                        // what passes the pass's own exact tests.
                        pass = contact_reach_wide(home, oa, ob, g, cskin, p2x, p2y, p2z, q2x, q2y, q2z, exact) &&
                               lines_may_touch(home, p2x, p2y, p2z, q2x, q2y, q2z, oa.w + cskin, line_eps);
                        exact = exact && pass && lines_may_touch(home, p2x, p2y, p2z, q2x, q2y, q2z, oa.w, line_eps);
                    } else {
                        pass = contact_reach(home, oa, ob, g, p2x, p2y, p2z, q2x, q2y, q2z) &&
                               lines_may_touch(home, p2x, p2y, p2z, q2x, q2y, q2z, oa.w, line_eps);
                    }
                    r2 = oa.w;
                    other_id = other;
                    owner = h;
                }
                const uint32_t ballot = __ballot_sync(FULL, pass);
                if (pass) {
                    const uint32_t at = queued + __popc(ballot & ((1u << lane) - 1u));
                    qg[2 * at] = make_float4(p2x, p2y, p2z, r2);
                    qg[2 * at + 1] = make_float4(q2x, q2y, q2z, __uint_as_float(other_id));
                    qo[at] = (uint8_t)(owner | (exact ? 0x80 : 0));
                }
                queued += __popc(ballot);
                __syncwarp();
            }
            if (queued >= 32 || (f0 + 32 >= total && queued)) {
                const uint32_t n = min(queued, 32u);
                PairTerms pt;
                bool hit = false, keep = false;
                int h = 0;
                if ((uint32_t)lane < n) {
                    const float4 ea = qg[2 * lane], eb = qg[2 * lane + 1];
                    h = qo[lane] & 31;
                    const Home home = make_home(hg[2 * h], hg[2 * h + 1], seg_of[h]);
                    if (MODE != CONTACT_REFRESH || (qo[lane] & 0x80))
                        hit = contact_solve(home, __float_as_uint(eb.w), ea.w, ea.x, ea.y, ea.z, eb.x, eb.y, eb.z,
                                            sp.correction_fraction, sp.contact_aggregation, pt);
                    if (MODE == CONTACT_REFRESH)
                        keep = within_contact_skin(home, ea.x, ea.y, ea.z, eb.x, eb.y, eb.z, ea.w, cskin,
                                                   A ? w.specs[lane_spec[A ? warp : 0][h]].line_eps : line_eps_world);
                }
                if (MODE == CONTACT_REFRESH) {
                    // Append the kept entries to the batch's chunk in queue
                    // order, which is list order owner after owner, so each
                    // owner's contact list is one contiguous, ordered run.
                    const uint32_t keeps = __ballot_sync(FULL, keep);
                    const uint32_t peers = __match_any_sync(FULL, keep ? (uint32_t)h : 32u + (uint32_t)lane);
                    if (keep) {
                        const uint32_t at = emitted + __popc(keeps & ((1u << lane) - 1u));
                        if (at < 32u * cblock)
                            w.contact_list[(size_t)base * cblock + at] = __float_as_uint(qg[2 * lane + 1].w);
                        else
                            spilled_owners |= 1u << h;
                    }
                    __syncwarp();
                    if (keep && lane == 31 - __clz(peers)) kept[h] += __popc(peers);
                    emitted += __popc(keeps);
                    __syncwarp();
                }
                if (__any_sync(FULL, hit)) {
                    // Each hit parks its terms in its own (already consumed)
                    // queue slot and the lowest lane of each owner's hits
                    // posts their mask; every owner then adds its own hits in
                    // ascending queue order, the order of the list, so the
                    // owners sum in parallel and bit for bit as one by one.
                    const uint32_t peers = __match_any_sync(FULL, hit ? (uint32_t)h : 32u + (uint32_t)lane);
                    if (hit) {
                        qg[2 * lane] = make_float4(pt.pen, pt.t0x, pt.t0y, pt.t0z);
                        qg[2 * lane + 1] = make_float4(pt.t1x, pt.t1y, pt.t1z, pt.aggw);
                        if (lane == __ffs(peers) - 1) hm[h] = peers;
                    }
                    __syncwarp();
                    uint32_t mine = hm[lane];
                    if (mine) hm[lane] = 0u;
                    while (mine) {
                        const int j = __ffs(mine) - 1;
                        mine &= mine - 1u;
                        const float4 ta = qg[2 * j], tb = qg[2 * j + 1];
                        add_hit(acc, sp.contact_aggregation, ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w);
                    }
                    __syncwarp();
                }
                const uint32_t rest = queued - n;
                float4 ma = make_float4(0.0f, 0.0f, 0.0f, 0.0f), mb = ma;
                uint8_t mo = 0;
                if ((uint32_t)lane < rest) {
                    ma = qg[2 * (n + lane)];
                    mb = qg[2 * (n + lane) + 1];
                    mo = qo[n + lane];
                }
                __syncwarp();
                if ((uint32_t)lane < rest) {
                    qg[2 * lane] = ma;
                    qg[2 * lane + 1] = mb;
                    qo[lane] = mo;
                }
                __syncwarp();
                queued = rest;
            }
        }
        if (listed) {
            finish_segment(w, segment, acc, sp.contact_aggregation);
            thread_max = max(thread_max, __float_as_uint(fmaxf(acc.maxpen, 0.0f)));
        }
        if (A && gate && listed && thread_max) {  // each specimen's own maximum
            atomicMax(&ctl_of<A>(w, my_spec)->acc[0], thread_max);
            thread_max = 0;
        }
        if (MODE == CONTACT_REFRESH) {
            spilled_owners = __reduce_or_sync(FULL, spilled_owners);
            const bool batch_refreshed = __any_sync(FULL, valid);
            if (valid)
                w.contact_count[base + lane] = !listed ? CONTACT_USE_SCAN
                                               : (spilled_owners >> lane) & 1u ? CONTACT_USE_VERLET
                                                                               : kept[lane];
            else if (A && in_range && batch_refreshed)
                // The chunk was rewritten for the refreshed slots: a slot of
                // another specimen in the batch (stopped, or with lists that
                // hold) has no list in it now; its Verlet list (or the cell
                // scan) serves it until its own specimen's next refresh.
                w.contact_count[base + lane] = w.nbr_count[segment] <= block ? CONTACT_USE_VERLET : CONTACT_USE_SCAN;
        }
        uint32_t spill = __ballot_sync(FULL, valid && !listed);
        while (spill) {
            const int j = __ffs(spill) - 1;
            spill &= spill - 1u;
            const uint32_t spilled = __shfl_sync(FULL, segment, j);
            ContactAcc o = overflow_segment<A>(w, sp, spilled, lane);
            if (lane == 0) finish_segment(w, spilled, o, sp.contact_aggregation);
            if (A) {
                const uint32_t bits = __float_as_uint(fmaxf(o.maxpen, 0.0f));
                if (gate && lane == 0 && bits) atomicMax(&ctl_of<A>(w, spec_of_seg<A>(w, spilled))->acc[0], bits);
            } else {
                thread_max = max(thread_max, __float_as_uint(fmaxf(o.maxpen, 0.0f)));
            }
        }
        __syncwarp();
    }
    thread_max = warp_max_u32(thread_max);
    if (lane == 0) warp_max[warp] = thread_max;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t m = 0;
        for (int k = 0; k < CONTACT_WARPS; ++k) m = max(m, warp_max[k]);
        if (gate && !A && m) atomicMax(&w.ctl->acc[0], m);
        __threadfence();
        is_last = atomicAdd(&w.ctl->done_blocks, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    if (threadIdx.x == 0) {  // every warp of every block is past its last batch
        w.ctl->next_batch = 0;
        if (!gate || refresh_follows) w.ctl->done_blocks = 0;
    }
    // In an arena whose refresh pass runs next, that pass's last block runs
    // the gates, over both passes' maxima.
    if (!gate || refresh_follows) return;
    if (!A) {
        if (threadIdx.x == 0) {
            __threadfence();
            Control *c = w.ctl;
            assess_reduced_metrics(c, sp, c->cell_overflow);
            c->done_blocks = 0;
            if (MODE == CONTACT_REFRESH) {
                c->contact_state[0] = 0;
                c->contact_state[1] += 1;
            }
            __threadfence();
        }
        return;
    }
    // Arena: every still-active specimen's own gate; the world stays active
    // while any specimen is.
    __shared__ int any_active;
    if (threadIdx.x == 0) any_active = 0;
    __threadfence();
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < w.P; p += blockDim.x) {
        Control *c = w.ctl + 1 + p;
        if (c->control[0] == 0) continue;
        if (MODE == CONTACT_REFRESH && c->contact_state[0]) {  // refreshed in this pass
            c->contact_state[0] = 0;
            c->contact_state[1] += 1;
        }
        assess_reduced_metrics(c, sp, w.ctl->cell_overflow);
        if (c->control[0]) any_active = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        w.ctl->control[0] = any_active ? 1u : 0u;
        w.ctl->done_blocks = 0;
        if (MODE == CONTACT_REFRESH) {
            w.ctl->contact_state[0] = 0;
            w.ctl->contact_state[1] += 1;
        }
        __threadfence();
    }
}

// ---------------------------------------------------------------- fiber update

struct Triplet {
    float scale, pw, cw, nw;
    float gux, guy, guz, cgx, cgy, cgz, gvx, gvy, gvz;
};

// project_curvature_triplet_in_place (kernels.rs:1165-1322), split into the
// test (does it move anything?) and the move, so that a warp can test many
// triplets at once and apply only the first that acts.
__device__ inline bool curvature_triplet_test(const float4 *P, const float4 *St, int prev, int center, int next,
                                              float stiffness, float safety_margin, Triplet &t) {
    float maximum_curvature = St[center].x * (1.0f - safety_margin);
    if (!(maximum_curvature > 0.0f)) return false;
    float4 pp = P[prev], pc = P[center], pn = P[next];
    float ux = pc.x - pp.x, uy = pc.y - pp.y, uz = pc.z - pp.z;
    float vx = pn.x - pc.x, vy = pn.y - pc.y, vz = pn.z - pc.z;
    const float uu = ux * ux + uy * uy + uz * uz;
    const float vv = vx * vx + vy * vy + vz * vz;
    if (uu > 1.0e-12f && vv > 1.0e-12f) {  // the rough rejection of lanes_test, below
        const float ru = rsqrtf(uu), rv = rsqrtf(vv);
        const float rough_half = 0.25f * maximum_curvature * (uu * ru + vv * rv);
        const float rough_limit = 1.0f - 2.0f * rough_half * rough_half;
        if ((ux * vx + uy * vy + uz * vz) * (ru * rv) > rough_limit + 1.0e-5f) return false;
    }
    float first_length = sqrtf(uu);
    float second_length = sqrtf(vv);
    if (!(first_length > 1.0e-7f && second_length > 1.0e-7f)) return false;
    float unx = ux / first_length, uny = uy / first_length, unz = uz / first_length;
    float vnx = vx / second_length, vny = vy / second_length, vnz = vz / second_length;
    float cosine = clampf(unx * vnx + uny * vny + unz * vnz, -1.0f, 1.0f);
    float sine_half = 0.25f * maximum_curvature * (first_length + second_length);
    if (!(sine_half < 1.0f)) return false;
    float minimum_cosine = 1.0f - 2.0f * sine_half * sine_half;
    float violation = minimum_cosine - cosine;
    float sine = sqrtf(fmaxf(1.0f - cosine * cosine, 0.0f));
    if (violation > 0.0f && sine > 1.0e-3f) violation = (acos_f32(cosine) - acos_f32(minimum_cosine)) * sine;
    if (!(violation > 0.0f)) return false;
    t.gux = (vnx - cosine * unx) / first_length;
    t.guy = (vny - cosine * uny) / first_length;
    t.guz = (vnz - cosine * unz) / first_length;
    t.gvx = (unx - cosine * vnx) / second_length;
    t.gvy = (uny - cosine * vny) / second_length;
    t.gvz = (unz - cosine * vnz) / second_length;
    t.cgx = t.gux - t.gvx;
    t.cgy = t.guy - t.gvy;
    t.cgz = t.guz - t.gvz;
    t.pw = pp.w != 0.0f ? 0.0f : 1.0f;  // w carries the pinned flag in shared memory
    t.cw = pc.w != 0.0f ? 0.0f : 1.0f;
    t.nw = pn.w != 0.0f ? 0.0f : 1.0f;
    float denominator = t.pw * (t.gux * t.gux + t.guy * t.guy + t.guz * t.guz) +
                        t.cw * (t.cgx * t.cgx + t.cgy * t.cgy + t.cgz * t.cgz) +
                        t.nw * (t.gvx * t.gvx + t.gvy * t.gvy + t.gvz * t.gvz);
    if (!(denominator > 1.0e-12f)) return false;
    t.scale = stiffness * violation / denominator;
    return t.pw > 0.0f || t.cw > 0.0f || t.nw > 0.0f;
}

__device__ inline float wall_clamp(float moved, float extent, int axis, const Grid &g) {
    return g.periodic[axis] ? moved : clampf(moved, g.lower[axis] + extent, g.upper[axis] - extent);
}

// wall_clamp that adds moved - kept to the vertex's wall reaction
// (kernels.rs:1440-1451, :1277-1305; R null = no reactions kept). The
// reference adds the difference after every projection; a zero difference
// leaves its running sum unchanged (the sum starts at +0 and a sum of
// differences is never -0), so only a clamp that moves a coordinate is
// written, by the one lane that owns the vertex at that point.
__device__ inline float wall_clamp_r(float moved, float extent, int axis, const Grid &g, float4 *R, int i) {
    const float kept = wall_clamp(moved, extent, axis, g);
    if (R != nullptr && !(kept == moved)) {
        float4 r = R[i];
        const float d = moved - kept;
        if (axis == 0)
            r.x += d;
        else if (axis == 1)
            r.y += d;
        else
            r.z += d;
        R[i] = r;
    }
    return kept;
}

__device__ inline void curvature_triplet_apply(float4 *P, const float4 *St, int prev, int center, int next,
                                               const Triplet &t, const Grid &g, float4 *R) {
    float4 pp = P[prev], pc = P[center], pn = P[next];
    float pe = St[prev].w, ce = St[center].w, ne = St[next].w;
    float mp, mc, mn;
    mp = pp.x - t.pw * t.scale * t.gux;
    mc = pc.x + t.cw * t.scale * t.cgx;
    mn = pn.x + t.nw * t.scale * t.gvx;
    if (t.pw > 0.0f) pp.x = wall_clamp_r(mp, pe, 0, g, R, prev);
    if (t.cw > 0.0f) pc.x = wall_clamp_r(mc, ce, 0, g, R, center);
    if (t.nw > 0.0f) pn.x = wall_clamp_r(mn, ne, 0, g, R, next);
    mp = pp.y - t.pw * t.scale * t.guy;
    mc = pc.y + t.cw * t.scale * t.cgy;
    mn = pn.y + t.nw * t.scale * t.gvy;
    if (t.pw > 0.0f) pp.y = wall_clamp_r(mp, pe, 1, g, R, prev);
    if (t.cw > 0.0f) pc.y = wall_clamp_r(mc, ce, 1, g, R, center);
    if (t.nw > 0.0f) pn.y = wall_clamp_r(mn, ne, 1, g, R, next);
    mp = pp.z - t.pw * t.scale * t.guz;
    mc = pc.z + t.cw * t.scale * t.cgz;
    mn = pn.z + t.nw * t.scale * t.gvz;
    if (t.pw > 0.0f) pp.z = wall_clamp_r(mp, pe, 2, g, R, prev);
    if (t.cw > 0.0f) pc.z = wall_clamp_r(mc, ce, 2, g, R, center);
    if (t.nw > 0.0f) pn.z = wall_clamp_r(mn, ne, 2, g, R, next);
    P[prev] = pp;
    P[center] = pc;
    P[next] = pn;
}

// Everything after the gate, one warp per fiber.
__global__ void __launch_bounds__(256) fiber_kernel(WorldDev w, StepParams sp) {
    if (w.ctl->control[0] == 0) return;
    extern __shared__ float4 fiber_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    const int maxv = (int)w.max_fiber;
    float4 *P = fiber_smem + (size_t)warp * 3 * maxv;  // positions, w = pinned
    float4 *T = P + maxv;                              // internal corrections
    float4 *St = T + maxv;                             // static vertex data
    const Grid &g = w.grid;
    const float md = 0.5f * w.skin;
    uint32_t smax = 0, cmax = 0;
    bool far = false;
    bool contact_far = false;
    const bool contact_lists = w.contact_skin > 0.0f;
    for (uint32_t k = blockIdx.x * warps + warp; k < w.FA; k += gridDim.x * warps) {
        const uint32_t f = w.fiber_order[k];
        const uint2 span = w.fiber_vspan[f];
        const uint32_t v0 = span.x;
        const int n = (int)span.y;
        const uint32_t s0 = w.fiber_s0[f];
        const float radius = w.seg_static[s0].x;
        float4 *const R = w.reaction != nullptr ? w.reaction + v0 : nullptr;
        for (int i = lane; i < n; i += 32) {
            float4 p = w.pos[v0 + i];
            p.w = w.pinned[v0 + i] ? 1.0f : 0.0f;
            P[i] = p;
            St[i] = w.vtx_static[v0 + i];
            if (R) R[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);  // clear_wall_reactions (kernels.rs:13-24)
        }
        __syncwarp();
        // find/apply_internal_corrections x constraint_iterations (Jacobi).
        for (uint32_t pass = 0; pass < sp.constraint_iterations; ++pass) {
            for (int i = lane; i < n; i += 32) {
                float4 x = P[i];
                float cx = 0.0f, cy = 0.0f, cz = 0.0f;
                if (x.w == 0.0f) {
                    if (i > 0) {
                        float4 o = P[i - 1];
                        float dx = o.x - x.x, dy = o.y - x.y, dz = o.z - x.z;
                        float length = sqrtf(dx * dx + dy * dy + dz * dz);
                        if (length > 1.0e-7f) {
                            float magnitude = 0.5f * sp.stretch_stiffness * (length - w.rest[s0 + i - 1]) / length;
                            cx += dx * magnitude;
                            cy += dy * magnitude;
                            cz += dz * magnitude;
                        }
                    }
                    if (i + 1 < n) {
                        float4 o = P[i + 1];
                        float dx = o.x - x.x, dy = o.y - x.y, dz = o.z - x.z;
                        float length = sqrtf(dx * dx + dy * dy + dz * dz);
                        if (length > 1.0e-7f) {
                            float magnitude = 0.5f * sp.stretch_stiffness * (length - w.rest[s0 + i]) / length;
                            cx += dx * magnitude;
                            cy += dy * magnitude;
                            cz += dz * magnitude;
                        }
                    }
                    if (i > 1) {
                        float4 o = P[i - 2];
                        float dx = o.x - x.x, dy = o.y - x.y, dz = o.z - x.z;
                        float length = sqrtf(dx * dx + dy * dy + dz * dz);
                        if (length > 1.0e-7f) {
                            float magnitude = 0.5f * sp.bend_stiffness * (length - St[i].y) / length;
                            cx += dx * magnitude;
                            cy += dy * magnitude;
                            cz += dz * magnitude;
                        }
                    }
                    if (i + 2 < n) {
                        float4 o = P[i + 2];
                        float dx = o.x - x.x, dy = o.y - x.y, dz = o.z - x.z;
                        float length = sqrtf(dx * dx + dy * dy + dz * dz);
                        if (length > 1.0e-7f) {
                            float magnitude = 0.5f * sp.bend_stiffness * (length - St[i].z) / length;
                            cx += dx * magnitude;
                            cy += dy * magnitude;
                            cz += dz * magnitude;
                        }
                    }
                }
                T[i] = make_float4(cx, cy, cz, 0.0f);
            }
            __syncwarp();
            for (int i = lane; i < n; i += 32) {
                float4 x = P[i];
                if (x.w != 0.0f) continue;
                float4 c = T[i];
                float e = St[i].w;
                x.x = wall_clamp_r(x.x + c.x, e, 0, g, R, i);
                x.y = wall_clamp_r(x.y + c.y, e, 1, g, R, i);
                x.z = wall_clamp_r(x.z + c.z, e, 2, g, R, i);
                P[i] = x;
            }
            __syncwarp();
        }
        // apply_contact_corrections (flexible).
        for (int i = lane; i < n; i += 32) {
            float4 x = P[i];
            float step = 0.0f;
            if (x.w == 0.0f) {
                float cx = 0.0f, cy = 0.0f, cz = 0.0f;
                if (i > 0) {
                    float4 c1 = w.corr[2 * (size_t)(s0 + i - 1) + 1];
                    cx += c1.x;
                    cy += c1.y;
                    cz += c1.z;
                }
                if (i + 1 < n) {
                    float4 c0 = w.corr[2 * (size_t)(s0 + i)];
                    cx += c0.x;
                    cy += c0.y;
                    cz += c0.z;
                }
                float length = sqrtf(cx * cx + cy * cy + cz * cz);
                if (length > sp.max_step) {
                    float scale = sp.max_step / length;
                    cx *= scale;
                    cy *= scale;
                    cz *= scale;
                }
                float e = St[i].w;
                x.x = wall_clamp_r(x.x + cx, e, 0, g, R, i);
                x.y = wall_clamp_r(x.y + cy, e, 1, g, R, i);
                x.z = wall_clamp_r(x.z + cz, e, 2, g, R, i);
                P[i] = x;
                step = sqrtf(cx * cx + cy * cy + cz * cz);
            }
            w.vertex_step[v0 + i] = step;
            smax = max(smax, __float_as_uint(fmaxf(step, 0.0f)));
        }
        __syncwarp();
        // project_fiber_curvature_in_place: forward then backward Gauss-Seidel
        // sweeps. Lanes test 32 consecutive triplets on the current
        // positions; every triplet before the first acting one is a no-op in
        // the serial order, so applying that one and resuming right after it
        // reproduces the serial sweep exactly.
        if (n >= 3) {
            const int last = n - 3;  // triplets t = 0..last: (t, t+1, t+2)
            // A pass that moves nothing leaves the positions as they were, so
            // every later pass would test the same triplets and move nothing
            // either: the sweeps end there.
            for (uint32_t sweep = 0; sweep < sp.curvature_cleanup_sweeps; ++sweep) {
                bool moved = false;
                int t0 = 0;
                while (t0 <= last) {
                    int t = t0 + lane;
                    Triplet tr;
                    bool act = t <= last &&
                               curvature_triplet_test(P, St, t, t + 1, t + 2, sp.curvature_limit_stiffness,
                                                      sp.curvature_limit_safety_margin, tr);
                    uint32_t ballot = __ballot_sync(FULL, act);
                    if (ballot == 0) {
                        t0 += 32;
                        continue;
                    }
                    moved = true;
                    int j = __ffs(ballot) - 1;
                    if (lane == j) curvature_triplet_apply(P, St, t, t + 1, t + 2, tr, g, R);
                    __syncwarp();
                    t0 += j + 1;
                }
                if (!moved) break;
                moved = false;
                t0 = last;
                while (t0 >= 0) {
                    int t = t0 - lane;
                    Triplet tr;
                    bool act = t >= 0 &&
                               curvature_triplet_test(P, St, t, t + 1, t + 2, sp.curvature_limit_stiffness,
                                                      sp.curvature_limit_safety_margin, tr);
                    uint32_t ballot = __ballot_sync(FULL, act);
                    if (ballot == 0) {
                        t0 -= 32;
                        continue;
                    }
                    moved = true;
                    int j = __ffs(ballot) - 1;
                    if (lane == j) curvature_triplet_apply(P, St, t, t + 1, t + 2, tr, g, R);
                    __syncwarp();
                    t0 -= j + 1;
                }
                if (!moved) break;
            }
        }
        __syncwarp();
        formation_targets_staged(w, f, P, n, v0, lane);
        // Write back; displacement check; next gate's curvature ratios;
        // geometry records for the next contact pass.
        for (int i = lane; i < n; i += 32) {
            float4 x = P[i];
            float4 out = make_float4(x.x, x.y, x.z, 0.0f);
            w.pos[v0 + i] = out;
            float4 r = w.ref_pos[v0 + i];
            float dx = x.x - r.x, dy = x.y - r.y, dz = x.z - r.z;
            if (dx * dx + dy * dy + dz * dz > md * md) far = true;
            if (contact_lists && contact_moved(w, v0 + i, x.x, x.y, x.z)) contact_far = true;
            if (i > 0 && i + 1 < n) {
                float maximum = St[i].x;
                if (maximum > 0.0f) {
                    float ratio = curvature_ratio_at([&](int k) { return P[k]; }, i, maximum);
                    cmax = max(cmax, __float_as_uint(fmaxf(ratio, 0.0f)));
                }
            }
            if (i + 1 < n) {
                float4 y = P[i + 1];
                float dx = y.x - x.x, dy = y.y - x.y, dz = y.z - x.z;
                const float half = 0.5f * sqrtf(dx * dx + dy * dy + dz * dz);
                w.geom[2 * (size_t)(s0 + i)] = make_float4(x.x, x.y, x.z, radius);
                w.geom[2 * (size_t)(s0 + i) + 1] = make_float4(y.x, y.y, y.z, half);
                if (contact_lists && half > w.contact_half_limit) contact_far = true;
            }
        }
        __syncwarp();
    }
    smax = warp_max_u32(smax);
    cmax = warp_max_u32(cmax);
    bool any_far = __any_sync(FULL, far);
    bool any_contact_far = __any_sync(FULL, contact_far);
    if (lane == 0) {
        if (smax) atomicMax(&w.ctl->acc[1], smax);
        if (cmax) atomicMax(&w.ctl->acc[2], cmax);
        if (any_far) w.ctl->neighbor_state[0] = 1;
        if (any_contact_far) w.ctl->contact_state[0] = 1;
    }
}

// ------------------------------------------------------ fiber update, lane per fiber

constexpr int LANES_KMAX = 8;  // vertices per lane in the cooperative passes: fibers <= 256

// Shared-memory vertex record of the lane-per-fiber update: xyz, and w =
// the vertex's curvature limit with the sign bit set when it is pinned
// (0 and -0 keep the flag for an unrestricted vertex).
__device__ inline bool lanes_pinned(float4 p) { return signbit(p.w); }
__device__ inline float lanes_limit(float4 p) { return fabsf(p.w); }

// project_curvature_triplet_in_place (kernels.rs:1165-1322) for triplet
// (t, t+1, t+2) of a staged fiber, split into the test (does the projection
// move anything?) and the move, so that a lane group can test several
// triplets at once and apply only the first that acts. A cheap test first
// rules out triplets that certainly satisfy their limit, before any IEEE
// square root or division: edge lengths and the cosine from rsqrtf (2 ulp).
// The rough limit cosine is within 2e-6 of the exact path's (whose lengths
// are correctly rounded square roots) wherever the exact path can act, and
// the rough cosine within 1e-6 of its cosine, so a 1e-5 margin never skips a
// triplet the exact computation would project; the exact path that follows
// is the reference's, operation for operation.
__device__ inline bool lanes_test(const float4 *P, int t, float stiffness, float safety_margin, Triplet &tr) {
    const float4 pp = P[t], pc = P[t + 1], pn = P[t + 2];
    const float maximum_curvature = lanes_limit(pc) * (1.0f - safety_margin);
    if (!(maximum_curvature > 0.0f)) return false;
    const float ux = pc.x - pp.x, uy = pc.y - pp.y, uz = pc.z - pp.z;
    const float vx = pn.x - pc.x, vy = pn.y - pc.y, vz = pn.z - pc.z;
    const float uu = ux * ux + uy * uy + uz * uz;
    const float vv = vx * vx + vy * vy + vz * vz;
    if (uu > 1.0e-12f && vv > 1.0e-12f) {
        const float ru = rsqrtf(uu), rv = rsqrtf(vv);
        const float rough_half = 0.25f * maximum_curvature * (uu * ru + vv * rv);
        const float rough_limit = 1.0f - 2.0f * rough_half * rough_half;
        if ((ux * vx + uy * vy + uz * vz) * (ru * rv) > rough_limit + 1.0e-5f) return false;
    }
    const float first_length = sqrtf(uu);
    const float second_length = sqrtf(vv);
    if (!(first_length > 1.0e-7f && second_length > 1.0e-7f)) return false;
    const float sine_half = 0.25f * maximum_curvature * (first_length + second_length);
    if (!(sine_half < 1.0f)) return false;
    const float minimum_cosine = 1.0f - 2.0f * sine_half * sine_half;
    const float unx = ux / first_length, uny = uy / first_length, unz = uz / first_length;
    const float vnx = vx / second_length, vny = vy / second_length, vnz = vz / second_length;
    const float cosine = clampf(unx * vnx + uny * vny + unz * vnz, -1.0f, 1.0f);
    float violation = minimum_cosine - cosine;
    const float sine = sqrtf(fmaxf(1.0f - cosine * cosine, 0.0f));
    if (violation > 0.0f && sine > 1.0e-3f) violation = (acos_f32(cosine) - acos_f32(minimum_cosine)) * sine;
    if (!(violation > 0.0f)) return false;
    tr.gux = (vnx - cosine * unx) / first_length;
    tr.guy = (vny - cosine * uny) / first_length;
    tr.guz = (vnz - cosine * unz) / first_length;
    tr.gvx = (unx - cosine * vnx) / second_length;
    tr.gvy = (uny - cosine * vny) / second_length;
    tr.gvz = (unz - cosine * vnz) / second_length;
    tr.cgx = tr.gux - tr.gvx;
    tr.cgy = tr.guy - tr.gvy;
    tr.cgz = tr.guz - tr.gvz;
    tr.pw = lanes_pinned(pp) ? 0.0f : 1.0f;
    tr.cw = lanes_pinned(pc) ? 0.0f : 1.0f;
    tr.nw = lanes_pinned(pn) ? 0.0f : 1.0f;
    const float denominator = tr.pw * (tr.gux * tr.gux + tr.guy * tr.guy + tr.guz * tr.guz) +
                              tr.cw * (tr.cgx * tr.cgx + tr.cgy * tr.cgy + tr.cgz * tr.cgz) +
                              tr.nw * (tr.gvx * tr.gvx + tr.gvy * tr.gvy + tr.gvz * tr.gvz);
    if (!(denominator > 1.0e-12f)) return false;
    tr.scale = stiffness * violation / denominator;
    return tr.pw > 0.0f || tr.cw > 0.0f || tr.nw > 0.0f;
}

__device__ inline void lanes_apply(float4 *P, int t, const Triplet &tr, float extent, const Grid &g, float4 *R) {
    const float4 pp = P[t], pc = P[t + 1], pn = P[t + 2];
    float4 a = pp, b = pc, c = pn;
    if (tr.pw > 0.0f) {
        a.x = wall_clamp_r(pp.x - tr.pw * tr.scale * tr.gux, extent, 0, g, R, t);
        a.y = wall_clamp_r(pp.y - tr.pw * tr.scale * tr.guy, extent, 1, g, R, t);
        a.z = wall_clamp_r(pp.z - tr.pw * tr.scale * tr.guz, extent, 2, g, R, t);
    }
    if (tr.cw > 0.0f) {
        b.x = wall_clamp_r(pc.x + tr.cw * tr.scale * tr.cgx, extent, 0, g, R, t + 1);
        b.y = wall_clamp_r(pc.y + tr.cw * tr.scale * tr.cgy, extent, 1, g, R, t + 1);
        b.z = wall_clamp_r(pc.z + tr.cw * tr.scale * tr.cgz, extent, 2, g, R, t + 1);
    }
    if (tr.nw > 0.0f) {
        c.x = wall_clamp_r(pn.x + tr.nw * tr.scale * tr.gvx, extent, 0, g, R, t + 2);
        c.y = wall_clamp_r(pn.y + tr.nw * tr.scale * tr.gvy, extent, 1, g, R, t + 2);
        c.z = wall_clamp_r(pn.z + tr.nw * tr.scale * tr.gvz, extent, 2, g, R, t + 2);
    }
    P[t] = a;
    P[t + 1] = b;
    P[t + 2] = c;
}

// Order of the grouped-lane update's fibers. A warp's lane groups step
// through their curvature sweeps together, so a warp takes as many rounds as
// its slowest fiber. Ranking the fibers by the rounds their sweeps take
// (most first) gives each warp fibers of about equal work: on the mid-size
// specimen's first few thousand iterations, when the update is bound by
// instruction issue, that makes it about 9 % faster than the creation order
// (descending vertex count). In a relaxed packing it makes it slower (warps
// of four of the heaviest fibers run the exact projection in nearly every
// round), so the kernel measures both: the update's blocks stamp their end
// (%globaltimer) and this kernel its own end, so every launch reads the last
// update's duration. Epochs of `period` launches go in cycles of
// ORDER_CYCLE: creation order, ranked order, creation order, then the order
// with the shorter mean update for the rest of the cycle (`ranked` forces
// the ranked order). The key is each fiber's rounds, averaged over the epochs
// (16 x rounds, the last epoch weighing 1/4).
// Any order gives the same positions: a fiber's update reads and writes only
// its own vertices and segments, and its maxima are order-free integer
// maxima. Within one rank the order is whatever the shared-memory counters
// hand out. One block of 1024 threads: a counting sort over ORDER_RANKS
// ranks (rounds at or above the last rank share it).
constexpr int ORDER_RANKS = 4096;
constexpr int ORDER_THREADS = 1024;
constexpr uint32_t ORDER_CYCLE = 10;

__device__ inline uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__global__ void __launch_bounds__(ORDER_THREADS) order_by_rounds_kernel(WorldDev w, uint32_t period, int ranked) {
    Control *const c = w.ctl;
    if (c->control[0] == 0) return;
    __shared__ uint32_t epoch_mode;  // 0: no new order, 1: creation order, 2: ranked order
    if (threadIdx.x == 0) {
        // The last update's duration counts toward the order it ran in.
        const uint64_t begin = c->order_begin, end = c->order_end;
        if (begin != 0 && end > begin) {
            c->order_ns[c->order_mode] += end - begin;
            c->order_runs[c->order_mode] += 1;
        }
        const uint32_t tick = c->order_tick;
        c->order_tick = tick + 1u;
        uint32_t mode = 0;
        if (tick % period == 0u) {
            const uint32_t epoch = tick / period % ORDER_CYCLE;
            uint32_t order = 0;  // 0 creation, 1 ranked
            if (epoch == 0) {
                for (int m = 0; m < 2; ++m) c->order_ns[m] = 0, c->order_runs[m] = 0;
            } else if (epoch == 1) {
                order = 1;
            } else if (epoch == 3) {
                // Ranked when its mean update was shorter: ns1 / runs1 < ns0 / runs0.
                const uint64_t n0 = c->order_runs[0], n1 = c->order_runs[1];
                c->order_best = n0 && n1 && c->order_ns[1] * n0 < c->order_ns[0] * n1 ? 1u : 0u;
            }
            if (epoch >= 3) order = c->order_best;
            if (ranked) order = 1;
            c->order_mode = order;
            mode = 1 + order;
        }
        epoch_mode = mode;
    }
    __syncthreads();
    const uint32_t mode = epoch_mode;
    __shared__ uint32_t start[ORDER_RANKS];
    __shared__ uint32_t warp_total[ORDER_THREADS / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (mode == 1) {
        for (uint32_t k = tid; k < w.FA; k += ORDER_THREADS) {
            const uint32_t f = w.fiber_order[k];
            const int average = (int)w.rounds_avg[f];
            w.rounds_avg[f] = (uint32_t)(average + (16 * (int)min(w.fiber_rounds[f], 1u << 20) - average) / 4);
            w.update_order[k] = f;
        }
    } else if (mode == 2) {
        // The thread that updates a fiber's average reads it back below.
        const auto rank_of = [&](uint32_t f) {
            return ORDER_RANKS - 1 - (int)min(w.rounds_avg[f] >> 4, ORDER_RANKS - 1u);
        };
        for (int i = tid; i < ORDER_RANKS; i += ORDER_THREADS) start[i] = 0;
        __syncthreads();
        for (uint32_t k = tid; k < w.FA; k += ORDER_THREADS) {
            const uint32_t f = w.fiber_order[k];
            const int average = (int)w.rounds_avg[f];
            w.rounds_avg[f] = (uint32_t)(average + (16 * (int)min(w.fiber_rounds[f], 1u << 20) - average) / 4);
            atomicAdd(&start[rank_of(f)], 1u);
        }
        __syncthreads();
        // Exclusive scan of the counts: ORDER_RANKS / ORDER_THREADS per thread.
        constexpr int PER = ORDER_RANKS / ORDER_THREADS;
        uint32_t count[PER], sum = 0;
#pragma unroll
        for (int j = 0; j < PER; ++j) sum += (count[j] = start[tid * PER + j]);
        uint32_t inclusive = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(FULL, inclusive, o);
            if (lane >= o) inclusive += v;
        }
        if (lane == 31) warp_total[warp] = inclusive;
        __syncthreads();
        if (warp == 0) {
            uint32_t t = warp_total[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(FULL, t, o);
                if (lane >= o) t += v;
            }
            warp_total[lane] = t;
        }
        __syncthreads();
        uint32_t base = inclusive - sum + (warp > 0 ? warp_total[warp - 1] : 0u);
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            start[tid * PER + j] = base;
            base += count[j];
        }
        __syncthreads();
        for (uint32_t k = tid; k < w.FA; k += ORDER_THREADS) {
            const uint32_t f = w.fiber_order[k];
            w.update_order[atomicAdd(&start[rank_of(f)], 1u)] = f;
        }
    }
    __syncthreads();
    // The update starts when this kernel ends.
    if (threadIdx.x == 0) {
        c->order_end = 0;
        c->order_begin = global_ns();
    }
}

// Everything after the gate for 32/LPF fibers per warp (fibers of at most
// 256 vertices), LPF lanes per fiber in the curvature sweeps. The warp stages
// the fibers in shared memory and runs the internal stretch/bend passes
// (kernels.rs:1027-1163, :1417-1453) and the contact step (:1455-1537)
// cooperatively, one fiber at a time. Then each group of LPF lanes runs
// project_fiber_curvature_in_place (:1324-1415) on its fiber: the group tests
// LPF consecutive triplets on the current positions; every triplet before
// the first acting one is a no-op in the serial order, so applying that one
// and resuming right after it reproduces the serial sweep exactly. Last the
// warp writes the fibers back with the displacement check
// (neighbor.rs:446-465) and the next gate's curvature and step maxima
// (:925-980, :95-127).
// In an arena (A) each fiber takes its specimen's grid and skin, fibers of
// stopped specimens are skipped, and the maxima and flags go to each
// fiber's specimen.
// FM compiles in the formation work (wall reactions, layer and vertex
// targets); without it the kernel carries none of it.
template <int LPF, bool A = false, bool FM = false>
__global__ void __launch_bounds__(128, 8) fiber_lanes_kernel(WorldDev w, StepParams sp, int stride) {
    constexpr int FPW = 32 / LPF;  // fibers per warp
    if (w.ctl->control[0] == 0) return;
    extern __shared__ float4 lanes_smem_all[];
    // Each warp works alone on its own fibers; a block holds up to 4 warps
    // only so that 32 warps fit on an SM (at most 32 blocks are resident).
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    float4 *const lanes_smem = lanes_smem_all + (size_t)wib * FPW * stride;
    const int group = lane / LPF, gl = lane % LPF;
    const uint32_t gmask = LPF == 32 ? FULL : (((1u << LPF) - 1u) << (group * LPF));
    uint32_t smax = 0, cmax = 0;
    bool far = false;
    bool contact_far = false;
    const bool contact_lists = w.contact_skin > 0.0f;
    for (uint32_t batch = blockIdx.x * wpb + wib; batch * FPW < w.FA; batch += gridDim.x * wpb) {
        const uint32_t slot = batch * FPW + group;
        uint32_t mine = slot < w.FA ? w.update_order[slot] : TGL_NONE;
        if (A && mine != TGL_NONE && ctl_of<A>(w, spec_of_fiber<A>(w, mine))->control[0] == 0) mine = TGL_NONE;
        for (int j = 0; j < FPW; ++j) {
            const uint32_t f = __shfl_sync(FULL, mine, j * LPF);
            if (f == TGL_NONE) continue;
            const uint32_t fspec = spec_of_fiber<A>(w, f);
            const Grid &g = grid_of<A>(w, fspec);
            const uint2 span = w.fiber_vspan[f];
            const uint32_t v0 = span.x;
            const int n = (int)span.y;
            const uint32_t s0 = w.fiber_s0[f];
            const float extent = w.seg_static[s0].x;
            float4 *P = lanes_smem + (size_t)j * stride;
            float4 *const R = FM && w.reaction != nullptr ? w.reaction + v0 : nullptr;
            for (int i = lane; i < n; i += 32) {
                float4 p = w.pos[v0 + i];
                const float limit = w.vtx_static[v0 + i].x;
                p.w = w.pinned[v0 + i] ? -limit : limit;
                if (w.pinned[v0 + i] && limit == 0.0f) p.w = -0.0f;
                P[i] = p;
                if (R) R[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);  // clear_wall_reactions (kernels.rs:13-24)
            }
            __syncwarp();
            // find/apply_internal_corrections x constraint_iterations (Jacobi).
            for (uint32_t pass = 0; pass < sp.constraint_iterations; ++pass) {
                float cxs[LANES_KMAX], cys[LANES_KMAX], czs[LANES_KMAX];
#pragma unroll
                for (int k = 0; k < LANES_KMAX; ++k) {
                    const int i = lane + 32 * k;
                    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
                    if (i < n) {
                        const float4 x = P[i];
                        if (!lanes_pinned(x)) {
                            if (i > 0) {
                                float4 o = P[i - 1];
                                float dx = o.x - x.x, dy = o.y - x.y, dz = o.z - x.z;
                                float length = sqrtf(dx * dx + dy * dy + dz * dz);
                                if (length > 1.0e-7f) {
                                    float magnitude = 0.5f * sp.stretch_stiffness * (length - w.rest[s0 + i - 1]) / length;
                                    cx += dx * magnitude;
                                    cy += dy * magnitude;
                                    cz += dz * magnitude;
                                }
                            }
                            if (i + 1 < n) {
                                float4 o = P[i + 1];
                                float dx = o.x - x.x, dy = o.y - x.y, dz = o.z - x.z;
                                float length = sqrtf(dx * dx + dy * dy + dz * dz);
                                if (length > 1.0e-7f) {
                                    float magnitude = 0.5f * sp.stretch_stiffness * (length - w.rest[s0 + i]) / length;
                                    cx += dx * magnitude;
                                    cy += dy * magnitude;
                                    cz += dz * magnitude;
                                }
                            }
                            if (i > 1) {
                                float4 o = P[i - 2];
                                float dx = o.x - x.x, dy = o.y - x.y, dz = o.z - x.z;
                                float length = sqrtf(dx * dx + dy * dy + dz * dz);
                                if (length > 1.0e-7f) {
                                    float magnitude = 0.5f * sp.bend_stiffness * (length - w.vtx_static[v0 + i].y) / length;
                                    cx += dx * magnitude;
                                    cy += dy * magnitude;
                                    cz += dz * magnitude;
                                }
                            }
                            if (i + 2 < n) {
                                float4 o = P[i + 2];
                                float dx = o.x - x.x, dy = o.y - x.y, dz = o.z - x.z;
                                float length = sqrtf(dx * dx + dy * dy + dz * dz);
                                if (length > 1.0e-7f) {
                                    float magnitude = 0.5f * sp.bend_stiffness * (length - w.vtx_static[v0 + i].z) / length;
                                    cx += dx * magnitude;
                                    cy += dy * magnitude;
                                    cz += dz * magnitude;
                                }
                            }
                        }
                    }
                    cxs[k] = cx;
                    cys[k] = cy;
                    czs[k] = cz;
                }
                __syncwarp();
#pragma unroll
                for (int k = 0; k < LANES_KMAX; ++k) {
                    const int i = lane + 32 * k;
                    if (i < n) {
                        float4 x = P[i];
                        if (!lanes_pinned(x)) {
                            x.x = wall_clamp_r(x.x + cxs[k], extent, 0, g, R, i);
                            x.y = wall_clamp_r(x.y + cys[k], extent, 1, g, R, i);
                            x.z = wall_clamp_r(x.z + czs[k], extent, 2, g, R, i);
                            P[i] = x;
                        }
                    }
                }
                __syncwarp();
            }
            // apply_contact_corrections (flexible).
            for (int i = lane; i < n; i += 32) {
                float4 x = P[i];
                float step = 0.0f;
                if (!lanes_pinned(x)) {
                    float cx = 0.0f, cy = 0.0f, cz = 0.0f;
                    if (i > 0) {
                        float4 c1 = w.corr[2 * (size_t)(s0 + i - 1) + 1];
                        cx += c1.x;
                        cy += c1.y;
                        cz += c1.z;
                    }
                    if (i + 1 < n) {
                        float4 c0 = w.corr[2 * (size_t)(s0 + i)];
                        cx += c0.x;
                        cy += c0.y;
                        cz += c0.z;
                    }
                    float length = sqrtf(cx * cx + cy * cy + cz * cz);
                    if (length > sp.max_step) {
                        float scale = sp.max_step / length;
                        cx *= scale;
                        cy *= scale;
                        cz *= scale;
                    }
                    x.x = wall_clamp_r(x.x + cx, extent, 0, g, R, i);
                    x.y = wall_clamp_r(x.y + cy, extent, 1, g, R, i);
                    x.z = wall_clamp_r(x.z + cz, extent, 2, g, R, i);
                    P[i] = x;
                    step = sqrtf(cx * cx + cy * cy + cz * cz);
                }
                w.vertex_step[v0 + i] = step;
                smax = max(smax, __float_as_uint(fmaxf(step, 0.0f)));
            }
            __syncwarp();
            if (A) {
                smax = warp_max_u32(smax);
                if (lane == 0 && smax) atomicMax(&ctl_of<A>(w, fspec)->acc[1], smax);
                smax = 0;
            }
        }
        // Curvature Gauss-Seidel, LPF lanes per fiber, forward then backward.
        // The warp's groups step together: every round each unfinished group
        // tests LPF triplets of its own fiber, one warp-wide ballot gives
        // every group its bits, and each group applies its own first acting
        // triplet. A group's sequence of tests and moves is exactly its
        // serial sweep; stepping together only shares the instruction issue
        // between the groups. A pass that moves nothing ends its group's
        // sweeps (every later pass would test the same positions).
        {
            const Grid &g = grid_of<A>(w, mine != TGL_NONE ? spec_of_fiber<A>(w, mine) : 0u);
            const int last = mine != TGL_NONE ? (int)w.fiber_vspan[mine].y - 3 : -1;
            const float extent = mine != TGL_NONE ? w.seg_static[w.fiber_s0[mine]].x : 0.0f;
            float4 *const R =
                FM && mine != TGL_NONE && w.reaction != nullptr ? w.reaction + w.fiber_vspan[mine].x : nullptr;
            float4 *P = lanes_smem + (size_t)group * stride;
            bool done = mine == TGL_NONE || sp.curvature_cleanup_sweeps == 0;
            bool forward = true, moved = false;
            uint32_t sweep = 0, rounds = 0;
            int t0 = 0;
            while (__any_sync(FULL, !done)) {
                rounds += done ? 0u : 1u;
                Triplet tr;
                const int t = forward ? t0 + gl : t0 - gl;
                const bool act = !done && (forward ? t <= last : t >= 0) &&
                                 lanes_test(P, t, sp.curvature_limit_stiffness, sp.curvature_limit_safety_margin, tr);
                const uint32_t ballot = __ballot_sync(FULL, act);
                const uint32_t bits = LPF == 32 ? ballot : (ballot >> (group * LPF)) & ((1u << LPF) - 1u);
                if (!done) {
                    if (bits) {
                        const int first = __ffs(bits) - 1;
                        if (gl == first) lanes_apply(P, t, tr, extent, g, R);
                        moved = true;
                        t0 = forward ? t0 + first + 1 : t0 - first - 1;
                    } else {
                        t0 = forward ? t0 + LPF : t0 - LPF;
                    }
                    if (forward ? t0 > last : t0 < 0) {  // the pass is over
                        if (!moved) {
                            done = true;
                        } else if (forward) {
                            forward = false;
                            moved = false;
                            t0 = last;
                        } else {
                            moved = false;
                            forward = true;
                            t0 = 0;
                            done = ++sweep >= sp.curvature_cleanup_sweeps;
                        }
                    }
                }
                __syncwarp();
            }
            // The rounds this fiber's sweeps took rank it for the next updates
            // (a fiber of a stopped specimen took none).
            if (!A && w.fiber_rounds != nullptr && mine != TGL_NONE && gl == 0) w.fiber_rounds[mine] = rounds;
            if (A && w.fiber_rounds != nullptr && gl == 0 && slot < w.FA) w.fiber_rounds[w.update_order[slot]] = rounds;
        }
        __syncwarp();
        // Write back; displacement check; next gate's curvature ratios;
        // geometry records for the next contact pass.
        for (int j = 0; j < FPW; ++j) {
            const uint32_t f = __shfl_sync(FULL, mine, j * LPF);
            if (f == TGL_NONE) continue;
            const uint32_t fspec = spec_of_fiber<A>(w, f);
            const float md = 0.5f * skin_of<A>(w, fspec);
            const uint2 span = w.fiber_vspan[f];
            const uint32_t v0 = span.x;
            const int n = (int)span.y;
            const uint32_t s0 = w.fiber_s0[f];
            const float radius = w.seg_static[s0].x;
            float4 *P = lanes_smem + (size_t)j * stride;
            if (FM) formation_targets_staged(w, f, P, n, v0, lane);
            for (int i = lane; i < n; i += 32) {
                const float4 x = P[i];
                w.pos[v0 + i] = make_float4(x.x, x.y, x.z, 0.0f);
                const float4 r = w.ref_pos[v0 + i];
                const float dx = x.x - r.x, dy = x.y - r.y, dz = x.z - r.z;
                if (dx * dx + dy * dy + dz * dz > md * md) far = true;
                if (contact_lists && contact_moved(w, v0 + i, x.x, x.y, x.z)) contact_far = true;
                if (i > 0 && i + 1 < n) {
                    const float maximum = lanes_limit(x);
                    if (maximum > 0.0f) {
                        const float ratio = curvature_ratio_at([&](int k) { return P[k]; }, i, maximum);
                        cmax = max(cmax, __float_as_uint(fmaxf(ratio, 0.0f)));
                    }
                }
                if (i + 1 < n) {
                    const float4 y = P[i + 1];
                    const float ex = y.x - x.x, ey = y.y - x.y, ez = y.z - x.z;
                    const float half = 0.5f * sqrtf(ex * ex + ey * ey + ez * ez);
                    w.geom[2 * (size_t)(s0 + i)] = make_float4(x.x, x.y, x.z, radius);
                    w.geom[2 * (size_t)(s0 + i) + 1] = make_float4(y.x, y.y, y.z, half);
                    if (contact_lists && half > w.contact_half_limit) contact_far = true;
                }
            }
            if (A) {
                cmax = warp_max_u32(cmax);
                const bool fiber_far = __any_sync(FULL, far);
                const bool fiber_contact_far = __any_sync(FULL, contact_far);
                if (lane == 0) {
                    if (cmax) atomicMax(&ctl_of<A>(w, fspec)->acc[2], cmax);
                    if (fiber_far) flag_rebuild<A>(w, fspec);
                    if (fiber_contact_far) flag_refresh<A>(w, fspec);
                }
                cmax = 0;
                far = false;
                contact_far = false;
            }
        }
        __syncwarp();
    }
    // The end of the update, for the fiber-order choice.
    if (lane == 0) atomicMax(&w.ctl->order_end, (unsigned long long)global_ns());
    if (A) return;
    smax = warp_max_u32(smax);
    cmax = warp_max_u32(cmax);
    const bool any_far = __any_sync(FULL, far);
    const bool any_contact_far = __any_sync(FULL, contact_far);
    if (lane == 0) {
        if (smax) atomicMax(&w.ctl->acc[1], smax);
        if (cmax) atomicMax(&w.ctl->acc[2], cmax);
        if (any_far) w.ctl->neighbor_state[0] = 1;
        if (any_contact_far) w.ctl->contact_state[0] = 1;
    }
}

// ------------------------------------------------------ rigid translation

// apply_rigid_contact_corrections (kernels.rs:1539-1646) for one fiber per
// warp: the fiber moves as a whole by its deepest segment's mean end
// correction (the first of equal maxima, as the serial loop picks it),
// capped at max_step and clamped on walled axes so that every vertex stays
// inside; pinned vertices move with it, as in the reference. Then the same
// write-back as the flexible update: geometry records, the displacement
// checks and the next gate's step and curvature maxima.
template <bool A>
__global__ void __launch_bounds__(256) rigid_kernel(WorldDev w, StepParams sp) {
    if (w.ctl->control[0] == 0) return;
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const bool contact_lists = w.contact_skin > 0.0f;
    uint32_t smax = 0, cmax = 0;
    bool far = false, contact_far = false;
    for (uint32_t k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); k < w.FA; k += warps) {
        const uint32_t f = w.fiber_order[k];
        const uint32_t spec = spec_of_fiber<A>(w, f);
        if (A && ctl_of<A>(w, spec)->control[0] == 0) continue;
        const Grid &g = grid_of<A>(w, spec);
        const uint2 span = w.fiber_vspan[f];
        const uint32_t v0 = span.x, n = span.y, m = n - 1, s0 = w.fiber_s0[f];
        // Deepest segment: each lane keeps its first strict maximum, then the
        // warp takes the largest, the lowest segment on ties.
        float best = 0.0f, bx = 0.0f, by = 0.0f, bz = 0.0f;
        uint32_t best_index = 0xFFFFFFFFu;
        for (uint32_t local = lane; local < m; local += 32) {
            const float4 c0 = w.corr[2 * (size_t)(s0 + local)], c1 = w.corr[2 * (size_t)(s0 + local) + 1];
            const float cx = 0.5f * (c0.x + c1.x), cy = 0.5f * (c0.y + c1.y), cz = 0.5f * (c0.z + c1.z);
            const float squared = cx * cx + cy * cy + cz * cz;
            if (squared > best) {
                best = squared;
                best_index = local;
                bx = cx;
                by = cy;
                bz = cz;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const float ob = __shfl_xor_sync(FULL, best, o);
            const uint32_t oi = __shfl_xor_sync(FULL, best_index, o);
            const float ox = __shfl_xor_sync(FULL, bx, o), oy = __shfl_xor_sync(FULL, by, o),
                        oz = __shfl_xor_sync(FULL, bz, o);
            if (ob > best || (ob == best && oi < best_index)) {
                best = ob;
                best_index = oi;
                bx = ox;
                by = oy;
                bz = oz;
            }
        }
        float tx = bx, ty = by, tz = bz;
        const float length = sqrtf(tx * tx + ty * ty + tz * tz);
        if (length > sp.max_step) {
            const float scale = sp.max_step / length;
            tx *= scale;
            ty *= scale;
            tz *= scale;
        }
        // The translation that keeps every vertex inside the walls.
        float lo[3] = {-INFINITY, -INFINITY, -INFINITY}, hi[3] = {INFINITY, INFINITY, INFINITY};
        for (uint32_t local = lane; local < n; local += 32) {
            const float4 x = w.pos[v0 + local];
            const float extent = w.vtx_static[v0 + local].w;
            const float xs[3] = {x.x, x.y, x.z};
            for (int a = 0; a < 3; ++a) {
                lo[a] = fmaxf(lo[a], g.lower[a] + extent - xs[a]);
                hi[a] = fminf(hi[a], g.upper[a] - extent - xs[a]);
            }
        }
        for (int a = 0; a < 3; ++a)
            for (int o = 16; o > 0; o >>= 1) {
                lo[a] = fmaxf(lo[a], __shfl_xor_sync(FULL, lo[a], o));
                hi[a] = fminf(hi[a], __shfl_xor_sync(FULL, hi[a], o));
            }
        float t[3] = {tx, ty, tz};
        for (int a = 0; a < 3; ++a)
            if (!g.periodic[a]) t[a] = t[a] < lo[a] ? lo[a] : (t[a] > hi[a] ? hi[a] : t[a]);
        const float applied = sqrtf(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        // The wall's share of the translation, spread over the vertices
        // (the reactions were cleared at the step's start).
        float4 *const R = !A && w.reaction != nullptr ? w.reaction + v0 : nullptr;
        const float4 reaction = make_float4((tx - t[0]) / (float)n, (ty - t[1]) / (float)n, (tz - t[2]) / (float)n, 0.0f);
        for (uint32_t local = lane; local < n; local += 32) {
            float4 x = w.pos[v0 + local];
            x.x += t[0];
            x.y += t[1];
            x.z += t[2];
            w.pos[v0 + local] = x;
            w.vertex_step[v0 + local] = applied;
            if (R) R[local] = reaction;
        }
        __syncwarp();
        if (!A) formation_targets_staged(w, f, w.pos + v0, (int)n, v0, lane);
        smax = max(smax, __float_as_uint(fmaxf(applied, 0.0f)));
        const float md = 0.5f * skin_of<A>(w, spec);
        const float radius = w.seg_static[s0].x;
        const float4 *P = w.pos + v0;
        for (uint32_t i = lane; i < n; i += 32) {
            const float4 x = P[i];
            const float4 r = w.ref_pos[v0 + i];
            const float dx = x.x - r.x, dy = x.y - r.y, dz = x.z - r.z;
            if (dx * dx + dy * dy + dz * dz > md * md) far = true;
            if (contact_lists && contact_moved(w, v0 + i, x.x, x.y, x.z)) contact_far = true;
            if (i > 0 && i + 1 < n) {
                const float maximum = w.vtx_static[v0 + i].x;
                if (maximum > 0.0f) {
                    const float ratio = curvature_ratio_at([&](int k) { return P[k]; }, (int)i, maximum);
                    cmax = max(cmax, __float_as_uint(fmaxf(ratio, 0.0f)));
                }
            }
            if (i + 1 < n) {
                const float4 y = P[i + 1];
                const float ex = y.x - x.x, ey = y.y - x.y, ez = y.z - x.z;
                const float half = 0.5f * sqrtf(ex * ex + ey * ey + ez * ez);
                w.geom[2 * (size_t)(s0 + i)] = make_float4(x.x, x.y, x.z, radius);
                w.geom[2 * (size_t)(s0 + i) + 1] = make_float4(y.x, y.y, y.z, half);
                if (contact_lists && half > w.contact_half_limit) contact_far = true;
            }
        }
        __syncwarp();
        if (A) {
            cmax = warp_max_u32(cmax);
            const bool fiber_far = __any_sync(FULL, far);
            const bool fiber_contact_far = __any_sync(FULL, contact_far);
            if (lane == 0) {
                if (smax) atomicMax(&ctl_of<A>(w, spec)->acc[1], smax);
                if (cmax) atomicMax(&ctl_of<A>(w, spec)->acc[2], cmax);
                if (fiber_far) flag_rebuild<A>(w, spec);
                if (fiber_contact_far) flag_refresh<A>(w, spec);
            }
            smax = cmax = 0;
            far = false;
            contact_far = false;
        }
    }
    if (A) return;
    smax = warp_max_u32(smax);
    cmax = warp_max_u32(cmax);
    const bool any_far = __any_sync(FULL, far);
    const bool any_contact_far = __any_sync(FULL, contact_far);
    if (lane == 0) {
        if (smax) atomicMax(&w.ctl->acc[1], smax);
        if (cmax) atomicMax(&w.ctl->acc[2], cmax);
        if (any_far) w.ctl->neighbor_state[0] = 1;
        if (any_contact_far) w.ctl->contact_state[0] = 1;
    }
}

// ---------------------------------------------------------------- host copies

// Raises *flag when any of the n staged floats is not finite (all exponent
// bits set: an infinity or a NaN).
__global__ void stage_nonfinite_kernel(const float *xyz, size_t n, unsigned int *flag) {
    bool bad = false;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        bad |= (__float_as_uint(xyz[i]) & 0x7F800000u) == 0x7F800000u;
    if (__any_sync(FULL, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

__global__ void positions_from_stage_kernel(WorldDev w) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < w.V; v += gridDim.x * blockDim.x)
        w.pos[v] = make_float4(w.xyz_stage[3 * (size_t)v], w.xyz_stage[3 * (size_t)v + 1],
                               w.xyz_stage[3 * (size_t)v + 2], 0.0f);
}

__global__ void refresh_geometry_kernel(WorldDev w) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < w.S; s += gridDim.x * blockDim.x) {
        uint32_t v0 = w.seg_v0[s];
        float4 a = w.pos[v0], b = w.pos[v0 + 1];
        float dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
        w.geom[2 * (size_t)s] = make_float4(a.x, a.y, a.z, w.seg_static[s].x);
        w.geom[2 * (size_t)s + 1] = make_float4(b.x, b.y, b.z, 0.5f * sqrtf(dx * dx + dy * dy + dz * dz));
    }
}

__global__ void positions_to_stage_kernel(WorldDev w) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < w.V; v += gridDim.x * blockDim.x) {
        float4 p = w.pos[v];
        w.xyz_stage[3 * (size_t)v] = p.x;
        w.xyz_stage[3 * (size_t)v + 1] = p.y;
        w.xyz_stage[3 * (size_t)v + 2] = p.z;
    }
}

__global__ void corrections_to_stage_kernel(WorldDev w, float *corr6, float *pen) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < w.S; s += gridDim.x * blockDim.x) {
        float4 a = w.corr[2 * (size_t)s], b = w.corr[2 * (size_t)s + 1];
        corr6[6 * (size_t)s] = a.x;
        corr6[6 * (size_t)s + 1] = a.y;
        corr6[6 * (size_t)s + 2] = a.z;
        corr6[6 * (size_t)s + 3] = b.x;
        corr6[6 * (size_t)s + 4] = b.y;
        corr6[6 * (size_t)s + 5] = b.z;
        pen[s] = a.w;
    }
}

int grid_for(uint64_t n, int threads, int cap) {
    uint64_t blocks = (n + threads - 1) / threads;
    if (blocks < 1) blocks = 1;
    if (blocks > (uint64_t)cap) blocks = cap;
    return (int)blocks;
}

}  // namespace

// A kernel's largest dynamic shared memory is a process-wide attribute of
// the function, shared by every world: raise it when a plan needs more, and
// never lower it below what another world (or an earlier plan of this one,
// whose captured graphs may still launch) needs.
template <typename Kernel>
static void allow_dynamic_smem(Kernel kernel, size_t bytes) {
    static std::mutex lock;
    static std::map<const void *, size_t> granted;
    const void *key = reinterpret_cast<const void *>(kernel);
    std::lock_guard<std::mutex> guard(lock);
    size_t &current = granted[key];
    if (bytes <= current) return;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess)
        current = bytes;
}

void plan_launches(const WorldDev &w, LaunchPlan &lp) {
    int device = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&lp.num_sms, cudaDevAttrMultiProcessorCount, device);
    if (lp.num_sms <= 0) lp.num_sms = 148;
    lp.contact_group = 32;
    // Absolute margin of the line-distance bound: 4e-6 of the largest box
    // edge, above the f32 rounding of coordinates that are unwrapped by up to
    // a box length either side.
    {
        float edge = 0.0f;
        for (int a = 0; a < 3; ++a) edge = std::max(edge, w.grid.length[a]);
        lp.line_eps = 4.0e-6f * edge;
    }
    // Three 256-thread blocks are resident per SM at the kernel's launch
    // bounds; fewer leave room to the kernels around it.
    const int contact_per_sm = lp.tune_contact_per_sm >= 1 && lp.tune_contact_per_sm <= 3 ? lp.tune_contact_per_sm : 3;
    lp.contact_blocks = grid_for((w.NS + 31) / 32, CONTACT_WARPS, lp.num_sms * contact_per_sm);
    // Update kernel: as many warps per block as fit 96 KB of staged fibers.
    size_t per_warp = (size_t)3 * w.max_fiber * sizeof(float4);
    int warps = 8;
    while (warps > 1 && per_warp * warps > 96 * 1024) warps >>= 1;
    lp.fiber_warps = warps;
    lp.fiber_smem = per_warp * warps;
    lp.fiber_blocks = grid_for(w.FA, warps, 1 << 20);
    // Lane-per-fiber update for fibers of at most 32 * LANES_KMAX vertices:
    // 32 fibers per warp, an odd float4 stride per fiber so that the lanes'
    // same-index accesses spread over the banks.
    if (const char *env = std::getenv("TGL_LANES_PER_FIBER")) lp.lanes_per_fiber = std::atoi(env);
    if (lp.tune_lanes) lp.lanes_per_fiber = lp.tune_lanes;
    if (lp.lanes_per_fiber != 2 && lp.lanes_per_fiber != 4 && lp.lanes_per_fiber != 8 && lp.lanes_per_fiber != 32)
        lp.lanes_per_fiber = 8;
    const int fpw = 32 / lp.lanes_per_fiber;
    lp.lanes_stride = (int)(w.max_fiber | 1u);
    lp.lanes_smem = (size_t)fpw * lp.lanes_stride * sizeof(float4);
    lp.fiber_lanes = w.max_fiber <= 32u * LANES_KMAX && lp.lanes_smem <= 200 * 1024;
    // Warps per block: 4 where their staged fibers fit, so that 32 warps
    // (the register file at the kernel's 64 registers, and 8 blocks of 4
    // warps) are resident per SM instead of the 28 that one-warp blocks get
    // (their shared memory and 1 KB reserve per block run out first); the
    // long tail of the grid then runs on a full SM.
    const int wpb_max = lp.tune_wpb == 1 || lp.tune_wpb == 2 ? lp.tune_wpb : 4;
    lp.lanes_wpb = 1;
    while (lp.lanes_wpb < wpb_max && lp.lanes_smem * (size_t)(2 * lp.lanes_wpb) <= 200 * 1024) lp.lanes_wpb *= 2;
    const uint32_t lane_warps = (w.FA + fpw - 1) / fpw;
    lp.lanes_blocks = (int)((lane_warps + lp.lanes_wpb - 1) / lp.lanes_wpb);
    // The update's fiber order is chosen in epochs of 16 launches where
    // there are enough fibers for the choice to pay for its kernel
    // (TGL_UPDATE_ORDER_PERIOD sets the epoch; 0 keeps the creation order).
    lp.order_period = w.FA >= 4096u ? 16 : 0;
    if (const char *env = std::getenv("TGL_UPDATE_ORDER_PERIOD")) lp.order_period = std::max(std::atoi(env), 0);
    if (!lp.fiber_lanes || w.fiber_rounds == nullptr) lp.order_period = 0;
    // TGL_UPDATE_ORDER_RANKED=1 keeps the ranked order instead of timing both.
    lp.order_ranked = 0;
    if (const char *env = std::getenv("TGL_UPDATE_ORDER_RANKED")) lp.order_ranked = std::atoi(env) != 0;
    lp.contact_lists = w.contact_skin > 0.0f;
    lp.build_ch = lp.tune_build_ch >= 512 && lp.tune_build_ch <= 4096 ? lp.tune_build_ch : lp.arena ? 1536 : 3072;
    lp.build_smem = (size_t)lp.build_ch * (sizeof(float4) + sizeof(uint32_t));
    // The sphere pre-test needs >= 3 cells on every periodic axis (see
    // rb_build_kernel); its absolute margin is 1e-6 of the largest box edge.
    lp.build_prefilter = 1;
    float edge = 0.0f;
    for (int a = 0; a < 3; ++a) {
        if (w.grid.periodic[a] && w.grid.cells[a] < 3) lp.build_prefilter = 0;
        edge = std::max(edge, w.grid.length[a]);
    }
    lp.build_sphere_eps = 1.0e-6f * edge;
    int sw = 8;
    while (sw > 1 && (size_t)sw * w.block * 4 > 96 * 1024) sw >>= 1;
    lp.sort_warps = sw;
    lp.sort_smem = (size_t)sw * w.block * 4;
    allow_dynamic_smem(fiber_kernel, std::max<size_t>(lp.fiber_smem, 1));
    if (lp.fiber_lanes) {
        const size_t smem = lp.lanes_smem * lp.lanes_wpb;
        const auto allow = [smem](auto kernel) { allow_dynamic_smem(kernel, smem); };
        allow(fiber_lanes_kernel<2, false, false>);
        allow(fiber_lanes_kernel<4, false, false>);
        allow(fiber_lanes_kernel<8, false, false>);
        allow(fiber_lanes_kernel<32, false, false>);
        allow(fiber_lanes_kernel<2, true, false>);
        allow(fiber_lanes_kernel<4, true, false>);
        allow(fiber_lanes_kernel<8, true, false>);
        allow(fiber_lanes_kernel<32, true, false>);
        allow(fiber_lanes_kernel<2, false, true>);
        allow(fiber_lanes_kernel<4, false, true>);
        allow(fiber_lanes_kernel<8, false, true>);
        allow(fiber_lanes_kernel<32, false, true>);
    }
    allow_dynamic_smem(rb_build_kernel<false>, lp.build_smem);
    allow_dynamic_smem(rb_build_kernel<true>, lp.build_smem);
    allow_dynamic_smem(rb_sort_lists_kernel<false>, std::max<size_t>(lp.sort_smem, 1));
    allow_dynamic_smem(rb_sort_lists_kernel<true>, std::max<size_t>(lp.sort_smem, 1));
}

int launch_begin_batch(const WorldDev &w, const LaunchPlan &lp, cudaStream_t st) {
    if (lp.arena)
        begin_batch_kernel<true><<<1, 256, 0, st>>>(w);
    else
        begin_batch_kernel<false><<<1, 32, 0, st>>>(w);
    return 1;
}

int launch_flag_displacement(const WorldDev &w, const LaunchPlan &lp, cudaStream_t st) {
    if (lp.arena)
        flag_displacement_kernel<true><<<grid_for(w.V, 256, 1 << 30), 256, 0, st>>>(w);
    else
        flag_displacement_kernel<false><<<grid_for(w.V, 256, 1 << 30), 256, 0, st>>>(w);
    return 1;
}

int launch_measure_start(const WorldDev &w, const LaunchPlan &lp, cudaStream_t st) {
    if (lp.arena)
        measure_start_kernel<true><<<grid_for(w.F, 8, lp.num_sms * 16), 256, 0, st>>>(w);
    else
        measure_start_kernel<false><<<grid_for(w.F, 8, lp.num_sms * 16), 256, 0, st>>>(w);
    return 1;
}

int launch_request_rebuild(const WorldDev &w, const LaunchPlan &lp, cudaStream_t st) {
    if (lp.arena)
        request_rebuild_kernel<true><<<1, 256, 0, st>>>(w);
    else
        request_rebuild_kernel<false><<<1, 32, 0, st>>>(w);
    return 1;
}

template <bool A>
static void enqueue_rebuild(const WorldDev &w, const LaunchPlan &lp, cudaStream_t st) {
    const int cap = lp.num_sms * 16;
    rb_clear_kernel<A><<<grid_for(w.C, 256, cap), 256, 0, st>>>(w);
    rb_count_kernel<A><<<grid_for(w.S, 256, cap), 256, 0, st>>>(w);
    rb_scan_kernel<A><<<A ? (int)w.P : 1, 1024, 0, st>>>(w);
    rb_scatter_kernel<A><<<grid_for(w.S, 256, cap), 256, 0, st>>>(w);
    rb_sort_cells_kernel<A><<<grid_for(w.C, 8, cap), 256, 8 * CELL_SORT_CAP * sizeof(uint32_t), st>>>(w);
    rb_gather_kernel<A><<<grid_for(w.S, 256, cap), 256, 0, st>>>(w);
    rb_boxes_kernel<A><<<grid_for(w.C, 8, cap), 256, 0, st>>>(w);
    rb_build_kernel<A><<<(int)std::min<uint64_t>(w.C, (uint64_t)lp.num_sms * 64), 256, lp.build_smem, st>>>(
        w, lp.build_ch, lp.build_prefilter, lp.build_sphere_eps);
    rb_sort_lists_kernel<A><<<grid_for(w.S, lp.sort_warps, cap), lp.sort_warps * 32, lp.sort_smem, st>>>(w);
    rb_snapshot_kernel<A><<<grid_for(w.V, 256, cap), 256, 0, st>>>(w);
    rb_finish_kernel<A><<<1, A ? 256 : 32, 0, st>>>(w);
}

int launch_cell_list(const WorldDev &w, const LaunchPlan &lp, cudaStream_t st) {
    const int cap = lp.num_sms * 16;
    rb_clear_kernel<false><<<grid_for(w.C, 256, cap), 256, 0, st>>>(w);
    rb_count_kernel<false><<<grid_for(w.S, 256, cap), 256, 0, st>>>(w);
    rb_scan_kernel<false><<<1, 1024, 0, st>>>(w);
    rb_scatter_kernel<false><<<grid_for(w.S, 256, cap), 256, 0, st>>>(w);
    rb_sort_cells_kernel<false><<<grid_for(w.C, 8, cap), 256, 8 * CELL_SORT_CAP * sizeof(uint32_t), st>>>(w);
    return 5;
}

int launch_rebuild(const WorldDev &w, const LaunchPlan &lp, cudaStream_t st) {
    if (lp.arena)
        enqueue_rebuild<true>(w, lp, st);
    else
        enqueue_rebuild<false>(w, lp, st);
    return REBUILD_KERNELS;
}

// The condition reads exactly the flag the gated rebuild kernels test on
// entry, at the same point of the step, so a skipped body is one whose
// kernels would all have returned at once. (Every kernel keeps its test.)
__global__ void rebuild_condition_kernel(WorldDev w, cudaGraphConditionalHandle rebuild) {
    const bool pending = w.ctl->neighbor_state[0] != 0;
    cudaGraphSetConditional(rebuild, pending ? 1u : 0u);
    if (pending) w.ctl->rebuild_bodies += 1;
}

int launch_rebuild_condition(const WorldDev &w, cudaGraphConditionalHandle rebuild, cudaStream_t st) {
    rebuild_condition_kernel<<<1, 1, 0, st>>>(w, rebuild);
    return 1;
}

// The step of a looped batch graph: the rebuild condition as above, and the
// loop's own condition for after this step -- another step follows while
// the gate keeps the batch active and fewer than `steps` have begun. A
// batch the gate stops runs one more step, whose kernels all return at once
// (they test the same active flag), and the loop ends.
__global__ void step_condition_kernel(WorldDev w, cudaGraphConditionalHandle rebuild, cudaGraphConditionalHandle loop,
                                      uint32_t steps) {
    const bool pending = w.ctl->neighbor_state[0] != 0;
    cudaGraphSetConditional(rebuild, pending ? 1u : 0u);
    if (pending) w.ctl->rebuild_bodies += 1;
    const uint32_t begun = ++w.ctl->loop_step;
    cudaGraphSetConditional(loop, (w.ctl->control[0] != 0 && begun < steps) ? 1u : 0u);
}

int launch_step_condition(const WorldDev &w, cudaGraphConditionalHandle rebuild, cudaGraphConditionalHandle loop,
                          uint32_t steps, cudaStream_t st) {
    step_condition_kernel<<<1, 1, 0, st>>>(w, rebuild, loop, steps);
    return 1;
}

int launch_contact(const WorldDev &w, const LaunchPlan &lp, const StepParams &sp, bool gate, cudaStream_t st) {
    if (lp.arena) {
        if (gate && lp.contact_lists) {
            contact_kernel<CONTACT_LISTED, true><<<lp.contact_blocks, CONTACT_WARPS * 32, 0, st>>>(w, sp, 1, lp.line_eps);
            contact_kernel<CONTACT_REFRESH, true><<<lp.contact_blocks, CONTACT_WARPS * 32, 0, st>>>(w, sp, 1, lp.line_eps);
            return 2;
        }
        contact_kernel<CONTACT_FULL, true><<<lp.contact_blocks, CONTACT_WARPS * 32, 0, st>>>(w, sp, gate ? 1 : 0,
                                                                                            lp.line_eps);
        return 1;
    }
    if (gate && lp.contact_lists) {
        // Listed first: the refresh pass clears the flag the listed pass reads.
        contact_kernel<CONTACT_LISTED><<<lp.contact_blocks, CONTACT_WARPS * 32, 0, st>>>(w, sp, 1, lp.line_eps);
        contact_kernel<CONTACT_REFRESH><<<lp.contact_blocks, CONTACT_WARPS * 32, 0, st>>>(w, sp, 1, lp.line_eps);
        return 2;
    }
    contact_kernel<CONTACT_FULL><<<lp.contact_blocks, CONTACT_WARPS * 32, 0, st>>>(w, sp, gate ? 1 : 0, lp.line_eps);
    return 1;
}

template <bool A, bool FM>
static void enqueue_lanes(const WorldDev &w, const LaunchPlan &lp, const StepParams &sp, cudaStream_t st) {
    const dim3 grid(lp.lanes_blocks), block(32 * lp.lanes_wpb);
    const size_t smem = lp.lanes_smem * lp.lanes_wpb;
    switch (lp.lanes_per_fiber) {
        case 2: fiber_lanes_kernel<2, A, FM><<<grid, block, smem, st>>>(w, sp, lp.lanes_stride); break;
        case 8: fiber_lanes_kernel<8, A, FM><<<grid, block, smem, st>>>(w, sp, lp.lanes_stride); break;
        case 32: fiber_lanes_kernel<32, A, FM><<<grid, block, smem, st>>>(w, sp, lp.lanes_stride); break;
        default: fiber_lanes_kernel<4, A, FM><<<grid, block, smem, st>>>(w, sp, lp.lanes_stride); break;
    }
}

int launch_fiber_update(const WorldDev &w, const LaunchPlan &lp, const StepParams &sp, cudaStream_t st) {
    if (sp.motion_model == 1) {
        const int blocks = grid_for(w.F, 8, lp.num_sms * 16);
        if (lp.arena)
            rigid_kernel<true><<<blocks, 256, 0, st>>>(w, sp);
        else
            rigid_kernel<false><<<blocks, 256, 0, st>>>(w, sp);
        return 1;
    }
    if (lp.fiber_lanes) {
        int kernels = 1;
        if (lp.order_period > 0) {
            order_by_rounds_kernel<<<1, ORDER_THREADS, 0, st>>>(w, (uint32_t)lp.order_period, lp.order_ranked);
            kernels += 1;
        }
        if (lp.arena)
            enqueue_lanes<true, false>(w, lp, sp, st);
        else if (w.reaction != nullptr || w.layer_target != nullptr || w.vertex_target != nullptr)
            enqueue_lanes<false, true>(w, lp, sp, st);
        else
            enqueue_lanes<false, false>(w, lp, sp, st);
        return kernels;
    } else {
        fiber_kernel<<<lp.fiber_blocks, lp.fiber_warps * 32, lp.fiber_smem, st>>>(w, sp);
    }
    return 1;
}

int launch_stage_nonfinite(const WorldDev &w, unsigned int *flag, cudaStream_t st) {
    stage_nonfinite_kernel<<<grid_for(3ull * w.V, 256, 1 << 14), 256, 0, st>>>(w.xyz_stage, 3ull * w.V, flag);
    return 1;
}

int launch_positions_from_stage(const WorldDev &w, cudaStream_t st) {
    positions_from_stage_kernel<<<grid_for(w.V, 256, 1 << 16), 256, 0, st>>>(w);
    refresh_geometry_kernel<<<grid_for(w.S, 256, 1 << 16), 256, 0, st>>>(w);
    return 2;
}

int launch_refresh_geometry(const WorldDev &w, cudaStream_t st) {
    refresh_geometry_kernel<<<grid_for(w.S, 256, 1 << 16), 256, 0, st>>>(w);
    return 1;
}

int launch_positions_to_stage(const WorldDev &w, cudaStream_t st) {
    positions_to_stage_kernel<<<grid_for(w.V, 256, 1 << 16), 256, 0, st>>>(w);
    return 1;
}

int launch_corrections_to_stage(const WorldDev &w, float *corr6, float *pen, cudaStream_t st) {
    corrections_to_stage_kernel<<<grid_for(w.S, 256, 1 << 16), 256, 0, st>>>(w, corr6, pen);
    return 1;
}

}  // namespace tgl
