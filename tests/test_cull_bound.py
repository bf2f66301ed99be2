"""The Verlet build's stencil-cell culling never skips a pair the sphere test passes.

rb_build_kernel (tangle_b200/csrc/kernels.cu) stages the 27 stencil cells'
bounding spheres, bounds each cell's spheres (radii x 1.0003) by a box in
that cell's own frame, and lets a home segment skip a cell whose box is
farther than its reach. This restates both tests in f32, operation for
operation (numpy rounds every f32 operation and contracts nothing, as the
kernel is compiled), on random grids: periodic and walled axes, unwrapped
coordinates several box lengths out, centres outside the walls, centres
within 1e-7 of a cell face and partners placed at the sphere test's limit
(half of them along an axis, where the box bound is tight).
Every pair that passes the sphere test must lie in a cell the home scans.
The GPU pair-set tests check the kernel itself bit for bit.
"""

import numpy as np
import pytest

f32 = np.float32


def proxy_cell(m, lower, width, cells, periodic):
    r = np.floor((m - lower) / width).astype(np.int64)
    return np.mod(r, cells) if periodic else np.clip(r, 0, cells - 1)


def make_grid(rng):
    cells = rng.integers(3, 7, size=3)
    periodic = rng.random(3) < 0.6
    lower = (rng.normal(size=3) * 10.0 ** rng.uniform(-4, 0.5, size=3)).astype(f32)
    width0 = f32(10.0 ** rng.uniform(-5, -3))
    length = (width0 * cells).astype(f32)
    width = (length / cells.astype(f32)).astype(f32)
    inv_length = (f32(1.0) / length).astype(f32)
    return cells, periodic, lower, width, length, inv_length


def make_spheres(rng, grid, n):
    cells, periodic, lower, width, length, _ = grid
    wmax = float(width.max())
    radius = (rng.random(n) * wmax * rng.uniform(0.05, 0.5)).astype(f32)
    skin = f32(wmax * rng.uniform(0.0, 0.4))
    c = np.empty((n, 3), f32)
    for a in range(3):
        x = lower[a] + rng.random(n) * length[a]
        if periodic[a]:
            x = x + rng.integers(-3, 4, size=n) * length[a]
        else:
            out = rng.random(n) < 0.1
            x = np.where(out, lower[a] + rng.uniform(-0.5, 1.5, size=n) * length[a], x)
        c[:, a] = x.astype(f32)
    face = rng.random(n) < 0.3  # centres within 1e-7 of a cell face
    for a in range(3):
        k = rng.integers(0, cells[a], size=n)
        x = (lower[a] + k.astype(f32) * width[a]).astype(f32) + (rng.normal(size=n) * 1e-7 * wmax).astype(f32)
        c[face, a] = x[face].astype(f32)
    sphere_eps = f32(1e-6 * float(length.max()))
    for _ in range(n // 3):  # partners at the sphere test's limit
        i, j = rng.integers(0, n, size=2)
        if i == j:
            continue
        if rng.random() < 0.5:  # along an axis: where the box bound is tight
            u = np.zeros(3)
            u[rng.integers(0, 3)] = rng.choice([-1.0, 1.0])
        else:
            u = rng.normal(size=3)
            u /= np.linalg.norm(u)
        limit = float((radius[i] + radius[j] + skin) * 1.0002) + float(sphere_eps)
        c[j] = (c[i].astype(np.float64) + u * limit * (1.0 - rng.uniform(0.0, 2e-6))).astype(f32)
    return c, radius, skin, sphere_eps


def wrap(d, axis, grid):
    _, periodic, _, _, length, inv_length = grid
    if periodic[axis]:
        d = (d - (np.rint((d * inv_length[axis]).astype(f32)).astype(f32) * length[axis]).astype(f32)).astype(f32)
    return d


def check_one(seed):
    rng = np.random.default_rng(seed)
    grid = make_grid(rng)
    cells, periodic, lower, width, length, _ = grid
    n = int(rng.integers(80, 300))
    c, radius, skin, sphere_eps = make_spheres(rng, grid, n)
    cell = np.stack([proxy_cell(c[:, a], lower[a], width[a], cells[a], periodic[a]) for a in range(3)], 1)
    grid_scale, wmax = f32(0.0), f32(0.0)
    for a in range(3):
        grid_scale = f32(grid_scale + f32(f32(abs(lower[a])) + f32(f32(2.0) * length[a])))
        wmax = max(wmax, width[a])
    # Each sphere's box in its own cell's frame (home-independent).
    face = (lower[None, :] + (cell.astype(f32) * width[None, :]).astype(f32)).astype(f32)
    r3 = (radius * f32(1.0003)).astype(f32)
    p = np.stack([wrap((c[:, a] - face[:, a]).astype(f32), a, grid) for a in range(3)], 1)
    lo_s, hi_s = (p - r3[:, None]).astype(f32), (p + r3[:, None]).astype(f32)
    mag_s = ((np.abs(c[:, 0]) + np.abs(c[:, 1])).astype(f32) + np.abs(c[:, 2])).astype(f32)
    key = (cell[:, 2] * cells[1] + cell[:, 1]) * cells[0] + cell[:, 0]
    members = {int(k): np.nonzero(key == k)[0] for k in np.unique(key)}
    box = {k: (lo_s[m].min(0), hi_s[m].max(0), mag_s[m].max()) for k, m in members.items()}
    passed = culled = skipped_passing = 0
    for i in range(n):
        hc = cell[i]
        q = np.array([wrap(f32(c[i, a] - face[i, a]), a, grid) for a in range(3)], f32)
        for k in range(27):
            off = np.array([k % 3 - 1, (k // 3) % 3 - 1, k // 9 - 1])
            nc = hc + off
            ok = True
            for a in range(3):
                if periodic[a]:
                    nc[a] %= cells[a]
                elif not 0 <= nc[a] < cells[a]:
                    ok = False
            if not ok:
                continue
            nk = int((nc[2] * cells[1] + nc[1]) * cells[0] + nc[0])
            if nk not in box:
                continue
            lo, hi, mag = box[nk]
            far2 = f32(0.0)
            for a in range(3):
                shift = f32(f32(f32(off[a]) * width[a]) - q[a])
                l, h = f32(lo[a] + shift), f32(hi[a] + shift)
                gap = max(f32(0.0), max(l, f32(-h)))
                if periodic[a]:
                    for sign in (1, -1):
                        ls, hs = f32(l + sign * length[a]), f32(h + sign * length[a])
                        gap = min(gap, max(f32(0.0), max(ls, f32(-hs))))
                far2 = f32(far2 + f32(gap * gap))
            hmag = f32(f32(f32(abs(c[i, 0])) + f32(abs(c[i, 1]))) + f32(abs(c[i, 2])))
            margin = f32(f32(f32(1e-3) * wmax) + f32(f32(8e-6) * f32(f32(f32(mag + hmag)) + grid_scale)))
            reach = f32(f32(f32(f32(radius[i] + skin) * f32(1.0002)) + sphere_eps) + margin)
            scan = not far2 > f32(reach * reach)
            m = members[nk]
            d = np.stack([wrap((c[m, a] - c[i, a]).astype(f32), a, grid) for a in range(3)], 1)
            limit = ((((radius[i] + radius[m]).astype(f32) + skin).astype(f32) * f32(1.0002)).astype(f32)
                     + sphere_eps).astype(f32)
            d2 = ((d[:, 0] * d[:, 0]).astype(f32) + (d[:, 1] * d[:, 1]).astype(f32)).astype(f32)
            d2 = (d2 + (d[:, 2] * d[:, 2]).astype(f32)).astype(f32)
            passes = d2 <= (limit * limit).astype(f32)
            passed += int(passes.sum())
            if not scan:
                culled += len(m)
                skipped_passing += int(passes.sum())
    return passed, culled, skipped_passing


SEEDS = range(12)
RESULTS = {}


@pytest.mark.parametrize("seed", SEEDS)
def test_culled_cells_hold_no_passing_pair(seed):
    RESULTS[seed] = passed, culled, skipped = check_one(seed)
    assert skipped == 0
    assert passed > 0


def test_the_random_grids_cull_cells():
    """Both sides are exercised: some grids cull a good share of the pairs."""
    results = [RESULTS.get(seed) or check_one(seed) for seed in SEEDS]
    assert sum(r[1] for r in results) > 0.2 * sum(r[0] for r in results)
