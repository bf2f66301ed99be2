"""Learned warm start: graph, forward/backward against the f64 CPU oracle,
training, and the accept-or-revert rule.

Tolerances (written in the asserts): the device stores activations and
gradients in bf16 (8-bit mantissa) between layers and accumulates in f32,
the oracle computes in f64 with the same bf16 rounding of the stored
activations; outputs agree to 2 % of their scale and each parameter
gradient to 5 % in norm with cosine similarity above 0.995.
"""

import numpy as np
import pytest

from tangle_b200.assembly import PackedAssembly
from tangle_b200.generate import mid_size_specimen
from tangle_b200.settings import RelaxationConfig, RelaxationSettings

pytestmark = pytest.mark.gpu


def small_world(seed=3, scale=0.2):
    from tangle_b200.device import DeviceWorld

    assembly = mid_size_specimen(scale=scale, seed=seed)
    d = assembly.smallest_diameter()
    config = RelaxationSettings(penetration_tolerance=1.0e-3 * d, neighbor_capacity=256,
                                max_list_bytes=1 << 30).to_config(d)
    packed = PackedAssembly.from_assembly(assembly)
    return DeviceWorld(packed, config.cell_list, config.max_step), config, packed


def host_pairs(positions, packed, lists, counts, cutoff, box, periodic):
    """Pairs (a < b) of the Verlet lists within `cutoff` of touching, in f64."""
    x = positions.reshape(-1, 3).astype(np.float64)
    sv = packed.segment_vertices.reshape(-1, 2)
    r = packed.segment_radii.astype(np.float64)
    keep, margin = set(), set()
    for a, entries in enumerate(lists):
        if entries is None:
            continue
        for b in entries:
            b = int(b)
            if b <= a:
                continue
            p1, q1, p2, q2 = x[sv[a, 0]], x[sv[a, 1]], x[sv[b, 0]].copy(), x[sv[b, 1]].copy()
            sep = 0.5 * (p2 + q2 - p1 - q1)
            shift = np.where(periodic, np.round(sep / box) * box, 0.0)
            p2 -= shift
            q2 -= shift
            d1, d2, rr = q1 - p1, q2 - p2, p1 - p2
            A, E, F, C, B = d1 @ d1, d2 @ d2, d2 @ rr, d1 @ rr, d1 @ d2
            den = A * E - B * B
            s = min(max((B * F - C * E) / den, 0.0), 1.0) if den > 1e-12 * A * E else 0.0
            t = (B * s + F) / E
            if t < 0.0:
                t, s = 0.0, min(max(-C / A, 0.0), 1.0)
            elif t > 1.0:
                t, s = 1.0, min(max((B - C) / A, 0.0), 1.0)
            gap = np.linalg.norm(rr + d1 * s - d2 * t) - r[a] - r[b]
            if abs(gap - cutoff) < 1e-4 * cutoff:
                margin.add((a, b))
            elif gap <= cutoff:
                keep.add((a, b))
    return keep, margin


def test_contact_graph_is_symmetric_sorted_and_complete(cuda_lib):
    from tangle_b200.warmstart import ContactGraph, graph_cutoff

    world, config, packed = small_world()
    world.run_batch(RelaxationConfig(**{**config.__dict__, "force_full_iterations": True}), 5)
    cutoff = graph_cutoff(world)
    g = ContactGraph.from_world(world, cutoff)
    E = g.E
    assert E > 0
    dst, src = g.dst[:E].cpu().numpy(), g.src[:E].cpu().numpy()
    twin, s, t = g.twin[:E].cpu().numpy(), g.s[:E].cpu().numpy(), g.t[:E].cpu().numpy()
    off = g.offsets.cpu().numpy()
    assert off[0] == 0 and off[-1] == E and np.all(np.diff(off) >= 0)
    assert np.array_equal(np.repeat(np.arange(g.S), np.diff(off)), dst)
    for a in range(g.S):
        assert np.all(np.diff(src[off[a]:off[a + 1]]) > 0)
    assert np.array_equal(twin[twin], np.arange(E))
    assert np.array_equal(dst[twin], src) and np.array_equal(src[twin], dst)
    assert np.array_equal(s[twin], t) and np.array_equal(t[twin], s)
    assert np.all((s >= 0) & (s <= 1) & (t >= 0) & (t <= 1))
    # The pair set against an f64 host computation on the same lists.
    counts, lists = world.debug_neighbor_lists()
    box = (packed.cell_upper - packed.cell_lower).astype(np.float64)
    keep, margin = host_pairs(world.download_positions(), packed, lists, counts, cutoff, box,
                              packed.cell_periodic.astype(bool))
    got = {(int(a), int(b)) for a, b in zip(dst, src) if a < b}
    assert keep - got == set() and got - keep - margin == set()
    # Node features: unit tangents, diameters in units of 10 um.
    nf = g.node_features.float().cpu().numpy()
    assert np.allclose(np.linalg.norm(nf[:, :3], axis=1), 1.0, atol=1e-2)
    assert np.all(np.isclose(nf[:, 5], 0.7, atol=1e-2) | np.isclose(nf[:, 5], 1.9, atol=1e-2))


def test_focused_graph_keeps_exactly_the_pairs_touching_the_focus(cuda_lib):
    """A graph restricted to focus fibers (a new ply's warm start) holds
    exactly the full graph's edges with an endpoint segment on a focus
    fiber, with the same closest-point parameters and edge features; the
    next unrestricted graph is the full one again."""
    from tangle_b200.warmstart import ContactGraph, graph_cutoff

    world, config, packed = small_world(seed=9)
    world.run_batch(RelaxationConfig(**{**config.__dict__, "force_full_iterations": True}), 3)
    cutoff = graph_cutoff(world)
    full = ContactGraph.from_world(world, cutoff)
    focus = np.arange(0, packed.fiber_count, 3)
    part = ContactGraph.from_world(world, cutoff, focus=focus)
    again = ContactGraph.from_world(world, cutoff)
    fiber = packed.segment_fibers.astype(np.int64)
    in_focus = np.zeros(packed.fiber_count, dtype=bool)
    in_focus[focus] = True

    def records(g):
        E = g.E
        dst, src = g.dst[:E].cpu().numpy(), g.src[:E].cpu().numpy()
        s, t = g.s[:E].cpu().numpy(), g.t[:E].cpu().numpy()
        feats = g.edge_features[:E].float().cpu().numpy()
        return {(int(a), int(b)): (float(x), float(y), tuple(f)) for a, b, x, y, f in zip(dst, src, s, t, feats)}

    r_full, r_part = records(full), records(part)
    expected = {k: v for k, v in r_full.items() if in_focus[fiber[k[0]]] or in_focus[fiber[k[1]]]}
    assert 0 < len(r_part) < len(r_full)
    assert r_part == expected
    assert records(again) == r_full


def _params(net):
    return [(layer.w.cpu().numpy().astype(np.float64), layer.b.cpu().numpy().astype(np.float64))
            for layer in net.layers()]


def test_forward_and_gradients_match_the_f64_oracle(cuda_lib):
    import torch

    from warmstart_oracle import graph_to_cpu, loss_and_gradients
    from tangle_b200.warmstart import WarmStartNet, make_sample

    world, config, _ = small_world(seed=5, scale=0.15)
    sample = make_sample(world, config, iterations=16)
    net = WarmStartNet(seed=7)
    # Give the decoder full-size weights so every layer carries gradient.
    net.dec2.w.mul_(10.0)
    net.dec2.wb = net.dec2.w.to(torch.bfloat16)
    net.zero_grad()
    y, cache = net.forward(sample.graph, keep=True)
    loss, dy, dyb = net.loss_and_gradient(y, sample.target, sample.graph.V)
    net.backward(sample.graph, cache, dy, dyb)
    torch.cuda.synchronize()
    ref_loss, ref_y, ref_grads = loss_and_gradients(graph_to_cpu(sample.graph), _params(net),
                                                    sample.target.cpu().numpy())
    got_y = y.cpu().numpy()
    scale = np.abs(ref_y[:, :3]).max()
    assert np.abs(got_y[:, :3] - ref_y[:, :3]).max() <= 2e-2 * scale
    assert abs(float(loss.item()) - ref_loss) <= 2e-2 * ref_loss
    for i, (layer, (gw, gb)) in enumerate(zip(net.layers(), ref_grads)):
        for got, ref, name in ((layer.gw.cpu().numpy(), gw, "w"), (layer.gb.cpu().numpy(), gb, "b")):
            norm = np.linalg.norm(ref)
            if norm == 0.0:
                assert np.linalg.norm(got) == 0.0
                continue
            rel = np.linalg.norm(got - ref) / norm
            cos = float((got * ref).sum() / (np.linalg.norm(got) * norm))
            assert rel < 5e-2 and cos > 0.995, (i, name, rel, cos)


def test_gradients_match_the_bf16_rounding_model(cuda_lib):
    """The device's gradients against the f64 oracle that rounds activations
    and each layer's incoming gradient to bf16 where the device does: within
    1 % in norm (cosine > 0.9999). What is left is f32 accumulation and the
    bf16 roundings it flips (a flip moves one value by 2^-8 of itself). The
    oracle without the gradient rounding differs from the device by more:
    that rounding is what the 5 % bound against plain f64 autograd allows."""
    import torch

    from warmstart_oracle import graph_to_cpu, loss_and_gradients
    from tangle_b200.warmstart import WarmStartNet, make_sample

    world, config, _ = small_world(seed=5, scale=0.15)
    sample = make_sample(world, config, iterations=16)
    net = WarmStartNet(seed=7)
    net.dec2.w.mul_(10.0)
    net.dec2.wb = net.dec2.w.to(torch.bfloat16)
    net.zero_grad()
    y, cache = net.forward(sample.graph, keep=True)
    loss, dy, dyb = net.loss_and_gradient(y, sample.target, sample.graph.V)
    net.backward(sample.graph, cache, dy, dyb)
    torch.cuda.synchronize()
    g = graph_to_cpu(sample.graph)
    target = sample.target.cpu().numpy()
    _, _, model = loss_and_gradients(g, _params(net), target, round_gradients=True)
    _, _, plain = loss_and_gradients(g, _params(net), target, round_bf16=True, round_gradients=False)
    worst_model = worst_plain = 0.0
    for i, (layer, (mw, mb), (pw, pb)) in enumerate(zip(net.layers(), model, plain)):
        for got, ref, other, name in ((layer.gw.cpu().numpy(), mw, pw, "w"), (layer.gb.cpu().numpy(), mb, pb, "b")):
            norm = np.linalg.norm(ref)
            if norm == 0.0:
                continue
            rel = np.linalg.norm(got - ref) / norm
            cos = float((got * ref).sum() / (np.linalg.norm(got) * norm))
            assert rel < 1e-2 and cos > 0.9999, (i, name, rel, cos)
            worst_model = max(worst_model, rel)
            worst_plain = max(worst_plain, np.linalg.norm(got - other) / np.linalg.norm(other))
    assert worst_model < worst_plain, (worst_model, worst_plain)


def test_training_reduces_the_loss(cuda_lib):
    from tangle_b200.warmstart import WarmStartNet, evaluate, make_sample, train

    samples = []
    for seed in (11, 12, 13):
        world, config, _ = small_world(seed=seed, scale=0.15)
        samples.append(make_sample(world, config, iterations=32))
        world.close()
    net = WarmStartNet(seed=1)
    before = evaluate(net, samples)["loss"]
    history = train(net, samples, epochs=25, lr=2e-3)
    after = evaluate(net, samples)["loss"]
    assert after < 0.7 * before, (before, after, history[-3:])


def test_warm_start_never_raises_the_residual(cuda_lib):
    from tangle_b200.warmstart import WarmStartNet, residual, warm_start

    world, config, _ = small_world(seed=17, scale=0.2)
    net = WarmStartNet(seed=2)
    pen0, curv0, total0 = residual(world, config)
    for scale in (1.0, 50.0):  # an untrained proposal, then a wild one
        report = warm_start(world, net, config, scale=scale)
        pen1, curv1, total1 = residual(world, config)
        assert total1 <= total0 * (1.0 + 1e-6)
        if not report.accepted:
            assert (pen1, total1) == (pen0, total0)
        pen0, curv0, total0 = pen1, curv1, total1


def test_residual_matches_the_contact_pass(cuda_lib):
    from tangle_b200.warmstart import residual

    world, config, _ = small_world(seed=19, scale=0.2)
    pen, ratio, total = residual(world, config)
    _, seg_pen = world.debug_corrections(config)
    assert np.float32(pen) == np.float32(seg_pen.max())
    assert total > 0.0 and ratio > 0.0


def test_trained_network_gains_over_plain_relaxation(cuda_lib):
    """The committed network, on specimens it was not trained on: its
    proposal is accepted, and after the same 64 plain iterations the summed
    overlap is at least 15 % below plain relaxation's."""
    import os

    from tangle_b200.device import DeviceWorld
    from tangle_b200.warmstart import WarmStartNet, relaxation_config, residual, training_specimen, warm_start

    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tangle_b200",
                        "warmstart_net.npz")
    net = WarmStartNet.load(path)
    for index in (3, 7):
        assembly = training_specimen(index, seed_base=700000)
        config = relaxation_config(assembly)
        fixed = RelaxationConfig(**{**config.__dict__, "force_full_iterations": True})
        packed = PackedAssembly.from_assembly(assembly)
        plain = DeviceWorld(packed, config.cell_list, config.max_step)
        plain.run_batch(fixed, 64)
        warm = DeviceWorld(packed, config.cell_list, config.max_step)
        report = warm_start(warm, net, config)
        assert report.accepted and report.residual_after < 0.6 * report.residual_before
        warm.run_batch(fixed, 64)
        assert residual(warm, config)[2] < 0.85 * residual(plain, config)[2]
