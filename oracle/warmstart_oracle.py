"""CPU f64 restatement of the warm-start network (test infrastructure only).

The learned warm start has no counterpart in the reference; its gradients
are checked against PyTorch CPU autograd in float64 on the same graph,
features and weights. `forward` mirrors tangle_b200/warmstart.py layer by
layer; with `round_bf16` it rounds to bf16 exactly where the device path
stores bf16 activations, and with `round_gradients` it also rounds every
layer's incoming gradient as the device does, so that what remains is the
device's f32 accumulation (and the bf16 roundings its f32 sums flip).
"""

from __future__ import annotations

import numpy as np
import torch

HIDDEN = 64


def _bf16(x, on: bool):
    return x.to(torch.bfloat16).to(torch.float64) if on else x


def graph_to_cpu(graph):
    """The device graph's arrays as CPU tensors."""
    E = graph.E
    return {
        "V": graph.V, "S": graph.S, "E": E,
        "seg_v0": graph.seg_v0.cpu().long(),
        "links": graph.links.cpu().long().view(-1, 4),
        "offsets": graph.offsets.cpu().long(),
        "dst": graph.dst[:E].cpu().long(), "src": graph.src[:E].cpu().long(),
        "twin": graph.twin[:E].cpu().long(),
        "s": graph.s[:E].cpu().double(), "t": graph.t[:E].cpu().double(),
        "node_features": graph.node_features.cpu().double(),
        "edge_features": graph.edge_features[:E].cpu().double(),
    }


class _DeviceLinear(torch.autograd.Function):
    """y = round(x) round(W)^T + b whose backward rounds the incoming
    gradient dy to bf16 where the device does (tangle_b200/warmstart.py
    Linear.backward: the weight gradient dy_bf16^T x_bf16 and the input
    gradient dy_bf16 W_bf16 take the rounded dy, the bias gradient the f32
    dy), with f64 arithmetic everywhere else."""

    @staticmethod
    def forward(ctx, x, w, b):
        xr, wr = _bf16(x, True), _bf16(w, True)
        ctx.save_for_backward(xr, wr)
        return xr @ wr.T + b

    @staticmethod
    def backward(ctx, dy):
        xr, wr = ctx.saved_tensors
        dyr = _bf16(dy, True)
        return dyr @ wr, dyr.T @ xr, dy.sum(0)


def forward(g, params, round_bf16: bool = True, round_gradients: bool = False):
    """params: list of (W [out x in], b [out]) f64 tensors in WarmStartNet.layers() order.
    With `round_gradients` (implies round_bf16), every layer's backward also
    rounds its incoming gradient to bf16 as the device does (_DeviceLinear)."""
    rb = round_bf16 or round_gradients
    V, E = g["V"], g["E"]
    it = iter(params)

    def lin(x, relu):
        w, b = next(it)
        y = _DeviceLinear.apply(x, w, b) if round_gradients else _bf16(x, rb) @ _bf16(w, rb).T + b
        return torch.relu(y) if relu else y

    a1 = _bf16(lin(g["node_features"], True), rb)
    h = lin(a1, False)
    links = g["links"]
    v0 = g["seg_v0"][g["src"]]
    dst_v0 = g["seg_v0"][g["dst"]]
    for _ in range(3):
        t = g["t"][:, None]
        xe = torch.cat([(1.0 - t) * h[v0] + t * h[v0 + 1], g["edge_features"]], dim=1) if E else None
        if E:
            z = _bf16(lin(_bf16(xe, rb), True), rb)
            m = lin(z, False)
            s = g["s"][:, None]
            agg = torch.zeros(V, HIDDEN, dtype=torch.float64)
            agg = agg.index_add(0, dst_v0, (1.0 - s) * m).index_add(0, dst_v0 + 1, s * m)
            weight = torch.zeros(V, dtype=torch.float64)
            weight = weight.index_add(0, dst_v0, 1.0 - g["s"]).index_add(0, dst_v0 + 1, g["s"])
            agg = agg / weight.clamp(min=1.0)[:, None]
        else:
            next(it)
            next(it)
            agg = torch.zeros(V, HIDDEN, dtype=torch.float64)
        prev, nxt = links[:, 0], links[:, 1]
        has_p, has_n = (prev >= 0).double()[:, None], (nxt >= 0).double()[:, None]
        count = (has_p + has_n).clamp(min=1.0)
        nb = (h[prev.clamp(min=0)] * has_p + h[nxt.clamp(min=0)] * has_n) / count
        xn = _bf16(torch.cat([h, agg, nb], dim=1), rb)
        u = _bf16(lin(xn, True), rb)
        h = h + lin(u, False)
    d1 = _bf16(lin(_bf16(h, rb), True), rb)
    return lin(d1, False)


def loss_and_gradients(g, params_np, target, round_bf16: bool = True, round_gradients: bool = False):
    """MSE of the first 3 outputs against target [V x 3]; returns
    (loss, output, [(dW, db)] as numpy) in f64."""
    params = [(torch.tensor(w, dtype=torch.float64, requires_grad=True),
               torch.tensor(b, dtype=torch.float64, requires_grad=True)) for w, b in params_np]
    y = forward(g, params, round_bf16, round_gradients)
    tgt = torch.as_tensor(np.asarray(target), dtype=torch.float64)
    loss = ((y[:, :3] - tgt) ** 2).mean()
    loss.backward()
    return float(loss.detach()), y.detach().numpy(), [(w.grad.numpy(), b.grad.numpy()) for w, b in params]
