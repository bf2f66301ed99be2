"""Learned warm start: a message-passing network over the contact graph.

An addition on top of the plain relaxation (which stays the drop-in and
always runs afterwards to the same gates): a small network predicts, per
vertex, the displacement (in fiber diameters) that the plain relaxer would
produce over the next K iterations; the proposal is applied once and
reverted when it raises the overlap residual.

Network (hidden width 64, bf16 weights and activations, f32 accumulation
and master weights):

* encoder: node features (16: unit tangent, curvature x d, rest
  curvature x d, d / 10 um, overlap / d, contact push / d) -> 64 -> 64;
* 3 message-passing rounds, each with its own weights:
  - edge MLP on [h of the source point (interpolated along its segment),
    edge features] (64 + 16) -> 64 -> 64;
  - messages averaged into the vertices of the destination segment,
    weighted by the vertex's share (the closest-point parameter);
  - node MLP on [h, messages, mean of the fiber neighbors' h]
    (192) -> 64 -> 64, added to h (residual);
* decoder: 64 -> 64 -> 16 (the first 3 outputs are the displacement / d).

Every matrix product runs on the tensor cores through `tgl_gemm_bf16`
(tcgen05), every gather/scatter, reduction, loss and Adam step through this
library's kernels; PyTorch only holds the device memory and the stream.
"""

from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np

from .device import DeviceWorld, _raise, config_struct, load_library
from .settings import RelaxationConfig

HIDDEN = 64
ROUNDS = 3
NODE_FEATURES = 16
EDGE_FEATURES = 16
EDGE_INPUT = HIDDEN + EDGE_FEATURES  # 80
NODE_INPUT = 3 * HIDDEN              # 192
OUTPUT = 16                          # 3 used
K_SPLIT = 8192                       # samples per CTA in weight-gradient products


class _Gemm(ctypes.Structure):
    _fields_ = [
        ("a", ctypes.c_void_p), ("b", ctypes.c_void_p), ("lda", ctypes.c_int64), ("ldb", ctypes.c_int64),
        ("m", ctypes.c_int32), ("n", ctypes.c_int32), ("k", ctypes.c_int64), ("a_mn", ctypes.c_int32),
        ("b_mn", ctypes.c_int32), ("k_split", ctypes.c_int64), ("bias", ctypes.c_void_p),
        ("relu", ctypes.c_int32), ("reserved", ctypes.c_int32), ("mask", ctypes.c_void_p),
        ("ld_mask", ctypes.c_int64), ("residual", ctypes.c_void_p), ("ld_res", ctypes.c_int64),
        ("out_f32", ctypes.c_void_p), ("ldo", ctypes.c_int64), ("out_bf16", ctypes.c_void_p),
        ("ldo_bf16", ctypes.c_int64), ("error", ctypes.c_void_p),
    ]


class _MpGraph(ctypes.Structure):
    _fields_ = [
        ("vertex_count", ctypes.c_int32), ("segment_count", ctypes.c_int32), ("edge_count", ctypes.c_int32),
        ("reserved", ctypes.c_int32), ("seg_v0", ctypes.c_void_p), ("links", ctypes.c_void_p),
        ("offsets", ctypes.c_void_p), ("dst", ctypes.c_void_p), ("src", ctypes.c_void_p), ("twin", ctypes.c_void_p),
        ("s", ctypes.c_void_p), ("t", ctypes.c_void_p),
    ]


class _MpGraphOut(ctypes.Structure):
    _fields_ = [
        ("seg_v0", ctypes.c_void_p), ("links", ctypes.c_void_p), ("offsets", ctypes.c_void_p),
        ("dst", ctypes.c_void_p), ("src", ctypes.c_void_p), ("twin", ctypes.c_void_p), ("s", ctypes.c_void_p),
        ("t", ctypes.c_void_p), ("node_features", ctypes.c_void_p), ("edge_features", ctypes.c_void_p),
    ]


_bound = False


def _lib():
    global _bound
    lib = load_library()
    if not _bound:
        P, I64, I32, F = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32, ctypes.c_float
        sigs = {
            "tgl_gemm_bf16": [ctypes.POINTER(_Gemm), P],
            "tgl_mp_edge_inputs": [ctypes.POINTER(_MpGraph), P, P, I64, P],
            "tgl_mp_node_inputs": [ctypes.POINTER(_MpGraph), P, P, P, P],
            "tgl_mp_node_inputs_backward": [ctypes.POINTER(_MpGraph), P, P, P, P, P],
            "tgl_mp_edge_inputs_backward": [ctypes.POINTER(_MpGraph), P, I64, P, P],
            "tgl_column_sums": [P, I64, I32, I64, P, I32, P, P],
            "tgl_adam_step": [I64, P, P, P, P, P, F, F, F, F, I32, P],
            "tgl_mse": [I64, P, I64, P, I32, P, P, I64, P, P, P],
            "tgl_convert_bf16": [I64, P, P, P],
            "tgl_warmstart_graph_count": [P, F, ctypes.POINTER(I64)],
            "tgl_warmstart_graph_fill": [P, ctypes.POINTER(_MpGraphOut)],
            "tgl_warmstart_set_focus": [P, P, ctypes.c_size_t],
            "tgl_world_displace": [P, P, I64, F, I32, F],
            "tgl_world_residual": [P, P, ctypes.POINTER(F), ctypes.POINTER(F), ctypes.POINTER(F)],
        }
        for name, args in sigs.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        lib.tgl_column_sums_scratch.argtypes = [I64, I32]
        lib.tgl_column_sums_scratch.restype = ctypes.c_int64
        _bound = True
    return lib


def _check(rc: int) -> None:
    if rc:
        _raise(load_library(), rc)


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t) -> Optional[int]:
    return None if t is None else t.data_ptr()


def gemm(a, b, m, n, k, *, a_mn=False, b_mn=False, lda, ldb, bias=None, relu=False, mask=None, ld_mask=0,
         residual=None, ld_res=0, out_f32=None, ldo=0, out_bf16=None, ldo_bf16=0, k_split=0) -> None:
    """tgl_gemm_bf16 on torch tensors (see include/tangle_cuda.h)."""
    g = _Gemm(_p(a), _p(b), lda, ldb, m, n, k, int(a_mn), int(b_mn), k_split, _p(bias), int(relu), 0, _p(mask),
              ld_mask, _p(residual), ld_res, _p(out_f32), ldo, _p(out_bf16), ldo_bf16, None)
    _check(_lib().tgl_gemm_bf16(ctypes.byref(g), _stream()))


def column_sums(x, rows: int, n: int, ld: int, out, accumulate: bool = False) -> None:
    import torch

    lib = _lib()
    scratch = torch.empty(max(int(lib.tgl_column_sums_scratch(rows, n)), 1), dtype=torch.float32, device=x.device)
    _check(lib.tgl_column_sums(_p(x), rows, n, ld, _p(out), int(accumulate), _p(scratch), _stream()))


def to_bf16(x, out=None):
    import torch

    out = torch.empty(x.shape, dtype=torch.bfloat16, device=x.device) if out is None else out
    _check(_lib().tgl_convert_bf16(x.numel(), _p(x), _p(out), _stream()))
    return out


# ---------------------------------------------------------------- the graph


class ContactGraph:
    """A contact graph held in device tensors (independent of its world)."""

    def __init__(self, V: int, S: int, E: int, device):
        import torch

        i32, f32, bf = torch.int32, torch.float32, torch.bfloat16
        self.V, self.S, self.E = V, S, E
        self.seg_v0 = torch.empty(S, dtype=i32, device=device)
        self.links = torch.empty(4 * V, dtype=i32, device=device)
        self.offsets = torch.empty(S + 1, dtype=i32, device=device)
        self.dst = torch.empty(max(E, 1), dtype=i32, device=device)
        self.src = torch.empty(max(E, 1), dtype=i32, device=device)
        self.twin = torch.empty(max(E, 1), dtype=i32, device=device)
        self.s = torch.empty(max(E, 1), dtype=f32, device=device)
        self.t = torch.empty(max(E, 1), dtype=f32, device=device)
        self.node_features = torch.empty(V, NODE_FEATURES, dtype=bf, device=device)
        self.edge_features = torch.empty(max(E, 1), EDGE_FEATURES, dtype=bf, device=device)

    @classmethod
    def from_world(cls, world: DeviceWorld, cutoff: float, focus=None) -> "ContactGraph":
        """tgl_warmstart_graph_count / _fill on the world's current positions.
        With `focus` (fiber indices), only pairs with a segment on one of
        those fibers become edges (tgl_warmstart_set_focus)."""
        import torch

        lib = _lib()
        if focus is not None:
            flags = np.zeros(world.packed().fiber_count, dtype=np.uint8)
            flags[np.asarray(focus, dtype=np.int64)] = 1
            _check(lib.tgl_warmstart_set_focus(world._handle, flags.ctypes.data_as(ctypes.c_void_p), flags.size))
        try:
            edges = ctypes.c_int64()
            _check(lib.tgl_warmstart_graph_count(world._handle, ctypes.c_float(cutoff), ctypes.byref(edges)))
            g = cls(world.vertex_count, world.segment_count, int(edges.value), torch.device("cuda"))
            out = _MpGraphOut(_p(g.seg_v0), _p(g.links), _p(g.offsets), _p(g.dst), _p(g.src), _p(g.twin), _p(g.s),
                              _p(g.t), _p(g.node_features), _p(g.edge_features))
            _check(lib.tgl_warmstart_graph_fill(world._handle, ctypes.byref(out)))
        finally:
            if focus is not None:
                _check(lib.tgl_warmstart_set_focus(world._handle, None, 0))
        return g

    def struct(self) -> _MpGraph:
        return _MpGraph(self.V, self.S, self.E, 0, _p(self.seg_v0), _p(self.links), _p(self.offsets), _p(self.dst),
                        _p(self.src), _p(self.twin), _p(self.s), _p(self.t))

    def diameters(self):
        """Per-vertex fiber diameter (metres), from the node features."""
        return self.node_features[:, 5].float() * 10.0e-6


# ---------------------------------------------------------------- layers


class Linear:
    """y = act(x W^T + b) with W f32 [out x in] (master) and its bf16 copy."""

    def __init__(self, fan_in: int, out: int, relu: bool, generator, device, zero: bool = False,
                 used_inputs: Optional[int] = None, used_outputs: Optional[int] = None, init_scale: float = 1.0):
        import torch

        self.fan_in, self.out, self.relu = fan_in, out, relu
        bound = math.sqrt(6.0 / (used_inputs or fan_in)) if relu else math.sqrt(3.0 / (used_inputs or fan_in))
        bound *= init_scale
        w = (torch.rand(out, fan_in, generator=generator) * 2.0 - 1.0) * bound
        if used_inputs is not None:
            w[:, used_inputs:] = 0.0
        if used_outputs is not None:
            w[used_outputs:, :] = 0.0
        if zero:
            w.zero_()
        self.w = w.to(device)
        self.b = torch.zeros(out, device=device)
        self.wb = to_bf16(self.w)
        self.gw = torch.zeros_like(self.w)
        self.gb = torch.zeros_like(self.b)
        self.mw, self.vw = torch.zeros_like(self.w), torch.zeros_like(self.w)
        self.mb, self.vb = torch.zeros_like(self.b), torch.zeros_like(self.b)

    @property
    def parameter_count(self) -> int:
        return self.w.numel() + self.b.numel()

    def forward(self, x_bf16, rows: int, out_f32=None, out_bf16=None, residual=None) -> None:
        gemm(x_bf16, self.wb, rows, self.out, self.fan_in, lda=self.fan_in, ldb=self.fan_in, bias=self.b,
             relu=self.relu, residual=residual, ld_res=self.out, out_f32=out_f32, ldo=self.out, out_bf16=out_bf16,
             ldo_bf16=self.out)

    def backward(self, x_bf16, rows: int, dy_bf16, dy_f32, dx_f32=None, dx_bf16=None, x_mask=None) -> None:
        """Accumulates gw, gb; writes dx = dy W (times the ReLU mask of x when
        x came out of a ReLU)."""
        import torch

        splits = max(1, (rows + K_SPLIT - 1) // K_SPLIT)
        partial = torch.empty(splits, self.out, self.fan_in, dtype=torch.float32, device=self.w.device)
        gemm(dy_bf16, x_bf16, self.out, self.fan_in, rows, a_mn=True, b_mn=True, lda=self.out, ldb=self.fan_in,
             out_f32=partial, ldo=self.fan_in, k_split=K_SPLIT if splits > 1 else 0)
        column_sums(partial, splits, self.out * self.fan_in, self.out * self.fan_in, self.gw, accumulate=True)
        column_sums(dy_f32, rows, self.out, self.out, self.gb, accumulate=True)
        if dx_f32 is not None or dx_bf16 is not None:
            gemm(dy_bf16, self.wb, rows, self.fan_in, self.out, b_mn=True, lda=self.out, ldb=self.fan_in,
                 mask=x_mask, ld_mask=self.fan_in, out_f32=dx_f32, ldo=self.fan_in, out_bf16=dx_bf16,
                 ldo_bf16=self.fan_in)

    def zero_grad(self) -> None:
        self.gw.zero_()
        self.gb.zero_()

    def adam(self, lr: float, step: int, beta1=0.9, beta2=0.999, eps=1.0e-8) -> None:
        lib, st = _lib(), _stream()
        _check(lib.tgl_adam_step(self.w.numel(), _p(self.w), _p(self.gw), _p(self.mw), _p(self.vw), _p(self.wb),
                                 lr, beta1, beta2, eps, step, st))
        _check(lib.tgl_adam_step(self.b.numel(), _p(self.b), _p(self.gb), _p(self.mb), _p(self.vb), None, lr,
                                 beta1, beta2, eps, step, st))


# ---------------------------------------------------------------- the network


class WarmStartNet:
    """The message-passing network (module docstring)."""

    def __init__(self, seed: int = 0, device=None):
        import torch

        device = device or torch.device("cuda")
        g = torch.Generator().manual_seed(seed)
        self.device = device
        self.enc1 = Linear(NODE_FEATURES, HIDDEN, True, g, device, used_inputs=10)
        self.enc2 = Linear(HIDDEN, HIDDEN, False, g, device)
        self.rounds = []
        for _ in range(ROUNDS):
            self.rounds.append({
                "e1": Linear(EDGE_INPUT, HIDDEN, True, g, device, used_inputs=HIDDEN + 6),
                "e2": Linear(HIDDEN, HIDDEN, False, g, device),
                "n1": Linear(NODE_INPUT, HIDDEN, True, g, device),
                "n2": Linear(HIDDEN, HIDDEN, False, g, device, init_scale=0.1),
            })
        self.dec1 = Linear(HIDDEN, HIDDEN, True, g, device)
        self.dec2 = Linear(HIDDEN, OUTPUT, False, g, device, used_outputs=3)
        self.dec2.w.mul_(0.1)
        self.dec2.wb = to_bf16(self.dec2.w)
        self.step = 0

    def layers(self) -> List[Linear]:
        out = [self.enc1, self.enc2]
        for r in self.rounds:
            out += [r["e1"], r["e2"], r["n1"], r["n2"]]
        return out + [self.dec1, self.dec2]

    @property
    def parameter_count(self) -> int:
        return sum(layer.parameter_count for layer in self.layers())

    # ---- forward
    def forward(self, graph: ContactGraph, keep: bool = False):
        """Predicted displacement / d in columns 0..2 of an f32 [V x 16]
        tensor; with `keep`, also the activations the backward pass needs."""
        import torch

        V, E, dev = graph.V, graph.E, self.device
        bf, f32 = torch.bfloat16, torch.float32
        gs = graph.struct()
        lib, st = _lib(), _stream()
        cache: Dict[str, object] = {}
        a1 = torch.empty(V, HIDDEN, dtype=bf, device=dev)
        self.enc1.forward(graph.node_features, V, out_bf16=a1)
        h = torch.empty(V, HIDDEN, dtype=f32, device=dev)
        hb = torch.empty(V, HIDDEN, dtype=bf, device=dev)
        self.enc2.forward(a1, V, out_f32=h, out_bf16=hb)
        if keep:
            cache["a1"] = a1
            cache["h0b"] = hb
        xe = torch.zeros(max(E, 1), EDGE_INPUT, dtype=bf, device=dev)
        if E:
            xe[:, HIDDEN:] = graph.edge_features[:E]
        rounds = []
        for r in self.rounds:
            if E:
                _check(lib.tgl_mp_edge_inputs(ctypes.byref(gs), _p(h), _p(xe), EDGE_INPUT, st))
            z = torch.empty(max(E, 1), HIDDEN, dtype=bf, device=dev)
            m = torch.empty(max(E, 1), HIDDEN, dtype=f32, device=dev)
            if E:
                r["e1"].forward(xe, E, out_bf16=z)
                r["e2"].forward(z, E, out_f32=m)
            xn = torch.empty(V, NODE_INPUT, dtype=bf, device=dev)
            _check(lib.tgl_mp_node_inputs(ctypes.byref(gs), _p(h), _p(m), _p(xn), st))
            u = torch.empty(V, HIDDEN, dtype=bf, device=dev)
            r["n1"].forward(xn, V, out_bf16=u)
            h_new = torch.empty(V, HIDDEN, dtype=f32, device=dev)
            hb_new = torch.empty(V, HIDDEN, dtype=bf, device=dev)
            r["n2"].forward(u, V, out_f32=h_new, out_bf16=hb_new, residual=h)
            if keep:
                rounds.append({"xe": xe.clone() if E else None, "z": z, "xn": xn, "u": u})
            h, hb = h_new, hb_new
        d1 = torch.empty(V, HIDDEN, dtype=bf, device=dev)
        self.dec1.forward(hb, V, out_bf16=d1)
        y = torch.empty(V, OUTPUT, dtype=f32, device=dev)
        self.dec2.forward(d1, V, out_f32=y)
        if keep:
            cache.update(rounds=rounds, hb=hb, d1=d1)
            return y, cache
        return y

    # ---- backward
    def backward(self, graph: ContactGraph, cache, dy_f32, dy_bf16) -> None:
        import torch

        V, E, dev = graph.V, graph.E, self.device
        bf, f32 = torch.bfloat16, torch.float32
        gs = graph.struct()
        lib, st = _lib(), _stream()
        dd1 = torch.empty(V, HIDDEN, dtype=f32, device=dev)
        dd1b = torch.empty(V, HIDDEN, dtype=bf, device=dev)
        self.dec2.backward(cache["d1"], V, dy_bf16, dy_f32, dx_f32=dd1, dx_bf16=dd1b, x_mask=cache["d1"])
        dh = torch.empty(V, HIDDEN, dtype=f32, device=dev)
        self.dec1.backward(cache["hb"], V, dd1b, dd1, dx_f32=dh)
        for r, saved in zip(reversed(self.rounds), reversed(cache["rounds"])):
            dhb = to_bf16(dh)
            du = torch.empty(V, HIDDEN, dtype=f32, device=dev)
            dub = torch.empty(V, HIDDEN, dtype=bf, device=dev)
            r["n2"].backward(saved["u"], V, dhb, dh, dx_f32=du, dx_bf16=dub, x_mask=saved["u"])
            dxn = torch.empty(V, NODE_INPUT, dtype=f32, device=dev)
            r["n1"].backward(saved["xn"], V, dub, du, dx_f32=dxn)
            dh_prev = dh.clone()  # the residual path
            dm = torch.empty(max(E, 1), HIDDEN, dtype=bf, device=dev)
            dm32 = torch.empty(max(E, 1), HIDDEN, dtype=f32, device=dev)
            _check(lib.tgl_mp_node_inputs_backward(ctypes.byref(gs), _p(dxn), _p(dh_prev), _p(dm), _p(dm32), st))
            if E:
                dz = torch.empty(E, HIDDEN, dtype=f32, device=dev)
                dzb = torch.empty(E, HIDDEN, dtype=bf, device=dev)
                r["e2"].backward(saved["z"], E, dm, dm32, dx_f32=dz, dx_bf16=dzb, x_mask=saved["z"])
                dxe = torch.empty(E, EDGE_INPUT, dtype=f32, device=dev)
                r["e1"].backward(saved["xe"], E, dzb, dz, dx_f32=dxe)
                _check(lib.tgl_mp_edge_inputs_backward(ctypes.byref(gs), _p(dxe), EDGE_INPUT, _p(dh_prev), st))
            dh = dh_prev
        dhb = to_bf16(dh)
        da1 = torch.empty(V, HIDDEN, dtype=f32, device=dev)
        da1b = torch.empty(V, HIDDEN, dtype=bf, device=dev)
        self.enc2.backward(cache["a1"], V, dhb, dh, dx_f32=da1, dx_bf16=da1b, x_mask=cache["a1"])
        self.enc1.backward(graph.node_features, V, da1b, da1)

    def zero_grad(self) -> None:
        for layer in self.layers():
            layer.zero_grad()

    def adam(self, lr: float) -> None:
        self.step += 1
        for layer in self.layers():
            layer.adam(lr, self.step)

    def loss_and_gradient(self, y, target, rows: int):
        """tgl_mse over the 3 displacement columns: (loss tensor, dy f32, dy bf16)."""
        import torch

        loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        dy = torch.empty(rows, OUTPUT, dtype=torch.float32, device=self.device)
        dyb = torch.empty(rows, OUTPUT, dtype=torch.bfloat16, device=self.device)
        scratch = torch.empty(1024, dtype=torch.float32, device=self.device)
        _check(_lib().tgl_mse(rows, _p(y), OUTPUT, _p(target), 3, _p(loss), _p(dy), OUTPUT, _p(dyb), _p(scratch),
                              _stream()))
        return loss, dy, dyb

    def train_step(self, graph: ContactGraph, target, lr: float) -> float:
        self.zero_grad()
        y, cache = self.forward(graph, keep=True)
        loss, dy, dyb = self.loss_and_gradient(y, target, graph.V)
        self.backward(graph, cache, dy, dyb)
        self.adam(lr)
        return loss

    # ---- persistence
    def state(self) -> Dict[str, np.ndarray]:
        out = {"step": np.array([self.step])}
        for i, layer in enumerate(self.layers()):
            out[f"w{i}"] = layer.w.cpu().numpy()
            out[f"b{i}"] = layer.b.cpu().numpy()
        return out

    def load_state(self, state) -> None:
        import torch

        for i, layer in enumerate(self.layers()):
            layer.w.copy_(torch.from_numpy(np.asarray(state[f"w{i}"], dtype=np.float32)))
            layer.b.copy_(torch.from_numpy(np.asarray(state[f"b{i}"], dtype=np.float32)))
            layer.wb = to_bf16(layer.w)
        self.step = int(np.asarray(state["step"])[0])

    def save(self, path) -> None:
        np.savez(path, **self.state())

    @classmethod
    def load(cls, path, device=None) -> "WarmStartNet":
        net = cls(device=device)
        with np.load(path) as data:
            net.load_state({k: data[k] for k in data.files})
        return net


# ---------------------------------------------------------------- training data and use


@dataclass
class Sample:
    graph: ContactGraph
    target: object  # f32 [V x 3] displacement / d


def graph_cutoff(world: DeviceWorld) -> float:
    """Edge gap cutoff: the world's neighbor skin (pairs its Verlet lists hold)."""
    return float(world.neighbor_skin)


def make_sample(world: DeviceWorld, config: RelaxationConfig, iterations: int = 64) -> Sample:
    """Graph of the current positions and the plain relaxer's displacement
    over the next `iterations` iterations, in diameters."""
    import torch

    graph = ContactGraph.from_world(world, graph_cutoff(world))
    x0 = torch.from_numpy(world.download_positions()).to(graph.node_features.device).view(-1, 3)
    fixed = RelaxationConfig(**{**config.__dict__, "force_full_iterations": True})
    world.run_batch(fixed, iterations)
    x1 = torch.from_numpy(world.download_positions()).to(graph.node_features.device).view(-1, 3)
    target = ((x1 - x0) / graph.diameters()[:, None]).contiguous()
    return Sample(graph, target)


def residual(world: DeviceWorld, config: RelaxationConfig):
    """(max penetration, max curvature ratio, sum of penetration / d) of the
    current positions, moving nothing."""
    lib = _lib()
    a, b, c = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
    _check(lib.tgl_world_residual(world._handle, ctypes.byref(config_struct(config)), ctypes.byref(a),
                                  ctypes.byref(b), ctypes.byref(c)))
    return float(a.value), float(b.value), float(c.value)


@dataclass
class WarmStartReport:
    accepted: bool
    residual_before: float
    residual_after: float
    max_penetration_before: float
    max_penetration_after: float
    seconds: float
    edges: int
    curvature_after: float = 0.0  # max curvature ratio right after the proposal


def warm_start(world: DeviceWorld, net: WarmStartNet, config: RelaxationConfig, scale: float = 1.0,
               max_step_diameters: float = 2.0, fibers=None) -> WarmStartReport:
    """Applies the network's proposal to the world's positions; reverts it
    unless it lowers the overlap residual (the sum over segments of their
    deepest penetration / d). Curvature is left to the plain iterations that
    always follow: their gate includes it, and the proposal's small kinks are
    removed within their first sweeps. With `fibers` (indices), only those
    fibers' vertices move (a newly deposited ply on a relaxed stack)."""
    import torch

    t0 = time.perf_counter()
    pen0, curv0, total0 = residual(world, config)
    saved = world.download_positions()
    # Only the moving fibers' contacts can carry their proposal: with
    # `fibers`, the graph holds the pairs that touch one of them.
    graph = ContactGraph.from_world(world, graph_cutoff(world), focus=fibers)
    y = net.forward(graph)
    if fibers is not None:
        spans = np.asarray(world.packed().fiber_vertex_spans, dtype=np.int64).reshape(-1, 2)
        keep = np.zeros(world.vertex_count, dtype=np.float32)
        for f in np.asarray(fibers, dtype=np.int64):
            keep[spans[f, 0]: spans[f, 0] + spans[f, 1]] = 1.0
        y = y * torch.from_numpy(keep).to(y.device)[:, None]
    d_max = float(graph.diameters().max().item()) if graph.V else 0.0
    _check(_lib().tgl_world_displace(world._handle, _p(y), OUTPUT, ctypes.c_float(scale), 1,
                                     ctypes.c_float(max_step_diameters * d_max)))
    pen1, curv1, total1 = residual(world, config)
    accepted = total1 < total0
    if not accepted:
        world.upload_positions(saved)
    torch.cuda.synchronize()
    return WarmStartReport(accepted, total0, total1 if accepted else total0, pen0, pen1 if accepted else pen0,
                           time.perf_counter() - t0, graph.E, curv1)


# ---------------------------------------------------------------- training driver


def training_specimen(index: int, seed_base: int = 1000):
    """A 2,000-fiber specimen drawn like the mid-size one: the same fibers
    and volume fraction in a cube scaled by (2,000 / 20,000)^(1/3)."""
    from .generate import mid_size_specimen

    return mid_size_specimen(scale=(2000.0 / 20000.0) ** (1.0 / 3.0), seed=seed_base + index)


def ply_training_specimen(index: int, seed_base: int = 1000):
    """Two plies of the 20-ply stack's kind on a 1 mm square: the first is
    relaxed before the second is activated on top of it."""
    from .generate import ply_stack_specimen

    return ply_stack_specimen(plies=2, side=1.0e-3, seed=seed_base + index)


def relaxation_config(assembly, neighbor_capacity: int = 256) -> RelaxationConfig:
    from .settings import RelaxationSettings

    d = assembly.smallest_diameter()
    return RelaxationSettings(penetration_tolerance=1.0e-3 * d, neighbor_capacity=neighbor_capacity,
                              max_list_bytes=8 << 30).to_config(d)


def generate_samples(count: int, iterations: int = 64, seed_base: int = 1000, progress=None,
                     geometry: str = "mid_size") -> List[Sample]:
    """Training samples from the plain relaxer's own trajectories: each
    specimen's graph at its start and its displacement after `iterations`.
    With geometry "ply": the first ply relaxed 256 iterations alone, then
    the second activated, and the sample taken from there."""
    from .assembly import PackedAssembly

    samples = []
    for i in range(count):
        assembly = (ply_training_specimen if geometry == "ply" else training_specimen)(i, seed_base)
        config = relaxation_config(assembly)
        world = DeviceWorld(PackedAssembly.from_assembly(assembly), config.cell_list, config.max_step)
        if geometry == "ply":
            world.activate_formation_step(0)
            world.run_batch(RelaxationConfig(**{**config.__dict__, "force_full_iterations": True}), 256)
            world.activate_formation_step(1)
        samples.append(make_sample(world, config, iterations))
        world.close()
        if progress:
            progress(i)
    return samples


def train(net: WarmStartNet, samples: List[Sample], epochs: int, lr: float = 1.0e-3, log=None) -> List[float]:
    """Adam over the samples, one graph per step; returns the mean loss per epoch."""
    import torch

    history = []
    order = np.arange(len(samples))
    rng = np.random.default_rng(net.step + 12345)
    for epoch in range(epochs):
        rng.shuffle(order)
        losses = []
        for i in order:
            losses.append(net.train_step(samples[i].graph, samples[i].target, lr))
        mean = float(torch.stack(losses).mean().item())
        history.append(mean)
        if log:
            log(epoch, mean)
    return history


def evaluate(net: WarmStartNet, samples: List[Sample]) -> Dict[str, float]:
    """Mean loss of the network and of predicting no motion, on samples."""
    import torch

    model, zero = [], []
    for s in samples:
        y = net.forward(s.graph)
        loss, _, _ = net.loss_and_gradient(y, s.target, s.graph.V)
        model.append(loss)
        zero.append((s.target.float() ** 2).mean())
    return {"loss": float(torch.stack(model).mean().item()), "zero_motion_loss": float(torch.stack(zero).mean().item())}


def measure_gain(net: WarmStartNet, count: int, iterations: int = 64, seed_base: int = 900000,
                 scale: float = 1.0) -> Dict[str, object]:
    """On fresh held-out specimens: the residual after `iterations` plain
    iterations from the start, without and with the warm start first."""
    from .assembly import PackedAssembly

    rows = []
    for i in range(count):
        assembly = training_specimen(i, seed_base)
        config = relaxation_config(assembly)
        fixed = RelaxationConfig(**{**config.__dict__, "force_full_iterations": True})
        packed = PackedAssembly.from_assembly(assembly)
        plain = DeviceWorld(packed, config.cell_list, config.max_step)
        start = residual(plain, config)
        plain.run_batch(fixed, iterations)
        plain_after = residual(plain, config)
        plain.close()
        warm = DeviceWorld(packed, config.cell_list, config.max_step)
        report = warm_start(warm, net, config, scale=scale)
        warm.run_batch(fixed, iterations)
        warm_after = residual(warm, config)
        warm.close()
        rows.append({"start_total": start[2], "plain_total": plain_after[2], "warm_total": warm_after[2],
                     "plain_max_pen": plain_after[0], "warm_max_pen": warm_after[0],
                     "accepted": report.accepted, "proposal_total": report.residual_after,
                     "proposal_curvature_ratio": report.curvature_after})
    mean = lambda k: float(np.mean([r[k] for r in rows]))
    return {"specimens": count, "iterations": iterations, "accepted": sum(r["accepted"] for r in rows),
            "start_total": mean("start_total"), "plain_total": mean("plain_total"),
            "warm_total": mean("warm_total"), "plain_max_pen": mean("plain_max_pen"),
            "warm_max_pen": mean("warm_max_pen"), "proposal_total": mean("proposal_total"), "rows": rows}


def _main(argv=None) -> int:
    import argparse
    import json

    ap = argparse.ArgumentParser(description="Train the warm-start network on the plain relaxer's trajectories.")
    ap.add_argument("--specimens", type=int, default=256)
    ap.add_argument("--held-out", type=int, default=16)
    ap.add_argument("--iterations", type=int, default=64)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--lr", type=float, default=1.0e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--gain-specimens", type=int, default=8)
    ap.add_argument("--load", default=None, help="evaluate a saved network on held-out specimens; no training")
    ap.add_argument("--geometry", choices=["mid_size", "ply"], default="mid_size",
                    help="training specimens: mid-size-like cubes, or a ply deposited on a relaxed ply")
    ap.add_argument("--out", default=None)
    ap.add_argument("--learning-curve", default=None,
                    help="comma-separated training-set sizes: one network per size, trained on the first that many "
                         "specimens for --epochs epochs and evaluated on the same held-out specimens; no --out")
    args = ap.parse_args(argv)
    if args.learning_curve:
        sizes = sorted({int(x) for x in args.learning_curve.split(",") if x.strip()})
        t0 = time.perf_counter()
        samples = generate_samples(max(sizes) + args.held_out, args.iterations, geometry=args.geometry)
        test_set = samples[max(sizes):]
        curve = []
        for size in sizes:
            t1 = time.perf_counter()
            net = WarmStartNet(seed=args.seed)
            history = train(net, samples[:size], args.epochs, args.lr)
            curve.append({"specimens": size, "adam_steps": size * args.epochs, "held_out": evaluate(net, test_set),
                          "final_train_loss": history[-1], "train_seconds": time.perf_counter() - t1})
            print(json.dumps(curve[-1]), flush=True)
        print(json.dumps({"learning_curve": curve, "held_out_specimens": args.held_out, "epochs": args.epochs,
                          "parameters": WarmStartNet(seed=args.seed).parameter_count,
                          "seconds": time.perf_counter() - t0}), flush=True)
        return 0
    if args.load:
        print(json.dumps(measure_gain(WarmStartNet.load(args.load), args.gain_specimens, args.iterations)),
              flush=True)
        return 0
    if not args.out:
        ap.error("--out is required when training")
    t0 = time.perf_counter()
    samples = generate_samples(args.specimens + args.held_out, args.iterations, geometry=args.geometry)
    train_set, test_set = samples[: args.specimens], samples[args.specimens:]
    t1 = time.perf_counter()
    net = WarmStartNet(seed=args.seed)
    before = evaluate(net, test_set)
    history = train(net, train_set, args.epochs, args.lr,
                    log=lambda e, l: print(json.dumps({"epoch": e, "train_loss": l}), flush=True))
    t2 = time.perf_counter()
    after = evaluate(net, test_set)
    net.save(args.out)
    gain = (measure_gain(net, args.gain_specimens, args.iterations)
            if args.gain_specimens and args.geometry == "mid_size" else None)
    print(json.dumps({"specimens": args.specimens, "held_out": args.held_out, "iterations": args.iterations,
                      "epochs": args.epochs, "parameters": net.parameter_count, "data_seconds": t1 - t0,
                      "train_seconds": t2 - t1, "held_out_before": before, "held_out_after": after,
                      "gain": gain, "history": history}), flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(_main())
