"""Benchmark of the plain relaxation path on B200.

Default workload: the mid-size specimen (periodic 2 mm cube, 20,000 wavy
fibers of 7 and 19 um split 50:50 by volume, segment length 2 d, curvature
limit 1/(5 d); about 2.0 M nodes), generated from a seed (synthetic: no
dataset involved). One step = one `run_batch` of `--iterations` relaxation
iterations (force_full_iterations, so every step does the same number of
iterations and neighbor-list rebuilds happen as the displacement check
requests them).

Printed JSON line (rank 0):
* value -- node-iterations/s over the K timed steps, whole job, inputs
  resident in HBM, CUDA events on the library's stream, max over ranks;
* e2e -- the same metric through the public API with host buffers: every
  step uploads positions from pinned host memory, runs the batch and
  downloads the positions;
* roofline -- the fiber update (the largest kernel): algorithmic bytes per
  launch (`update_bytes`) over its CUDA-event duration inside the timed
  region, against the measured HBM copy bandwidth, with the DRAM traffic of
  the committed ncu capture; roofline_contact -- the same for the contact
  pass: sum_s (60 + 4 K_s) bytes per launch;
* cpu_baseline -- the CPU oracle on the same specimen, all host threads,
  a bounded sample of iterations;
* time_to_admissible -- seconds from the initial specimen to max overlap
  < 1e-3 d with curvature <= limit (or the iteration cap), for plain PBD and
  for the learned warm start followed by plain PBD, with the time at which
  the max overlap first fell below 0.1, 0.05, 0.03, 0.02, 0.01 and 0.001 d.

`--impl reference` times the reference algorithm's CPU restatement (the
oracle; the reference is Rust and cannot be built here) on the same
workload, rank 0 only. `--workload ply_stack` deposits the 20-ply stack ply
by ply (its own JSON line: whole-job seconds, plain and warm-started).
Multi-GPU: one independent replica specimen per rank (replicas only; the
relaxation of one specimen runs on one GPU).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s to overlap<1e-3·d & node-iter/s: learned warm-start vs plain PBD, 1 B200"
UNIT = "node-iter/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["cuda", "reference"], default="cuda")
    ap.add_argument("--workload", choices=["mid_size", "cpu_runnable", "batched", "ply_stack", "gemm"],
                    default="mid_size")
    ap.add_argument("--plies", type=int, default=20, help="plies of the ply_stack workload")
    ap.add_argument("--ply-budget", type=int, default=1024, help="iteration cap per ply of the ply_stack workload")
    ap.add_argument("--ply-side", type=float, default=2.0e-3, help="ply edge of the ply_stack workload (m)")
    ap.add_argument("--specimens", type=int, default=512, help="specimens of the batched workload")
    ap.add_argument("--iterations", type=int, default=128, help="relaxation iterations per step")
    ap.add_argument("--scale", type=float, default=1.0, help="shrink the mid-size cell (tests only)")
    ap.add_argument("--capacity", type=int, default=256, help="neighbor slots per segment")
    ap.add_argument("--gemm-scale", type=float, default=1.0,
                    help="scale the row counts of the gemm workload's network shapes (small profiling cases)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-tta", action="store_true")
    ap.add_argument("--tta-iterations", type=int, default=20000, help="iteration cap of each time-to-admissible run")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--autotune", action="store_true", help="also time the steps with the autotuner's launch shapes")
    ap.add_argument("--no-autotune", action="store_true", help="skip the autotuner comparison of the batched workload")
    ap.add_argument("--cpu-iterations", type=int, default=40)
    ap.add_argument("--cpu-specimens", type=int, default=16, help="arena specimens the CPU baseline relaxes")
    ap.add_argument("--reference-iterations", type=int, default=4,
                    help="relaxation iterations per step of the reference arm (CPU)")
    ap.add_argument("--beta", type=float, default=1.0 / 0.3,
                    help="Schladitz beta of the mid-size specimen's orientation about z (0.3: z-aligned)")
    ap.add_argument("--tta-betas", default="3.3333333333333335,0.3",
                    help="betas of the time-to-admissible runs (comma separated; empty: the workload's only)")
    ap.add_argument("--save-positions", default=None, help="write the positions after the timed steps (.npy)")
    ap.add_argument("--load-positions", default=None, help="start from saved positions (.npy)")
    return ap.parse_args()


def beta_label(beta: float) -> str:
    if abs(beta - 1.0 / 0.3) < 1.0e-9:
        return "Schladitz beta 1/0.3 about z (xy-biased)"
    if abs(beta - 0.3) < 1.0e-9:
        return "Schladitz beta 0.3 about z (z-aligned)"
    return f"Schladitz beta {beta:g} about z"


def bench_config(name, packs, config):
    """The workload as both arms name it (same keys, same values)."""
    return {"workload": name, "nodes": sum(p.vertex_count for p in packs),
            "segments": sum(p.segment_count for p in packs), "fibers": sum(p.fiber_count for p in packs),
            "specimens": len(packs), "neighbor_capacity": config.cell_list.neighbor_capacity}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def replica_throughput(seconds: float, work: float, world_size: int, device: str = "cuda"):
    """Whole-job throughput of independent replicas (no data-path
    collective): every rank's work summed, over the slowest rank's time (max
    over ranks), reduced through the process group (NCCL on the GPUs, gloo in
    the CPU tests). Returns (value, seconds, work)."""
    if world_size > 1:
        import torch
        import torch.distributed as dist

        t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
        w = torch.tensor([float(work)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(w, op=dist.ReduceOp.SUM)
        seconds, work = float(t.item()), float(w.item())
    return work / seconds, seconds, work


def workload(args, rank):
    """(assembly or list of assemblies for the arena, config, name, smallest diameter)."""
    from tangle_b200.generate import batched_specimens, cpu_runnable_specimen, mid_size_specimen
    from tangle_b200.settings import RelaxationSettings

    if args.workload == "batched":
        assemblies = batched_specimens(count=args.specimens, seed=1 + rank)
        d_min = min(a.smallest_diameter() for a in assemblies)
        name = (f"batched: {args.specimens} specimens in one arena, fiber count log-uniform 40-5,000, d 10 um, "
                "length 0.3-1 mm, segment 2d, fiber volume fraction 5-25 %, isotropic, curvature limit 1/(5d)")
        settings = RelaxationSettings(penetration_tolerance=1.0e-3 * d_min, neighbor_capacity=args.capacity,
                                      max_list_bytes=32 << 30, iterations_per_batch=args.iterations,
                                      max_iterations=100000)
        return assemblies, settings.to_config(d_min), name, d_min
    if args.workload == "cpu_runnable":
        assembly = cpu_runnable_specimen(seed=1 + rank)
        name = "cpu_runnable: periodic 300 um cube, 40 straight 10 um fibers x 30 segments (1,240 nodes)"
    else:
        assembly = mid_size_specimen(scale=args.scale, seed=1 + rank, beta=args.beta)
        name = ("mid_size: periodic 2x2x2 mm, 20,000 wavy fibers 1.5 mm, d 7/19 um 50:50 by volume, "
                f"segment 2d, {beta_label(args.beta)}, curvature limit 1/(5d)")
        if args.scale != 1.0:
            name += f", scaled {args.scale}"
    d_min = assembly.smallest_diameter()
    settings = RelaxationSettings(penetration_tolerance=1.0e-3 * d_min, neighbor_capacity=args.capacity,
                                  max_list_bytes=8 << 30, iterations_per_batch=args.iterations,
                                  max_iterations=100000)
    config = settings.to_config(d_min)
    return assembly, config, name, d_min


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        self.file.flush()
        self.file.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.file.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() in ("active", "1", "yes"):
                    reasons.add(name)
        os.unlink(self.file.name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def contact_bytes(world):
    """Algorithmic bytes of the two kinds of contact pass.

    A pass reads each segment's own record and writes its outputs (60 B) and
    reads 4 B per list entry it walks: the Verlet list (K_s entries) in a
    refresh pass, which also writes the contact lists (4 B per kept entry and
    4 B per count) and the position snapshot (16 B read + 16 B written per
    node); the contact list in a listed pass (the Verlet list where a slot's
    contact list overflowed). Returns (listed, refresh) bytes; without
    contact lists both are the full-list bytes sum_s (60 + 4 K_s).
    """
    import numpy as np

    counts, _ = world.debug_neighbor_lists()
    S = counts.size
    block = world.neighbor_block
    listed_verlet = np.where(counts <= block, counts, 0).astype(np.float64)
    full = 60.0 * S + 4.0 * float(listed_verlet.sum())
    info = world.contact_list_info()
    if info["block"] == 0:
        return full, full
    from tangle_b200.device import CONTACT_USE_VERLET

    states = world.debug_contact_states()
    _, _, slot_segment = world.debug_cell_list()
    verlet_by_slot = listed_verlet[slot_segment]
    on_verlet = states == CONTACT_USE_VERLET
    scanned = states == 0xFFFFFFFF
    chunked = np.where(on_verlet | scanned, 0, states).astype(np.float64)
    walked = np.where(on_verlet, verlet_by_slot, chunked)
    listed = 60.0 * S + 4.0 * float(walked.sum())
    kept = chunked
    refresh = full + 4.0 * float(kept.sum()) + 4.0 * S + 32.0 * world.vertex_count
    return listed, refresh


def ncu_traffic(refresh_share: float, lists_on: bool):
    """Per-pass DRAM bytes of the contact pass from the committed ncu summary
    (listed and refresh passes weighted by their share of the passes)."""
    path = os.path.join(ROOT, "profiles", "contact_traffic.json")
    try:
        with open(path) as fh:
            data = json.load(fh)
        if not lists_on:
            return float(data["dram_bytes_per_full_pass"])
        return (refresh_share * float(data["dram_bytes_per_refresh_pass"]) +
                (1.0 - refresh_share) * float(data["dram_bytes_per_listed_pass"]))
    except (OSError, KeyError, ValueError):
        return None


def update_bytes(nodes: int, segments: int, contact_lists: bool) -> float:
    """Algorithmic bytes of one fiber-update launch: per vertex the position
    read and written (16 + 16), its static record (16), pinned flag (4),
    list snapshot (16) and step (4), plus the contact-list snapshot (16) when
    contact lists are on; per segment its rest length (4), two correction
    records (32) and two geometry records written (32)."""
    return float(nodes) * (72.0 + (16.0 if contact_lists else 0.0)) + float(segments) * 68.0


def issue_bound(profile: str, refresh_share=None):
    """A kernel against its instruction-issue bound, from the committed
    full-size ncu capture (one pass per launch): the warp instructions of a
    launch over the same launch's duration, against 4 warp instructions per
    clock on each of the 148 SMs at the 1,965 MHz the capture ran at; for the
    contact pass, listed and refresh passes weighted by their share of this
    run's passes. Both figures come from the same launches (the capture's
    state, early in the trajectory), so the fraction does not mix states
    with this run's timing. None without the capture."""
    path = os.path.join(ROOT, "profiles", profile)
    try:
        with open(path) as fh:
            data = json.load(fh)
        if refresh_share is None:
            inst = float(data["warp_instructions_per_launch"])
            us = float(data["capture_us_per_launch"])
        else:
            inst = (refresh_share * float(data["warp_instructions_per_refresh_pass"]) +
                    (1.0 - refresh_share) * float(data["warp_instructions_per_listed_pass"]))
            us = (refresh_share * float(data["capture_us_per_refresh_pass"]) +
                  (1.0 - refresh_share) * float(data["capture_us_per_listed_pass"]))
        peak = 4.0 * 148 * 1965.0e6
    except (OSError, KeyError, ValueError):
        return None
    achieved = inst / (us * 1.0e-6)
    return {"achieved": achieved, "peak": peak, "unit": "warp instructions/s", "frac": achieved / peak,
            "warp_instructions_per_launch": inst, "capture_us_per_launch": us,
            "source": f"profiles/{profile} (ncu smsp__inst_executed.sum and gpu__time_duration.sum, full size)"}


def update_traffic(nodes: int):
    """Per-launch DRAM bytes of the fiber update from the committed ncu
    summary, scaled to `nodes` (traffic grows with the nodes)."""
    path = os.path.join(ROOT, "profiles", "update_traffic.json")
    try:
        with open(path) as fh:
            data = json.load(fh)
        return float(data["dram_bytes_per_launch"]) * nodes / float(data["nodes"])
    except (OSError, KeyError, ValueError, ZeroDivisionError):
        return None


MILESTONES = (0.1, 0.05, 0.03, 0.02, 0.01, 0.001)  # max overlap / d


def time_to_admissible(packed, config, d_min, net, limit):
    """Relaxes a fresh world to the gate (max overlap < tolerance, curvature
    within its limit) or `limit` iterations, recording when the max overlap
    first falls below each milestone; with `net`, the warm start runs first
    (its time included)."""
    import torch

    from tangle_b200.device import DeviceWorld

    world = DeviceWorld(packed, config.cell_list, config.max_step)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    report = None
    if net is not None:
        from tangle_b200.warmstart import warm_start

        report = warm_start(world, net, config)
    reached = {}
    status = None
    while True:
        status = world.run_batch(config, config.iterations_per_batch)
        elapsed = time.perf_counter() - t0
        for m in MILESTONES:
            if m not in reached and status.max_penetration <= m * d_min:
                reached[m] = {"seconds": elapsed, "iterations": status.total_iterations}
        if status.converged or status.total_iterations >= limit:
            break
    out = {"seconds": time.perf_counter() - t0, "iterations": status.total_iterations, "converged": status.converged,
           "max_penetration_over_d": status.max_penetration / d_min,
           "max_curvature_ratio": status.max_curvature_ratio,
           "milestones_over_d": {str(m): reached.get(m) for m in MILESTONES},
           "method": "plain PBD" if net is None else "learned warm start, then plain PBD"}
    if report is not None:
        out["warm_start"] = {"accepted": report.accepted, "seconds": report.seconds, "edges": report.edges,
                             "residual_before": report.residual_before, "residual_after": report.residual_after}
    world.close()
    return out


def arena_time_to_admissible(packs, config, limit):
    """A fresh arena relaxed batch after batch until every specimen's gate
    holds (or `limit` iterations): each specimen's iterations and the wall
    time of the batch in which it first converged, as percentiles."""
    import numpy as np
    import torch

    from tangle_b200.device import DeviceWorld

    world = DeviceWorld.arena(packs, config.cell_list, config.max_step)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    seconds = [None] * len(packs)
    iterations = [None] * len(packs)
    while True:
        status = world.run_batch(config, config.iterations_per_batch)
        elapsed = time.perf_counter() - t0
        for i, st in enumerate(world.specimen_statuses(config)):
            if st.converged and seconds[i] is None:
                seconds[i] = elapsed
                iterations[i] = st.total_iterations
        if all(s is not None for s in seconds) or status.total_iterations >= limit:
            break
    world.close()
    done = [s for s in seconds if s is not None]
    its = [i for i in iterations if i is not None]
    pct = lambda xs, q: float(np.percentile(xs, q)) if xs else None
    return {"specimens": len(packs), "converged": len(done), "seconds": time.perf_counter() - t0,
            "iterations_cap": limit, "seconds_p50": pct(done, 50), "seconds_p90": pct(done, 90),
            "seconds_max": max(done) if done else None, "iterations_p50": pct(its, 50),
            "iterations_p90": pct(its, 90), "iterations_max": max(its) if its else None, "method": "plain PBD"}


PLY_MILESTONES = (0.2, 0.1, 0.05)


def ply_stack_deposition(assembly, packed, config, d_min, plies, budget, net):
    """The 20-ply formation sequence on one resident world: for each ply,
    activate its formation step (the ply was generated in place, one ply
    thickness above the previous), optionally apply the learned warm start to
    the new ply's fibers, and relax until the gate holds or `budget`
    iterations. Returns the whole job's wall time (host-driven, inputs
    resident), per-ply records and the node-iterations done."""
    import numpy as np
    import torch

    from tangle_b200.device import DeviceWorld

    world = DeviceWorld(packed, config.cell_list, config.max_step)
    records = []
    node_iterations = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(plies):
        tk = time.perf_counter()
        _, vertices = world.activate_formation_step(k)
        accepted = None
        if net is not None:
            from tangle_b200.warmstart import warm_start

            new_ply = np.nonzero(np.asarray(packed.fiber_formation_steps) == k)[0]
            accepted = warm_start(world, net, config, fibers=new_ply).accepted
        start = None
        status = None
        reached = {}
        while True:
            status = world.run_batch(config, min(config.iterations_per_batch, budget))
            if start is None:
                start = status.total_iterations - status.batch_iterations
            done = status.total_iterations - start
            for m in PLY_MILESTONES:
                if m not in reached and status.max_penetration <= m * d_min:
                    reached[m] = {"iterations": done, "seconds": time.perf_counter() - tk}
            if status.converged or done >= budget:
                break
        node_iterations += vertices * done
        records.append({"ply": k, "active_vertices": vertices, "iterations": done, "converged": status.converged,
                        "seconds": time.perf_counter() - tk,
                        "max_penetration_over_d": status.max_penetration / d_min,
                        "max_curvature_ratio": status.max_curvature_ratio, "warm_start_accepted": accepted,
                        "milestones_over_d": {str(m): reached.get(m) for m in PLY_MILESTONES}})
    torch.cuda.synchronize()
    seconds = time.perf_counter() - t0
    world.close()
    return seconds, node_iterations, records


def run_ply_stack(args):
    """The 20-ply stack (2 x 2 x 0.1 mm plies, periodic x/y, z walls, 7/19
    um at 15 % per ply, rest curvature up to half the limit, ~2.9 M
    segments), deposited ply by ply on one world, with plain PBD and with the
    learned warm start per ply: whole-job seconds (lower is better) and the
    node-iterations per second of the relaxation."""
    import torch

    from tangle_b200.assembly import PackedAssembly
    from tangle_b200.build import build
    from tangle_b200.generate import ply_stack_specimen
    from tangle_b200.settings import RelaxationSettings

    build()
    torch.cuda.set_device(0)
    assembly = ply_stack_specimen(plies=args.plies, side=args.ply_side)
    packed = PackedAssembly.from_assembly(assembly)
    d_min = assembly.smallest_diameter()
    settings = RelaxationSettings(penetration_tolerance=1.0e-3 * d_min, neighbor_capacity=args.capacity,
                                  max_list_bytes=8 << 30, iterations_per_batch=64, max_iterations=1 << 30)
    config = settings.to_config(d_min)
    runs = {}
    ply_net = os.path.join(ROOT, "tangle_b200", "warmstart_ply_net.npz")
    if os.path.exists(ply_net):
        from tangle_b200.warmstart import WarmStartNet

        net = WarmStartNet.load(ply_net)
    else:
        net = load_warmstart_net()
    for label, use_net in (("plain", None), ("warm_start", net)):
        if label == "warm_start" and net is None:
            continue
        seconds, node_iterations, records = ply_stack_deposition(assembly, packed, config, d_min, args.plies,
                                                                 args.ply_budget, use_net)
        runs[label] = {"seconds": seconds, "node_iterations": node_iterations,
                       "node_iter_per_s": node_iterations / seconds if seconds > 0 else None,
                       "iterations": sum(r["iterations"] for r in records),
                       "plies_converged": sum(1 for r in records if r["converged"]), "plies": records}
    plain = runs["plain"]
    line = {"metric": "s to deposit and relax a 20-ply stack ply by ply (gate: overlap < 1e-3 d per ply)",
            "value": plain["seconds"], "unit": "s", "n_gpus": 1, "higher_is_better": False, "dtype": "f32",
            "data": "synthetic", "impl": "cuda",
            "config": {"workload": (f"ply_stack: {args.plies} plies {args.ply_side * 1e3:g} x {args.ply_side * 1e3:g}"
                                    " x 0.1 mm, periodic xy, z walls, 7/19 um 50:50 by volume at 15 % per ply, "
                                    "xy directions with N(0, 3 deg) tilt, rest curvature up to 0.5 x limit 1/(5d), "
                                    "segment 0.8 d, 1 mm fibers"),
                       "nodes": packed.vertex_count, "segments": packed.segment_count,
                       "fibers": packed.fiber_count, "ply_iteration_cap": args.ply_budget},
            "runs": runs}
    print(json.dumps(line), flush=True)
    return 0


def load_warmstart_net():
    path = os.path.join(ROOT, "tangle_b200", "warmstart_net.npz")
    if not os.path.exists(path):
        return None
    from tangle_b200.warmstart import WarmStartNet

    return WarmStartNet.load(path)


def cpu_model() -> str:
    """The host CPU's model name (from /proc/cpuinfo), or the platform's."""
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.lower().startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform

    return platform.processor() or platform.machine()


def cpu_baseline(packed, config, iterations, d_min=None, start=None, compare=True):
    """The oracle on the same specimen from the same start state (or, for an
    arena, on its first specimens, one after another), all host threads: one
    list-building iteration, then `iterations` timed. With `compare`, a fresh
    CUDA world runs the same iterations from the same state and the line
    carries the parity of the final positions (max |dx| / d and whether they
    are bit-identical)."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    cores = os.cpu_count() or 1
    orc.set_threads(cores)
    packs = packed if isinstance(packed, list) else [packed]
    fixed = type(config)(**{**config.__dict__, "force_full_iterations": True})
    work, elapsed, done = 0.0, 0.0, 0
    parity = None
    for i, p in enumerate(packs):
        world = orc.OracleWorld(p, config.cell_list, config.max_step)
        if start is not None and i == 0:
            world.upload_positions(start)
        world.run_batch(fixed, 1)  # builds the lists
        t0 = time.perf_counter()
        status = world.run_batch(fixed, iterations)
        elapsed += time.perf_counter() - t0
        done = max(status.batch_iterations, 1)
        work += p.vertex_count * done
        if compare and i == 0 and d_min is not None:
            from tangle_b200.device import DeviceWorld

            cuda = DeviceWorld(p, config.cell_list, config.max_step)
            if start is not None:
                cuda.upload_positions(start)
            cuda.run_batch(fixed, 1)
            cuda_status = cuda.run_batch(fixed, iterations)
            po, pd = world.download_positions(), cuda.download_positions()
            cuda.close()
            parity = {"iterations": 1 + iterations,
                      "max_abs_over_d": float(np.abs(po.astype(np.float64) - pd.astype(np.float64)).max()) / d_min,
                      "bit_exact": bool(np.array_equal(po.view(np.uint32), pd.view(np.uint32))),
                      "tolerance_over_d": 1.0e-5,
                      "verdict_identical": bool(status.converged == cuda_status.converged and
                                                status.total_iterations == cuda_status.total_iterations),
                      "specimen": "the first" if len(packs) > 1 else "the benchmarked one"}
        world.close()
    what = "the same specimen" if len(packs) == 1 else f"the first {len(packs)} specimens of the arena"
    state = " from the timed region's start state" if start is not None else ""
    out = {"value": work / elapsed, "unit": UNIT, "cores": cores, "cpu_model": cpu_model(), "kind": "port",
           "sample": f"{done} plain iterations of {what}{state} after one list-building iteration, "
                     f"{elapsed:.1f} s, OpenMP over {cores} threads"}
    if parity is not None:
        out["parity"] = parity
    return out


def run_reference(args):
    rank, world_size, _ = dist_env()
    if rank != 0:
        return 0
    from tangle_b200.assembly import PackedAssembly

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc

    assembly, config, name, d_min = workload(args, 0)
    # The arena's reference is the same algorithm world by world: a bounded
    # sample of its specimens relaxed one after another.
    all_assemblies = assembly if isinstance(assembly, list) else [assembly]
    all_packs = [PackedAssembly.from_assembly(a) for a in all_assemblies]
    packs = all_packs[: args.cpu_specimens]
    cores = os.cpu_count() or 1
    orc.set_threads(cores)
    worlds = [orc.OracleWorld(p, config.cell_list, config.max_step) for p in packs]
    fixed = type(config)(**{**config.__dict__, "force_full_iterations": True})
    per_step = args.reference_iterations
    for _ in range(max(args.warmup, 1)):
        for world in worlds:
            world.run_batch(fixed, per_step)
    t0 = time.perf_counter()
    work = 0.0
    for _ in range(args.steps):
        for p, world in zip(packs, worlds):
            st = world.run_batch(fixed, per_step)
            work += p.vertex_count * st.batch_iterations
    elapsed = time.perf_counter() - t0
    nodes = sum(p.vertex_count for p in packs)
    value = work / elapsed
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * elapsed / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator)",
        "config": bench_config(name, all_packs, config),
        "timing": {"iterations_per_step": per_step, "specimens_timed": len(packs),
                   "start_state": "the initial specimen",
                   "window": f"iterations {max(args.warmup, 1) * per_step} to "
                             f"{(max(args.warmup, 1) + args.steps) * per_step} of the relaxation"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "cpu_model": cpu_model(), "kind": "port",
                         "sample": f"{args.steps} steps of {per_step} iterations of "
                                   + ("the same specimen" if len(packs) == 1
                                      else f"the first {len(packs)} specimens of the arena, one after another")
                                   + f", OpenMP over {cores} threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_cuda(args):
    import numpy as np
    import torch

    rank, world_size, local = dist_env()
    if world_size > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    from tangle_b200.assembly import PackedAssembly
    from tangle_b200.build import build
    from tangle_b200.device import DeviceWorld

    build()
    assembly, config, name, d_min = workload(args, rank)
    batched = isinstance(assembly, list)
    if batched:
        packs = [PackedAssembly.from_assembly(a) for a in assembly]
        packed = None
        nodes = sum(p.vertex_count for p in packs)
        world = DeviceWorld.arena(packs, config.cell_list, config.max_step)
    else:
        packed = PackedAssembly.from_assembly(assembly)
        nodes = packed.vertex_count
        world = DeviceWorld(packed, config.cell_list, config.max_step)
    fixed = type(config)(**{**config.__dict__, "force_full_iterations": True})
    if args.load_positions:
        world.upload_positions(np.load(args.load_positions))
    stream = torch.cuda.ExternalStream(world.stream_handle)

    def barrier():
        torch.cuda.synchronize()
        if world_size > 1:
            torch.distributed.barrier()
            torch.cuda.synchronize()

    # The production batch graphs (one device-side loop per batch) serve the
    # warm-up and the timed steps; per-kernel times come from an instrumented
    # replay of the same steps afterwards.
    for _ in range(args.warmup):
        world.run_batch(fixed, args.iterations)
    # The timed steps start from the initial specimen again (the warm-up
    # batches only capture the graph and load the kernels), the state the
    # reference arm and the CPU baseline start from too; an arena keeps the
    # state the warm-up left. The end-to-end leg and the instrumented replay
    # run the same trajectory from this state.
    host = torch.empty(3 * nodes, dtype=torch.float32, pin_memory=True)
    host_np = host.numpy()
    if not batched and not args.load_positions:
        world.upload_positions(packed.positions)
    world.download_positions(host_np)
    start_state = host_np.copy()
    iterations_done = 0
    rebuilds0 = world.neighbor_list_rebuilds()
    launches0 = world.kernel_launches
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    barrier()
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            start.record(stream)
        for _ in range(args.steps):
            st = world.run_batch(fixed, args.iterations)
            iterations_done += st.batch_iterations
        with torch.cuda.stream(stream):
            end.record(stream)
        end.synchronize()
    launches = world.kernel_launches - launches0
    rebuilds = world.neighbor_list_rebuilds() - rebuilds0
    if args.save_positions and rank == 0:
        np.save(args.save_positions, world.download_positions())
    elapsed_ms = start.elapsed_time(end)
    barrier()
    value, elapsed_s, total_work = replica_throughput(elapsed_ms / 1000.0, float(nodes * iterations_done),
                                                     world_size)
    elapsed_ms = elapsed_s * 1000.0
    clock_summary = clocks.summary()

    # Per-kernel device times: the same steps from the same state, with CUDA
    # events recorded around every step's kernels (an unrolled graph holding
    # the same kernels). One untimed batch captures it first.
    world.set_kernel_timing(True)
    world.upload_positions(start_state)
    world.run_batch(fixed, args.iterations)
    world.upload_positions(start_state)
    bytes_start = contact_bytes(world)
    refreshes0 = world.contact_list_info()["refreshes"]
    contact_ms = update_ms = rebuild_ms = 0.0
    contact_passes = updates = 0
    for _ in range(args.steps):
        world.run_batch(fixed, args.iterations)
        kt = world.last_kernel_times()
        contact_ms += kt["contact_ms"]
        contact_passes += kt["contact_passes"]
        update_ms += kt["update_ms"]
        updates += kt["updates"]
        rebuild_ms += kt["rebuild_ms"]
    bytes_end = contact_bytes(world)
    contact_info = world.contact_list_info()
    refreshes = contact_info["refreshes"] - refreshes0
    world.set_kernel_timing(False)
    host_np[:] = start_state

    # Roofline of the contact pass: the passes' algorithmic bytes (listed and
    # refresh passes weighted by their counts, list sizes averaged over the
    # start and end of the timed region) over their mean duration.
    avg_contact_s = (contact_ms / max(contact_passes, 1)) / 1000.0
    listed_bytes = 0.5 * (bytes_start[0] + bytes_end[0])
    refresh_bytes = 0.5 * (bytes_start[1] + bytes_end[1])
    refresh_share = min(refreshes, contact_passes) / max(contact_passes, 1)
    algorithmic = refresh_share * refresh_bytes + (1.0 - refresh_share) * listed_bytes
    peak, peak_kind = measured_peak()
    achieved = algorithmic / avg_contact_s / 1.0e9 if avg_contact_s > 0 else 0.0
    roofline_contact = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "traffic": ncu_traffic(refresh_share, contact_info["block"] > 0),
                        "peak_source": f"{peak_kind} hbm_gbs", "kernel": "contact_kernel (find_segment_corrections)",
                        "algorithmic_bytes_per_launch": algorithmic, "avg_launch_ms": avg_contact_s * 1000.0,
                        "contact_passes": contact_passes, "refresh_passes": refreshes,
                        "contact_skin_m": contact_info["skin"]}
    if not batched and contact_info["block"] > 0:
        roofline_contact["issue_bound"] = issue_bound("contact_traffic.json", refresh_share)
    # Roofline of the fiber update, the largest kernel (about 55 % of the
    # step): its algorithmic bytes per launch over its mean duration.
    segments = world.segment_count
    avg_update_s = (update_ms / max(updates, 1)) / 1000.0
    update_algorithmic = update_bytes(nodes, segments, contact_info["block"] > 0)
    update_achieved = update_algorithmic / avg_update_s / 1.0e9 if avg_update_s > 0 else 0.0
    roofline = {"bound": "hbm", "achieved": update_achieved, "peak": peak, "unit": "GB/s",
                "frac": update_achieved / peak, "traffic": update_traffic(nodes),
                "peak_source": f"{peak_kind} hbm_gbs",
                "kernel": "fiber_lanes_kernel (internal, contact and curvature corrections)",
                "algorithmic_bytes_per_launch": update_algorithmic, "avg_launch_ms": avg_update_s * 1000.0,
                "launches": updates}
    if not batched:
        roofline["issue_bound"] = issue_bound("update_traffic.json")

    # End to end through the public API with pinned host buffers: the timed
    # steps again, from the same start state, each step uploading the
    # positions, running the batch and downloading the result (which the next
    # step uploads). The batch's graph already exists, so no warm-up is needed.
    e2e = None
    if not args.no_e2e:
        barrier()
        t0 = time.perf_counter()
        done = 0
        for _ in range(args.steps):
            world.upload_positions(host_np)
            st = world.run_batch(fixed, args.iterations)
            world.download_positions(host_np)
            done += st.batch_iterations
        e2e_value, _, _ = replica_throughput(time.perf_counter() - t0, float(nodes * done), world_size)
        e2e = {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 12 * nodes,
               "d2h_bytes_per_step": 12 * nodes + 64}
    # The reference arm's own window of the same trajectory, on the GPU: from
    # the initial specimen, max(W, 1) untimed steps then K timed steps of
    # --reference-iterations iterations each (CUDA events, one host
    # synchronisation per step as there).
    window = None
    if not batched and not args.load_positions:
        world.upload_positions(packed.positions)
        per_step = args.reference_iterations
        for _ in range(max(args.warmup, 1)):
            world.run_batch(fixed, per_step)
        barrier()
        done = 0
        with torch.cuda.stream(stream):
            start.record(stream)
        for _ in range(args.steps):
            done += world.run_batch(fixed, per_step).batch_iterations
        with torch.cuda.stream(stream):
            end.record(stream)
        end.synchronize()
        window_value, _, _ = replica_throughput(start.elapsed_time(end) / 1000.0, float(nodes * done), world_size)
        window = {"value": window_value, "unit": UNIT, "iterations_per_step": per_step, "steps": args.steps,
                  "first_iteration": max(args.warmup, 1) * per_step,
                  "what": "the reference arm's iterations of the same trajectory from the initial specimen, "
                          "timed on the GPU with CUDA events"}
    # The launch-shape autotuner on this workload. After the search, the
    # default and the tuned shapes each time the same steps from the same
    # state on the production graph with CUDA events, alternately and twice
    # each (default, tuned, default, tuned), so that neither gains from
    # running later; each value is the better of its two.
    tuned = None
    if args.autotune or (batched and not args.no_autotune):
        from tangle_b200.autotune import autotune

        default_params = world.launch_params()
        world.upload_positions(start_state)
        choice = autotune(world, fixed, trial_iterations=min(args.iterations, 32), force=True)

        def time_shapes(params):
            world.set_launch_params(params)
            world.upload_positions(start_state)
            world.run_batch(fixed, args.iterations)  # captures this shape's graph
            world.upload_positions(start_state)
            barrier()
            done = 0
            with torch.cuda.stream(stream):
                start.record(stream)
            for _ in range(args.steps):
                done += world.run_batch(fixed, args.iterations).batch_iterations
            with torch.cuda.stream(stream):
                end.record(stream)
            end.synchronize()
            return replica_throughput(start.elapsed_time(end) / 1000.0, float(nodes * done), world_size)[0]

        runs = {"default": [], "tuned": []}
        for _ in range(2):
            runs["default"].append(time_shapes(default_params))
            runs["tuned"].append(time_shapes(choice["params"]))
        tuned = {"default_value": max(runs["default"]), "tuned_value": max(runs["tuned"]), "unit": UNIT,
                 "runs": runs, "timed_region_value": value, "default_params": default_params,
                 "tuned_params": choice["params"], "search": choice["report"],
                 "what": "the timed steps again after the search, from the same state, default and tuned "
                         "launch shapes alternately (two runs each, the better kept)"}
    world.close()

    # Time to admissible from the initial specimen, plain PBD and with the
    # learned warm start first (device-resident, same gates, same cap), for
    # each orientation reading of the mid-size specimen.
    tta = None
    if not args.no_tta and batched:
        tta = {"plain": arena_time_to_admissible(packs, config, args.tta_iterations)}
    elif not args.no_tta:
        from tangle_b200.generate import mid_size_specimen

        net = load_warmstart_net()
        betas = [float(b) for b in args.tta_betas.split(",") if b.strip()] or [args.beta]
        tta = {}
        for beta in betas:
            if args.workload == "mid_size" and abs(beta - args.beta) > 1.0e-9:
                spec = PackedAssembly.from_assembly(mid_size_specimen(scale=args.scale, seed=1 + rank, beta=beta))
            else:
                spec = packed
            entry = {"specimen": beta_label(beta),
                     "plain": time_to_admissible(spec, config, d_min, None, args.tta_iterations)}
            if net is not None:
                entry["warm_start"] = time_to_admissible(spec, config, d_min, net, args.tta_iterations)
            else:
                entry["warm_start"] = {"unavailable": "no trained network (tangle_b200/warmstart_net.npz)"}
            tta["beta_" + f"{beta:.2f}".rstrip("0").rstrip(".").replace(".", "_")] = entry

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu:
        cpu = cpu_baseline(packs[: args.cpu_specimens] if batched else packed, config, args.cpu_iterations,
                           d_min=d_min, start=np.load(args.load_positions) if args.load_positions else None)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world_size, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded generator)",
            "config": bench_config(name, packs if batched else [packed], config),
            "timing": {"iterations_per_step": args.iterations,
                       "start_state": ("the state after the warm-up steps" if batched or args.load_positions
                                       else "the initial specimen"),
                       "l2": "inputs larger than L2 (positions, geometry and lists exceed 126 MB)",
                       "parallelism": f"replicas x{world_size}"},
            "gpu_launches": int(launches),
            "neighbor_list_rebuilds": int(rebuilds),
            "kernel_ms": {"contact": contact_ms, "update": update_ms, "rebuild_and_gated": rebuild_ms},
            "roofline": roofline,
            "roofline_contact": roofline_contact,
            "clocks": clock_summary,
            "e2e": e2e,
            "reference_window": window,
            "autotune": tuned,
            "time_to_admissible": tta,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world_size > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def measured_tensor_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def run_gemm(args):
    """tgl_gemm_bf16 (the warm-start network's tensor-core kernel) timed with
    CUDA events on the network's own shapes at the mid-size specimen's scale
    (rows = directed contact edges or vertices, the layer widths as N and
    K) and on one large square-ish product, against the measured HBM and
    bf16 peaks. Each shape: 3 untimed launches, then the mean of --steps."""
    import ctypes

    import torch

    from tangle_b200.build import build
    from tangle_b200.device import load_library

    build()
    torch.cuda.set_device(0)
    lib = load_library()

    class Gemm(ctypes.Structure):
        _fields_ = [("a", ctypes.c_void_p), ("b", ctypes.c_void_p), ("lda", ctypes.c_int64), ("ldb", ctypes.c_int64),
                    ("m", ctypes.c_int32), ("n", ctypes.c_int32), ("k", ctypes.c_int64), ("a_mn", ctypes.c_int32),
                    ("b_mn", ctypes.c_int32), ("k_split", ctypes.c_int64), ("bias", ctypes.c_void_p),
                    ("relu", ctypes.c_int32), ("reserved", ctypes.c_int32), ("mask", ctypes.c_void_p),
                    ("ld_mask", ctypes.c_int64), ("residual", ctypes.c_void_p), ("ld_res", ctypes.c_int64),
                    ("out_f32", ctypes.c_void_p), ("ldo", ctypes.c_int64), ("out_bf16", ctypes.c_void_p),
                    ("ldo_bf16", ctypes.c_int64), ("error", ctypes.c_void_p)]

    fn = lib.tgl_gemm_bf16
    fn.argtypes = [ctypes.POINTER(Gemm), ctypes.c_void_p]
    fn.restype = ctypes.c_int
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    hbm, hbm_kind = measured_peak()
    tensor, tensor_kind = measured_tensor_peak()
    rows = lambda m: max(128, int(m * args.gemm_scale))
    shapes = [
        # (label, m, n, k): forward products, K-major operands, bf16 output.
        ("edge MLP layer 1 (E x 80 -> 64)", rows(16_000_000), 64, 80),
        ("edge MLP layer 2 (E x 64 -> 64)", rows(16_000_000), 64, 64),
        ("node MLP layer 1 (V x 192 -> 64)", rows(2_000_000), 64, 192),
        ("large product (16384 x 8192 -> 256)", 16384, 256, 8192),
    ]
    results = []
    for label, m, n, k in shapes:
        a = (torch.randn(m, k, device=dev) * 0.1).to(torch.bfloat16)
        b = (torch.randn(n, k, device=dev) * 0.1).to(torch.bfloat16)
        out = torch.empty(m, n, dtype=torch.bfloat16, device=dev)
        err = torch.zeros(1, dtype=torch.int32, device=dev)
        g = Gemm(a.data_ptr(), b.data_ptr(), k, k, m, n, k, 0, 0, 0, None, 0, 0, None, 0, None, 0, None, n,
                 out.data_ptr(), n, err.data_ptr())
        for _ in range(3):
            assert fn(ctypes.byref(g), stream.cuda_stream) == 0, lib.tgl_last_error()
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(args.steps):
            fn(ctypes.byref(g), stream.cuda_stream)
        end.record(stream)
        end.synchronize()
        assert int(err.item()) == 0
        seconds = start.elapsed_time(end) / 1000.0 / args.steps
        flops = 2.0 * m * n * k
        traffic = 2.0 * (m * k + n * k + m * n)  # bf16 operands read once, bf16 result written
        ref = (a[:4096].float() @ b.float().T)
        rel = float(((out[:4096].float() - ref).abs().max() / (ref.abs().max() + 1e-30)).item())
        results.append({"shape": label, "m": m, "n": n, "k": k, "ms": seconds * 1000.0,
                        "tflops": flops / seconds / 1.0e12, "tensor_frac": flops / seconds / 1.0e12 / tensor,
                        "gbs": traffic / seconds / 1.0e9, "hbm_frac": traffic / seconds / 1.0e9 / hbm,
                        "max_rel_err_vs_f32": rel})
        del a, b, out
    line = {"metric": "tgl_gemm_bf16 throughput on the warm-start network's shapes", "impl": "cuda",
            "unit": "TFLOP/s", "value": max(r["tflops"] for r in results), "steps": args.steps,
            "dtype": "bf16 operands, f32 accumulate (tensor memory)", "data": "synthetic normal operands",
            "peaks": {"bf16_tflops": tensor, "bf16_source": tensor_kind, "hbm_gbs": hbm, "hbm_source": hbm_kind},
            "shapes": results}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "ply_stack":
        return run_ply_stack(args)
    if args.workload == "gemm":
        return run_gemm(args)
    return run_cuda(args)


if __name__ == "__main__":
    sys.exit(main())
