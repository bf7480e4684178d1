"""Benchmark: body-substeps/s of the Solver6DOF substep on the 100k-box pile.

Workload (the metric's configuration): 100,000 OBBs, half extents uniform in
[0.2, 0.4] m, random orientations, density 1000, on a 100x100x10 jittered
grid (1.4 m spacing) over a floor, one box in 500 corner-pinned with a
breakable pin (5e4 N); dt 1/60, 4 substeps, 10 iterations + post-stabilization,
Jones-Plassmann coloring.  The pile is settled (untimed) before the warm-up so
the timed frames run on a resting pile (~1M dynamic contact rows).

A "step" is one frame (4 substeps).  value = bodies x substeps x steps / device
time of the timed steps (CUDA events on the solver's stream, L2 flushed between
steps outside the events); with torchrun, N independent replicas (one pile per
GPU, no collective in the loop) and the max time over ranks.

`--impl reference` times the CPU port of the reference substep (the oracle:
the C++ restatement, which reproduces the reference's own kernels bit for bit;
the reference's Warp CPU path itself cannot be installed here) on all host
cores, on the same settled 100k pile (state prepared untimed on the GPU), one
substep per step; a 20x20x10 tile on all cores and on one core is reported
beside it.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "body-substeps/s @100k boxes; iters to 1e-4 m violation, learned vs plain λ0"
UNIT = "body-substeps/s"
PARAMS = dict(dt=1.0 / 60.0, iterations=10, substeps=4, friction_static_mult=1.25, coloring_mode="jones_plassmann")
FULL = dict(nx=100, nz=100, ny=10)
SAMPLE = dict(nx=20, nz=20, ny=10)


def dyn_bodies(s) -> int:
    return int(sum(1 for m in s._mass if m > 0.0))


# ---------------------------------------------------------------------------
# Per-launch algorithmic bytes (the per-unit figures of the survey's
# measurement section; units from the live counters of the same run).
# ---------------------------------------------------------------------------
def algorithmic_bytes(n_bodies: int, r1: int, r2: int, n_pairs: int, pairs_with_contacts: int, contacts: int,
                      iterations: int) -> dict:
    T = iterations + 1
    solve = (n_bodies * 184 + (r1 + r2) * (124 + 24) + T * (n_bodies * 112 + r1 * 44 + 2 * r2 * 84)
             + (T - 1) * (r1 * 100 + r2 * 128) + n_bodies * 104 + contacts * 64)
    collide = n_bodies * 64 + n_pairs * 108 + pairs_with_contacts * 140 + contacts * (3 * 72 + 40)
    return {"solve": solve, "collide": collide, "substep": solve + collide}


def collision_stage_bytes(n: int, pairs: int, pairs_with: int, contacts: int) -> dict:
    """Algorithmic bytes of each collision stage (what the stage must read
    and write at least once; N bodies, P pairs, Pc pairs with contacts, K
    contacts = dynamic groups, 2K incidences):
      k_aabb       N x (pose 32 + half extents 16 + box out 32)           80 N
      k_morton     N x (box 32 + code 4 + index 4)                        40 N
      radix_sort   4 passes x N x (keys+indices in 8 + out 8 + hist 4)    80 N
      k_lbvh_build (N-1) x (4 codes 16 + children/parent 16)             32 (N-1)
      k_lbvh_leaves N x (box in 32 + leaf box out 32)                     64 N
      k_lbvh_refit (N-1) x (2 child boxes 64 + box out 32)               96 (N-1)
      k_lbvh_pack  (N-1) x (children and grandchildren indices 24 + four
                   entry boxes 128 + leaf body and mass lookups 40 + record
                   out 128)                                            320 (N-1)
      k_bp_count   N x (own box 32 + count 4) + packed tree 128 (N-1)
      k_bp_fill    as k_bp_count + pairs out 8 P
      k_narrow     108 P + 140 Pc (two poses and extents, SAT / manifold out)
      k_emit       K x (3 rows x 72 + cache probe 40)                    256 K
      scans        12 B per scanned element (read twice, write once)
      k_dg_fill    4 N (zero) + K x (bodies 8) + 2K x (entry 8)     4 N + 24 K
      k_dg_sort    2K x (entry 8 read + 8 write)                          32 K"""
    tree = 128 * max(n - 1, 0)
    return {"k_aabb": 80 * n, "k_morton": 40 * n, "radix_sort": 80 * n, "k_lbvh_build": 32 * max(n - 1, 0),
            "k_lbvh_leaves": 64 * n, "k_lbvh_refit": 96 * max(n - 1, 0), "k_lbvh_pack": 320 * max(n - 1, 0),
            "k_bp_count": 36 * n + tree, "scan_pair_offsets": 12 * n, "k_bp_fill": 36 * n + tree + 8 * pairs,
            "k_narrow": 108 * pairs + 140 * pairs_with, "scan_contact_offsets": 24 * pairs, "k_emit": 256 * contacts,
            "scan_incidence_offsets": 12 * n, "k_dg_fill": 4 * n + 24 * contacts, "k_dg_sort": 32 * contacts}


def collision_report(s, substeps: int = 8) -> dict:
    """Per-stage device time (event-record nodes between the stages of a
    one-off graph of the pipeline) over
    `substeps` profiled substeps -- one LBVH rebuild and the refits between
    -- with algorithmic GB/s from collision_stage_bytes."""
    acc: dict = {}
    for _ in range(substeps):
        for k, v in s.collision_profile().items():
            acc.setdefault(k, []).append(v)
    st = s.stats()
    p = s.pairs()
    nb = len(s._x)
    by = collision_stage_bytes(nb, int(st["n_pairs"]), int(np.sum(p["count"] > 0)), int(st["n_dyn_groups"]))
    out = {}
    for k, v in acc.items():
        ms = float(np.mean(v))
        row = {"ms": round(ms, 4), "runs_per_substep": round(len(v) / substeps, 3)}
        if k in by and ms > 0:
            row["gb_per_s"] = round(by[k] / (ms * 1e-3) / 1e9, 1)
        out[k] = row
    total = sum(r["ms"] * r["runs_per_substep"] for r in out.values())
    return {"stages": out, "ms_per_substep": round(total, 4),
            "note": "one-off graph of the pipeline with an event-record node after each stage; scans are three launches each"}


def barrier_sweep_report(s) -> dict:
    """Per-color pass time of the grid-barrier sweep (the option the flag
    sweep replaces): one substep with phase stamps (globaltimer after each
    grid barrier)."""
    keep = (s.flag_sweep, s.timing)
    s.flag_sweep, s.timing = False, True
    try:
        s.substep()
        ph = s.phase_profile()
        s.substep()
        ph = s.phase_profile()
    finally:
        s.flag_sweep, s.timing = keep
    ms, passes = ph.get("primal", (0.0, 0))
    return {"passes": passes, "ms_per_pass": ms / max(1, passes), "primal_ms": ms,
            "phases_ms": {k: round(v[0], 4) for k, v in ph.items()}}


# ---------------------------------------------------------------------------
# nvidia-smi clock sampler (runs during the timed region).
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        # nvidia-smi numbers GPUs physically: map the CUDA ordinal through
        # CUDA_VISIBLE_DEVICES (index or UUID) when it is set.
        vis = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
        self.gpu = vis[gpu_index] if gpu_index < len(vis) else str(gpu_index)
        self.proc = None
        self.lines = []

    def start(self, wait_s: float = 3.0):
        """Starts sampling every 50 ms; returns once the first sample is in
        (or after wait_s), so the timed region that follows is covered."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while not self.lines and time.time() - t0 < wait_s:
            time.sleep(0.01)
        self.lines.clear()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (C++ restatement of the reference substep, FP32,
# OpenMP), which reproduces the reference's own kernels bit for bit
# (tests/test_reference_pin.py).
# ---------------------------------------------------------------------------
def cpu_rate(steps: int, warmup: int, threads: int, settle: int = 120, also_threads=()) -> dict:
    """The port on a 20x20x10 tile of the pile, settled on the CPU with all
    `threads`; then `steps` frames are timed with `threads` and with each
    count in `also_threads` (reported under "by_threads")."""
    from avbd_b200 import scenes
    from oracle.oracle import OracleSolver6DOF
    s = OracleSolver6DOF(precision="float32", threads=threads, **PARAMS)
    scenes.pile(s, **SAMPLE)
    for _ in range(settle + warmup):
        s.step()
    nb = dyn_bodies(s)
    c = s.counts()
    by = {}
    for th in (threads, *also_threads):
        s.threads = th
        t0 = time.perf_counter()
        for _ in range(steps):
            s.step()
        by[th] = time.perf_counter() - t0
    s.threads = threads
    dt = by[threads]
    return {"value": nb * PARAMS["substeps"] * steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"{SAMPLE['nx']}x{SAMPLE['nz']}x{SAMPLE['ny']} tile of the pile ({nb} boxes, "
                       f"{c['n_rows'] - c['n_static']} dynamic rows), settled {settle} frames, "
                       f"{steps} timed frames; FP32 C++ restatement of the reference substep"),
            "seconds": dt, "by_threads": {str(th): nb * PARAMS["substeps"] * steps / t for th, t in by.items()}}


def settled_pile_state(settle: int, size=None) -> dict:
    """The benchmark pile settled on the GPU by this package (untimed input
    preparation: settling 100k boxes for 240 frames would take the port the
    better part of an hour).  Returns the Solver6DOF state_dict."""
    from avbd_b200 import Solver6DOF, scenes
    s = Solver6DOF(**PARAMS)
    scenes.pile(s, **(size or FULL))
    for _ in range(settle):
        s._enqueue_step()
    s._after_frame()
    sd = s.state_dict()
    del s
    return sd


def port_full_rate(sd: dict, substeps: int, warmup: int, threads: int, size=None, settle: int = 240) -> dict:
    """The port on the full settled pile: the state is loaded into the
    oracle's FP32 build, `warmup` substeps run untimed, then `substeps`
    substeps are timed (one substep is a bounded sample of one frame)."""
    from avbd_b200 import scenes
    from oracle.oracle import OracleSolver6DOF
    size = size or FULL
    s = OracleSolver6DOF(precision="float32", threads=threads, **PARAMS)
    scenes.pile(s, **size)
    s._flush()
    s.set_bodies(sd["x"], sd["q"], sd["v"], sd["w"], sd["pv"], sd["pw"])
    s.set_static_rows(sd["row_lam"], sd["row_pen"], sd["row_active"], sd["row_was"])
    s.set_cache(sd["cache_abc"], sd["cache_state"])
    s.set_colors(sd["colors"], sd["n_colors"], sd["color_dirty"])
    for _ in range(warmup):
        s.substep()
    nb = dyn_bodies(s)
    t0 = time.perf_counter()
    for _ in range(substeps):
        s.substep()
    dt = time.perf_counter() - t0
    c = s.counts()
    return {"value": nb * substeps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": (f"full {size['nx']}x{size['nz']}x{size['ny']} pile ({nb} boxes, "
                       f"{c['n_rows'] - c['n_static']} dynamic rows, {c['n_pairs']} pairs) settled {settle} frames "
                       f"(state prepared untimed on the GPU), {substeps} timed substeps after {warmup} warm-up "
                       "substeps; FP32 C++ restatement of the reference substep"),
            "seconds": dt, "dyn_rows": c["n_rows"] - c["n_static"]}


def run_reference(args) -> None:
    """The reference arm: the port of the reference substep on the host
    cores, on the same settled 100k pile as the GPU arm (one substep per
    step), with the tile sample on all cores and on one core beside it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    extra = {}
    try:
        import torch
        have_gpu = torch.cuda.is_available()
    except Exception:
        have_gpu = False
    if have_gpu:
        sd = settled_pile_state(args.settle)
        r = port_full_rate(sd, args.steps, args.warmup, threads, settle=args.settle)
        same = True
        workload = ("pile 100x100x10 (100000 OBBs, he U[0.2,0.4], 200 corner pins fracture 5e4), dt 1/60, "
                    "4 substeps, 10 iterations + post-stab, JP coloring; one substep per step")
    else:  # no GPU to prepare the settled state: the tile alone
        r = cpu_rate(args.steps, args.warmup, threads)
        same = False
        extra["same_config_reason"] = "no GPU to prepare the settled 100k pile; 20x20x10 tile timed instead"
        workload = "pile tile 20x20x10 (bounded sample)"
    tile = cpu_rate(3, 2, threads, also_threads=(1,))
    extra["tile"] = {"sample": tile["sample"], "body_substeps_per_s_by_threads": tile["by_threads"]}
    line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * r["seconds"] / max(1, args.steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "same_config": same,
            "config": {"workload": workload, "sample": r["sample"]},
            "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": r["sample"]},
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            **extra}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Second half of the metric: iterations to a violation tolerance, learned vs
# plain (zero) warm start of new contacts.
# ---------------------------------------------------------------------------
def warm_start_eval(seeds=tuple(range(1000, 1010)), frames=(240, 400), iterations=256) -> dict:
    """Held-out 16x16x8 piles of the benchmark distribution (the shipped
    network was trained on seeds 0..49), at two snapshots each: one substep
    of up to 256 iterations from the plain zero start and from the learned
    start (both with the contact cache emptied, so every contact is new) and
    from the full contact cache.  Score: iterations until the max violation
    over all rows <= 1e-4 m (257 = not reached); the max over the box-box
    contact rows alone beside it."""
    from avbd_b200.learned import WarmStartMLP
    from avbd_b200.train_warm_start import make_pile, score_snapshot, snapshots, summarize
    model = WarmStartMLP.load()
    rows = []
    for seed in seeds:
        s = make_pile(seed, 16, 16, 8, model=model)
        for f in snapshots(s, frames):
            rows.append(dict(seed=seed, frame=f, **score_snapshot(s, iterations)))
    d = summarize(rows)
    return {"workload": (f"held-out 16x16x8 piles, seeds {seeds[0]}..{seeds[-1]}, frames {list(frames)}, one "
                         "substep from each start"),
            "max_iterations": iterations,
            "iters_to_1e-4m_max_violation": {"plain": d["plain_max_iters"], "learned": d["learned_max_iters"],
                                              "cached": d["cached_max_iters"],
                                              "learned_reduction": d["learned_max_reduction"],
                                              "cached_reduction": d["cached_max_reduction"]},
            "iters_to_1e-4m_max_box_contact_violation": {"plain": d["plain_box_iters"],
                                                          "learned": d["learned_box_iters"],
                                                          "cached": d["cached_box_iters"]},
            "learned_applied_fraction": d["applied_fraction"]}


def warm_start_throughput(s, frames: int, warm: int = 3) -> dict:
    """Body-substeps/s of the benchmark pile with the learned warm start on
    and off (the network attached; `enabled` toggled), device time."""
    import torch
    from avbd_b200.learned import WarmStartMLP
    model = WarmStartMLP.load()
    s.warm_start = model
    st = s._cuda_stream
    nb = dyn_bodies(s)
    out = {}
    for arm, on in (("learned", True), ("plain", False)):
        model.enabled = on
        for _ in range(warm):
            s.step()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(st):
            t0.record(st)
        for _ in range(frames):
            s._enqueue_step()
        with torch.cuda.stream(st):
            t1.record(st)
        s._after_frame()
        out[arm] = nb * PARAMS["substeps"] * frames / (t0.elapsed_time(t1) / 1e3)
    s.warm_start = None
    return {"body_substeps_per_s": out, "frames": frames, "learned_vs_plain": out["learned"] / out["plain"]}


def batched_summary(frames: int = 5, seq_frames: int = 3, settle: int = 60) -> dict:
    """The batched-scenes comparison in a form short enough for the main
    bench line: the 512 scenes batched (one CUDA graph per frame, lanes per
    body 4 with the flag sweep), and the same 512 scenes as 512 Solver6DOF
    stepped one at a time.  The single solvers start from the batch's
    settled bodies (positions, orientations, velocities copied per scene,
    so the 512 of them need not settle again); each runs 4 untimed frames
    (contacts, cache and coloring rebuild, and every LBVH rebuild pattern's
    frame graph is captured) before its timed ones."""
    import torch
    from avbd_b200.batch import c4_batch, c4_single, c4_specs
    specs = c4_specs(512, seed=0)
    b = c4_batch(specs)
    b.solver.primal_group_size = 4
    for _ in range(settle):
        b.solver._enqueue_step()
    b.solver._after_frame()
    for _ in range(2):
        b.step()
    st = b.solver._cuda_stream
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(st):
        t0.record(st)
    for _ in range(frames):
        b.solver._enqueue_step()
    with torch.cuda.stream(st):
        t1.record(st)
    b.solver._after_frame()
    ms_b = t0.elapsed_time(t1) / frames
    value_b = b.body_substeps_per_frame() / (ms_b * 1e-3)
    x, q, v, w = b.solver.x4, b.solver.q, b.solver.v4, b.solver.w4
    singles = []
    for sc, spec in zip(b.scenes, specs):
        s1 = c4_single(spec)
        s1._flush()
        idx = torch.as_tensor([bd.index for bd in sc.bodies], device=x.device)
        org = torch.as_tensor(np.append(sc.origin, 0.0), dtype=torch.float32, device=x.device)
        with torch.cuda.stream(s1._cuda_stream):
            s1.x4[: len(idx)].copy_(x[idx] - org)
            s1.q[: len(idx)].copy_(q[idx])
            s1.v4[: len(idx)].copy_(v[idx])
            s1.w4[: len(idx)].copy_(w[idx])
        singles.append(s1)
    torch.cuda.synchronize()
    for _ in range(4):
        for s1 in singles:
            s1._enqueue_step()
        for s1 in singles:
            s1._after_frame()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(seq_frames):
        for s1 in singles:
            s1._enqueue_step()
        for s1 in singles:
            s1._cuda_stream.synchronize()
    e1.record()
    torch.cuda.synchronize()
    ms_s = e0.elapsed_time(e1) / seq_frames
    units = sum(sum(1 for m in s1._mass if m > 0) * s1.substeps for s1 in singles)
    value_s = units / (ms_s * 1e-3)
    return {"workload": ("512 scenes, bodies log-uniform [16, 2048] (OBB heaps with 4 walls), substeps {2,4,8}, "
                         f"iterations {{5,10,20}}, settled {settle} frames; batched: one CUDA graph per frame; "
                         "one at a time: 512 Solver6DOF, one frame graph each, frames enqueued back to back"),
            "batched": {"value": value_b, "ms_per_frame": ms_b},
            "one_at_a_time": {"value": value_s, "ms_per_frame": ms_s},
            "speedup": value_b / value_s, "unit": UNIT}


# ---------------------------------------------------------------------------
# Multi-GPU: replicas only.  Each rank runs its own pile; the only collective
# is this max of the per-rank timings (the job is as fast as its slowest rank).
# ---------------------------------------------------------------------------
def max_over_ranks(v: float, world: int, device) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_units(bodies_per_rank: int, substeps: int, steps: int, world: int) -> int:
    """Body-substeps of the whole job: every rank steps its own replica."""
    return bodies_per_rank * substeps * steps * world


# ---------------------------------------------------------------------------
# GPU arm.
# ---------------------------------------------------------------------------
def run_gpu(args) -> None:
    import torch
    import torch.distributed as dist
    from avbd_b200 import Solver6DOF, scenes

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    size = dict(FULL) if not args.small else dict(nx=40, nz=40, ny=10)
    s = Solver6DOF(device=str(dev), **PARAMS)
    if args.row_capacity:
        s.dyn_row_capacity = args.row_capacity  # smaller arena for profiler captures
    if args.group_size:
        s.primal_group_size = args.group_size
    if args.blocks_per_sm:
        s.blocks_per_sm = args.blocks_per_sm
    if args.sweep:
        s.flag_sweep = args.sweep == "flags"
        s.adaptive_lanes = args.sweep == "barrier-adaptive"
    if args.no_resting_floor:
        s.resting_floor = False
    t_build = time.perf_counter()
    scenes.pile(s, **size)  # the caller's add_box / add_floor_contact_box / add_pin_corner calls
    t_api = time.perf_counter()
    s._flush()  # the library's build: arena, body arrays, static groups on the device, upload
    s.stream.synchronize()
    t_flush = time.perf_counter() - t_api
    t_api -= t_build
    t_build = t_api + t_flush
    nb = dyn_bodies(s)
    for _ in range(args.settle):
        s._enqueue_step()
    s._after_frame()
    tuned = None
    if args.tune and not (args.group_size or args.blocks_per_sm or args.sweep):
        from avbd_b200.autotune import autotune
        tuned = autotune(s)  # launch shape for this scene; the scene state is restored
    for _ in range(args.warmup):
        s.step()
    stream = s._cuda_stream
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    if args.profile:
        torch.cuda.profiler.start()
    k0 = s.stats()["kernels_launched"]
    coll_list, solve_list = [], []
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            ev[k][0].record(stream)
        s._enqueue_step()
        with torch.cuda.stream(stream):
            ev[k][1].record(stream)
        s._after_frame()
        # device time of the frame's last substep, per part (events on the
        # solver's stream between the collision and solve graph launches)
        coll_list.append(s.broadphase_ms)
        solve_list.append(s.solve_ms)
    barrier()
    if args.profile:
        torch.cuda.profiler.stop()
    kernels = s.stats()["kernels_launched"] - k0
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    st = s.stats()
    coll_ms, solve_ms = float(np.mean(coll_list)), float(np.mean(solve_list))

    # end to end through the public API: pinned host state in, step, poses out
    n = len(s._x)
    pin_in = [torch.empty((n, 4), dtype=torch.float32).pin_memory() for _ in range(4)]
    pin_out = [torch.empty((n, 4), dtype=torch.float32).pin_memory() for _ in range(2)]
    with torch.cuda.stream(stream):
        for h, t in zip(pin_in, (s.x4, s.q, s.v4, s.w4)):
            h.copy_(t[:n], non_blocking=True)
    stream.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.upload_body_state(*pin_in)
        s.step()
        s.download_poses(*pin_out)
    barrier()
    e2e_s = time.perf_counter() - t0
    h2d = sum(int(t.numel() * 4) for t in pin_in)
    d2h = sum(int(t.numel() * 4) for t in pin_out)

    ms = max_over_ranks(ms, world, dev)
    e2e_s = max_over_ranks(e2e_s, world, dev)
    units = job_units(nb, PARAMS["substeps"], args.steps, world)
    value = units / (ms / 1e3)
    e2e_value = units / e2e_s
    r1 = len(s._rows)
    r2 = int(st["n_dyn_rows"])
    p = s.pairs()
    pairs_with = int(np.sum(p["count"] > 0))
    ab = algorithmic_bytes(n, r1, r2, int(st["n_pairs"]), pairs_with, int(st["n_dyn_groups"]), PARAMS["iterations"])
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = ab["solve"] / (solve_ms / 1e3) / 1e9 if solve_ms > 0 else 0.0
    # DRAM bytes of one solve launch from an ncu capture of this workload
    # (dram__bytes_read.sum + dram__bytes_write.sum), committed with its
    # command; the capture's pile settled fewer frames, so its bytes are
    # scaled by the ratio of the two launches' algorithmic bytes
    traffic = None
    tf = os.path.join(ROOT, "profiles", "solve_traffic.json")
    if os.path.exists(tf) and not args.small:
        try:
            cap = json.load(open(tf))
            traffic = cap["bytes_per_launch"] * ab["solve"] / cap.get("algorithmic_bytes_per_launch", ab["solve"])
        except Exception:
            traffic = None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": (f"pile {size['nx']}x{size['nz']}x{size['ny']} ({nb} OBBs, he U[0.2,0.4], "
                                f"{sum(1 for g in s._groups if g[0] == 1)} corner pins fracture 5e4), dt 1/60, "
                                "4 substeps, 10 iterations + post-stab, JP coloring; settled "
                                f"{args.settle} frames before warm-up"),
                   "global_batch": nb * world, "seq_len": None, "parallelism": f"replicas x{world}",
                   "l2": "flushed (256 MiB write) between timed steps, outside the events",
                   "live": {"dyn_rows": r2, "static_rows": r1, "pairs": int(st["n_pairs"]),
                            "contacts": int(st["n_dyn_groups"]), "colors": int(st["n_colors"])},
                   "launch_shape": {"group_size": s.primal_group_size, "blocks_per_sm": s.blocks_per_sm,
                                    "flag_sweep": bool(s.flag_sweep), "adaptive_lanes": bool(s.adaptive_lanes),
                                    "autotuned": tuned is not None},
                   "scene_build_s": {"total": round(t_build, 3), "api_calls": round(t_api, 3),
                                     "flush": round(t_flush, 3)}},
        "roofline": {"bound": "hbm", "kernel": "solve (k_solve_persistent head + k_flag_sweep + tail)", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "algorithmic_bytes_per_launch": ab["solve"], "launch_ms": solve_ms,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(kernels),
        "clocks": clk,
        "phase_ms_per_substep": {"collide": coll_ms, "solve": solve_ms},
    }
    line["collision_kernels"] = collision_report(s)
    line["barrier_sweep"] = barrier_sweep_report(s)
    if tuned is not None:
        line["autotune_ms_per_frame"] = {
            (f"G{r['group_size']}x{r['blocks_per_sm']}{'-flags' if r['flag_sweep'] else ''}"
             f"{'-adapt' if r['adaptive_lanes'] else ''}"): round(r["ms_per_frame"], 3)
            for r in tuned["table"]}
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        # the port on this run's own settled pile (the GPU state loaded into
        # the oracle), a few substeps: the same configuration as `value`
        cb = port_full_rate(s.state_dict(), substeps=3, warmup=1, threads=threads, size=size, settle=args.settle)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if rank == 0 and world == 1 and not args.no_batched:
        line["batched_scenes_512"] = batched_summary()
    if rank == 0 and not args.no_warm_start:
        line["warm_start"] = warm_start_eval()
        line["warm_start"]["throughput_100k_pile"] = warm_start_throughput(s, frames=10)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_batched(args) -> None:
    """Batched scenes: 512 independent scenes (bodies log-uniform in
    [16, 2048], OBB heap distribution, per-scene friction, substeps in
    {2, 4, 8}, iterations in {5, 10, 20}) stepped by one solver -- a frame
    is one CUDA graph: every substep slot's collision launches and persistent
    solve -- against launching the scenes one at a time (one Solver6DOF
    each, every scene's frame enqueued back to back, one synchronisation per
    frame), on the first `--seq-scenes` scenes (default all 512) for the
    ratio."""
    import torch
    import torch.distributed as dist
    from avbd_b200.autotune import autotune
    from avbd_b200.batch import c4_batch, c4_single, c4_specs

    # Several GPUs: the scenes are dealt round-robin to the ranks (scenes are
    # independent: no collective in the loop); the job's rate is all ranks'
    # body-substeps over the slowest rank's time.
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    specs = c4_specs(512, seed=0)[rank::world]
    dev = torch.device("cuda", local)

    def time_frames(step_all, sync, frames):
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        t0.record()
        for _ in range(frames):
            step_all()
        sync()
        t1.record()
        torch.cuda.synchronize(dev)
        return t0.elapsed_time(t1) / 1e3

    def batched(spec_list, frames):
        b = c4_batch(spec_list)
        for _ in range(args.settle_batched):
            b.solver._enqueue_step()
        b.solver._after_frame()
        tuned = autotune(b.solver) if not args.no_tune else None
        for _ in range(args.warmup):
            b.step()
        st = b.solver._cuda_stream
        k0 = b.stats()["kernels_launched"]
        sec = time_frames(lambda: b.solver._enqueue_step(), lambda: st.synchronize(), frames)
        b.solver._after_frame()
        units = b.body_substeps_per_frame() * frames
        return {"value": units / sec, "ms_per_frame": 1e3 * sec / frames,
                "launches_per_frame": (b.stats()["kernels_launched"] - k0) / frames,
                "bodies": len(b.solver._mass), "static_rows": len(b.solver._rows),
                "launch_shape": tuned["best"] if tuned else None}

    def one_at_a_time(spec_list, frames):
        ss = [c4_single(sp) for sp in spec_list]
        for s in ss:
            for _ in range(args.settle_batched):
                s._enqueue_step()
            s._after_frame()
            for _ in range(args.warmup):
                s.step()

        def step_all():
            for s in ss:
                s._enqueue_step()

        def sync():
            for s in ss:
                s._cuda_stream.synchronize()

        sec = time_frames(step_all, sync, frames)
        for s in ss:
            s._after_frame()
        units = sum(sum(1 for m in s._mass if m > 0) * s.substeps for s in ss) * frames
        return {"value": units / sec, "ms_per_frame": 1e3 * sec / frames}

    full = batched(specs, args.steps)
    if world > 1:
        units = torch.tensor([full["value"] * full["ms_per_frame"]], dtype=torch.float64, device=dev)
        dist.all_reduce(units)  # body-substeps per ms-frame summed over ranks
        slowest = max_over_ranks(full["ms_per_frame"], world, dev)
        full["value"] = float(units.item()) / slowest
        full["ms_per_frame"] = slowest
        dist.barrier()
        dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"metric": "body-substeps/s, 512 batched scenes", "value": full["value"], "unit": UNIT,
                              "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                              "ms_per_step": full["ms_per_frame"], "higher_is_better": True, "scaling": "strong",
                              "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                              "config": {"workload": "512 scenes dealt round-robin to the ranks",
                                         "parallelism": f"scenes x{world}"}}), flush=True)
        return
    sub = specs[: args.seq_scenes]
    b_sub = batched(sub, args.steps)
    seq = one_at_a_time(sub, max(3, args.steps // 3))
    line = {"metric": "body-substeps/s, 512 batched scenes", "value": full["value"], "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": full["ms_per_frame"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": (f"512 scenes, bodies log-uniform [16, 2048] ({full['bodies']} bodies incl. 4 "
                                    f"walls per scene, {full['static_rows']} static rows), OBB heaps, mu_s U[0.3,0.8], "
                                    f"substeps {{2,4,8}}, iterations {{5,10,20}}, settled {args.settle_batched} "
                                    "frames"),
                       "launch_shape": full["launch_shape"], "launches_per_frame": full["launches_per_frame"]},
            "one_at_a_time": {"scenes": len(sub), "batched": b_sub["value"], "one_at_a_time": seq["value"],
                              "speedup": b_sub["value"] / seq["value"],
                              "ms_per_frame": {"batched": b_sub["ms_per_frame"],
                                               "one_at_a_time": seq["ms_per_frame"]}}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--settle", type=int, default=240)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--small", action="store_true", help="40x40x10 pile (profiling captures)")
    ap.add_argument("--profile", action="store_true", help="cudaProfilerStart/Stop around the timed steps")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--group-size", type=int, default=0, help="lanes per body (0 = the solver default)")
    ap.add_argument("--blocks-per-sm", type=int, default=0, help="solve CTAs per SM (0 = the solver default)")
    ap.add_argument("--sweep", default="", choices=["", "barrier", "barrier-adaptive", "flags"],
                    help="color-pass ordering (empty = the solver default)")
    ap.add_argument("--tune", action="store_true",
                    help="run the launch-shape autotuner before timing and report its table (the default "
                         "times Solver6DOF's own default shape, as a drop-in user gets it)")
    ap.add_argument("--no-tune", action="store_true", help="batched bench: skip the autotuner")
    ap.add_argument("--no-warm-start", action="store_true", help="skip the learned warm-start evaluation")
    ap.add_argument("--no-batched", action="store_true", help="skip the 512-scene batched comparison key")
    ap.add_argument("--no-resting-floor", action="store_true",
                    help="read every floor corner group (Solver6DOF.resting_floor = False)")
    ap.add_argument("--row-capacity", type=int, default=0, help="initial dynamic-row pool (0 = reference size)")
    ap.add_argument("--batched", action="store_true", help="512 batched scenes vs one scene at a time")
    ap.add_argument("--seq-scenes", type=int, default=512, help="scenes in the one-at-a-time comparison")
    ap.add_argument("--settle-batched", type=int, default=60)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.batched:
        run_batched(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
