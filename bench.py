#!/usr/bin/env python
"""Throughput of the Stable Cosserat Rods substep on B200: vertex-substeps/s.

Workload (config 2): RopeBatch.from_positions with 4096 ropes x 64 vertices per GPU (seg 0.02 m,
straight down + N(0, 1e-3) m jitter, vertex 0 pinned), density 0.117 kg/m, EA 11473 N,
EI 4.48e-3 N m^2, h = 1/6000 s, 8 iterations, 100 substeps per 1/60 s control frame, plane
z = 0 (radius 6.35 mm), roots on the second-order program: p0 in a 1 m cube (z in [1.4, 2.4]),
v0 ~ N(0, 0.5) m/s, p1 = p0 + N(0, 0.05) m. Damping 0 and drag 0.2 /s set explicitly.
One step = one control frame (one persistent kernel launch). Synthetic seeded inputs.

  value   device time of the K timed frames (CUDA events on the solver stream, inputs already
          resident; L2 flushed between frames outside the events), max over ranks
  e2e     the same frames through the public API with host buffers: every step copies its
          root program from pinned host memory and reads the resulting positions back
  --impl reference: the CPU restatement of the reference's algorithm (the reference itself
          does not build here: GLM is absent) timed on all host cores, bounded sample.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "cosserat-rod-solver-cuda_b200")
for p in (PKG, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "vertex-substeps/s"
N_ROPES, V, S, ITERS, DT = 4096, 64, 100, 8, 1.0 / 60.0
H = 1.0 / 6000.0


def c2_inputs(n_ropes, frames, seed):
    import scenarios as Sc

    pos, roots = Sc.c2_positions(n_ropes, V, seed)
    rng = np.random.default_rng(seed + 1000)
    p0 = np.empty((frames, n_ropes, 3), np.float32)
    v0 = rng.normal(0, 0.5, (frames, n_ropes, 3)).astype(np.float32)
    p1 = np.empty_like(p0)
    cur = roots.copy()
    for f in range(frames):
        p0[f] = cur
        p1[f] = (cur + rng.normal(0, 0.05, (n_ropes, 3))).astype(np.float32)
        cur = p1[f]
    return pos, p0, v0, p1


def configure(b):
    b.set_gravity(np.array([0, 0, -9.81], np.float32))
    b.damping = 0.0
    b.drag = 0.2
    b.set_planes(np.array([[0, 0, 1, 0]], np.float32), radius=0.00635)


def read_flops():
    path = os.path.join(ROOT, "profiles", "flop_count_config2.txt")
    for line in open(path):
        if line.startswith("flops_per_vertex_substep:"):
            return float(line.split(":")[1])
    raise RuntimeError("flops_per_vertex_substep missing in " + path)


def read_traffic():
    path = os.path.join(ROOT, "profiles", "frame_kernel_config2.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":")[1])
    return None


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return json.load(open(path)), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.dev)], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_leg(seconds_target=15.0, threads=None):
    """The CPU restatement (FP32 instantiation of the oracle) on all host cores: bounded sample
    of the config-2 workload, ropes split over threads (ropes are independent)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ropesim_oracle

    threads = threads or os.cpu_count() or 1

    def run(n_ropes, frames):
        pos, p0, v0, p1 = c2_inputs(n_ropes, frames, 7)
        chunks = np.array_split(np.arange(n_ropes), threads)
        sims = []
        for c in chunks:
            if len(c) == 0:
                continue
            b = ropesim_oracle.RopeBatch.from_positions(pos[c], 0.117, 11473.0, 4.48e-3, H, ITERS, precision="f32")
            configure(b)
            sims.append((b, c))
        t0 = time.perf_counter()

        def work(b, c):
            for f in range(frames):
                b.step(p0[f][c], v0[f][c], DT, S, root_pos_end=p1[f][c])

        ts = [threading.Thread(target=work, args=bc) for bc in sims]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        return time.perf_counter() - t0

    probe_ropes = threads
    t = run(probe_ropes, 1)
    per = t / (probe_ropes * V * S)
    n_ropes = int(max(threads, min(N_ROPES, seconds_target / max(per, 1e-12) / (V * S) / 2)))
    frames = 2
    t = run(n_ropes, frames)
    value = n_ropes * V * S * frames / t
    return {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{n_ropes} of the {N_ROPES} config-2 ropes x {frames} frames x {S} substeps "
                      f"(FP32 CPU restatement, {threads} threads, {t:.1f} s)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ropesim_oracle

    threads = os.cpu_count() or 1
    n_ropes = max(threads, int(os.environ.get("RS_REF_ROPES", str(8 * threads))))
    pos, p0, v0, p1 = c2_inputs(n_ropes, args.warmup + args.steps, 11)
    chunks = [c for c in np.array_split(np.arange(n_ropes), threads) if len(c)]
    sims = []
    for c in chunks:
        b = ropesim_oracle.RopeBatch.from_positions(pos[c], 0.117, 11473.0, 4.48e-3, H, ITERS, precision="f32")
        configure(b)
        sims.append((b, c))

    def frame(f):
        def work(b, c):
            b.step(p0[f][c], v0[f][c], DT, S, root_pos_end=p1[f][c])

        ts = [threading.Thread(target=work, args=bc) for bc in sims]
        for t in ts:
            t.start()
        for t in ts:
            t.join()

    for f in range(args.warmup):
        frame(f)
    t0 = time.perf_counter()
    for f in range(args.warmup, args.warmup + args.steps):
        frame(f)
    el = time.perf_counter() - t0
    value = n_ropes * V * S * args.steps / el
    sample = (f"{n_ropes} of the {N_ROPES} config-2 ropes per step (64 verts, {S} substeps, {ITERS} itr), "
              f"FP32 CPU restatement of the reference's algorithm on {threads} threads")
    line = {"metric": METRIC, "value": value, "unit": METRIC, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "config2-program-4096x64 (bounded CPU sample)", "ropes_per_step": n_ropes,
                       "verts_per_rope": V, "substeps": S, "num_itr": ITERS},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference CUDA build unavailable (GLM headers absent); the reference arm is the oracle port"}
    print(json.dumps(line), flush=True)


def config3_scene(n_ropes, seed=3):
    """Config 3: n_ropes uneven ropes, V ~ U{16..256} at 2 cm, EA log-U[1e2, 1e4] and
    EI log-U[1e-5, 1e-2] per rope, per-vertex masses x U[0.8, 1.2], two planes, eight meshes
    (sphere, box, capsule closed forms baked to 64^3 float32 lattices) with per-env poses."""
    from ropesim import sdf

    rng = np.random.default_rng(seed)
    verts = rng.integers(16, 257, n_ropes)
    g = int(np.ceil(np.sqrt(n_ropes)))
    ropes = []
    for r in range(n_ropes):
        L = 0.02 * (verts[r] - 1)
        root = np.array([(r % g) * 0.7, (r // g) * 0.7, 0.06 + 0.97 * L])
        tilt = np.deg2rad(rng.uniform(5, 20))
        az = rng.uniform(0, 2 * np.pi)
        d = np.array([np.sin(tilt) * np.cos(az), np.sin(tilt) * np.sin(az), -np.cos(tilt)])
        pts = root + np.outer(np.arange(verts[r]) * 0.02, d)
        pts[1:] += rng.normal(0, 1e-3, (verts[r] - 1, 3))
        ropes.append(pts.astype(np.float32))
    ea = np.exp(rng.uniform(np.log(1e2), np.log(1e4), n_ropes))
    ei = np.exp(rng.uniform(np.log(1e-5), np.log(1e-2), n_ropes))
    ea_v = np.concatenate([np.full(v, ea[i]) for i, v in enumerate(verts)]).astype(np.float32)
    ei_v = np.concatenate([np.full(v, ei[i]) for i, v in enumerate(verts)]).astype(np.float32)
    m_v = []
    for i, rope in enumerate(ropes):
        seg = np.linalg.norm(np.diff(rope.astype(np.float64), axis=0), axis=1)
        m = np.zeros(len(rope))
        m[:-1] += 0.5 * 0.117 * seg
        m[1:] += 0.5 * 0.117 * seg
        m_v.append(m * rng.uniform(0.8, 1.2, len(rope)))
    m_v = np.concatenate(m_v).astype(np.float32)
    n64 = lambda lo, hi: (hi - lo) / 63.0
    grids = [sdf.from_function(sdf.sdf_sphere(0.12), [-0.2] * 3, [0.2] * 3, n64(-0.2, 0.2)),
             sdf.from_function(sdf.sdf_box([0.12, 0.08, 0.06], round=0.01), [-0.2] * 3, [0.2] * 3, n64(-0.2, 0.2)),
             sdf.from_function(sdf.sdf_capsule(0.06, 0.12, axis=0), [-0.2] * 3, [0.2] * 3, n64(-0.2, 0.2))]
    grids = [grids[i % 3] for i in range(8)]
    return ropes, verts, ea_v, ei_v, m_v, grids


def build_config3(ropesim, scene, engine):
    ropes, verts, ea_v, ei_v, m_v, grids = scene
    b = ropesim.RopeBatch.from_ropes(ropes, 0.117, 1000.0, 1e-3, H, ITERS)
    b.set_stretch_stiffnesses(ea_v)
    b.set_bend_stiffnesses(ei_v)
    b.set_masses(m_v)
    b.set_engine(engine)
    b.set_gravity(np.array([0, 0, -9.81], np.float32))
    b.damping = 0.0
    b.drag = 0.2
    b.set_planes(np.array([[0, 0, 1, 0], [0.05, 0.0, 1.0, -0.02]], np.float32), radius=0.005, mu_s=0.5, mu_k=0.4)
    for gd in grids:
        b.add_mesh(*gd.as_args())
    return b


def run_config3(args):
    """Config 3 forward: persistent (autotuned bins) vs the plain per-substep path, same inputs."""
    import torch

    import ropesim
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import scenarios as Sc

    torch.cuda.set_device(0)
    R = args.ropes if args.ropes != 4096 else 8192
    scene = config3_scene(R)
    ropes, verts = scene[0], scene[1]
    nv = int(np.sum(verts))
    rng = np.random.default_rng(17)
    M = 8
    frames = args.warmup + args.steps
    # per-env mesh poses: next to each rope along its length, then a random rigid walk
    pos0 = np.zeros((R, M, 3), np.float32)
    for r, rope in enumerate(ropes):
        L = 0.02 * (len(rope) - 1)
        for m in range(M):
            pos0[r, m] = rope[0] + np.array([0.25 * np.cos(0.8 * m), 0.25 * np.sin(0.8 * m), -(0.15 + 0.1 * m) * L])
    q0 = np.zeros((R, M, 4), np.float32)
    q0[..., 3] = 1.0
    poses = []
    p, q = pos0, q0
    for f in range(frames):
        poses.append((torch.as_tensor(p, device="cuda"), torch.as_tensor(q, device="cuda")))
        p, q = Sc.walk_poses(rng, p, q, step=0.003, ang=0.02)
    roots = np.stack([r[0] for r in ropes]).astype(np.float32)
    prog = []
    cur = roots.copy()
    for f in range(frames):
        v0 = rng.normal(0, 0.1, (R, 3)).astype(np.float32)
        p1 = (cur + rng.normal(0, 0.01, (R, 3))).astype(np.float32)
        prog.append(tuple(torch.as_tensor(x, device="cuda") for x in (cur, v0, p1)))
        cur = p1
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    out = {}
    for engine in ("persistent",) if args.no_plain else ("persistent", "plain"):
        b = build_config3(ropesim, scene, engine)
        st = torch.cuda.ExternalStream(b.stream_ptr())
        ms = []
        for f in range(frames):
            b.set_mesh_poses_all(poses[f][0], poses[f][1], teleport=(f == 0))
            if f >= args.warmup:
                flush.fill_(float(f))
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
            b.step(prog[f][0], prog[f][1], DT, S, root_pos_end=prog[f][2])
            if f >= args.warmup:
                e1.record(st)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
        pos = torch.as_tensor(b.positions()).cpu().numpy()
        out[engine] = {"ms_per_step": float(np.mean(ms)), "value": nv * S * len(ms) / (sum(ms) * 1e-3),
                       "finite": bool(np.isfinite(pos).all()), "layout": list(b.layout())}
        del b
    if not args.no_plain:
        out["plain_per_length"] = plain_per_length(ropesim, scene, prog, poses, args, flush)
    line = {"metric": METRIC, "value": out["persistent"]["value"], "unit": METRIC, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": out["persistent"]["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded config-3 scene)",
            "config": {"workload": f"config3-uneven-{R}", "ropes": R, "verts": nv, "verts_per_rope": "U{16..256}",
                       "substeps": S, "num_itr": ITERS, "planes": 2, "meshes": M, "lattice": "64^3",
                       "l2": "flushed between frames (256 MB write)"},
            "persistent": out["persistent"]}
    if not args.no_plain:
        line.update({"plain_path": out["plain"], "speedup_vs_plain": out["persistent"]["value"] / out["plain"]["value"],
                     "plain_per_length": out["plain_per_length"],
                     "speedup_vs_plain_per_length": out["persistent"]["value"] / out["plain_per_length"]["value"]})
    print(json.dumps(line), flush=True)


def plain_per_length(ropesim, scene, prog, poses, args, flush):
    """The plain path as the reference's API can run uneven ropes: RopeBatch holds num_envs ropes
    of one length, so the scene becomes one plain-engine batch per distinct vertex count (each
    with its own copy of the lattices), stepped in sequence on one stream every frame. Same
    ropes, stiffnesses, masses, planes, mesh poses and root programs as the single packed batch;
    a frame is timed with CUDA events on the legacy default stream, which every batch's blocking
    stream is ordered with."""
    import torch

    ropes, verts, ea_v, ei_v, m_v, grids = scene
    starts = np.concatenate([[0], np.cumsum(verts)[:-1]])
    batches = []
    for V in np.unique(verts):
        idx = np.nonzero(verts == V)[0]
        b = ropesim.RopeBatch.from_positions(np.stack([ropes[r] for r in idx]), 0.117, 1000.0, 1e-3, H, ITERS)
        sel = np.stack([starts[r] + np.arange(V) for r in idx])  # [n_V, V] flat vertex indices
        b.set_stretch_stiffnesses(ea_v[sel[:, :-1]])
        b.set_bend_stiffnesses(ei_v[sel[:, :-1]])
        b.set_masses(m_v[sel])
        b.set_engine("plain")
        b.set_gravity(np.array([0, 0, -9.81], np.float32))
        b.damping = 0.0
        b.drag = 0.2
        b.set_planes(np.array([[0, 0, 1, 0], [0.05, 0.0, 1.0, -0.02]], np.float32), radius=0.005, mu_s=0.5, mu_k=0.4)
        for gd in grids:
            b.add_mesh(*gd.as_args())
        batches.append((b, torch.as_tensor(idx, device="cuda")))
    nv = int(np.sum(verts))
    ms = []
    nwarm, nsteps = min(args.warmup, 3), min(args.steps, 3)
    for f in range(nwarm + nsteps):
        sub = [(b, poses[f][0][i].contiguous(), poses[f][1][i].contiguous(),
                [prog[f][k][i].contiguous() for k in range(3)]) for b, i in batches]
        if f >= nwarm:
            flush.fill_(float(f))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
        for b, pp, pq, pr in sub:
            b.set_mesh_poses_all(pp, pq, teleport=(f == 0))
            b.step(pr[0], pr[1], DT, S, root_pos_end=pr[2])
        if f >= nwarm:
            e1.record()
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
    finite = all(bool(torch.isfinite(torch.as_tensor(b.positions())).all()) for b, _ in batches)
    res = {"ms_per_step": float(np.mean(ms)), "value": nv * S * len(ms) / (sum(ms) * 1e-3), "batches": len(batches),
           "steps": nsteps, "finite": finite,
           "note": "one plain-engine RopeBatch per distinct vertex count (the reference's RopeBatch takes ropes of "
                   "one length), stepped in sequence"}
    del batches
    return res


def max_over_ranks(x, dist, device):
    """The maximum of a per-rank scalar over every rank: whole-job times are the slowest rank's."""
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, units_per_rank, seconds):
    """Whole-job throughput: every rank processes its own shard of ropes (weak scaling)."""
    return world * units_per_rank / seconds


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))

    import ctypes

    import ropesim

    lib = ctypes.CDLL(os.path.join(PKG, "ropesim", "libropesim_b200.so"))
    frames = args.warmup + args.steps
    # frames [0, W+K) drive the device-timed leg; the end-to-end leg continues the same root
    # programs over frames [W+K, 2(W+K)) (its own W warm-up frames, then K timed)
    pos, p0, v0, p1 = c2_inputs(N_ROPES, 2 * frames, 1234 + rank)
    b = ropesim.RopeBatch.from_positions(pos, 0.117, 11473.0, 4.48e-3, H, ITERS, deterministic=True)
    configure(b)
    if args.block:
        b.set_block(args.block)
    b.set_timing(True)
    dev = torch.device("cuda", local)
    P0 = torch.as_tensor(p0, device=dev)
    V0 = torch.as_tensor(v0, device=dev)
    P1 = torch.as_tensor(p1, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    torch.cuda.synchronize()

    # ---- device-timed leg: one persistent launch per frame
    for f in range(args.warmup):
        b.step(P0[f], V0[f], DT, S, root_pos_end=P1[f])
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    kernel_ms = []
    frame_ms = []
    stream = torch.cuda.ExternalStream(b.stream_ptr())
    sampler = ClockSampler(local)
    with sampler:
        for f in range(args.warmup, frames):
            flush.fill_(float(f))
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.step(P0[f], V0[f], DT, S, root_pos_end=P1[f])
            e1.record(stream)
            e1.synchronize()
            frame_ms.append(e0.elapsed_time(e1))
            kernel_ms.append(b.last_frame_ms())
    torch.cuda.synchronize()
    total_ms = float(sum(frame_ms))
    if world > 1:
        total_ms = max_over_ranks(total_ms, dist, dev)
        dist.barrier()
    vs_per_rank = N_ROPES * V * S * args.steps
    value = job_rate(world, vs_per_rank, total_ms * 1e-3)

    # ---- end-to-end leg: host inputs in, host positions out, through the public API
    if args.no_e2e:
        frames = args.warmup  # no timed e2e frames
    hp0 = torch.as_tensor(p0).pin_memory()
    hv0 = torch.as_tensor(v0).pin_memory()
    hp1 = torch.as_tensor(p1).pin_memory()
    out = torch.empty((N_ROPES, V, 3), dtype=torch.float32).pin_memory()
    view = torch.as_tensor(b.positions())
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    def e2e_frame(f):
        a0 = hp0[f].to(dev, non_blocking=True)
        a1 = hv0[f].to(dev, non_blocking=True)
        a2 = hp1[f].to(dev, non_blocking=True)
        b.step(a0, a1, DT, S, root_pos_end=a2)
        out.copy_(view)

    e2e_first = args.warmup + args.steps
    for f in range(e2e_first, e2e_first + args.warmup):
        e2e_frame(f)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for f in range(e2e_first + args.warmup, e2e_first + frames):
        e2e_frame(f)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    if world > 1:
        e2e_s = max_over_ranks(e2e_s, dist, dev)
    e2e_value = job_rate(world, vs_per_rank, e2e_s) if not args.no_e2e else None
    h2d = 3 * N_ROPES * 3 * 4
    d2h = N_ROPES * V * 3 * 4

    # ---- plain path: the same frames through the per-substep-launch engine (the reference's
    # launch structure, in-repo), same inputs and device timing
    plain = None
    if not args.no_plain:
        pb = ropesim.RopeBatch.from_positions(pos, 0.117, 11473.0, 4.48e-3, H, ITERS, deterministic=True)
        configure(pb)
        pb.set_engine("plain")
        pstream = torch.cuda.ExternalStream(pb.stream_ptr())
        for f in range(args.warmup):
            pb.step(P0[f], V0[f], DT, S, root_pos_end=P1[f])
        torch.cuda.synchronize()
        pms = []
        nplain = min(args.steps, 3)
        for f in range(args.warmup, args.warmup + nplain):
            flush.fill_(float(f))
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(pstream)
            pb.step(P0[f], V0[f], DT, S, root_pos_end=P1[f])
            e1.record(pstream)
            e1.synchronize()
            pms.append(e0.elapsed_time(e1))
        pvalue = N_ROPES * V * S * nplain / (sum(pms) * 1e-3)
        plain = {"value": pvalue, "unit": METRIC, "ms_per_step": sum(pms) / nplain, "steps": nplain,
                 "launches_per_step": S * (3 + 2 * ITERS) + 1, "speedup_of_persistent": value / world / pvalue,
                 "note": "per-substep-launch plain path (reference launch structure, in-repo; the reference's own "
                         "CUDA build is unavailable)"}
        del pb

    if rank == 0:
        peaks, source = measured_peaks()
        tf = ctypes.c_double(0)
        lib.rs_probe_fp32_peak(ctypes.byref(tf), None)
        fp32_peak = tf.value
        flops_vs = read_flops()
        avg_kernel_ms = float(np.mean(kernel_ms))
        flops_launch = flops_vs * N_ROPES * V * S
        achieved = flops_launch / (avg_kernel_ms * 1e-3) / 1e12
        state_bytes = N_ROPES * V * (6 * 16 + 4 * 16 + 40)  # state in (6 float4), out (4 float4), views
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded config-2 ropes and root programs)",
            "config": {"workload": "config2-program-4096x64", "ropes_per_gpu": N_ROPES, "verts_per_rope": V,
                       "substeps": S, "num_itr": ITERS, "h": H, "planes": 1, "l2": "flushed between frames (256 MB write)",
                       "bins": list(b.layout()), "parallelism": f"replicas x{world} (ropes independent)"},
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": args.steps,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved / fp32_peak, "traffic": read_traffic(),
                         "peak_source": "measured FP32 FMA probe (rs_probe_fp32_peak) on this GPU",
                         "flops_per_vertex_substep": flops_vs,
                         "hbm_view": {"algorithmic_bytes_per_launch": state_bytes,
                                      "achieved_gbs": state_bytes / (avg_kernel_ms * 1e-3) / 1e9,
                                      "peak_gbs": peaks.get("hbm_gbs"), "peak_source": source}},
            "kernel_ms_per_frame": avg_kernel_ms,
            "plain_path": plain,
            "clocks": sampler.summary(),
        }
        if world == 1 and not args.no_cpu:
            line["cpu_baseline"] = cpu_leg()
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_config4(args):
    """Config 4: differentiable rollouts of 1024 ropes x 64 vertices (config-1 rope: 3 cm segments,
    0.1 kg/m, EA 500 N, EI 1e-4 N m^2), 30 control frames x 100 substeps, program roots, loss = mean
    squared tip distance to a seeded target curve. One step = one 30-frame rollout: forward only
    (RopeBatch.step), forward + backward (ropesim.grad.frame + loss.backward(), gradients of the
    programs, EA, EI, mass and the initial state), and the plain per-substep path's forward."""
    import torch

    import ropesim
    import ropesim.grad as rg

    torch.cuda.set_device(0)
    R = args.ropes if args.ropes != 4096 else 1024
    V, F, S4 = 64, args.frames or 30, 100
    seg, density, ea, ei = 0.03, 0.1, 500.0, 1e-4
    rng = np.random.default_rng(4)
    roots = np.stack([rng.uniform(-0.5, 0.5, R), rng.uniform(-0.5, 0.5, R), rng.uniform(2.5, 3.5, R)], 1).astype(np.float32)
    pos = np.repeat(roots[:, None], V, 1) - np.array([0, 0, seg], np.float32) * np.arange(V, dtype=np.float32)[None, :, None]
    pos[:, 1:] += rng.normal(0, 1e-3, (R, V - 1, 3)).astype(np.float32)
    prog = []
    cur = roots.copy()
    for f in range(F):
        v0 = rng.normal(0, 0.3, (R, 3)).astype(np.float32)
        p1 = (cur + rng.normal(0, 0.02, (R, 3))).astype(np.float32)
        prog.append((cur.copy(), v0, p1))
        cur = p1
    P = [torch.tensor(np.stack([p[k] for p in prog]), device="cuda") for k in range(3)]
    t_amp = rng.normal(0, 0.05, (1, R, 3))
    tgt = pos[:, -1][None] + t_amp * np.sin(2 * np.pi * np.arange(1, F + 1)[:, None, None] / F)
    tgt = torch.tensor(tgt, device="cuda", dtype=torch.float32)

    def make(engine):
        b = ropesim.RopeBatch.from_positions(pos, density, ea, ei, 1 / 6000, ITERS)
        b.set_gravity(np.array([0, 0, -9.81], np.float32))
        b.damping = 0.0
        b.drag = 0.2
        if engine == "plain":
            b.set_engine("plain")
        return b

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    nv = R * V

    def timed(fn, rollouts):
        ms = []
        for k in range(rollouts):
            flush.fill_(float(k))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return ms

    out = {}
    for engine in ("persistent", "plain"):
        b = make(engine)
        st0 = rg.state(b)

        def fwd(b=b, st0=st0):
            b.set_state(*st0)
            for f in range(F):
                b.step(P[0][f], P[1][f], DT, S4, root_pos_end=P[2][f])

        timed(fwd, args.warmup)
        ms = timed(fwd, args.steps)
        out[engine] = {"ms_per_rollout": float(np.mean(ms)), "value": nv * S4 * F * len(ms) / (sum(ms) * 1e-3)}
        if engine == "persistent":
            par0 = rg.parameters(b)
            grads = {}

            def fwd_bwd(b=b, st0=st0, par0=par0):
                st = [t.clone().requires_grad_() for t in st0]
                par = [t.clone().requires_grad_() for t in par0]
                pr = [t.clone().requires_grad_() for t in P]
                cur = st
                loss = 0.0
                for f in range(F):
                    cur = rg.frame(b, cur, par, pr[0][f], pr[1][f], pr[2][f], DT, S4,
                                   tape=False if args.no_tape else ("iterates" if args.iterate_tape else True))
                    loss = loss + ((cur[0].view(R, V, 3)[:, -1] - tgt[f]) ** 2).sum(-1).mean()
                loss.backward()
                grads["tensors"] = [t.grad for t in st + par + pr]  # checked after the timed rollouts
                grads["loss_t"] = loss.detach()

            timed(fwd_bwd, args.warmup)
            msb = timed(fwd_bwd, args.steps)
            grads["finite"] = bool(all(torch.isfinite(t).all() for t in grads["tensors"]))
            grads["loss"] = float(grads["loss_t"])
            out["fwd_bwd"] = {"ms_per_rollout": float(np.mean(msb)), "value": nv * S4 * F * len(msb) / (sum(msb) * 1e-3),
                              "grads_finite": grads["finite"], "loss": grads["loss"]}
        del b
    line = {"metric": "vertex-substeps/s (fwd+bwd)", "value": out["fwd_bwd"]["value"], "unit": "vertex-substeps/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": out["fwd_bwd"]["ms_per_rollout"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded config-4 rollouts)",
            "config": {"workload": f"config4-diff-{R}x{V}", "ropes": R, "verts_per_rope": V, "frames": F,
                       "substeps": S4, "num_itr": ITERS, "step": f"one {F}-frame rollout",
                       "backward": "replays each frame" if args.no_tape else (
                           "from the forward's substep and iterate tapes" if args.iterate_tape
                           else "from the forward's substep tapes"),
                       "counted": "forward vertex-substeps of the rollout", "l2": "flushed between rollouts (256 MB write)"},
            "forward": out["persistent"], "fwd_bwd": out["fwd_bwd"], "plain_path_forward": out["plain"],
            "fwd_bwd_over_fwd": out["fwd_bwd"]["ms_per_rollout"] / out["persistent"]["ms_per_rollout"],
            "fwd_bwd_speedup_vs_plain_fwd": out["fwd_bwd"]["value"] / out["plain"]["value"],
            "fwd_speedup_vs_plain": out["persistent"]["value"] / out["plain"]["value"]}
    print(json.dumps(line), flush=True)


def config5_scene(R=256, V=128, seed=5):
    """Config 5 stand-in (seeded): R free ropes of V vertices, 1 cm segments (density 0.117 kg/m),
    per-rope EA log-uniform [1e2, 1e3] N and EI log-uniform [1e-5, 1e-3] N m^2 (at 8 sweeps the
    adjoint of stiffer stretch, k / (m / h^2) above ~7 or EA above ~3e3 N here, grows without bound:
    the Jacobi map's linearisation is unstable there, in FP64 as well), dropped in layers of
    8 parallel straight ropes 15 mm apart in z (each layer a random rotation about z and a random
    offset within a 0.3 m footprint; ropes 4 cm apart within a layer, so no pair starts closer than
    the 10 mm contact distance; the lowest layer 5 cm up), onto the plane z = 0 inside a shallow
    spherical bowl (radius 6 m, its lowest point 5 cm below the plane, rising to 8 cm above it at
    the lattice edge) baked to a 128^3 lattice. Returns (positions [R, V, 3],
    EA [R], EI [R], lattice args)."""
    sys.path.insert(0, PKG)
    from ropesim import sdf

    rng = np.random.default_rng(seed)
    seg, per_layer = 0.01, 8
    layers = (R + per_layer - 1) // per_layer
    pos = np.zeros((R, V, 3), np.float32)
    t = (np.arange(V) - (V - 1) / 2) * seg
    for r in range(R):
        L, k = r // per_layer, r % per_layer
        if k == 0:
            th = rng.uniform(0, np.pi)
            off = rng.uniform(-0.05, 0.05, 2)
            d, nrm = np.array([np.cos(th), np.sin(th)]), np.array([-np.sin(th), np.cos(th)])
        c = off + nrm * (k - (per_layer - 1) / 2) * 0.04
        pos[r, :, 0] = c[0] + d[0] * t
        pos[r, :, 1] = c[1] + d[1] * t
        pos[r, :, 2] = 0.05 + 0.015 * L
    ea = np.exp(rng.uniform(np.log(1e2), np.log(1e3), R)).astype(np.float32)
    ei = np.exp(rng.uniform(np.log(1e-5), np.log(1e-3), R)).astype(np.float32)
    sp = 0.0165  # 128 nodes per axis: 2.0955 m
    lo = np.array([-1.05, -1.05, -0.25])
    g = sdf.from_function(sdf.sdf_bowl(6.0, centre=(0.0, 0.0, 5.95)), lo, lo + 126.5 * sp, sp)
    assert g.values.shape == (128, 128, 128)
    phi = sdf.sdf_bowl(6.0, centre=(0.0, 0.0, 5.95))(pos.reshape(-1, 3))
    assert phi.min() > 0.02, "a rope starts outside the bowl"
    return pos, ea, ei, g.as_args()


def run_config5(args):
    """Config 5: contact-heavy forward + backward. 256 x 128 free ropes (config5_scene) with one
    rope-rope contact group of all ropes (radius 0.9 R, barrier 0.2 R for R = 5 mm, k_collision
    0.025, mu 0.4, k_friction 1e7), the plane z = 0 and the bowl (R = 5 mm, mu_s 0.5, mu_k 0.4);
    dt 1/60, 100 substeps, 8 iterations. The group (32,768 vertices) is larger than a CTA, so frames
    run the per-substep-launch path (grid broad phase) and the backward the per-launch adjoint.

    Stiffness fitting: targets are the rollout with the seeded per-rope EA / EI (its full state at
    every frame). Through the pile the exact gradient of the 8-sweep map grows by ~1e4 per frame
    (the compressed barrier is far stiffer than m / h^2), so the fit is one-step-ahead (teacher
    forced): every frame starts from the target state, the loss is the predicted frame-end
    positions' mean squared distance to the target (mm^2) summed over the frames, and each frame
    is differentiated on its own (a frame whose gradient overflows FP32 is left out and counted).
    One step = --frames such frames forward (with tapes) and backward, then one Adam step on
    per-rope log EA / log EI. Reported: fitting steps/s, forward + backward vertex-substeps/s, the
    forward-only rollout, and with --fit-steps N the parameter errors after N steps."""
    import torch

    import ropesim
    import ropesim.grad as rg

    torch.cuda.set_device(0)
    R = args.ropes if args.ropes != 4096 else 256
    V, F, S5 = 128, args.frames or 60, 100
    iters = args.iters or ITERS
    pos, ea_true, ei_true, lattice = config5_scene(R, V)
    Rc = 0.005
    b = ropesim.RopeBatch.from_positions(pos, 0.117, 1000.0, 1e-3, 1 / 6000, iters, pinned=np.zeros(V, bool))
    b.set_gravity(np.array([0, 0, -9.81], np.float32))
    b.damping = 0.0
    b.drag = 0.2
    b.set_planes(np.array([[0.0, 0.0, 1.0, 0.0]], np.float32), radius=Rc, mu_s=0.5, mu_k=0.4)
    b.set_contact(Rc, mu_s=0.5, mu_k=0.4)
    b.add_mesh(*lattice, pos=np.zeros((R, 3), np.float32), quat=np.tile(np.float32([0, 0, 0, 1]), (R, 1)), mu_s=0.5, mu_k=0.4)
    b.set_rope_contact(True, radius=0.9 * Rc, barrier=0.2 * Rc, k_collision=0.025, mu=0.4, k_friction=1e7, group_ropes=R)
    st0 = rg.state(b)
    _, _, mass = rg.parameters(b)
    n = R * V
    seg_mask = torch.ones(R, V, device="cuda")
    seg_mask[:, -1] = 0.0

    def per_vertex(x):  # per-rope values onto the vertices that own a segment
        return (x[:, None] * seg_mask).reshape(n)

    true_ea = torch.tensor(ea_true, device="cuda")
    true_ei = torch.tensor(ei_true, device="cuda")
    with torch.no_grad():  # the trajectories the method itself generates, with the seeded parameters
        cur, traj = st0, [st0]
        for f in range(F):
            cur = rg.frame(b, cur, (per_vertex(true_ea), per_vertex(true_ei), mass), None, None, None, DT, S5)
            traj.append(tuple(t.clone() for t in cur))
    drop = float((st0[0][:, 2] - traj[-1][0][:, 2]).mean())
    rng = np.random.default_rng(6)
    log_ea = torch.tensor(np.log(ea_true) + rng.normal(0, 0.3, R), device="cuda", dtype=torch.float32, requires_grad=True)
    log_ei = torch.tensor(np.log(ei_true) + rng.normal(0, 0.3, R), device="cuda", dtype=torch.float32, requires_grad=True)
    opt = torch.optim.Adam([log_ea, log_ei], lr=0.05, eps=1e-12)

    def errors():
        with torch.no_grad():
            e_ea = (log_ea.exp() / true_ea).log().abs().median()
            e_ei = (log_ei.exp() / true_ei).log().abs().median()
        return float(e_ea), float(e_ei)

    info = {"dropped_frames": 0}

    def fit_step():
        g_ea, g_ei = torch.zeros_like(log_ea), torch.zeros_like(log_ei)
        total = 0.0
        for f in range(F):
            par = (per_vertex(log_ea.exp()), per_vertex(log_ei.exp()), mass)
            out = rg.frame(b, traj[f], par, None, None, None, DT, S5)
            loss = ((out[0] - traj[f + 1][0]) ** 2).sum(-1).mean() * 1e6  # mm^2
            ga, gi = torch.autograd.grad(loss, (log_ea, log_ei))
            if bool(torch.isfinite(ga).all() and torch.isfinite(gi).all()):
                g_ea += ga
                g_ei += gi
            else:
                info["dropped_frames"] += 1
            total += float(loss.detach())
        log_ea.grad, log_ei.grad = g_ea, g_ei
        info["loss"] = total
        opt.step()

    def fwd_only():
        b.set_state(*st0)
        for f in range(F):
            b.step_free(DT, S5)

    def timed(fn, k):
        ms = []
        for _ in range(k):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return ms

    err0 = errors()
    timed(fit_step, 1)
    loss_first = info["loss"]
    timed(fit_step, args.warmup - 1)
    msb = timed(fit_step, args.steps)
    fit = {"steps_done": args.warmup + args.steps}
    if args.fit_steps > fit["steps_done"]:
        timed(fit_step, args.fit_steps - fit["steps_done"])
        fit["steps_done"] = args.fit_steps
    err1 = errors()
    fit.update({"objective": "one-step-ahead (teacher forced) frame-end positions, mm^2 summed over frames",
                "loss_first_step": loss_first, "loss_last_step": info["loss"],
                "frames_dropped_for_overflow": info["dropped_frames"],
                "median_abs_log_error_ea": [err0[0], err1[0]], "median_abs_log_error_ei": [err0[1], err1[1]]})
    timed(fwd_only, 1)
    msf = timed(fwd_only, max(1, min(args.steps, 3)))
    ms_step = float(np.mean(msb))
    line = {"metric": "stiffness-fitting steps/s (forward + backward)", "value": 1e3 / ms_step, "unit": "steps/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded config-5 pile: layered drop into a baked bowl)",
            "config": {"workload": f"config5-contact-{R}x{V}", "ropes": R, "verts_per_rope": V, "frames": F,
                       "substeps": S5, "num_itr": iters, "contact_group_vertices": n,
                       "step": f"one fitting step: {F} teacher-forced frames forward (taped) + backward, Adam on "
                               "per-rope log EA / log EI", "engine": "per-substep launches, grid broad phase "
                               "(group larger than a CTA)", "mean_drop_m": drop},
            "fwd_bwd_vertex_substeps_per_s": n * S5 * F / (ms_step * 1e-3),
            "forward_only": {"ms_per_rollout": float(np.mean(msf)), "value": n * S5 * F / (float(np.mean(msf)) * 1e-3)},
            "fwd_bwd_over_fwd": ms_step / float(np.mean(msf)), "fit": fit}
    print(json.dumps(line), flush=True)


def run_exchange(args):
    """The rigid-body exchange loop at scale (the reference's Isaac bridge, ropesim/isaac_bridge.py:236-271):
    per exchange, mesh poses from CUDA tensors (set_mesh_poses_all), one rope step, and the
    frame-averaged wrenches read back through mesh_wrenches_view (a device copy, as the bridge's
    wrenches()). Config-3 scene (uneven ropes, 2 planes, 8 meshes per env) with the contact-force
    readout on, exchanged once per control frame (K = 1, 100 substeps) and sub-cycled (K = 10
    steps of 10 substeps, the bridge's --exchange 10), next to the same frames with the readout
    off. One step = one control frame; CUDA events on the solver stream around the whole loop."""
    import torch

    import ropesim
    import scenarios as Sc

    torch.cuda.set_device(0)
    R = args.ropes if args.ropes != 4096 else 8192
    scene = config3_scene(R)
    ropes, verts = scene[0], scene[1]
    nv = int(np.sum(verts))
    M = 8
    rng = np.random.default_rng(23)
    frames = args.warmup + args.steps
    pos0 = np.zeros((R, M, 3), np.float32)
    for r, rope in enumerate(ropes):
        L = 0.02 * (len(rope) - 1)
        for m in range(M):
            pos0[r, m] = rope[0] + np.array([0.25 * np.cos(0.8 * m), 0.25 * np.sin(0.8 * m), -(0.15 + 0.1 * m) * L])
    q0 = np.zeros((R, M, 4), np.float32)
    q0[..., 3] = 1.0
    roots = np.stack([r[0] for r in ropes]).astype(np.float32)

    def leg(K, forces):
        b = build_config3(ropesim, scene, "persistent")
        b.enable_contact_forces(forces)
        st = torch.cuda.ExternalStream(b.stream_ptr())
        wview = torch.as_tensor(b.mesh_wrenches_view()) if forces else None
        prng = np.random.default_rng(29)
        p, q, cur = pos0, q0, roots.copy()
        poses, progs = [], []
        for f in range(frames * K):  # per exchange: poses and a root program over dt / K
            poses.append((torch.as_tensor(p, device="cuda"), torch.as_tensor(q, device="cuda")))
            p, q = Sc.walk_poses(prng, p, q, step=0.003 / K, ang=0.02 / K)
            v0 = prng.normal(0, 0.1, (R, 3)).astype(np.float32)
            p1 = (cur + prng.normal(0, 0.01 / K, (R, 3))).astype(np.float32)
            progs.append(tuple(torch.as_tensor(x, device="cuda") for x in (cur, v0, p1)))
            cur = p1
        out = []
        ms, wall = [], []
        for f in range(frames):
            if f >= args.warmup:
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                t0 = time.perf_counter()
            for k in range(K):
                x = f * K + k
                b.set_mesh_poses_all(poses[x][0], poses[x][1], teleport=(x == 0))
                b.step(progs[x][0], progs[x][1], DT / K, S // K, root_pos_end=progs[x][2])
                if forces:
                    out.append(wview[:, :M].clone())
            if f >= args.warmup:
                e1.record(st)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
                wall.append(time.perf_counter() - t0)
        torch.cuda.synchronize()
        res = {"K": K, "readout": forces, "ms_per_frame": float(np.mean(ms)), "wall_ms_per_frame": 1e3 * float(np.mean(wall)),
               "value": nv * S * len(ms) / (sum(ms) * 1e-3)}
        if forces:
            w = torch.stack(out[-K:]).float()
            res["wrench_max_abs"] = float(w.abs().max())
            res["finite"] = bool(torch.isfinite(w).all())
        del b
        return res

    legs = [leg(1, False), leg(1, True), leg(10, True)]
    line = {"metric": "vertex-substeps/s (exchange loop)", "value": legs[2]["value"], "unit": METRIC, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": legs[2]["ms_per_frame"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded config-3 scene)",
            "config": {"workload": f"exchange-config3-{R}", "ropes": R, "verts": nv, "meshes": M, "substeps": S,
                       "step": "one control frame of K exchanges: poses in (CUDA), rope step, wrenches out (device copy)"},
            "legs": legs,
            "readout_cost": legs[1]["ms_per_frame"] / legs[0]["ms_per_frame"],
            "subcycle_cost_k10": legs[2]["ms_per_frame"] / legs[1]["ms_per_frame"]}
    print(json.dumps(line), flush=True)


# Operations of one evaluation, counted from the kernel source (add/sub/mul/div/sqrt = 1): a
# point-triangle distance on its longest path (the face interior, FP32), a line-triangle crossing
# test (three edge predicates, FP64) and one solid angle (FP32, atan2 counted as 1).
BAKE_FLOP_DIST, BAKE_FLOP_CROSS, BAKE_FLOP_SOLID = 80, 15, 66


def run_bake(args):
    """Mesh baking (the reference's sdf.bake_mesh, on Warp there): an icosphere of `--bake-subdiv`
    subdivisions (default 5: 20,480 triangles, r 0.15 m) baked with 2.5 mm cells and a 5 cm margin
    (162^3 = 4.25 M nodes). value: lattice nodes per second of the whole call (CUDA events on the
    bake's stream around it; the host's triangle sort and upload are inside); kernel_ms_per_bake:
    the kernels alone; e2e: sdf.bake_mesh from host arrays to a host lattice (wall clock);
    cpu_baseline: the FP64 brute-force oracle on all host cores over one slab of the lattice."""
    import ctypes

    import torch

    import meshes
    from ropesim import sdf

    torch.cuda.set_device(0)
    lib = ctypes.CDLL(os.path.join(PKG, "ropesim", "libropesim_b200.so"))
    v, f = meshes.icosphere(args.bake_subdiv, 0.15)
    spacing, margin = 0.0025, 0.05
    origin, dims = sdf._lattice(v.min(0) - margin, v.max(0) + margin, spacing)
    nodes = int(np.prod(dims))
    out = torch.empty(dims, dtype=torch.float32, device="cuda")
    st = torch.cuda.Stream()
    cnt = (ctypes.c_ulonglong * 4)()
    vp, fp = np.ascontiguousarray(v, np.float32), np.ascontiguousarray(f, np.int32)
    org = np.ascontiguousarray(origin, np.float32)

    def bake(counters=None):
        rc = lib.rs_sdf_bake(vp.ctypes.data_as(ctypes.c_void_p), len(v), fp.ctypes.data_as(ctypes.c_void_p), len(f),
                             org.ctypes.data_as(ctypes.c_void_p), ctypes.c_double(spacing), dims[0], dims[1], dims[2],
                             ctypes.c_float(0.0), ctypes.c_float(0.0), ctypes.c_void_p(out.data_ptr()), 1,
                             ctypes.c_void_p(st.cuda_stream), counters)
        if rc != 0:
            raise RuntimeError("rs_sdf_bake failed")

    bake(cnt)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        bake()
    torch.cuda.synchronize()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    ms, kms = [], []
    sampler = ClockSampler(0)
    with sampler:
        for k in range(args.steps):
            flush.fill_(float(k))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            bake(cnt)
            e1.record(st)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            kms.append(cnt[3] * 1e-6)
    dev_ms = float(np.mean(ms))
    kernel_ms = float(np.mean(kms))
    # end to end: host mesh in, host lattice out, through the public Python API
    sdf.bake_mesh(v, f, spacing, margin)
    t0 = time.perf_counter()
    ke = max(1, min(args.steps, 5))
    for _ in range(ke):
        g = sdf.bake_mesh(v, f, spacing, margin)
    e2e_s = (time.perf_counter() - t0) / ke
    assert g.values.shape == tuple(dims) and np.isfinite(g.values).all()
    assert np.array_equal(out.cpu().numpy(), g.values)
    ev_d, ev_x, ev_w = int(cnt[0]), int(cnt[1]), int(cnt[2])
    flops = ev_d * BAKE_FLOP_DIST + ev_w * BAKE_FLOP_SOLID  # FP32 work (the FP64 crossing tests are few)
    tf = ctypes.c_double(0)
    lib.rs_probe_fp32_peak(ctypes.byref(tf), None)
    achieved = flops / (kernel_ms * 1e-3) / 1e12
    line = {"metric": "lattice nodes/s (mesh bake)", "value": nodes / (dev_ms * 1e-3), "unit": "nodes/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (icosphere mesh)",
            "config": {"workload": f"bake-icosphere{args.bake_subdiv}", "triangles": len(f), "lattice": list(dims),
                       "nodes": nodes, "spacing_m": spacing, "margin_m": margin, "signed": True,
                       "l2": "flushed between bakes (256 MB write)"},
            "e2e": {"value": nodes / e2e_s, "unit": "nodes/s", "h2d_bytes_per_step": int(vp.nbytes + fp.nbytes),
                    "d2h_bytes_per_step": nodes * 4},
            "kernel_ms_per_bake": kernel_ms,
            "timing": "value: CUDA events around the whole rs_sdf_bake call on its stream (host triangle sort and "
                      "upload included); kernel_ms_per_bake and roofline: the two kernels alone",
            "gpu_launches": 2 * args.steps,
            "evaluations": {"point_triangle_distances": ev_d, "crossing_tests": ev_x, "solid_angles": ev_w,
                            "brute_force_pairs": nodes * len(f), "distance_fraction_of_brute_force": ev_d / (nodes * len(f))},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": tf.value, "unit": "TFLOP/s",
                         "frac": achieved / tf.value, "traffic": None,
                         "flops_per_eval": {"distance": BAKE_FLOP_DIST, "crossing_fp64": BAKE_FLOP_CROSS,
                                            "solid_angle": BAKE_FLOP_SOLID},
                         "peak_source": "measured FP32 FMA probe (rs_probe_fp32_peak) on this GPU"},
            "clocks": sampler.summary()}
    if not args.no_cpu:
        import _oracle

        i1 = 1
        t0 = time.perf_counter()
        _oracle.bake_sdf(vp, fp, org, spacing, [i1, dims[1], dims[2]], 0.0, 0.0, 0)
        t = time.perf_counter() - t0
        thr = _oracle.hardware_threads()
        line["cpu_baseline"] = {"value": i1 * dims[1] * dims[2] / t, "unit": "nodes/s", "cores": thr, "kind": "port",
                                "sample": f"{i1} of {dims[0]} x-slabs of the lattice (FP64 brute-force oracle, "
                                          f"{thr} threads, {t:.1f} s)"}
    print(json.dumps(line), flush=True)


def main():
    global N_ROPES
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--ropes", type=int, default=N_ROPES, help="ropes per GPU (profiling of smaller cases)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling)")
    ap.add_argument("--block", type=int, default=0, help="bin size (CTA threads); 0 = the library's choice")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-path leg")
    ap.add_argument("--frames", type=int, default=0,
                    help="control frames per rollout (0 = the workload's own: 30 for config4, 60 for config5)")
    ap.add_argument("--no-tape", action="store_true", help="config4: backward replays frames instead of keeping tapes")
    ap.add_argument("--no-iterate-tape", dest="iterate_tape", action="store_false",
                    help="config4: keep only the substep tapes (the backward recomputes the iterates)")
    ap.add_argument("--fit-steps", type=int, default=0, help="config5: total fitting steps to run (e.g. 50)")
    ap.add_argument("--iters", type=int, default=0, help="config5: Jacobi sweeps per substep (0 = the default 8)")
    ap.add_argument("--bake-subdiv", type=int, default=5, help="bake: icosphere subdivisions of the baked mesh")
    ap.add_argument("--workload", default="config2",
                    choices=["config2", "config3", "config4", "config5", "bake", "exchange"],
                    help="config2 (the headline line), config3 (uneven ropes, planes and meshes vs the plain path) "
                         "or config4 (differentiable rollouts: forward and forward + backward)")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    N_ROPES = args.ropes
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "config3":
        run_config3(args)
    elif args.workload == "config4":
        run_config4(args)
    elif args.workload == "config5":
        run_config5(args)
    elif args.workload == "exchange":
        run_exchange(args)
    elif args.workload == "bake":
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        run_bake(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
