#!/usr/bin/env python
"""Throughput of the Stable Cosserat Rods substep on B200: vertex-substeps/s, forward and
forward + backward, against the plain per-substep-launch path on the same GPU.

Default workload (the target configuration): 8192 uneven ropes, V ~ U{16..256} at 2 cm
(1,107,975 vertices), EA log-U[1e2, 1e4] N and EI log-U[1e-5, 1e-2] N m^2 per rope, per-vertex
masses x U[0.8, 1.2], two planes, eight kinematic meshes (sphere / box / capsule closed forms on
64^3 float32 lattices) with per-env random-walk poses every frame, root programs (v0 ~ N(0, 0.1),
p1 = p0 + N(0, 0.01)), h = 1/6000 s, 8 iterations, 100 substeps per 1/60 s control frame.
Seeded synthetic inputs (tests/scenarios.py: bench_c3_scene / bench_c3_inputs). One step = one
control frame: mesh poses in, one persistent kernel launch, status read.

  value     device time of the K timed frames (CUDA events on the solver stream; inputs resident
            in HBM; L2 flushed between frames outside the events), max over ranks
  e2e       the same frames through the public API from pinned host buffers: every step copies
            its mesh poses and root program in and reads the positions view back
  speedup_vs_plain  the same frames through the plain per-substep-launch engine (the
            reference's launch structure), and the plain engine as the reference's API must run
            uneven ropes (one RopeBatch per rope length)
  config2 / config4 / fwd_bwd_over_fwd  the 4096 x 64 config-2 workload and the 1024 x 64
            differentiable rollouts (forward vs forward + backward), measured in the same run
  --impl reference: the CPU restatement of the reference's algorithm (the reference's CUDA
            build needs GLM, absent here) on all host cores, bounded samples of the same scene

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload ...]
With --gpus N > 1 and no torchrun environment the script re-launches itself under
torch.distributed.run with N ranks (one per GPU; ropes sharded by rank, no collective on the
data path).
"""
from __future__ import annotations

import argparse
import json
import os
import socket
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

import scenarios as Sc  # noqa: E402  (the seeded bench scenes, shared with the parity tests)

METRIC = "vertex-substeps/s fwd and fwd+bwd vs plain path, same B200, ≤1e-5 m deviation"
UNIT = "vertex-substeps/s"
V, S, ITERS, DT, H = 64, Sc.BENCH_S, Sc.BENCH_ITERS, Sc.BENCH_DT, Sc.BENCH_H
C2_ROPES, C3_ROPES, M3 = 4096, 8192, 8


def read_profile_value(name, key):
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith(key + ":"):
            return float(line.split(":")[1])
    return None


def read_parity():
    """Summary of tests/test_bench_parity.py's last run on a B200 (profiles/parity_bench_scenes.txt)."""
    path = os.path.join(ROOT, "profiles", "parity_bench_scenes.txt")
    if not os.path.exists(path):
        return None
    body = "".join(l for l in open(path) if not l.startswith("#"))
    try:
        d = json.loads(body)
    except ValueError:
        return None
    d["source"] = "profiles/parity_bench_scenes.txt (tests/test_bench_parity.py on a B200)"
    return d


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


# ------------------------------------------------------------------ process plumbing
def maybe_relaunch(args):
    """`--gpus N` (N > 1) outside torchrun: re-run this command under torch.distributed.run with
    N ranks on this node. Inside torchrun, --gpus must equal the world size."""
    world = os.environ.get("WORLD_SIZE")
    if world is not None:
        if int(world) != args.gpus:
            raise SystemExit(f"--gpus {args.gpus} does not match the launcher's WORLD_SIZE {world}")
        return
    if args.gpus <= 1:
        return
    import torch

    if torch.cuda.device_count() < args.gpus:
        raise SystemExit(f"--gpus {args.gpus} needs {args.gpus} visible GPUs; {torch.cuda.device_count()} found")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    raise SystemExit(subprocess.call(cmd))


def dist_setup():
    """(world, rank, local rank, device, dist module or None): one process per GPU over NCCL."""
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
        return world, rank, local, dev, dist
    return world, rank, local, dev, None


def max_over_ranks(x, dist, device):
    """The maximum of a per-rank scalar over every rank: whole-job times are the slowest rank's."""
    import torch

    if dist is None:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, units_per_rank, seconds):
    """Whole-job throughput: every rank processes its own shard of ropes (weak scaling)."""
    return world * units_per_rank / seconds


def barrier(dist):
    if dist is not None:
        dist.barrier()


def fp32_peak_tflops():
    import ctypes

    lib = ctypes.CDLL(os.path.join(PKG, "ropesim", "libropesim_b200.so"))
    tf = ctypes.c_double(0)
    lib.rs_probe_fp32_peak(ctypes.byref(tf), None)
    return tf.value


def timed_frames(fn, frames, stream, flush, kernel_ms=None, b=None):
    """CUDA-event time of each call of fn(f) on `stream`, L2 flushed before each (outside the events)."""
    import torch

    ms = []
    for f in frames:
        flush.fill_(float(f))
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn(f)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        if kernel_ms is not None:
            kernel_ms.append(b.last_frame_ms())
    return ms


# ------------------------------------------------------------------ CPU legs (the oracle port)
def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ropesim_oracle

    return ropesim_oracle


def _threads_run(sims, work):
    ts = [threading.Thread(target=work, args=s) for s in sims]
    for t in ts:
        t.start()
    for t in ts:
        t.join()


def c3_cpu_sims(scene, ropes, threads, precision="f32"):
    ro = _oracle()
    chunks = [c for c in np.array_split(np.asarray(ropes), threads) if len(c)]
    return [(Sc.bench_c3_build(ro, scene, sel=c, precision=precision), c) for c in chunks]


def c3_cpu_frame(sims, inputs, f):
    PP, QQ, p0, v0, p1 = inputs

    def work(o, c):
        o.set_mesh_poses_all(PP[f][c], QQ[f][c], teleport=(f == 0))
        o.step(p0[f][c], v0[f][c], DT, S, root_pos_end=p1[f][c])

    _threads_run(sims, work)


def cpu_leg_c3(scene, inputs, seconds_target=15.0, threads=None):
    """The FP32 CPU restatement on all host cores: a bounded sample of the config-3 ropes
    (ropes split over threads), frames 0..2 of the same inputs."""
    threads = threads or os.cpu_count() or 1
    verts = scene[1]
    probe = np.arange(threads)
    sims = c3_cpu_sims(scene, probe, threads)
    t0 = time.perf_counter()
    c3_cpu_frame(sims, inputs, 0)
    per = (time.perf_counter() - t0) / max(1, int(verts[probe].sum()))  # s per vertex-frame (all threads)
    n = int(np.clip(seconds_target / 2 / max(per, 1e-12) / np.mean(verts), threads, len(verts)))
    sel = np.arange(n)
    sims = c3_cpu_sims(scene, sel, threads)
    frames = 2
    t0 = time.perf_counter()
    for f in range(frames):
        c3_cpu_frame(sims, inputs, f)
    t = time.perf_counter() - t0
    nv = int(verts[sel].sum())
    return {"value": nv * S * frames / t, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"the first {n} of the {len(verts)} config-3 ropes ({nv} vertices) x {frames} frames x {S} substeps "
                      f"(FP32 CPU restatement, {threads} threads, {t:.1f} s)"}


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's algorithm (its CUDA build needs
    GLM, absent on this image) on all host cores, each step one frame of a bounded sample of the
    same scene. Rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from ropesim import sdf

    threads = os.cpu_count() or 1
    frames = args.warmup + args.steps
    if args.workload == "config2":
        n_ropes = max(threads, int(os.environ.get("RS_REF_ROPES", str(8 * threads))))
        pos, p0, v0, p1 = Sc.bench_c2_inputs(n_ropes, frames, 11)
        ro = _oracle()
        sims = []
        for c in [c for c in np.array_split(np.arange(n_ropes), threads) if len(c)]:
            b = ro.RopeBatch.from_positions(pos[c], 0.117, 11473.0, 4.48e-3, H, ITERS, precision="f32")
            Sc.bench_c2_configure(b)
            sims.append((b, c))

        def frame(f):
            _threads_run(sims, lambda b, c: b.step(p0[f][c], v0[f][c], DT, S, root_pos_end=p1[f][c]))

        nv, workload = n_ropes * V, "config2-program-4096x64"
        sample = f"{n_ropes} of the 4096 config-2 ropes per step (64 verts)"
    else:
        scene = Sc.bench_c3_scene(sdf, C3_ROPES)
        inputs = Sc.bench_c3_inputs(scene, frames)
        n_ropes = max(threads, int(os.environ.get("RS_REF_ROPES", str(32 * threads))))
        sims = c3_cpu_sims(scene, np.arange(n_ropes), threads)
        nv, workload = int(scene[1][:n_ropes].sum()), f"config3-uneven-{C3_ROPES}"
        sample = f"the first {n_ropes} of the {C3_ROPES} config-3 ropes per step ({nv} vertices)"

        def frame(f):
            c3_cpu_frame(sims, inputs, f)

    for f in range(args.warmup):
        frame(f)
    t0 = time.perf_counter()
    for f in range(args.warmup, frames):
        frame(f)
    el = time.perf_counter() - t0
    value = nv * S * args.steps / el
    sample += f", {S} substeps, {ITERS} itr; FP32 CPU restatement of the reference's algorithm on {threads} threads"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload + " (bounded CPU sample)", "ropes_per_step": n_ropes, "verts_per_step": nv,
                       "substeps": S, "num_itr": ITERS},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference CUDA build unavailable (GLM headers absent); the reference arm is the oracle port"}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ config 3 (the target)
def c3_legs(args, world, rank, local, dev, dist, extras):
    """Config 3 on this rank's shard: the persistent device-timed leg, the end-to-end leg and (with
    `extras`, one rank) the plain paths and the CPU baseline. Returns the line's fields."""
    import torch

    import ropesim
    from ropesim import sdf

    R = args.ropes or C3_ROPES
    scene = Sc.bench_c3_scene(sdf, R, seed=3 + 7919 * rank)
    verts = scene[1]
    nv = int(np.sum(verts))
    W, K = args.warmup, args.steps
    F = 2 * (W + K)
    inputs = Sc.bench_c3_inputs(scene, F, seed=17 + rank)
    PP, QQ, p0, v0, p1 = inputs
    Td = [tuple(torch.as_tensor(x[f], device=dev) for x in inputs) for f in range(W + K)]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2

    b = Sc.bench_c3_build(ropesim, scene)
    b.set_timing(True)
    st = torch.cuda.ExternalStream(b.stream_ptr())

    def frame(bb, f, T):
        bb.set_mesh_poses_all(T[0], T[1], teleport=(f == 0))
        bb.step(T[2], T[3], DT, S, root_pos_end=T[4])

    for f in range(W):
        frame(b, f, Td[f])
    torch.cuda.synchronize()
    barrier(dist)
    kernel_ms = []
    sampler = ClockSampler(local)
    with sampler:
        ms = timed_frames(lambda f: frame(b, f, Td[f]), range(W, W + K), st, flush, kernel_ms, b)
    torch.cuda.synchronize()
    total_ms = max_over_ranks(sum(ms), dist, dev)
    barrier(dist)
    value = job_rate(world, nv * S * K, total_ms * 1e-3)
    pos_ok = bool(torch.isfinite(torch.as_tensor(b.positions())).all())

    layout = list(b.layout())
    del b, Td
    torch.cuda.empty_cache()

    # ---- end to end: pinned host poses and programs in, positions out, through the public API,
    # on the same frames: a second batch of the same scene takes the W warm-up frames through the
    # host path too (stepping is deterministic, so it reaches the device-timed run's frame-W state),
    # then the K timed frames
    e2e_value = None
    if not args.no_e2e:
        b2 = Sc.bench_c3_build(ropesim, scene)
        hs = [torch.as_tensor(x[:W + K]).pin_memory() for x in inputs]
        out = torch.empty((nv, 3), dtype=torch.float32).pin_memory()
        view = torch.as_tensor(b2.positions()).reshape(nv, 3)

        def e2e_frame(f):
            T = tuple(h[f].to(dev, non_blocking=True) for h in hs)
            frame(b2, f, T)
            out.copy_(view)

        for f in range(W):
            e2e_frame(f)
        torch.cuda.synchronize()
        barrier(dist)
        t0 = time.perf_counter()
        for f in range(W, W + K):
            e2e_frame(f)
        torch.cuda.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t0, dist, dev)
        e2e_value = job_rate(world, nv * S * K, e2e_s)
        del b2
        torch.cuda.empty_cache()
    h2d = R * M3 * 7 * 4 + R * 9 * 4
    d2h = nv * 3 * 4

    res = {"value": value, "ms_per_step": total_ms / K, "kernel_ms_per_frame": float(np.mean(kernel_ms)),
           "R": R, "nv": nv, "layout": layout, "finite": pos_ok, "clocks": sampler.summary(),
           "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                   "inputs": "per step: mesh poses [R, 8, 7] + root program [R, 9] float32 from pinned host memory; "
                             "out: positions view [n, 3] to pinned host memory"}}
    if not extras:
        return res

    # ---- the plain per-substep-launch engine on the same inputs (one packed batch)
    nplain_w, nplain = min(W, 3), min(K, 3)
    pb = Sc.bench_c3_build(ropesim, scene)
    pb.set_engine("plain")
    pst = torch.cuda.ExternalStream(pb.stream_ptr())
    Tp = [tuple(torch.as_tensor(x[f], device=dev) for x in inputs) for f in range(nplain_w + nplain)]
    for f in range(nplain_w):
        frame(pb, f, Tp[f])
    pms = timed_frames(lambda f: frame(pb, f, Tp[f]), range(nplain_w, nplain_w + nplain), pst, flush)
    pvalue = nv * S * nplain / (sum(pms) * 1e-3)
    res["plain_path"] = {"value": pvalue, "unit": UNIT, "ms_per_step": float(np.mean(pms)), "steps": nplain,
                         "launches_per_step": S * (3 + 2 * ITERS) + 3,
                         "note": "per-substep-launch plain engine over one packed batch of the same ropes (the "
                                 "reference's launch structure, in-repo; the reference's own CUDA build is unavailable)"}
    res["speedup_vs_plain"] = res["value"] / world / pvalue
    del pb, Tp
    torch.cuda.empty_cache()
    if not args.no_per_length:
        res["plain_per_length"] = plain_per_length(ropesim, scene, inputs, dev, flush)
        res["speedup_vs_plain_per_length"] = res["value"] / world / res["plain_per_length"]["value"]
    if not args.no_cpu and world == 1:
        res["cpu_baseline"] = cpu_leg_c3(scene, inputs)
    return res


def plain_per_length(ropesim, scene, inputs, dev, flush, nwarm=2, nsteps=2):
    """The plain path as the reference's API can run uneven ropes: RopeBatch holds ropes of one
    length, so the scene becomes one plain-engine batch per distinct vertex count (each with its
    own copy of the lattices), stepped in sequence on one stream every frame. Same ropes,
    stiffnesses, masses, planes, mesh poses and root programs as the packed batch; a frame is
    timed with CUDA events on the legacy default stream, which every batch's blocking stream is
    ordered with."""
    import torch

    verts = scene[1]
    PP, QQ, p0, v0, p1 = inputs
    batches = []
    for Vr in np.unique(verts):
        idx = np.nonzero(verts == Vr)[0]
        b = Sc.bench_c3_build(ropesim, scene, sel=idx)
        b.set_engine("plain")
        batches.append((b, idx))
    nv = int(np.sum(verts))
    ms = []
    for f in range(nwarm + nsteps):
        sub = [(b, *(torch.as_tensor(np.ascontiguousarray(x[f][i]), device=dev) for x in (PP, QQ, p0, v0, p1)))
               for b, i in batches]
        if f >= nwarm:
            flush.fill_(float(f))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
        for b, pp, pq, a0, a1, a2 in sub:
            b.set_mesh_poses_all(pp, pq, teleport=(f == 0))
            b.step(a0, a1, DT, S, root_pos_end=a2)
        if f >= nwarm:
            e1.record()
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
    finite = all(bool(torch.isfinite(torch.as_tensor(b.positions())).all()) for b, _ in batches)
    res = {"value": nv * S * len(ms) / (sum(ms) * 1e-3), "unit": UNIT, "ms_per_step": float(np.mean(ms)),
           "batches": len(batches), "steps": nsteps, "finite": finite,
           "note": "one plain-engine RopeBatch per distinct vertex count (the reference's RopeBatch takes ropes of "
                   "one length), stepped in sequence"}
    del batches
    torch.cuda.empty_cache()
    return res


# ------------------------------------------------------------------ config 2
def c2_legs(args, world, rank, local, dev, dist, steps, warmup, e2e=True, plain=True, sampler=None):
    """Config 2 (4096 x 64 ropes per rank, plane z = 0, program roots): device-timed frames, the
    end-to-end frames and the plain engine on the same inputs."""
    import torch

    import ropesim

    N = C2_ROPES
    frames = warmup + steps
    pos, p0, v0, p1 = Sc.bench_c2_inputs(N, 2 * frames, 1234 + rank)
    b = ropesim.RopeBatch.from_positions(pos, 0.117, 11473.0, 4.48e-3, H, ITERS, deterministic=True)
    Sc.bench_c2_configure(b)
    if args.block:
        b.set_block(args.block)
    b.set_timing(True)
    P0, V0, P1 = (torch.as_tensor(x, device=dev) for x in (p0, v0, p1))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    for f in range(warmup):
        b.step(P0[f], V0[f], DT, S, root_pos_end=P1[f])
    torch.cuda.synchronize()
    barrier(dist)
    stream = torch.cuda.ExternalStream(b.stream_ptr())
    kernel_ms = []

    def step(f):
        b.step(P0[f], V0[f], DT, S, root_pos_end=P1[f])

    if sampler is not None:
        with sampler:
            ms = timed_frames(step, range(warmup, frames), stream, flush, kernel_ms, b)
    else:
        ms = timed_frames(step, range(warmup, frames), stream, flush, kernel_ms, b)
    torch.cuda.synchronize()
    total_ms = max_over_ranks(sum(ms), dist, dev)
    barrier(dist)
    vs = N * V * S * steps
    res = {"value": job_rate(world, vs, total_ms * 1e-3), "unit": UNIT, "ms_per_step": total_ms / steps,
           "kernel_ms_per_frame": float(np.mean(kernel_ms)), "steps": steps, "bins": list(b.layout())}
    if e2e:
        hp0, hv0, hp1 = (torch.as_tensor(x).pin_memory() for x in (p0, v0, p1))
        out = torch.empty((N, V, 3), dtype=torch.float32).pin_memory()
        view = torch.as_tensor(b.positions())

        def e2e_frame(f):
            a0 = hp0[f].to(dev, non_blocking=True)
            a1 = hv0[f].to(dev, non_blocking=True)
            a2 = hp1[f].to(dev, non_blocking=True)
            b.step(a0, a1, DT, S, root_pos_end=a2)
            out.copy_(view)

        for f in range(frames, frames + warmup):
            e2e_frame(f)
        torch.cuda.synchronize()
        barrier(dist)
        t0 = time.perf_counter()
        for f in range(frames + warmup, 2 * frames):
            e2e_frame(f)
        torch.cuda.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t0, dist, dev)
        res["e2e"] = {"value": job_rate(world, vs, e2e_s), "unit": UNIT, "h2d_bytes_per_step": 3 * N * 3 * 4,
                      "d2h_bytes_per_step": N * V * 3 * 4}
    del b
    if plain:
        pb = ropesim.RopeBatch.from_positions(pos, 0.117, 11473.0, 4.48e-3, H, ITERS, deterministic=True)
        Sc.bench_c2_configure(pb)
        pb.set_engine("plain")
        pstream = torch.cuda.ExternalStream(pb.stream_ptr())
        for f in range(min(warmup, 3)):
            pb.step(P0[f], V0[f], DT, S, root_pos_end=P1[f])
        nplain = min(steps, 3)
        pms = timed_frames(lambda f: pb.step(P0[f], V0[f], DT, S, root_pos_end=P1[f]), range(warmup, warmup + nplain),
                           pstream, flush)
        pvalue = N * V * S * nplain / (sum(pms) * 1e-3)
        res["plain_path"] = {"value": pvalue, "unit": UNIT, "ms_per_step": sum(pms) / nplain, "steps": nplain,
                             "launches_per_step": S * (3 + 2 * ITERS) + 1}
        res["speedup_vs_plain"] = res["value"] / world / pvalue
        del pb
    torch.cuda.empty_cache()
    return res


def c2_roofline(c2, fp32_peak):
    flops_vs = read_profile_value("flop_count_config2.txt", "flops_per_vertex_substep")
    achieved = flops_vs * C2_ROPES * V * S / (c2["kernel_ms_per_frame"] * 1e-3) / 1e12
    return {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
            "flops_per_vertex_substep": flops_vs}


def run_config2(args):
    """The config-2 line on its own (4096 x 64 ropes per GPU), as in the earlier headline."""
    world, rank, local, dev, dist = dist_setup()
    sampler = ClockSampler(local)
    c2 = c2_legs(args, world, rank, local, dev, dist, args.steps, args.warmup, e2e=not args.no_e2e,
                 plain=not args.no_plain, sampler=sampler)
    if rank == 0:
        peaks, source = measured_peaks()
        fp32 = fp32_peak_tflops()
        roof = c2_roofline(c2, fp32)
        state_bytes = C2_ROPES * V * (6 * 16 + 4 * 16 + 40)
        roof.update({"traffic": read_profile_value("frame_kernel_config2.txt", "dram_bytes_per_launch"),
                     "peak_source": "measured FP32 FMA probe (rs_probe_fp32_peak) on this GPU",
                     "hbm_view": {"algorithmic_bytes_per_launch": state_bytes,
                                  "achieved_gbs": state_bytes / (c2["kernel_ms_per_frame"] * 1e-3) / 1e9,
                                  "peak_gbs": peaks.get("hbm_gbs"), "peak_source": source}})
        line = {"metric": METRIC, "value": c2["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": c2["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded config-2 ropes and root programs)",
                "config": {"workload": "config2-program-4096x64", "ropes_per_gpu": C2_ROPES, "verts_per_rope": V,
                           "substeps": S, "num_itr": ITERS, "h": H, "planes": 1,
                           "l2": "flushed between frames (256 MB write)", "bins": c2["bins"],
                           "parallelism": f"ropes sharded by rank x{world} (independent)"},
                "e2e": c2.get("e2e"), "gpu_launches": args.steps, "roofline": roof,
                "kernel_ms_per_frame": c2["kernel_ms_per_frame"], "plain_path": c2.get("plain_path"),
                "speedup_vs_plain": c2.get("speedup_vs_plain"), "clocks": sampler.summary()}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ config 4 (differentiable)
def c4_legs(args, rollouts_warm=3, rollouts=3, R=1024):
    """Config 4: differentiable rollouts of 1024 ropes x 64 vertices (config-1 rope: 3 cm segments,
    0.1 kg/m, EA 500 N, EI 1e-4 N m^2), 30 control frames x 100 substeps, program roots, loss = mean
    squared tip distance to a seeded target curve. One step = one 30-frame rollout: forward only
    (RopeBatch.step), forward + backward (ropesim.grad.frame + loss.backward(), gradients of the
    programs, EA, EI, mass and the initial state), and the plain per-substep path's forward."""
    import torch

    import ropesim
    import ropesim.grad as rg

    Vr, F, S4 = 64, args.frames or 30, 100
    seg, density, ea, ei = 0.03, 0.1, 500.0, 1e-4
    rng = np.random.default_rng(4)
    roots = np.stack([rng.uniform(-0.5, 0.5, R), rng.uniform(-0.5, 0.5, R), rng.uniform(2.5, 3.5, R)], 1).astype(np.float32)
    pos = np.repeat(roots[:, None], Vr, 1) - np.array([0, 0, seg], np.float32) * np.arange(Vr, dtype=np.float32)[None, :, None]
    pos[:, 1:] += rng.normal(0, 1e-3, (R, Vr - 1, 3)).astype(np.float32)
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
    nv = R * Vr

    def timed(fn, n):
        ms = []
        for k in range(n):
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
    tape = False if args.no_tape else ("iterates" if args.iterate_tape else True)
    for engine in ("persistent",) if args.no_plain else ("persistent", "plain"):
        b = make(engine)
        st0 = rg.state(b)

        def fwd(b=b, st0=st0):
            b.set_state(*st0)
            for f in range(F):
                b.step(P[0][f], P[1][f], DT, S4, root_pos_end=P[2][f])

        timed(fwd, rollouts_warm)
        ms = timed(fwd, rollouts)
        out[engine] = {"ms_per_rollout": float(np.mean(ms)), "value": nv * S4 * F * len(ms) / (sum(ms) * 1e-3),
                       "bins": list(b.layout())}
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
                    cur = rg.frame(b, cur, par, pr[0][f], pr[1][f], pr[2][f], DT, S4, tape=tape)
                    loss = loss + ((cur[0].view(R, Vr, 3)[:, -1] - tgt[f]) ** 2).sum(-1).mean()
                loss.backward()
                grads["tensors"] = [t.grad for t in st + par + pr]  # checked after the timed rollouts
                grads["loss_t"] = loss.detach()

            timed(fwd_bwd, rollouts_warm)
            msb = timed(fwd_bwd, rollouts)
            grads["finite"] = bool(all(torch.isfinite(t).all() for t in grads["tensors"]))
            out["fwd_bwd"] = {"ms_per_rollout": float(np.mean(msb)), "value": nv * S4 * F * len(msb) / (sum(msb) * 1e-3),
                              "grads_finite": grads["finite"], "loss": float(grads["loss_t"])}
            del grads
        del b
    torch.cuda.empty_cache()
    res = {"workload": f"config4-diff-{R}x{Vr}", "frames": F, "substeps": S4, "rollouts": rollouts,
           "backward": "replays each frame" if args.no_tape else (
               "from the forward's substep and iterate tapes" if args.iterate_tape else "from the forward's substep tapes"),
           "forward": out["persistent"], "fwd_bwd": out["fwd_bwd"],
           "fwd_bwd_over_fwd": out["fwd_bwd"]["ms_per_rollout"] / out["persistent"]["ms_per_rollout"]}
    if "plain" in out:
        res["plain_path_forward"] = out["plain"]
        res["fwd_speedup_vs_plain"] = out["persistent"]["value"] / out["plain"]["value"]
        res["fwd_bwd_speedup_vs_plain_fwd"] = out["fwd_bwd"]["value"] / out["plain"]["value"]
    return res


def run_config4(args):
    import torch

    torch.cuda.set_device(0)
    c4 = c4_legs(args, rollouts_warm=args.warmup, rollouts=args.steps, R=args.ropes or 1024)
    line = {"metric": METRIC + " (config-4 fwd+bwd)", "value": c4["fwd_bwd"]["value"], "unit": UNIT,
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": c4["fwd_bwd"]["ms_per_rollout"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded config-4 rollouts)",
            "config": {"workload": c4["workload"], "frames": c4["frames"], "substeps": c4["substeps"], "num_itr": ITERS,
                       "step": f"one {c4['frames']}-frame rollout", "backward": c4["backward"],
                       "counted": "forward vertex-substeps of the rollout", "l2": "flushed between rollouts (256 MB write)"},
            **{k: v for k, v in c4.items() if k not in ("workload", "frames", "substeps", "backward")}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ the default line
def run_target(args):
    """The default line: config 3 (the target configuration) with the plain paths beside it, and
    config 2 and config 4 measured in the same run (one rank; with N > 1 ranks each rank runs its
    own shard of config 3 and the extras are skipped)."""
    import torch

    world, rank, local, dev, dist = dist_setup()
    extras = world == 1
    c3 = c3_legs(args, world, rank, local, dev, dist, extras)
    c2 = c4 = None
    if extras and not args.no_extras:
        c2 = c2_legs(args, world, rank, local, dev, dist, steps=min(args.steps, 10), warmup=args.warmup)
        c4 = c4_legs(args)
    if rank == 0:
        peaks, source = measured_peaks()
        fp32 = fp32_peak_tflops()
        flops_vs = read_profile_value("flop_count_config3.txt", "flops_per_vertex_substep")
        kms = c3["kernel_ms_per_frame"]
        roof = {"bound": "fp32", "unit": "TFLOP/s", "peak": fp32,
                "peak_source": "measured FP32 FMA probe (rs_probe_fp32_peak) on this GPU; MEASURED_PEAKS.json carries "
                               "no FP32 figure",
                "kernel": "frame_kernel<256, SURF_MESHES> (one launch per frame)", "kernel_ms_per_frame": kms}
        if flops_vs:
            achieved = flops_vs * c3["nv"] * S / (kms * 1e-3) / 1e12
            roof.update({"achieved": achieved, "frac": achieved / fp32, "flops_per_vertex_substep": flops_vs})
        t = read_profile_value("frame_kernel_config3.txt", "dram_bytes_per_launch")
        roof["traffic"] = t
        state_bytes = c3["nv"] * (6 * 16 + 4 * 16 + 40)
        roof["hbm_view"] = {"algorithmic_bytes_per_launch": state_bytes,
                            "achieved_gbs": state_bytes / (kms * 1e-3) / 1e9, "peak_gbs": peaks.get("hbm_gbs"),
                            "peak_source": source}
        line = {"metric": METRIC, "value": c3["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": c3["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded config-3 scene: uneven ropes, per-rope EA/EI, per-vertex masses, two planes, "
                        "eight 64^3 lattices with per-env random-walk poses, root programs)",
                "config": {"workload": f"config3-uneven-{c3['R']}", "ropes_per_gpu": c3["R"], "verts_per_gpu": c3["nv"],
                           "verts_per_rope": "U{16..256}", "substeps": S, "num_itr": ITERS, "h": H, "planes": 2,
                           "meshes": M3, "lattice": "64^3 float32", "l2": "flushed between frames (256 MB write)",
                           "bins": c3["layout"], "parallelism": f"ropes sharded by rank x{world} (independent)"},
                "e2e": c3["e2e"], "gpu_launches": 4 * args.steps,
                "gpu_launches_note": "per frame: scatter_targets, stage_motion, frame_kernel, commit",
                "roofline": roof, "kernel_ms_per_frame": kms, "finite": c3["finite"], "clocks": c3["clocks"]}
        for k in ("speedup_vs_plain", "plain_path", "speedup_vs_plain_per_length", "plain_per_length", "cpu_baseline"):
            if k in c3:
                line[k] = c3[k]
        if c4 is not None:
            line["fwd_bwd_over_fwd"] = c4["fwd_bwd_over_fwd"]
            line["config4"] = c4
        if c2 is not None:
            c2["roofline"] = c2_roofline(c2, fp32)
            line["config2"] = c2
        par = read_parity()
        if par is not None:
            line["parity"] = par
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ config 3 alone (profiling)
def run_config3(args):
    """Config 3 forward alone, persistent vs the packed plain path (no extras): the profiling entry."""
    world, rank, local, dev, dist = dist_setup()
    args.no_e2e = True
    c3 = c3_legs(args, world, rank, local, dev, dist, extras=not args.no_plain)
    if rank == 0:
        line = {"metric": METRIC, "value": c3["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": c3["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded config-3 scene)",
                "config": {"workload": f"config3-uneven-{c3['R']}", "verts": c3["nv"], "bins": c3["layout"]},
                "kernel_ms_per_frame": c3["kernel_ms_per_frame"], "clocks": c3["clocks"]}
        for k in ("speedup_vs_plain", "plain_path", "speedup_vs_plain_per_length", "plain_per_length"):
            if k in c3:
                line[k] = c3[k]
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


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
    One step = the frames of --fit-window (default: all --frames) forward (with tapes) and
    backward, then one Adam step (--lr) on per-rope log EA / log EI, each frame's gradient clipped
    to --clip (norm over both parameter vectors; 0 = no clipping). Reported: fitting steps/s,
    forward + backward vertex-substeps/s, the forward-only rollout, and with --fit-steps N the
    parameter errors after N steps (with the loss and errors of every step)."""
    import torch

    import ropesim
    import ropesim.grad as rg

    torch.cuda.set_device(0)
    R = args.ropes or 256
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
    opt = torch.optim.Adam([log_ea, log_ei], lr=args.lr, eps=1e-12)

    def errors():
        with torch.no_grad():
            e_ea = (log_ea.exp() / true_ea).log().abs().median()
            e_ei = (log_ei.exp() / true_ei).log().abs().median()
        return float(e_ea), float(e_ei)

    info = {"dropped_frames": 0, "clipped_frames": 0, "history": []}
    f0, f1 = (int(x) for x in args.fit_window.split(":")) if args.fit_window else (0, F)
    fit_frames = range(max(0, f0), min(F, f1))

    def fit_step():
        g_ea, g_ei = torch.zeros_like(log_ea), torch.zeros_like(log_ei)
        total = 0.0
        for f in fit_frames:
            par = (per_vertex(log_ea.exp()), per_vertex(log_ei.exp()), mass)
            out = rg.frame(b, traj[f], par, None, None, None, DT, S5)
            loss = ((out[0] - traj[f + 1][0]) ** 2).sum(-1).mean() * 1e6  # mm^2
            ga, gi = torch.autograd.grad(loss, (log_ea, log_ei))
            if bool(torch.isfinite(ga).all() and torch.isfinite(gi).all()):
                gn = float(torch.sqrt((ga * ga).sum() + (gi * gi).sum()))
                if args.clip > 0 and gn > args.clip:
                    ga, gi = ga * (args.clip / gn), gi * (args.clip / gn)
                    info["clipped_frames"] += 1
                g_ea += ga
                g_ei += gi
            else:
                info["dropped_frames"] += 1
            total += float(loss.detach())
        log_ea.grad, log_ei.grad = g_ea, g_ei
        info["loss"] = total
        opt.step()
        info["history"].append([round(total, 6), *[round(e, 5) for e in errors()]])

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
                "window": [fit_frames.start, fit_frames.stop], "lr": args.lr, "clip": args.clip,
                "loss_first_step": loss_first, "loss_last_step": info["loss"],
                "frames_dropped_for_overflow": info["dropped_frames"], "frames_clipped": info["clipped_frames"],
                "history_loss_err_ea_err_ei": info["history"],
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

    torch.cuda.set_device(0)
    R = args.ropes or C3_ROPES
    from ropesim import sdf

    scene = Sc.bench_c3_scene(sdf, R)
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
        b = Sc.bench_c3_build(ropesim, scene)
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
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="target",
                    choices=["target", "config2", "config3", "config4", "config5", "bake", "exchange"],
                    help="target (default: config 3 with the plain paths, plus config 2 and config 4 in the same run), "
                         "config2 / config3 / config4 / config5 alone, exchange (the Isaac-bridge loop), bake (mesh baking)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--ropes", type=int, default=0, help="ropes per GPU (0 = the workload's own; profiling of smaller cases)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling)")
    ap.add_argument("--block", type=int, default=0, help="config2: bin size (CTA threads); 0 = the library's choice")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-path legs")
    ap.add_argument("--no-per-length", action="store_true", help="skip the one-batch-per-rope-length plain leg")
    ap.add_argument("--no-extras", action="store_true", help="target: skip the config-2 and config-4 legs")
    ap.add_argument("--frames", type=int, default=0,
                    help="control frames per rollout (0 = the workload's own: 30 for config4, 60 for config5)")
    ap.add_argument("--no-tape", action="store_true", help="config4: backward replays frames instead of keeping tapes")
    ap.add_argument("--no-iterate-tape", dest="iterate_tape", action="store_false",
                    help="config4: keep only the substep tapes (the backward recomputes the iterates)")
    ap.add_argument("--fit-steps", type=int, default=0, help="config5: total fitting steps to run (e.g. 50)")
    ap.add_argument("--iters", type=int, default=0, help="config5: Jacobi sweeps per substep (0 = the default 8)")
    ap.add_argument("--fit-window", default="", help="config5: frames a:b the fit's loss uses (default all)")
    ap.add_argument("--clip", type=float, default=0.0, help="config5: clip each frame's gradient norm to this (0 = off)")
    ap.add_argument("--lr", type=float, default=0.05, help="config5: Adam learning rate on log EA / log EI")
    ap.add_argument("--bake-subdiv", type=int, default=5, help="bake: icosphere subdivisions of the baked mesh")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    maybe_relaunch(args)
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "config2":
        run_config2(args)
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
        run_target(args)


if __name__ == "__main__":
    main()
