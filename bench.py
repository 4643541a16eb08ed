#!/usr/bin/env python
"""Benchmark: body-steps per second of the batched uneven-worlds workload.

Workload: 4096 independent worlds (per GPU) of 8-512 bodies each (log-uniform), 70% boxes and 30% spheres
in a seeded stack or scatter above a half-space, dt 1/60, 4 substeps. Every step runs the whole contact
pipeline of every world on the device (broadphase, narrowphase, coloring, the substepped soft solve,
restitution, sleep) from one CUDA graph per step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--worlds 4096] [--impl b200|reference]

value: awake dynamic bodies summed over the K timed steps of all worlds on all GPUs, divided by the device
time of those steps (CUDA events on the library's stream; max over ranks). Under torchrun the world set holds
4096 worlds per GPU and is split over the ranks by longest-processing-time on body counts (weak scaling, no
collective in the step; one gather of per-world results after timing).

parity: the end-to-end batch's every 4th world against the reference stepping the same worlds the same steps
(the CPU baseline's own run): states within 1e-5, bit-identical worlds and identical candidate pairs.

e2e: the same metric through the public C ABI on a fresh batch stepped the same way, with each step's
inputs (per-body forces, from pinned host memory) copied in and every body's pose copied out inside the
timed region, timed by the host clock.

--impl reference: the unmodified reference World::step (compiled from its own sources into
oracle/_ref/libtwofold_ref.so) on a bounded sample of the same worlds, one world per thread from a pool of
every host core.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "body-steps/s"
UNIT = "body-steps/s"
SAMPLE_STRIDE = 4  # the CPU sample steps every 4th world


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--worlds", type=int, default=4096)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the plain-path and adjoint measurements")
    ap.add_argument("--shapes", default=None,
                    help="launch shapes as JSON {kernel: [threads, big-world bodies, shared bytes]} in place of the "
                         "autotuner's, e.g. the launch_shapes of an earlier run (for profiling that run's kernels)")
    ap.add_argument("--single", default=None, choices=list(SINGLE_WORLDS),
                    help="run only this single-world configuration, without the reference, and print its entry "
                         "(for profiling its kernels)")
    return ap.parse_args()


def config(args, n_gpus):
    return {
        "workload": "batched_uneven_worlds",
        "worlds_per_gpu": args.worlds,
        "bodies_per_world": "log-uniform 8-512, 70% boxes / 30% spheres, stack or scatter, half-space ground",
        "dt": "1/60",
        "substeps": 4,
        "timed_steps": f"{args.warmup + 1}..{args.warmup + args.steps} of the 240-step run",
        "parallelism": f"independent worlds, {n_gpus} GPU(s), no collective in the step",
        "l2_flush": "not needed: the step's resident state (bodies, contacts, axes) is far larger than L2",
    }


# ------------------------------------------------------------------------------------------------------------
# Distributed plumbing


class Dist:
    """One process per GPU from torchrun's environment. The ranks share nothing inside a step; the process group
    carries the barriers around the timed region and the reductions of its results (max of the device times,
    sum of the body-steps). NCCL on GPUs; gloo on CPU (`backend`), which the multi-process tests use."""

    def __init__(self, backend=None, timeout_s=300):
        self.world_size = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.cuda = False
        if self.world_size > 1:
            import datetime

            import torch
            import torch.distributed as dist

            backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
            self.cuda = backend == "nccl"
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if self.cuda:
                torch.cuda.set_device(self.local_rank)
                kw["device_id"] = torch.device("cuda", self.local_rank)
            dist.init_process_group(backend, **kw)
            self.pg = dist

    def barrier(self):
        import torch

        if torch.cuda.is_available():
            torch.cuda.synchronize()
        if self.pg:
            self.pg.barrier()
            if torch.cuda.is_available():
                torch.cuda.synchronize()

    def reduce(self, value, op):
        if not self.pg:
            return value
        import torch

        device = f"cuda:{self.local_rank}" if self.cuda else "cpu"
        t = torch.tensor([float(value)], dtype=torch.float64, device=device)
        self.pg.all_reduce(t, op=getattr(self.pg.ReduceOp, op))
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ------------------------------------------------------------------------------------------------------------
# Clocks during the timed region


class ClockSampler:
    FIELDS = ["clocks.sm", "clocks.max.sm", "clocks_event_reasons.active", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown",
              "clocks_event_reasons.sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []  # (host time, csv line)
        self.window_start = self.window_stop = None

    def start(self):
        """Starts sampling ahead of the timed region: nvidia-smi takes a fraction of a second to begin, longer
        than the whole timed region can be; only samples inside the window count."""
        if self.proc:
            return self
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", "--query-gpu=" + ",".join(self.FIELDS), "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def __enter__(self):
        self.start()
        self.window_start = time.monotonic()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def __exit__(self, *exc):
        self.window_stop = time.monotonic()

    def close(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.proc = None

    def summary(self):
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lo, hi = self.window_start or 0.0, (self.window_stop or time.monotonic()) + 0.05
        for t, line in list(self.lines):
            if not lo <= t <= hi:
                continue
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[3:7]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------------------------------------------
# The reference on the host cores


def reference_rate(worlds, settings, dt, warmup, steps, threads):
    """Reference World::step on `worlds`, one world per thread; body-steps/s over the last `steps` steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reference as R

    refs = [R.RefWorld(w, settings) for w in worlds]
    if warmup:
        R.step_parallel(refs, dt, warmup, threads)
    t0 = time.perf_counter()
    body_steps = R.step_parallel(refs, dt, steps, threads)
    elapsed = time.perf_counter() - t0
    return body_steps / elapsed, body_steps, elapsed


def run_reference(args, dist):
    if dist.rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reference as R
    from twofold_b200 import scenes

    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libtwofold_ref.so was not built"}))
        return
    sc = scenes.config4(n_worlds=args.worlds)
    sample = sc.worlds[::SAMPLE_STRIDE]
    threads = R.hardware_threads()
    rate, body_steps, elapsed = reference_rate(sample, sc.settings, sc.dt, args.warmup, args.steps, threads)
    desc = (f"every {SAMPLE_STRIDE}th world ({len(sample)} of {args.worlds}), steps {args.warmup + 1}-"
            f"{args.warmup + args.steps}, {body_steps} body-steps in {elapsed:.2f} s")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3 * SAMPLE_STRIDE,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config(args, args.gpus),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference", "sample": desc},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


# ------------------------------------------------------------------------------------------------------------
# The B200 library


def substep_bytes(work):
    """Algorithmic bytes of one k_substep launch: each awake body read and written once (160 B) and, in each
    of its 3 passes (warm start, biased solve, relax), each active contact (64 B) and contact point (84 B)."""
    return 160 * work["awake"] + 3 * (64 * work["active_contacts"] + 84 * work["active_points"])


def load_traffic(mode):
    """The k_substep DRAM traffic of one ncu capture for the substep's launch mode ("world": the world kernel,
    "flat": the flat solve), with the work counts of the step it was captured on."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            t = json.load(f).get(mode)
        if t and "work" in t and "k_substep_bytes_per_launch" in t:
            return t
    return None


PLAIN_STRIDE = 64  # every 64th world stepped on its own


def plain_rate(sc, args, device):
    """Body-steps/s of the plain path: worlds stepped one by one, each a batch of one world on the same GPU
    (its own graph per step, launch shapes from the autotuner on that world after the warm-up, as the batch
    has), over a sample of the workload's worlds; device time summed over the worlds."""
    from twofold_b200.world import Batch

    ms, body_steps = 0.0, 0
    sample = sc.worlds[::PLAIN_STRIDE]
    for w in sample:
        one = Batch([w], sc.settings, device=device)
        for _ in range(args.warmup):
            one.step_checked(sc.dt, 1, graph=True)
        one.autotune(sc.dt, trial_steps=1)
        b0 = one.body_steps()
        for _ in range(args.steps):
            one.step_checked(sc.dt, 1, graph=True)
            ms += one.elapsed_ms()
        body_steps += one.body_steps() - b0
        one.close()
    return {"value": body_steps / (ms / 1e3), "unit": UNIT, "device_ms": ms,
            "sample": f"every {PLAIN_STRIDE}th world ({len(sample)} of {len(sc.worlds)}), each alone and tuned, steps "
                      f"{args.warmup + 1}-{args.warmup + args.steps}"}


def single_worlds(device, warmup=20, steps=40, only=None, reference=True):
    """The plain path on the single-world configurations (box pyramid, terrain, planar pile): device ms per
    step through the C ABI (a CUDA graph per step, launch shapes from the autotuner after the warm-up) over
    steps warmup+1..warmup+steps, beside the reference
    stepping the same world the same steps on one host core. A reported comparison, not the headline."""
    from twofold_b200 import scenes
    from twofold_b200.world import Batch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reference as R

    out = {}
    for name in SINGLE_WORLDS:
        if only and name != only:
            continue
        sc = getattr(scenes, SINGLE_WORLDS[name])()
        one = Batch(sc.worlds, sc.settings, device=device)
        for _ in range(warmup):
            one.step_checked(sc.dt, 1, graph=True)
        one.autotune(sc.dt, trial_steps=1)  # launch shapes for this world, as for the batch
        ms = 0.0
        b0 = one.body_steps()
        for _ in range(steps):
            one.step_checked(sc.dt, 1, graph=True)
            ms += one.elapsed_ms()
        body_steps = one.body_steps() - b0
        # Per-kernel times of the next steps, from graphs with an event pair around each kernel group.
        one.set_profiling(True)
        for _ in range(SINGLE_BREAKDOWN_STEPS):
            one.step_checked(sc.dt, 1, graph=True)
        kt = one.kernel_times()
        one.set_profiling(False)
        one.close()
        entry = {"gpu_ms_per_step": ms / steps, "body_steps_per_s": body_steps / (ms / 1e3),
                 "kernel_ms_per_step": {k: v[0] / SINGLE_BREAKDOWN_STEPS for k, v in kt.items()},
                 "kernel_steps": f"{warmup + steps + 1}-{warmup + steps + SINGLE_BREAKDOWN_STEPS}"}
        if reference and R.available():
            r = R.RefWorld(sc.worlds[0], sc.settings)
            r.step(sc.dt, warmup)
            t0 = time.perf_counter()
            r.step(sc.dt, steps)
            el = time.perf_counter() - t0
            entry.update({"reference_ms_per_step": 1e3 * el / steps, "reference_cores": 1})
        entry["steps"] = f"{warmup + 1}-{warmup + steps}"
        out[name] = entry
    return out


def adjoint_cost(device, n_worlds=1024, steps=120):
    """The differentiable impact workload: record 120 steps of 1024 worlds, run the model forward and the adjoint
    backward in float; device times of both, and of the pipeline's own 120 steps of the same worlds."""
    from twofold_b200 import scenes
    from twofold_b200.world import Batch

    sc = scenes.config5(n_worlds=n_worlds)
    pipe = Batch.from_scene(sc, device=device)
    pipe_ms = 0.0
    for _ in range(steps):
        pipe.step_checked(sc.dt, 1, graph=True)
        pipe_ms += pipe.elapsed_ms()
    pipe.close()
    b = Batch.from_scene(sc, device=device)
    b.tape_record(sc.dt, steps)
    n_shapes = sum(len(w.shapes) for w in sc.worlds)
    final = b.adjoint_forward(32)
    grad = np.zeros_like(final)
    boxes = np.zeros(len(final), bool)
    for wi in range(n_worlds):
        boxes[b.offsets[wi] + 1:b.offsets[wi] + 65] = True
    grad[boxes, 0] = 2 * final[boxes, 0]  # loss: sum of the boxes' squared final x
    b.adjoint_backward(grad, n_shapes)
    fwd, bwd = b.adjoint_ms()
    recompute, reverse = b.adjoint_backward_ms()
    b.close()
    return {"workload": f"impact walls, {n_worlds} worlds x 66 bodies, {steps} steps, checkpoint every step",
            "precision": "f32", "model_forward_ms": fwd, "backward_ms": bwd, "backward_over_forward": bwd / fwd,
            "pipeline_forward_ms": pipe_ms, "backward_over_pipeline_forward": bwd / pipe_ms,
            "backward_parts_ms": {"recompute_summed": recompute, "reverse_summed": reverse}}


SINGLE_WORLDS = {"box_pyramid_210": "config1", "terrain_32768": "config2", "planar_16384": "config3"}
SINGLE_BREAKDOWN_STEPS = 5  # profiled steps after each single world's timed ones
BREAKDOWN_STEPS = 10  # graph-replayed steps after the timed region, with an event pair around each kernel group
TUNE_AHEAD = 10       # the autotuner's batch is stepped this far past the warm-up


def world_set(args, dist):
    """This rank's shard of the one seeded world set: args.worlds worlds per GPU in total, split over the ranks
    by longest-processing-time on body counts (a single GPU takes the whole set, in order)."""
    from twofold_b200 import scenes, shard

    total = args.worlds * dist.world_size
    counts = scenes.config4_bodies(total)
    shards = shard.lpt_partition(counts, dist.world_size)
    mine = shards[dist.rank]
    return scenes.config4(n_worlds=total, only=mine), shards, counts


def state_parity(batch, refs, stride):
    """World states of the GPU batch against the reference worlds (the batch's every stride-th world, stepped
    the same steps): normwise relative error of positions, rotations and velocities, bit-identical worlds, and
    worlds whose candidate pair keys are identical."""
    worst, same, cands = 0.0, 0, 0
    for k, r in enumerate(refs):
        wi = k * stride
        mine, theirs = batch.world_states(wi), r.states()
        for key in ("p", "q", "v", "w"):
            a = np.asarray(mine[key], np.float64)
            b = np.asarray(theirs[key], np.float64)
            if a.size:
                worst = max(worst, float(np.max(np.abs(a - b)) / max(float(np.max(np.abs(b))), 1e-6)))
        same += all(np.array_equal(np.asarray(mine[key]).view(np.uint32), np.asarray(theirs[key]).view(np.uint32))
                    for key in ("p", "q", "v", "w"))
        cands += bool(np.array_equal(batch.candidates(wi), r.candidates()))
    return {"worlds": len(refs), "max_rel_err": worst, "tolerance": 1e-5, "bit_identical_worlds": same,
            "candidates_equal_worlds": cands}


def run_b200(args, dist):
    from twofold_b200 import abi
    from twofold_b200.world import Batch

    abi.load()
    n = dist.world_size
    sc, shards, counts = world_set(args, dist)
    dt = sc.dt
    batch = Batch.from_scene(sc, device=dist.local_rank)
    for _ in range(args.warmup):
        batch.step_checked(dt, 1, graph=True)
    # Launch shapes chosen by the library's autotuner, on a second batch of the same worlds stepped to the middle
    # of the timed window (the worlds' contacts build up over it, and the shapes that suit a step without
    # contacts do not suit one full of them); shapes never change results.
    t_tune = time.perf_counter()
    if args.shapes:
        shapes = {k: tuple(int(x) for x in v) for k, v in json.loads(args.shapes).items()}
    else:
        tuner = Batch.from_scene(sc, device=dist.local_rank)
        for _ in range(args.warmup + TUNE_AHEAD):
            tuner.step_checked(dt, 1, graph=True)
        shapes = tuner.autotune(dt, trial_steps=1)
        tuner.close()
        del tuner
    for k, (threads, big, smem) in shapes.items():
        batch.set_launch(k, threads, big, smem)
    tune_s = time.perf_counter() - t_tune
    launches0 = batch.launches()
    steps0 = batch.body_steps()
    clocks = ClockSampler(dist.local_rank).start()
    time.sleep(1.0)  # nvidia-smi is sampling by the time the timed region starts
    dist.barrier()
    device_ms = 0.0
    t0 = time.perf_counter()
    with clocks:
        for _ in range(args.steps):
            batch.step_checked(dt, 1, graph=True)
            device_ms += batch.elapsed_ms()
    wall = time.perf_counter() - t0
    clocks.close()
    dist.barrier()
    body_steps = batch.body_steps() - steps0
    launches = batch.launches() - launches0
    max_ms = dist.reduce(device_ms, "MAX")
    total_body_steps = dist.reduce(body_steps, "SUM")
    value = total_body_steps / (max_ms / 1e3)

    # Per-kernel times of the next steps, replayed from graphs that hold an event pair around each kernel group,
    # with the algorithmic bytes of every k_substep launch from the work counts of its own step.
    batch.set_profiling(True)
    prof_ms, sub_bytes, works = 0.0, 0, []
    for _ in range(BREAKDOWN_STEPS):
        batch.step_checked(dt, 1, graph=True)
        prof_ms += batch.elapsed_ms()
        works.append(batch.work_counts())
        sub_bytes += substep_bytes(works[-1]) * 4
    kt = batch.kernel_times()
    batch.set_profiling(False)
    top = max(kt, key=lambda k: kt[k][0])
    peaks = {}
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            peaks = json.load(f)
    peak = float(peaks.get("hbm_gbs", 6650.0))
    sub_ms_total = kt["k_substep"][0]
    sub_launches = max(kt["k_substep"][1], 1)
    achieved = sub_bytes / (sub_ms_total / 1e3) / 1e9
    substep_mode = "flat" if shapes.get("substep", (0, 0, 0))[1] == -1 else "world"
    traffic = load_traffic(substep_mode)
    breakdown = {k: v[0] / BREAKDOWN_STEPS for k, v in kt.items()}

    # End to end: a fresh batch, the same warm-up, then per step: forces in, step, poses out. The poses of a step
    # travel to the host (two pinned buffers in turn) while the next step runs; the timed region ends once the
    # last step's poses have arrived.
    del batch
    e2e_batch = Batch.from_scene(sc, device=dist.local_rank)
    for k, (threads, big, smem) in shapes.items():
        e2e_batch.set_launch(k, threads, big, smem)
    total = int(e2e_batch.offsets[-1])
    try:
        import torch

        forces = torch.zeros((total, 3), dtype=torch.float32).pin_memory().numpy()
        poses = [torch.zeros((total, 3), dtype=torch.float32).pin_memory().numpy() for _ in range(2)]
        rots = [torch.zeros((total, 4), dtype=torch.float32).pin_memory().numpy() for _ in range(2)]
    except Exception:
        forces = np.zeros((total, 3), np.float32)
        poses = [np.zeros((total, 3), np.float32) for _ in range(2)]
        rots = [np.zeros((total, 4), np.float32) for _ in range(2)]
    for _ in range(args.warmup):
        e2e_batch.step_checked(dt, 1, graph=True)
    e_steps0 = e2e_batch.body_steps()
    dist.barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        e2e_batch.add_forces(forces)
        e2e_batch.step_checked(dt, 1, graph=True)
        e2e_batch.read_poses_async(poses[k % 2], rots[k % 2])
    e2e_batch.poses_wait()
    e_wall = time.perf_counter() - t0
    dist.barrier()
    e_body_steps = dist.reduce(e2e_batch.body_steps() - e_steps0, "SUM")
    e_wall = dist.reduce(e_wall, "MAX")

    # Every rank's per-world results to rank 0 (outside every timed region): one gather of each world's pose
    # checksum, keyed by its number in the whole set.
    digests = {}
    for k, w in enumerate(shards[dist.rank]):
        st = e2e_batch.world_states(k)
        digests[int(w)] = float(np.abs(np.asarray(st["p"], np.float64)).sum())
    gathered = [digests]
    if dist.pg:
        gathered = [None] * n
        dist.pg.all_gather_object(gathered, digests)
    worlds_gathered = sum(len(g) for g in gathered)

    cpu = None
    parity = None
    if dist.rank == 0 and n == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import reference as R

        if R.available():
            threads = R.hardware_threads()
            sample = sc.worlds[::SAMPLE_STRIDE]
            refs = [R.RefWorld(w, sc.settings) for w in sample]
            if args.warmup:
                R.step_parallel(refs, dt, args.warmup, threads)
            t_ref = time.perf_counter()
            bsteps = R.step_parallel(refs, dt, args.steps, threads)
            el = time.perf_counter() - t_ref
            cpu = {"value": bsteps / el, "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"every {SAMPLE_STRIDE}th world ({len(sample)} of {args.worlds}), steps "
                             f"{args.warmup + 1}-{args.warmup + args.steps}, {bsteps} body-steps in {el:.2f} s"}
            # The same worlds of the end-to-end batch, after the same steps, against those reference worlds.
            parity = state_parity(e2e_batch, refs, SAMPLE_STRIDE)
            parity["steps"] = args.warmup + args.steps
            parity["compared"] = "end-to-end batch (forces of zero added every step) against the reference sample"
    del e2e_batch

    # The plain path for comparison: a sample of the same worlds, each stepped alone as a batch of one.
    plain = None
    if dist.rank == 0 and not args.no_extras:
        plain = plain_rate(sc, args, dist.local_rank)
    adjoint = None
    if dist.rank == 0 and not args.no_extras:
        adjoint = adjoint_cost(dist.local_rank)
    singles = None
    if dist.rank == 0 and n == 1 and not args.no_extras:
        singles = single_worlds(dist.local_rank)

    if dist.rank == 0:
        roof = {"bound": "hbm", "kernel": "k_substep", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": None,
                "peak_source": "measured hbm_gbs (MEASURED_PEAKS.json)" if "hbm_gbs" in peaks else "fallback",
                "algorithmic_bytes_per_launch": sub_bytes / sub_launches, "avg_launch_ms": sub_ms_total / sub_launches,
                "timed_on": f"{BREAKDOWN_STEPS} graph-replayed steps after the timed region, an event pair per kernel",
                "top_kernel_by_time": top}
        if traffic:
            # Measured on a smaller batch: the ratio of traffic to algorithmic bytes at the captured state, and
            # the traffic it implies for this run's launches.
            ratio = traffic["k_substep_bytes_per_launch"] / substep_bytes(traffic["work"])
            roof["traffic"] = ratio * sub_bytes / sub_launches
            roof["traffic_over_algorithmic"] = ratio
            roof["traffic_captured"] = {"substep_mode": substep_mode,
                                        "bytes_per_launch": traffic["k_substep_bytes_per_launch"],
                                        "work": traffic["work"], "source": traffic.get("source")}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": n, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic: one seeded world set, split over the GPUs by body count",
            "config": config(args, n),
            "e2e": {"value": e_body_steps / e_wall, "unit": UNIT, "h2d_bytes_per_step": int(forces.nbytes),
                    "d2h_bytes_per_step": int(poses[0].nbytes + rots[0].nbytes),
                    "copies": "forces in before each step; each step's poses out while the next step runs"},
            "gpu_launches": int(launches),
            "roofline": roof,
            "parity": parity,
            "kernel_breakdown": {"ms_per_step": breakdown, "sum_ms": sum(breakdown.values()),
                                 "steps_ms_per_step": prof_ms / BREAKDOWN_STEPS,
                                 "steps": f"{args.warmup + args.steps + 1}..{args.warmup + args.steps + BREAKDOWN_STEPS}",
                                 "mode": "graph replay, the graph holding an event pair around each kernel group"},
            "launch_shapes": {k: list(v) for k, v in shapes.items()},
            "autotune_s": tune_s,
            "autotune_state": f"a second batch of the same worlds at step {args.warmup + TUNE_AHEAD}",
            "work_last_step": works[-1],
            "shards": {"worlds": [len(s) for s in shards],
                       "bodies": [int(counts[s].sum()) for s in shards], "worlds_gathered": worlds_gathered},
            "wall_s_timed_region": wall,
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
            "plain_one_by_one": plain,
            "adjoint": adjoint,
            "single_world_configs": singles,
        }
        print(json.dumps(line))


def main():
    args = parse()
    if args.single:
        print(json.dumps(single_worlds(0, only=args.single, reference=False)))
        return
    dist = Dist()
    try:
        if args.impl == "reference":
            run_reference(args, dist)
        else:
            run_b200(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
