#!/usr/bin/env python
"""Benchmark of the adaptive GIMP substep on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl agimp|reference] [--config 3]

Metric: particle-substeps/s (particles x substeps / time) of the whole job.
Default workload: the 3D dynamic-adaptivity scene (3 levels, 64^3..256^3,
~1.9M particles, snow plasticity, slab collider, prescribed levels recomputed
every 10 substeps), synthetic seeded data.  A step is one substep of the
whole scene; the refinement every 10th step is inside the timed region.

--impl agimp (default): the CUDA path.  `value` is device time (CUDA events
  on the launching stream, max over ranks) with the state resident in HBM;
  `e2e` is the same metric through the public Python API with host buffers:
  the scene is uploaded from pinned host memory and x_p is read back to
  pinned host memory after every substep, all inside the timed region.
--surrogate NPZ: the snow return map goes through the trained surrogate MLP
  (tensor-core inference, exact fallback); the line adds the plain path's
  throughput on the same scene and the position error against it.
--impl reference: the reference's algorithm on the host cores (the CPU
  oracle restatement, OpenMP on all host threads) on the same scene; rank 0
  only.

Multi-GPU: replicas only (one independent scene per rank, seeded by rank);
the single-scene substep does not shard.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "adaptive-gimp_b200"))
sys.path.insert(0, os.path.join(REPO, "oracle"))

METRIC = "particle-substeps/s"
# the end-to-end run takes at least this many substeps (a wall-clock figure
# over a few milliseconds is dominated by host-side jitter)
E2E_MIN_STEPS = 100
FALLBACK_HBM_GBS = 6650.0
# algorithmic bytes per particle-substep (f32 SoA), counted once per kernel
BYTES = {  # (dim, with Jp) -> (P2G, G2P)
    (2, False): (52, 72), (2, True): (56, 80),
    (3, False): (100, 144), (3, True): (104, 152),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="agimp", choices=["agimp", "reference"])
    ap.add_argument("--config", type=int, default=3)
    ap.add_argument("--scale", type=float, default=1.0, help="body scale of the scene (profiling cases)")
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="budget of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--parity-substeps", type=int, default=100,
                    help="substeps of the full scene compared with the f32 / f64 oracle in the CPU leg (0: none)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--surrogate", default=None, metavar="NPZ",
                    help="snow return map through this trained surrogate (agimp.train_surrogate output); the line "
                         "then also reports the plain path's throughput and the position error against it")
    ap.add_argument("--sur-tol", type=float, default=1e-3, help="surrogate residual tolerance")
    ap.add_argument("--snow", action="store_true",
                    help="config 4 with config 2's snow material (each box thrown at a random velocity)")
    ap.add_argument("--accuracy-substeps", type=int, default=1000,
                    help="config 4 with --surrogate: substeps of the accuracy comparison against the plain batch")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch sizes")
    ap.add_argument("--tuning", default=None, metavar="CHUNK,CTAS_PER_SM",
                    help="fixed launch sizes instead of the autotuner (e.g. 64,16)")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profile_traffic(kernel, workload):
    """dram bytes per particle for `kernel` from the committed ncu summary
    (profiles/*.md lines 'TRAFFIC <kernel> <workload> <bytes per particle>')."""
    pdir = os.path.join(REPO, "profiles")
    if not os.path.isdir(pdir):
        return None
    for fn in sorted(os.listdir(pdir)):
        if not fn.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(pdir, fn)):
            m = re.match(r"\s*TRAFFIC\s+(\S+)\s+(\S+)\s+([0-9.eE+-]+)", line)
            if m and m.group(1) == kernel and m.group(2) == workload:
                return float(m.group(3))
    return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.p = None
        self.path = os.path.join("/tmp", "agimp_clocks_%d_%d.csv" % (os.getpid(), gpu))

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [t.strip() for t in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def refine_kernels(scene):
    """Kernels of one refinement: bounding box (2), occupancy (2), one
    distance-transform pass per axis, level assignment."""
    return 5 + scene.dim


def scene_config(scene, world=1):
    """The `config` object of a single-scene line: the workload and every
    interpretation of the configuration as a structured key (both arms print
    the same object)."""
    import numpy as np

    from agimp import scenes
    sk = scene.sim_kwargs
    k = int(scene.name[6]) if scene.name.startswith("config") and scene.name[6].isdigit() else None
    rho = scenes.RHO.get(k)
    d = scene.dim
    vel = np.unique(np.asarray(scene.v, np.float32), axis=0)
    mat = {"model": "fixed-corotated" + (" + snow plasticity" if sk.get("plasticity") == "snow" else ""),
           "E": sk["E"] * rho if rho else sk["E"], "rho": rho, "E_over_rho": sk["E"], "nu": sk["nu"]}
    if sk.get("plasticity") == "snow":
        mat.update(theta_c=sk.get("theta_c", 2.5e-2), theta_s=sk.get("theta_s", 7.5e-3),
                   hardening=sk.get("hardening", 10.0))
    return {
        "workload": scene.name, "particles": scene.n, "levels": scene.level,
        "coarsest": scene.coarsest, "finest": scene.coarsest << (scene.level - 1), "dt": scene.dt,
        "refine_every": scene.refine_every, "parallelism": "replicas" if world > 1 else "single",
        "material": mat,
        "gravity": list(sk.get("gravity", ())),
        "initial_velocity": vel.tolist() if len(vel) <= 4 else "per body",
        "colliders": [list(c) for c in sk.get("colliders", ())],
        "boundary": sk.get("boundary_mode", "ref_slip"),
        "invalid_nodes": sk.get("invalid_nodes", "raw"),
        "refinement": ({"rule": "free-surface depth (Chebyshev, finest cells)", "band": scene.refine_band,
                        "every": scene.refine_every} if scene.refine_every else "static level map"),
        "l2": "inputs exceed L2 (particle state %.0f MB)" % (scene.n * (4 * (2 * d + 2 * d * d + 2)) / 1e6),
        "seed": 0,
        "description": scene.description,
    }


def run_steps(sim, scene, first, count, stream=None):
    for i in range(first, first + count):
        if scene.refine_every and i % scene.refine_every == 0:
            sim.refine_levels(scene.refine_band, stream=stream)
        sim.substep(scene.dt, stream=stream)


def cpu_oracle_run(scene, seconds, threads, steps_cap=None, warmup=1):
    """Time the oracle (OpenMP, `threads` threads) on the full scene; returns
    (particle-substeps/s, substeps timed, seconds)."""
    import numpy as np

    import oracle as O
    from agimp.simulator import tabulate_level_map
    d, n = scene.dim, scene.n
    kw = {}
    sk = scene.sim_kwargs
    if "gravity" in sk:
        kw["gravity"] = tuple(sk["gravity"]) + (0.0,) * (3 - len(sk["gravity"]))
    for k in ("E", "nu", "theta_c", "theta_s", "hardening"):
        if k in sk:
            kw[k] = sk[k]
    kw["boundary_mode"] = {"ref_slip": 0, "sticky": 1}[sk.get("boundary_mode", "ref_slip")]
    kw["plasticity"] = {None: 0, "snow": 1}[sk.get("plasticity")]
    kw["colliders"] = tuple(sk.get("colliders", ()))
    kw["invalid_nodes"] = {"raw": 0, "normalize": 1}[sk.get("invalid_nodes", "raw")]
    o = O.Oracle(d, scene.level, scene.coarsest, n, **kw)
    o.set_particles(scene.x, scene.v, np.tile(np.eye(d), (n, 1, 1)), np.zeros((n, d, d)), scene.m, scene.g)
    if scene.grid_initializer is not None:
        t, H = tabulate_level_map(scene.grid_initializer, d, scene.level, scene.coarsest)
        o.set_level_map(t, H)

    def one(i):
        if scene.refine_every and i % scene.refine_every == 0:
            o.refine_levels(scene.refine_band)
        o.substep(scene.dt, 1, threads)

    for i in range(warmup):
        one(i)
    t0 = time.perf_counter()
    done = 0
    while True:
        one(warmup + done)
        done += 1
        el = time.perf_counter() - t0
        if (steps_cap and done >= steps_cap) or el >= seconds:
            break
    el = time.perf_counter() - t0
    return n * done / el, done, el


def cpu_parity_leg(a, scene, local, tuning):
    """The CPU baseline, and from the same oracle run the long-horizon parity
    of the GPU path.  The full scene runs from its initial state for
    --parity-substeps substeps (refinement included) on the GPU, on the f32
    oracle (OpenMP on all host threads; after one warm-up substep, the
    substeps finished within --cpu-seconds are the timed CPU sample) and on
    the f64 oracle; positions, velocities and per-level grid momentum are
    compared (oracle/parity.py).  Returns (cpu_baseline, parity or None)."""
    import parity as PY
    from agimp.simulator import tabulate_level_map
    threads = os.cpu_count() or 1
    steps = max(0, a.parity_substeps)
    lm = (tabulate_level_map(scene.grid_initializer, scene.dim, scene.level, scene.coarsest)
          if scene.grid_initializer is not None else None)
    par = None
    if steps:
        sim = scene.build(device=local)
        sim.set_tuning(tuning["chunk"], tuning["ctas_per_sm"])
        run_steps(sim, scene, 0, steps)
        gpu = {"x": sim.x_p.to_numpy(), "v": sim.v_p.to_numpy(), "g": sim.g_p.to_numpy()}
        errors = sim.errors()
        boxes = PY.grid_boxes(gpu["x"], scene.coarsest, scene.level)
        grids = [(sim.ad_grid_m[l].read(lo, n), sim.ad_grid_v[l].read(lo, n)) for l, (lo, n) in enumerate(boxes)]
        sim.close()
    o32 = PY.make_oracle(scene, False, lm)
    PY.step(o32, scene, 0, threads)  # warm-up
    if steps:
        t0 = time.perf_counter()
        done, el = PY.timed_run(o32, scene, 1, steps - 1, threads, a.cpu_seconds)
        total32 = time.perf_counter() - t0
    else:
        done, el = 0, 0.0
        t0 = time.perf_counter()
        while True:
            PY.step(o32, scene, 1 + done, threads)
            done += 1
            el = time.perf_counter() - t0
            if el >= a.cpu_seconds:
                break
    cpu = {"value": scene.n * done / el, "unit": METRIC, "cores": threads, "kind": "port",
           "sample": "%s: %d substeps of the full %d-particle scene after 1 warm-up, %.1f s, OpenMP%s"
                     % (scene.name, done, scene.n, el,
                        ", the first substeps of the parity run" if steps else "")}
    if steps:
        t1 = time.perf_counter()
        o64 = PY.make_oracle(scene, True, lm)
        PY.run(o64, scene, 0, steps, threads)
        par = PY.report(gpu, grids, o32, o64, scene.x, boxes, steps)
        par["gpu_device_errors"] = errors
        par["oracle_seconds"] = {"f32": round(total32, 1), "f64": round(time.perf_counter() - t1, 1)}
        par["grid_boxes"] = [[lo, n] for lo, n in boxes]
    return cpu, par


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from agimp import scenes
    threads = os.cpu_count() or 1
    budget = max(10.0, min(150.0, 2.0 * a.steps))
    if a.config == 4:
        sc = scenes.make_batch_config(scale=a.scale)
        val, done, el, ns = cpu_oracle_batch(sc, budget, threads)
        sample = "%d of the %d scenes one at a time, %d substeps each after 1 warm-up, %.1f s" % (ns, len(sc), done, el)
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": val, "unit": METRIC, "n_gpus": a.gpus, "steps": done,
            "warmup": 1, "ms_per_step": 1e3 * el / (done * ns), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "config4_batched_2d", "scenes": len(sc), "particles": sum(s.n for s in sc)},
            "cpu_baseline": {"value": val, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference is Taichi code and Taichi cannot be installed offline; this arm runs the CPU "
                    "restatement of its algorithm (oracle/oracle.cpp) with OpenMP on all host threads"}))
        return
    scene = scenes.make_config(a.config, scale=a.scale)
    warm = min(a.warmup, 10)
    val, done, el = cpu_oracle_run(scene, budget, threads, steps_cap=a.steps, warmup=warm)
    sample = "%s: %d substeps of the full %d-particle scene after %d warm-up, %.1f s" % (
        scene.name, done, scene.n, warm, el)
    out = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": METRIC, "n_gpus": a.gpus, "steps": done,
        "warmup": warm, "ms_per_step": 1e3 * el / done, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": scene_config(scene, a.gpus),
        "cpu_baseline": {"value": val, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference is Taichi code and Taichi cannot be installed offline; this arm runs the CPU "
                "restatement of its algorithm (oracle/oracle.cpp) with OpenMP on all host threads",
    }
    print(json.dumps(out))


def timed_steps(sim, scene, a, stream, dist=None, clocks=None):
    """Warm-up, then K timed substeps between CUDA events on `stream`; returns ms."""
    import contextlib

    import torch
    st = __import__("ctypes").c_void_p(stream.cuda_stream)
    run_steps(sim, scene, 0, a.warmup, st)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with (clocks or contextlib.nullcontext()):
        e0.record(stream)
        run_steps(sim, scene, a.warmup, a.steps, st)
        e1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    return e0.elapsed_time(e1)


def job_totals(dist, device, times_ms, units):
    """Whole-job figures over the ranks: each entry of `times_ms` is replaced
    by its maximum over the ranks (the slowest rank's time) and `units` by
    their sum (ranks may hold scenes of different sizes).  Without a process
    group (one rank) the inputs come back unchanged."""
    import torch
    t = torch.tensor(list(times_ms), dtype=torch.float64, device=device)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()], float(u.item())


def surrogate_report(a, scene, sim, ms, local, tuning):
    """Plain (SVD return map) run of the same scene for comparison: its
    throughput and the surrogate run's position error against it."""
    import numpy as np
    import torch
    st = sim.stats()
    plain = scene.build(device=local)
    plain.set_tuning(tuning["chunk"], tuning["ctas_per_sm"])
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        ms_plain = timed_steps(plain, scene, a, stream)
    xs, xp = sim.x_p.to_numpy(), plain.x_p.to_numpy()
    plain.close()
    d = np.abs(xs.astype(np.float64) - xp)
    return {"weights": os.path.relpath(a.surrogate, REPO) if os.path.isabs(a.surrogate) else a.surrogate,
            "tol": a.sur_tol, "ms_per_step": ms / a.steps, "plain_ms_per_step": ms_plain / a.steps,
            "plain_value": scene.n * a.steps / (ms_plain / 1e3), "speedup_vs_plain": ms_plain / ms,
            "substeps_compared": a.warmup + a.steps,
            "position_error_vs_plain": {"max": float(d.max()), "mean": float(d.mean()), "unit": "domain lengths"},
            "last_substep": {"handed_off": st["n_surrogate"], "rejected": st["n_fallback"]}}


def run_agimp(a):
    import numpy as np
    import torch

    from agimp import scenes
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    scene = scenes.make_config(a.config, seed=rank, scale=a.scale)
    sim = scene.build(device=local)
    import ctypes
    stream = torch.cuda.Stream()
    st = ctypes.c_void_p(stream.cuda_stream)
    if a.tuning:
        ch, cps = (int(v) for v in a.tuning.split(","))
        sim.set_tuning(ch, cps)
    elif not a.no_autotune:
        with torch.cuda.stream(stream):
            # tune on the level layout the run steps with: the schedule's
            # first refinement (substep 0) comes before the candidates run
            if scene.refine_every:
                sim.refine_levels(scene.refine_band, stream=st)
            sim.autotune(scene.dt, trials=10, stream=st)
    tuning = sim.tuning
    mlp = None
    if a.surrogate:
        from agimp.surrogate import load
        mlp, xmax = load(a.surrogate, device=local)
        sim.set_surrogate(mlp, xmax, a.sur_tol)
    with torch.cuda.stream(stream):
        clk = Clocks(local)
        ms = timed_steps(sim, scene, a, stream, dist, clk)
        errors = sim.errors()
        stats = sim.stats()
        # per-phase timing of single substeps (direct launches, CUDA events)
        prof = [sim.profile_substep(scene.dt, stream=st) for _ in range(5)]
    (ms_max,), units = job_totals(dist, "cuda", [ms], scene.n * a.steps)
    value = units / (ms_max / 1e3)
    phases = {k: statistics.median(p[k] for p in prof) for k in prof[0]}
    d = scene.dim
    jp = scene.sim_kwargs.get("plasticity") == "snow"
    b_p2g, b_g2p = BYTES[(d, jp)]
    nb = stats["n_binned"]
    hbm, src = peaks()
    dom = "p2g" if phases["p2g"] >= phases["g2p"] else "g2p"
    dom_bytes = nb * (b_p2g if dom == "p2g" else b_g2p)
    achieved = dom_bytes / (phases[dom] / 1e3) / 1e9
    tr = profile_traffic("k_" + dom, scene.name)
    roof = {"bound": "hbm", "kernel": "k_" + dom, "achieved": achieved, "peak": hbm, "peak_source": src,
            "unit": "GB/s", "frac": achieved / hbm, "traffic": (tr * nb) if tr is not None else None,
            "algorithmic_bytes": dom_bytes,
            "p2g_g2p_combined_frac": (nb * (b_p2g + b_g2p) / ((phases["p2g"] + phases["g2p"]) / 1e3) / 1e9) / hbm}
    n_refines = sum(1 for i in range(a.warmup, a.warmup + a.steps) if scene.refine_every and i % scene.refine_every == 0)
    launches = a.steps * sim.kernels_per_substep() + n_refines * refine_kernels(scene)
    out = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": scene_config(scene, world),
        "roofline": roof,
        "phases_ms": phases,
        "tuning": tuning,
        "gpu_launches": launches,
        "clocks": clk.summary(),
        "device_errors": errors,
    }
    if mlp is not None:
        # the per-phase profile above ran extra substeps: rebuild for the comparison
        sim.close()
        sim = scene.build(device=local)
        sim.set_tuning(tuning["chunk"], tuning["ctas_per_sm"])
        sim.set_surrogate(mlp, xmax, a.sur_tol)
        with torch.cuda.stream(stream):
            timed_steps(sim, scene, a, stream)
        out["surrogate"] = surrogate_report(a, scene, sim, ms, local, tuning)
    if not a.no_e2e:
        out["e2e"] = e2e_median(lambda: e2e_run(a, scene, local, a.surrogate and (mlp, xmax, a.sur_tol), tuning))
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        out["cpu_baseline"], par = cpu_parity_leg(a, scene, local, tuning)
        if par is not None:
            out["parity"] = par
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    sim.close()
    if rank == 0:
        print(json.dumps(out))


def run_batch(a):
    """Config 4: a batch of independent 2D scenes stepped by shared launches
    (one launch per kernel for all scenes, one CUDA graph per substep), with
    launch sizes from the autotuner; compared with the same scenes stepped one
    at a time (each with its own graph)."""
    import ctypes

    import numpy as np
    import torch

    from agimp import scenes
    from agimp.batch import SceneBatch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    sc = scenes.make_batch_config(seed=rank, scale=a.scale, material="snow" if a.snow else "elastic")
    dt = sc[0].dt
    n_tot = sum(s.n for s in sc)
    stream = torch.cuda.Stream()
    st = ctypes.c_void_p(stream.cuda_stream)
    sims = [s.build(device=local) for s in sc]
    batch = SceneBatch(sims)
    mlp = None
    if a.surrogate:
        from agimp.surrogate import load
        mlp, xmax = load(a.surrogate, device=local)
        batch.set_surrogate(mlp, xmax, a.sur_tol)
    if a.tuning:
        ch, cps = (int(v) for v in a.tuning.split(","))
        batch.set_tuning(ch, cps)
        tuning = batch.tuning
    else:
        tuning = batch.autotune(dt, trials=10, stream=st) if not a.no_autotune else batch.tuning

    def timed(step, clocks=None):
        import contextlib
        with torch.cuda.stream(stream):
            for _ in range(a.warmup):
                step()
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            with (clocks or contextlib.nullcontext()):
                e0.record(stream)
                for _ in range(a.steps):
                    step()
                e1.record(stream)
                torch.cuda.synchronize()
            if dist:
                dist.barrier()
            return e0.elapsed_time(e1)

    clk = Clocks(local)
    ms = timed(lambda: batch.substep(dt, 1, stream=st), clk)
    errors = [s.errors() for s in sims]
    with torch.cuda.stream(stream):
        prof = [batch.profile_substep(dt, stream=st) for _ in range(5)]
    nb = sum(s.stats()["n_binned"] for s in sims)
    # the same scenes one at a time, each through its own graph
    alone = [s.build(device=local) for s in sc]

    def one_at_a_time():
        for s in alone:
            s.substep(dt, stream=st)

    ms_alone = timed(one_at_a_time)
    ms_plain_batch = None
    if mlp is not None:
        plain = [s.build(device=local) for s in sc]
        pbatch = SceneBatch(plain)
        pbatch.set_tuning(tuning["chunk"], tuning["ctas_per_sm"])
        ms_plain_batch = timed(lambda: pbatch.substep(dt, 1, stream=st))
        pbatch.close()
        for s in plain:
            s.close()
    # both runs took warmup + steps substeps; the batch ran 5 more for its profile
    for s in alone:
        with torch.cuda.stream(stream):
            s.substep(dt, 5, stream=st)
    torch.cuda.synchronize()
    errs = []
    for s, b in zip(alone, sims):
        if s.n_particles:
            errs.append(float(np.abs(s.x_p.to_numpy().astype(np.float64) - b.x_p.to_numpy()).max()))
    for s in alone:
        s.close()
    (ms_max, ms_alone_max), units = job_totals(dist, "cuda", [ms, ms_alone], n_tot * a.steps)
    value = units / (ms_max / 1e3)
    phases = {k: statistics.median(p[k] for p in prof) for k in prof[0]}
    b_p2g, b_g2p = BYTES[(2, False)]
    hbm, src = peaks()
    dom = "p2g" if phases["p2g"] >= phases["g2p"] else "g2p"
    dom_bytes = nb * (b_p2g if dom == "p2g" else b_g2p)
    achieved = dom_bytes / (phases[dom] / 1e3) / 1e9
    tr = profile_traffic("k_" + dom, "config4_batched")
    roof = {"bound": "hbm", "kernel": "k_" + dom, "achieved": achieved, "peak": hbm, "peak_source": src,
            "unit": "GB/s", "frac": achieved / hbm, "traffic": (tr * nb) if tr is not None else None,
            "algorithmic_bytes": dom_bytes,
            "p2g_g2p_combined_frac": (nb * (b_p2g + b_g2p) / ((phases["p2g"] + phases["g2p"]) / 1e3) / 1e9) / hbm}
    levels = [s.level for s in sc]
    out = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "config4_batched_2d" + ("_snow" if a.snow else ""), "scenes": len(sc),
                   "particles": n_tot, "material": "snow (config 2)" if a.snow else "elastic (config 1)",
                   "levels": {str(k): levels.count(k) for k in sorted(set(levels))},
                   "particles_per_scene": [int(min(s.n for s in sc)), int(max(s.n for s in sc))],
                   "dt": dt, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs exceed L2 (particle state %.0f MB)" % (n_tot * 4 * 14 / 1e6),
                   "description": "256 independent 2D scenes, 2-4 levels, finest 256^2 or 512^2, 1-3 elastic "
                                  "boxes, lognormal 2k-60k particles, static level maps, one launch per kernel "
                                  "for all scenes under a CUDA graph"},
        "tuning": tuning,
        "one_at_a_time": {"value": units / (ms_alone_max / 1e3),
                          "ms_per_step": ms_alone_max / a.steps, "speedup_of_batch": ms_alone_max / ms_max,
                          "position_error_vs_batch": {"max_over_scenes": max(errs), "median": float(np.median(errs)),
                                                      "unit": "domain lengths"}},
        "roofline": roof,
        "phases_ms": phases,
        "gpu_launches": a.steps * batch.kernels_per_substep(),
        "clocks": clk.summary(),
        "device_errors": int(np.bitwise_or.reduce(errors)),
    }
    if mlp is not None:
        (ms_pb,), _ = job_totals(dist, "cuda", [ms_plain_batch], 0)
        out["surrogate"] = batch_surrogate_report(a, sc, local, tuning, mlp, xmax, ms_max, ms_pb, ms_alone_max,
                                                  rank == 0 and world == 1 and not a.no_cpu_baseline)
    if not a.no_e2e:
        out["e2e"] = e2e_median(lambda: e2e_batch(a, sc, local, tuning))
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        threads = os.cpu_count() or 1
        val, done, el, ns = cpu_oracle_batch(sc, a.cpu_seconds, threads)
        out["cpu_baseline"] = {"value": val, "unit": METRIC, "cores": threads, "kind": "port",
                               "sample": "%d of the %d scenes one at a time, %d substeps each, %.1f s, OpenMP"
                                         % (ns, len(sc), done, el)}
    batch.close()
    for s in sims:
        s.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


def batch_surrogate_report(a, sc, local, tuning, mlp, xmax, ms_sur, ms_plain_batch, ms_alone, cpu_leg):
    """The batched+surrogate form against the plain forms on the same scenes.
    Speed: device time of the timed substeps of the batch with the surrogate,
    of the plain batch (exact return map) and of the plain scenes stepped one
    at a time.  Accuracy: from the initial state, --accuracy-substeps
    substeps of the surrogate batch and of the plain batch; per scene the
    position error of the surrogate run against the plain run, relative to
    the plain run's RMS displacement.  In the CPU leg (rank 0, one GPU) the
    f64 oracle runs the three smallest snow scenes over the same substeps and
    both GPU runs are compared with it (the plain run's error is the floor)."""
    import numpy as np

    from agimp.batch import SceneBatch
    K = a.accuracy_substeps
    dt = sc[0].dt
    runs = {}
    for name, use in (("surrogate", True), ("plain", False)):
        sims = [s.build(device=local) for s in sc]
        b = SceneBatch(sims)
        b.set_tuning(tuning["chunk"], tuning["ctas_per_sm"])
        if use:
            b.set_surrogate(mlp, xmax, a.sur_tol)
        handed = rejected = 0
        for i in range(K):
            b.substep(dt, 1)
            if use and (i % 50 == 0 or i == K - 1):
                stt = b.surrogate_stats()
                handed += stt["handed_off"]
                rejected += stt["rejected"]
        runs[name] = ([s.x_p.to_numpy().astype(np.float64) for s in sims], handed, rejected,
                      int(np.bitwise_or.reduce([s.errors() for s in sims])))
        b.close()
        for s in sims:
            s.close()
    xs, xp = runs["surrogate"][0], runs["plain"][0]
    rel = []
    for s, u, p in zip(sc, xs, xp):
        if not s.n:
            continue
        disp = np.sqrt(((p - s.x) ** 2).sum(1).mean())
        rel.append(float(np.sqrt(((u - p) ** 2).sum(1).mean()) / disp) if disp > 0 else 0.0)
    rep = {
        "weights": os.path.relpath(a.surrogate, REPO) if os.path.isabs(a.surrogate) else a.surrogate,
        "tol": a.sur_tol,
        "ms_per_step": ms_sur / a.steps, "plain_batch_ms_per_step": ms_plain_batch / a.steps,
        "plain_one_at_a_time_ms_per_step": ms_alone / a.steps,
        "speedup_vs_plain_batch": ms_plain_batch / ms_sur, "speedup_vs_plain_one_at_a_time": ms_alone / ms_sur,
        "accuracy": {"substeps": K,
                     "position_rel_vs_plain": {"max_over_scenes": max(rel), "median": float(np.median(rel)),
                                               "mean": float(np.mean(rel))},
                     "sampled_handed_off": runs["surrogate"][1], "sampled_rejected": runs["surrogate"][2],
                     "device_errors": [runs["surrogate"][3], runs["plain"][3]]},
    }
    if cpu_leg:
        import parity as PY
        from agimp.simulator import tabulate_level_map
        threads = os.cpu_count() or 1
        idx = [i for i in np.argsort([s.n if s.n else 1 << 30 for s in sc])[:3] if sc[i].n]
        vs = []
        for i in idx:
            s = sc[i]
            o = PY.make_oracle(s, True, tabulate_level_map(s.grid_initializer, s.dim, s.level, s.coarsest))
            PY.run(o, s, 0, K, threads)
            x64 = o.particles()["x"]
            disp = np.sqrt(((x64 - s.x) ** 2).sum(1).mean())

            def err(x):
                return float(np.sqrt(((x - x64) ** 2).sum(1).mean()) / disp)
            vs.append({"scene": s.name, "particles": s.n, "surrogate_vs_f64": err(xs[i]), "plain_vs_f64": err(xp[i])})
        rep["accuracy"]["vs_f64_oracle"] = vs
    return rep


def cpu_oracle_batch(sc, seconds, threads, steps=3):
    """The oracle stepping scenes one at a time (as the reference would), over
    as many scenes as fit the time budget (setup and one warm-up substep per
    scene untimed); returns (particle-substeps/s, substeps per scene, timed
    seconds, scenes)."""
    import parity as PY
    from agimp.simulator import tabulate_level_map
    el, work, k = 0.0, 0, 0
    for s in sc:
        n = s.n
        o = PY.make_oracle(s, False, tabulate_level_map(s.grid_initializer, s.dim, s.level, s.coarsest))
        o.substep(s.dt, 1, threads)
        t1 = time.perf_counter()
        o.substep(s.dt, steps, threads)
        el += time.perf_counter() - t1
        work += n * steps
        k += 1
        if el >= seconds:
            break
    return work / el, steps, el, k


E2E_RUNS = 3


def e2e_median(run):
    """The end-to-end measurement repeated E2E_RUNS times (wall clock over the
    host's copies varies from run to run); the median run is reported, every
    run's value beside it."""
    runs = [run() for _ in range(E2E_RUNS)]
    vals = [r["value"] for r in runs]
    out = dict(sorted(runs, key=lambda r: r["value"])[len(runs) // 2])
    out["runs"] = vals
    return out


def e2e_batch(a, sc, local, tuning=None):
    """Same metric through the public API with host buffers: all scenes are
    uploaded from pinned host memory in one batch upload, then per substep the
    batch steps and all scenes' positions are read back into pinned host
    memory."""
    import numpy as np
    import torch

    from agimp.batch import SceneBatch
    sims = [s.build(device=local) for s in sc]
    batch = SceneBatch(sims)
    # every scene's initial state concatenated in batch order, in pinned host
    # memory: one upload call for the batch (agimp_batch_set_particles)
    n_tot = sum(s.n for s in sc)
    d = sc[0].dim
    h = {k: torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()
         for k, shape in (("x", (n_tot, d)), ("v", (n_tot, d)), ("F", (n_tot, d, d)), ("C", (n_tot, d, d)),
                          ("m", (n_tot,)))}
    h["g"] = torch.empty((n_tot,), dtype=torch.int32, pin_memory=True).numpy()
    h["x"][:] = np.concatenate([s.x for s in sc])
    h["v"][:] = np.concatenate([s.v for s in sc])
    h["F"][:] = np.eye(d, dtype=np.float32)
    h["C"][:] = 0
    h["m"][:] = np.concatenate([s.m for s in sc])
    h["g"][:] = np.concatenate([s.g for s in sc])
    if tuning:
        batch.set_tuning(tuning["chunk"], tuning["ctas_per_sm"])
    import ctypes
    main_s, copy_s = torch.cuda.Stream(), torch.cuda.Stream()
    sm, scp = ctypes.c_void_p(main_s.cuda_stream), ctypes.c_void_p(copy_s.cuda_stream)
    outs = [torch.empty((n_tot, 2), dtype=torch.float32, pin_memory=True).numpy() for _ in range(2)]
    done = [None, None]
    steps = max(a.steps, E2E_MIN_STEPS)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    batch.set_particles(x=h["x"], v=h["v"], F=h["F"], C=h["C"], m=h["m"], g=h["g"])
    for i in range(steps):
        batch.substep(sc[0].dt, stream=sm)
        # every scene's x_p in one gathered copy on a copy stream, overlapping
        # the next substep; double-buffered
        k = i % 2
        if done[k] is not None:
            done[k].synchronize()
        batch.positions(out=outs[k], blocking=False, stream=scp)
        done[k] = torch.cuda.Event()
        done[k].record(copy_s)
    for e in done:
        if e is not None:
            e.synchronize()
    el = time.perf_counter() - t0
    batch.close()
    for s in sims:
        s.close()
    h2d = sum(s.n * 4 * (2 * 2 + 2 * 4 + 2) for s in sc)
    return {"value": n_tot * steps / el, "unit": METRIC, "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": n_tot * 2 * 4, "substeps": steps,
            "timing": "wall clock; every substep's positions of all scenes read back to pinned host memory in one "
                      "asynchronous gathered copy overlapping the next substep, double-buffered, all landed before "
                      "the clock stops",
            "note": "h2d is the one-time upload of the scenes spread over the timed substeps"}


def e2e_run(a, scene, local, sur=None, tuning=None):
    """Same metric through the public API with host buffers: upload the scene
    from pinned host memory, then per substep call substep() and read x_p back
    into pinned host memory."""
    import numpy as np
    import torch
    n, d = scene.n, scene.dim

    def pinned(shape, dt=torch.float32):
        return torch.empty(shape, dtype=dt, pin_memory=True).numpy()

    hx, hv, hF, hC, hm, hg, hJ = (pinned((n, d)), pinned((n, d)), pinned((n, d, d)), pinned((n, d, d)), pinned((n,)),
                                  pinned((n,), torch.int32), pinned((n,)))
    hx[:] = scene.x
    hv[:] = scene.v
    hF[:] = np.eye(d, dtype=np.float32)
    hC[:] = 0
    hm[:] = scene.m
    hg[:] = scene.g
    hJ[:] = 1
    outs = [pinned((n, d)), pinned((n, d))]
    steps = max(a.steps, E2E_MIN_STEPS)
    sim = scene.build(device=local)
    if tuning:
        sim.set_tuning(tuning["chunk"], tuning["ctas_per_sm"])
    if sur:
        sim.set_surrogate(*sur)
    import ctypes
    main_s, copy_s = torch.cuda.Stream(), torch.cuda.Stream()
    sm, sc = ctypes.c_void_p(main_s.cuda_stream), ctypes.c_void_p(copy_s.cuda_stream)
    done = [None, None]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    sim.set_particles(x=hx, v=hv, F=hF, C=hC, m=hm, g=hg, Jp=hJ)
    for i in range(steps):
        if scene.refine_every and i % scene.refine_every == 0:
            sim.refine_levels(scene.refine_band, stream=sm)
        sim.substep(scene.dt, stream=sm)
        # x_p of this substep into one of two pinned buffers on a copy stream;
        # the next substep runs meanwhile.  The host takes a buffer back only
        # after its copy has landed.
        k = i % 2
        if done[k] is not None:
            done[k].synchronize()
        sim.x_p.to_numpy(out=outs[k], blocking=False, stream=sc)
        done[k] = torch.cuda.Event()
        done[k].record(copy_s)
    for e in done:
        if e is not None:
            e.synchronize()
    el = time.perf_counter() - t0
    sim.close()
    h2d = n * 4 * (2 * d + 2 * d * d + 3)
    return {"value": n * steps / el, "unit": METRIC, "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": n * d * 4, "substeps": steps,
            "timing": "wall clock; every substep's x_p read back to pinned host memory (asynchronous copy on a "
                      "second stream overlapping the next substep, double-buffered, all landed before the clock stops)",
            "note": "h2d is the one-time upload of the scene state spread over the timed substeps"}


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.config == 4:
        run_batch(a)
    else:
        run_agimp(a)


if __name__ == "__main__":
    main()
