#!/usr/bin/env python
"""Benchmark of the MPM substep: particle-substeps/s on the 3D sand-column
workload (Drucker-Prager sand cylinder, 4.74 M particles at h = 1/256, a
rigid cuboid and a floor; slosh's launch_step semantics).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One process per GPU (torchrun for N > 1).  Every rank runs its own replica
of the scene (independent scenes, no collective on the data path; weak
scaling); the timed region is bracketed by a barrier and a device
synchronisation, timed with CUDA events on the launch stream, and the max
over ranks is reported.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "particle-substeps/s (4M 3D sand)"
UNIT = "particle-substeps/s"
# Algorithmic bytes per particle-substep of the whole substep (x, v, C, F
# read and written once in FP32, m/V0/material read, plastic state r/w, sort
# key and permutation, grid nodes): 3D sand = 254 B.
B_ALG_SAND = 254.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--h", type=float, default=1.0 / 256.0)
    ap.add_argument("--profile-steps", type=int, default=10)
    ap.add_argument("--e2e-substeps", type=int, default=500)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument(
        "--no-extras",
        action="store_true",
        help="default workload: skip the batched and served runs added to the N=1 line",
    )
    ap.add_argument("--batched-substeps", type=int, default=1000, help="batched run of the N=1 line: substeps")
    ap.add_argument(
        "--workload",
        choices=["sand", "dam_break_2d", "elastic_drop_3d", "batched", "served", "precision"],
        default="sand",
        help="sand: the 4.74 M-particle sand column (default); dam_break_2d, elastic_drop_3d: the other "
        "plain scenes; batched: 256 independent scenes in one batch vs the plain per-scene loop; served: "
        "Poisson request stream through the serving loop; precision: sand column vs the FP64 oracle",
    )
    ap.add_argument("--scenes", type=int, default=256, help="batched: number of scenes")
    ap.add_argument("--scene-max", type=int, default=256000, help="batched: largest scene (particles)")
    ap.add_argument("--requests", type=int, default=200, help="served: requests in the trace")
    ap.add_argument("--rate", type=float, default=20.0, help="served: mean arrivals per second")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="served: HBM budget")
    ap.add_argument("--tick", type=int, default=100, help="served: substeps per batched step at most")
    ap.add_argument("--no-plain", action="store_true", help="served: skip the one-in-flight baseline")
    ap.add_argument(
        "--ncu-case",
        action="store_true",
        help="profiling case for ncu: build the scene at --h (column radius --radius), or the --workload scene, run "
        "--steps substeps as direct launches, print stats, exit",
    )
    ap.add_argument("--radius", type=float, default=0.15, help="ncu case: radius of the sand column")
    return ap.parse_args()


def main_ncu_case(args):
    from slosh_b200 import scenes
    from slosh_b200.pipeline import MpmPipeline

    if args.workload == "batched":
        from slosh_b200.batch import MpmBatch

        scs = batched_scenes(args.scenes, max_particles=args.scene_max)
        total = int(sum(sc.n for sc in scs))
        b = MpmBatch(3, max_particles=total + 1024, grid_capacity=int(sum(max(64, 2.5 * sc.n / 512.0) for sc in scs)),
                     max_scenes=max(args.scenes, 1), max_bodies=4 * args.scenes + 16)
        for sc in scs:
            b.add(sc)
        b.set_tuning(5, 64, 8, 3)  # the shape the autotuner picks for this workload
        b.step(args.steps)
        b.sync()
        print(json.dumps({"ncu_case": "batched", "scenes": len(scs), "particles": total, **b.stats()}))
        b.close()
        return 0
    if args.workload == "dam_break_2d":
        sc = scenes.dam_break_2d()
    elif args.workload == "elastic_drop_3d":
        sc = scenes.elastic_drop_3d()
    else:
        sc = scenes.sand_column_3d(h=args.h, substeps=500, radius=args.radius)
    data = scenes.build_mpm_data(sc)
    # direct launches (the substep's kernels one by one, no graph): a
    # profiler does not see the kernels of graphs with conditional nodes
    data.profile_substeps(args.steps)
    data.sync()
    print(json.dumps({"ncu_case": sc.name, "h": sc.cell_width, "particles": sc.n, **data.stats()}))
    data.close()
    return 0


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(ms: float, pg, device=None) -> float:
    """The slowest rank's time: every rank passes its own timed region and
    gets the maximum (all ranks take this collective at the same point)."""
    if pg is None:
        return ms
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, units_per_rank: float, ms: float) -> float:
    """Whole-job throughput of replicas: units of all ranks over the slowest
    rank's time (weak scaling: every rank runs the full workload)."""
    return world * units_per_rank / (ms / 1e3)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel: str, workload: str | None = None):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary
    (profiles/ncu_traffic.txt lines: `<kernel> <bytes_per_launch> ...` for
    the sand column, `<workload>:<kernel> <bytes_per_launch> ...` for the
    other workloads)."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(p):
        return None
    name = f"{workload}:{kernel}" if workload else kernel
    with open(p) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2 and parts[0] == name and not line.startswith("#"):
                try:
                    return float(parts[1])
                except ValueError:
                    return None
    return None


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"),
                stderr=subprocess.DEVNULL,
            )
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                cols = [c.strip() for c in line.split(",")]
                if len(cols) < 9:
                    continue
                try:
                    sm.append(float(cols[1]))
                    smax.append(float(cols[2]))
                except ValueError:
                    continue
                for name, val in zip(names, cols[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(name)
        os.unlink(self.path)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def timed_launches(data, st0: dict, st1: dict, steps: int):
    """Kernels launched by `steps` substeps between two stats snapshots, and
    how many of them kept their grid: with conditional graphs a substep that
    keeps its grid launches 7 kernels fewer than one that rebuilds it."""
    reused = st1["n_grid_reuses"] - st0["n_grid_reuses"]
    rebuilt = st1["n_grid_rebuilds"] - st0["n_grid_rebuilds"]
    full = data.kernels_per_substep
    if st1["conditional_graphs"]:
        launches = full * rebuilt + (full - 7) * reused
    else:
        launches = data.kernels_per_substep * steps
    return launches, {"reused_substeps": reused, "rebuilt_substeps": rebuilt,
                      "conditional_graphs": bool(st1["conditional_graphs"])}


def bench_scene(h: float):
    from slosh_b200 import scenes

    return scenes.sand_column_3d(h=h, substeps=500)


L2_BYTES = 126 * 1024 * 1024
# particle storage a substep touches, per particle (3D): both copies of the
# 128-byte state, the original-index planes, sort key, permutation, cell slot
STORAGE_BYTES = 280


def l2_note(state_bytes: int) -> str:
    """How the timed substeps meet the L2 rule: no flush between substeps,
    so say whether the particle storage outgrows the 126 MB L2."""
    size = f"about {state_bytes / 1e9:.2g} GB of particle storage" if state_bytes >= 1e8 else \
        f"about {state_bytes / 1e6:.2g} MB of particle storage"
    if state_bytes > L2_BYTES:
        return f"inputs larger than L2 ({size})"
    return (f"inputs smaller than L2 ({size}): the configuration's whole state stays resident in L2 "
            "across substeps, as in any run of it; no flush")


def workload_config(scene, extra=None):
    cfg = {
        "workload": f"sand_column_3d: Drucker-Prager sand cylinder r=0.15 h=0.5 at 8 ppc, dx={scene.cell_width:.6g}, "
        f"{scene.n} particles, rigid cuboid 0.1^3 + Separate floor, dt=2e-5",
        "particles": scene.n,
        "dim": 3,
        "material": "sand_linear (Drucker-Prager 30 deg, E=3.5e5, nu=0.3, rho=2200)",
        "l2": l2_note(scene.n * STORAGE_BYTES),
        "parallelism": "independent replica per GPU",
    }
    if extra:
        cfg.update(extra)
    return cfg


def run_cpu(h: float, steps: int, warmup: int, budget_s: float | None):
    """The oracle (FP32, OpenMP on every host core) on the full sand column:
    `warmup` untimed substeps, then `steps` timed ones (or as many as fit in
    `budget_s` seconds, at least 2)."""
    from oracle import oracle as O

    sc = bench_scene(h)
    threads = os.cpu_count() or 1
    orc = O.from_scene(sc, threads=threads)
    if warmup:
        orc.step(warmup)
    done = 0
    t0 = time.perf_counter()
    while True:
        orc.step(1)
        done += 1
        el = time.perf_counter() - t0
        if budget_s is not None:
            if (el >= budget_s and done >= 2) or done >= steps:
                break
        elif done >= steps:
            break
    el = time.perf_counter() - t0
    orc.close()
    sample = f"the full sand column ({sc.n} particles), {done} substeps after {warmup} warm-up"
    return sc.n * done / el, threads, sample, el, done


def main_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    value, cores, sample, el, done = run_cpu(args.h, args.steps, args.warmup, None)
    sc_cfg = bench_scene(args.h)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": done,
        "warmup": args.warmup,
        "ms_per_step": el / done * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded lattice + jitter)",
        "config": workload_config(sc_cfg),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's own step runs only through wgpu (no CPU path, no graphics stack here); "
        "this arm times the oracle's C++ restatement of its shader math with OpenMP on the host cores",
    }
    print(json.dumps(line))
    return 0


def main_ours(args):
    import numpy as np
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
        pg = dist

    from slosh_b200 import scenes
    from slosh_b200._lib import PARTICLE_DTYPE
    from slosh_b200.pipeline import MpmPipeline

    sc = bench_scene(args.h)
    n = sc.n
    data = scenes.build_mpm_data(sc, device=local)
    stream = torch.cuda.Stream(device=dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    pipe = MpmPipeline()

    # warm-up (untimed)
    pipe.launch_step(data, max(args.warmup, 3), sptr)
    data.sync(sptr)

    # timed region: K substeps launched as CUDA graphs
    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize(dev)

    clocks = ClockSampler(local)
    st0 = data.stats()
    barrier()
    clocks.start()
    time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    pipe.launch_step(data, args.steps, sptr)
    ev1.record(stream)
    barrier()
    ck = clocks.stop()
    data.sync(sptr)
    ms = max_over_ranks(ev0.elapsed_time(ev1), pg, dev)
    value = aggregate_rate(world, n * args.steps, ms)
    st1 = data.stats()
    launches, grid_reuse = timed_launches(data, st0, st1, args.steps)
    svd_fp64 = st1["n_svd_fp64"] - st0["n_svd_fp64"]

    # per-kernel device time right after the timed region (direct launches
    # with events around each kernel; same scene state)
    prof = data.profile_substeps(args.profile_steps, sptr)

    # median of 5 timed regions of max(K, 100) substeps each (same stream,
    # same graphs), beside the single K-substep region above
    rep_k = max(args.steps, 100)
    reps = []
    st_r0 = data.stats()
    for _ in range(5):
        r0 = torch.cuda.Event(enable_timing=True)
        r1 = torch.cuda.Event(enable_timing=True)
        barrier()
        r0.record(stream)
        pipe.launch_step(data, rep_k, sptr)
        r1.record(stream)
        barrier()
        reps.append(max_over_ranks(r0.elapsed_time(r1), pg, dev))
    rep_ms = statistics.median(reps)
    repeat = {
        "substeps_per_region": rep_k,
        "regions": len(reps),
        "value": aggregate_rate(world, n * rep_k, rep_ms),
        "ms_per_step": rep_ms / rep_k,
        "ms_per_step_all": [r / rep_k for r in reps],
    }
    _, repeat["grid_reuse"] = timed_launches(data, st_r0, data.stats(), rep_k * len(reps))

    per_substep = {k: v / args.profile_steps for k, v in prof.items()}
    dom = max(per_substep, key=per_substep.get)
    peak, peak_kind = measured_peaks()
    stats = data.stats()
    nb = stats["n_blocks"]
    n_nodes = nb * 64
    alg_bytes = {
        # x+m, perm, V0, flags, F, plastic read; x, v, C, F, plastic written; node velocities read
        "k_g2p_update": n * (16 + 4 + 4 + 4 + 36 + 12 + 12 + 12 + 36 + 36 + 12) + n_nodes * 12,
        # perm, x+m, v, C read; node momentum/mass written
        "k_p2g": n * (4 + 16 + 12 + 36) + n_nodes * 16,
    }
    dom_bytes = alg_bytes.get(dom)
    roof = None
    if dom_bytes is not None:
        achieved = dom_bytes / (per_substep[dom] / 1e3) / 1e9
        roof = {
            "kernel": dom,
            "bound": "hbm",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": achieved / peak,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6650 GB/s",
            "algorithmic_bytes_per_launch": dom_bytes,
            "launch_ms": per_substep[dom],
            "traffic": ncu_traffic(dom),
        }
    substep_roof = {
        "bytes_per_particle_substep": B_ALG_SAND,
        "achieved_gbs": value / world * B_ALG_SAND / 1e9,
        "frac_of_peak": value / world * B_ALG_SAND / 1e9 / peak,
    }

    # end to end through the public API: upload from pinned host memory,
    # E substeps, positions read back, every e2e step.
    e2e = None
    if args.e2e_steps > 0:
        buf = torch.empty(n * PARTICLE_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
        host = buf.numpy().view(PARTICLE_DTYPE)
        host[:] = sc.particles
        outbuf = torch.empty(n * 16, dtype=torch.uint8, pin_memory=True)
        out = outbuf.numpy().view(np.float32).reshape(n, 4)
        # warm run of the e2e path
        data.upload(host, sptr)
        pipe.launch_step(data, 2, sptr)
        data.positions(out, sptr)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.e2e_steps):
            data.upload(host, sptr)
            pipe.launch_step(data, args.e2e_substeps, sptr)
            data.positions(out, sptr)
        e1.record(stream)
        barrier()
        ems = max_over_ranks(e0.elapsed_time(e1), pg, dev)
        e2e = {
            "value": aggregate_rate(world, n * args.e2e_substeps * args.e2e_steps, ems),
            "unit": UNIT,
            "h2d_bytes_per_step": int(n * PARTICLE_DTYPE.itemsize),
            "d2h_bytes_per_step": int(n * 16),
            "substeps_per_step": args.e2e_substeps,
            "steps": args.e2e_steps,
            "api": "slosh_upload_particles + slosh_step + slosh_download_positions (host buffers)",
        }

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, cores, sample, _, _ = run_cpu(args.h, 10**9, 1, args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded lattice + jitter; no dataset)",
            "config": workload_config(sc),
            "roofline": roof,
            "substep_roofline": substep_roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": ck,
            "kernel_ms_per_substep": per_substep,
            "active_blocks": nb,
            "repeat_median": repeat,
            "grid_reuse": grid_reuse,
            "svd_fp64_fallbacks_timed": svd_fp64,
        }
    data.close()
    if rank == 0:
        if world == 1 and not args.no_extras:
            # the batched and served configurations, measured in the same run
            drop = ("n_gpus", "higher_is_better", "scaling", "vs_baseline", "dtype", "data")
            for wl, k in (("dam_break_2d", 1000), ("elastic_drop_3d", 2000)):  # their whole runs
                line[wl] = {key: v for key, v in plain_line(args, wl, k, args.warmup, 5.0).items() if key not in drop}
            line["batched"] = {k: v for k, v in batched_line(args, args.batched_substeps, args.warmup).items() if k not in drop}
            # configuration 3's precision study: 500 substeps against the FP64 oracle
            line["precision"] = precision_line(args, 500, 1.0 / 64.0)
            line["served"] = {k: v for k, v in served_line(args).items() if k not in drop}
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()
    return 0


def batched_scenes(count: int, seed: int = 4, max_particles: int = 256000):
    """Scenes of the batched workload: particle counts log-uniform in
    [4k, max_particles] (256k for the configuration), material uniform over
    {fluid, fixed-corotated, Drucker-Prager sand}, cell width 1/64 or 1/128
    (seeded)."""
    import numpy as np

    from slosh_b200 import scenes

    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(4000.0), np.log(float(max(max_particles, 4000))), count))
    mats = rng.choice(["fluid", "elastic", "sand"], count)
    hs = rng.choice([1.0 / 64.0, 1.0 / 128.0], count)
    return [
        scenes.random_scene_3d(int(n), str(m), float(h), seed=seed * 1000 + i, substeps=1000)
        for i, (n, m, h) in enumerate(zip(ns, mats, hs))
    ]


def batched_line(args, steps: int, warmup: int) -> dict:
    """Config: 256 independent 3D scenes advanced by one batch (per substep
    one graph launch of 13 kernels over all scenes, or one persistent
    cooperative kernel, whichever the autotuner picks) against the plain loop
    of per-scene contexts (one graph launch of 13 kernels per scene and
    substep), same scenes, same substeps, same stream."""
    import numpy as np
    import torch

    from slosh_b200 import scenes as S
    from slosh_b200.batch import MpmBatch
    from slosh_b200.pipeline import MpmPipeline

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    scs = batched_scenes(args.scenes, max_particles=args.scene_max)
    total = int(sum(sc.n for sc in scs))
    stream = torch.cuda.Stream(device=dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    # active blocks with their neighbour-only blocks: about 2.5 per 512
    # particles, and at least 256 a scene (a small blob's shell of neighbour
    # blocks outweighs its interior)
    blocks_est = int(sum(max(256, 2.5 * sc.n / 512.0) for sc in scs))
    b = MpmBatch(
        3,
        max_particles=total + 1024,
        grid_capacity=blocks_est,
        max_scenes=max(args.scenes, 1),
        max_bodies=4 * args.scenes + 16,
        device=local,
    )
    slots = [b.add(sc) for sc in scs]
    tuning = b.autotune(2, sptr)
    b.step(max(warmup, 3), sptr)
    b.sync(sptr)
    clocks = ClockSampler(local)
    torch.cuda.synchronize(dev)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.step(steps, sptr)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ck = clocks.stop()
    b.sync(sptr)
    ms = e0.elapsed_time(e1)
    value = total * steps / (ms / 1e3)
    st = b.stats()

    # both substep forms on the same scenes: the 13-kernel graph (the shape
    # the autotuner picks for it) and the one persistent cooperative kernel
    forms = {}
    n_form = min(steps, 200)
    for name, shape in (("graph_13_kernels", (5, 64, 8, 3, 0)), ("fused_cooperative", (5, 64, 8, 3, 1))):
        b.set_tuning(*shape)
        b.step(3, sptr)
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        b.step(n_form, sptr)
        f1.record(stream)
        torch.cuda.synchronize(dev)
        fms = f0.elapsed_time(f1) / n_form
        forms[name] = {"ms_per_step": fms, "value": total / (fms / 1e3), "substeps": n_form}
        if shape[4]:
            forms[name]["inside_graph"] = bool(b.stats()["fused_graph"])
    b.set_tuning(tuning["p2g_ctas_per_sm"], tuning["g2p_threads"], tuning["g2p_ctas_per_sm"], tuning["p2g_stages"],
                 tuning["fused"])
    b.sync(sptr)

    # end to end through the public API: every scene uploaded from host
    # records in pinned memory, K substeps, every scene's positions read back
    # into pinned memory.
    from slosh_b200._lib import PARTICLE_DTYPE

    rec_buf = torch.empty(total * PARTICLE_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
    out_buf = torch.empty(total * 16, dtype=torch.uint8, pin_memory=True)
    recs = rec_buf.numpy().view(PARTICLE_DTYPE)
    pos = out_buf.numpy().view(np.float32).reshape(total, 4)
    host, outs, at = [], [], 0
    for sc in scs:
        recs[at : at + sc.n] = sc.particles
        host.append(recs[at : at + sc.n])
        outs.append(pos[at : at + sc.n])
        at += sc.n
    for sl in slots:
        b.remove_scene(sl)
    b.step(1, sptr)
    t0 = time.perf_counter()
    slots = [b.add_scene(h, sc.cell_width, sc.params, sc.bodies, sptr) for h, sc in zip(host, scs)]
    b.step(steps, sptr)
    for sl, o in zip(slots, outs):
        b.positions(sl, o, sptr)
    e2e_s = time.perf_counter() - t0
    b.close()

    # plain loop: one context per scene, each stepped through its own graph
    pipe = MpmPipeline()
    datas = [S.build_mpm_data(sc, device=local) for sc in scs]
    for d in datas:
        pipe.launch_step(d, max(warmup, 3), sptr)
    torch.cuda.synchronize(dev)
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for d in datas:
        pipe.launch_step(d, steps, sptr)
    p1.record(stream)
    torch.cuda.synchronize(dev)
    pms = p0.elapsed_time(p1)
    plain = total * steps / (pms / 1e3)
    for d in datas:
        d.close()

    mats = {}
    for sc in scs:
        k = sc.name.split("_")[1]
        mats[k] = mats.get(k, 0) + 1
    line = {
        "metric": f"particle-substeps/s (batched {args.scenes} scenes)",
        "value": value,
        "unit": UNIT,
        "n_gpus": 1,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": ms / steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded box blobs; no dataset)",
        "config": {
            "workload": f"batched: {len(scs)} independent 3D scenes, particles log-uniform [4k, {args.scene_max // 1000}k] "
            f"(total {total}), materials {mats}, dx 1/64 or 1/128, Separate floor each; one batch launch per substep "
            f"({'fused cooperative kernel' if tuning['fused'] else 'graph of 13 kernels'}, autotuned)",
            "scenes": len(scs),
            "particles": total,
            "tuning": tuning,
            "active_blocks": st["n_blocks"],
            "l2": l2_note(total * STORAGE_BYTES),
        },
        "plain_loop": {
            "value": plain,
            "ms_per_step": pms / steps,
            "desc": "one single-scene context per scene, each substep a graph launch per scene",
        },
        "speedup_vs_plain": value / plain,
        "substep_forms": forms,
        "e2e": {
            "value": total * steps / e2e_s,
            "unit": UNIT,
            "h2d_bytes_per_step": int(total * 192),
            "d2h_bytes_per_step": int(total * 16),
            "api": "slosh_batch_add_scene x scenes + slosh_batch_step + slosh_batch_download_positions x scenes "
            "(host buffers, wall clock)",
        },
        "gpu_launches": (1 if tuning["fused"] else 12 + st["g2p_launches"]) * steps,
        "clocks": ck,
    }
    return line


def main_batched(args):
    print(json.dumps(batched_line(args, args.steps, args.warmup)))
    return 0


def served_trace(count: int, seed: int = 5):
    """Requests of the served workload: unit-rate exponential gaps (scaled
    by 1 / rate), particle counts log-uniform in [8k, 2M], substeps uniform
    in [200, 2000], materials and cell widths as in the batched workload."""
    import numpy as np

    from slosh_b200 import scenes

    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0, count)
    ns = np.exp(rng.uniform(np.log(8000.0), np.log(2.0e6), count))
    subs = rng.integers(200, 2001, count)
    mats = rng.choice(["fluid", "elastic", "sand"], count)
    hs = rng.choice([1.0 / 64.0, 1.0 / 128.0], count)
    reqs = [
        (scenes.random_scene_3d(int(n), str(m), float(h), seed=seed * 1000 + i), int(s))
        for i, (n, m, h, s) in enumerate(zip(ns, mats, hs, subs))
    ]
    arrivals = np.cumsum(gaps) - gaps[0]
    return reqs, arrivals


def run_trace(srv, reqs, arrivals, rate: float):
    """Feeds the requests at arrivals / rate seconds (a feeder thread) and
    collects every completion.  Latency = completion - submission (queueing
    included), on the server's clock."""
    import threading

    import numpy as np

    t0 = time.perf_counter()

    def feeder():
        for (sc, sub), a in zip(reqs, arrivals):
            delay = t0 + a / rate - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            srv.submit(sc.particles, sc.cell_width, sc.params, sc.bodies, sub)

    th = threading.Thread(target=feeder)
    th.start()
    done = []
    while len(done) < len(reqs):
        done += srv.poll()
        time.sleep(0.002)
    th.join()
    lat = np.array([d["done_s"] - d["submit_s"] for d in done])
    work = float(sum(d["n"] * d["substeps"] for d in done))
    span = max(d["done_s"] for d in done) - min(d["submit_s"] for d in done)
    st = srv.stats()
    return {
        "rate_req_s": rate,
        "requests": len(done),
        "failed": int(sum(d["status"] != 0 for d in done)),
        "p50_s": float(np.percentile(lat, 50)),
        "p99_s": float(np.percentile(lat, 99)),
        "mean_s": float(lat.mean()),
        "throughput": work / span,
        "span_s": span,
        "gpu_busy_frac": st["busy_s"] / max(st["now_s"], 1e-9),
        "max_in_flight": st["max_in_flight_seen"],
        "tuning": st["tuning"],
    }


def served_line(args) -> dict:
    """Config: Poisson stream (mean 20 requests/s, seeded) of 3D scenes with
    8k-2M particles and 200-2000 substeps through the serving loop (HBM
    budget 150 GB, continuous batching); then the same trace at 0.7 of the
    measured capacity; then the plain loop (one request in flight at a time)
    on the 20 requests/s trace."""
    import numpy as np
    import torch

    from slosh_b200.serving import MpmServer

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    count = args.requests
    reqs, arrivals = served_trace(count)
    mean_work = float(np.mean([sc.n * s for sc, s in reqs]))
    budget = int(args.budget_gb * 1e9)
    clocks = ClockSampler(local)

    def server(max_in_flight=0):
        srv = MpmServer(budget, max_scenes=1024, tick_substeps=args.tick, max_in_flight=max_in_flight, device=local)
        # warm-up request (graphs, launch-shape autotuning); not part of the trace
        sc, _ = reqs[0]
        srv.submit(sc.particles, sc.cell_width, sc.params, sc.bodies, 24)
        srv.wait_idle(600)
        srv.poll()
        return srv

    srv = server()
    clocks.start()
    full = run_trace(srv, reqs, arrivals, args.rate)
    ck = clocks.stop()
    pool_gb = srv.stats()["pool_bytes"] / 1e9
    srv.close()
    cap_req_s = full["throughput"] / mean_work
    srv = server()
    steady = run_trace(srv, reqs, arrivals, 0.7 * cap_req_s)
    srv.close()
    plain = None
    if not args.no_plain:
        srv = server(max_in_flight=1)
        plain = run_trace(srv, reqs, arrivals, args.rate)
        srv.close()
    mean_n = float(np.mean([sc.n for sc, _ in reqs]))
    line = {
        "metric": "served particle-substeps/s (Poisson 20 req/s)",
        "value": full["throughput"],
        "unit": UNIT,
        "n_gpus": 1,
        "steps": count,
        "warmup": 1,
        "ms_per_step": full["span_s"] * 1e3 / count,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded box blobs, seeded Poisson arrivals; no dataset)",
        "config": {
            "workload": f"served: {count} requests, Poisson {args.rate} req/s, particles log-uniform [8k, 2M], "
            f"substeps uniform [200, 2000], fluid/elastic/sand, dx 1/64 or 1/128; HBM budget {args.budget_gb} GB "
            f"(batch pool {pool_gb:.1f} GB), tick {args.tick} substeps",
            "mean_request_particles": mean_n,
            "mean_request_work": mean_work,
            "offered_load": args.rate * mean_work,
        },
        "latency_s": {"p50": full["p50_s"], "p99": full["p99_s"], "mean": full["mean_s"]},
        "run_offered_load": full,
        "run_0p7_capacity": steady,
        "plain_one_in_flight": plain,
        "speedup_vs_plain": (full["throughput"] / plain["throughput"]) if plain else None,
        "e2e": {
            "value": full["throughput"],
            "unit": UNIT,
            "h2d_bytes_per_step": int(mean_n * 192),
            "d2h_bytes_per_step": int(mean_n * 16),
            "api": "slosh_server_submit (host records) to completion with positions in host memory; a step is a request",
        },
        "gpu_launches": None,
        "clocks": ck,
    }
    return line


def main_served(args):
    print(json.dumps(served_line(args)))
    return 0


def plain_alg_bytes(dim: int, sand: bool, n: int, n_nodes: int) -> dict:
    """Algorithmic bytes per launch of the two transfer kernels."""
    d2 = dim * dim
    pl = 12 if sand else 0
    return {
        # x+m, perm, V0, flags, F, plastic read; x, v, C, F, plastic written; node velocities read
        "k_g2p_update": n * (16 + 4 + 4 + 4 + 4 * d2 + pl + 4 * dim + 4 * dim + 4 * d2 + 4 * d2 + pl)
        + n_nodes * 4 * dim,
        # perm, x+m, v, C read; node partial tiles written
        "k_p2g": n * (4 + 16 + 4 * dim + 4 * d2) + n_nodes * 16,
    }


def plain_line(args, workload: str, steps: int, warmup: int, cpu_seconds: float) -> dict:
    """The other plain single-scene configurations: the 2D dam break
    (62.6 k particles, Tait fluid) and the 3D elastic drop (524 k particles,
    two fixed-corotated cubes), timed like the sand column."""
    import numpy as np
    import torch

    from oracle import oracle as O
    from slosh_b200 import scenes
    from slosh_b200._lib import PARTICLE_DTYPE
    from slosh_b200.pipeline import MpmPipeline

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if workload == "dam_break_2d":
        sc = scenes.dam_break_2d()
        desc = "dam_break_2d: Tait fluid column 0.4x0.6 at 2x2 ppc, dx=1/256, stick walls, dt=1e-4"
        b_alg, sand = 129.0, False
    else:
        sc = scenes.elastic_drop_3d()
        desc = "elastic_drop_3d: two fixed-corotated cubes (E=1e5, nu=0.3) at 8 ppc, dx=1/128, slip floor, dt=5e-5"
        b_alg, sand = 230.0, False
    n = sc.n
    data = scenes.build_mpm_data(sc, device=local)
    stream = torch.cuda.Stream(device=dev)
    sptr = ctypes.c_void_p(stream.cuda_stream)
    pipe = MpmPipeline()
    pipe.launch_step(data, max(warmup, 3), sptr)
    data.sync(sptr)
    clocks = ClockSampler(local)
    st0 = data.stats()
    torch.cuda.synchronize(dev)
    clocks.start()
    time.sleep(0.3)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    pipe.launch_step(data, steps, sptr)
    ev1.record(stream)
    torch.cuda.synchronize(dev)
    ck = clocks.stop()
    data.sync(sptr)
    ms = ev0.elapsed_time(ev1)
    value = n * steps / (ms / 1e3)
    launches, grid_reuse = timed_launches(data, st0, data.stats(), steps)
    prof = data.profile_substeps(args.profile_steps, sptr)
    per_substep = {k: v / args.profile_steps for k, v in prof.items()}
    # the roofline of the larger transfer kernel (a small scene's other
    # kernels are launch-bound and move O(blocks) bytes)
    dom = max(("k_g2p_update", "k_p2g"), key=lambda k: per_substep.get(k, 0.0))
    peak, peak_kind = measured_peaks()
    nb = data.stats()["n_blocks"]
    ab = plain_alg_bytes(sc.dim, sand, n, nb * 64).get(dom)
    roof = None
    if ab is not None:
        achieved = ab / (per_substep[dom] / 1e3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind, "algorithmic_bytes_per_launch": ab,
                "launch_ms": per_substep[dom], "traffic": ncu_traffic(dom, workload)}
    # e2e: upload + K substeps + positions through the public API
    buf = torch.empty(n * PARTICLE_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
    host = buf.numpy().view(PARTICLE_DTYPE)
    host[:] = sc.particles
    outbuf = torch.empty(n * 16, dtype=torch.uint8, pin_memory=True)
    out = outbuf.numpy().view(np.float32).reshape(n, 4)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    data.upload(host, sptr)
    pipe.launch_step(data, steps, sptr)
    data.positions(out, sptr)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    e2e = n * steps / (e0.elapsed_time(e1) / 1e3)
    data.close()
    cpu = None
    if cpu_seconds > 0:
        orc = O.from_scene(sc, threads=os.cpu_count() or 1)
        orc.step(1)
        done, t0 = 0, time.perf_counter()
        while done < 2 or (time.perf_counter() - t0 < cpu_seconds and done < sc.substeps):
            orc.step(1)
            done += 1
        el = time.perf_counter() - t0
        orc.close()
        cpu = {"value": n * done / el, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": f"full scene, {done} substeps after 1 warm-up"}
    line = {
        "metric": f"particle-substeps/s ({workload})",
        "value": value,
        "unit": UNIT,
        "n_gpus": 1,
        "steps": steps,
        "warmup": warmup,
        "ms_per_step": ms / steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded lattice + jitter; no dataset)",
        "config": {"workload": desc, "particles": n, "dim": sc.dim, "active_blocks": nb, "l2": l2_note(n * STORAGE_BYTES)},
        "roofline": roof,
        "substep_roofline": {"bytes_per_particle_substep": b_alg, "achieved_gbs": value * b_alg / 1e9,
                             "frac_of_peak": value * b_alg / 1e9 / peak},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": n * 192, "d2h_bytes_per_step": n * 16},
        "gpu_launches": launches,
        "grid_reuse": grid_reuse,
        "clocks": ck,
        "kernel_ms_per_substep": per_substep,
    }
    return line


def main_plain(args):
    print(json.dumps(plain_line(args, args.workload, args.steps, args.warmup,
                                0.0 if args.no_cpu_baseline else args.cpu_seconds)))
    return 0


def precision_line(args, steps: int, h: float) -> dict:
    """Precision study of the sand column: the FP32 GPU substep and the FP32
    oracle against the FP64 oracle after `steps` substeps, on the column at
    dx = h (the FP64 oracle cannot run the 4.74 M-particle column for 500
    substeps in minutes; the material, geometry, bodies and dt are those of
    the full configuration)."""
    import numpy as np
    import torch

    from oracle import oracle as O
    from slosh_b200 import scenes
    from slosh_b200.pipeline import MpmPipeline

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    sc = scenes.sand_column_3d(h=h, substeps=steps)
    data = scenes.build_mpm_data(sc, device=local)
    MpmPipeline().launch_step(data, steps)
    g = data.download_particles()
    fp64_fallbacks = data.stats()["n_svd_fp64"]
    data.close()
    threads = os.cpu_count() or 1
    o32 = O.from_scene(sc, threads=threads)
    o64 = O.from_scene(sc, double=True, threads=threads)
    t0 = time.perf_counter()
    o32.step(steps)
    o64.step(steps)
    cpu_s = time.perf_counter() - t0
    r32, r64 = o32.get_particles(), o64.get_particles()
    o32.close()
    o64.close()

    def err(a, b, k, cols=None):
        x = np.asarray(a[k], np.float64)
        y = np.asarray(b[k], np.float64)
        if cols is not None:
            x, y = x[:, cols], y[:, cols]
        d = np.abs(x - y)
        return {"max": float(d.max()), "rms": float(np.sqrt((d**2).mean())), "scale": float(np.abs(y).max())}

    res = {}
    for name, a in (("gpu_fp32", g), ("oracle_fp32", r32)):
        res[name] = {
            "position": err(a, r64, "position"),
            "velocity": err(a, r64, "velocity"),
            "def_grad": err(a, r64, "def_grad"),
            "plastic_q": err(a, r64, "model", [1]),
        }
    line = {
        "metric": "error vs FP64 oracle (sand column)",
        "workload": f"sand_column_3d at dx={sc.cell_width:.6g}: {sc.n} particles, {steps} substeps, dt=2e-5",
        "particles": sc.n,
        "substeps": steps,
        "cell_width": sc.cell_width,
        "errors": res,
        "position_max_err_in_cells": res["gpu_fp32"]["position"]["max"] / sc.cell_width,
        "gpu_svd_fp64_fallbacks": fp64_fallbacks,
        "oracle_cpu_seconds": cpu_s,
        "oracle_threads": threads,
    }
    return line


def main_precision(args):
    print(json.dumps(precision_line(args, args.steps, args.h if args.h > 1.0 / 100 else 1.0 / 64)))
    return 0


def main():
    args = parse()
    if args.ncu_case:
        return main_ncu_case(args)
    if args.workload in ("dam_break_2d", "elastic_drop_3d"):
        return main_plain(args)
    if args.workload == "precision":
        return main_precision(args)
    if args.workload == "batched":
        return main_batched(args)
    if args.workload == "served":
        return main_served(args)
    if args.impl == "reference":
        return main_reference(args)
    return main_ours(args)


if __name__ == "__main__":
    sys.exit(main())
