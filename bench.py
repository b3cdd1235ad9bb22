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
        "--ncu-case",
        action="store_true",
        help="profiling case for ncu: build the scene at --h, run --steps substeps, print stats, exit",
    )
    return ap.parse_args()


def main_ncu_case(args):
    from slosh_b200 import scenes
    from slosh_b200.pipeline import MpmPipeline

    sc = bench_scene(args.h)
    data = scenes.build_mpm_data(sc)
    MpmPipeline().launch_step(data, args.steps)
    data.sync()
    print(json.dumps({"ncu_case": sc.name, "h": sc.cell_width, "particles": sc.n, **data.stats()}))
    data.close()
    return 0


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary
    (profiles/ncu_traffic.txt lines: `<kernel> <bytes_per_launch> ...`)."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2 and parts[0] == kernel and not line.startswith("#"):
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


def bench_scene(h: float):
    from slosh_b200 import scenes

    return scenes.sand_column_3d(h=h, substeps=500)


def workload_config(scene, extra=None):
    cfg = {
        "workload": f"sand_column_3d: Drucker-Prager sand cylinder r=0.15 h=0.5 at 8 ppc, dx={scene.cell_width:.6g}, "
        f"{scene.n} particles, rigid cuboid 0.1^3 + Separate floor, dt=2e-5",
        "particles": scene.n,
        "dim": 3,
        "material": "sand_linear (Drucker-Prager 30 deg, E=3.5e5, nu=0.3, rho=2200)",
        "l2": "inputs larger than L2 (about 0.7 GB of particle state resident per GPU)",
        "parallelism": "independent replica per GPU",
    }
    if extra:
        cfg.update(extra)
    return cfg


def cpu_sample_scene(h: float):
    """Bounded sample of the workload for the CPU runs: the bottom quarter of
    the sand column (same material, spacing and bodies)."""
    sc = bench_scene(h)
    y = sc.particles["position"][:, 1]
    keep = y < 0.05 + 0.125
    sc.particles = sc.particles[keep].copy()
    return sc


def run_cpu(h: float, steps: int, warmup: int, budget_s: float | None):
    from oracle import oracle as O

    sc = cpu_sample_scene(h)
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
    sample = f"bottom quarter of the sand column ({sc.n} particles, y < 0.175), {done} substeps after {warmup} warm-up"
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
    ms = ev0.elapsed_time(ev1)
    if pg is not None:
        t = torch.tensor([ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    value = world * n * args.steps / (ms / 1e3)
    launches = data.kernels_per_substep * args.steps

    # per-kernel device time (direct launches with events around each kernel)
    prof = data.profile_substeps(args.profile_steps, sptr)
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
        ems = e0.elapsed_time(e1)
        if pg is not None:
            t = torch.tensor([ems], device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {
            "value": world * n * args.e2e_substeps * args.e2e_steps / (ems / 1e3),
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
            "config": workload_config(sc, {"timed_substeps": args.steps}),
            "roofline": roof,
            "substep_roofline": substep_roof,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": ck,
            "kernel_ms_per_substep": per_substep,
            "active_blocks": nb,
        }
        print(json.dumps(line))
    data.close()
    if pg is not None:
        pg.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.ncu_case:
        return main_ncu_case(args)
    if args.impl == "reference":
        return main_reference(args)
    return main_ours(args)


if __name__ == "__main__":
    sys.exit(main())
