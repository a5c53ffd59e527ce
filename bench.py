"""Benchmark of the coupled RK4 phase-field step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload magnetoelastic|fm_demag|ferroelectric]

Workload (default): the coupled magnetoelastic + elastodynamics + Maxwell FDTD
run on a 128x128x96 grid (56-layer garnet substrate, 32-layer YIG film,
8 vacuum layers), FP64, synthetic seeded initial state.  One step = one full
RK4 step of all active physics.  The metric is cell-steps/s (grid cells x
steps / device time), whole job over all ranks.

`--impl ours` times the engine (CUDA events on the engine stream, max over
ranks), measures the end-to-end rate through the C ABI with host buffers,
reports the dominant kernel's roofline from per-launch events and, on rank 0,
the CPU reference (GO-Ferro's own solver, serial) on a bounded sample.
`--impl reference` times GO-Ferro's own solver (oracle/_ref, built from the
reference sources) on the host; it is serial (OpenACC pragmas are ignored on
the host), so it uses one core.
With N > 1 each rank runs an independent replica of the workload on its own
GPU (the grid is not decomposed; there is no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "magnetoelastic": dict(preset="magnetoelastic", kw=dict(nx=128, ny=128, nz=96, sub=56, film=32),
                           sample_kw=dict(nx=32, ny=32, nz=96, sub=56, film=32),
                           desc="coupled magnetoelastic + elastodynamics + FDTD, 128x128x96, dx=2nm"),
    "fm_demag": dict(preset="fm_demag", kw=dict(nx=64, ny=64, nz=16),
                     sample_kw=dict(nx=64, ny=64, nz=16),
                     desc="FM LLG + FFT magnetostatics, 64x64x16, dx=2nm"),
    "ferroelectric": dict(preset="ferroelectric", kw=dict(nx=128, ny=128, nz=128),
                          sample_kw=dict(nx=32, ny=32, nz=128),
                          desc="FE TDGL + electrostriction + elastodynamics + FDTD, 128^3, dx=1nm"),
}

# Algorithmic bytes per unit (cell, or edge/face for the Yee kernels) of one
# launch, averaged over the four RK stages: every array the kernel must read
# or write, once (stage-dependent terms weighted 3/4 where they occur in 3 of
# the 4 stages); neighbour re-reads are not counted.
def alg_bytes_per_unit(kernel: str, info, mfe_frac: float = 0.0) -> float:
    """Bytes one unit (cell, Yee vertex) of a launch must move, averaged over
    the four RK stages (stage outputs are written at stages 1-3, the
    accumulators read at stages 2-4, the step value read at stages 1-3).
    mfe_frac: fraction of cells that are ferromagnetic or ferroelectric."""
    D = 8.0
    if kernel == "k_elastic":
        # tiled stress-divergence kernel: u_in, m and p for the eigenstrain,
        # material ids; writes the divergence and the crystal-frame strain of
        # magnetic/ferroelectric cells
        reads = 3 + 3 * info.fm + 3 * info.fe
        writes = 3 + 6 * mfe_frac
        return (reads + writes) * D + 1
    if kernel == "k_elastic_rk":
        # divergence, force_store, v_x, v_in, u_x (stages 1-3), v/u accumulators
        # (stages 2-4); writes v/u stage outputs, accumulators, force_store (stage 1)
        reads = 3 + 3 + 3 + 3 + 3 * 0.75 + 6 * 0.75
        writes = 6 * 0.75 + 6 + 3 * 0.25
        return (reads + writes) * D + 1
    if kernel == "k_llg_fm":
        reads = 3 + 3 + 3 * 0.75 + 3 + 6 * info.elastic + 3 * info.em
        writes = 3 * 0.75 + 3 + 3 * info.em
        return (reads + writes) * D + 1
    if kernel == "k_fe":
        reads = 3 + 3 + 3 * 0.75 + 3 + 3 + 3 * 0.75 + 6 + 6 + 3 + 3 * info.em
        writes = 3 * 0.75 * 2 + 3 * 2
        return (reads + writes) * D + 1
    if kernel == "k_em_fused":
        # per Yee vertex: three E edges and three H faces, each with stage input,
        # step value, accumulator read/write and stage output; dM/dt and dP/dt
        per_comp = 1 + 0.75 + 0.75 + 0.75 + 1
        return (6 * per_comp + 3 * info.fm + 3 * info.fe) * D + 1
    return float("nan")


def units_per_launch(kernel: str, info) -> int:
    nx, ny, nz = info.nx, info.ny, info.nz
    edges = {"x": nx * (ny + 1) * (nz + 1), "y": (nx + 1) * ny * (nz + 1), "z": (nx + 1) * (ny + 1) * nz}
    faces = {"x": (nx + 1) * ny * nz, "y": nx * (ny + 1) * nz, "z": nx * ny * (nz + 1)}
    if kernel.startswith("k_em_E_"):
        return edges[kernel[-1]]
    if kernel.startswith("k_em_H_"):
        return faces[kernel[-1]]
    return nx * ny * nz


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(kernel: str, workload: str):
    """dram read+write bytes per launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get("dram_bytes_per_launch_full_size")


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu),
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
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
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def build_deck(gf, wl: str, sample: bool):
    spec = WORKLOADS[wl]
    kw = dict(spec["sample_kw"] if sample else spec["kw"])
    d = gf.decks.PRESETS[spec["preset"]](**kw)
    return d


def cpu_reference(gf, wl: str, steps: int, tmp: str, warmup: int = 0):
    """GO-Ferro's own solver on the bounded CPU sample: `warmup` untimed steps,
    then `steps` timed ones; returns (cell-steps/s, info)."""
    from oracle import refrun
    if not refrun.available():
        return None, "oracle binary not built"
    d = build_deck(gf, wl, sample=True)
    d.steps = steps + warmup
    ddir = os.path.join(tmp, "ref_deck")
    gf.decks.write_deck(d, ddir)
    r = refrun.run(ddir, os.path.join(tmp, "ref_out"), steps=steps + warmup, trace_every=max(steps + warmup, 1),
                   warmup=warmup)
    t = r["timing"]
    value = d.n * steps / t["seconds"]
    sample = f"{d.nx}x{d.ny}x{d.nz} sub-grid of the workload's layer stack, {steps} steps, serial reference build"
    return value, {"seconds": t["seconds"], "sample": sample, "cells": d.n}


def run_reference_arm(args, rank, world):
    import __graft_entry__
    gf = __graft_entry__.import_package()
    if rank != 0:
        return
    spec = WORKLOADS[args.workload]
    with tempfile.TemporaryDirectory() as tmp:
        steps = max(1, min(args.steps, args.ref_steps))
        warm = min(args.warmup, 3)
        value, info = cpu_reference(gf, args.workload, steps, tmp, warm)
    if value is None:
        print(json.dumps({"impl": "reference", "unavailable": info}))
        return
    line = {
        "impl": "reference", "metric": "cell-steps/s FP64", "value": value, "unit": "cell-steps/s",
        "n_gpus": world, "steps": steps, "warmup": warm, "ms_per_step": 1e3 * info["seconds"] / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": spec["desc"], "sample": info["sample"]},
        "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": 1, "kind": "reference", "sample": info["sample"]},
        "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_ours(args, rank, world, local_rank):
    import torch
    import __graft_entry__
    gf = __graft_entry__.import_package()
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        dist = dist_mod
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local_rank)
    spec = WORKLOADS[args.workload]
    with tempfile.TemporaryDirectory() as tmp:
        d = build_deck(gf, args.workload, sample=False)
        m0 = d.m0
        d.m0 = None          # uploaded below instead of written as text
        p0, q0 = d.p0, d.q0
        d.p0 = None
        ddir = os.path.join(tmp, "deck")
        gf.decks.write_deck(d, ddir)
        eng = gf.Engine(ddir, device=local_rank)
        if m0 is not None:
            eng.upload("m", m0)
        if p0 is not None:
            eng.upload("p", p0)
            eng.upload("q", q0)
        info = eng.info
        ncell = d.n
        mc = d.material_cell()
        mfe_ids = [q + 1 for q, mt in enumerate(d.materials) if mt.fm or mt.fe]
        mfe_frac = float(np.isin(mc, mfe_ids).mean()) if mfe_ids else 0.0
        stream = torch.cuda.ExternalStream(eng.stream(), device=local_rank)

        # warm-up (also builds and uploads the CUDA graphs)
        eng.advance(max(args.warmup, 1))
        eng.synchronize()

        # ---- device-timed region ----
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(local_rank) as cs:
            ev0.record(stream)
            eng.advance(args.steps)
            ev1.record(stream)
            ev1.synchronize()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ms = ev0.elapsed_time(ev1)
        if dist:
            t = torch.tensor([ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        clocks = cs.summary()
        info = eng.get_info()
        value = world * ncell * args.steps / (ms / 1e3)

        # ---- end-to-end through the C ABI with host buffers ----
        e2e_steps = max(1, min(args.steps, 20))
        obs = [o for o, on in (("m", info.fm), ("m_afm1", info.afm), ("m_afm2", info.afm), ("p", info.fe),
                               ("u", info.elastic)) if on]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            eng.advance(1)                      # uploads the step's drive row (pinned H2D)
            for o in obs:                       # D2H reads of the step's observables
                eng.average(o)
            if info.em:
                eng.probe_em(d.nx // 2, d.ny // 2, min(d.nz - 1, sum(l[0] for l in d.layers[:2]) - 2))
        e2e_s = time.perf_counter() - t0
        if dist:
            t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e_value = world * ncell * e2e_steps / e2e_s
        h2d = 520     # one StepDrive row per step (time + 4 stage rows of 128 B)
        d2h = 8 * 3 * len(obs) + (8 * 6 if info.em else 0)  # averages, E and H at the probe cell

        # ---- per-kernel device time for the roofline ----
        prof = eng.profile_steps(2)
        eng.check_finite()
        eng.close()

    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return
    kname = max(prof, key=lambda k: prof[k][1])
    launches, total_ms = prof[kname]
    avg_s = total_ms / launches / 1e3
    units = units_per_launch(kname, info)
    bpu = alg_bytes_per_unit(kname, info, mfe_frac)
    achieved = bpu * units / avg_s / 1e9
    peak, peak_kind = load_peaks()
    step_ms_prof = sum(v[1] for v in prof.values()) / 2.0
    roof = {"kernel": kname, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "traffic": committed_traffic(kname, args.workload),
            "alg_bytes_per_launch": bpu * units, "avg_launch_ms": avg_s * 1e3,
            "share_of_step": total_ms / 2.0 / step_ms_prof}

    cpu = None
    if not args.no_cpu_baseline:
        with tempfile.TemporaryDirectory() as tmp:
            v, ci = cpu_reference(gf, args.workload, args.ref_steps, tmp, 3)
        if v is not None:
            cpu = {"value": v, "unit": "cell-steps/s", "cores": 1, "kind": "reference", "sample": ci["sample"]}
    line = {
        "metric": "cell-steps/s FP64", "value": value, "unit": "cell-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": spec["desc"], "cells": ncell, "steps_timed": args.steps,
                   "parallelism": f"replicas{world}" if world > 1 else "single",
                   "l2": f"state resident in HBM ({info.device_bytes / 1e9:.2f} GB) > L2 (126 MB): no flush needed",
                   "graph": "one CUDA graph per step parity"},
        "roofline": roof,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps},
        "clocks": clocks,
        "gpu_launches": int(info.launches_per_step) * args.steps,
        "kernels_ms_per_step": {k: v[1] / 2.0 for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="magnetoelastic")
    ap.add_argument("--ref-steps", type=int, default=40)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
