"""Benchmark of the coupled RK4 phase-field step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ferroelectric|magnetoelastic|fm_demag|sweep]
                    [--precision both|fp64|mixed]

Workload (default): the ferroelectric TDGL + electrostriction +
elastodynamics + Maxwell FDTD run on a 128^3 grid (PbTiO3-like film, dx =
1 nm, seeded random P within +-1e-3 C/m^2, z-polarised Gaussian sheet
current), the largest single-GPU workload, run in both FP64 and FP32-mixed.
One step = one full RK4 step of all active physics.  The metric is
cell-steps/s (grid cells x steps / device time), whole job over all ranks: the
headline `value` is the FP64 form (the reference's arithmetic); with
--precision both (the default) the line also carries `mixed`, the same
measurement of the FP32 mixed form, its speed-up over FP64 and its trace error
against the FP64 engine on the same initial state.  At N=1 it also carries
`step_roofline` (the whole step's algorithmic bytes per cell-step over the
measured copy peak), `other_workloads` (the coupled magnetoelastic 128x128x96
film and the 64x64x16 FM + magnetostatics run, both forms), `adjoint` (the
cost of the discrete adjoint against the forward step, FP32 mixed and FP64, on a 256x256x32
ferromagnetic film) and `batched` (48 ferroelectric instances per graph).

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
                          sample_kw=dict(nx=16, ny=16, nz=128),
                          desc="FE TDGL + electrostriction + elastodynamics + FDTD, 128^3, dx=1nm"),
}

# Algorithmic bytes per unit (cell, or edge/face for the Yee kernels) of one
# launch, averaged over the four RK stages: every array the kernel must read
# or write, once (stage-dependent terms weighted 3/4 where they occur in 3 of
# the 4 stages); neighbour re-reads are not counted.
def alg_bytes_per_unit(kernel: str, info, mfe_frac: float = 0.0, mixed: bool = False) -> float:
    """Bytes one unit (cell, Yee vertex) of a launch must move, averaged over
    the four RK stages (stage outputs are written at stages 1-3, the
    accumulators read at stages 2-4, the step value read at stages 1-3).
    mfe_frac: fraction of cells that are ferromagnetic or ferroelectric.
    Mixed form: 4-byte reals, plus the compensation word of every state
    scalar read and written in the last stage (0.5 accesses per launch)."""
    D = 4.0 if mixed else 8.0
    comp = 0.5 if mixed else 0.0
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
        return (reads + writes + comp * 6) * D + 1
    if kernel == "k_llg_fm":
        reads = 3 + 3 + 3 * 0.75 + 3 + 6 * info.elastic + 3 * info.em
        writes = 3 * 0.75 + 3 + 3 * info.em
        return (reads + writes + comp * 3) * D + 1
    if kernel == "k_fe":
        reads = 3 + 3 + 3 * 0.75 + 3 + 3 + 3 * 0.75 + 6 + 6 + 3 + 3 * info.em
        writes = 3 * 0.75 * 2 + 3 * 2
        return (reads + writes + comp * 6) * D + 1
    if kernel == "k_em_fused":
        # per Yee vertex: three E edges and three H faces, each with stage input,
        # step value, accumulator read/write and stage output; dM/dt and dP/dt
        per_comp = 1 + 0.75 + 0.75 + 0.75 + 1 + comp
        return (6 * per_comp + 3 * info.fm + 3 * info.fe) * D + 1
    return float("nan")


# Algorithmic bytes per cell-step of each physics block: the compulsory
# traffic of classical RK4 with one read and one write per array per kernel
# (18 accesses per state scalar per step: FP64 144 B, FP32-mixed 72 B + 8 B of
# compensation word), plus the per-stage static-field reads, stencil halo
# re-reads free; a block counts over the cells it is active on.
STEP_BYTES = {  # block: (FP64, FP32-mixed)
    "fm": (532.0, 292.0), "afm": (964.0, 532.0), "fe": (864.0, 480.0), "elastic": (984.0, 540.0),
    "em": (864.0, 480.0), "drude": (1296.0, 720.0), "demag": (672.0, 336.0),
}


def step_alg_bytes(d, info, mixed: bool) -> float:
    """Algorithmic bytes of one step of deck `d` per grid cell."""
    mc = d.material_cell()
    n = float(mc.size)
    col = 1 if mixed else 0

    def frac(pred):
        ids = [q + 1 for q, mt in enumerate(d.materials) if pred(mt)]
        return float(np.isin(mc, ids).sum()) / n if ids else 0.0
    b = 0.0
    if info.fm:
        b += STEP_BYTES["fm"][col] * frac(lambda m: m.fm)
    if info.afm:
        b += STEP_BYTES["afm"][col] * frac(lambda m: m.afm)
    if info.fe:
        b += STEP_BYTES["fe"][col] * frac(lambda m: m.fe)
    if info.elastic:
        b += STEP_BYTES["elastic"][col] * float((mc != 0).sum()) / n
    if info.em:
        b += STEP_BYTES["em"][col]
        if any(m.drude[0][1] != 0 or m.drude[1][1] != 0 or m.drude[2][1] != 0 for m in d.materials):
            b += STEP_BYTES["drude"][col]
    if info.demag_per_stage:
        b += STEP_BYTES["demag"][col]
    return b


def step_roofline(d, info, ms_per_step: float, mixed: bool) -> dict:
    bpc = step_alg_bytes(d, info, mixed)
    achieved = bpc * d.n / (ms_per_step / 1e3) / 1e9
    peak, kind = load_peaks()
    return {"bound": "hbm", "alg_bytes_per_cell_step": bpc, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": kind}


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


def committed_traffic(kernel: str, workload: str, mixed: bool = False):
    """dram read+write bytes per launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{workload}{'_mixed' if mixed else ''}.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    return d.get("dram_bytes_per_launch_full_size")


class ClockSampler:
    """SM clock and clock-event reasons sampled through NVML by a host thread
    every ~2 ms while the timed region runs.  A timed region of a few tens of
    milliseconds is shorter than nvidia-smi's start-up and first sampling
    interval, so polling NVML directly is what yields samples inside it;
    `mark_start` / `mark_end` bracket the region in host time and `summary`
    keeps the samples taken between them (the nearest ones if the region was
    shorter than one poll).  Only reads the GPU's state."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.samples = []
        self.t0 = self.t1 = None
        self.err = None
        self._stop = False
        self._thread = None
        self.smax = None

    def _poll(self, nv, h):
        while not self._stop:
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((time.perf_counter(), float(sm), int(rs)))
            except Exception as e:      # keep the region's timing unaffected
                self.err = str(e)
                return
            time.sleep(0.002)

    def __enter__(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            # CUDA device index -> NVML handle through the device UUID (NVML
            # enumerates every GPU of the node, CUDA only the visible ones)
            import torch
            h = None
            try:
                h = nv.nvmlDeviceGetHandleByUUID("GPU-" + str(torch.cuda.get_device_properties(self.gpu).uuid))
            except Exception:
                h = None
            if h is None:
                vis = os.environ.get("CUDA_VISIBLE_DEVICES")
                idx = int(vis.split(",")[self.gpu]) if vis and vis.split(",")[self.gpu].strip().isdigit() else self.gpu
                h = nv.nvmlDeviceGetHandleByIndex(idx)
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self._thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self._thread.start()
            deadline = time.perf_counter() + 2.0
            while not self.samples and self.err is None and time.perf_counter() < deadline:
                time.sleep(0.001)
        except Exception as e:
            self.err = str(e)
        return self

    def mark_start(self):
        self.t0 = time.perf_counter()

    def mark_end(self):
        self.t1 = time.perf_counter()
        # one more poll after the region so that a short region has a sample on each side
        time.sleep(0.005)

    def __exit__(self, *a):
        self._stop = True
        if self._thread:
            self._thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": [], "samples": 0,
                    "note": f"no NVML samples: {self.err}"}
        t0 = self.t0 if self.t0 is not None else self.samples[0][0]
        t1 = self.t1 if self.t1 is not None else self.samples[-1][0]
        inside = [s for s in self.samples if t0 <= s[0] <= t1]
        where = "inside the timed region"
        if not inside:
            inside = sorted(self.samples, key=lambda s: min(abs(s[0] - t0), abs(s[0] - t1)))[:2]
            where = "nearest to the timed region (shorter than one poll)"
        reasons = sorted({nm for _, _, rs in inside for nm, bit in self.REASONS.items() if rs & bit})
        return {"sm_mhz": statistics.median(s[1] for s in inside), "sm_max_mhz": self.smax, "reasons": reasons,
                "samples": len(inside), "source": f"NVML, {where}"}


GRID_OVERRIDE = None    # (nx, ny, nz) from --grid: a smaller copy of the workload for profiling


def build_deck(gf, wl: str, sample: bool):
    spec = WORKLOADS[wl]
    kw = dict(spec["sample_kw"] if sample else spec["kw"])
    if GRID_OVERRIDE and not sample:
        nx, ny, nz = GRID_OVERRIDE
        if spec["preset"] == "magnetoelastic":
            # keep the layer stack's proportions (substrate, film, vacuum)
            sub = max(1, round(kw["sub"] * nz / kw.get("nz", 96)))
            film = max(1, round(kw["film"] * nz / kw.get("nz", 96)))
            kw.update(sub=min(sub, nz - 1), film=min(film, nz - min(sub, nz - 1)))
        kw.update(nx=nx, ny=ny, nz=nz)
    d = gf.decks.PRESETS[spec["preset"]](**kw)
    return d


def cpu_reference(gf, wl: str, steps: int, tmp: str, warmup: int = 0, procs: int = 1):
    """GO-Ferro's own solver on the bounded CPU sample: `warmup` untimed steps,
    then `steps` timed ones; returns (cell-steps/s, info).  The reference's
    host build is serial (its OpenACC pragmas are ignored on the host), so
    the whole host is used by running `procs` copies of the sample at once,
    one per core; the rate is procs x cells x steps over the slowest copy's
    time loop."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import refrun
    if not refrun.available():
        return None, "oracle binary not built"
    d = build_deck(gf, wl, sample=True)
    d.steps = steps + warmup
    ddir = os.path.join(tmp, "ref_deck")
    gf.decks.write_deck(d, ddir)

    def one(q):
        return refrun.run(ddir, os.path.join(tmp, f"ref_out{q}"), steps=steps + warmup,
                          trace_every=max(steps + warmup, 1), warmup=warmup)
    with ThreadPoolExecutor(max_workers=procs) as ex:
        runs = list(ex.map(one, range(procs)))
    secs = max(r["timing"]["seconds"] for r in runs)
    value = procs * d.n * steps / secs
    sample = (f"{d.nx}x{d.ny}x{d.nz} sub-grid of the workload's layer stack, {steps} steps after {warmup} untimed, "
              f"serial reference build" + (f", {procs} concurrent copies (one per core)" if procs > 1 else ""))
    return value, {"seconds": secs, "sample": sample, "cells": d.n, "procs": procs}


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_reference_arm(args, rank, world):
    import __graft_entry__
    gf = __graft_entry__.import_package()
    if rank != 0:
        return
    spec = WORKLOADS[args.workload]
    procs = max(1, min(host_cores(), args.ref_procs))
    with tempfile.TemporaryDirectory() as tmp:
        steps = max(1, min(args.steps, args.ref_steps))
        warm = min(args.warmup, 3)
        value, info = cpu_reference(gf, args.workload, steps, tmp, warm, procs=procs)
    if value is None:
        print(json.dumps({"impl": "reference", "unavailable": info}))
        return
    line = {
        "impl": "reference", "metric": "cell-steps/s FP64", "value": value, "unit": "cell-steps/s",
        "n_gpus": world, "steps": steps, "warmup": warm, "ms_per_step": 1e3 * info["seconds"] / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": spec["desc"], "sample": info["sample"]},
        "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": procs, "kind": "reference",
                         "sample": info["sample"]},
        "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def max_over_ranks(x: float, dist, torch, device: str) -> float:
    """The largest value of x over all ranks (x itself without a process
    group): replicas are timed by the slowest rank."""
    if not dist:
        return x
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, cells: int, steps: int, seconds: float) -> float:
    """Whole-job cell-steps/s of `world` replicas, each advancing `cells`
    cells by `steps` steps, timed by the slowest rank."""
    return world * cells * steps / seconds


TRACE_GROUPS = {"m": (0, 3), "p": (3, 6), "u": (6, 9), "E": (9, 12), "H": (12, 15)}


def observe(eng, info, probe):
    """<m>, <p>, <u>, probed E and H (zeros where a physics is off)."""
    row = np.zeros(15)
    if info.fm:
        row[0:3] = eng.average("m")
    if info.fe:
        row[3:6] = eng.average("p")
    if info.elastic:
        row[6:9] = eng.average("u")
    if info.em:
        e, h = eng.probe_em(*probe)
        row[9:12] = e
        row[12:15] = h
    return row


def trace_error(mine, ref):
    """Largest deviation of each vector observable over a trace, relative to
    the observable's largest component magnitude in the FP64 trace."""
    out = {}
    for name, (a, b) in TRACE_GROUPS.items():
        scale = float(np.max(np.abs(ref[:, a:b])))
        if scale > 0.0:
            out[name] = float(np.max(np.abs(mine[:, a:b] - ref[:, a:b]))) / scale
    return out


def measure(gf, torch, dist, args, world, local_rank, precision, d, ddir, uploads, probe):
    """Trace, warm-up, device-timed steps, end-to-end steps and per-kernel
    times of one engine on the deck in `ddir`."""
    eng = gf.Engine(ddir, device=local_rank, precision=precision)
    for name, arr in uploads:
        eng.upload(name, arr)
    info = eng.info
    ncell = d.n
    stream = torch.cuda.ExternalStream(eng.stream(), device=local_rank)

    # observable trace from the initial state (compared across the two forms)
    trace = [observe(eng, info, probe)]
    for _ in range(args.trace_steps):
        eng.advance(1)
        trace.append(observe(eng, info, probe))
    trace = np.array(trace)

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
        cs.mark_start()
        ev0.record(stream)
        eng.advance(args.steps)
        ev1.record(stream)
        ev1.synchronize()
        cs.mark_end()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms, dist, torch, "cuda")
    clocks = cs.summary()
    info = eng.get_info()
    value = aggregate_rate(world, ncell, args.steps, ms / 1e3)

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
            eng.probe_em(*probe)
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s, dist, torch, "cuda")
    e2e_value = aggregate_rate(world, ncell, e2e_steps, e2e_s)
    h2d = 520     # one StepDrive row per step (time + 4 stage rows of 128 B)
    d2h = 8 * 3 * len(obs) + (8 * 6 if info.em else 0)  # averages, E and H at the probe cell

    # ---- per-kernel device time for the roofline ----
    prof = eng.profile_steps(2)
    eng.check_finite()
    eng.close()
    return dict(value=value, ms=ms, clocks=clocks, info=info, trace=trace, prof=prof,
                e2e={"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                     "steps": e2e_steps})


def roofline(r, args, mfe_frac, mixed):
    prof, info = r["prof"], r["info"]
    kname = max(prof, key=lambda k: prof[k][1])
    launches, total_ms = prof[kname]
    avg_s = total_ms / launches / 1e3
    units = units_per_launch(kname, info)
    bpu = alg_bytes_per_unit(kname, info, mfe_frac, mixed)
    achieved = bpu * units / avg_s / 1e9
    peak, peak_kind = load_peaks()
    step_ms_prof = sum(v[1] for v in prof.values()) / 2.0
    return {"kernel": kname, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "traffic": committed_traffic(kname, args.workload, mixed),
            "alg_bytes_per_launch": bpu * units, "avg_launch_ms": avg_s * 1e3,
            "share_of_step": total_ms / 2.0 / step_ms_prof}


def adjoint_cost(gf, torch, args, local_rank):
    """Cost of the discrete adjoint against a forward pass: FM LLG + FFT
    magnetostatics + magnetoelastic elastodynamics on 256x256x32 (the adjoint
    configuration's grid and physics: YIG-like magnetoelastic film with free
    surfaces and the Liao boundary at k = 0, 1 T bias, per-cell damping 1e-3
    with 10 % seeded noise, a 256-sample x waveform), in the FP32 mixed form
    (the configuration's form) and in FP64.  Every time is device time on the
    engine's stream (CUDA events around the enqueued work, host launch gaps
    included): the engine's graph-replayed forward step of the same
    precision, the adjoint's own forward run (checkpoints every 100 steps,
    <m_x> trace) and its backward run (each checkpoint block recomputed once
    with its stages kept in the stage store, then the reverse sweep).  The mixed entry also gives the relative difference of
    its gradients from the FP64 adjoint's on the same inputs."""
    mu0 = 1.256637061e-6
    steps, K, nw = args.adjoint_steps, args.adjoint_checkpoint, 256
    gx, gy, gz = (int(v) for v in args.adjoint_grid.lower().split("x"))
    out = {}
    grads = {}
    with tempfile.TemporaryDirectory() as tmp:
        d = gf.decks.preset_fm_demag(nx=gx, ny=gy, nz=gz, steps=steps)
        d.Hext_table = None
        d.Hext_stat = (0.0, 0.0, 1.0 / mu0)
        d.materials = [gf.decks.yig(1e-3, magnetoelastic=True)]
        d.elastic, d.elasto_back, d.elasto_on = True, True, True
        d.abc_1D, d.liao_w = False, 0.5
        gf.decks.write_deck(d, tmp)
        rng = np.random.default_rng(20241208)
        alpha = 1e-3 * (1.0 + 0.1 * rng.random(d.n))
        tt = (np.arange(nw) + 0.5) / nw
        wave = (1e-3 / mu0) * np.sin(2 * np.pi * 8 * tt) * np.exp(-((tt - 0.3) / 0.1) ** 2)
        for prec in ("mixed", "fp64"):
            with gf.Engine(tmp, device=local_rank, precision=prec) as eng:
                stream = torch.cuda.ExternalStream(eng.stream(), device=local_rank)
                eng.advance(3)
                eng.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                eng.advance(steps)
                e1.record(stream)
                e1.synchronize()
                t_eng = e0.elapsed_time(e1) / 1e3
                with gf.Adjoint(eng, nw, K) as adj:
                    adj.set_alpha(alpha)
                    adj.set_waveform(wave)
                    # warm-up: one forward run of the timed length, so the
                    # checkpoint and trace buffers it sizes are allocated
                    # outside the timed run
                    adj.forward(steps)
                    eng.synchronize()
                    e0.record(stream)
                    tr = adj.forward(steps)
                    e1.record(stream)
                    e1.synchronize()
                    t_fwd = e0.elapsed_time(e1) / 1e3
                    # d loss / d <m_x>: spectral power of the trace in 0.1-0.5 THz
                    X = np.fft.rfft(tr)
                    f = np.fft.rfftfreq(tr.size, d.dt)
                    band = np.nonzero((f >= 0.1e12) & (f <= 0.5e12))[0]
                    n = np.arange(tr.size)
                    g = np.zeros(tr.size)
                    for k in band:
                        g += 2.0 * np.real(np.conj(X[k]) * np.exp(-2j * np.pi * k * n / tr.size))
                    eng.synchronize()
                    e0.record(stream)
                    gw, ga = adj.backward(g)
                    e1.record(stream)
                    e1.synchronize()
                    t_bwd = e0.elapsed_time(e1) / 1e3
                    grads[prec] = (gw, ga)
                    store_used, store_bytes = adj.store_info()
            out[prec] = {"steps": steps, "checkpoint_every": K,
                         "forward_ms_per_step": 1e3 * t_eng / steps,
                         "adjoint_forward_ms_per_step": 1e3 * t_fwd / steps,
                         "backward_ms_per_step": 1e3 * t_bwd / steps,
                         "backward_over_forward": t_bwd / t_eng,
                         "forward_plus_backward_over_forward": (t_fwd + t_bwd) / t_eng,
                         "loss_band_bins": int(len(band)),
                         "backward_layout": "stage store" if store_used else "recompute",
                         "backward_layout_bytes": store_bytes}
    (gw, ga), (gw64, ga64) = grads["mixed"], grads["fp64"]
    out["mixed"]["grad_wave_rel_diff_vs_fp64"] = float(np.max(np.abs(gw - gw64)) / max(np.max(np.abs(gw64)), 1e-300))
    out["mixed"]["grad_alpha_rel_diff_vs_fp64"] = float(np.max(np.abs(ga - ga64)) / max(np.max(np.abs(ga64)), 1e-300))
    out["workload"] = (f"FM LLG + FFT magnetostatics + magnetoelastic elastodynamics, {gx}x{gy}x{gz}, "
                       "per-cell alpha and 256-sample waveform; FP32 mixed (the configuration's form) and FP64")
    out["timing"] = "device time (CUDA events on the engine stream)"
    out["definition"] = ("backward = recompute of every checkpoint block (stage store layout: keeping each step's stages; "
                         "recompute layout: a second per-step stage recompute) + reverse sweep; "
                         "forward = the engine's step of the same precision (CUDA graph)")
    return out


SWEEP_SIZES = [(32, 32, 32), (48, 48, 32), (64, 64, 32), (96, 96, 24)]


def sweep_decks(gf, count, steps, seed=20241207):
    """Instances of the batched sweep: ferroelectric TDGL + electrostriction +
    elastodynamics + FDTD (PbTiO3-like, dx = 1 nm), grid drawn by seed from
    SWEEP_SIZES, z-polarised sheet current J_f type 6 (Gaussian x sine) with
    amplitude log-uniform over 10-500 kV/cm and carrier uniform over
    0.5-3 THz.  The Courant-limited step (2.45e-18 s) makes a run of
    `steps` steps last a few fs, so the Gaussian envelope is centred inside
    the run (sigma = steps*dt/10) instead of a THz-scale width."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        nx, ny, nz = SWEEP_SIZES[int(rng.integers(len(SWEEP_SIZES)))]
        kvcm = 10.0 ** rng.uniform(1.0, np.log10(500.0))
        f0 = rng.uniform(0.5e12, 3e12)
        d = gf.decks.preset_ferroelectric(nx=nx, ny=ny, nz=nz, steps=steps)
        d.name = f"sweep_{i:02d}_{nx}x{ny}x{nz}"
        d.jf_type = 6
        d.jf_freq = f0
        d.jf_sigma = steps * d.dt / 10.0
        d.jf_amp = d.jf_amp * kvcm / 100.0        # the preset radiates ~100 kV/cm
        out.append((d, kvcm, f0))
    return out


def run_sweep(gf, torch, args, local_rank, count, steps, fp64_check):
    """Batched mixed-form sweep: all instances advanced by one graph per step
    (gf_batch in its phase mode: each RK stage a few launches over the work
    items of every instance, autotuned tile chunks and phase-A fusion)
    against the same engines advanced one after another with their own
    graphs and against the batch's branch mode (one graph branch per
    engine); optional FP64 error per instance."""
    import shutil
    decks = sweep_decks(gf, count, steps)
    tmp = tempfile.mkdtemp()
    engines = []
    try:
        t_create = time.perf_counter()
        dirs = []
        for d, _, _ in decks:
            p0, q0 = d.p0, d.q0
            d.p0 = None
            ddir = os.path.join(tmp, d.name)
            gf.decks.write_deck(d, ddir)
            d.p0, d.q0 = p0, q0
            dirs.append(ddir)
            e = gf.Engine(ddir, device=local_rank, precision="mixed")
            e.upload("p", p0)
            e.upload("q", q0)
            engines.append(e)
        t_create = time.perf_counter() - t_create
        cells = sum(d.n for d, _, _ in decks)
        # sequential: every engine with its own graph, one after another
        for e in engines:
            e.advance(2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for e in engines:
            e.advance(steps)
        for e in engines:
            e.synchronize()
        t_seq = time.perf_counter() - t0
        def timed_batch(mode):
            with gf.Batch(engines, autotune=True, mode=mode) as b:
                chunks = sorted({b.tuned_chunk(i) for i in range(len(engines))})
                plan = b.plan()
                stream = torch.cuda.ExternalStream(b.stream(), device=local_rank)
                b.advance(2)
                b.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                b.advance(steps)
                e1.record(stream)
                e1.synchronize()
                return e0.elapsed_time(e1) / 1e3, chunks, plan

        # one graph branch per engine, then the phase mode (13 launches per
        # step for all engines of these decks), the batch's default for them
        t_branch, _, _ = timed_batch("branches")
        t_batch, chunks, plan = timed_batch("auto")
        pz = [float(e.average("p")[2]) for e in engines]
        result = {"instances": count, "cells": cells, "steps_timed": steps,
                  "value": cells * steps / t_batch, "unit": "cell-steps/s", "ms_per_step": 1e3 * t_batch / steps,
                  "sequential_ms_per_step": 1e3 * t_seq / steps, "speedup_vs_sequential": t_seq / t_batch,
                  "branches_ms_per_step": 1e3 * t_branch / steps, "speedup_vs_branches": t_branch / t_batch,
                  "plan": plan,
                  "tuned_elastic_chunks": chunks, "create_s": t_create,
                  "grids": {f"{a}x{b_}x{c}": sum(1 for d, _, _ in decks if (d.nx, d.ny, d.nz) == (a, b_, c))
                            for a, b_, c in SWEEP_SIZES}}
        if fp64_check:
            # the same instances from the same state in FP64, one trace point per step
            n_check = 3 * steps + 6     # sequential, branch-mode and phase-mode runs: 2 warm-up + timed steps each
            errs, resp = [], []
            for (d, kvcm, f0), ddir, pzm in zip(decks, dirs, pz):
                with gf.Engine(ddir, device=local_rank, precision="fp64") as e64:
                    e64.upload("p", d.p0)
                    e64.upload("q", d.q0)
                    e64.advance(n_check)
                    p64 = e64.average("p")
                scale = max(abs(float(x)) for x in p64)
                errs.append(abs(pzm - float(p64[2])) / scale)
                resp.append({"kV_per_cm": kvcm, "f0_THz": f0 / 1e12, "grid": f"{d.nx}x{d.ny}x{d.nz}",
                             "pz_mixed": pzm, "pz_fp64": float(p64[2]), "rel_err": errs[-1]})
            result["fp64_check_steps"] = n_check
            result["max_rel_err_vs_fp64"] = max(errs)
            result["instances_detail"] = resp
        return result
    finally:
        for e in engines:
            e.close()
        shutil.rmtree(tmp, ignore_errors=True)


def measure_workload(gf, torch, dist, args, world, local_rank, wl, forms):
    """Deck of workload `wl` (initial state uploaded, not written as text),
    and the measurement of each form in `forms`."""
    results = {}
    with tempfile.TemporaryDirectory() as tmp:
        d = build_deck(gf, wl, sample=False)
        uploads = []
        if d.m0 is not None:
            uploads.append(("m", d.m0))
        if d.p0 is not None:
            uploads += [("p", d.p0), ("q", d.q0)]
        m0, p0 = d.m0, d.p0
        d.m0 = None
        d.p0 = None
        ddir = os.path.join(tmp, "deck")
        gf.decks.write_deck(d, ddir)
        d.m0, d.p0 = m0, p0
        mc = d.material_cell()
        mfe_ids = [q + 1 for q, mt in enumerate(d.materials) if mt.fm or mt.fe]
        mfe_frac = float(np.isin(mc, mfe_ids).mean()) if mfe_ids else 0.0
        probe = (d.nx // 2, d.ny // 2, min(d.nz - 1, sum(l[0] for l in d.layers[:2]) - 2))
        for form in forms:
            results[form] = measure(gf, torch, dist, args, world, local_rank, form, d, ddir, uploads, probe)
    return d, results, mfe_frac


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
    if args.workload == "sweep":
        # the batched configuration on its own: one JSON line of the sweep
        sw = run_sweep(gf, torch, args, local_rank, count=48, steps=args.steps, fp64_check=True)
        if dist:
            dist.destroy_process_group()
        if rank == 0:
            line = {"metric": "cell-steps/s FP32-mixed batched sweep", "value": sw.pop("value") * world,
                    "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps, "warmup": 2,
                    "ms_per_step": sw["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                    "config": {"workload": "48 ferroelectric + FDTD instances, grids drawn from 32^3, 48x48x32, "
                                           "64x64x32, 96x96x24; J_f type 6, 10-500 kV/cm, 0.5-3 THz",
                               "parallelism": f"replicas{world}" if world > 1 else "single"},
                    "sweep": sw}
            print(json.dumps(line))
        return
    spec = WORKLOADS[args.workload]
    forms = ["fp64", "mixed"] if args.precision == "both" else [args.precision]
    d, results, mfe_frac = measure_workload(gf, torch, dist, args, world, local_rank, args.workload, forms)
    others = {}
    if world == 1 and not args.no_other_workloads and args.workload == "ferroelectric":
        # the other single-GPU workloads, both forms, on the same box (context
        # for the headline; the headline is the largest single-GPU workload)
        import copy
        a2 = copy.copy(args)
        a2.trace_steps = 20
        for wl in ("magnetoelastic", "fm_demag"):
            dw, rw, _ = measure_workload(gf, torch, dist, a2, world, local_rank, wl, ["fp64", "mixed"])
            ent = {"workload": WORKLOADS[wl]["desc"], "cells": dw.n}
            for form, rr in rw.items():
                ent[form] = {"value": rr["value"], "ms_per_step": rr["ms"] / args.steps, "clocks": rr["clocks"],
                             "step_roofline": step_roofline(dw, rr["info"], rr["ms"] / args.steps, form == "mixed")}
            ent["speedup_mixed_vs_fp64"] = rw["mixed"]["value"] / rw["fp64"]["value"]
            ent["mixed_trace_error_vs_fp64"] = trace_error(rw["mixed"]["trace"], rw["fp64"]["trace"])
            others[wl] = ent

    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return
    head_form = forms[0]
    r = results[head_form]
    info = r["info"]
    ncell = d.n

    cpu = None
    if not args.no_cpu_baseline:
        with tempfile.TemporaryDirectory() as tmp:
            v, ci = cpu_reference(gf, args.workload, args.ref_steps, tmp, 3)
        if v is not None:
            cpu = {"value": v, "unit": "cell-steps/s", "cores": 1, "kind": "reference", "sample": ci["sample"]}
    head_mixed = head_form == "mixed"
    line = {
        "metric": "cell-steps/s FP32-mixed" if head_mixed else "cell-steps/s FP64", "value": r["value"],
        "unit": "cell-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32" if head_mixed else "f64",
        "data": "synthetic",
        "config": {"workload": spec["desc"], "cells": ncell, "steps_timed": args.steps,
                   "parallelism": f"replicas{world}" if world > 1 else "single",
                   "l2": f"state resident in HBM ({info.device_bytes / 1e9:.2f} GB) > L2 (126 MB): no flush needed",
                   "graph": "one CUDA graph per step parity"},
        "roofline": roofline(r, args, mfe_frac, head_mixed),
        "step_roofline": step_roofline(d, info, r["ms"] / args.steps, head_mixed),
        "cpu_baseline": cpu,
        "e2e": r["e2e"],
        "clocks": r["clocks"],
        "gpu_launches": int(info.launches_per_step) * args.steps,
        "kernels_ms_per_step": {k: v[1] / 2.0 for k, v in sorted(r["prof"].items(), key=lambda kv: -kv[1][1])},
    }
    if "fp64" in results and "mixed" in results:
        rm = results["mixed"]
        err = trace_error(rm["trace"], results["fp64"]["trace"])
        line["mixed"] = {
            "metric": "cell-steps/s FP32-mixed", "value": rm["value"], "unit": "cell-steps/s",
            "ms_per_step": rm["ms"] / args.steps, "speedup_vs_fp64": rm["value"] / r["value"],
            "trace_error_vs_fp64": err, "trace_steps": args.trace_steps,
            "max_trace_error": max(err.values()) if err else None,
            "error_definition": "max over the trace of |mixed - fp64| / max|fp64 component| per vector observable",
            "roofline": roofline(rm, args, mfe_frac, True),
            "step_roofline": step_roofline(d, rm["info"], rm["ms"] / args.steps, True),
            "e2e": rm["e2e"], "clocks": rm["clocks"],
            "gpu_launches": int(rm["info"].launches_per_step) * args.steps,
            "kernels_ms_per_step": {k: v[1] / 2.0 for k, v in sorted(rm["prof"].items(), key=lambda kv: -kv[1][1])},
            "device_bytes": int(rm["info"].device_bytes),
        }
    if others:
        line["other_workloads"] = others
    if world == 1 and not args.no_adjoint:
        line["adjoint"] = adjoint_cost(gf, torch, args, local_rank)
    if world == 1 and not args.no_batch:
        sw = run_sweep(gf, torch, args, local_rank, count=48, steps=args.sweep_steps, fp64_check=True)
        sw["workload"] = ("batched sweep: 48 ferroelectric + FDTD instances, grids drawn from 32^3, 48x48x32, "
                          "64x64x32, 96x96x24, FP32 mixed, one CUDA graph per step in the layout the batch's tuner "
                          "timed faster (see plan: one branch per engine, or launches per stage phase over every engine's work items)")
        line["batched"] = sw
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["sweep"], default="ferroelectric")
    ap.add_argument("--ref-steps", type=int, default=100)
    ap.add_argument("--no-other-workloads", action="store_true")
    ap.add_argument("--grid", default=None,
                    help="NXxNYxNZ: run a smaller copy of the workload (profiling captures); not a bench line")

    ap.add_argument("--ref-procs", type=int, default=64,
                    help="most concurrent copies of the serial reference in --impl reference (one per host core)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", choices=["both", "fp64", "mixed"], default="both")
    ap.add_argument("--trace-steps", type=int, default=100)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--sweep-steps", type=int, default=100)
    ap.add_argument("--adjoint-steps", type=int, default=400)
    ap.add_argument("--adjoint-grid", default="256x256x32", help="grid of the adjoint cost measurement (NXxNYxNZ)")
    ap.add_argument("--adjoint-checkpoint", type=int, default=100, help="steps between the adjoint's stored states")
    args = ap.parse_args()
    global GRID_OVERRIDE
    if args.grid:
        GRID_OVERRIDE = tuple(int(x) for x in args.grid.lower().split("x"))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
