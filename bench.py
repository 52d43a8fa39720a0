#!/usr/bin/env python
"""Benchmark of the engine on the FP32 dispersive-sphere workload.

Workload (one "step" = one FDTD time step over the whole grid): 384^3 inner
cells + 12-cell CPML on all faces = 408^3 = 67.9 M cells, dl = 1 mm, sphere
r = 0.1 m of a Drude (wp = 2e10, gamma = 1e9) + Lorentz (d_eps = 2, w0 = 3e10,
delta = 5e8) ADE medium, x-propagating TFSF Gaussian, NF2FF at 1/3/5 GHz
accumulated in FP64; fields, CPML psi and ADE state in FP32.  Inputs are
synthetic (no dataset is involved); the 3.3 GB of resident field state is far
larger than the 126 MB L2, so every step streams from HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Prints one JSON line.  `value` is device-timed Mcell-updates/s over K steps
(CUDA events on the engine's stream, max over ranks); `e2e` is the same metric
through the public run path (scene compile + upload + K steps + read-back of
all fields and NF2FF currents, wall clock), the path the reference's own
benchmark times (test/benchmark.cu:174-216).  With N > 1 every rank runs its
own copy of the scene (independent scenes, no data-path collective): weak
scaling.  `--impl reference` times the CPU restatement of the reference's
algorithm (oracle/, OpenMP over all host cores) on a bounded sample of the
same scene.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mcell-updates/s and % HBM roofline, FP32/batched/learned vs FP64 plain, 1 B200"
UNIT = "Mcell-updates/s"


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def esize(precision):
    return 8 if precision == "fp64" else 4


def algorithmic_bytes(gi, kernel, precision):
    """Compulsory DRAM bytes of one launch of `kernel` on grid `gi`.

    Bulk half-step (H or E): read the 3 updated and the 3 dual components,
    write the 3 updated ones, read the 1-byte material id: 9 T + 1 per cell.
    CPML: read + write psi of the 2 tangential components of every slab cell.
    ADE (E only): per dispersive cell and component, read + write J (per
    pole), J_prev (per pole) and E_prev (M-Lorentz).
    """
    T = esize(precision)
    nx, ny, nz = gi.nx, gi.ny, gi.nz
    cells = nx * ny * nz
    # slab cells per axis
    b = 0
    Ls = list(getattr(gi, "_pml", [0] * 6))
    for a, n_a in enumerate((nx, ny, nz)):
        L = Ls[2 * a] + Ls[2 * a + 1]
        b += L * cells // n_a
    ade = 0
    if gi.ade_kind:
        P = gi.ade_poles
        per_comp = 2 * T * P + ((2 * T * P + 2 * T) if gi.ade_kind == 3 else 0)
        ade = gi.n_dispersive_cells * 3 * per_comp
    if kernel in (0, 2):  # H or E half-step
        byt = cells * (9 * T + 1) + b * 2 * 2 * T
        return byt + (ade if kernel == 2 else 0)
    if kernel == 6:  # one-sweep step: read E^n, H^{n-1/2}; write H^{n+1/2}, E^{n+1}
        return cells * (12 * T + 1) + b * 4 * 2 * T + ade
    return None


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(tempfile.mkstemp(suffix=".csv")[1])

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[q] for r in rows for q in range(4) if r[5 + q].lower() == "active"})
        loaded = sorted(sm)[len(sm) // 4:] if len(sm) > 4 else sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def max_over_ranks(x, dist):
    """Max of x over all ranks (a time: the job's is the slowest rank's).
    dist = (torch, torch.distributed) or None; NCCL reduces on the device,
    gloo on the host."""
    if not dist:
        return x
    torch, tdist = dist
    dev = "cuda" if tdist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def job_rate(cells, steps, world, ms):
    """Whole-job Mcell-updates/s: every rank steps its own copy of `cells`
    cells `steps` times in `ms` (the slowest rank's time)."""
    return cells * steps * world / (ms / 1e3) / 1e6


def workload_label(scene, gi, cells):
    dims = f"{gi.nx}x{gi.ny}x{gi.nz}"
    if scene == "dispersive":
        return (f"dispersive sphere {dims} ({cells}^3 + 12-cell CPML), Drude+Lorentz ADE, TFSF Gaussian, "
                "NF2FF 1/3/5 GHz (FP64 accumulation)")
    parts = {"vacuum": "PEC box only", "pml": "12-cell CPML", "tfsf": "12-cell CPML + TFSF Gaussian",
             "nf2ff": "12-cell CPML + TFSF Gaussian + NF2FF 1/3/5 GHz"}[scene]
    return f"diagnostic variant of the dispersive-sphere workload, {dims}: {parts}"


def build_scene(cells, precision, scene="dispersive"):
    """The benchmark workload, or a reduced variant for kernel diagnostics
    (vacuum: PEC box only; pml: + CPML; tfsf: + CPML + TFSF; nf2ff: + NF2FF)."""
    from xfdtd_cuda_b200 import configs
    if scene == "dispersive":
        return configs.dispersive_sphere(cells=cells, precision=precision)
    s = configs.dispersive_sphere(cells=cells, precision=precision, freqs=(1e9, 3e9, 5e9) if scene == "nf2ff" else ())
    s.objects = s.objects[:1]
    if scene == "vacuum":
        s.boundaries = []
        s.sources = []
    elif scene == "pml":
        s.sources = []
    return s


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _omp_threads(n):
    """Set the OpenMP thread count of the calling thread (the CPU restatement
    runs its parallel loops from it)."""
    import ctypes
    try:
        ctypes.CDLL("libgomp.so.1").omp_set_num_threads(int(n))
    except OSError:
        pass


def cpu_sample(cells: int, steps: int, precision="fp64", threads: int | None = None):
    """Time the CPU restatement on a bounded sample of the workload."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import xfdtd_cuda_b200 as X
    from oracle import OracleSim
    sim = build_scene(cells, "fp64")
    sc, keep = sim.lower()
    h = X.Handle(sc, keep)
    o = OracleSim(h, steps + 2)
    threads = threads or int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    _omp_threads(threads)
    o.run(2)  # warm-up (first touch of the arrays)
    gi = h.info()
    t0 = time.perf_counter()
    o.run(steps)
    dt = time.perf_counter() - t0
    _omp_threads(int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)))
    n = gi.nx * gi.ny * gi.nz
    return {"value": n * steps / dt / 1e6, "unit": UNIT, "cores": threads, "kind": "port", "cpu": cpu_model(),
            "sample": f"dispersive sphere {gi.nx}x{gi.ny}x{gi.nz} ({cells}^3 + 12-cell CPML), FP64, {steps} steps, "
                      f"CPU restatement (oracle/, OpenMP {threads} threads), {dt:.1f} s"}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    cells = args.ref_cells
    sample = cpu_sample(cells, max(1, args.warmup))  # warm-up steps
    res = cpu_sample(cells, max(1, args.steps))
    out = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": "dispersive sphere (Drude+Lorentz ADE, TFSF, 12-cell CPML, NF2FF 1/3/5 GHz), "
                                  f"bounded CPU sample {cells}^3 inner cells", "cells_per_step": None},
           "cpu_baseline": res,
           "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    del sample
    print(json.dumps(out))
    return 0


def plain_compare(local: int, steps: int, warmup: int):
    """Mcell-updates/s of the dielectric-sphere workload (dielectric sphere 140^3 + 8-cell CPML
    = 156^3, TFSF, NF2FF at 1 GHz) in the FP64 plain form (the reference's
    kernel structure: per-cell coefficient arrays, one launch per component,
    separate CPML/TFSF corrector launches) next to the FP32 and FP64 fused
    one-sweep kernel, device-timed the same way as the headline number."""
    import xfdtd_cuda_b200 as X
    from xfdtd_cuda_b200 import _lib as L
    from xfdtd_cuda_b200 import configs
    res = {}
    for key, prec, path in (("fp64_plain", "fp64", L.PATH_PLAIN), ("fp64_fused", "fp64", L.PATH_FUSED),
                            ("fp32_fused", "fp32", L.PATH_FUSED)):
        sim = configs.dielectric_sphere(precision=prec)
        sc, keep = sim.lower()
        h = X.Handle(sc, keep)
        h.set_device(local)
        h.set_kernel_path(path)
        h.init(warmup + steps)
        gi = h.info()
        h.step(warmup)
        h.sync()
        ms = h.timed_step(steps)
        res[key] = gi.nx * gi.ny * gi.nz * steps / (ms / 1e3) / 1e6
        h.close()
    return {"workload": "dielectric sphere 156x156x156 (140^3 + 8-cell CPML), eps_r=3 mu_r=2, TFSF, NF2FF 1 GHz",
            "unit": UNIT, "steps": steps, **res, "fp32_fused_over_fp64_plain": res["fp32_fused"] / res["fp64_plain"]}


def batched_compare(local: int, steps: int, warmup: int, solo_steps: int = 8):
    """The batched sweep: 64 seeded 3-D scenes (64^3..256^3 inner cells + 8-cell CPML, random
    sphere/cube scatterer, TFSF Gaussian, FP32) stepped as one batch (tile
    rows and launch form -- one launch of the one-sweep kernel per step, or
    one persistent launch per chunk of steps -- autotuned on the warm-up
    steps, CUDA-graph replay), device-timed; next to the same scenes stepped
    one after another through their own handles (each a separate launch
    sequence)."""
    import xfdtd_cuda_b200 as X
    from xfdtd_cuda_b200 import configs
    sims = configs.batched_sweep()
    # one scene at a time: device time of solo_steps steps per scene, summed
    solo_ms, cells = 0.0, 0
    for s in sims:
        sc, keep = s.lower()
        h = X.Handle(sc, keep)
        h.set_device(local)
        h.init(solo_steps + 2)
        h.step(2)
        solo_ms += h.timed_step(solo_steps)
        gi = h.info()
        cells += gi.nx * gi.ny * gi.nz
        h.close()
    hs = []
    for s in sims:
        sc, keep = s.lower()
        h = X.Handle(sc, keep)
        h.set_device(local)
        hs.append(h)
    b = X.Batch(hs)
    b.init(warmup + steps)
    b.step(warmup)
    b.sync()
    ms = b.timed_step(steps)
    info = b.info()
    b.close()
    for h in hs:
        h.close()
    return {"workload": "batched sweep: 64 scenes, inner sides U{64..256} (seed 4) + 8-cell CPML, random sphere/cube "
                        "scatterer (eps_r 1..10, sigma 0..0.1 S/m), TFSF Gaussian, FP32",
            "unit": UNIT, "cells_per_step": cells, "steps": steps, "value": cells * steps / (ms / 1e3) / 1e6,
            "ms_per_step": ms / steps, "tile_rows": info["tile_rows"], "launch": info["launch"],
            "work_items_per_step": info["work_items"],
            "one_at_a_time": {"value": cells * solo_steps / (solo_ms / 1e3) / 1e6, "steps": solo_steps,
                              "ms_per_step": solo_ms / solo_steps}}


def cylinder2d_compare(local: int, steps: int = 4000):
    """The 2-D cylinder: TMz PEC cylinder (r = 50 cells) in 1024^2 cells + 10-cell CPML
    (1044^2), TFSF Gaussian, 4000 steps, in FP32 and FP64 on the temporally
    blocked kernel (9 steps per launch), and FP32 with one launch per step;
    device-timed Mcell-updates/s of each and the relative L2 error of the
    FP32 probe series against the FP64 run (the FP64 engine is bit-identical
    to the CPU restatement of the reference)."""
    import numpy as np
    import xfdtd_cuda_b200 as X
    from xfdtd_cuda_b200 import configs
    out, series = {"workload": "2-D TMz PEC cylinder, 1044^2 cells (1024^2 + 10-cell CPML), TFSF, 8 probes, "
                               f"{steps} steps", "unit": UNIT}, {}
    for key, prec, tb in (("fp32", "fp32", 9), ("fp64", "fp64", 9), ("fp32_one_launch_per_step", "fp32", 0)):
        sim = configs.cylinder_2d(precision=prec)
        sc, keep = sim.lower()
        h = X.Handle(sc, keep)
        h.set_device(local)
        h.set_temporal_block(tb)
        h.init(steps)
        ms = h.timed_step(steps)
        gi = h.info()
        cells = gi.nx * gi.ny
        series[key] = np.concatenate([h.read_probe(p) for p in range(len(h.probe_desc))])
        out[key] = {"value": cells * steps / (ms / 1e3) / 1e6, "ms_per_step": ms / steps,
                    "launches_per_step": gi.launches_per_step if tb == 0 else 1.0 / tb,
                    "steps_per_launch": tb or 1}
        h.close()
    out["fp32_probe_rel_l2_vs_fp64"] = float(np.linalg.norm(series["fp32"] - series["fp64"]) /
                                             np.linalg.norm(series["fp64"]))
    return out


def learned_abc_compare(local: int, steps: int, warmup: int, side: int = 768):
    """The learned boundary: a side^3 FP32 scattering domain whose walls use the learned
    absorbing boundary (shipped weights) against the same interior wrapped in
    a 12-cell CPML ((side+24)^3) and in a 3-cell CPML ((side+6)^3, the depth
    of the learned stencil), device-timed, with k_labc_apply's share of the
    learned step; and the probe error of the learned boundary, of the plain
    Mur boundary, of bare PEC walls and of the 3-cell CPML against the 12-cell
    CPML judge on a 48^3 validation scene."""
    import xfdtd_cuda_b200 as X
    from xfdtd_cuda_b200 import _lib as L
    from xfdtd_cuda_b200 import labc
    w = labc.shipped_weights()
    out = {"workload": f"scatterer in {side}^3 FP32, learned 3-cell boundary vs 12-cell CPML ({side + 24}^3) and "
                       f"3-cell CPML ({side + 6}^3)", "unit": UNIT}
    for mode in ("learned", "cpml", "cpml3"):
        thick = {"cpml": 12, "cpml3": 3}.get(mode, 0)
        sim = labc.scatter_scene(5, interior=side, pml=thick, dl=1e-3, inset=64)
        sc, keep = sim.lower()
        h = X.Handle(sc, keep)
        h.set_device(local)
        h.set_kernel_path(L.PATH_FUSED)
        h.init(warmup + steps + 3)
        if mode == "learned":
            h.set_learned_abc(w)
        h.step(warmup)
        h.sync()
        ms = h.timed_step(steps)
        gi = h.info()
        cells = gi.nx * gi.ny * gi.nz
        out[mode] = {"cells": cells, "value": cells * steps / (ms / 1e3) / 1e6, "ms_per_step": ms / steps,
                     "interior_cell_updates_per_s": side ** 3 * steps / (ms / 1e3) / 1e6}
        if mode == "learned":  # k_labc_apply's share of the step (launches bracketed by events)
            kms, kcnt = h.profile_kernels(3)
            out[mode]["k_labc_apply_share"] = kms[L.K_CORRECT] / sum(kms)
        h.close()
    out["probe_error_vs_cpml"] = labc.reflection_errors(w, seed=10, interior=48, steps=300, device=local,
                                                        modes=("pec", "mur", "learned", "cpml3"))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--cells", type=int, default=384)
    ap.add_argument("--precision", choices=["fp32", "fp64"], default="fp32")
    ap.add_argument("--profile-steps", type=int, default=6)
    ap.add_argument("--ref-cells", type=int, default=128)
    ap.add_argument("--cpu-steps", type=int, default=50)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--path", choices=["auto", "split", "fused", "plain"], default="auto")
    ap.add_argument("--scene", choices=["dispersive", "vacuum", "pml", "tfsf", "nf2ff"], default="dispersive")
    ap.add_argument("--tile-rows", type=int, default=16)
    ap.add_argument("--no-plain", action="store_true", help="skip the FP64 plain-form comparison")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched 64-scene leg")
    ap.add_argument("--no-labc", action="store_true", help="skip the learned-boundary leg")
    ap.add_argument("--no-2d", action="store_true", help="skip the 2-D cylinder leg")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the full-size FP32-vs-FP64 accuracy leg")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        # host-side CPU run: rank 0 alone works and prints, the others exit at
        # once; no rank takes a collective step, so no process group is needed
        return run_reference(args, rank, world)
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        dist = (torch, tdist)

    import xfdtd_cuda_b200 as X
    from xfdtd_cuda_b200 import _lib as L

    sim = build_scene(args.cells, args.precision, args.scene)
    sc, keep = sim.lower()
    h = X.Handle(sc, keep)
    h.set_device(local)
    path = {"auto": L.PATH_AUTO, "split": L.PATH_SPLIT, "fused": L.PATH_FUSED, "plain": L.PATH_PLAIN}[args.path]
    h.set_kernel_path(path)
    h.set_launch_hint((1, 1, 1), (32, args.tile_rows, 1))
    total = args.warmup + args.steps + args.profile_steps
    h.init(total)
    gi = h.info()
    gi._pml = [sc.pml.cells[q] for q in range(6)]
    cells = gi.nx * gi.ny * gi.nz

    h.step(args.warmup)
    h.sync()

    def barrier():
        if dist:
            dist[1].barrier()

    barrier()
    with ClockSampler(local) as clk:
        ms = h.timed_step(args.steps)
    barrier()
    ms = max_over_ranks(ms, dist)
    value = job_rate(cells, args.steps, world, ms)

    # per-kernel device time (launches bracketed by events, no graph)
    kms, kcnt = h.profile_kernels(args.profile_steps)
    tot = sum(kms)
    kernels = {L.KERNEL_NAMES[q]: {"launches": kcnt[q], "ms_per_launch": kms[q] / kcnt[q], "share": kms[q] / tot}
               for q in range(L.K_COUNT) if kcnt[q]}
    # roofline of the costliest kernel class that has a byte model
    modelled = [q for q in range(L.K_COUNT) if kcnt[q] and algorithmic_bytes(gi, q, args.precision)]
    dom = max(modelled or [max(range(L.K_COUNT), key=lambda q: kms[q])], key=lambda q: kms[q])
    peak, peak_kind = peaks()
    alg = algorithmic_bytes(gi, dom, args.precision) or 0.0
    launch_ms = kms[dom] / kcnt[dom]
    achieved = alg / (launch_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "kernel": L.KERNEL_NAMES[dom], "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": alg}
    traffic_file = ROOT / "profiles" / "traffic.txt"
    if traffic_file.exists():
        for line in traffic_file.read_text().splitlines():
            parts = line.split()
            if len(parts) == 3 and parts[0] == "traffic_bytes_per_cell" and parts[1] == L.KERNEL_NAMES[dom].split()[0]:
                roofline["traffic"] = float(parts[2]) * cells
    step_bytes = cells * (12 * esize(args.precision) + 1)
    step_roof = {"bytes_per_cell": 12 * esize(args.precision) + 1, "achieved": step_bytes / (ms / args.steps / 1e3) / 1e9,
                 "peak": peak, "unit": "GB/s"}
    step_roof["frac"] = step_roof["achieved"] / peak
    launches = gi.launches_per_step * args.steps + (args.steps + 63) // 64

    e2e = None
    if not args.no_e2e:
        barrier()
        t0 = time.perf_counter()
        hd = X.SimulationHD(sim)  # the reference's run(n) flow
        hd.setDevice(local)
        hd.kernel_path = path
        hd.setGridDim((1, 1, 1))
        hd.setBlockDim((32, args.tile_rows, 1))
        hd.init(args.steps)  # host scene compile, host result arrays (faulted in by host threads), device state
        t1 = time.perf_counter()
        hd.handle.step(args.steps)
        hd.handle.sync()
        t2 = time.perf_counter()
        hd.copyDeviceToHost()  # six fields into sim.emf (float64), NF2FF currents
        t3 = time.perf_counter()
        wall = max_over_ranks(t3 - t0, dist)
        gi2 = hd.handle.info()  # bytes the library copied each way (its own counters)
        parts = {"compile": hd.timings["compile"], "init": t1 - t0 - hd.timings["compile"], "step": t2 - t1,
                 "read_back": t3 - t2}
        e2e = {"value": job_rate(cells, args.steps, world, wall * 1e3), "unit": UNIT,
               "h2d_bytes_per_step": gi2.h2d_bytes / args.steps, "d2h_bytes_per_step": gi2.d2h_bytes / args.steps,
               "seconds": {**parts, "wall": t3 - t0},
               "path": "SimulationHD(sim).run(n) flow: init (host compile, host result arrays, device state and "
                       "uploads) + n steps (host threads fault in the result arrays during init and steps) + "
                       "copyDeviceToHost (six fields as float64 into sim.emf, NF2FF currents), wall clock; bytes "
                       "counted by the library"}
        hd.releaseDevice()
        sim.emf = None

    h.close()
    plain = None
    if not args.no_plain and world == 1:
        plain = plain_compare(local, 50, 3)
    batched = None
    if not args.no_batch and world == 1:
        try:
            batched = batched_compare(local, 30, 16)
        except Exception as exc:  # reported, not fatal for the headline
            batched = {"error": str(exc)}
    cyl2d = None
    if not args.no_2d and world == 1:
        try:
            cyl2d = cylinder2d_compare(local)
        except Exception as exc:
            cyl2d = {"error": str(exc)}
    learned = None
    if not args.no_labc and world == 1:
        try:
            learned = learned_abc_compare(local, 20, 3)
        except Exception as exc:
            learned = {"error": str(exc)}

    accuracy = None
    if not args.no_accuracy and world == 1:
        try:
            from xfdtd_cuda_b200 import accuracy as A
            accuracy = {"what": "relative L2 of the FP32 one-sweep engine against the FP64 engine (bit-identical "
                                "to the CPU restatement) at full size, per output",
                        "dielectric_sphere_156cube_2400_steps": A.fp32_vs_fp64("dielectric", 2400, local),
                        "dispersive_sphere_408cube_6000_steps": A.fp32_vs_fp64("dispersive", 6000, local),
                        "coefficient_storage_trial": {
                            "what": "dielectric sphere (156^3, 2400 steps) with the FP32 engine's coefficient LUT rounded to 16 bits",
                            "fp16": A.fp32_vs_fp64("dielectric", 2400, local, fields=False, coeff_storage=1),
                            "bf16": A.fp32_vs_fp64("dielectric", 2400, local, fields=False, coeff_storage=2)}}
        except Exception as exc:
            accuracy = {"error": str(exc)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_sample(args.ref_cells, args.cpu_steps)
        one = cpu_sample(args.ref_cells // 2, max(10, args.cpu_steps // 5), threads=1)
        cpu["one_core"] = {"value": one["value"], "sample": one["sample"]}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic",
               "config": {"workload": workload_label(args.scene, gi, args.cells),
                          "cells_per_step": cells, "parallelism": f"scene-replica x{world}" if world > 1 else "1 GPU",
                          "l2": "resident state 3.3 GB >> 126 MB L2 (no flush needed)"},
               "e2e": e2e, "roofline": roofline, "step_roofline": step_roof, "cpu_baseline": cpu,
               "clocks": clk.summary(), "gpu_launches": launches, "kernels": kernels, "vs_fp64_plain": plain,
               "batched": batched, "learned_abc": learned, "cylinder_2d": cyl2d, "accuracy": accuracy}
        print(json.dumps(out))
    if dist:
        dist[1].barrier()
        dist[1].destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
