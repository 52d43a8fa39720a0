"""FP32 engine against the FP64 engine on the same scene, output by output.

The FP64 one-sweep engine reproduces the CPU restatement of the reference
bit for bit (FP64 unit compiled without contraction, reference operation
order), so it stands in for the FP64 oracle at sizes the CPU cannot run in a
test.  For each output of a run this reports the relative L2 error of the FP32
run against the FP64 run:

* probes: every probe series (seeded points in the total- and scattered-field
  regions), concatenated, and the worst single probe;
* far field: E_theta and E_phi of the xz (phi = 0) and yz (phi = pi/2) cuts at
  360 angles from -pi to pi, per NF2FF frequency, as the reference's sphere
  tests request them (test/dielectric_sphere_scatter.cu:85-91,
  test/dispersive_sphere_scatter/dispersive_sphere_scatter.cuh:113-124);
* final fields: each of the six components after the last step, relative
  and (largest difference, largest value) absolute.
"""
from __future__ import annotations

import math

import numpy as np

from . import configs
from .simulation import EMF, Handle


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    dt = complex if (np.iscomplexobj(a) or np.iscomplexobj(b)) else np.float64
    a = a.astype(dt, copy=False).ravel()
    b = b.astype(dt, copy=False).ravel()
    den = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def seeded_probes(half_side: float, n: int = 8, seed: int = 3):
    """n probe points (seeded) spread over the inner domain, alternating Ez and Ex."""
    rng = np.random.default_rng(seed)
    pts = []
    for q in range(n):
        p = rng.uniform(-0.9 * half_side, 0.9 * half_side, size=3)
        pts.append(((float(p[0]), float(p[1]), float(p[2])), EMF.Field.EZ if q % 2 == 0 else EMF.Field.EX))
    return pts


def scene(name: str, precision: str, cells: int | None = None):
    """The dielectric sphere (140^3 + 8-cell CPML, 1 GHz) or the dispersive
    sphere (384^3 + 12-cell CPML, 1/3/5 GHz) workload with seeded probes."""
    if name == "dielectric":
        c = cells or 140
        return configs.dielectric_sphere(cells=c, precision=precision, probes=seeded_probes(c * 2.5e-3 / 2))
    c = cells or 384
    return configs.dispersive_sphere(cells=c, precision=precision, probes=seeded_probes(c * 1e-3 / 2))


def run_outputs(sim, steps: int, device: int = 0, fields: bool = True, coeff_storage: int = 0):
    """Run `steps` steps and collect probes, far-field cuts and final fields."""
    sc, keep = sim.lower()
    h = Handle(sc, keep)
    h.set_device(device)
    if coeff_storage:
        h.set_coeff_storage(coeff_storage)
    h.init(steps)
    h.step(steps)
    h.sync()
    gi = h.info()
    out = {"probes": [h.read_probe(p) for p in range(len(h.probe_desc))], "far": {}, "fields": {}}
    theta = np.linspace(-math.pi, math.pi, 360)
    for f in range(gi.n_freqs):
        for cut, phi in (("xz", 0.0), ("yz", math.pi / 2)):
            eth, eph = h.far_field(f, theta, np.full_like(theta, phi))
            out["far"][(f, cut)] = np.concatenate([eth, eph])
    if fields:
        for q in range(6):
            out["fields"][q] = h.read_field(q).astype(np.float32 if sim.precision == "fp32" else np.float64)
    h.close()
    return out


def fp32_vs_fp64(name: str, steps: int, device: int = 0, cells: int | None = None, fields: bool = True,
                 coeff_storage: int = 0):
    """Relative L2 error of every output of the FP32 run (its coefficient LUT
    optionally rounded to FP16 / BF16, the storage trial) against the FP64 run."""
    r32 = run_outputs(scene(name, "fp32", cells), steps, device, fields, coeff_storage)
    r64 = run_outputs(scene(name, "fp64", cells), steps, device, fields)
    per_probe = [rel_l2(a, b) for a, b in zip(r32["probes"], r64["probes"])]
    res = {
        "steps": steps,
        "probes": rel_l2(np.concatenate(r32["probes"]), np.concatenate(r64["probes"])),
        "probe_worst": max(per_probe) if per_probe else None,
        "far_field": {f"{k[1]}@f{k[0]}": rel_l2(r32["far"][k], r64["far"][k]) for k in r64["far"]},
    }
    if fields:
        names = ["exeyezhxhyhz"[2 * q:2 * q + 2] for q in range(6)]
        res["fields"] = {names[q]: rel_l2(r32["fields"][q], r64["fields"][q]) for q in range(6)}
        # the same differences on an absolute scale: largest |FP32 - FP64| and
        # largest |FP64| of each final component (the incident pulse has
        # amplitude 1 in E, 1 / 377 in H)
        res["fields_max_abs_error"] = {names[q]: float(np.abs(r32["fields"][q].astype(np.float64) - r64["fields"][q]).max())
                                       for q in range(6)}
        res["fields_max_abs"] = {names[q]: float(np.abs(r64["fields"][q]).max()) for q in range(6)}
    res["far_field_worst"] = max(res["far_field"].values()) if res["far_field"] else None
    return res
