"""Standard scenes: the benchmark workloads and their scaled-down test twins.

Each builder returns a ``Simulation``; ``cells`` scales the inner domain while
keeping the physics (materials, source, boundary, NF2FF) of the workload.

* ``dielectric_sphere``  -- 3-D FP64 dielectric sphere scatter: 0.35 m cube,
  dl = 2.5 mm (140^3) + 8-cell CPML, sphere r = 0.1 m, eps_r = 3, mu_r = 2,
  TFSF 15 cells inset, x-propagating Gaussian tau = 20 dl / 6e8, t0 = 4.5 tau,
  Courant 0.9, 2400 steps, NF2FF at 1 GHz 11 cells inset
  (the scene of the reference's test/dielectric_sphere_scatter.cu).
* ``cylinder_2d``        -- 2-D TMz PEC cylinder: 1024^2 cells, dl = 1 mm,
  10-cell CPML, r = 0.05 m, TFSF Gaussian, 4000 steps, seeded probes
  (test/cylinder_scatter_2d.cu with the sizes of the 2-D benchmark).
* ``dispersive_sphere``  -- 3-D FP32 sphere of Drude (wp = 2e10, gamma = 1e9)
  + Lorentz (d_eps = 2, w0 = 3e10, delta = 5e8) medium, eps_inf = 1: 384^3,
  dl = 1 mm, 12-cell CPML, TFSF Gaussian, NF2FF at 1/3/5 GHz in FP64,
  6000 steps (test/dispersive_sphere_scatter/*).
"""
from __future__ import annotations

import math

import numpy as np

from .simulation import (PML, TFSF2D, TFSF3D, Cube, Cylinder, DispersiveMaterial, DrudePole, ElectroMagneticProperty,
                         LorentzPole, Material, NFFFTFrequencyDomain, Object, PointMonitor, Simulation, Sphere,
                         Vector, Waveform)


def _gaussian(dl):
    tau = 20 * dl / 6e8
    return Waveform.gaussian(tau, 4.5 * tau)


def dielectric_sphere(cells: int = 140, dl: float = 2.5e-3, pml: int = 8, precision: str = "fp64",
                      tfsf_inset: int = 15, nf2ff_inset: int = 11, freqs=(1e9,), radius: float | None = None,
                      probes=()):
    side = cells * dl
    s = Simulation(dl, dl, dl, 0.9, precision=precision)
    h = side / 2
    s.addObject(Object("domain", Cube(Vector(-h, -h, -h), Vector(side, side, side)), Material.createAir()))
    r = radius if radius is not None else 0.1 * cells / 140 * 2.5e-3 / dl
    s.addObject(Object("dielectric_sphere", Sphere(Vector(0, 0, 0), r),
                       Material("a", ElectroMagneticProperty(3, 2, 0, 0))))
    s.addWaveformSource(TFSF3D(tfsf_inset, tfsf_inset, tfsf_inset, math.pi / 2, 0, 0, _gaussian(dl)))
    for d in range(6):
        s.addBoundary(PML(pml, d))
    if freqs:
        s.addNF2FF(NFFFTFrequencyDomain(nf2ff_inset, nf2ff_inset, nf2ff_inset, list(freqs)))
    for p, f in probes:
        s.addMonitor(PointMonitor(Vector(*p), f))
    return s


def cylinder_2d(cells: int = 1024, dl: float = 1e-3, pml: int = 10, precision: str = "fp32", radius: float | None = None,
                tfsf_inset: int = 15, n_probes: int = 8, seed: int = 2):
    side = cells * dl
    s = Simulation(dl, dl, 1.0, 0.9, precision=precision)
    h = side / 2
    s.addObject(Object("domain", Cube(Vector(-h, -h, -math.inf), Vector(side, side, math.inf)), Material.createAir()))
    r = radius if radius is not None else 0.05 * cells / 1024 * 1e-3 / dl
    s.addObject(Object("cylinder", Cylinder(Vector(0, 0, 0), r, math.inf, 2), Material.createPec()))
    s.addWaveformSource(TFSF2D(tfsf_inset, tfsf_inset, 0.0, _gaussian(dl)))
    for d in range(4):
        s.addBoundary(PML(pml, d))
    rng = np.random.default_rng(seed)
    from .simulation import EMF
    for q in range(n_probes):
        x, y = rng.uniform(-0.45 * side, 0.45 * side, size=2)
        s.addMonitor(PointMonitor(Vector(float(x), float(y), 0.0), EMF.Field.EZ))
    return s


def dispersive_material():
    return DispersiveMaterial("drude_lorentz", 1.0, [DrudePole(2e10, 1e9), LorentzPole(2.0, 3e10, 5e8)])


def dispersive_sphere(cells: int = 384, dl: float = 1e-3, pml: int = 12, precision: str = "fp32",
                      freqs=(1e9, 3e9, 5e9), tfsf_inset: int = 15, nf2ff_inset: int = 11, radius: float | None = None,
                      material=None, probes=()):
    side = cells * dl
    s = Simulation(dl, dl, dl, 0.9, precision=precision)
    h = side / 2
    s.addObject(Object("domain", Cube(Vector(-h, -h, -h), Vector(side, side, side)), Material.createAir()))
    r = radius if radius is not None else 0.1 * cells / 384 * 1e-3 / dl
    s.addObject(Object("sphere", Sphere(Vector(0, 0, 0), r), material or dispersive_material()))
    s.addWaveformSource(TFSF3D(tfsf_inset, tfsf_inset, tfsf_inset, math.pi / 2, 0, 0, _gaussian(dl)))
    for d in range(6):
        s.addBoundary(PML(pml, d))
    if freqs:
        s.addNF2FF(NFFFTFrequencyDomain(nf2ff_inset, nf2ff_inset, nf2ff_inset, list(freqs)))
    for p, f in probes:
        s.addMonitor(PointMonitor(Vector(*p), f))
    return s


def batched_sweep(n: int = 64, seed: int = 4, lo: int = 64, hi: int = 256, pml: int = 8, dl: float = 1e-3,
                  precision: str = "fp32"):
    """Batched sweep: `n` 3-D scenes with inner sides drawn uniformly from [lo, hi] cells
    (seeded), each holding one random sphere or cube scatterer (eps_r in
    [1, 10], sigma in [0, 0.1] S/m) inside an 8-cell CPML, lit by a TFSF
    Gaussian pulse.  Returns the list of Simulation objects."""
    rng = np.random.default_rng(seed)
    sims = []
    for q in range(n):
        side_cells = int(rng.integers(lo, hi + 1))
        side = side_cells * dl
        s = Simulation(dl, dl, dl, 0.9, precision=precision)
        h = side / 2
        s.addObject(Object("domain", Cube(Vector(-h, -h, -h), Vector(side, side, side)), Material.createAir()))
        eps = float(rng.uniform(1, 10))
        sig = float(rng.uniform(0, 0.1))
        size = float(rng.uniform(0.15, 0.35)) * side
        c = [float(rng.uniform(-0.1, 0.1)) * side for _ in range(3)]
        mat = Material(f"m{q}", ElectroMagneticProperty(eps, 1.0, sig, 0.0))
        if rng.integers(2):
            shape = Sphere(Vector(*c), size / 2)
        else:
            shape = Cube(Vector(*(x - size / 2 for x in c)), Vector(size, size, size))
        s.addObject(Object(f"scatterer{q}", shape, mat))
        inset = max(3, side_cells // 16)
        s.addWaveformSource(TFSF3D(inset, inset, inset, float(rng.uniform(0, math.pi)), float(rng.uniform(0, 2 * math.pi)),
                                   float(rng.uniform(0, math.pi)), _gaussian(dl)))
        for d in range(6):
            s.addBoundary(PML(pml, d))
        sims.append(s)
    return sims
