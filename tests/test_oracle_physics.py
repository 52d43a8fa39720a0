"""Known-answer tests that pin the CPU restatement (the parity oracle).

The reference ships no golden vectors, so the oracle is anchored by physics
with closed-form answers:
  * TFSF: for axis-aligned incidence the 1-D auxiliary grid and the 3-D Yee
    grid share their numerical dispersion, so the scattered-field region stays
    at round-off and the total field equals the auxiliary solution exactly;
  * TMz/3-D PEC cavities ring at their analytic resonances (up to the known
    Yee dispersion at ~10 cells per wavelength);
  * the CPML reflects less than -40 dB of a scattered pulse;
  * a lossless PEC cavity keeps its energy bounded (the leapfrog is stable).
"""
import math

import numpy as np
import pytest

import xfdtd_cuda_b200 as X
from xfdtd_cuda_b200 import configs
from helpers import oracle_of


def vacuum_tfsf_3d(theta=math.pi / 2, phi=0.0, cells=24, dl=5e-3):
    s = configs.dielectric_sphere(cells=cells, dl=dl, pml=6, tfsf_inset=4, nf2ff_inset=2, radius=0.001, freqs=())
    s.objects = s.objects[:1]  # vacuum only
    s.sources[0].theta, s.sources[0].phi = theta, phi
    return s


def sf_tf_ratio(o, box, f=2, margin=2):
    e = o.field(f)
    is_, ie, js, je, ks, ke = box
    tf = np.abs(e[is_ + 1:ie, js + 1:je, ks + 1:ke]).max()
    mask = np.ones(e.shape, bool)
    mask[is_ - margin:ie + margin + 1, js - margin:je + margin + 1, ks - margin:ke + margin + 1] = False
    return np.abs(e[mask]).max() / tf, tf


def test_tfsf_axis_aligned_no_leakage_3d():
    s = vacuum_tfsf_3d()
    o = oracle_of(s, 110)
    o.run(110)
    ratio, tf = sf_tf_ratio(o, list(o.view.tfsf_box))
    assert tf > 0.5
    assert ratio < 1e-12


def test_tfsf_oblique_leakage_small():
    s = vacuum_tfsf_3d(theta=1.1, phi=0.6, cells=28)
    o = oracle_of(s, 120)
    o.run(120)
    e = {f: o.field(f) for f in range(3)}
    b = list(o.view.tfsf_box)
    tf = max(np.abs(e[f][b[0] + 2:b[1] - 1, b[2] + 2:b[3] - 1, b[4] + 2:b[5] - 1]).max() for f in range(3))
    sf = 0.0
    for f in range(3):
        m = np.ones(e[f].shape, bool)
        m[b[0] - 2:b[1] + 3, b[2] - 2:b[3] + 3, b[4] - 2:b[5] + 3] = False
        sf = max(sf, np.abs(e[f][m]).max())
    assert tf > 0.3
    assert sf / tf < 3e-2  # linear interpolation of the incident field: about -35 dB


def test_total_field_equals_auxiliary_solution():
    n = 100
    s = vacuum_tfsf_3d()
    o = oracle_of(s, n)
    o.run(n - 1)  # fields are E^{n-1}; incident row n-1 is E_aux at (n-1) dt
    e_inc, h_inc = o.incident_tables()
    b = list(o.view.tfsf_box)
    ez = o.field(2)
    tre = o.view.tfsf_transform_e[2]
    j, k = (b[2] + b[3]) // 2, (b[4] + b[5]) // 2
    got = ez[b[0] + 1:b[1], j, k]
    want = tre * e_inc[n - 1, np.arange(b[0] + 1, b[1]) - b[0] + 2]
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    assert np.abs(want).max() > 0.5


def test_tfsf_axis_aligned_no_leakage_2d():
    s = configs.cylinder_2d(cells=80, dl=1e-3, pml=8, precision="fp64", radius=1e-9, tfsf_inset=10, n_probes=0)
    s.objects = s.objects[:1]
    o = oracle_of(s, 150)
    o.run(150)
    ez = o.field(2)[:, :, 0]
    b = list(o.view.tfsf_box)
    tf = np.abs(ez[b[0] + 1:b[1], b[2] + 1:b[3]]).max()
    mask = np.ones(ez.shape, bool)
    mask[b[0] - 1:b[1] + 2, b[2] - 1:b[3] + 2] = False
    assert tf > 0.5 and np.abs(ez[mask]).max() / tf < 1e-12


def test_pec_cavity_resonance_3d():
    a, bb, c, dl = 0.06, 0.04, 0.03, 2e-3
    s = X.Simulation(dl, dl, dl, 0.95)
    s.addObject(X.Object("domain", X.Cube(X.Vector(0, 0, 0), X.Vector(a, bb, c)), X.Material.createAir()))
    n = 3000
    o = oracle_of(s, n)
    rng = np.random.default_rng(3)
    ey = rng.standard_normal(o.shape(1)) * 0.0
    ny, nz = o.shape(1)[1], o.shape(1)[2]
    # seed the TE101-like mode (Ey ~ sin(pi x/a) sin(pi z/c))
    xs = np.arange(o.shape(1)[0]) * dl
    zs = np.arange(nz) * dl
    ey[:] = np.sin(np.pi * xs / a)[:, None, None] * np.sin(np.pi * zs / c)[None, None, :] + 0.1 * rng.standard_normal(ey.shape)
    o.set_field(1, ey)
    series = []
    for _ in range(n // 10):
        o.run(10)
        series.append(o.field(1)[15, 10, 7])
    dt = o.view.dt * 10
    spec = np.abs(np.fft.rfft(np.array(series) * np.hanning(len(series)), 8 * len(series)))
    freqs = np.fft.rfftfreq(8 * len(series), dt)
    f_peak = freqs[np.argmax(spec[1:]) + 1]
    f_101 = X.C_0 / 2 * math.sqrt((1 / a) ** 2 + (1 / c) ** 2)
    assert abs(f_peak - f_101) / f_101 < 0.01


def test_lossless_cavity_energy_bounded():
    s = X.Simulation(2e-3, 2e-3, 2e-3, 0.9)
    s.addObject(X.Object("domain", X.Cube(X.Vector(0, 0, 0), X.Vector(0.03, 0.024, 0.02)), X.Material.createAir()))
    o = oracle_of(s, 600)
    rng = np.random.default_rng(5)
    nx, ny, nz = o.view.nx, o.view.ny, o.view.nz
    # random values only where the update acts (tangential E on the PEC walls
    # must be zero, otherwise it is a static source that pumps H linearly)
    upd = {0: (slice(0, nx), slice(1, ny), slice(1, nz)), 1: (slice(1, nx), slice(0, ny), slice(1, nz)),
           2: (slice(1, nx), slice(1, ny), slice(0, nz))}
    for f in range(6):
        v = np.zeros(o.shape(f))
        sl = upd[f] if f < 3 else (slice(0, nx), slice(0, ny), slice(0, nz))
        v[sl] = rng.standard_normal(v[sl].shape)
        o.set_field(f, v)
    energies = []
    for _ in range(30):
        o.run(20)
        en = sum(X.EPSILON_0 * (o.field(f) ** 2).sum() for f in range(3)) + \
            sum(X.MU_0 * (o.field(f) ** 2).sum() for f in range(3, 6))
        energies.append(en)
    energies = np.array(energies)
    assert np.isfinite(energies).all()
    assert energies.max() / energies.min() < 1.5


def _cpml_probe(cells, inset, n):
    s = configs.cylinder_2d(cells=cells, dl=1e-3, pml=10, precision="fp64", radius=0.01, tfsf_inset=inset, n_probes=0)
    s.addMonitor(X.PointMonitor(X.Vector(0.0, 0.042, 0.0), X.EMF.Field.EZ))
    s.addMonitor(X.PointMonitor(X.Vector(-0.042, 0.0, 0.0), X.EMF.Field.EZ))
    o = oracle_of(s, n)
    o.run(n)
    return o.probe(0), o.probe(1)


def test_cpml_reflection_below_minus_40db():
    n = 320
    small = _cpml_probe(100, 15, n)    # TF box 70 cells, probes 7 cells outside it, 8 from the CPML
    big = _cpml_probe(300, 115, n)     # same box and probes, CPML 108 cells away
    for a, b in zip(small, big):
        assert np.abs(b).max() > 1e-3
        assert np.abs(a - b).max() / np.abs(b).max() < 1e-2
