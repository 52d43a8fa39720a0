"""Independent anchors from tests/golden/ (made by tests/golden/make_golden.py).

* mie_sphere.npz: the analytic Mie radar cross-section of the eps_r = 3,
  mu_r = 2 sphere of radius 5 cm at 1 GHz.  The oracle's far field (and, on
  a GPU, the engine's, through xfb_far_field) normalised by the spectrum of
  the unit Gaussian pulse must follow it in the E-plane and H-plane cuts:
  sigma = 4 pi |r E_far|^2 / |G(f)|^2.  The tolerance (rel-L2 3 %) covers the
  staircased sphere (20 cells per radius) and the finite run.
* mie_dispersive.npz: the same for the dispersive sphere of the benchmark
  workload (radius 0.1 m, Drude + Lorentz ADE) at 1, 3 and 5 GHz, which the
  FP32 engine at full size (408^3, 6000 steps) must follow.
* oracle_small.npz: probes, field sums and one NF2FF current plane of the
  oracle on a small FP64 sphere; pins the CPU restatement against drift.
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest

import xfdtd_cuda_b200 as X
from xfdtd_cuda_b200 import configs
from helpers import engine, oracle_of
from oracle import far_field_numpy

GOLD = Path(__file__).resolve().parent / "golden"
MIE_TOL = 0.03


def mie_scene(precision="fp64", cells=60, dl=2.5e-3):
    g = np.load(GOLD / "mie_sphere.npz")
    return configs.dielectric_sphere(cells=cells, dl=dl, pml=8, precision=precision, tfsf_inset=4, nf2ff_inset=2,
                                     freqs=(float(g["freq"]),), radius=float(g["radius"]))


def rcs_cuts(far, dl, f=None, sc=None):
    """sigma / lambda^2 in the E-plane (x-z) and H-plane (x-y) cuts at the
    scattering angles sc (default: the dielectric fixture's) at frequency f;
    far(theta, phi) -> (E_theta, E_phi)."""
    g = np.load(GOLD / "mie_sphere.npz")
    f = float(g["freq"]) if f is None else float(f)
    sc = g["theta"] if sc is None else sc
    tau = 20 * dl / 6e8  # the scene's Gaussian exp(-((t - t0) / tau)^2)
    spec = tau * math.sqrt(math.pi) * math.exp(-((math.pi * f * tau) ** 2))
    lam = 299792458.0 / f
    out = []
    for th, ph in ((math.pi / 2 - sc, np.zeros_like(sc)), (np.full_like(sc, math.pi / 2), sc)):
        et, ep = far(th, ph)
        out.append(4 * math.pi * (np.abs(et) ** 2 + np.abs(ep) ** 2) / spec ** 2 / lam ** 2)
    return out, (g["sigma_e"], g["sigma_h"])


# the dispersive sphere of the benchmark workload against its Mie series
# (mie_dispersive.npz): 100 cells per radius, 6000 steps.  Measured on the
# FP32 engine: 3.4 % (1 GHz, eps = -6.8 - 1.6j), 0.6 % (3 GHz, eps = 3.2 -
# 0.17j), 9.9 % (5 GHz, next to the Lorentz pole at 4.8 GHz: eps = -17.7 -
# 6.6j, where the field hugs the staircased surface and the discrete
# permittivity departs most from the model); rel-L2 bars per frequency:
DISP_TOL = {1e9: 0.05, 3e9: 0.02, 5e9: 0.15}


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_oracle_follows_mie():
    sim = mie_scene()
    n = 1000
    o = oracle_of(sim, n)
    o.run(n)
    sc, keep = sim.lower()
    gi = X.Handle(sc, keep).info()
    cur = [[o.nf2ff(0, face, w) for w in range(4)] for face in range(6)]
    f = sim.nf2ff_list[0].freqs[0]
    (se, sh), (me, mh) = rcs_cuts(
        lambda th, ph: far_field_numpy(cur, list(gi.nf2ff_box), list(gi.origin), (gi.dx, gi.dy, gi.dz), f, th, ph),
        2.5e-3)
    assert rel(se, me) <= MIE_TOL
    assert rel(sh, mh) <= MIE_TOL


def test_oracle_matches_fixture():
    g = np.load(GOLD / "oracle_small.npz")
    sim = configs.dielectric_sphere(cells=20, dl=5e-3, pml=4, precision="fp64", tfsf_inset=3, nf2ff_inset=2,
                                    freqs=(2e9,), radius=0.02,
                                    probes=[((0.0, 0.0, 0.0), 2), ((0.03, -0.02, 0.01), 1), ((-0.04, 0.03, 0.0), 5)])
    n = int(g["steps"])
    o = oracle_of(sim, n)
    o.run(n)
    probes = np.stack([o.probe(p) for p in range(3)])
    np.testing.assert_allclose(probes, g["probes"], rtol=1e-12, atol=1e-12 * np.abs(g["probes"]).max())
    fields = [o.field(f) for f in range(6)]
    np.testing.assert_allclose([f.sum() for f in fields], g["field_sum"], rtol=1e-10,
                               atol=1e-12 * np.abs(g["field_abs"]).max())
    np.testing.assert_allclose([np.abs(f).sum() for f in fields], g["field_abs"], rtol=1e-12)
    np.testing.assert_allclose(o.nf2ff(0, 1, 0), g["nf2ff_xp_ja"], rtol=1e-12,
                               atol=1e-12 * np.abs(g["nf2ff_xp_ja"]).max())


@pytest.mark.gpu
@pytest.mark.parametrize("precision,path", [("fp64", 2), ("fp32", 2), ("fp64", 3), ("fp32", 1)])
def test_engine_follows_mie(precision, path):
    sim = mie_scene(precision)
    n = 1000
    h = engine(sim, n, path=path)
    h.step(n)
    h.sync()
    (se, sh), (me, mh) = rcs_cuts(lambda th, ph: h.far_field(0, th, ph), 2.5e-3)
    assert rel(se, me) <= MIE_TOL
    assert rel(sh, mh) <= MIE_TOL


@pytest.mark.gpu
def test_engine_mie_refined():
    # the same sphere at 1.25 mm (40 cells per radius), FP32 one-sweep path
    sim = mie_scene("fp32", cells=120, dl=1.25e-3)
    n = 2000
    h = engine(sim, n, path=2)
    h.step(n)
    h.sync()
    (se, sh), (me, mh) = rcs_cuts(lambda th, ph: h.far_field(0, th, ph), 1.25e-3)
    assert rel(se, me) <= MIE_TOL
    assert rel(sh, mh) <= MIE_TOL


@pytest.mark.gpu
def test_engine_follows_dispersive_mie():
    g = np.load(GOLD / "mie_dispersive.npz")
    sim = configs.dispersive_sphere(precision="fp32")
    n = 6000
    h = engine(sim, n, path=2)
    h.step(n)
    h.sync()
    errs = []
    for q, f in enumerate(g["freqs"]):
        (se, sh), _ = rcs_cuts(lambda th, ph: h.far_field(q, th, ph), 1e-3, f, g["theta"])
        errs.append((float(f), rel(se, g["sigma_e"][q]), rel(sh, g["sigma_h"][q])))
    print("dispersive Mie rel-L2 (f, E-plane, H-plane):", errs)
    for f, ee, eh in errs:
        assert ee <= DISP_TOL[f] and eh <= DISP_TOL[f], (f, ee, eh)
