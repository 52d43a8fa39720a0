"""Time-domain NF2FF (the reference's NFFFTTimeDomain path,
src/nf2ff/time_domain/nf2ff_time_domain_data.cu:113-175).

CPU: the oracle's time-domain far field, Fourier-transformed at a frequency,
agrees with its frequency-domain far field from the same surface (a physics
anchor of the restatement).  GPU: the engine's potentials against the
oracle's sequential sums (the engine sums the face points in a different,
fixed order: FP64 agreement to round-off, 1e-12 relative L2), the device far
field against numpy, and reproducibility across graph on/off and a
checkpoint round trip.
"""
import math

import numpy as np
import pytest

import xfdtd_cuda_b200 as X
from conftest import has_gpu, rel_l2
from oracle import OracleSim, far_field_numpy, far_field_td_numpy
from xfdtd_cuda_b200 import configs

TH, PH = math.pi / 3, math.pi / 4
F0 = 2e9


def _scene(precision="fp64", td=True, fd=True):
    sim = configs.dielectric_sphere(cells=20, dl=5e-3, pml=5, precision=precision, tfsf_inset=4, nf2ff_inset=2,
                                    radius=0.025, freqs=(F0,) if fd else ())
    if td:
        sim.addNF2FF(X.NFFFTTimeDomain(2, 2, 2, "", TH, PH))
    return sim


def _oracle(sim, n):
    sc, keep = sim.lower()
    o = OracleSim(X.Handle(sc, keep), n)
    o.run(n)
    return o


def test_td_far_field_of_oracle_matches_frequency_domain():
    n = 700
    sim = _scene()
    sc, keep = sim.lower()
    h = X.Handle(sc, keep)
    o = OracleSim(h, n)
    o.run(n)
    v = o.view
    pot = [o.nf2ff_td(w) for w in range(6)]
    et, ep = far_field_td_numpy(pot, TH, PH, v.dt)
    # the transform of the time signal at F0 (the bins are observation times n dt)
    w0 = 2 * np.pi * F0
    ph = np.exp(-1j * w0 * np.arange(len(et)) * v.dt) * v.dt
    ft, fp = np.sum(et * ph), np.sum(ep * ph)
    cur = [[o.nf2ff(0, face, w) for w in range(4)] for face in range(6)]
    gi = h.info()
    et_fd, ep_fd = far_field_numpy(cur, list(v.nf2ff_box), list(gi.origin), (v.dx, v.dy, v.dz), F0,
                                   np.array([TH]), np.array([PH]))
    # same surface, same direction: magnitudes agree (the time-domain form
    # differs by its first difference in time and linear bin weights)
    assert abs(abs(ft) - abs(et_fd[0])) <= 0.01 * abs(et_fd[0])
    assert abs(abs(fp) - abs(ep_fd[0])) <= 0.01 * abs(ep_fd[0])
    # the pulse has left the box: the last bins are empty
    assert np.abs(et[-20:]).max() <= 1e-3 * np.abs(et).max()


gpu = pytest.mark.gpu


@gpu
def test_td_potentials_match_oracle_fp64():
    n = 300
    sim = _scene()
    sc, keep = sim.lower()
    h = X.Handle(sc, keep)
    h.init(n)
    h.step(n)
    h.sync()
    o = _oracle(_scene(), n)
    for w in range(6):
        a, b = h.read_nf2ff_td(w), o.nf2ff_td(w)
        assert a.shape == b.shape
        assert rel_l2(a, b) <= 1e-12, (w, rel_l2(a, b))
    et, ep = h.far_field_td()
    rt, rp = far_field_td_numpy([o.nf2ff_td(w) for w in range(6)], TH, PH, h.info().dt)
    assert rel_l2(et, rt) <= 1e-12 and rel_l2(ep, rp) <= 1e-12
    # the frequency-domain currents of the same run stay bit-identical
    for face in range(6):
        for w in range(4):
            assert np.array_equal(h.read_nf2ff(0, face, w), o.nf2ff(0, face, w))
    h.close()


@gpu
def test_td_reproducible_graph_and_checkpoint():
    n = 200

    def run(graph, steps_per_graph, split=None):
        sc, keep = _scene().lower()
        h = X.Handle(sc, keep)
        h.set_graph(graph, steps_per_graph)
        h.init(n)
        if split is None:
            h.step(n)
        else:
            h.step(split)
            st = h.get_state()
            h.step(n - split)  # overwritten by the restore below
            h.set_state(st)
            h.step(n - split)
        h.sync()
        out = [h.read_nf2ff_td(w) for w in range(6)]
        h.close()
        return out

    ref = run(True, 64)
    for other in (run(False, 1), run(True, 7), run(True, 64, split=77)):
        for a, b in zip(ref, other):
            assert np.array_equal(a, b)


@gpu
def test_td_only_scene_and_simulation_hd_flow(tmp_path):
    sim = _scene(td=True, fd=False)
    nf = sim.nf2ff_list[0]
    nf.setOutputDir(str(tmp_path))
    hd = X.SimulationHD(sim)
    hd.setGridDim((1, 1, 1))
    hd.setBlockDim((32, 8, 1))
    hd.run(150)
    t, et, ep = nf.processFarField()
    assert len(t) == len(et) == len(ep) and np.isfinite(et).all()
    assert (tmp_path / "far_field_td.npy").exists()
    o = _oracle(_scene(td=True, fd=False), 150)
    for w in range(6):
        assert rel_l2(nf.potentials[w], o.nf2ff_td(w)) <= 1e-12
    hd.releaseDevice()
