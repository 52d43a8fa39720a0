"""Temporally blocked 2-D TMz step (k_step2_tb): S steps per launch in
shared-memory tiles with an S-cell halo, probes recorded inside.

Against the one-launch-per-step kernel and the CPU restatement: FP64 fields,
probes and the CPML state bit-identical for several block lengths (including
run lengths that are not multiples of it), random initial fields, thick and
thin CPML, checkpoints taken between blocked launches; FP32 to round-off.
"""
import numpy as np
import pytest

import xfdtd_cuda_b200 as X
from conftest import rel_l2
from helpers import oracle_of
from xfdtd_cuda_b200 import _lib as L
from xfdtd_cuda_b200 import configs

pytestmark = pytest.mark.gpu


def _scene(prec="fp64", cells=150, pml=10, inset=12):
    return configs.cylinder_2d(cells=cells, dl=1e-3, pml=pml, precision=prec, radius=0.02, tfsf_inset=inset,
                               n_probes=9, seed=4)


def _run(sim, steps, tb, init_fields=None, graph=True, chunks=None):
    sc, keep = sim.lower()
    h = X.Handle(sc, keep)
    h.set_temporal_block(tb)
    h.set_graph(graph, 16)
    h.init(steps)
    if init_fields is not None:
        for f, a in init_fields.items():
            h.write_field(f, a)
    for n in chunks or [steps]:
        h.step(n)
    h.sync()
    return h


def _fields(h):
    return {f: h.read_field(f) for f in (L.EZ, L.HX, L.HY)}


@pytest.mark.parametrize("tb", [1, 3, 7, 15])
def test_blocked_equals_per_step_fp64(tb):
    steps = 97
    a = _run(_scene(), steps, 0)
    b = _run(_scene(), steps, tb, chunks=[40, 57])
    assert b.info().launches_per_step == 1
    fa, fb = _fields(a), _fields(b)
    for f in fa:
        assert np.array_equal(fa[f], fb[f]), f
    for p in range(len(a.probe_desc)):
        assert np.array_equal(a.read_probe(p), b.read_probe(p)), p
    a.close()
    b.close()


def test_blocked_matches_oracle_thin_cpml():
    steps = 160
    h = _run(_scene(cells=90, pml=4, inset=6), steps, 7)
    o = oracle_of(_scene(cells=90, pml=4, inset=6), steps)
    o.run(steps)
    for f in (L.EZ, L.HX, L.HY):
        assert np.array_equal(h.read_field(f), o.field(f)), f
    for p in range(len(h.probe_desc)):
        assert np.array_equal(h.read_probe(p), o.probe(p)), p
    h.close()


def test_blocked_random_fields_equal_per_step():
    steps = 45
    rng = np.random.default_rng(8)
    ref = _run(_scene(cells=90, pml=4, inset=6), 1, 0)
    init = {f: rng.standard_normal(ref.read_field(f).shape) for f in (L.EZ, L.HX, L.HY)}
    ref.close()
    a = _run(_scene(cells=90, pml=4, inset=6), steps, 0, init_fields=init)
    b = _run(_scene(cells=90, pml=4, inset=6), steps, 5, init_fields=init)
    for f in (L.EZ, L.HX, L.HY):
        assert np.array_equal(a.read_field(f), b.read_field(f)), f
    a.close()
    b.close()


def test_blocked_checkpoint_resume_and_graph_off():
    steps = 70
    ref = _run(_scene(), steps, 7)
    sc, keep = _scene().lower()
    h = X.Handle(sc, keep)
    h.set_temporal_block(7)
    h.set_graph(False, 1)
    h.init(steps)
    h.step(33)
    st = h.get_state()
    h.step(20)
    h.set_state(st)
    h.step(steps - 33)
    h.sync()
    for f in (L.EZ, L.HX, L.HY):
        assert np.array_equal(h.read_field(f), ref.read_field(f)), f
    for p in range(len(h.probe_desc)):
        assert np.array_equal(h.read_probe(p), ref.read_probe(p)), p
    h.close()
    ref.close()


def test_blocked_fp32_to_round_off():
    steps = 120
    a = _run(_scene("fp32"), steps, 0)
    b = _run(_scene("fp32"), steps, 9)
    for f in (L.EZ, L.HX, L.HY):
        assert rel_l2(b.read_field(f), a.read_field(f)) <= 1e-6
    a.close()
    b.close()
