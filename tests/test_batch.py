"""Batches of scenes (xfb_batch_*): every scene stepped in a batch ends in the
same state as the same scene stepped alone, with CPML, TFSF, ADE (deferred
box pass), probes and NF2FF — bit for bit in FP64 (both follow the
reference's operation order with no contraction); in FP32 within 1e-5
relative, since a batch cuts its scenes into different work items (whole
tile columns) than a single scene does, so some cells run another body of the
step kernel, which the compiler contracts into FMAs differently; and an FP64
batch agrees with the CPU restatement bit for bit."""
import numpy as np
import pytest

import xfdtd_cuda_b200 as X
from xfdtd_cuda_b200 import _lib as L
from xfdtd_cuda_b200 import configs
from conftest import max_rel
from helpers import bit_equal, compare_fields, fields_of, oracle_of

FP32_TOL = 1e-5

pytestmark = pytest.mark.gpu


def _scenes(precision):
    return [
        configs.dielectric_sphere(cells=28, dl=5e-3, pml=6, precision=precision, tfsf_inset=5, nf2ff_inset=3,
                                  freqs=(1.5e9,), radius=0.03, probes=[((0.0, 0.0, 0.0), 2)]),
        configs.dispersive_sphere(cells=30, dl=4e-3, pml=5, precision=precision, freqs=(2e9,), tfsf_inset=4,
                                  nf2ff_inset=2, radius=0.02, probes=[((0.01, 0.0, 0.0), 1)]),
        *configs.batched_sweep(n=3, seed=11, lo=20, hi=44, pml=5, dl=2e-3, precision=precision),
    ]


def _handle(sim, n, path=2):
    sc, keep = sim.lower()
    h = X.Handle(sc, keep)
    h.set_kernel_path(path)
    h.init(n)
    return h


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("tile", [0, 8, 14, 16])
def test_batch_matches_scenes_stepped_alone(precision, tile):
    n = 45
    sims = _scenes(precision)
    alone = []
    for s in sims:
        h = _handle(s, n)
        h.step(n)
        h.sync()
        alone.append(h)
    hs = [X.Handle(*s.lower()) for s in sims]
    b = X.Batch(hs, tile_rows=tile)
    b.init(n)
    b.step(7)   # the first call autotunes the tile when tile == 0
    b.step(n - 7)
    b.sync()
    info = b.info()
    assert info["tile_rows"] in (8, 14, 16) and info["work_items"] > 0
    for h, a in zip(hs, alone):
        if precision == "fp64":
            assert bit_equal(fields_of(h, 3), fields_of(a, 3))
            for p in range(len(h.probe_desc)):
                assert np.array_equal(h.read_probe(p), a.read_probe(p))
            if h.info().n_freqs:
                assert np.array_equal(h.read_nf2ff(0, 1, 2), a.read_nf2ff(0, 1, 2))
        else:
            assert compare_fields(fields_of(h, 3), fields_of(a, 3)) <= FP32_TOL
            for p in range(len(h.probe_desc)):
                assert max_rel(h.read_probe(p), a.read_probe(p)) <= FP32_TOL
            if h.info().n_freqs:
                assert max_rel(h.read_nf2ff(0, 1, 2), a.read_nf2ff(0, 1, 2)) <= FP32_TOL
    b.close()
    # released handles step on their own from where the batch left them
    with pytest.raises(X.XfbError):
        hs[0].step(1)  # the run was sized for n steps
    for h in hs + alone:
        h.close()


def test_fp64_batch_against_oracle():
    n = 40
    sims = _scenes("fp64")[:2]
    hs = [X.Handle(*s.lower()) for s in sims]
    b = X.Batch(hs)
    b.init(n)
    b.step(n)
    b.sync()
    for s, h in zip(sims, hs):
        o = oracle_of(s, n)
        o.run(n)
        assert bit_equal(fields_of(h, 3), fields_of(o, 3))
    b.close()


@pytest.mark.gpu
def test_autotune_cache_reused(tmp_path, monkeypatch):
    # the first batch autotunes and records its choice per (GPU, precision,
    # scene sizes); a second batch of the same scenes takes it without probing
    cache = tmp_path / "tiles.txt"
    monkeypatch.setenv("XFB_AUTOTUNE_CACHE", str(cache))
    sims = configs.batched_sweep(n=3, lo=20, hi=30, seed=12)

    def batch():
        hs = [X.Handle(*s.lower()) for s in sims]
        b = X.Batch(hs)
        b.init(30)
        return b, hs

    b, hs = batch()
    b.step(20)
    b.sync()
    rows = b.info()["tile_rows"]
    form = b.info()["launch"]
    b.close()
    lines = cache.read_text().splitlines()
    # one line per autotune: key, then tile index + 3 * launch form (1 per step, 2 persistent)
    assert len(lines) == 1 and int(lines[0].split()[-1]) in range(3, 9)
    b2, hs2 = batch()
    b2.step(1)  # too few steps to autotune: without the cache it would take 16-row tiles
    b2.sync()
    assert b2.info()["tile_rows"] == rows and b2.info()["launch"] == form
    b2.close()


def _sweep(precision, n=5, seed=21):
    # scenes without monitors or a separate ADE pass: the persistent form applies
    return configs.batched_sweep(n=n, seed=seed, lo=18, hi=46, pml=5, dl=2e-3, precision=precision)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("tile", [8, 16])
def test_persistent_batch_matches_per_step_and_alone(precision, tile):
    # several persistent launches (chunks of at most 64 steps, odd chunk
    # lengths so launches start on both field sets) against the per-step
    # form and against every scene stepped alone
    n = 150
    sims = _sweep(precision)
    runs = {}
    for form in (L.BATCH_PERSISTENT, L.BATCH_PER_STEP):
        hs = [X.Handle(*s.lower()) for s in sims]
        b = X.Batch(hs, tile_rows=tile, launch=form)
        b.init(n)
        for chunk in (1, 37, 64, 48):
            b.step(chunk)
        b.sync()
        assert b.info()["launch"] == ("persistent" if form == L.BATCH_PERSISTENT else "per_step")
        runs[form] = [fields_of(h, 3) for h in hs]
        b.close()
        for h in hs:
            h.close()
    for q, s in enumerate(sims):
        a = _handle(s, n)
        a.step(n)
        a.sync()
        alone = fields_of(a, 3)
        a.close()
        if precision == "fp64":
            assert bit_equal(runs[L.BATCH_PERSISTENT][q], runs[L.BATCH_PER_STEP][q])
            assert bit_equal(runs[L.BATCH_PERSISTENT][q], alone)
        else:
            assert compare_fields(runs[L.BATCH_PERSISTENT][q], runs[L.BATCH_PER_STEP][q]) <= FP32_TOL
            # the persistent form computes the TFSF incident values in place,
            # the per-step form and a single scene take them from the line
            # tables of k_tfsf_lines, which the FP32 engine contracts
            # differently: round-off, within the FP32 engine's 1e-4 bar
            assert compare_fields(runs[L.BATCH_PERSISTENT][q], alone) <= 1e-4


def test_persistent_batch_refused_with_monitors():
    sims = _scenes("fp64")[:1]  # records probes and NF2FF between steps
    hs = [X.Handle(*s.lower()) for s in sims]
    b = X.Batch(hs, launch=L.BATCH_PERSISTENT)
    with pytest.raises(X.XfbError) as e:
        b.init(10)
    assert e.value.status == L.XFB_ERR_INVALID
    b.close()
    b = X.Batch(hs)  # the automatic choice keeps the per-step form
    b.init(30)
    b.step(30)
    b.sync()
    assert b.info()["launch"] == "per_step"
    b.close()
    for h in hs:
        h.close()
