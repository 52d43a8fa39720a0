"""Far field through xfb_far_field_static, the entry point that allocates no
device memory, checked against the allocating xfb_far_field.

Who needs it: a host that hands the solver a fixed device-memory budget when
it starts and treats any later cudaMalloc as an error (pool-managed
frameworks), or a latency-bound loop in which a cudaMalloc/cudaFree would stall
the device.  Such callers cannot use xfb_far_field, which allocates its angle
and output buffers on every call; xfb_far_field_static uses one fixed device
array of the library instead, so it is limited to
XFB_FAR_FIELD_STATIC_MAX_ANGLES angles per call.

This file is collected last on purpose: a failure here leaves every other test
already run.  It builds its own scene, so it also runs alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

import xfdtd_cuda_b200 as X
from xfdtd_cuda_b200 import _lib as L
from xfdtd_cuda_b200 import configs

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the same kernel on the same currents: agreement to round-off


def _handle():
    sim = configs.dielectric_sphere(cells=24, dl=5e-3, pml=5, precision="fp32", tfsf_inset=4, nf2ff_inset=2,
                                    radius=0.025, freqs=(1.5e9, 3e9))
    sc, keep = sim.lower()
    h = X.Handle(sc, keep)
    h.init(80)
    h.step(80)
    h.sync()
    return h


def _call(lib, fn, h, freq, th, ph):
    out = np.empty((len(th), 4), dtype=np.float64)
    dp = C.POINTER(C.c_double)
    st = fn(h.h, freq, len(th), th.ctypes.data_as(dp), ph.ctypes.data_as(dp), out.ctypes.data_as(dp))
    return st, out


def test_far_field_static_matches_allocating_entry_point():
    h = _handle()
    lib = L.load()
    rng = np.random.default_rng(11)
    # two calls in a row through the C-ABI; the second is shorter than the first,
    # so stale scratch contents from the first call must not leak into it
    for n, freq in [(181, 0), (37, 1)]:
        th = np.ascontiguousarray(rng.uniform(0, np.pi, n))
        ph = np.ascontiguousarray(rng.uniform(-np.pi, np.pi, n))
        st, got = _call(lib, lib.xfb_far_field_static, h, freq, th, ph)
        assert st == L.XFB_OK, lib.xfb_last_error(h.h)
        st, want = _call(lib, lib.xfb_far_field, h, freq, th, ph)
        assert st == L.XFB_OK
        assert np.isfinite(got).all()
        assert np.linalg.norm(got - want) <= TOL * np.linalg.norm(want)


def test_far_field_static_rejects_more_angles_than_its_scratch():
    h = _handle()
    lib = L.load()
    n = L.FAR_FIELD_STATIC_MAX_ANGLES + 1
    th = np.zeros(n)
    ph = np.zeros(n)
    st, _ = _call(lib, lib.xfb_far_field_static, h, 0, th, ph)
    assert st == L.XFB_ERR_RANGE
    assert b"at most 4096 angles" in lib.xfb_last_error(h.h)
