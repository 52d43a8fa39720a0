"""Bounded waits of the one-sweep step kernel.

The step kernel stages its planes with asynchronous bulk copies and waits for
each with a bounded poll loop.  A wait that runs out must not hang the device:
the work item lets its copies in flight land, sets the handle's (or batch's)
error flag and ends, and the host reports XFB_ERR_TIMEOUT.  The tests make the
waits run out with a poll limit of 0 (xfb_set_wait_limit), so no copy is ever
abandoned and the device context stays usable: a fresh init then runs
bit-identically to a handle that never timed out.
"""
import numpy as np
import pytest

import xfdtd_cuda_b200 as X
from xfdtd_cuda_b200 import _lib as L
from xfdtd_cuda_b200 import configs

pytestmark = pytest.mark.gpu


def _scene(seed_shift=0.0):
    return configs.dispersive_sphere(cells=40 + int(seed_shift), dl=3e-3, pml=6, precision="fp64", freqs=(2e9,),
                                     tfsf_inset=4, nf2ff_inset=2, radius=0.03)


def _handle(sim, n):
    sc, keep = sim.lower()
    h = X.Handle(sc, keep)
    h.set_launch_hint((1, 1, 1), (32, 16, 1))
    h.init(n)
    return h


def test_step_wait_runs_out_reports_timeout_and_recovers():
    h = _handle(_scene(), 12)
    h.step(2)
    h.sync()
    h.set_wait_limit(0)
    h.step(1)
    with pytest.raises(L.XfbError) as e:
        h.sync()
    assert e.value.status == L.XFB_ERR_TIMEOUT
    # read-back of an incomplete run reports the same status
    with pytest.raises(L.XfbError) as e:
        h.read_field(L.EZ)
    assert e.value.status == L.XFB_ERR_TIMEOUT
    # the device is fine: a new run equals one that never timed out
    h.init(12)
    h.step(5)
    h.sync()
    ref = _handle(_scene(), 12)
    ref.step(5)
    ref.sync()
    for f in range(6):
        assert np.array_equal(h.read_field(f), ref.read_field(f))
    h.close()
    ref.close()


def test_batch_wait_runs_out_reports_timeout():
    hs = [_handle(_scene(q * 8), 10) for q in range(2)]
    b = X.Batch(hs, tile_rows=16)
    b.init(10)
    b.step(1)
    b.sync()
    b.set_wait_limit(0)
    b.step(1)
    with pytest.raises(L.XfbError) as e:
        b.sync()
    assert e.value.status == L.XFB_ERR_TIMEOUT
    b.init(10)  # the limit and the flag start over
    b.step(2)
    b.sync()
    b.close()
    for h in hs:
        h.close()


def test_persistent_batch_wait_runs_out_reports_timeout():
    # the persistent launch's staging waits and its waits on the previous
    # step of a scene share the batch's poll limit: with 0 they run out, the
    # CTAs stop at their next ticket and the host reports the timeout
    sims = configs.batched_sweep(n=3, seed=21, lo=18, hi=30, pml=5, dl=2e-3, precision="fp64")
    hs = [X.Handle(*s.lower()) for s in sims]
    b = X.Batch(hs, tile_rows=16, launch=L.BATCH_PERSISTENT)
    b.init(20)
    b.step(2)
    b.sync()
    b.set_wait_limit(0)
    b.step(5)
    with pytest.raises(L.XfbError) as e:
        b.sync()
    assert e.value.status == L.XFB_ERR_TIMEOUT
    b.init(20)  # the limit and the flag start over
    b.step(4)
    b.sync()
    b.close()
    for h in hs:
        h.close()


def test_wait_limit_rejects_negative_and_paths_without_waits():
    h = _handle(_scene(), 4)
    with pytest.raises(L.XfbError) as e:
        h.set_wait_limit(-1)
    assert e.value.status == L.XFB_ERR_INVALID
    h.close()
    sc, keep = _scene().lower()
    s = X.Handle(sc, keep)
    s.set_kernel_path(L.PATH_SPLIT)
    s.init(4)
    with pytest.raises(L.XfbError) as e:
        s.set_wait_limit(0)
    assert e.value.status == L.XFB_ERR_STATE
    s.close()
