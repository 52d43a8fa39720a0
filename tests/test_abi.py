"""The C-ABI library loads, exports every declared symbol and validates input
(no device work: these run on a CPU-only machine)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import xfdtd_cuda_b200 as X
from xfdtd_cuda_b200 import _lib as L
from xfdtd_cuda_b200 import configs
from conftest import has_gpu

HEADER = Path(__file__).resolve().parents[1] / "include" / "xfdtd_b200.h"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(xfb_\w+)\s*\(", text, re.M)))


def test_every_declared_symbol_is_exported_and_bound():
    lib = C.CDLL(str(L.LIB_PATH))
    names = declared()
    assert len(names) >= 45
    for n in names:
        assert hasattr(lib, n), f"{n} not exported"
    bound = {s[0] for s in L.SIGNATURES}
    assert set(names) <= bound, f"unbound: {set(names) - bound}"


def test_status_strings_and_version():
    lib = L.load()
    assert lib.xfb_abi_version() == 2
    for s in range(9):
        assert lib.xfb_status_string(s)
    assert lib.xfb_status_string(99) == b"unknown status"


def _scene(**kw):
    sim = configs.dielectric_sphere(cells=20, dl=5e-3, pml=4, tfsf_inset=3, nf2ff_inset=2, radius=0.02, **kw)
    return sim.lower()


def test_create_destroy_without_device_and_view():
    sc, keep = _scene()
    h = X.Handle(sc, keep)
    gi = h.info()
    assert (gi.nx, gi.ny, gi.nz) == (28, 28, 28)
    assert gi.dim == 3 and gi.n_materials == 2
    v = h.compiled_view()
    assert v.nx == 28 and v.tfsf_enabled == 1 and v.nf2ff_enabled == 1
    ids = np.ctypeslib.as_array(v.material_id, shape=(28, 28, 28))
    assert set(np.unique(ids)) == {0, 1}
    h.close()


@pytest.mark.parametrize("mutate,msg", [
    (lambda s: setattr(s, "dim", 4), "dim"),
    (lambda s: setattr(s, "courant", 1.5), "courant"),
    (lambda s: setattr(s, "dx", -1.0), "cell sizes"),
    (lambda s: s.domain_cells.__setitem__(0, 0), "domain_cells"),
    (lambda s: setattr(s, "n_materials", 0), "materials"),
    (lambda s: s.pml.cells.__setitem__(0, 200), "pml"),
])
def test_invalid_scenes_rejected(mutate, msg):
    sc, keep = _scene()
    mutate(sc)
    with pytest.raises(X.XfbError) as e:
        X.Handle(sc, keep)
    assert e.value.status == L.XFB_ERR_INVALID
    assert msg in str(e.value)


def test_tfsf_box_must_fit():
    sim = configs.dielectric_sphere(cells=20, dl=5e-3, pml=4, tfsf_inset=12, nf2ff_inset=2, radius=0.02)
    sc, keep = sim.lower()
    with pytest.raises(X.XfbError, match="TFSF box"):
        X.Handle(sc, keep)


def test_state_calls_before_init():
    sc, keep = _scene()
    h = X.Handle(sc, keep)
    with pytest.raises(X.XfbError) as e:
        h.step(1)
    assert e.value.status == L.XFB_ERR_STATE


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_init_without_device_fails_loudly():
    sc, keep = _scene()
    h = X.Handle(sc, keep)
    with pytest.raises(X.XfbError) as e:
        h.init(10)
    assert e.value.status == L.XFB_ERR_NO_DEVICE


def test_missing_library_raises(tmp_path):
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        L.load(tmp_path / "libxfdtd_b200.so")


def _handle(sim):
    sc, keep = sim.lower()
    return X.Handle(sc, keep)


def test_batch_validates_its_scenes():
    a = _handle(configs.dielectric_sphere(cells=20, dl=5e-3, pml=4, precision="fp32", tfsf_inset=3, freqs=()))
    b = _handle(configs.dielectric_sphere(cells=24, dl=5e-3, pml=4, precision="fp32", tfsf_inset=3, freqs=()))
    c64 = _handle(configs.dielectric_sphere(cells=20, dl=5e-3, pml=4, precision="fp64", tfsf_inset=3, freqs=()))
    flat = _handle(configs.cylinder_2d(cells=32, dl=1e-3, pml=4, precision="fp32", radius=0.004, tfsf_inset=3, n_probes=1))
    with pytest.raises(X.XfbError, match="one precision"):
        X.Batch([a, c64])
    with pytest.raises(X.XfbError, match="3-D"):
        X.Batch([a, flat])
    with pytest.raises(X.XfbError, match="twice"):
        X.Batch([a, a])
    batch = X.Batch([a, b])
    with pytest.raises(X.XfbError, match="already belongs"):
        X.Batch([b])
    with pytest.raises(X.XfbError, match="tile rows"):
        batch._c(batch.lib.xfb_batch_set_tile(batch.b, 12))
    # a batched handle refuses to be destroyed on its own; the batch releases it
    assert a.lib.xfb_destroy(a.h) == L.XFB_ERR_STATE
    with pytest.raises(X.XfbError, match="not initialised"):
        batch.step(1)
    batch.close()
    assert a.lib.xfb_destroy(a.h) == L.XFB_OK
    a.h = None


def test_batched_sweep_config_is_seeded():
    s1 = configs.batched_sweep(n=8, seed=4)
    s2 = configs.batched_sweep(n=8, seed=4)
    sides = [s.objects[0].shape.size.x for s in s1]
    assert sides == [s.objects[0].shape.size.x for s in s2]
    assert all(0.064 - 1e-12 <= x <= 0.256 + 1e-12 for x in sides)
