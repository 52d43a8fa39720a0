"""Scenes handed over as the arrays XFDTD_CORE compiles
(xfb_create_from_arrays): the 18 per-cell coefficient arrays in their field
shapes, per-cell ADE coefficients, CPML profiles, TFSF projections and
incident tables, NF2FF box, monitors.  A scene compiled by the engine is
expanded into that form (the incident tables taken from the CPU
restatement's recurrence) and handed back: the handle steps bit-identically
to the scene's own, FP64.  The compression refuses non-isotropic sets.
"""
import ctypes as C

import numpy as np
import pytest

import xfdtd_cuda_b200 as X
from oracle import OracleSim
from xfdtd_cuda_b200 import _lib as L
from xfdtd_cuda_b200 import configs

_dp = C.POINTER(C.c_double)


def _ptr(a):
    return a.ctypes.data_as(_dp)


def core_arrays_of(sim, steps):
    """xfb_core_arrays of a scene: what XFDTD_CORE would hand over."""
    sc, keep = sim.lower()
    h = X.Handle(sc, keep)
    h.prepare_tables(steps)
    v = h.compiled_view()
    nx, ny, nz, nm = v.nx, v.ny, v.nz, v.n_materials
    mid = np.ctypeslib.as_array(v.material_id, shape=(nx, ny, nz)).astype(np.int64)
    coeff = np.ctypeslib.as_array(v.coeff, shape=(nm, 18))
    keep_arrays = []
    a = L.CoreArrays()
    a.precision = sc.precision
    a.nx, a.ny, a.nz = nx, ny, nz
    a.dx, a.dy, a.dz, a.dt = v.dx, v.dy, v.dz, v.dt
    a.origin = (C.c_double * 3)(*h.info().origin)
    for q in range(18):
        f = q // 3
        shp = (nx + (f in (1, 2, 3)), ny + (f in (0, 2, 4)), nz + (f in (0, 1, 5)))
        arr = np.full(shp, 7.0)  # entries past the cells: never read
        arr[:nx, :ny, :nz] = coeff[mid, q]
        keep_arrays.append(arr)
        a.coeff[q] = _ptr(arr)
    if v.ade_kind:
        P = v.ade_poles
        am = np.ctypeslib.as_array(v.ade_mat, shape=(nm, 3))
        ap = np.ctypeslib.as_array(v.ade_pole, shape=(nm, P, 7))
        a.ade_kind, a.ade_poles = v.ade_kind, P
        for q in range(3):
            arr = np.ascontiguousarray(am[mid, q])
            keep_arrays.append(arr)
            a.ade_cell[q] = _ptr(arr)
        for q in range(7):
            arr = np.ascontiguousarray(ap[mid, :, q])
            keep_arrays.append(arr)
            a.ade_pole[q] = _ptr(arr)
    n = (nx, ny, nz)
    for f in range(6):
        a.pml[f] = v.pml_cells[f]
    for ax in range(3):
        for name, ln in (("pml_ae", n[ax] + 1), ("pml_be", n[ax] + 1), ("pml_ah", n[ax]), ("pml_bh", n[ax])):
            arr = np.ctypeslib.as_array(getattr(v, name)[ax], shape=(ln,)).copy()
            keep_arrays.append(arr)
            getattr(a, name)[ax] = _ptr(arr)
    if v.tfsf_enabled:
        a.tfsf_enabled = 1
        a.tfsf_box = (C.c_int * 6)(*v.tfsf_box)
        for ax in range(3):
            nb = v.tfsf_box[2 * ax + 1] - v.tfsf_box[2 * ax]
            pi = np.ctypeslib.as_array(v.tfsf_proj_int[ax], shape=(nb + 1,)).copy()
            ph = np.ctypeslib.as_array(v.tfsf_proj_half[ax], shape=(nb + 2,)).copy()
            keep_arrays += [pi, ph]
            a.tfsf_proj_int[ax], a.tfsf_proj_half[ax] = _ptr(pi), _ptr(ph)
        a.tfsf_transform_e = (C.c_double * 3)(*v.tfsf_transform_e)
        a.tfsf_transform_h = (C.c_double * 3)(*v.tfsf_transform_h)
        a.tfsf_ca = (C.c_double * 3)(*v.tfsf_ca)
        a.tfsf_cb = (C.c_double * 3)(*v.tfsf_cb)
        e, hh = OracleSim(h, steps).incident_tables()  # rows 0..steps-1 of E and H
        nl = v.aux_nl
        e_full = np.zeros((steps + 1, nl + 1))
        e_full[:steps] = e  # row `steps` (after the last step) is never read
        keep_arrays += [e_full, np.ascontiguousarray(hh)]
        a.aux_nl, a.inc_steps = nl, steps
        a.e_inc, a.h_inc = _ptr(e_full), _ptr(keep_arrays[-1])
    if v.nf2ff_enabled:
        a.nf2ff_enabled = 1
        a.nf2ff_box = (C.c_int * 6)(*v.nf2ff_box)
        fr = np.ctypeslib.as_array(v.freqs, shape=(v.n_freqs,)).copy()
        keep_arrays.append(fr)
        a.n_freqs, a.freqs = v.n_freqs, _ptr(fr)
    if v.nf2ff_td_enabled:
        a.nf2ff_td_enabled = 1
        a.nf2ff_td_box = (C.c_int * 6)(*v.nf2ff_td_box)
        a.nf2ff_td_theta, a.nf2ff_td_phi = v.nf2ff_td_theta, v.nf2ff_td_phi
    a.n_probes, a.probes = sc.n_probes, sc.probes
    a.n_movies, a.movies = sc.n_movies, sc.movies
    keep_arrays += [keep, h]
    return a, keep_arrays


def test_core_arrays_rejected_when_not_isotropic():
    a, keep = core_arrays_of(configs.dielectric_sphere(cells=12, dl=5e-3, pml=3, precision="fp64", tfsf_inset=2,
                                                        nf2ff_inset=1, radius=0.01), 4)
    bad = np.ctypeslib.as_array(a.coeff[1], shape=(1,))  # cexhy of cell 0 -> breaks cexhy == -ceyhx
    bad[0] = bad[0] * 1.5
    with pytest.raises(L.XfbError) as e:
        X.Handle.from_core_arrays(a, keep)
    assert e.value.status == L.XFB_ERR_INVALID and "isotropic" in str(e.value)


@pytest.mark.gpu
@pytest.mark.parametrize("scene", ["dielectric", "dispersive"])
def test_core_arrays_step_like_the_scene(scene):
    steps = 70
    if scene == "dielectric":
        def build():
            sim = configs.dielectric_sphere(cells=24, dl=5e-3, pml=5, precision="fp64", tfsf_inset=4,
                                            nf2ff_inset=2, radius=0.025, freqs=(2e9,),
                                            probes=[((0.0, 0.0, 0.0), L.EZ), ((0.02, -0.01, 0.0), L.HX)])
            sim.addNF2FF(X.NFFFTTimeDomain(3, 3, 3, "", 0.7, 1.9))
            return sim
    else:
        build = lambda: configs.dispersive_sphere(cells=30, dl=3e-3, pml=5, precision="fp64", freqs=(2e9,),
                                                  tfsf_inset=4, nf2ff_inset=2, radius=0.025,
                                                  probes=[((0.0, 0.0, 0.0), L.EX)])
    ref = X.Handle(*build().lower())
    ref.init(steps)
    ref.step(steps)
    ref.sync()
    a, keep = core_arrays_of(build(), steps)
    h = X.Handle.from_core_arrays(a, keep)
    h.init(steps)
    h.step(steps)
    h.sync()
    for f in range(6):
        assert np.array_equal(h.read_field(f), ref.read_field(f)), f
    for p in range(len(ref.probe_desc)):
        assert np.array_equal(h.read_probe(p), ref.read_probe(p)), p
    for face in range(6):
        for w in range(4):
            assert np.array_equal(h.read_nf2ff(0, face, w), ref.read_nf2ff(0, face, w))
    if scene == "dielectric":
        for w in range(6):
            assert np.array_equal(h.read_nf2ff_td(w), ref.read_nf2ff_td(w)), w
    with pytest.raises(L.XfbError):
        h.init(steps + 1)  # longer than the incident tables handed over
    h.close()
    ref.close()


def test_xfdtd_core_adapter_against_accessor_stand_in(tmp_path):
    """include/xfdtd_b200/xfdtd_core_adapter.hpp compiled against the
    stand-in accessor surface in tests/core_adapter/fake and run: the packed
    scene goes through xfb_create_from_arrays and is checked entry by entry
    (materials, ADE, CPML profiles with the c_psi ratio folded in, TFSF,
    NF2FF frequencies read back from the transforms, time-domain box and
    direction, movies, and the two refusals)."""
    import shutil
    import subprocess
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    lib = root / "xfdtd_cuda_b200"
    if not shutil.which("g++"):
        pytest.skip("no g++")
    exe = tmp_path / "adapter_test"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", str(root / "tests/core_adapter/fake"),
           "-I", str(root / "include"), str(root / "tests/core_adapter/adapter_test.cpp"), "-L", str(lib),
           "-lxfdtd_b200", f"-Wl,-rpath,{lib}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=300)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stderr
