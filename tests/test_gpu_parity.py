"""Parity of the CUDA engine against the CPU restatement of the reference.

FP64: the engine evaluates every update, correction and accumulation in the
reference's order without FMA contraction, so fields, CPML/ADE state, NF2FF
currents, probes and movies must agree to <= 1e-12 relative (and are expected
to agree bit for bit).  FP32: relative L2 <= 1e-4 against the FP64 oracle on
probe series and far field, the accuracy budget of the FP32 fused path.
"""
import math

import numpy as np
import pytest

import xfdtd_cuda_b200 as X
from xfdtd_cuda_b200 import configs
from conftest import rel_l2, max_rel
from helpers import bit_equal, compare_fields, engine, fields_of, oracle_of
from oracle import far_field_numpy

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def small_sphere(precision="fp64", **kw):
    # 28^3 inner cells of 5 mm: sphere r = 6 cells, TFSF 4 cells in, NF2FF 2 in
    args = dict(cells=28, dl=5e-3, pml=6, precision=precision, tfsf_inset=5, nf2ff_inset=3,
                freqs=(1.5e9, 4e9), radius=0.03,
                probes=[((0.0, 0.0, 0.0), 2), ((0.05, -0.03, 0.02), 4), ((-0.06, 0.06, -0.06), 0)])
    args.update(kw)
    return configs.dielectric_sphere(**args)


def add_movie(sim, field=0, interval=7):
    sim.addMonitor(X.MovieMonitor(X.FieldMonitor(X.Cube(X.Vector(-0.07, 0.0, -0.07), X.Vector(0.14, 5e-3, 0.14)), field),
                                  interval))
    return sim


PATHS = [1, 2]  # XFB_PATH_SPLIT (H and E half-step kernels), XFB_PATH_FUSED (one-sweep step)
PLAIN = 3        # XFB_PATH_PLAIN (reference kernel structure; no ADE, 3-D only)


def run_pair(sim, n, path=0):
    h = engine(sim, n, path=path)
    h.step(n)
    h.sync()
    o = oracle_of(sim, n)
    o.run(n)
    return h, o


def check_all(h, o, dim, n_probes, n_movies, nf, tol=FP64_TOL, expect_exact=True):
    gf, of = fields_of(h, dim), fields_of(o, dim)
    err = compare_fields(gf, of)
    assert err <= tol, f"field mismatch {err:.3e}"
    for p in range(n_probes):
        assert max_rel(h.read_probe(p), o.probe(p)) <= tol
    for m in range(n_movies):
        assert max_rel(h.read_movie(m), o.movie(m)) <= tol
    if nf:
        gi = h.info()
        for f in range(gi.n_freqs):
            for face in range(6):
                for w in range(4):
                    a, b = h.read_nf2ff(f, face, w), o.nf2ff(f, face, w)
                    assert np.abs(a - b).max() <= tol * max(np.abs(b).max(), 1e-300)
    if expect_exact:
        assert bit_equal(gf, of), "FP64 fields agree within tolerance but not bit for bit"


@pytest.mark.parametrize("path", PATHS + [PLAIN])
def test_fp64_dielectric_sphere_bitexact(path):
    sim = add_movie(small_sphere())
    h, o = run_pair(sim, 90, path)
    check_all(h, o, 3, 3, 1, nf=True)


@pytest.mark.parametrize("path", PATHS)
def test_fp64_h_field_movies_bitexact(path):
    # movies of the three H components (the reference instantiates
    # MovieMonitor<HX..HZ>, movie_monitor.cu:136-138, but never dispatches them)
    sim = small_sphere()
    for f in (3, 4, 5):
        add_movie(sim, field=f, interval=6)
    h, o = run_pair(sim, 60, path)
    check_all(h, o, 3, 3, 3, nf=False)
    for m in range(3):
        assert np.array_equal(h.read_movie(m), o.movie(m))
        assert np.abs(h.read_movie(m)).max() > 0


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("kind", ["drude", "debye", "drude_lorentz", "mlorentz"])
@pytest.mark.parametrize("radius", [0.03, 0.018])
def test_fp64_ade_bitexact(kind, path, radius):
    # radius 0.03 puts TFSF face planes next to the dispersive box (ADE inside
    # the step kernel); 0.018 keeps them apart (ADE as a separate box pass)
    mats = {
        "drude": X.DrudeMedium("d", 1.0, [2e10], [1e9]),
        "debye": X.DebyeMedium("b", 2.0, [6.0], [2e-11]),
        "drude_lorentz": configs.dispersive_material(),
        "mlorentz": X.MLorentzMaterial.makeMLorentz("m", 2.0, (5 - 2) * (2 * math.pi * 2e9) ** 2, 0.0,
                                                   (2 * math.pi * 2e9) ** 2, 2 * math.pi * 2e9, 1.0),
    }
    sim = configs.dispersive_sphere(cells=26, dl=4e-3, pml=6, precision="fp64", freqs=(1e9, 3e9), tfsf_inset=4,
                                    nf2ff_inset=2, radius=radius, material=mats[kind],
                                    probes=[((0.0, 0.0, 0.0), 2), ((0.01, 0.0, 0.0), 1)])
    h, o = run_pair(sim, 80, path)
    check_all(h, o, 3, 2, 0, nf=True)


@pytest.mark.parametrize("path", PATHS)
def test_fp64_cylinder_2d_bitexact(path):
    # 2-D TMz: H and E half-step kernels, and the one-sweep 2-D step
    sim = configs.cylinder_2d(cells=96, dl=1e-3, pml=8, precision="fp64", radius=0.012, tfsf_inset=6, n_probes=5)
    sim.addMonitor(X.MovieMonitor(X.FieldMonitor(X.Cube(X.Vector(-0.04, -0.04, -math.inf), X.Vector(0.08, 0.08, math.inf)),
                                                 X.EMF.Field.EZ), 9))
    h, o = run_pair(sim, 150, path)
    check_all(h, o, 2, 5, 1, nf=False)


@pytest.mark.parametrize("path", PATHS + [PLAIN])
def test_fp64_no_tfsf_no_pml_initial_field(path):
    # PEC box with random initial fields: pure Yee update, no correctors
    sim = X.Simulation(3e-3, 3e-3, 3e-3, 0.9)
    sim.addObject(X.Object("domain", X.Cube(X.Vector(0, 0, 0), X.Vector(0.051, 0.042, 0.039)), X.Material.createAir()))
    sim.addObject(X.Object("blk", X.Cube(X.Vector(0.01, 0.01, 0.01), X.Vector(0.01, 0.02, 0.01)),
                           X.Material("lossy", X.ElectroMagneticProperty(4.0, 1.5, 0.02, 0.0))))
    n = 60
    h = engine(sim, n, path=path)
    o = oracle_of(sim, n)
    rng = np.random.default_rng(7)
    for f in range(6):
        v = rng.standard_normal(h.shape(f))
        h.write_field(f, v)
        o.set_field(f, v)
    h.step(n)
    h.sync()
    o.run(n)
    gf, of = fields_of(h, 3), fields_of(o, 3)
    assert compare_fields(gf, of) <= FP64_TOL
    assert bit_equal(gf, of)


def test_fp64_nf2ff_reads_between_steps():
    # surface samples wait in a ring for several steps before they reach the
    # NF2FF accumulators; reads in the middle of a run (which flush the ring)
    # at step counts on and off the ring length change no bit of the result
    sim = small_sphere()
    n = 61
    h = engine(sim, n, path=2)
    for chunk in (5, 3, 8, 13, 1, 31):
        h.step(chunk)
        h.read_nf2ff(1, 3, 2)
    h.sync()
    o = oracle_of(sim, n)
    o.run(n)
    for f in range(2):
        for face in range(6):
            for w in range(4):
                assert np.array_equal(h.read_nf2ff(f, face, w), o.nf2ff(f, face, w))


def elongated_scene(precision="fp64"):
    # 36 x 56 x 104 inner cells of 3 mm + 6-cell CPML: the one-sweep tiles at
    # k0 = 32 and 64 away from the TFSF faces are lean interior work items
    # (the bulk-copy body); TFSF box, a lossy block and CPML around them
    sim = X.Simulation(3e-3, 3e-3, 3e-3, 0.9, precision=precision)
    sim.addObject(X.Object("domain", X.Cube(X.Vector(0, 0, 0), X.Vector(0.108, 0.168, 0.312)), X.Material.createAir()))
    sim.addObject(X.Object("blk", X.Cube(X.Vector(0.04, 0.06, 0.12), X.Vector(0.02, 0.04, 0.06)),
                           X.Material("lossy", X.ElectroMagneticProperty(4.0, 1.5, 0.02, 0.0))))
    tau = 20 * 3e-3 / 6e8
    sim.addWaveformSource(X.TFSF3D(5, 5, 5, math.pi / 3, math.pi / 5, 0.4, X.Waveform.gaussian(tau, 4.5 * tau)))
    for d in range(6):
        sim.addBoundary(X.PML(6, d))
    sim.addMonitor(X.PointMonitor(X.Vector(0.05, 0.08, 0.15), 2))
    return sim


@pytest.mark.parametrize("rows", [8, 16])
def test_fp64_lean_interior_bitexact(rows):
    # random initial fields inside the CPML (H scaled to free-space impedance),
    # so the interior tiles carry data from the first step; zero on the walls
    # and in the CPML, whose corrections the reference also applies to wall
    # cells; both tile heights of the one-sweep kernel
    sim = elongated_scene()
    n = 70
    h = engine(sim, n, path=2, block=(32, rows, 1))
    o = oracle_of(sim, n)
    rng = np.random.default_rng(11)
    for f in range(6):
        sh = h.shape(f)
        v = np.zeros(sh)
        inner = tuple(slice(8, s - 8) for s in sh)
        v[inner] = rng.standard_normal(v[inner].shape) * (1.0 if f < 3 else 1.0 / 377.0)
        h.write_field(f, v)
        o.set_field(f, v)
    h.step(n)
    h.sync()
    o.run(n)
    gf, of = fields_of(h, 3), fields_of(o, 3)
    assert compare_fields(gf, of) <= FP64_TOL
    assert bit_equal(gf, of)
    assert max_rel(h.read_probe(0), o.probe(0)) == 0.0


@pytest.mark.parametrize("rows", [8, 16])
def test_fp32_lean_interior_against_fp64_oracle(rows):
    n = 200
    h = engine(elongated_scene("fp32"), n, path=2, block=(32, rows, 1))
    h.step(n)
    h.sync()
    o = oracle_of(elongated_scene(), n)
    o.run(n)
    assert rel_l2(h.read_probe(0), o.probe(0)) <= 1e-4
    gf, of = fields_of(h, 3), fields_of(o, 3)
    for f in of:
        assert rel_l2(gf[f], of[f]) <= 1e-4


@pytest.mark.parametrize("path", PATHS + [PLAIN])
def test_fp32_against_fp64_oracle(path):
    sim32 = small_sphere("fp32")
    sim64 = small_sphere("fp64")
    n = 240
    h = engine(sim32, n, path=path)
    h.step(n)
    h.sync()
    o = oracle_of(sim64, n)
    o.run(n)
    for p in range(3):
        assert rel_l2(h.read_probe(p), o.probe(p)) <= 1e-4
    gi = h.info()
    th = np.linspace(0.05, math.pi - 0.05, 37)
    for f in range(gi.n_freqs):
        cur = [[o.nf2ff(f, face, w) for w in range(4)] for face in range(6)]
        et_o, ep_o = far_field_numpy(cur, list(gi.nf2ff_box), list(gi.origin), (gi.dx, gi.dy, gi.dz),
                                     sim64.nf2ff_list[0].freqs[f], th, 0.0)
        et_g, ep_g = h.far_field(f, th, np.zeros_like(th))
        assert rel_l2(np.concatenate([et_g, ep_g]), np.concatenate([et_o, ep_o])) <= 1e-4


def test_far_field_kernel_matches_numpy():
    sim = small_sphere()
    n = 120
    h = engine(sim, n)
    h.step(n)
    h.sync()
    gi = h.info()
    th = np.linspace(-math.pi, math.pi, 61)
    ph = np.full_like(th, 0.3)
    for f in range(gi.n_freqs):
        cur = [[h.read_nf2ff(f, face, w) for w in range(4)] for face in range(6)]
        et_n, ep_n = far_field_numpy(cur, list(gi.nf2ff_box), list(gi.origin), (gi.dx, gi.dy, gi.dz),
                                     sim.nf2ff_list[0].freqs[f], th, ph)
        et_g, ep_g = h.far_field(f, th, ph)
        assert rel_l2(np.concatenate([et_g, ep_g]), np.concatenate([et_n, ep_n])) <= 1e-10


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_graph_tile_and_path_invariance(precision):
    # Graph replay never changes a bit, nor does the tile shape in FP64 (no
    # FMA contraction).  In FP32 a different tile height moves cells between
    # the step kernel's bodies (bulk-copy or general), which the compiler
    # contracts differently, so there they agree to round-off; likewise across
    # kernel paths.
    sim = configs.dispersive_sphere(cells=30, dl=4e-3, pml=5, precision=precision, freqs=(2e9,), tfsf_inset=4,
                                    nf2ff_inset=2, radius=0.035)
    n = 50
    refs = {}
    for path in (1, 2):
        r = engine(sim, n, graph=False, block=(32, 8, 1), path=path)
        r.step(n)
        r.sync()
        refs[path] = r
    for graph, block, path in [(True, (32, 8, 1), 1), (True, (32, 4, 1), 1), (True, (64, 16, 1), 1),
                               (True, (32, 8, 1), 2), (True, (32, 4, 1), 2), (True, (64, 16, 1), 2)]:
        h = engine(sim, n, graph=graph, block=block, path=path)
        h.step(17)
        h.step(n - 17)
        h.sync()
        if precision == "fp64" or block[1] <= 8:  # the reference runs' tile height (8 rows)
            assert bit_equal(fields_of(h, 3), fields_of(refs[path], 3))
            assert np.array_equal(h.read_nf2ff(0, 1, 2), refs[path].read_nf2ff(0, 1, 2))
        else:
            assert compare_fields(fields_of(h, 3), fields_of(refs[path], 3)) < 1e-5
            assert max_rel(h.read_nf2ff(0, 1, 2), refs[path].read_nf2ff(0, 1, 2)) < 1e-5
    a, b = fields_of(refs[1], 3), fields_of(refs[2], 3)
    if precision == "fp64":
        assert bit_equal(a, b)
    else:
        assert compare_fields(a, b) < 1e-4


def test_checkpoint_resume_equivalence():
    sim = configs.dispersive_sphere(cells=24, dl=4e-3, pml=5, precision="fp32", freqs=(2e9,), tfsf_inset=4,
                                    nf2ff_inset=2, radius=0.03, probes=[((0.0, 0.0, 0.0), 2)])
    n, k = 60, 23
    a = engine(sim, n)
    a.step(n)
    a.sync()
    b = engine(sim, n)
    b.step(k)
    blob = b.get_state()
    b.step(n - k)  # diverge, then roll back
    b.set_state(blob)
    b.step(n - k)
    b.sync()
    assert bit_equal(fields_of(b, 3), fields_of(a, 3))
    assert np.array_equal(a.read_probe(0), b.read_probe(0))
    for face in range(6):  # NF2FF accumulators across a checkpoint taken off the sample-ring boundary
        for w in range(4):
            assert np.array_equal(a.read_nf2ff(0, face, w), b.read_nf2ff(0, face, w))


def test_watchdog_and_errors():
    sim = small_sphere("fp32")
    h = engine(sim, 10)
    h.step(10)
    assert h.check_finite() == 0
    with pytest.raises(X.XfbError):
        h.step(1)  # beyond the sized run
    bad = np.zeros(h.shape(2))
    bad[3, 3, 3] = np.nan
    h.write_field(2, bad)
    assert h.check_finite() == 1


def test_simulation_hd_dropin_flow(tmp_path):
    sim = small_sphere("fp32")
    movie = X.MovieMonitor(X.FieldMonitor(X.Cube(X.Vector(-0.07, 0.0, -0.07), X.Vector(0.14, 5e-3, 0.14)), 0), 10,
                           "movie_ex_xz", str(tmp_path / "movie"))
    sim.addMonitor(movie)
    hd = X.SimulationHD(sim)
    hd.setGridDim((4, 4, 4))
    hd.setBlockDim((8, 8, 8))
    hd.run(60)
    assert movie.data.shape[0] == 6
    assert (tmp_path / "movie" / "00005.npy").exists()
    nf = sim.nf2ffs()[0]
    et, ep = nf.processFarField(np.linspace(-math.pi, math.pi, 36), 0.0, "xz")
    assert et.shape == (2, 36) and np.isfinite(et).all()


def test_plain_path_rejects_dispersive_and_2d():
    for sim in (configs.dispersive_sphere(cells=20, dl=4e-3, pml=4, precision="fp64", freqs=(), tfsf_inset=3,
                                          radius=0.02),
                configs.cylinder_2d(cells=40, dl=1e-3, pml=6, precision="fp64", radius=0.005, tfsf_inset=4)):
        sc, keep = sim.lower()
        h = X.Handle(sc, keep)
        h.set_kernel_path(PLAIN)
        with pytest.raises(X.XfbError, match="plain path"):
            h.init(10)


def test_fp32_2d_cylinder_against_fp64():
    # the 2-D cylinder at reduced size: the FP32 engine against the FP64 engine (which is
    # bit-identical to the CPU restatement) on all probe series
    n = 900
    series = {}
    for prec in ("fp32", "fp64"):
        sim = configs.cylinder_2d(cells=256, precision=prec, tfsf_inset=10, n_probes=8)
        h = engine(sim, n)
        h.step(n)
        h.sync()
        series[prec] = np.concatenate([h.read_probe(p) for p in range(8)])
    assert rel_l2(series["fp32"], series["fp64"]) <= 1e-4
