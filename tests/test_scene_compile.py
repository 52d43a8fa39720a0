"""Host scene compiler: coefficients, CPML profiles, voxelisation, TFSF and
NF2FF geometry, ADE coefficients (checked against their published formulas and
against the analytic permittivity of each dispersive model)."""
import math

import numpy as np
import pytest

import xfdtd_cuda_b200 as X
from xfdtd_cuda_b200 import configs

EPS0, MU0 = X.EPSILON_0, X.MU_0


def compile_sim(sim):
    sc, keep = sim.lower()
    h = X.Handle(sc, keep)
    return h, h.compiled_view(), h.info()


def lut(v):
    return np.ctypeslib.as_array(v.coeff, shape=(v.n_materials, 18))


def box_sim(mat, dl=(2e-3, 3e-3, 4e-3), courant=0.8):
    s = X.Simulation(*dl, courant)
    s.addObject(X.Object("domain", X.Cube(X.Vector(0, 0, 0), X.Vector(0.04, 0.048, 0.06)), X.Material.createAir()))
    s.addObject(X.Object("blk", X.Cube(X.Vector(0.01, 0.012, 0.02), X.Vector(0.01, 0.012, 0.02)), mat))
    return s


def test_time_step_courant():
    h, v, gi = compile_sim(box_sim(X.Material.createAir()))
    dt = 0.8 / (X.C_0 * math.sqrt(1 / 2e-3 ** 2 + 1 / 3e-3 ** 2 + 1 / 4e-3 ** 2))
    assert gi.dt == pytest.approx(dt, rel=1e-14)


def test_yee_coefficients_lossy_magnetic():
    prop = X.ElectroMagneticProperty(4.0, 2.5, 0.3, 150.0)
    h, v, gi = compile_sim(box_sim(X.Material("m", prop)))
    c = lut(v)[1]
    dt, (dx, dy, dz) = gi.dt, (2e-3, 3e-3, 4e-3)
    eps, mu, se, sm = 4 * EPS0, 2.5 * MU0, 0.3, 150.0
    ce = (2 * eps - se * dt) / (2 * eps + se * dt)
    cb = 2 * dt / (2 * eps + se * dt)
    ch = (2 * mu - sm * dt) / (2 * mu + sm * dt)
    db = 2 * dt / (2 * mu + sm * dt)
    want = [ce, -cb / dz, cb / dy, ce, -cb / dx, cb / dz, ce, -cb / dy, cb / dx,
            ch, db / dz, -db / dy, ch, db / dx, -db / dz, ch, db / dy, -db / dx]
    np.testing.assert_allclose(c, want, rtol=1e-14)
    # background is vacuum: ce = ch = 1, cb = dt / eps0
    c0 = lut(v)[0]
    assert c0[0] == 1.0 and c0[9] == 1.0
    assert c0[2] == pytest.approx(gi.dt / EPS0 / dy, rel=1e-14)


def test_pec_zeroes_e_coefficients():
    h, v, gi = compile_sim(box_sim(X.Material.createPec()))
    c = lut(v)[1]
    assert np.all(c[:9] == 0)
    assert c[9] == 1.0


def test_voxelisation_counts():
    dl = 2e-3
    s = X.Simulation(dl, dl, dl, 0.9)
    s.addObject(X.Object("domain", X.Cube(X.Vector(-0.05, -0.05, -0.05), X.Vector(0.1, 0.1, 0.1)), X.Material.createAir()))
    s.addObject(X.Object("sph", X.Sphere(X.Vector(0, 0, 0), 0.03), X.Material("d", X.ElectroMagneticProperty(2))))
    s.addObject(X.Object("cube", X.Cube(X.Vector(0.032, 0.032, 0.032), X.Vector(0.01, 0.01, 0.01)),
                         X.Material("e", X.ElectroMagneticProperty(3))))
    h, v, gi = compile_sim(s)
    ids = np.ctypeslib.as_array(v.material_id, shape=(gi.nx, gi.ny, gi.nz))
    n_sph = int((ids == 1).sum())
    assert abs(n_sph - 4 / 3 * math.pi * (0.03 / dl) ** 3) / n_sph < 0.03
    assert int((ids == 2).sum()) == 5 ** 3


def test_cylinder_2d_voxels():
    sim = configs.cylinder_2d(cells=200, dl=1e-3, pml=10, precision="fp64", radius=0.04, n_probes=0)
    h, v, gi = compile_sim(sim)
    assert gi.dim == 2 and gi.nz == 1
    ids = np.ctypeslib.as_array(v.material_id, shape=(gi.nx, gi.ny, 1))
    n = int((ids == 1).sum())
    assert abs(n - math.pi * 40 ** 2) / n < 0.02
    assert lut(v)[1][6] == 0.0  # PEC


def test_cpml_profiles():
    sim = configs.dielectric_sphere(cells=30, dl=5e-3, pml=8, tfsf_inset=4, nf2ff_inset=2, radius=0.03)
    h, v, gi = compile_sim(sim)
    dt, L, m = gi.dt, 8, 3.0
    smax = 0.8 * (m + 1) / (X.ETA_0 * 5e-3)
    n = gi.nx
    ae = np.ctypeslib.as_array(v.pml_ae[0], shape=(n + 1,))
    be = np.ctypeslib.as_array(v.pml_be[0], shape=(n + 1,))
    ah = np.ctypeslib.as_array(v.pml_ah[0], shape=(n,))

    def ab(rho):
        sg, al = smax * rho ** m, 0.05 * (1 - rho)
        b = math.exp(-(sg + al) * dt / EPS0)
        return sg / (sg + al) * (b - 1), b

    for q in range(1, L):
        a, b = ab((L - q) / L)
        assert ae[q] == pytest.approx(a, rel=1e-12) and be[q] == pytest.approx(b, rel=1e-12)
    for q in range(n - L, n):
        assert ae[q] == pytest.approx(ab((q - (n - L)) / L)[0], rel=1e-12, abs=1e-300)
        assert ah[q] == pytest.approx(ab((q + 0.5 - (n - L)) / L)[0], rel=1e-12)
    assert np.all(ae[L + 1:n - L] == 0) and ae[L] == 0
    assert np.all(np.diff(ae[1:L]) > 0)  # |a| grows towards the outer wall (a < 0)


def test_tfsf_geometry():
    sim = configs.dielectric_sphere(cells=30, dl=5e-3, pml=6, tfsf_inset=5, nf2ff_inset=3, radius=0.03)
    h, v, gi = compile_sim(sim)
    assert list(gi.tfsf_box) == [11, 31, 11, 31, 11, 31]
    assert list(gi.nf2ff_box) == [9, 33, 9, 33, 9, 33]
    te = np.array(v.tfsf_transform_e[:])
    th = np.array(v.tfsf_transform_h[:])
    k = np.array([1.0, 0, 0])
    assert np.linalg.norm(te) == pytest.approx(1.0)
    assert abs(te @ k) < 1e-15 and np.allclose(np.cross(k, te), th)
    pi = np.ctypeslib.as_array(v.tfsf_proj_int[0], shape=(21,))
    np.testing.assert_allclose(pi, np.arange(21) + 2.0)  # x-propagation: integer projections
    assert v.aux_ceih == pytest.approx(-gi.dt / (EPS0 * 5e-3))


@pytest.mark.parametrize("theta,phi", [(math.pi / 2, 0.3), (0.7, 1.1), (2.5, -2.0), (math.pi / 2, math.pi)])
def test_tfsf_oblique_stencils_inside_aux_grid(theta, phi):
    s = configs.dielectric_sphere(cells=24, dl=5e-3, pml=5, tfsf_inset=4, nf2ff_inset=2, radius=0.02)
    s.sources[0].theta, s.sources[0].phi = theta, phi
    h, v, gi = compile_sim(s)
    b = list(gi.tfsf_box)
    n = [b[1] - b[0], b[3] - b[2], b[5] - b[4]]
    lo = hi = 0.0
    for a in range(3):
        pi = np.ctypeslib.as_array(v.tfsf_proj_int[a], shape=(n[a] + 1,))
        ph = np.ctypeslib.as_array(v.tfsf_proj_half[a], shape=(n[a] + 2,))
        lo += min(pi.min(), ph.min())
        hi += max(pi.max(), ph.max())
    assert lo - 0.5 >= -1e-9 and hi + 1 <= v.aux_nl


def test_nf2ff_dft_tables():
    sim = configs.dielectric_sphere(cells=24, dl=5e-3, pml=5, tfsf_inset=4, nf2ff_inset=2, radius=0.02,
                                    freqs=(1e9, 2.5e9))
    h, v, gi = compile_sim(sim)
    h.prepare_tables(50)
    v = h.compiled_view()
    te = np.ctypeslib.as_array(v.nf2ff_te, shape=(2, 50, 2))
    th = np.ctypeslib.as_array(v.nf2ff_th, shape=(2, 50, 2))
    t = np.arange(50)
    for f, fr in enumerate((1e9, 2.5e9)):
        w = 2 * math.pi * fr
        np.testing.assert_allclose(te[f, :, 0] + 1j * te[f, :, 1], gi.dt * np.exp(-1j * w * (t + 1) * gi.dt), rtol=1e-13)
        np.testing.assert_allclose(th[f, :, 0] + 1j * th[f, :, 1], gi.dt * np.exp(-1j * w * (t + 0.5) * gi.dt), rtol=1e-13)
    src = np.ctypeslib.as_array(v.aux_source, shape=(51,))
    tau = 20 * 5e-3 / 6e8
    np.testing.assert_allclose(src, np.exp(-(((t.tolist() + [50]) * np.ones(1) * gi.dt - 4.5 * tau) / tau) ** 2), rtol=1e-13)


# ---- ADE: numerical permittivity of the discrete recursions ---------------
def numerical_eps_r(v, gi, m, omega):
    """eps_r of the discrete Ampere law + J recursion at frequency omega."""
    dt = gi.dt
    z = np.exp(1j * omega * dt)
    P = v.ade_poles
    pole = np.ctypeslib.as_array(v.ade_pole, shape=(v.n_materials, P, 7))[m]
    cf = lut(v)[m]
    eps_inf_term = None
    jsum = 0
    for p in range(P):
        cjj, cjjp, cjen, cje, cjep = pole[p][:5]
        if v.ade_kind == 2:    # Drude: J+ = cjj J + cje (E+ + E)
            je = cje * (z + 1) / (z - cjj)
        elif v.ade_kind == 1:  # Debye: J+ = cjj J + cje (E+ - E)
            je = cje * (z - 1) / (z - cjj)
        else:
            je = (cjen * z + cje + cjep / z) / (z - cjj - cjjp / z)
        jsum = jsum + (z + 1) / 2 * je
    del eps_inf_term
    return jsum / (EPS0 * (z - 1) / dt)


@pytest.mark.parametrize("name,mat,kind", [
    ("drude", X.DrudeMedium("d", 1.0, [2e10], [1e9]), 2),
    ("debye", X.DebyeMedium("b", 2.0, [6.0], [2e-11]), 1),
    ("drude_lorentz", configs.dispersive_material(), 3),
    ("lorentz", X.LorentzMedium("l", 1.5, [4.0], [3e10], [5e8]), 3),
])
def test_ade_discrete_susceptibility_matches_model(name, mat, kind):
    sim = configs.dispersive_sphere(cells=30, dl=1e-3, pml=5, precision="fp64", freqs=(), tfsf_inset=4,
                                    nf2ff_inset=2, radius=0.008, material=mat)
    h, v, gi = compile_sim(sim)
    assert v.ade_kind == kind
    assert gi.n_dispersive_cells > 0
    for f in (0.5e9, 2e9, 5e9):
        w = 2 * math.pi * f
        chi_num = numerical_eps_r(v, gi, 1, w)
        chi_ana = mat.relativePermittivity(f) - mat.prop.epsilon_r
        assert abs(chi_num - chi_ana) / abs(chi_ana) < 2e-3 * (1 + (w * gi.dt / 0.01) ** 2), (f, chi_num, chi_ana)


def test_ade_e_coefficients_consistent():
    mat = configs.dispersive_material()
    sim = configs.dispersive_sphere(cells=30, dl=1e-3, pml=5, precision="fp64", freqs=(), tfsf_inset=4,
                                    nf2ff_inset=2, radius=0.008, material=mat)
    h, v, gi = compile_sim(sim)
    am = np.ctypeslib.as_array(v.ade_mat, shape=(v.n_materials, 3))
    pole = np.ctypeslib.as_array(v.ade_pole, shape=(v.n_materials, v.ade_poles, 7))
    dt = gi.dt
    D = EPS0 / dt + pole[1, :, 2].sum() / 2
    assert am[1, 0] == 1 and am[0, 0] == 0
    assert am[1, 2] == pytest.approx(-1 / (2 * D), rel=1e-14)
    assert lut(v)[1][0] == pytest.approx((EPS0 / dt - pole[1, :, 3].sum() / 2) / D, rel=1e-14)
    np.testing.assert_allclose(pole[1, :, 5], 1 + pole[1, :, 0])


def dispersive_bounds(v, gi):
    ids = np.ctypeslib.as_array(v.material_id, shape=(gi.nx, gi.ny, gi.nz))
    am = np.ctypeslib.as_array(v.ade_mat, shape=(v.n_materials, 3))
    cells = np.argwhere(am[ids, 0] != 0)
    if len(cells) == 0:
        return [0] * 6
    lo, hi = cells.min(axis=0), cells.max(axis=0) + 1
    return [int(lo[0]), int(hi[0]), int(lo[1]), int(hi[1]), int(lo[2]), int(hi[2])]


@pytest.mark.parametrize("layout", ["sphere", "sphere_cut_by_cube", "two_spheres", "dispersive_fill", "none"])
def test_ade_box_is_the_dispersive_cell_bounds(layout):
    """The ADE box (storage of the recursions' state) equals the bounds of
    the cells that hold a dispersive material, however objects overlap."""
    mat = X.DrudeMedium("d", 1.0, [2e10], [1e9])
    s = X.Simulation(1e-3, 1e-3, 1e-3, 0.9)
    fill = mat if layout == "dispersive_fill" else X.Material.createAir()
    s.addObject(X.Object("domain", X.Cube(X.Vector(-0.02, -0.02, -0.02), X.Vector(0.04, 0.04, 0.04)), fill))
    if layout in ("sphere", "sphere_cut_by_cube", "two_spheres"):
        s.addObject(X.Object("s1", X.Sphere(X.Vector(0.003, -0.002, 0.001), 0.009), mat))
    if layout == "two_spheres":
        s.addObject(X.Object("s2", X.Sphere(X.Vector(-0.012, 0.01, 0.008), 0.004), mat))
    if layout == "sphere_cut_by_cube":  # a later object takes half of the sphere's cells
        s.addObject(X.Object("cut", X.Cube(X.Vector(-0.02, -0.02, -0.02), X.Vector(0.04, 0.04, 0.021)),
                             X.Material.createPec()))
    if layout == "dispersive_fill":  # an air block in a dispersive domain
        s.addObject(X.Object("hole", X.Cube(X.Vector(-0.01, -0.01, -0.01), X.Vector(0.02, 0.02, 0.02)),
                             X.Material.createAir()))
    h, v, gi = compile_sim(s)
    want = dispersive_bounds(v, gi)
    assert list(v.ade_box) == want
    if layout != "none":
        assert want[0] < want[1]
