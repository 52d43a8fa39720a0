"""Generates the golden fixtures of tests/golden/ (run from the repository root:
python tests/golden/make_golden.py).

mie_sphere.npz   analytic bistatic radar cross-section sigma / lambda^2 of a
                 homogeneous sphere (Mie series, Bohren & Huffman, "Absorption
                 and Scattering of Light by Small Particles", eqs. 4.53, 4.74,
                 with the sphere's permeability mu_r) in the E-plane (S2) and
                 H-plane (S1) against the scattering angle: an independent
                 anchor for the whole engine path (scene compilation, TFSF,
                 Yee/CPML update, NF2FF accumulation, far field).
mie_dispersive.npz the same cross-section for the dispersive sphere of the
                 benchmark workload (radius 0.1 m; eps_inf = 1, a Drude pole
                 and a Lorentz pole) at 1, 3 and 5 GHz, with the complex
                 permittivity of the material model: an anchor for the ADE
                 path and the multi-frequency NF2FF.
oracle_small.npz probe series and field checksums of the CPU restatement on a
                 small FP64 dielectric sphere: pins the oracle against drift.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
from scipy import special

ROOT = Path(__file__).resolve().parents[2]
OUT = Path(__file__).resolve().parent
C0 = 299792458.0

# the Mie case: sphere of radius A, eps_r EPS, mu_r MU, at FREQ
A, EPS, MU, FREQ = 0.05, 3.0, 2.0, 1.0e9


def mie_s1_s2(x: float, m: complex, mu1: float, theta: np.ndarray, nmax: int | None = None):
    """Amplitude functions S1, S2 at scattering angles theta (radians) for size
    parameter x, relative refractive index m and relative permeability mu1 of
    the sphere (the medium has mu = 1)."""
    nmax = nmax or int(x + 4 * x ** (1 / 3) + 10)
    n = np.arange(1, nmax + 1)
    mx = m * x
    jx, djx = special.spherical_jn(n, x), special.spherical_jn(n, x, derivative=True)
    yx, dyx = special.spherical_yn(n, x), special.spherical_yn(n, x, derivative=True)
    jm, djm = special.spherical_jn(n, mx), special.spherical_jn(n, mx, derivative=True)
    hx, dhx = jx + 1j * yx, djx + 1j * dyx
    psi_x = jx + x * djx          # [x j_n(x)]'
    xi_x = hx + x * dhx           # [x h_n(x)]'
    psi_m = jm + mx * djm         # [mx j_n(mx)]'
    a = (m * m * jm * psi_x - mu1 * jx * psi_m) / (m * m * jm * xi_x - mu1 * hx * psi_m)
    b = (mu1 * jm * psi_x - jx * psi_m) / (mu1 * jm * xi_x - hx * psi_m)
    mu = np.cos(theta)
    pi = np.zeros((nmax + 1, len(theta)))
    tau = np.zeros((nmax + 1, len(theta)))
    pi[1] = 1.0
    tau[1] = mu
    for k in range(2, nmax + 1):
        pi[k] = (2 * k - 1) / (k - 1) * mu * pi[k - 1] - k / (k - 1) * pi[k - 2]
        tau[k] = k * mu * pi[k] - (k + 1) * pi[k - 1]
    f = ((2 * n + 1) / (n * (n + 1)))[:, None]
    s1 = np.sum(f * (a[:, None] * pi[1:] + b[:, None] * tau[1:]), axis=0)
    s2 = np.sum(f * (a[:, None] * tau[1:] + b[:, None] * pi[1:]), axis=0)
    return s1, s2


def make_mie():
    k = 2 * np.pi * FREQ / C0
    x = k * A
    m = np.sqrt(EPS * MU + 0j)
    theta = np.linspace(0.0, np.pi, 37)
    s1, s2 = mie_s1_s2(x, m, MU, theta)
    # sigma = 4 pi |S|^2 / k^2, in units of lambda^2 = (2 pi / k)^2
    norm = 4 * np.pi / k ** 2 / (2 * np.pi / k) ** 2
    np.savez(OUT / "mie_sphere.npz", theta=theta, sigma_e=norm * np.abs(s2) ** 2, sigma_h=norm * np.abs(s1) ** 2,
             radius=A, eps_r=EPS, mu_r=MU, freq=FREQ)


def make_mie_dispersive():
    sys.path.insert(0, str(ROOT))
    from xfdtd_cuda_b200 import configs
    mat = configs.dispersive_material()
    radius, freqs = 0.1, (1e9, 3e9, 5e9)
    theta = np.linspace(0.0, np.pi, 37)
    se, sh = [], []
    for f in freqs:
        k = 2 * np.pi * f / C0
        # the model's permittivity is in the exp(+j w t) convention; the
        # series (Bohren & Huffman) uses exp(-i w t): the conjugate
        m = np.sqrt(np.conj(complex(mat.relativePermittivity(f))))
        s1, s2 = mie_s1_s2(k * radius, m, 1.0, theta)
        norm = 4 * np.pi / k ** 2 / (2 * np.pi / k) ** 2
        se.append(norm * np.abs(s2) ** 2)
        sh.append(norm * np.abs(s1) ** 2)
    np.savez(OUT / "mie_dispersive.npz", theta=theta, sigma_e=np.array(se), sigma_h=np.array(sh), radius=radius,
             freqs=np.array(freqs))


def make_oracle_small():
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    import xfdtd_cuda_b200 as X
    from xfdtd_cuda_b200 import configs
    from oracle import OracleSim
    sim = configs.dielectric_sphere(cells=20, dl=5e-3, pml=4, precision="fp64", tfsf_inset=3, nf2ff_inset=2,
                                    freqs=(2e9,), radius=0.02,
                                    probes=[((0.0, 0.0, 0.0), 2), ((0.03, -0.02, 0.01), 1), ((-0.04, 0.03, 0.0), 5)])
    n = 80
    sc, keep = sim.lower()
    o = OracleSim(X.Handle(sc, keep), n)
    o.run(n)
    fields = [o.field(f) for f in range(6)]
    np.savez(OUT / "oracle_small.npz", steps=n, probes=np.stack([o.probe(p) for p in range(3)]),
             field_sum=np.array([f.sum() for f in fields]), field_abs=np.array([np.abs(f).sum() for f in fields]),
             nf2ff_xp_ja=o.nf2ff(0, 1, 0))


if __name__ == "__main__":
    make_mie()
    make_mie_dispersive()
    make_oracle_small()
    print("wrote", sorted(p.name for p in OUT.glob("*.npz")))
