"""Python side of the CPU restatement (TEST INFRASTRUCTURE, see xfb_oracle.c).

Only the test-suite, the smoke check and the bench's CPU-baseline leg use
this module, and only as the checker of the CUDA engine.

``OracleSim(handle, probes, movies)`` builds the CPU restatement from the same
compiled scene the engine uses (xfb_compiled_view), runs steps, and exposes
fields, probes, movies and NF2FF currents in the reference layout.
``far_field_numpy`` restates the NF2FF far-field integral (Balanis,
Advanced Engineering Electromagnetics, 2nd ed., eqs. 6.122-6.125) for the
surface currents; the reference delegates this step to XFDTD_CORE's
processFarField (test/dielectric_sphere_scatter.cu:85-91).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lib = None

EPSILON_0 = 8.854187817e-12
MU_0 = 4 * np.pi * 1e-7
C_0 = 1.0 / np.sqrt(EPSILON_0 * MU_0)
ETA_0 = np.sqrt(MU_0 / EPSILON_0)


def build() -> Path:
    src = HERE / "xfb_oracle.c"
    if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(str(LIB))
        lib.orc_create.restype = C.c_void_p
        lib.orc_create.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]
        lib.orc_run.restype = C.c_int
        lib.orc_run.argtypes = [C.c_void_p, C.c_longlong]
        for name in ("orc_field", "orc_field_mut", "orc_probe", "orc_movie"):
            getattr(lib, name).restype = C.POINTER(C.c_double)
            getattr(lib, name).argtypes = [C.c_void_p, C.c_int]
        lib.orc_nf2ff.restype = C.POINTER(C.c_double)
        lib.orc_nf2ff.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
        lib.orc_field_shape.argtypes = [C.c_void_p, C.c_int, C.c_int * 3]
        lib.orc_nf2ff_td.restype = C.POINTER(C.c_double)
        lib.orc_nf2ff_td.argtypes = [C.c_void_p, C.c_int]
        lib.orc_nf2ff_td_bins.restype = C.c_longlong
        lib.orc_nf2ff_td_bins.argtypes = [C.c_void_p]
        lib.orc_step.restype = C.c_longlong
        lib.orc_step.argtypes = [C.c_void_p]
        lib.orc_e_inc.restype = C.POINTER(C.c_double)
        lib.orc_e_inc.argtypes = [C.c_void_p]
        lib.orc_h_inc.restype = C.POINTER(C.c_double)
        lib.orc_h_inc.argtypes = [C.c_void_p]
        lib.orc_destroy.argtypes = [C.c_void_p]
        _lib = lib
    return _lib


class OracleSim:
    """CPU restatement of one scene.  ``handle`` is an engine Handle (host
    scene compiler only; no device needed) whose tables were sized with
    prepare_tables(total_steps) or init(total_steps)."""

    def __init__(self, handle, total_steps: int | None = None):
        self.lib = load()
        if total_steps is not None:
            handle.prepare_tables(total_steps)
        self.view = handle.compiled_view()
        self.total = self.view.total_steps
        sc_probes, sc_movies = self._monitors(handle)
        pr = (C.c_int * max(1, len(sc_probes)))(*sc_probes) if sc_probes else None
        mv = (C.c_int * max(1, len(sc_movies)))(*sc_movies) if sc_movies else None
        self.n_probes = len(sc_probes) // 4
        self.movie_desc = [sc_movies[8 * m: 8 * m + 8] for m in range(len(sc_movies) // 8)]
        self.s = self.lib.orc_create(C.byref(self.view), self.n_probes, pr, len(self.movie_desc), mv)
        self._handle = handle  # keep the compiled arrays alive

    @staticmethod
    def _monitors(handle):
        probes, movies = [], []
        for p in getattr(handle, "probe_desc", []):
            probes += list(p)
        for m in getattr(handle, "movie_desc", []):
            movies += list(m)
        return probes, movies

    def close(self):
        if getattr(self, "s", None):
            self.lib.orc_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, n: int):
        if self.lib.orc_run(self.s, int(n)) != 0:
            raise RuntimeError("oracle: steps beyond the sized run")

    @property
    def step(self) -> int:
        return int(self.lib.orc_step(self.s))

    def shape(self, f):
        s = (C.c_int * 3)()
        self.lib.orc_field_shape(self.s, f, s)
        return tuple(s)

    def field(self, f) -> np.ndarray:
        shp = self.shape(f)
        p = self.lib.orc_field(self.s, f)
        return np.ctypeslib.as_array(p, shape=shp).copy()

    def set_field(self, f, arr):
        shp = self.shape(f)
        p = self.lib.orc_field_mut(self.s, f)
        np.ctypeslib.as_array(p, shape=shp)[...] = arr

    def probe(self, p) -> np.ndarray:
        return np.ctypeslib.as_array(self.lib.orc_probe(self.s, p), shape=(self.total,))[: self.step].copy()

    def movie(self, m) -> np.ndarray:
        d = self.movie_desc[m]
        frames = (self.total + d[7] - 1) // d[7]
        shp = (frames, d[4] - d[1], d[5] - d[2], d[6] - d[3])
        return np.ctypeslib.as_array(self.lib.orc_movie(self.s, m), shape=shp).copy()

    def nf2ff(self, freq, face, which) -> np.ndarray:
        b = list(self.view.nf2ff_box)
        n = [b[1] - b[0], b[3] - b[2], b[5] - b[4]]
        n[face // 2] = 1
        a = np.ctypeslib.as_array(self.lib.orc_nf2ff(self.s, freq, face, which), shape=tuple(n) + (2,))
        return a[..., 0] + 1j * a[..., 1]

    def nf2ff_td(self, which) -> np.ndarray:
        """Time-domain NF2FF potential `which` (0..2 W_x..W_z, 3..5 U_x..U_z)."""
        n = int(self.lib.orc_nf2ff_td_bins(self.s))
        return np.ctypeslib.as_array(self.lib.orc_nf2ff_td(self.s, which), shape=(n,)).copy()

    def incident_tables(self):
        nl = self.view.aux_nl
        e = np.ctypeslib.as_array(self.lib.orc_e_inc(self.s), shape=(self.total, nl + 1)).copy()
        h = np.ctypeslib.as_array(self.lib.orc_h_inc(self.s), shape=(self.total, nl)).copy()
        return e, h


def far_field_numpy(currents, box, origin, d, freq, theta, phi):
    """Far field r*E (e^{-jkr} removed) from face currents.

    currents[face][w] (w = ja, jb, ma, mb) are complex arrays of the face
    extent; box = (is, ie, js, je, ks, ke); returns (E_theta, E_phi).
    N = sum J exp(+jk r.r') dS, L = sum M exp(+jk r.r') dS;
    E_theta = -jk/(4 pi) (L_phi + eta N_theta), E_phi = jk/(4 pi) (L_theta - eta N_phi).
    """
    theta = np.atleast_1d(np.asarray(theta, dtype=float))
    phi = np.atleast_1d(np.asarray(phi, dtype=float))
    theta, phi = np.broadcast_arrays(theta, phi)
    k = 2 * np.pi * freq / C_0
    st, ct, sp, cp = np.sin(theta), np.cos(theta), np.sin(phi), np.cos(phi)
    r = np.stack([st * cp, st * sp, ct], axis=-1)  # [n, 3]
    N = np.zeros((len(theta), 3), dtype=complex)
    Lm = np.zeros((len(theta), 3), dtype=complex)
    is_, ie, js, je, ks, ke = box
    comps = {0: (1, 2), 1: (2, 0), 2: (0, 1)}
    for face in range(6):
        ax, pos = face // 2, face % 2
        n = [ie - is_, je - js, ke - ks]
        n[ax] = 1
        idx = np.indices(n).reshape(3, -1).T.astype(float)  # local (i, j, k)
        start = [is_, js, ks]
        if pos:
            start[ax] = [ie, je, ke][ax]
        pos_xyz = np.empty_like(idx)
        for a in range(3):
            off = 0.0 if a == ax else 0.5
            pos_xyz[:, a] = origin[a] + (start[a] + idx[:, a] + off) * d[a]
        ds = np.prod([d[a] for a in range(3) if a != ax])
        ph = np.exp(1j * k * (r @ pos_xyz.T)) * ds  # [n_ang, n_pts]
        ca, cb = comps[ax]
        cur = [np.asarray(currents[face][w]).reshape(-1) for w in range(4)]
        N[:, ca] += ph @ cur[0]
        N[:, cb] += ph @ cur[1]
        Lm[:, ca] += ph @ cur[2]
        Lm[:, cb] += ph @ cur[3]
    n_th = N[:, 0] * ct * cp + N[:, 1] * ct * sp - N[:, 2] * st
    n_ph = -N[:, 0] * sp + N[:, 1] * cp
    l_th = Lm[:, 0] * ct * cp + Lm[:, 1] * ct * sp - Lm[:, 2] * st
    l_ph = -Lm[:, 0] * sp + Lm[:, 1] * cp
    f = k / (4 * np.pi)
    e_th = -1j * f * (l_ph + ETA_0 * n_th)
    e_ph = 1j * f * (l_th - ETA_0 * n_ph)
    return e_th, e_ph


def far_field_td_numpy(pot, theta, phi, dt):
    """r E_theta(t_n), r E_phi(t_n) from the time-domain NF2FF potentials
    pot[6] = (W_x, W_y, W_z, U_x, U_y, U_z) (time differences of the retarded
    surface-current integrals): Luebbers et al., "A finite-difference
    time-domain near zone to far zone transformation", IEEE Trans. Antennas
    Propag. 39(4), 1991: r E_theta = -(U_phi + eta W_theta) / (4 pi c dt),
    r E_phi = (U_theta - eta W_phi) / (4 pi c dt)."""
    c0 = 299792458.0
    wx, wy, wz, ux, uy, uz = pot
    st, ct, sp, cp = np.sin(theta), np.cos(theta), np.sin(phi), np.cos(phi)
    w_th = wx * ct * cp + wy * ct * sp - wz * st
    w_ph = -wx * sp + wy * cp
    u_th = ux * ct * cp + uy * ct * sp - uz * st
    u_ph = -ux * sp + uy * cp
    f = 1.0 / (4 * np.pi * c0 * dt)
    return -f * (u_ph + ETA_0 * w_th), f * (u_th - ETA_0 * w_ph)
