"""Host-side scene API and the SimulationHD drop-in.

The reference's users build an XFDTD_CORE ``xfdtd::Simulation`` (objects,
boundaries, waveform sources, monitors, NF2FF) and hand it to
``xfdtd::cuda::SimulationHD`` (include/xfdtd_cuda/simulation/simulation_hd.cuh:37-88),
then call ``setGridDim``/``setBlockDim``/``run(n)`` (readme.md:100-145,
test/dielectric_sphere_scatter.cu:78-83).  This module keeps those names and
that flow; the scene is lowered to the C-ABI ``xfb_scene`` and every time step
runs in the CUDA library.  There is no CPU path: a missing library raises.

    s = Simulation(dl, dl, dl, 0.9)
    s.addObject(Object("domain", Cube(Vector(-0.175, -0.175, -0.175), Vector(0.35, 0.35, 0.35)), Material.createAir()))
    s.addObject(Object("sphere", Sphere(Vector(0, 0, 0), 0.1), Material("a", ElectroMagneticProperty(3, 2, 0, 0))))
    s.addWaveformSource(TFSF3D(15, 15, 15, 0, 0, 0, Waveform.gaussian(tau, t0)))
    for d in Axis.Direction.ALL: s.addBoundary(PML(8, d))
    nf = NFFFTFrequencyDomain(11, 11, 11, [1e9]); s.addNF2FF(nf)
    hd = SimulationHD(s); hd.setGridDim((4, 4, 4)); hd.setBlockDim((8, 8, 8)); hd.run(2400)
    e_theta, e_phi = nf.processFarField(np.linspace(-np.pi, np.pi, 360), 0.0, "xz")
"""
from __future__ import annotations

import ctypes as C
import math
import os
import time
from dataclasses import dataclass, field
from pathlib import Path
from typing import Sequence

import numpy as np

from . import _lib as L

EPSILON_0 = 8.854187817e-12
MU_0 = 4 * math.pi * 1e-7
C_0 = 1.0 / math.sqrt(EPSILON_0 * MU_0)
ETA_0 = math.sqrt(MU_0 / EPSILON_0)


@dataclass
class Vector:
    x: float
    y: float
    z: float

    def __iter__(self):
        return iter((self.x, self.y, self.z))


class Axis:
    class Direction:
        XN, XP, YN, YP, ZN, ZP = range(6)
        ALL = (0, 1, 2, 3, 4, 5)

    class XYZ:
        X, Y, Z = 0, 1, 2


class EMF:
    """XFDTD_CORE's EMF: the component enum and, after a SimulationHD run,
    the host field arrays ex ... hz in their Yee shapes (float64), filled by
    SimulationHD.copyDeviceToHost."""

    class Field:
        EX, EY, EZ, HX, HY, HZ = range(6)

    names = ("ex", "ey", "ez", "hx", "hy", "hz")

    def __init__(self):
        for n in self.names:
            setattr(self, n, None)

    def field(self, f: int):
        return getattr(self, self.names[f])


# ---- shapes ---------------------------------------------------------------
class Shape:
    def to_object(self, material: int) -> L.Object:
        raise NotImplementedError


class Cube(Shape):
    def __init__(self, origin: Vector, size: Vector):
        self.origin, self.size = origin, size

    def to_object(self, material):
        o = L.Object(shape=L.SHAPE_CUBE, material=material)
        for a, v in enumerate(list(self.origin) + list(self.size)):
            o.p[a] = v
        return o


class Sphere(Shape):
    def __init__(self, center: Vector, radius: float):
        self.center, self.radius = center, radius

    def to_object(self, material):
        o = L.Object(shape=L.SHAPE_SPHERE, material=material)
        for a, v in enumerate(list(self.center) + [self.radius]):
            o.p[a] = v
        return o


class Cylinder(Shape):
    """Circular cylinder; ``axis`` 0/1/2, ``length`` may be ``inf``."""

    def __init__(self, center: Vector, radius: float, length: float = math.inf, axis: int = 2):
        self.center, self.radius, self.length, self.axis = center, radius, length, axis

    def to_object(self, material):
        o = L.Object(shape=L.SHAPE_CYLINDER, material=material)
        for a, v in enumerate(list(self.center) + [self.radius, float(self.axis), self.length]):
            o.p[a] = v
        return o


# ---- materials --------------------------------------------------------------
@dataclass
class ElectroMagneticProperty:
    epsilon_r: float = 1.0
    mu_r: float = 1.0
    sigma_e: float = 0.0
    sigma_m: float = 0.0


@dataclass
class Pole:
    kind: int
    params: tuple

    def chi(self, omega: np.ndarray) -> np.ndarray:
        s = 1j * omega
        p = self.params
        if self.kind == L.POLE_DEBYE:
            return p[0] / (1 + s * p[1])
        if self.kind == L.POLE_DRUDE:
            return p[0] ** 2 / (s * p[1] + s * s)
        if self.kind == L.POLE_LORENTZ:
            return p[0] * p[1] ** 2 / (p[1] ** 2 + 2 * p[2] * s + s * s)
        a0, a1, b0, b1, b2 = p
        return (a0 + a1 * s) / (b0 + b1 * s + b2 * s * s)


def DebyePole(delta_eps, tau):
    return Pole(L.POLE_DEBYE, (delta_eps, tau))


def DrudePole(omega_p, gamma):
    return Pole(L.POLE_DRUDE, (omega_p, gamma))


def LorentzPole(delta_eps, omega_0, delta):
    return Pole(L.POLE_LORENTZ, (delta_eps, omega_0, delta))


def MLorentzPole(a0, a1, b0, b1, b2):
    return Pole(L.POLE_MLORENTZ, (a0, a1, b0, b1, b2))


class Material:
    def __init__(self, name: str, prop: ElectroMagneticProperty | None = None, pec: bool = False,
                 poles: Sequence[Pole] = ()):
        self.name = name
        self.prop = prop or ElectroMagneticProperty()
        self.pec = pec
        self.poles = list(poles)
        if len(self.poles) > L.MAX_POLES:
            raise ValueError(f"at most {L.MAX_POLES} poles per material")

    @staticmethod
    def createAir():
        return Material("air")

    @staticmethod
    def createPec():
        return Material("pec", pec=True)

    def relativePermittivity(self, freq) -> np.ndarray:
        w = 2 * np.pi * np.asarray(freq, dtype=float)
        eps = np.full(w.shape, self.prop.epsilon_r, dtype=complex)
        for p in self.poles:
            eps = eps + p.chi(w)
        if self.prop.sigma_e:
            eps = eps + self.prop.sigma_e / (1j * w * EPSILON_0)
        return eps

    def to_c(self) -> L.Material:
        m = L.Material(eps_r=self.prop.epsilon_r, mu_r=self.prop.mu_r, sigma_e=self.prop.sigma_e,
                       sigma_m=self.prop.sigma_m, is_pec=int(self.pec), n_poles=len(self.poles))
        for q, p in enumerate(self.poles):
            m.poles[q].kind = p.kind
            for a, v in enumerate(p.params):
                m.poles[q].p[a] = v
        return m


class DispersiveMaterial(Material):
    """Linear dispersive medium eps(w) = eps_inf + sum_p chi_p(w) (ADE)."""

    def __init__(self, name, eps_inf, poles, mu_r=1.0, sigma_e=0.0):
        super().__init__(name, ElectroMagneticProperty(eps_inf, mu_r, sigma_e, 0.0), poles=poles)


def DrudeMedium(name, eps_inf, omega_p, gamma):
    return DispersiveMaterial(name, eps_inf, [DrudePole(w, g) for w, g in zip(np.atleast_1d(omega_p), np.atleast_1d(gamma))])


def DebyeMedium(name, eps_inf, eps_static, tau):
    return DispersiveMaterial(name, eps_inf, [DebyePole(es - eps_inf, t) for es, t in zip(np.atleast_1d(eps_static), np.atleast_1d(tau))])


def LorentzMedium(name, eps_inf, eps_static, omega_p, nv):
    return DispersiveMaterial(name, eps_inf, [LorentzPole(es - eps_inf, w, d) for es, w, d in
                                              zip(np.atleast_1d(eps_static), np.atleast_1d(omega_p), np.atleast_1d(nv))])


class MLorentzMaterial:
    @staticmethod
    def makeMLorentz(name, eps_inf, a0, a1, b0, b1, b2):
        arrs = [np.atleast_1d(np.asarray(v, dtype=float)) for v in (a0, a1, b0, b1, b2)]
        n = max(len(a) for a in arrs)
        arrs = [np.broadcast_to(a, (n,)) for a in arrs]
        return DispersiveMaterial(name, eps_inf, [MLorentzPole(*(float(a[q]) for a in arrs)) for q in range(n)])


class Object:
    def __init__(self, name: str, shape: Shape, material: Material):
        self.name, self.shape, self.material = name, shape, material


# ---- sources, boundaries, monitors ------------------------------------------
class Waveform:
    def __init__(self, kind: int, tau: float, t0: float, freq: float = 0.0):
        self.kind, self.tau, self.t0, self.freq = kind, tau, t0, freq
        self._time = None

    @staticmethod
    def gaussian(tau, t0):
        """exp(-((t - t0) / tau)^2)"""
        return Waveform(L.WAVE_GAUSSIAN, tau, t0)

    @staticmethod
    def cosineModulatedGaussian(tau, t0, freq):
        """exp(-((t - t0) / tau)^2) cos(2 pi f (t - t0))"""
        return Waveform(L.WAVE_COS_GAUSSIAN, tau, t0, freq)

    def __call__(self, t):
        t = np.asarray(t, dtype=float)
        g = np.exp(-(((t - self.t0) / self.tau) ** 2))
        if self.kind == L.WAVE_COS_GAUSSIAN:
            g = g * np.cos(2 * np.pi * self.freq * (t - self.t0))
        return g

    def time(self):
        return self._time

    def value(self):
        return None if self._time is None else self(self._time)


class TFSF3D:
    """Plane-wave total-field/scattered-field box ``distance_*`` cells inside the domain."""

    def __init__(self, distance_x, distance_y, distance_z, theta, phi, psi, waveform: Waveform):
        self.inset = (int(distance_x), int(distance_y), int(distance_z))
        self.theta, self.phi, self.psi = theta, phi, psi
        self._waveform = waveform

    def waveform(self):
        return self._waveform


class TFSF2D(TFSF3D):
    def __init__(self, distance_x, distance_y, phi, waveform: Waveform):
        super().__init__(distance_x, distance_y, 0, math.pi / 2, phi, 0.0, waveform)


class PML:
    def __init__(self, thickness: int, direction: int, order_m: float = 3.0, sigma_ratio: float = 1.0,
                 alpha_max: float = 0.05):
        self.thickness, self.direction = int(thickness), int(direction)
        self.order_m, self.sigma_ratio, self.alpha_max = order_m, sigma_ratio, alpha_max

    def mainAxis(self):
        return self.direction // 2


class FieldMonitor:
    def __init__(self, shape: Shape, field_: int, name: str = "", out_dir: str = ""):
        self.shape, self._field, self.name, self.out_dir = shape, field_, name, out_dir

    def field(self):
        return self._field


class PointMonitor:
    """Time series of one field component at the node nearest to ``point``."""

    def __init__(self, point: Vector, field_: int, name: str = "", out_dir: str = ""):
        self.point, self._field, self.name, self.out_dir = point, field_, name, out_dir
        self.data: np.ndarray | None = None
        self.index = None

    def field(self):
        return self._field


class MovieMonitor:
    """Frames of one field component on a box every `frame_interval` steps.
    `index_box=(lo, hi)` gives the box in component indices (half-open)
    instead of the frame's physical shape."""

    def __init__(self, frame: FieldMonitor, frame_interval: int, name: str = "", out_dir: str = "", index_box=None):
        self._frame, self._interval, self.name, self.out_dir = frame, int(frame_interval), name, out_dir
        self.data: np.ndarray | None = None
        self.box = None
        self.index_box = index_box

    def frame(self):
        return self._frame

    def frameInterval(self):
        return self._interval

    def output(self):
        if self.data is None or not self.out_dir:
            return
        os.makedirs(self.out_dir, exist_ok=True)
        for t in range(self.data.shape[0]):
            np.save(Path(self.out_dir) / f"{t:05d}.npy", self.data[t])


class NFFFTFrequencyDomain:
    def __init__(self, distance_x, distance_y, distance_z, freqs, out_dir: str = ""):
        self.inset = (int(distance_x), int(distance_y), int(distance_z))
        self.freqs = np.atleast_1d(np.asarray(freqs, dtype=float))
        self.out_dir = out_dir
        self._hd: "SimulationHD | None" = None
        self.currents = None  # [freq][face][ja jb ma mb] complex arrays after run()

    def freqCount(self):
        return len(self.freqs)

    def setOutputDir(self, d: str):
        self.out_dir = d

    def equivalentSurfaceCurrent(self, face: int, which: int, freq_index: int) -> np.ndarray:
        return self.currents[freq_index][face][which]

    def processFarField(self, theta, phi, tag: str = "", freq_index: int | None = None):
        """Far field on the device; returns (E_theta, E_phi) of r*E, shape [n_freq, n_angles].

        ``theta`` and ``phi`` may each be a scalar or an array (broadcast),
        like XFDTD_CORE's processFarField(theta[], phi) / (theta, phi[]).
        Writes ``far_field_<tag>.npy`` under the output directory when set.
        """
        if self._hd is None:
            raise RuntimeError("run the simulation first")
        th, ph = np.broadcast_arrays(np.asarray(theta, dtype=float), np.asarray(phi, dtype=float))
        th = np.ascontiguousarray(th.ravel())
        ph = np.ascontiguousarray(ph.ravel())
        freqs = range(self.freqCount()) if freq_index is None else [freq_index]
        et, ep = [], []
        for f in freqs:
            a, b = self._hd.far_field(f, th, ph)
            et.append(a)
            ep.append(b)
        et, ep = np.array(et), np.array(ep)
        if self.out_dir and tag:
            os.makedirs(self.out_dir, exist_ok=True)
            np.save(Path(self.out_dir) / f"far_field_{tag}.npy",
                    {"theta": th, "phi": ph, "freqs": self.freqs, "e_theta": et, "e_phi": ep}, allow_pickle=True)
        return et, ep


class NFFFTTimeDomain:
    """Time-domain near-to-far-field transformation for one observation
    direction (the reference's NFFFTTimeDomain, constructed as in its sphere
    test: NFFFTTimeDomain(dx, dy, dz, out_dir, theta, phi))."""

    def __init__(self, distance_x, distance_y, distance_z, out_dir: str = "", theta: float = 0.0, phi: float = 0.0):
        self.inset = (int(distance_x), int(distance_y), int(distance_z))
        self.out_dir = out_dir
        self.theta, self.phi = float(theta), float(phi)
        self._hd: "SimulationHD | None" = None
        self.potentials = None  # [6][bins]: W_x W_y W_z U_x U_y U_z after run()

    def setOutputDir(self, d: str):
        self.out_dir = d

    def observationDirection(self):
        st = math.sin(self.theta)
        return Vector(st * math.cos(self.phi), st * math.sin(self.phi), math.cos(self.theta))

    def processFarField(self):
        """(t, r E_theta(t), r E_phi(t)) in the observation direction, t = n dt
        from the moment the wave leaves the box point farthest along it.
        Writes ``far_field_td.npy`` under the output directory when set."""
        if self._hd is None:
            raise RuntimeError("run the simulation first")
        et, ep = self._hd.handle.far_field_td()
        t = np.arange(len(et)) * self._hd.handle.info().dt
        if self.out_dir:
            os.makedirs(self.out_dir, exist_ok=True)
            np.save(Path(self.out_dir) / "far_field_td.npy",
                    {"t": t, "theta": self.theta, "phi": self.phi, "e_theta": et, "e_phi": ep}, allow_pickle=True)
        return t, et, ep


class Simulation:
    """Scene container with the XFDTD_CORE Simulation surface used by the reference drivers."""

    def __init__(self, dx, dy, dz, courant, thread_config=None, precision: str = "fp64"):
        self.dx, self.dy, self.dz, self.courant = float(dx), float(dy), float(dz), float(courant)
        self.precision = precision
        self.objects: list[Object] = []
        self.sources: list = []
        self.boundaries: list[PML] = []
        self.monitor_list: list = []
        self.nf2ff_list: list[NFFFTFrequencyDomain] = []
        self.dimension = 3
        self.emf = None  # host field arrays of the last SimulationHD run (EMF)

    def addObject(self, o: Object):
        self.objects.append(o)

    def addWaveformSource(self, w):
        self.sources.append(w)
        if isinstance(w, TFSF2D):
            self.dimension = 2

    def addBoundary(self, b: PML):
        self.boundaries.append(b)

    def addMonitor(self, m):
        self.monitor_list.append(m)

    def addNF2FF(self, n):
        """Add an NFFFTFrequencyDomain or an NFFFTTimeDomain (one of each at most)."""
        self.nf2ff_list.append(n)

    def monitors(self):
        return self.monitor_list

    def nf2ffs(self):
        return self.nf2ff_list

    def waveformSources(self):
        return self.sources

    def isRoot(self):
        return True

    # ---- lowering to the C-ABI -------------------------------------------
    def _domain(self):
        if not self.objects or not isinstance(self.objects[0].shape, Cube):
            raise ValueError("the first object must be the domain cube")
        return self.objects[0]

    def _dim(self):
        dom = self._domain().shape
        return 2 if (math.isinf(dom.size.z) or self.dimension == 2) else 3

    def lower(self):
        """Build the C scene; returns (scene, keep-alive list, index helpers)."""
        dim = self._dim()
        dom = self._domain().shape
        d = (self.dx, self.dy, self.dz if dim == 3 else 1.0)
        cells = [int(round(dom.size.x / d[0])), int(round(dom.size.y / d[1])), 1]
        lo = [dom.origin.x, dom.origin.y, 0.0]
        if dim == 3:
            cells[2] = int(round(dom.size.z / d[2]))
            lo[2] = dom.origin.z
        mats: list[Material] = []
        ids: dict[int, int] = {}

        def mid(m: Material) -> int:
            if id(m) not in ids:
                ids[id(m)] = len(mats)
                mats.append(m)
            return ids[id(m)]

        mid(self._domain().material)
        objs = [o.shape.to_object(mid(o.material)) for o in self.objects[1:]]
        cm = (L.Material * len(mats))(*[m.to_c() for m in mats])
        co = (L.Object * max(1, len(objs)))(*objs) if objs else (L.Object * 1)()
        sc = L.Scene()
        sc.dim = dim
        sc.precision = L.XFB_FP64 if self.precision == "fp64" else L.XFB_FP32
        sc.dx, sc.dy, sc.dz = d
        sc.courant = self.courant
        for a in range(3):
            sc.domain_min[a] = lo[a]
            sc.domain_cells[a] = cells[a]
        sc.n_materials, sc.materials = len(mats), cm
        sc.n_objects, sc.objects = len(objs), co
        pml_cfg = None
        for b in self.boundaries:
            sc.pml.cells[b.direction] = b.thickness
            pml_cfg = b
        if pml_cfg is not None:
            sc.pml.order_m, sc.pml.sigma_ratio, sc.pml.alpha_max = pml_cfg.order_m, pml_cfg.sigma_ratio, pml_cfg.alpha_max
        else:
            sc.pml.order_m, sc.pml.sigma_ratio, sc.pml.alpha_max = 3.0, 1.0, 0.05
        tf = next((w for w in self.sources if isinstance(w, TFSF3D)), None)
        if tf is not None:
            sc.tfsf.enabled = 1
            for a in range(3):
                sc.tfsf.inset[a] = tf.inset[a]
            sc.tfsf.theta, sc.tfsf.phi, sc.tfsf.psi = tf.theta, tf.phi, tf.psi
            w = tf.waveform()
            sc.tfsf.waveform, sc.tfsf.tau, sc.tfsf.t0, sc.tfsf.freq = w.kind, w.tau, w.t0, w.freq
        keep = [cm, co]
        td = next((n for n in self.nf2ff_list if isinstance(n, NFFFTTimeDomain)), None)
        if td is not None:
            sc.nf2ff_td.enabled = 1
            for a in range(3):
                sc.nf2ff_td.inset[a] = td.inset[a]
            sc.nf2ff_td.theta, sc.nf2ff_td.phi = td.theta, td.phi
        fds = [n for n in self.nf2ff_list if isinstance(n, NFFFTFrequencyDomain)]
        if fds:
            nf = fds[0]
            fr = (C.c_double * len(nf.freqs))(*nf.freqs)
            keep.append(fr)
            sc.nf2ff.enabled = 1
            for a in range(3):
                sc.nf2ff.inset[a] = nf.inset[a]
            sc.nf2ff.n_freqs = len(nf.freqs)
            sc.nf2ff.freqs = fr
        pml = [b.thickness if b else 0 for b in [None] * 6]
        for b in self.boundaries:
            pml[b.direction] = b.thickness
        origin = [lo[0] - pml[0] * d[0], lo[1] - pml[2] * d[1], (lo[2] - pml[4] * d[2]) if dim == 3 else 0.0]
        n_tot = [cells[0] + pml[0] + pml[1], cells[1] + pml[2] + pml[3], cells[2] + pml[4] + pml[5]]

        def comp_shape(f):
            s = [n_tot[0] + (f in (L.EY, L.EZ, L.HX)), n_tot[1] + (f in (L.EX, L.EZ, L.HY)),
                 n_tot[2] + (f in (L.EX, L.EY, L.HZ))]
            if dim == 2:
                s[2] = 1
            return s

        probes, movies = [], []
        for m in self.monitor_list:
            if isinstance(m, PointMonitor):
                shp = comp_shape(m.field())
                idx = [int(round((v - o) / dd)) for v, o, dd in zip(m.point, origin, d)]
                idx = [min(max(0, i), s - 1) for i, s in zip(idx, shp)]
                if dim == 2:
                    idx[2] = 0
                m.index = idx
                probes.append(L.Probe(field=m.field(), index=(C.c_int * 3)(*idx)))
            elif isinstance(m, MovieMonitor):
                fm = m.frame()
                cube = fm.shape
                shp = comp_shape(fm.field())
                lo_i, hi_i = [], []
                for a in range(3 if m.index_box is None else 0):
                    if dim == 2 and a == 2:
                        lo_i.append(0); hi_i.append(1)
                        continue
                    org = list(cube.origin)[a]
                    sz = list(cube.size)[a]
                    l0 = 0 if math.isinf(org) else int(round((org - origin[a]) / d[a]))
                    h0 = shp[a] if math.isinf(sz) else int(round((org + sz - origin[a]) / d[a]))
                    l0 = min(max(0, l0), shp[a] - 1)
                    h0 = min(max(l0 + 1, h0), shp[a])
                    lo_i.append(l0); hi_i.append(h0)
                if m.index_box is not None:
                    for a in range(3):
                        l0 = min(max(0, int(m.index_box[0][a])), shp[a] - 1)
                        lo_i.append(l0)
                        hi_i.append(min(max(l0 + 1, int(m.index_box[1][a])), shp[a]))
                m.box = (lo_i, hi_i)
                movies.append(L.Movie(field=fm.field(), lo=(C.c_int * 3)(*lo_i), hi=(C.c_int * 3)(*hi_i),
                                      interval=m.frameInterval()))
        if probes:
            arr = (L.Probe * len(probes))(*probes)
            keep.append(arr)
            sc.n_probes, sc.probes = len(probes), arr
        if movies:
            arr = (L.Movie * len(movies))(*movies)
            keep.append(arr)
            sc.n_movies, sc.movies = len(movies), arr
        return sc, keep


class Handle:
    """Owns one engine handle (xfb_handle*)."""

    def __init__(self, scene: L.Scene, keep=()):
        self.lib = L.load()
        self._keep = list(keep)
        self.probe_desc = [(scene.probes[q].field, *scene.probes[q].index) for q in range(scene.n_probes)]
        self.movie_desc = [(scene.movies[q].field, *scene.movies[q].lo, *scene.movies[q].hi, scene.movies[q].interval)
                           for q in range(scene.n_movies)]
        h = C.c_void_p()
        L.check(self.lib.xfb_create(C.byref(scene), C.byref(h)))
        self.h = h

    @classmethod
    def from_core_arrays(cls, arrays: L.CoreArrays, keep=()):
        """A handle from a scene XFDTD_CORE compiled (xfb_create_from_arrays);
        `keep` holds the numpy arrays the struct points into."""
        self = cls.__new__(cls)
        self.lib = L.load()
        self._keep = list(keep)
        self.probe_desc = [(arrays.probes[q].field, *arrays.probes[q].index) for q in range(arrays.n_probes)]
        self.movie_desc = [(arrays.movies[q].field, *arrays.movies[q].lo, *arrays.movies[q].hi, arrays.movies[q].interval)
                           for q in range(arrays.n_movies)]
        h = C.c_void_p()
        L.check(self.lib.xfb_create_from_arrays(C.byref(arrays), C.byref(h)))
        self.h = h
        return self

    def close(self):
        if getattr(self, "h", None):
            self.lib.xfb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, status):
        L.check(status, self.h)

    def info(self) -> L.GridInfo:
        gi = L.GridInfo()
        self._c(self.lib.xfb_get_grid_info(self.h, C.byref(gi)))
        return gi

    def shape(self, f):
        gi = self.info()
        s = [gi.nx + (f in (L.EY, L.EZ, L.HX)), gi.ny + (f in (L.EX, L.EZ, L.HY)), gi.nz + (f in (L.EX, L.EY, L.HZ))]
        if gi.dim == 2:
            s[2] = 1
        return tuple(s)

    def set_launch_hint(self, grid, block):
        g = (C.c_uint * 3)(*grid)
        b = (C.c_uint * 3)(*block)
        self._c(self.lib.xfb_set_launch_hint(self.h, g, b))

    def set_device(self, ordinal: int):
        self._c(self.lib.xfb_set_device(self.h, int(ordinal)))

    def set_kernel_path(self, path: int):
        self._c(self.lib.xfb_set_kernel_path(self.h, int(path)))

    def set_temporal_block(self, steps: int):
        """Steps per launch of the blocked 2-D kernel (odd; 0: one launch per step)."""
        self._c(self.lib.xfb_set_temporal_block(self.h, int(steps)))

    def set_coeff_storage(self, storage: int):
        """Round the coefficient LUT to FP16 / BF16 at init (storage trial)."""
        self._c(self.lib.xfb_set_coeff_storage(self.h, int(storage)))

    def set_graph(self, enabled: bool, steps: int = 64):
        self._c(self.lib.xfb_set_graph(self.h, int(enabled), int(steps)))

    def init(self, n):
        self._c(self.lib.xfb_init(self.h, int(n)))

    def run(self, n):
        self._c(self.lib.xfb_run(self.h, int(n)))

    def step(self, n):
        self._c(self.lib.xfb_step(self.h, int(n)))

    def sync(self):
        self._c(self.lib.xfb_sync(self.h))

    def set_wait_limit(self, polls: int):
        """Poll limit of the step kernel's bounded staging waits (diagnostics)."""
        self._c(self.lib.xfb_set_wait_limit(self.h, int(polls)))

    def timed_step(self, n) -> float:
        ms = C.c_double()
        self._c(self.lib.xfb_timed_step(self.h, int(n), C.byref(ms)))
        return ms.value

    def profile_kernels(self, n):
        ms = (C.c_double * L.K_COUNT)()
        cnt = (C.c_longlong * L.K_COUNT)()
        self._c(self.lib.xfb_profile_kernels(self.h, int(n), ms, cnt))
        return list(ms), list(cnt)

    def read_field(self, f, out: np.ndarray | None = None) -> np.ndarray:
        """Component f (reference shape, float64); into `out` when given."""
        s = self.shape(f)
        if out is None:
            out = np.empty(s, dtype=np.float64)
        elif out.shape != s or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous float64 array of shape {s}")
        self._c(self.lib.xfb_read_field(self.h, f, out.ctypes.data_as(L._dp), out.size))
        self._prefault_keep = []
        return out

    def prefault(self, arr: np.ndarray):
        """Fault in the pages of a result array on background host threads
        (xfb_host_prefault) while the device works; the array is kept alive
        until the next read."""
        if not hasattr(self, "_prefault_keep"):
            self._prefault_keep = []
        self._prefault_keep.append(arr)
        self._c(self.lib.xfb_host_prefault(self.h, arr.ctypes.data, arr.nbytes))

    def prefault_wait(self):
        self._c(self.lib.xfb_host_prefault_wait(self.h))
        self._prefault_keep = []

    def write_field(self, f, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        if arr.shape != self.shape(f):
            raise ValueError(f"shape {arr.shape} != {self.shape(f)}")
        self._c(self.lib.xfb_write_field(self.h, f, arr.ctypes.data_as(L._dp), arr.size))

    def read_probe(self, p) -> np.ndarray:
        gi = self.info()
        out = np.empty(max(1, gi.current_step), dtype=np.float64)
        n = C.c_longlong()
        self._c(self.lib.xfb_read_probe(self.h, p, out.ctypes.data_as(L._dp), out.size, C.byref(n)))
        return out[: n.value]

    def read_movie(self, m) -> np.ndarray:
        s = (C.c_int * 4)()
        self._c(self.lib.xfb_movie_shape(self.h, m, s))
        out = np.empty(tuple(s), dtype=np.float64)
        self._c(self.lib.xfb_read_movie(self.h, m, out.ctypes.data_as(L._dp), out.size))
        return out

    def nf2ff_face_shape(self, face) -> tuple:
        s = (C.c_int * 3)()
        self._c(self.lib.xfb_nf2ff_face_shape(self.h, face, s))
        return tuple(s)

    def read_nf2ff(self, freq, face, which, out: np.ndarray | None = None) -> np.ndarray:
        """Surface current `which` (J_a, J_b, M_a, M_b) of one face and
        frequency, complex128 (the library's interleaved re/im pairs are
        numpy's complex layout); into `out` when given."""
        s = self.nf2ff_face_shape(face)
        if out is None:
            out = np.empty(s, dtype=np.complex128)
        elif out.shape != s or out.dtype != np.complex128 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous complex128 array of shape {s}")
        self._c(self.lib.xfb_read_nf2ff(self.h, freq, face, which, out.ctypes.data_as(L._dp), 2 * out.size))
        self._prefault_keep = []
        return out

    def read_nf2ff_all(self, freq, out: np.ndarray | None = None) -> np.ndarray:
        """All surface currents of one frequency in one read: complex128
        [4 (J_a, J_b, M_a, M_b), points], the six faces one after another
        (nf2ff_split cuts them into per-face arrays); into `out` when given."""
        pts = C.c_longlong()
        n = sum(int(np.prod(self.nf2ff_face_shape(f))) for f in range(6))
        if out is None:
            out = np.empty((4, n), dtype=np.complex128)
        elif out.shape != (4, n) or out.dtype != np.complex128 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous complex128 array of shape {(4, n)}")
        self._c(self.lib.xfb_read_nf2ff_all(self.h, freq, out.ctypes.data_as(L._dp), 2 * out.size, C.byref(pts)))
        self._prefault_keep = []
        return out

    def nf2ff_split(self, cur: np.ndarray):
        """[face][which] views (face shapes) into a read_nf2ff_all array."""
        res, o = [], 0
        for face in range(6):
            s = self.nf2ff_face_shape(face)
            m = int(np.prod(s))
            res.append([cur[w, o:o + m].reshape(s) for w in range(4)])
            o += m
        return res

    def far_field(self, freq, theta, phi):
        th = np.ascontiguousarray(theta, dtype=np.float64)
        ph = np.ascontiguousarray(phi, dtype=np.float64)
        out = np.empty((len(th), 4), dtype=np.float64)
        self._c(self.lib.xfb_far_field(self.h, freq, len(th), th.ctypes.data_as(L._dp), ph.ctypes.data_as(L._dp),
                                       out.ctypes.data_as(L._dp)))
        return out[:, 0] + 1j * out[:, 1], out[:, 2] + 1j * out[:, 3]

    def read_nf2ff_td(self, which) -> np.ndarray:
        """Time-domain NF2FF potential `which` (0..2 W_x..W_z, 3..5 U_x..U_z)."""
        n = C.c_longlong()
        self._c(self.lib.xfb_nf2ff_td_bins(self.h, C.byref(n)))
        out = np.empty(n.value, dtype=np.float64)
        self._c(self.lib.xfb_read_nf2ff_td(self.h, which, out.ctypes.data_as(L._dp), out.size))
        return out

    def far_field_td(self):
        """(r E_theta(t_n), r E_phi(t_n)) of the time-domain NF2FF."""
        n = C.c_longlong()
        self._c(self.lib.xfb_nf2ff_td_bins(self.h, C.byref(n)))
        et = np.empty(n.value, dtype=np.float64)
        ep = np.empty(n.value, dtype=np.float64)
        self._c(self.lib.xfb_far_field_td(self.h, et.ctypes.data_as(L._dp), ep.ctypes.data_as(L._dp), n.value))
        return et, ep

    def set_learned_abc(self, weights):
        """Learned absorbing boundary on every wall (3-D one-sweep scene
        without CPML, after init); None switches it off."""
        if weights is None:
            self._c(self.lib.xfb_set_learned_abc(self.h, None, 0))
            return
        w = np.ascontiguousarray(weights, dtype=np.float32)
        self._c(self.lib.xfb_set_learned_abc(self.h, w.ctypes.data_as(C.POINTER(C.c_float)), w.size))

    def far_field_static(self, freq, theta, phi):
        """xfb_far_field without device allocation (fixed device scratch of the
        library, at most FAR_FIELD_STATIC_MAX_ANGLES angles per call)."""
        th = np.ascontiguousarray(theta, dtype=np.float64)
        ph = np.ascontiguousarray(phi, dtype=np.float64)
        out = np.empty((len(th), 4), dtype=np.float64)
        self._c(self.lib.xfb_far_field_static(self.h, freq, len(th), th.ctypes.data_as(L._dp),
                                              ph.ctypes.data_as(L._dp), out.ctypes.data_as(L._dp)))
        return out[:, 0] + 1j * out[:, 1], out[:, 2] + 1j * out[:, 3]

    def get_state(self) -> bytes:
        n = C.c_size_t()
        self._c(self.lib.xfb_state_size(self.h, C.byref(n)))
        buf = C.create_string_buffer(n.value)
        self._c(self.lib.xfb_get_state(self.h, buf, n.value))
        return buf.raw

    def set_state(self, data: bytes):
        buf = C.create_string_buffer(data, len(data))
        self._c(self.lib.xfb_set_state(self.h, buf, len(data)))

    def check_finite(self) -> int:
        bad = C.c_longlong()
        st = self.lib.xfb_check_finite(self.h, C.byref(bad))
        if st not in (L.XFB_OK, L.XFB_ERR_NUMERIC):
            self._c(st)
        return bad.value

    def compiled_view(self) -> L.CompiledView:
        v = L.CompiledView()
        self._c(self.lib.xfb_compiled_view_get(self.h, C.byref(v)))
        return v

    def prepare_tables(self, n):
        self._c(self.lib.xfb_prepare_tables(self.h, int(n)))


class Batch:
    """Steps many 3-D scenes of one precision together (xfb_batch_*): one
    launch of the one-sweep kernel per step over the work items of every
    scene, or one persistent launch per chunk of steps (``launch``:
    L.BATCH_AUTO picks the faster on the first steps).  The Handles stay
    usable for read-back after ``sync()``."""

    def __init__(self, handles, tile_rows: int = 0, launch: int = L.BATCH_AUTO):
        self.lib = L.load()
        self.handles = list(handles)
        arr = (C.c_void_p * len(self.handles))(*[h.h for h in self.handles])
        b = C.c_void_p()
        st = self.lib.xfb_batch_create(arr, len(self.handles), C.byref(b))
        if st != L.XFB_OK:
            raise L.XfbError(st, self.lib.xfb_last_error(None).decode())
        self.b = b
        self._c(self.lib.xfb_batch_set_tile(self.b, tile_rows))
        self._c(self.lib.xfb_batch_set_launch(self.b, launch))

    def _c(self, status):
        if status != L.XFB_OK:
            raise L.XfbError(status, self.lib.xfb_batch_last_error(self.b).decode())

    def init(self, total_steps: int):
        self._c(self.lib.xfb_batch_init(self.b, total_steps))

    def step(self, n: int):
        self._c(self.lib.xfb_batch_step(self.b, n))

    def sync(self):
        self._c(self.lib.xfb_batch_sync(self.b))

    def set_wait_limit(self, polls: int):
        """Poll limit of the batch step's bounded staging waits (diagnostics)."""
        self._c(self.lib.xfb_batch_set_wait_limit(self.b, int(polls)))

    def timed_step(self, n: int) -> float:
        ms = C.c_double()
        self._c(self.lib.xfb_batch_timed_step(self.b, n, C.byref(ms)))
        return ms.value

    def info(self):
        cells, rows, items = C.c_longlong(), C.c_int(), C.c_int()
        self._c(self.lib.xfb_batch_info(self.b, C.byref(cells), C.byref(rows), C.byref(items)))
        form = C.c_int()
        self._c(self.lib.xfb_batch_launch_form(self.b, C.byref(form)))
        return {"cells": cells.value, "tile_rows": rows.value, "work_items": items.value,
                "launch": {0: "unchosen", 1: "per_step", 2: "persistent"}[form.value]}

    def close(self):
        if getattr(self, "b", None):
            self.lib.xfb_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SimulationHD:
    """Drop-in for ``xfdtd::cuda::SimulationHD`` (simulation_hd.cuh:37-88).

    init(n) compiles the host scene, allocates the host result arrays (the
    fields in ``host().emf``, the NF2FF surface currents), as XFDTD_CORE's
    Simulation::init does, and uploads the device state; background host
    threads fault in the result arrays' pages meanwhile and while the device
    steps.
    copyDeviceToHost() fills them, as the reference copies results back into
    the host objects (simulation_hd.cu:228-247)."""

    def __init__(self, host: Simulation):
        self._host = host
        self._grid = (1, 1, 1)
        self._block = (1, 1, 1)
        self.handle: Handle | None = None
        self.device = None        # CUDA ordinal (None: the current device)
        self.kernel_path = None   # xfb_set_kernel_path value (None: automatic)
        self.timings = {}

    def setDevice(self, ordinal: int):
        self.device = int(ordinal)

    def host(self):
        return self._host

    def setGridDim(self, g):
        self._grid = tuple(int(v) for v in g)

    def setBlockDim(self, b):
        self._block = tuple(int(v) for v in b)

    def init(self, time_step: int):
        t0 = time.perf_counter()
        sc, keep = self._host.lower()
        if self.handle is not None:
            self.handle.close()
        self.handle = Handle(sc, keep)
        t1 = time.perf_counter()
        if self.device is not None:
            self.handle.set_device(self.device)
        if self.kernel_path is not None:
            self.handle.set_kernel_path(self.kernel_path)
        self.handle.set_launch_hint(self._grid, self._block)
        # the host result arrays' pages are faulted in by host threads while
        # the device state is set up and stepped
        self._alloc_host_results()
        self.prefaultHostResults()
        self.handle.init(time_step)
        self.timings = {"compile": t1 - t0, "init": time.perf_counter() - t1}
        gi = self.handle.info()
        for w in self._host.sources:
            if isinstance(w, TFSF3D):
                w.waveform()._time = (np.arange(time_step) + 1) * gi.dt

    def run(self, time_step: int):
        """Reference run(n): initialise, advance n steps, copy results back
        into the host objects.  The pages of the host result arrays are
        faulted in on host threads while the device initialises and steps."""
        self.init(time_step)
        self.handle.step(time_step)
        self.handle.sync()
        self.copyDeviceToHost()

    def prefaultHostResults(self):
        """Start faulting in the host result arrays on background host threads
        (xfb_host_prefault); the next read joins them.  init() starts it; a
        second call before the next read queues nothing."""
        if getattr(self.handle, "_prefault_keep", None):
            return
        emf = self._host.emf
        for f in range(6):
            a = emf.field(f) if emf is not None else None
            if a is not None:
                self.handle.prefault(a)
        for a in self._nf_out or ():
            self.handle.prefault(a)

    def _alloc_host_results(self):
        h = self.handle
        gi = h.info()
        emf = EMF()
        for f in ((L.EZ, L.HX, L.HY) if gi.dim == 2 else range(6)):
            setattr(emf, EMF.names[f], np.empty(h.shape(f), dtype=np.float64))
        self._host.emf = emf
        self._nf_out = None
        if gi.n_freqs:
            n = sum(int(np.prod(h.nf2ff_face_shape(face))) for face in range(6))
            self._nf_out = [np.empty((4, n), dtype=np.complex128) for _ in range(gi.n_freqs)]

    def copyHostToDevice(self):
        pass  # buffers are uploaded by init()

    def copyDeviceToHost(self):
        h = self.handle
        emf = self._host.emf
        for f in range(6):
            a = emf.field(f)
            if a is not None:
                h.read_field(f, out=a)
        pi = mi = 0
        for m in self._host.monitor_list:
            if isinstance(m, PointMonitor):
                m.data = h.read_probe(pi)
                pi += 1
            elif isinstance(m, MovieMonitor):
                m.data = h.read_movie(mi)
                mi += 1
                m.output()
        for nf in self._host.nf2ff_list:
            nf._hd = self
            if isinstance(nf, NFFFTTimeDomain):
                nf.potentials = [h.read_nf2ff_td(w) for w in range(6)]
                continue
            nf.currents = [h.nf2ff_split(h.read_nf2ff_all(f, out=self._nf_out[f] if self._nf_out else None))
                           for f in range(nf.freqCount())]

    def releaseDevice(self):
        if self.handle is not None:
            self.handle.close()
            self.handle = None

    def field(self, f) -> np.ndarray:
        return self.handle.read_field(f)

    def far_field(self, freq, theta, phi):
        return self.handle.far_field(freq, theta, phi)
