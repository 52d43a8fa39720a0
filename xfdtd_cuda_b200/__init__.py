"""B200-native FDTD engine with the xfdtd::cuda::SimulationHD surface.

The time-stepping hot path (Yee update, CPML, TFSF, ADE dispersive media,
NF2FF accumulation, monitors) runs in hand-written CUDA kernels for sm_100a in
``libxfdtd_b200.so`` behind the C-ABI of ``include/xfdtd_b200.h``; this package
is the host-side scene API over that library.
"""
from ._lib import XfbError  # noqa: F401
from .simulation import (  # noqa: F401
    C_0, EPSILON_0, ETA_0, MU_0, EMF, Axis, Batch, Cube, Cylinder, DebyeMedium, DebyePole, DispersiveMaterial, DrudeMedium,
    DrudePole, ElectroMagneticProperty, FieldMonitor, Handle, LorentzMedium, LorentzPole, Material, MLorentzMaterial,
    MLorentzPole, MovieMonitor, NFFFTFrequencyDomain, NFFFTTimeDomain, Object, PML, PointMonitor, Simulation, SimulationHD, Sphere,
    TFSF2D, TFSF3D, Vector, Waveform,
)

__all__ = [n for n in dir() if not n.startswith("_")]
