"""Shared helpers: build a scene twice (engine handle + CPU oracle) and compare."""
from __future__ import annotations

import numpy as np

import xfdtd_cuda_b200 as X
from oracle import OracleSim

FIELDS_3D = (0, 1, 2, 3, 4, 5)
FIELDS_2D = (2, 3, 4)


def engine(sim: X.Simulation, n_steps: int, graph=True, block=(32, 8, 1), path=0) -> X.Handle:
    sc, keep = sim.lower()
    h = X.Handle(sc, keep)
    h.set_kernel_path(path)
    h.set_launch_hint((1, 1, 1), block)
    h.set_graph(graph, 16)
    h.init(n_steps)
    return h


def oracle_of(sim: X.Simulation, n_steps: int) -> OracleSim:
    sc, keep = sim.lower()
    h = X.Handle(sc, keep)
    return OracleSim(h, n_steps)


def fields_of(obj, dim):
    names = FIELDS_3D if dim == 3 else FIELDS_2D
    if isinstance(obj, OracleSim):
        return {f: obj.field(f) for f in names}
    return {f: obj.read_field(f) for f in names}


def compare_fields(a, b):
    """max |a-b| / max |b| over all components."""
    worst = 0.0
    for f in b:
        scale = np.abs(b[f]).max()
        if scale == 0:
            worst = max(worst, float(np.abs(a[f]).max()))
            continue
        worst = max(worst, float(np.abs(a[f] - b[f]).max() / scale))
    return worst


def bit_equal(a, b):
    return all(np.array_equal(a[f], b[f]) for f in b)
