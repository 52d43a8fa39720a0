"""x-slab decomposition of one grid.

CPU: the partition (balanced, every inner boundary's lower plane outside the x
CPML) and the halo-exchange schedule of slabs.exchange on two and three gloo
ranks: a leapfrog stencil over x with the engine's halo pattern (each slab
recomputes the H plane below it from the E and H halos; the lower halo is the
lower neighbour's last plane, the upper halo the upper neighbour's first)
matches the undivided run bit for bit.

GPU: slabs of one scene stepped by a SlabGroup on one device (update, peer
copies, record) against the same scene on one handle, FP64: fields, probes,
movie frames and NF2FF currents (frequency and time domain) bit-identical,
with CPML, TFSF, ADE media and NF2FF boxes crossing the slab boundaries.
"""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

import xfdtd_cuda_b200 as X
from xfdtd_cuda_b200 import _lib as L
from xfdtd_cuda_b200 import configs, slabs

ROOT = Path(__file__).resolve().parents[1]


def test_partition_balanced_and_outside_x_cpml():
    for nx, n, lo, hi in ((156, 2, 8, 8), (156, 3, 8, 8), (408, 8, 12, 12), (40, 4, 6, 6), (30, 5, 0, 0)):
        r = slabs.partition(nx, n, lo, hi)
        assert r[0][0] == 0 and r[-1][1] == nx and len(r) == n
        assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
        for i0, _ in r[1:]:
            assert lo <= i0 - 1 < nx - hi
        sizes = [b - a for a, b in r]
        assert max(sizes) - min(sizes) <= 1 or (lo and max(sizes) - min(sizes) <= lo + 1)
    with pytest.raises(ValueError):
        slabs.partition(20, 12, 8, 8)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _leapfrog_full(e, h, steps):
    e, h = e.copy(), h.copy()
    n = e.shape[0]
    for _ in range(steps):
        h[: n - 1] = h[: n - 1] + 0.5 * (e[1:] - e[: n - 1])
        e[1 : n - 1] = e[1 : n - 1] + 0.5 * (h[1 : n - 1] - h[: n - 2])
    return e, h


def _rank_main(rank, world, port, steps, out):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    from xfdtd_cuda_b200 import slabs as S
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    rng = np.random.default_rng(5)
    n = 23
    e0, h0 = rng.standard_normal((n, 4)), rng.standard_normal((n, 4))
    i0, i1 = S.partition(n - 1, world)[rank]  # cells 0..n-2, E nodes 0..n-1
    # local planes i0-1 .. i1 (halos included), global plane p at local p - i0 + 1
    lo = i0 - 1
    e = torch.zeros((i1 - lo + 1, 4), dtype=torch.float64)
    h = torch.zeros_like(e)
    for p in range(max(lo, 0), min(i1, n - 1) + 1):
        e[p - lo] = torch.from_numpy(e0[p])
        h[p - lo] = torch.from_numpy(h0[p])
    for _ in range(steps):
        # H of planes i0-1 .. i1-1 (the plane below recomputed from the halos), E of i0 .. i1-1
        for p in range(max(i0 - 1, 0), i1):
            h[p - lo] = h[p - lo] + 0.5 * (e[p + 1 - lo] - e[p - lo])
        for p in range(max(i0, 1), min(i1, n - 1)):
            e[p - lo] = e[p - lo] + 0.5 * (h[p - lo] - h[p - 1 - lo])
        send_down = [e[i0 - lo].clone(), h[i0 - lo].clone()]
        send_up = [e[i1 - 1 - lo].clone(), h[i1 - 1 - lo].clone()]
        recv_below = [torch.empty(4, dtype=torch.float64) for _ in range(2)]
        recv_above = [torch.empty(4, dtype=torch.float64) for _ in range(2)]
        S.exchange(send_down, send_up, recv_below, recv_above, rank, world, dist)
        if rank > 0:
            e[0], h[0] = recv_below
        if rank + 1 < world:
            e[i1 - lo], h[i1 - lo] = recv_above
    out.put((rank, i0, i1, e.numpy().copy(), h.numpy().copy()))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_exchange_schedule_gloo(world):
    steps = 9
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, steps, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rng = np.random.default_rng(5)
    n = 23
    e_ref, h_ref = _leapfrog_full(rng.standard_normal((n, 4)), rng.standard_normal((n, 4)), steps)
    for rank, i0, i1, e, h in res:
        lo = i0 - 1
        top = i1 + 1 if rank + 1 == world else i1  # the last slab also holds node plane n-1
        for p in range(i0, min(top, n)):
            assert np.array_equal(e[p - lo], e_ref[p]), (rank, p)
            if p < n - 1:
                assert np.array_equal(h[p - lo], h_ref[p]), (rank, p)


gpu = pytest.mark.gpu


def _dielectric(prec="fp64"):
    sim = configs.dielectric_sphere(cells=28, dl=5e-3, pml=5, precision=prec, tfsf_inset=4, nf2ff_inset=2,
                                    radius=0.03, freqs=(2e9,),
                                    probes=[((0.0, 0.0, 0.0), L.EZ), ((-0.04, 0.01, 0.0), L.HY), ((0.05, -0.02, 0.03), L.EX)])
    sim.addNF2FF(X.NFFFTTimeDomain(2, 2, 2, "", 0.7, 1.9))
    from xfdtd_cuda_b200.simulation import Cube, FieldMonitor, MovieMonitor, Vector
    sim.addMonitor(MovieMonitor(FieldMonitor(Cube(Vector(-0.07, -0.07, 0.0), Vector(0.14, 0.14, 0.005)), L.EZ), 7))
    sim.addMonitor(MovieMonitor(FieldMonitor(Cube(Vector(-0.07, 0.0, -0.07), Vector(0.14, 0.005, 0.14)), L.HY), 5))
    return sim


def _dispersive():
    return configs.dispersive_sphere(cells=36, dl=3e-3, pml=6, precision="fp64", freqs=(2e9,), tfsf_inset=4,
                                     nf2ff_inset=2, radius=0.03, probes=[((0.0, 0.0, 0.0), L.EX)])


def _whole(sim, steps):
    sc, keep = sim.lower()
    h = X.Handle(sc, keep)
    h.init(steps)
    h.step(steps)
    h.sync()
    return h


@gpu
@pytest.mark.parametrize("scene,n", [("dielectric", 2), ("dielectric", 3), ("dispersive", 2)])
def test_slab_group_matches_whole_grid_fp64(scene, n):
    steps = 60
    build = _dielectric if scene == "dielectric" else _dispersive
    ref = _whole(build(), steps)
    g = slabs.SlabGroup(build(), n, devices=(0,), total_steps=steps)
    g.step(steps)
    g.sync()
    for f in range(6):
        assert np.array_equal(g.read_field(f), ref.read_field(f)), f"field {f}"
    for p in range(len(ref.probe_desc)):
        assert np.array_equal(g.read_probe(p), ref.read_probe(p)), f"probe {p}"
    for face in range(6):
        for w in range(4):
            assert np.array_equal(g.read_nf2ff(0, face, w), ref.read_nf2ff(0, face, w)), (face, w)
    if scene == "dielectric":
        for m in range(2):  # an E-field and an H-field movie across the slab boundaries
            assert np.array_equal(g.read_movie(m), ref.read_movie(m))
        for w in range(6):  # time-domain sums: the same terms split by slab, then added
            a, b = g.read_nf2ff_td(w), ref.read_nf2ff_td(w)
            assert np.linalg.norm(a - b) <= 1e-12 * max(np.linalg.norm(b), 1e-300)
    g.close()
    ref.close()


@gpu
def test_slab_rules():
    sc, keep = _dielectric().lower()
    h = X.Handle(sc, keep)
    with pytest.raises(L.XfbError):
        h._c(h.lib.xfb_set_slab(h.h, 3, 20))  # plane 2 lies in the 5-cell x CPML
    h._c(h.lib.xfb_set_slab(h.h, 0, 20))
    h.init(5)
    with pytest.raises(L.XfbError) as e:
        h.step(1)
    assert e.value.status == L.XFB_ERR_STATE
    with pytest.raises(L.XfbError) as e:
        h._c(h.lib.xfb_slab_record(h.h))
    assert e.value.status == L.XFB_ERR_STATE
    h.close()
