"""x-slab decomposition of one grid over several devices.

A slab handle (xfb_set_slab) updates the cells [i0, i1) along x of the full
grid.  One time step of a decomposed run is

  1. xfb_slab_update on every slab (the one-sweep update of the owned planes),
  2. the halo exchange: each slab sends its first owned plane down and its
     last owned plane (with the H-side CPML psi of the y and z slabs) up,
  3. xfb_slab_record on every slab (monitors of the owned planes, counter).

Every monitor records only what its slab owns, so the sum over the slabs of
each read-back (probes, NF2FF currents and potentials, movie frames) is the
whole grid's, and a field is the owned planes of each slab side by side.

SlabGroup runs the slabs of one process (any devices, peer copies between
neighbours).  RankSlab is one slab per process, the exchange done with
torch.distributed point-to-point (NCCL on GPUs) on tensors that alias the
library's plane buffers.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .simulation import Handle


def partition(nx: int, n: int, pml_lo: int = 0, pml_hi: int = 0):
    """[(i0, i1)] of n slabs covering cells 0..nx-1 as evenly as possible,
    with every inner boundary s keeping plane s - 1 outside the x CPML
    (pml_lo cells at the low end, pml_hi at the high end)."""
    if n < 1 or n > nx:
        raise ValueError("need 1 <= slabs <= nx")
    lo_min, hi_max = pml_lo + 1, nx - pml_hi  # allowed boundaries s: lo_min <= s <= hi_max
    if n > 1 and hi_max - lo_min + 1 < n - 1:
        raise ValueError("too many slabs for the interior between the x CPML slabs")
    cuts = [0]
    for q in range(1, n):
        s = round(q * nx / n)
        s = min(max(s, lo_min, cuts[-1] + 1), hi_max - (n - 1 - q))
        cuts.append(s)
    cuts.append(nx)
    return [(cuts[q], cuts[q + 1]) for q in range(n)]


def _buffers(h: Handle, which: int):
    ptrs = (C.c_void_p * 10)()
    sizes = (C.c_size_t * 10)()
    n = C.c_int()
    h._c(h.lib.xfb_slab_planes(h.h, which, ptrs, sizes, C.byref(n)))
    return [(ptrs[q], sizes[q]) for q in range(n.value)]


class _Slab(Handle):
    def __init__(self, sim, i0, i1, device):
        sc, keep = sim.lower()
        super().__init__(sc, keep)
        self.set_device(device)
        self._c(self.lib.xfb_set_slab(self.h, int(i0), int(i1)))
        self.i0, self.i1 = i0, i1

    def update(self):
        self._c(self.lib.xfb_slab_update(self.h))

    def record(self):
        self._c(self.lib.xfb_slab_record(self.h))


class SlabGroup:
    """The slabs of one scene in one process, slab q on devices[q % len(devices)]."""

    def __init__(self, sim, n: int, devices=(0,), total_steps: int = 0):
        probe = Handle(*sim.lower())
        gi = probe.info()
        v = probe.compiled_view()
        self.nx = gi.nx
        self.ranges = partition(gi.nx, n, v.pml_cells[0], v.pml_cells[1])
        probe.close()
        self.slabs = [_Slab(sim, i0, i1, devices[q % len(devices)]) for q, (i0, i1) in enumerate(self.ranges)]
        if total_steps:
            self.init(total_steps)

    def init(self, total_steps: int):
        for s in self.slabs:
            s.init(total_steps)

    def step(self, n: int = 1):
        for _ in range(n):
            for s in self.slabs:
                s.update()
            for lo, hi in zip(self.slabs, self.slabs[1:]):
                lo._c(lo.lib.xfb_slab_exchange(lo.h, hi.h))
            for s in self.slabs:
                s.record()

    def sync(self):
        for s in self.slabs:
            s.sync()

    def read_field(self, f) -> np.ndarray:
        """The component over the whole grid: each slab's owned planes (the
        last slab also holds the node plane i = nx)."""
        out = None
        for q, s in enumerate(self.slabs):
            a = s.read_field(f)
            if out is None:
                out = np.zeros_like(a)
            hi = s.i1 if q + 1 < len(self.slabs) else a.shape[0]
            out[s.i0:hi] = a[s.i0:hi]
        return out

    def read_probe(self, p) -> np.ndarray:
        return sum(s.read_probe(p) for s in self.slabs)

    def read_movie(self, m) -> np.ndarray:
        return sum(s.read_movie(m) for s in self.slabs)

    def read_nf2ff(self, freq, face, which) -> np.ndarray:
        return sum(s.read_nf2ff(freq, face, which) for s in self.slabs)

    def read_nf2ff_td(self, which) -> np.ndarray:
        return sum(s.read_nf2ff_td(which) for s in self.slabs)

    def close(self):
        for s in self.slabs:
            s.close()


class _DeviceBuffer:
    """A device buffer of the library exposed to torch (no copy)."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3,
                                         "strides": None}


def exchange(send_down, send_up, recv_below, recv_above, rank: int, world: int, dist):
    """Point-to-point halo exchange of one step between neighbouring ranks.
    send_down / send_up / recv_below / recv_above are equal-length lists of
    tensors (rank 0 has no neighbour below, the last rank none above):
    send_up[q] of rank r lands in recv_below[q] of rank r + 1 and send_down[q]
    of rank r + 1 in recv_above[q] of rank r."""
    ops = []
    if rank + 1 < world:
        ops += [dist.P2POp(dist.isend, t, rank + 1) for t in send_up]
        ops += [dist.P2POp(dist.irecv, t, rank + 1) for t in recv_above]
    if rank > 0:
        ops += [dist.P2POp(dist.isend, t, rank - 1) for t in send_down]
        ops += [dist.P2POp(dist.irecv, t, rank - 1) for t in recv_below]
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()


class RankSlab:
    """One slab per process of a torch.distributed job (rank q holds slab q
    on its local device)."""

    def __init__(self, sim, rank: int, world: int, device: int, total_steps: int):
        import torch
        import torch.distributed as dist
        self.torch, self.dist = torch, dist
        self.rank, self.world = rank, world
        probe = Handle(*sim.lower())
        gi = probe.info()
        v = probe.compiled_view()
        self.ranges = partition(gi.nx, world, v.pml_cells[0], v.pml_cells[1])
        probe.close()
        i0, i1 = self.ranges[rank]
        self.slab = _Slab(sim, i0, i1, device)
        self.slab.init(total_steps)
        self.device = torch.device("cuda", device)

    def _tensors(self, which):
        if (which in (0, 2) and self.rank == 0) or (which in (1, 3) and self.rank + 1 == self.world):
            return []
        return [self.torch.as_tensor(_DeviceBuffer(p, n), device=self.device) for p, n in _buffers(self.slab, which)]

    def step(self, n: int = 1):
        for _ in range(n):
            self.slab.update()
            self.slab.sync()  # the update has written the planes the exchange reads
            exchange(self._tensors(0), self._tensors(1), self._tensors(2), self._tensors(3), self.rank, self.world,
                     self.dist)
            self.torch.cuda.synchronize(self.device)
            self.slab.record()

    def sync(self):
        self.slab.sync()

    def close(self):
        self.slab.close()
