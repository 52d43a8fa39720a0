"""Result read-back into caller arrays.

CPU: xfb_host_prefault faults in a host range on background threads without
changing its contents (including ranges with partial first and last pages),
and a wait joins them.

GPU: SimulationHD.run fills the host result arrays it allocated at init (the
fields in host().emf, the NF2FF surface currents) with exactly what the
handle's own reads return; reads into caller arrays (out=) match reads into
fresh ones; the one-call read of all currents of a frequency matches the
per-face reads.
"""
import numpy as np
import pytest

import xfdtd_cuda_b200 as X
from xfdtd_cuda_b200 import _lib as L
from xfdtd_cuda_b200 import configs


def test_prefault_keeps_contents():
    sc, keep = configs.dielectric_sphere(cells=12, dl=5e-3, pml=3, precision="fp64", tfsf_inset=2,
                                         nf2ff_inset=1, radius=0.01).lower()
    h = X.Handle(sc, keep)
    rng = np.random.default_rng(3)
    big = rng.standard_normal(9_000_000)  # 72 MB: several threads
    ref = big.copy()
    h.prefault(big)
    odd = rng.standard_normal(1234)  # smaller than a page pair, unaligned
    ref_odd = odd.copy()
    h.prefault(odd[1:])
    h.prefault(np.empty(0))
    h.prefault_wait()
    assert np.array_equal(big, ref) and np.array_equal(odd, ref_odd)
    fresh = np.empty(5_000_000)
    h.prefault(fresh)
    h.close()  # joins the threads first
    h2 = X.Handle(sc, keep)
    with pytest.raises(L.XfbError):
        h2._c(h2.lib.xfb_host_prefault(h2.h, None, 16))
    h2.close()


@pytest.mark.gpu
def test_simulation_hd_fills_host_results():
    steps = 40

    def build():
        return configs.dielectric_sphere(cells=24, dl=5e-3, pml=5, precision="fp32", tfsf_inset=4, nf2ff_inset=2,
                                         radius=0.025, freqs=(1e9, 2e9))

    sim = build()
    hd = X.SimulationHD(sim)
    hd.run(steps)
    ref = X.Handle(*build().lower())
    ref.init(steps)
    ref.step(steps)
    ref.sync()
    for f in range(6):
        a = sim.emf.field(f)
        assert a is not None and np.array_equal(a, ref.read_field(f)), f
        out = np.full(ref.shape(f), np.nan)
        assert ref.read_field(f, out=out) is out and np.array_equal(out, a)
    nf = sim.nf2ff_list[0]
    for fr in range(2):
        for face in range(6):
            for w in range(4):
                b = ref.read_nf2ff(fr, face, w)
                assert np.array_equal(nf.currents[fr][face][w], b)
                out = np.empty_like(b)
                assert np.array_equal(ref.read_nf2ff(fr, face, w, out=out), b)
    for fr in range(2):
        split = ref.nf2ff_split(ref.read_nf2ff_all(fr))
        for face in range(6):
            for w in range(4):
                assert np.array_equal(split[face][w], ref.read_nf2ff(fr, face, w))
    with pytest.raises(ValueError):
        ref.read_field(0, out=np.empty((2, 2)))
    hd.releaseDevice()
    ref.close()
