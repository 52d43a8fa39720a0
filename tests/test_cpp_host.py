"""The C++ host header (include/xfdtd_b200/simulation_hd.hpp): a program
written like the reference's drivers compiles and links against the library
with g++, reports errors as exceptions, and on a GPU produces the same
results as the Python host path for the same scene."""
import math
import subprocess
from pathlib import Path

import numpy as np
import pytest

import xfdtd_cuda_b200 as X
from xfdtd_cuda_b200 import configs
from conftest import has_gpu

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "sphere_demo.cpp"
LIBDIR = ROOT / "xfdtd_cuda_b200"


@pytest.fixture(scope="module")
def demo(tmp_path_factory):
    exe = tmp_path_factory.mktemp("cpp") / "sphere_demo"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", str(ROOT / "include"), str(SRC), "-o", str(exe),
           "-L", str(LIBDIR), "-lxfdtd_b200", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_host_compiles_and_reports_errors_as_exceptions(demo):
    if has_gpu():
        pytest.skip("covered by the GPU comparison")
    r = subprocess.run([str(demo), "5"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 3 and r.stdout.startswith("error: xfdtd_b200: "), r.stdout


@pytest.mark.gpu
def test_cpp_host_matches_python_host(demo):
    n = 60
    r = subprocess.run([str(demo), str(n)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    tag, sez, shx, pr, ff = r.stdout.split()
    assert tag == "ok"
    sim = configs.dielectric_sphere(cells=28, dl=5e-3, pml=6, precision="fp64", tfsf_inset=5, nf2ff_inset=3,
                                    freqs=(1.5e9,), radius=0.03)
    sim.addMonitor(X.PointMonitor(X.Vector(0, 0, 0), X.EMF.Field.EZ))
    sc, keep = sim.lower()
    h = X.Handle(sc, keep)
    h.init(n)
    h.step(n)
    h.sync()
    assert float(sez) == pytest.approx(float(h.read_field(2).sum()), rel=1e-12, abs=1e-300)
    assert float(shx) == pytest.approx(float(np.abs(h.read_field(3)).sum()), rel=1e-12)
    et, _ = h.far_field(0, np.array([math.pi / 2]), np.array([0.0]))
    assert float(ff) == pytest.approx(abs(et[0]), rel=1e-10)
    assert h.probe_desc[0][1:] == (20, 20, 20)
    assert float(pr) == pytest.approx(float(h.read_probe(0)[-1]), rel=1e-12, abs=1e-300)
