"""Host logic of the engine's work lists, without a GPU.

tests/host_workitems.cu is compiled against the engine's headers and run on
the CPU.  On seeded random scenes, with every tile configuration and the ADE
update both in the step kernel and deferred, it checks two things.

- The one-sweep work items cover every (tile, plane) exactly once.  Each item
  has a kind whose body handles every CPML, ADE and TFSF cell it updates,
  including the H halo plane and the tile's halo row and column.  Lean
  interior items lie inside the grid.
- The deferred ADE pass's run list covers every dispersive cell of the box
  exactly once, and nothing else.  Its runs stay inside one 32-aligned k
  segment and come in (i, j, k) order.

Those lists decide which specialised body the step kernel runs for every
cell: a cell left uncovered, or covered by a body without its CPML, ADE or
TFSF code, would be updated wrongly.
"""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_work_items_and_ade_runs(tmp_path):
    from xfdtd_cuda_b200 import build
    try:
        nvcc = build.nvcc()
    except RuntimeError as e:
        pytest.skip(str(e))
    exe = tmp_path / "host_workitems"
    subprocess.run([nvcc, "-std=c++17", "-O2", *build.ARCH, "-I", str(ROOT), "-I", str(ROOT / "include"),
                    "-o", str(exe), str(ROOT / "tests" / "host_workitems.cu")], check=True, timeout=600)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:]
    ok, items, runs = out.stdout.split()
    assert ok == "ok" and int(items) > 100000 and int(runs) > 1000
