"""The step kernels' phases run on the host, thread by thread, in the
kernels' order (tests/host_phases/phases.cpp): for elastic media the fused
kernel's tiles on planes [6, ny-6), the marching kernel's y-wall slabs and
the face SAT pass, for acoustic media the marching kernel over every plane,
against the per-point step (and the imaging kernel's interior taps against
its per-point code), on seeded grids whose tiles, chunks and closure
rows differ per axis.  Every phase is a host/device function, so this checks
the kernels' index arithmetic, ring slots, closure handling and the per-model
closure-weight tables without a GPU (the GPU tests run the same code as
kernels against the reference)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "fwi3d_b200", "csrc")


@pytest.fixture(scope="module")
def phases(tmp_path_factory):
    cxx = shutil.which("g++")
    if not cxx:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path_factory.mktemp("phases") / "phases")
    cmd = [cxx, "-O2", "-std=c++17", "-fopenmp", "-w", "-I", CSRC, "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "host_phases", "phases.cpp"), os.path.join(CSRC, "host_ops.cpp"),
           os.path.join(CSRC, "sbp_tables.cpp"), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True, timeout=600)
    return exe


# (physics, nx, ny, nz, y chunks, bc set, taper width, closure-weight tables)
CASES = [
    (2, 60, 40, 76, 1, 0, 5, 0),
    (2, 63, 33, 101, 3, 1, 3, 0),
    (2, 45, 50, 47, 2, 2, 4, 0),
    (3, 60, 40, 76, 1, 0, 5, 0),
    (3, 60, 40, 76, 2, 1, 5, 1),
    (3, 63, 33, 101, 3, 2, 3, 1),   # odd sizes: shifted last tiles, partial tiles
    (6, 60, 40, 76, 2, 1, 5, 1),
    (6, 45, 30, 47, 1, 2, 4, 0),
    (6, 70, 30, 90, 2, 2, 3, 1),
    (13, 40, 30, 36, 1, 0, 0, 0),   # imaging: interior taps vs per-point code
    (16, 40, 30, 36, 1, 0, 0, 0),
]


@pytest.mark.parametrize("case", CASES)
def test_kernel_phases_match_per_point(phases, case):
    out = subprocess.run([phases] + [str(v) for v in case], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    f = out.stdout.split()
    rel, nan = float(f[1]), int(f[5])
    assert nan == 0
    assert rel < 2e-6
