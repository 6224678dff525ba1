"""The site indexing of the kernels, checked on the CPU over every site: the
index functions of qws_b200/csrc/lattice.cuh are __host__ __device__, so
tests/geometry_check.cu (built here with nvcc, run without a GPU) drives the
exact device code -- the DD-order bijection, the in-block hops with the
rotated fastest direction, the face hops with their periodic wrap and
colours, every index inside [0, V) -- on every lattice and block grid the
GPU tests and the benchmark use, and on blocks one and two sites wide.
A stand-in for a device bounds checker for the index arithmetic."""
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent
NVCC = shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc"
                                if Path("/usr/local/cuda/bin/nvcc").exists() else None)

GEOMETRIES = [
    # the reference's golden lattices (CASE0-9, CASE_4111_1111) with their block grids
    "32,6,4,3/2,1,1,1", "32,6,4,6/2,1,1,2", "32,3,4,8/2,1,1,2", "32,3,6,8/2,1,1,2",
    "32,6,6,4/2,1,1,2", "32,6,6,8/2,1,1,2", "32,6,6,16/2,1,1,2", "32,12,8,6/2,2,2,2",
    "128,24,4,3/8,4,1,1", "32,6,16,12/2,1,4,4", "4,1,1,1/2,1,1,1",
    # edge cases of the GPU tests: periodic t, odd block extents, V not a multiple of 128
    "8,4,4,8/2,1,1,1", "12,6,6,6/2,2,2,2", "6,6,2,10/2,1,1,2", "12,6,4,6/2,1,1,1",
    "8,8,8,16/2,2,2,2", "8,8,8,16/2,1,1,1",
    # the benchmark's and the service's volumes at their tuned and reference partitions
    "8,8,8,8/2,2,2,2", "12,12,12,24/2,2,2,2", "16,16,16,32/2,2,2,4", "24,24,24,48/2,2,2,2",
    "32,32,32,64/2,1,1,1", "32,32,32,64/2,2,2,2", "32,32,32,64/4,2,2,2",
    "48,48,48,96/2,4,2,2", "48,48,48,96/2,1,1,1",
    # blocks one or two sites wide
    "8,4,4,4/8,4,4,4", "16,2,2,2/2,2,2,2", "4,4,4,4/4,2,2,2", "6,2,4,2/2,2,2,2",
]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if NVCC is None:
        pytest.skip("nvcc not found")
    exe = tmp_path_factory.mktemp("geom") / "geometry_check"
    r = subprocess.run([NVCC, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                        str(HERE / "geometry_check.cu"), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return exe


def test_site_indexing_on_every_site(checker):
    r = subprocess.run([str(checker), *GEOMETRIES], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:]
    lines = r.stdout.strip().splitlines()
    assert len(lines) == len(GEOMETRIES) and all(s.startswith("ok ") for s in lines), r.stdout


def test_checker_catches_a_planted_mistake(checker):
    """The checker is not vacuous: with two in-block strides swapped after
    the layout is made (a mistake planted on the CPU), it fails."""
    r = subprocess.run([str(checker), "planted:8,4,4,8/2,1,1,1"], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode == 1 and r.stdout.startswith("FAIL"), r.stdout
    r = subprocess.run([str(checker), "8,8,8/2,1,1,1"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "bad argument" in r.stdout
