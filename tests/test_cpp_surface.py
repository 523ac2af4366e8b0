"""The C++ operator surface (include/libtensor_b200/libtensor.h) compiled
with g++ and run: the ladder contraction written as a libtensor user writes
it, checked against the golden fixtures produced by the reference."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from tests.test_golden import G, golden_blocks

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "surface_test.cpp")
LIBDIR = os.path.join(ROOT, "libtensor_b200", "_lib")
CUDA_LIB = "/usr/local/cuda/lib64"


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    if not os.path.exists(os.path.join(LIBDIR, "libltg.so")):
        pytest.skip("libltg.so not built")
    out = str(tmp_path_factory.mktemp("cpp") / "surface_test")
    cmd = ["g++", "-std=c++14", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC, "-o", out,
           "-L", LIBDIR, "-lltg", f"-Wl,-rpath,{LIBDIR}", "-L", CUDA_LIB, f"-Wl,-rpath,{CUDA_LIB}", "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_surface_schedule_matches_golden(exe):
    r = subprocess.run([exe, "schedule"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    sched = [int(x) for x in r.stdout.split()]
    assert sched == [int(x) for x in G["c0_schedule"]]


@pytest.mark.gpu
def test_surface_compute_matches_golden(exe, tmp_path):
    out = str(tmp_path / "result.txt")
    r = subprocess.run([exe, "compute", out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = open(out).read().split("\n")
    nblk = int(lines[0])
    pos = 1
    gold = golden_blocks(0)
    seen = []
    for _ in range(nblk):
        b0, b1, b2, b3, n = (int(x) for x in lines[pos].split())
        data = np.array([float(x) for x in lines[pos + 1:pos + 1 + n]])
        pos += 1 + n
        a = ((b0 * 2 + b1) * 4 + b2) * 4 + b3            # block index dims (2, 2, 4, 4)
        seen.append(a)
        ref = gold[a].ravel()
        assert np.max(np.abs(data - ref)) <= 1e-13 * np.max(np.abs(ref)), a
    assert seen == sorted(gold)
    dot_tt, dot_ts, dot_pp = (float(x) for x in lines[pos].split())
    assert abs(dot_ts - 1.25 * dot_tt) <= 1e-13 * dot_tt
    assert abs(dot_pp - 0.25 * dot_tt) <= 1e-13 * dot_tt
    # letter interface against the operations written out: the ladder, an
    # antisymmetrising difference, dot products (one permuted), K = 3 and
    # K = 1 contractions, assignment then -=, symmetrizers, intermediates
    d = [float(x) for x in lines[pos + 1].split()]
    rmax = max(float(np.max(np.abs(v))) for v in gold.values())
    assert d[0] == 0.0                                  # the same plan and kernels
    assert d[1] <= 1e-15 * rmax
    assert d[2] <= 1e-13 * dot_tt and d[3] <= 1e-13 * dot_tt
    assert d[4] == 0.0 and d[5] == 0.0
    assert d[6] <= 1e-15 * rmax
    assert d[7] <= 1e-15 * rmax                         # symm(i|a, j|b, r) = 2 r
    assert d[8] == 0.0                                  # asymm(a, b, contraction) = btod_symmetrize2
    assert d[9] == 0.0                                  # graph replay = eager operations
    # intermediates: nested contraction, contraction of sums (same symmetry,
    # and a spin-only term), result on the right-hand side, dot of a sum, and
    # the assignment replayed as one graph (bit-identical to its eager run)
    gmax = max(1.0, rmax)
    assert d[10] <= 1e-13 * gmax and d[11] <= 1e-13 * gmax and d[12] <= 1e-13 * gmax
    assert d[13] <= 1e-15 * rmax                        # r - hr / 2, hr = r + r
    assert d[14] <= 1e-13 * dot_tt
    assert d[15] == 0.0
    assert d[16] == 2                                   # the add into the intermediate, the contraction
    assert d[17] == 0.0                                 # btod_contract3, direct_block_tensor = explicit ops
    # btod_symmetrize2 over the contraction (fused into its epilogue) against
    # the symmetrizer over the contraction's result (same terms; the k
    # summation of the contraction may be cut differently)
    assert d[18] <= 1e-15 * gmax
    assert d[19] <= 1e-12 * gmax                        # the same in the modular mode (13 moduli)
