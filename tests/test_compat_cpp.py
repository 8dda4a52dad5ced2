"""The C++ class surface (include/gdiamond_compat.hpp), compiled with g++ and run.

Mirrors the reference's own tests: seq vs omp and omp_dt (unittests/checker_omp.cpp,
checker_omp_dt.cpp) on the CPU, and on
the GPU seq vs update_FDTD_gpu_2D (unittests/checker_gpu.cu) and the 3D-fix baseline vs
mix-mapping ver3 (examples/gpu_mm_ver3.cu), all at the reference's |a-b| < 1e-8.  The seq
fields are also checked bit for bit against the golden fixture generated from the reference.
"""
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

import gdiamond_b200 as gd

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "compat_checker.cpp")
GOLDEN = os.path.join(ROOT, "tests", "golden", "ref_100cube_T100.json")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("compat") / "compat_checker")
    libdir = os.path.dirname(gd.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-O2", "-fopenmp", "-ffp-contract=off",
           "-I" + os.path.join(ROOT, "include"), SRC, "-o", out, "-L" + libdir,
           "-lgdiamond_b200", "-Wl,-rpath," + libdir]
    subprocess.run(cmd, check=True)
    return out


def run(exe, *args):
    r = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=600)
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
    return r.returncode, json.loads(line)


def test_cpp_seq_matches_golden_and_omp(checker, tmp_path):
    g = json.load(open(GOLDEN))
    rc, res = run(checker, "cpu", 100, 100, 100, 100, str(tmp_path / "seq_"))
    assert rc == 0 and res["omp_matches_seq"] and res["omp_dt_matches_seq"]
    for c, n in enumerate(("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")):
        data = (tmp_path / f"seq_{c}.bin").read_bytes()
        assert hashlib.sha256(data).hexdigest() == g["seq"][n]["sha256"], n
        assert res["seq_l2"][c] == pytest.approx(g["seq"][n]["l2"], rel=1e-12)


@pytest.mark.gpu
def test_cpp_gpu_paths_match_reference_checks(checker, tmp_path):
    shape, T = (64, 56, 48), 90
    rc, res = run(checker, "gpu", *shape, T, str(tmp_path / "g_"))
    assert res["gpu_2D_matches_seq"] and res["ver3_matches_3D_fix"]
    assert res["vectorized_matches_ver3"]
    assert res["figures_nf"] == 26 and res["figures_dft_max"] > 0
    assert rc == 0
    # the figures path's Ex DFT (Jx point source, plane Nz/2) against the oracle's FP64 DFT,
    # bit for bit, from the waveform, frequencies and coefficients the class used
    import oracle
    nx, ny, nz = shape
    rd = lambda name, dt: np.fromfile(tmp_path / f"g_{name}.bin", dtype=dt)
    wave, freqs = rd("fig_wave", np.float32), rd("fig_freqs", np.float64)
    coefs = [rd(f"coef{a}", np.float32) for a in range(12)]
    mon = oracle.Monitor("Ex", nz // 2, freqs, scale=50.0 / T)
    oracle.run(shape, coefs, T, sources=[oracle.Source("Jx", wave, i=nx // 2, j=ny // 2, k=nz // 2)],
               monitors=[mon], dt=float(np.float32(0.05)))
    re, im = rd("fig_re", np.float64), rd("fig_im", np.float64)
    assert np.array_equal(re, mon.re.reshape(-1)) and np.array_equal(im, mon.im.reshape(-1))
