"""Pins the CPU oracle to the reference (CPU only).

The oracle (oracle/fdtd_oracle.c) must reproduce gDiamond's own constructor coefficients and
update_FDTD_seq fields bit for bit:
  * against the committed golden fixtures (generated from the reference by
    tests/golden/make_golden.py) -- always;
  * against the reference compiled here (oracle/_ref/libgdref.so) -- when it is built.
Mirrors the reference's own correctness tests (unittests/checker_omp.cpp,
unittests/checker_omp_dt.cpp: 100^3 cells, 100 steps, all six components).
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                          np.asarray(b, np.float32).view(np.uint32))


def ref_mz_source(shape, src_idx, T):
    nx, ny, _ = shape
    return oracle.Source("Mz", oracle.reference_mz_wave(T), i=src_idx % nx,
                         j=(src_idx // nx) % ny, k=src_idx // (nx * ny))


@pytest.mark.parametrize("name", ["ref_seq_17x13x11_T25.npz", "ref_seq_24x20x16_T30.npz"])
def test_oracle_matches_golden_fields(name):
    d = np.load(os.path.join(GOLDEN, name))
    shape, T = tuple(int(v) for v in d["shape"]), int(d["T"])
    coefs = oracle.coefficients(shape)
    for a, n in enumerate(oracle.COEFFS):
        assert bits_equal(coefs[a], d[f"coef_{n}"]), n
    F = oracle.run(shape, coefs, T, sources=[ref_mz_source(shape, int(d["source_idx"]), T)])
    for c, n in enumerate(oracle.COMPONENTS):
        assert bits_equal(F[c], d[f"field_{n}"]), n


def test_oracle_matches_golden_100cube():
    g = json.load(open(os.path.join(GOLDEN, "ref_100cube_T100.json")))
    shape, T = tuple(g["shape"]), g["T"]
    coefs = oracle.coefficients(shape)
    for a, n in enumerate(oracle.COEFFS):
        assert sha(coefs[a]) == g["coef_sha256"][n], n
    F = oracle.run(shape, coefs, T, sources=[ref_mz_source(shape, g["source_idx"], T)])
    for c, n in enumerate(oracle.COMPONENTS):
        assert sha(F[c]) == g["seq"][n]["sha256"], n
        assert np.linalg.norm(F[c].astype(np.float64)) == pytest.approx(g["seq"][n]["l2"], rel=1e-12)
    # The reference's own omp and omp_dt paths agree with seq bit for bit.
    for v in ("omp", "omp_dt"):
        for n in oracle.COMPONENTS:
            assert g[v][n]["sha256"] == g["seq"][n]["sha256"]


def test_reference_params_match_golden():
    g = json.load(open(os.path.join(GOLDEN, "ref_100cube_T100.json")))
    p = oracle.reference_params()
    for k, v in g["params"].items():
        assert np.float32(p[k]) == np.float32(v), k


needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")


@needs_ref
@pytest.mark.parametrize("shape,T", [((9, 8, 7), 12), ((31, 17, 23), 20), ((40, 40, 40), 15)])
def test_oracle_matches_compiled_reference(shape, T):
    r = oracle.Reference(*shape)
    coefs_ref = r.coefficients()
    coefs = oracle.coefficients(shape)
    for a in range(12):
        assert bits_equal(coefs[a], coefs_ref[a]), oracle.COEFFS[a]
    r.run_seq(T)
    F_ref = r.fields("seq")
    F = oracle.run(shape, coefs, T, sources=[ref_mz_source(shape, r.source_idx(), T)])
    for c in range(6):
        assert bits_equal(F[c], F_ref[c]), oracle.COMPONENTS[c]


@needs_ref
def test_reference_omp_matches_seq():
    """The reference's own checker_omp test, with the harness's vector-resize workaround."""
    r = oracle.Reference(30, 28, 26)
    r.run_seq(20)
    r.run_omp(20)
    for a, b in zip(r.fields("seq"), r.fields("omp")):
        assert bits_equal(a, b)


def test_fp64_oracle_tracks_fp32():
    shape, T = (20, 18, 16), 40
    coefs = oracle.coefficients(shape)
    src = [oracle.Source("Jz", np.float32(5e4) * np.sin(np.arange(T) / 3.0).astype(np.float32),
                         i=10, j=9, k=8)]
    F32 = oracle.run(shape, coefs, T, sources=src)
    F64 = oracle.run(shape, coefs, T, sources=src, precision="f64")
    for a, b in zip(F32, F64):
        rel = np.linalg.norm(a.astype(np.float64) - b) / max(np.linalg.norm(b), 1e-30)
        assert rel < 1e-5


def test_dft_tables_are_fp64_trig():
    f = np.array([0.5, 1.0, 1.7])
    ct, st = oracle.dft_tables(f, 0.05, 10)
    t = np.arange(10)[:, None] * 0.05
    assert np.allclose(ct, np.cos(2 * np.pi * f[None, :] * t), rtol=0, atol=1e-15)
    assert np.allclose(st, np.sin(2 * np.pi * f[None, :] * t), rtol=0, atol=1e-15)


def test_monitor_accumulates_plane_dft():
    """Monitor sums equal an explicit FP64 DFT of the recorded plane history."""
    shape, T = (14, 12, 10), 16
    coefs = oracle.coefficients(shape)
    wave = np.float32(1e3) * np.sin(np.arange(T) * 0.7).astype(np.float32)
    src = [oracle.Source("Jz", wave, i=7, j=6, k=5)]
    freqs = np.array([0.4, 0.9])
    mon = oracle.Monitor("Ez", 5, freqs, scale=0.5)
    oracle.run(shape, coefs, T, sources=src, monitors=[mon])
    F = None
    hist = []
    for t in range(T):
        F = oracle.run(shape, coefs, 1, sources=src, fields=F, t0=t)
        hist.append(F[2].reshape(shape[2], shape[1], shape[0])[5].astype(np.float64))
    ct, st = oracle.dft_tables(freqs, float(np.float32(0.05)), T)
    re = sum((hist[t][None] * ct[t][:, None, None]) * 0.5 for t in range(T))
    im = -sum((hist[t][None] * st[t][:, None, None]) * 0.5 for t in range(T))
    assert np.allclose(mon.re, re, rtol=1e-12, atol=1e-9)
    assert np.allclose(mon.im, im, rtol=1e-12, atol=1e-9)
