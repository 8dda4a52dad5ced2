"""Generates the golden fixtures of tests/golden/ from the REFERENCE itself.

Runs gDiamond's own constructor and update_FDTD_seq / update_FDTD_omp / update_FDTD_omp_dt,
compiled from the reference sources into oracle/_ref/libgdref.so (``make -C oracle``), and
stores their outputs:

* ``ref_seq_17x13x11_T25.npz`` -- all 6 fields after 25 steps and the 12 coefficient arrays
  of a 17 x 13 x 11 grid (small enough to store whole);
* ``ref_seq_24x20x16_T30.npz`` -- the same for 24 x 20 x 16, 30 steps;
* ``ref_100cube_T100.json`` -- the reference unit-test configuration (100^3 cells, 100 steps,
  unittests/checker_*.cpp): per-component L2 norm and SHA-256 of the FP32 field bytes of seq,
  omp and omp_dt(16,16,16,5), and SHA-256 of the 12 coefficient arrays;
* ``ref_png_37x23.npz`` -- a seeded 37 x 23 field slice (values beyond +-vmax, zeros, -0.0
  included), its vmax, and the PNG file the reference's save_field_png (utils.h:210-255) writes
  for it, as bytes.

Run from the repository root:  python tests/golden/make_golden.py [small cube png]
(no arguments: every fixture).
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def small(shape, T):
    r = oracle.Reference(*shape)
    coefs = r.coefficients()
    r.run_seq(T)
    F = r.fields("seq")
    out = {f"field_{oracle.COMPONENTS[c]}": F[c] for c in range(6)}
    out.update({f"coef_{oracle.COEFFS[a]}": coefs[a] for a in range(12)})
    out["shape"] = np.array(shape)
    out["T"] = np.array(T)
    out["source_idx"] = np.array(r.source_idx())
    nx, ny, nz = shape
    np.savez_compressed(os.path.join(HERE, f"ref_seq_{nx}x{ny}x{nz}_T{T}.npz"), **out)


def cube():
    shape, T = (100, 100, 100), 100
    r = oracle.Reference(*shape)
    coefs = r.coefficients()
    res = {"shape": shape, "T": T, "source_idx": r.source_idx(), "params": r.params(),
           "coef_sha256": {oracle.COEFFS[a]: sha(coefs[a]) for a in range(12)}}
    r.run_seq(T)
    r.run_omp(T)
    r.run_omp_dt(16, 16, 16, 5, T)
    for v in ("seq", "omp", "omp_dt"):
        F = r.fields(v)
        res[v] = {oracle.COMPONENTS[c]: {"l2": float(np.linalg.norm(F[c].astype(np.float64))),
                                         "sha256": sha(F[c])} for c in range(6)}
    with open(os.path.join(HERE, "ref_100cube_T100.json"), "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)


def png():
    import tempfile
    rng = np.random.default_rng(21)
    u = (rng.standard_normal((23, 37)) * 1.5).astype(np.float32)
    u[0, :5] = [0.0, -0.0, 2.0, -2.0, 1e-30]
    vmax = np.float32(2.0)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "slice.png")
        oracle.ref_save_field_png(u, path, vmax)
        data = np.frombuffer(open(path, "rb").read(), np.uint8)
    np.savez_compressed(os.path.join(HERE, "ref_png_37x23.npz"), u=u, vmax=vmax, png=data)


if __name__ == "__main__":
    if not oracle.ref_available():
        oracle.build()
    which = set(sys.argv[1:]) or {"small", "cube", "png"}
    if "small" in which:
        small((17, 13, 11), 25)
        small((24, 20, 16), 30)
    if "cube" in which:
        cube()
    if "png" in which:
        png()
    print("golden fixtures written to", HERE)
