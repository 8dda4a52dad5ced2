"""Host-side helpers of bench.py (CPU only).

* the DRAM-traffic lookup the benchmark line reports as roofline.traffic: it must match the
  measured configuration exactly -- kernel family, row width, BLT, rows and z-chunks -- and
  report nothing for a configuration that was not measured;
* the relative spectral errors: a reference spectrum that is zero everywhere (a monitor the
  pulse has not reached in a short run) gives 0 for an exact result and inf otherwise, never a
  division error.
"""
import importlib.util
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    return b


def entries():
    out = []
    for ln in open(os.path.join(ROOT, "profiles", "fdtd_tiled_256cube_traffic.txt")):
        ln = ln.split("#", 1)[0].strip()
        if ln:
            out.append(dict(part.split("=", 1) for part in ln.split()))
    return out


def test_traffic_lookup_matches_the_measured_configuration_only():
    b = load_bench()
    rows = entries()
    assert rows
    for kv in rows:
        cfg = {"pairs": kv["kernel"] == "fdtd_tiled2", "width": int(kv["width"]),
               "blt": int(kv["blt"]), "tile_rows": int(kv["tile_rows"]),
               "z_chunks": int(kv["z_chunks"])}
        assert b.traffic_from_profile(cfg) == float(kv["dram_bytes_per_launch"])
        # the same numbers for the other row width or the one-cell kernel were not measured
        other = dict(cfg, width=96 - cfg["width"])
        if not any(int(r["width"]) == other["width"] and r["blt"] == kv["blt"] and
                   r["tile_rows"] == kv["tile_rows"] and r["z_chunks"] == kv["z_chunks"]
                   for r in rows):
            assert b.traffic_from_profile(other) is None
        assert b.traffic_from_profile(dict(cfg, pairs=False)) is None
    assert b.traffic_from_profile({"pairs": True, "width": 32, "blt": 5, "tile_rows": 8,
                                   "z_chunks": 1}) is None


def test_spectral_errors_with_a_zero_reference():
    b = load_bench()
    z = (np.zeros((2, 3, 4)), np.zeros((2, 3, 4)))
    one = (np.ones((2, 3, 4)), np.zeros((2, 3, 4)))
    assert b._spectral_error([z], [z]) == 0.0
    assert b._plane_spectrum_error([z], [z]) == 0.0
    assert b._spectral_error([one], [z]) == float("inf")
    assert b._plane_spectrum_error([one], [z]) == float("inf")
    half = (np.full((2, 3, 4), 0.5), np.zeros((2, 3, 4)))
    assert np.isclose(b._spectral_error([half], [one]), 0.5)
    assert np.isclose(b._plane_spectrum_error([half], [one]), 0.5)
