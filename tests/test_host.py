"""Host-side logic and the C-ABI library, without a GPU.

* the product's coefficient builder and source waveform reproduce the oracle bit for bit;
* libgdiamond_b200.so loads and exports every symbol include/fdtd_capi.h declares;
* argument validation returns status codes (no exit, no crash) before any device call.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle
import gdiamond_b200 as gd
from gdiamond_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                          np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("shape", [(24, 20, 16), (17, 13, 11), (40, 33, 29)])
@pytest.mark.parametrize("random_eps", [False, True])
def test_reference_coefficients_match_oracle(shape, random_eps):
    eps = None
    if random_eps:
        eps = np.random.default_rng(0).uniform(1, 12, int(np.prod(shape))).astype(np.float32)
    a = W.reference_coefficients(shape, eps_re=eps)
    b = oracle.coefficients(shape, eps_re=eps)
    for x, y in zip(a, b):
        assert bits_equal(x, y)


def test_reference_mz_wave_matches_oracle():
    assert bits_equal(W.reference_mz_wave(500), oracle.reference_mz_wave(500))


def test_vacuum_coefficients_are_courant_half():
    c = W.vacuum_coefficients((4, 4, 4))
    assert all((c[a] == 1).all() for a in (0, 1, 2, 6, 7, 8))
    assert all((c[a] == 0.5).all() for a in (3, 4, 5, 9, 10, 11))


def test_source_band_and_wave():
    f = W.source_band(8)
    assert len(f) == 8 and abs(f.mean() - 1.0) < 1e-6
    w = W.gaussian_wave(100)
    assert w.dtype == np.float32 and np.argmax(np.abs(w)) in range(30, 50)


def test_geometry_generators_are_seeded():
    a = W.spheres_eps((40, 30, 20), n_spheres=10, seed=3)
    b = W.spheres_eps((40, 30, 20), n_spheres=10, seed=3)
    assert np.array_equal(a, b) and a.max() > 1
    s = W.slab_eps((64, 96, 128), np.random.default_rng(5))
    assert s.max() >= 2 and s.min() == 1
    bx = W.box_eps((96, 96, 96), (48, 48, 48, 20, 7.0))
    assert (bx == 7.0).sum() == 20 ** 3


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "fdtd_capi.h")).read()
    return sorted(set(re.findall(r"\b(fdtd_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = C.CDLL(gd.LIB_PATH)
    decl = declared_symbols()
    assert len(decl) >= 15
    for name in decl:
        assert hasattr(L, name), name
    assert set(decl) == set(gd.EXPORTS)


def test_library_loads_and_reports_version():
    assert b"sm_100a" in gd.library().fdtd_version()
    assert gd.library().fdtd_status_string(4) == b"unsupported configuration"


def test_create_validates_arguments_without_device():
    with pytest.raises(gd.FdtdError) as e:
        gd.Simulation(2, 10, 10)
    assert e.value.status == 1  # FDTD_ERR_INVALID_ARG
    with pytest.raises(gd.FdtdError) as e:
        gd.Simulation(10, 10, 10, blt=9)
    assert e.value.status == 1
    with pytest.raises(gd.FdtdError) as e:
        gd.Simulation(10, 10, 10, tile_rows=12)
    assert e.value.status == 1


def test_null_handle_calls_return_invalid_arg():
    L = gd.library()
    assert L.fdtd_step(None, 1, None) == 1
    assert L.fdtd_sync(None) == 1
    assert L.fdtd_destroy(None) == 1
    assert L.fdtd_cpml_psi_bytes(None, 0, None) == 1
    assert L.fdtd_get_cpml_psi(None, 0, None) == 1
    assert L.fdtd_set_cpml_psi(None, 0, None) == 1


def test_surrogate_fallback_bucket_sizes():
    """Fallback calls are padded to a few batch sizes (powers of two from 4, at most the group)."""
    from gdiamond_b200 import surrogate as S
    assert [S.bucket(n, 256) for n in (1, 3, 4, 5, 9, 100, 256, 300)] == \
        [4, 4, 4, 8, 16, 128, 256, 256]
    assert S.bucket(7, 6) == 6


def test_surrogate_solver_boundary_arguments():
    """CPML layers must leave the source and flux planes outside them (checked before any
    device work); 8-cell layers are the default with CPML and keep the stated z = 10 / z = 86
    planes of the 96^3 grid outside."""
    import pytest
    from gdiamond_b200 import surrogate as S
    with pytest.raises(ValueError):
        S.SpectrumSolver(boundary="cpml", t_pml=10)  # z = 86 lies in a 10-cell top layer
    with pytest.raises(ValueError):
        S.SpectrumSolver(boundary="cpml", source_k=6)  # z = 6 lies in the bottom layer
    with pytest.raises(ValueError):
        S.SpectrumSolver(boundary="absorbing")
    assert 8 <= S.SOURCE_K and S.MONITOR_K <= S.SHAPE[2] - 2 - 8
