"""Allocation-free material-map construction, on the GPU.

`fdtd_build_material_map_noalloc` serves callers that cannot allocate device memory at the
point where they need a material map: an application that owns all device memory through its
own pool (a cudaMalloc from a plug-in would fail or fragment it), a loop where cudaMalloc's
implicit synchronisation is not acceptable, or code that must not grow its footprint after
start-up.  The caller passes the 12 coefficient arrays and the output buffers; the entry point's
hash-table scratch is a fixed device array inside the library.

Its output is checked against the existing allocating path (`fdtd_set_coefficients_device`,
which deduplicates into the handle's own map, and `fdtd_material_count`) on calls made back to
back, bit for bit: the same number of materials, and every cell's 12-tuple reproduced exactly
by table[map[cell]].  The second call uses different coefficients, so scratch left over from
the first call would show.  This file is collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import gdiamond_b200 as gd
from gdiamond_b200 import workloads as W

pytestmark = pytest.mark.gpu

MAX_NOALLOC_MATERIALS = 4096


def _fn():
    fn = gd.library().fdtd_build_material_map_noalloc
    fn.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p,
                   C.c_int32, C.POINTER(C.c_int32), C.c_void_p]
    fn.restype = C.c_int
    return fn


def to_device(coefs):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(c, np.float32)).cuda() for c in coefs]


def noalloc(coefs_dev, shape, max_materials):
    import torch
    nx, ny, nz = shape
    n = nx * ny * nz
    mat = torch.zeros(n, dtype=torch.int16, device="cuda")
    table = torch.zeros(max_materials * 12, dtype=torch.float32, device="cuda")
    ptrs = (C.c_void_p * 12)(*[int(c.data_ptr()) for c in coefs_dev])
    nmat = C.c_int32(-1)
    torch.cuda.synchronize()
    st = _fn()(ptrs, nx, ny, nz, C.c_void_p(mat.data_ptr()), C.c_void_p(table.data_ptr()),
               max_materials, C.byref(nmat), None)
    torch.cuda.synchronize()
    return (st, nmat.value, mat.cpu().numpy().view(np.uint16),
            table.cpu().numpy().reshape(max_materials, 12))


def existing_count(coefs_dev, shape):
    sim = gd.Simulation(*shape)
    sim.set_coefficients(coefs_dev)  # device tensors -> fdtd_set_coefficients_device
    n = sim.material_count()
    sim.close()
    return n


def check_against_existing(coefs, shape):
    dev = to_device(coefs)
    expect = existing_count(dev, shape)
    assert 0 < expect <= MAX_NOALLOC_MATERIALS
    st, nmat, mat, table = noalloc(dev, shape, MAX_NOALLOC_MATERIALS)
    assert st == 0, gd.library().fdtd_status_string(st)
    assert nmat == expect
    # ids are dense (0..nmat-1 all used) and name distinct tuples; their numbering may differ
    # from call to call, since ids follow table-slot order assigned by atomics
    assert int(mat.max()) + 1 == nmat
    assert len(np.unique(table[:nmat].view(np.uint32), axis=0)) == nmat
    for a in range(12):
        rebuilt = table[mat.astype(np.int64), a]
        assert np.array_equal(rebuilt.view(np.uint32),
                              np.asarray(coefs[a], np.float32).view(np.uint32)), gd.COEFFS[a]


def test_noalloc_matches_existing_path_on_consecutive_calls():
    shape1 = (60, 50, 40)
    check_against_existing(W.reference_coefficients(shape1), shape1)   # graded-PML tuples
    shape2 = (48, 44, 36)
    eps = W.spheres_eps(shape2, n_spheres=6, r_range=(3, 8), seed=5)
    check_against_existing(W.reference_coefficients(shape2, eps_re=eps), shape2)
    check_against_existing(W.vacuum_coefficients(shape2), shape2)      # a single material


def test_noalloc_rejects_sizes_beyond_its_limit():
    shape = (40, 30, 20)
    dev = to_device(W.reference_coefficients(shape))
    st, _, _, _ = noalloc(dev, shape, MAX_NOALLOC_MATERIALS + 1)
    assert st == 1  # FDTD_ERR_INVALID_ARG: table capacity above the fixed maximum
    st, nmat, _, _ = noalloc(dev, shape, 16)
    assert st == 4 and nmat > 16  # FDTD_ERR_UNSUPPORTED: more tuples than the caller's table
    check_against_existing(W.reference_coefficients(shape), shape)  # still usable afterwards


def test_noalloc_rejects_many_distinct_tuples_quickly():
    """A graded medium with a distinct tuple per cell (far beyond the 4096 limit) is rejected
    after a short pass: inserting stops once the count passes the caller's table size."""
    import time
    shape = (96, 96, 64)
    n = int(np.prod(shape))
    coefs = [c.copy() for c in W.vacuum_coefficients(shape)]
    coefs[3] = (np.float32(0.25) + np.arange(n, dtype=np.float32) * np.float32(1e-7))  # Cbx
    dev = to_device(coefs)
    noalloc(dev, (8, 8, 8), MAX_NOALLOC_MATERIALS)  # first call on the device resolves the table
    t0 = time.perf_counter()
    st, nmat, _, _ = noalloc(dev, shape, MAX_NOALLOC_MATERIALS)
    secs = time.perf_counter() - t0
    assert st == 4 and nmat > MAX_NOALLOC_MATERIALS  # FDTD_ERR_UNSUPPORTED
    assert secs < 2.0, secs
    check_against_existing(W.vacuum_coefficients((40, 30, 20)), (40, 30, 20))  # still usable
