"""The tiled kernel's schedule, emulated on the CPU, against the oracle (CPU only).

tests/tiled_emulator.py replays fdtd_tiled<BLT, ROWS> (gdiamond_b200/csrc/k_tiled.cu) CTA by
CTA.  These cases cover every (BLT, ROWS) instance the library builds, z-chunking with its
warm-up planes, odd grid sizes, the reference PML coefficients, random per-cell permittivity,
point and plane J/M sources and FP64 DFT monitors -- all bit for bit.
"""
import numpy as np
import pytest

import oracle
import tiled_emulator as TE

DX = np.float32(0.1)
DT = np.float32(0.05)


def wave(T, amp=5e4):
    n = np.arange(T)
    return (amp * np.exp(-(n - 3.0) ** 2 / 8.0) * np.sin(2 * np.pi * n / 5)).astype(np.float32)


def bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                          np.asarray(b, np.float32).view(np.uint32))


# (blt, rows, z-chunks, row width, x-pair family): the one-cell kernel (32-cell rows) and the
# x-pair kernel's 64- and 32-cell rows, at every instance the library builds
CONFIGS = [(b, r, z, 32, False) for r, bs in ((8, (1, 2, 3)), (16, (1, 2, 3, 4, 5, 6)),
                                              (32, (1, 2, 3, 4, 6)))
           for b in bs for z in (1, 3)]
CONFIGS += [(b, r, z, 64, True) for r, bs in ((8, (1, 2, 3)), (16, (1, 2, 3, 4)), (20, (1, 2, 3)),
                                              (24, (1, 2)), (32, (1, 2)))
            for b in bs for z in (1, 3)]
CONFIGS += [(b, r, z, 32, True) for r, bs in ((24, (1, 2)), (32, (1, 2, 3)), (48, (1, 2)))
            for b in bs for z in (1, 3)]


@pytest.mark.parametrize("blt,rows,zc,width,pairs", CONFIGS)
def test_schedule_point_sources(blt, rows, zc, width, pairs):
    shape, T = (71 if width == 64 else 37, 21, 19), 7
    coefs = oracle.coefficients(shape)
    w = wave(T)
    F_ref = oracle.run(shape, coefs, T, sources=[
        oracle.Source("Jz", w, i=18, j=10, k=9), oracle.Source("Mx", w * np.float32(0.5), i=5, j=6, k=7)])
    F = TE.run(shape, coefs, T, blt, rows, zc, DX, sources=[
        dict(comp=2, kind=0, i=18, j=10, k=9, wave=w),
        dict(comp=3, kind=0, i=5, j=6, k=7, wave=w * np.float32(0.5))], width=width,
        pairs=pairs)
    for c in range(6):
        assert bits_equal(F[c], F_ref[c]), oracle.COMPONENTS[c]


@pytest.mark.parametrize("blt,rows,zc,width,pairs",
                         [(2, 8, 2, 32, False), (4, 16, 3, 32, False), (3, 16, 1, 32, False),
                          (6, 32, 2, 32, False), (3, 16, 2, 64, True), (2, 32, 1, 64, True),
                          (1, 24, 2, 32, True), (3, 32, 1, 32, True)])
def test_schedule_plane_source_and_monitors(blt, rows, zc, width, pairs):
    shape, T = (29, 23, 17), 9
    nx, ny, nz = shape
    rng = np.random.default_rng(1)
    eps = np.ones(nx * ny * nz, np.float32)
    eps[rng.random(nx * ny * nz) < 0.3] = 4.0
    coefs = oracle.coefficients(shape, eps_re=eps)
    w = wave(T)
    freqs = np.array([0.5, 1.0, 1.3])
    mons = [oracle.Monitor("Ez", 6, freqs, 0.25), oracle.Monitor("Hy", 5, freqs, 1.0)]
    F_ref = oracle.run(shape, coefs, T, sources=[oracle.Source("Jz", w, k=4, kind=oracle.PLANE_Z)],
                       monitors=mons)
    ct, st = oracle.dft_tables(freqs, float(DT), T)
    emons = [dict(comp=2, k=6, cos=ct, sin=st, scale=0.25, re=np.zeros((3, ny, nx)),
                  im=np.zeros((3, ny, nx))),
             dict(comp=4, k=5, cos=ct, sin=st, scale=1.0, re=np.zeros((3, ny, nx)),
                  im=np.zeros((3, ny, nx)))]
    F = TE.run(shape, coefs, T, blt, rows, zc, DX,
               sources=[dict(comp=2, kind=1, i=0, j=0, k=4, wave=w)], monitors=emons,
               width=width, pairs=pairs)
    for c in range(6):
        assert bits_equal(F[c], F_ref[c]), oracle.COMPONENTS[c]
    for em, om in zip(emons, mons):
        assert np.abs(om.re).max() > 0
        assert np.array_equal(em["re"], om.re) and np.array_equal(em["im"], om.im)


def test_output_windows_tile_the_grid():
    """Every cell is written exactly once per pass and nothing outside the grid."""
    for (width, pairs), blt, rows in [(wp, b, r) for wp in ((32, False), (32, True), (64, True))
                                      for b in range(1, 7) for r in (8, 16, 20, 24, 32, 48)]:
        if rows - 2 * blt < 1:
            continue
        for shape in ((3, 3, 3), (33, 17, 9), (100, 61, 5)):
            nx, ny, nz = shape
            sx, xbase, sy = TE.tile_geometry(blt, rows, width, pairs)
            align = 2 if pairs else 4  # x-pairs: even starts; one cell: 16-byte TMA starts
            assert sx % align == 0 and xbase % align == 0 and xbase + blt <= 0
            assert sx <= width - 2 * blt
            ntx, nty, nzc, zlen = TE.grid_dims(shape, blt, rows, 2, width, pairs)
            cover = np.zeros(nx, int)
            for bx in range(ntx):
                lo = bx * sx + xbase + blt
                for x in range(lo, lo + sx):
                    if 0 <= x < nx:
                        cover[x] += 1
            assert (cover == 1).all()
            assert xbase + blt + ntx * sx >= nx and nty * sy >= ny and nzc * zlen >= nz
