"""Synthetic workloads and host-side set-up helpers.

* ``reference_coefficients`` -- the 12 coefficient arrays gDiamond's constructor builds
  (gDiamond/gdiamond.hpp:20-73 -> set_FDTD_matrices_3D_structure, gDiamond/utils.h:542-690),
  generalised to a per-cell relative permittivity, evaluated with the same operation order and
  rounding (FP32 complex arithmetic, FP64 where the reference promotes) so the arrays are
  bit-identical to the reference's.
* ``vacuum_coefficients`` -- Ca = Da = 1, Cb = Db = dt/dx everywhere (no PML).
* ``gaussian_wave`` -- the benchmark source J(n) = A exp(-(n-delay)^2 / (2 width^2)) sin(2 pi n /
  period) in FP32.
* Seeded permittivity generators for the dielectric-sphere, slab and box workloads.
"""
from __future__ import annotations

import math

import numpy as np

# gDiamond/gdiamond.hpp:893-906 and gDiamond/utils.h:17-22 (eps0 = mu0 = c0 = eta0 = 1).
REF_PI_F32 = np.float32(3.14159265359)
DX = np.float32(1.0) / np.float32(10)
DT = np.float32(0.05)
SOURCE_OMEGA = np.float32(2) * REF_PI_F32 * np.float32(1.0)
J_AMP = np.float32(5e4)
M_AMP = np.float32(5e4)
T_PML = 10


def reference_mz_wave(T):
    """update_FDTD_seq's source M_amp * sin(omega * t * dt), FP32 (gDiamond/gdiamond.hpp:1189).

    The sine is the C library's single-precision sinf, which std::sin(float) calls in the
    reference (numpy's float32 sin is a different implementation).
    """
    import ctypes
    import ctypes.util
    libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
    libm.sinf.restype = ctypes.c_float
    libm.sinf.argtypes = [ctypes.c_float]
    t = np.arange(T, dtype=np.float32)
    arg = (SOURCE_OMEGA * t) * DT
    return np.array([M_AMP * np.float32(libm.sinf(float(a))) for a in arg], np.float32)


def gaussian_wave(T, amp=5e4, period=20.0, width=10.0, delay=40.0):
    n = np.arange(T, dtype=np.float64)
    w = amp * np.exp(-((n - delay) ** 2) / (2.0 * width * width)) * np.sin(2.0 * np.pi * n / period)
    return w.astype(np.float32)


def source_band(n_freqs, dt=DT, period=20.0, width=10.0):
    """n_freqs frequencies evenly spaced over f0 +- 2 sigma_f of the Gaussian source."""
    f0 = 1.0 / (period * float(dt))
    sig = 1.0 / (2.0 * np.pi * width * float(dt))
    return np.linspace(f0 - 2 * sig, f0 + 2 * sig, n_freqs)


def vacuum_coefficients(shape, dx=DX, dt=DT):
    n = int(np.prod(shape))
    cb = np.float32(np.float64(dt) / np.float64(dx))
    one = np.ones(n, np.float32)
    half = np.full(n, cb, np.float32)
    return [one, one, one, half, half, half, one, one, one, half, half, half]


def _stretch_1d(n, t_pml, a_max, sigma_max, omega0):
    """Per-index complex stretch factor along one axis (gDiamond/utils.h:585-619)."""
    re = np.empty(n, np.float32)
    im = np.empty(n, np.float32)
    for i in range(n):
        dist = np.float32(0)
        if i < t_pml:
            dist = np.float32(1.0 - float(np.float32(i) / np.float32(t_pml)))
        if i + t_pml >= n:
            dist = np.float32(1.0 - float(np.float32(n - i - 1) / np.float32(t_pml)))
        d3 = math.pow(float(dist), 3.0)
        re[i] = np.float32(1.0 + float(a_max) * d3)
        im[i] = np.float32(float(sigma_max) * d3 / float(np.float32(omega0 * np.float32(1.0))))
    return re, im


def _cmul(ar, ai, br, bi):
    return (ar * br - ai * bi).astype(np.float32), (ar * bi + ai * br).astype(np.float32)


def _cdiv(ar, ai, br, bi):
    den = (br * br + bi * bi).astype(np.float32)
    return ((ar * br + ai * bi) / den).astype(np.float32), ((ai * br - ar * bi) / den).astype(np.float32)


def _pair(mre, mim, omega0, dt, dx):
    re = np.where(mre < 1, np.float32(1), mre).astype(np.float32)
    sigma = np.abs((omega0 * np.float32(1.0)) * mim).astype(np.float32)
    tmp = ((sigma * dt).astype(np.float64) / (2.0 * re.astype(np.float64) * 1.0)).astype(np.float32)
    t64 = tmp.astype(np.float64)
    ca = ((1.0 - t64) / (1.0 + t64)).astype(np.float32)
    cb = ((dt / (re * np.float32(1.0))).astype(np.float32).astype(np.float64) / (1.0 + t64)
          / np.float64(dx)).astype(np.float32)
    return ca, cb


def reference_coefficients(shape, eps_re=None, eps_im=None, dx=DX, dt=DT, omega0=SOURCE_OMEGA,
                           t_pml=T_PML):
    """12 FP32 arrays (Cax..Dbz, flat, x-fastest) with the reference's graded pseudo-PML."""
    nx, ny, nz = shape
    a_max = np.float32(2.0)
    denom = np.float32(2) * np.float32(1.0) * np.float32(t_pml) * np.float32(dx)
    # t_pml = 0: no graded layer (e.g. under CPML layers), every stretch factor 1
    sigma_max = np.float32(-4.0 * math.log(1e-5) / float(denom)) if t_pml > 0 else np.float32(0)
    sxr, sxi = _stretch_1d(nx, t_pml, a_max, sigma_max, omega0)
    syr, syi = _stretch_1d(ny, t_pml, a_max, sigma_max, omega0)
    szr, szi = _stretch_1d(nz, t_pml, a_max, sigma_max, omega0)
    X = (slice(None),)
    sxr = np.broadcast_to(sxr[None, None, :], (nz, ny, nx))
    sxi = np.broadcast_to(sxi[None, None, :], (nz, ny, nx))
    syr = np.broadcast_to(syr[None, :, None], (nz, ny, nx))
    syi = np.broadcast_to(syi[None, :, None], (nz, ny, nx))
    szr = np.broadcast_to(szr[:, None, None], (nz, ny, nx))
    szi = np.broadcast_to(szi[:, None, None], (nz, ny, nx))
    del X
    if eps_re is None:
        er = np.ones((nz, ny, nx), np.float32)
    else:
        er = np.asarray(eps_re, np.float32).reshape(nz, ny, nx)
    ei = np.zeros((nz, ny, nx), np.float32) if eps_im is None else \
        np.asarray(eps_im, np.float32).reshape(nz, ny, nx)
    one = np.ones((nz, ny, nx), np.float32)
    zero = np.zeros((nz, ny, nx), np.float32)
    out = [None] * 12

    def axis(mr, mi, a, b, c):
        # (m * s_a * s_b) / s_c
        r, i = _cmul(mr, mi, a[0], a[1])
        r, i = _cmul(r, i, b[0], b[1])
        return _cdiv(r, i, c[0], c[1])

    sx, sy, sz = (sxr, sxi), (syr, syi), (szr, szi)
    for comp, (a, b, c) in enumerate(((sy, sz, sx), (sx, sz, sy), (sx, sy, sz))):
        r, i = axis(er, ei, a, b, c)
        ca, cb = _pair(r, i, omega0, dt, dx)
        out[comp], out[3 + comp] = ca.reshape(-1), cb.reshape(-1)
        r, i = axis(one, zero, a, b, c)
        da, db = _pair(r, i, omega0, dt, dx)
        out[6 + comp], out[9 + comp] = da.reshape(-1), db.reshape(-1)
    return out


# ------------------------------------------------------------------ seeded geometries


def spheres_eps(shape, n_spheres=200, r_range=(4, 24), eps_range=(1.0, 12.0), seed=0):
    """Dielectric spheres, centres uniform in the grid, later spheres overwrite earlier ones."""
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    eps = np.ones((nz, ny, nx), np.float32)
    for _ in range(n_spheres):
        c = rng.uniform([0, 0, 0], [nx, ny, nz])
        r = rng.uniform(*r_range)
        e = np.float32(rng.uniform(*eps_range))
        x0, x1 = max(int(c[0] - r), 0), min(int(c[0] + r) + 1, nx)
        y0, y1 = max(int(c[1] - r), 0), min(int(c[1] + r) + 1, ny)
        z0, z1 = max(int(c[2] - r), 0), min(int(c[2] + r) + 1, nz)
        zz, yy, xx = np.ogrid[z0:z1, y0:y1, x0:x1]
        inside = (xx - c[0]) ** 2 + (yy - c[1]) ** 2 + (zz - c[2]) ** 2 <= r * r
        eps[z0:z1, y0:y1, x0:x1][inside] = e
    return eps.reshape(-1)


def slab_eps(shape, rng):
    """One dielectric slab: thickness U[8,32], eps U[2,12], axis random."""
    nx, ny, nz = shape
    eps = np.ones((nz, ny, nx), np.float32)
    axis = int(rng.integers(0, 3))
    n_ax = (nx, ny, nz)[axis]
    th = int(rng.integers(8, 33))
    th = min(th, n_ax - 2)
    lo = int(rng.integers(1, n_ax - th))
    e = np.float32(rng.uniform(2.0, 12.0))
    sl = [slice(None)] * 3
    sl[2 - axis] = slice(lo, lo + th)
    eps[tuple(sl)] = e
    return eps.reshape(-1)


def box_eps(shape, params):
    """Axis-aligned dielectric box from (cx, cy, cz, side, eps) (side in cells)."""
    nx, ny, nz = shape
    cx, cy, cz, side, e = params
    eps = np.ones((nz, ny, nx), np.float32)
    h = side / 2.0
    x0, x1 = int(round(cx - h)), int(round(cx + h))
    y0, y1 = int(round(cy - h)), int(round(cy + h))
    z0, z1 = int(round(cz - h)), int(round(cz + h))
    eps[max(z0, 0):z1, max(y0, 0):y1, max(x0, 0):x1] = np.float32(e)
    return eps.reshape(-1)
