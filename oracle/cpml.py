"""Test infrastructure only: CPU restatement of the CPML stepper (numpy, FP32).

The reference has no CPML (its absorber is the graded pseudo-PML of gDiamond/utils.h:585-660);
this is the checker for the GPU's CPML layers (fdtd_set_cpml).  One step is the reference's
E sweep then H sweep (gDiamond/gdiamond.hpp:1193-1221) over interior cells, except that a
spatial difference d along an axis where the position lies inside a layer becomes
d * (1/kappa) + psi, psi <- b * psi + a * d.  A component whose differences all lie outside
every layer uses the reference's formula unchanged.  numpy float32 arithmetic rounds every
operation to nearest even and never fuses, as the GPU kernels do, so fields agree bit for bit.

`profile` restates the profile formula (in FP64, cast to FP32) for comparison with the tables
the library computed; `run` takes those tables (b, a, 1/kappa, slot per axis and position
kind) so the stepper check does not depend on libm's last bit of exp/pow.
"""
from __future__ import annotations

import math

import numpy as np

F32 = np.float32


def profile(n, L, lo, hi, dx, dt, order=3.0, reflection=1e-6, kappa_max=1.0, alpha_max=0.05,
            half=False):
    """(slot, b, a, inv_kappa) of one axis: E positions x = p, H positions x = p + 1/2."""
    sigma_max = -(order + 1.0) * math.log(reflection) / (2.0 * L * dx)
    slot = np.full(n, -1, np.int32)
    b = np.ones(n, np.float32)
    a = np.zeros(n, np.float32)
    ik = np.ones(n, np.float32)
    for p in range(n):
        x = p + (0.5 if half else 0.0)
        rho, s = 0.0, -1
        if lo and x < L:
            rho, s = (L - x) / L, p
        if hi and x > n - 1 - L:
            rho, s = (x - (n - 1 - L)) / L, L + (p - (n - 1 - L))
        if not rho > 0.0:
            continue
        rho = min(rho, 1.0)
        rm = rho ** order
        sigma = sigma_max * rm
        kappa = 1.0 + (kappa_max - 1.0) * rm
        alpha = alpha_max * (1.0 - rho)
        bb = math.exp(-(sigma / kappa + alpha) * dt)
        den = sigma * kappa + kappa * kappa * alpha
        slot[p] = s
        b[p] = bb
        a[p] = sigma / den * (bb - 1.0) if den > 0 else 0.0
        ik[p] = 1.0 / kappa
    return slot, b, a, ik


def _axis_view(v, axis):
    """Broadcast a per-position table of `axis` (0 x, 1 y, 2 z) over [z][y][x]."""
    shape = [1, 1, 1]
    shape[2 - axis] = v.shape[0]
    return v.reshape(shape)


def axis_tables(tables, shape):
    """Per axis (E positions, H positions) the tables of `run` restricted to interior positions
    and broadcast over [z][y][x]: (inside-layer mask, b, a, 1/kappa)."""
    nx, ny, nz = shape

    def tab(axis, kind):
        slot, b, a, ik = tables[axis][kind]
        sl = (slice(1, (nz, ny, nx)[2 - axis] - 1),)
        return (_axis_view(np.asarray(slot)[sl] >= 0, axis),
                _axis_view(np.asarray(b, F32)[sl], axis), _axis_view(np.asarray(a, F32)[sl], axis),
                _axis_view(np.asarray(ik, F32)[sl], axis))

    return [tab(ax, 0) for ax in range(3)], [tab(ax, 1) for ax in range(3)]


def _source_terms(shape, sources, comp_base, t):
    """Per-component FP32 sums of the waveforms of the sources covering each interior cell
    (the device's source_value), and where any covers."""
    nx, ny, nz = shape
    inner = (nz - 2, ny - 2, nx - 2)
    acc = [np.zeros(inner, F32) for _ in range(3)]
    hit = [np.zeros(inner, bool) for _ in range(3)]
    names = ("Jx", "Jy", "Jz") if comp_base == 0 else ("Mx", "My", "Mz")
    for s in sources:
        if s.component not in names:
            continue
        c = names.index(s.component)
        w = F32(s.wave[t]) if t < len(s.wave) else F32(0)
        if s.kind == 0:
            idx = (s.k - 1, s.j - 1, s.i - 1)
            if all(0 <= q < e for q, e in zip(idx, inner)):
                acc[c][idx] = acc[c][idx] + w
                hit[c][idx] = True
        elif 1 <= s.k <= nz - 2:
            acc[c][s.k - 1] = acc[c][s.k - 1] + w
            hit[c][s.k - 1] = True
    return acc, hit


def step(shape, C, Fi, Fo, TE, TH, psi_e, psi_h, t, sources=(), dx=0.1, mask_e=None,
         mask_h=None):
    """One step: E from the fields of step t in Fi into Fo, then H from Fi's H and Fo's new E
    into Fo (Fi is Fo: in place), on the interior cells where mask_e / mask_h (None: all) hold;
    psi changes only there.  C: the 12 coefficient arrays [z][y][x]; TE, TH from axis_tables;
    psi_e, psi_h: six interior-shaped arrays each (exy exz eyz eyx ezx ezy; hxz hxy hyx hyz hzy
    hzx)."""
    nx, ny, nz = shape
    dx = F32(dx)
    I = (slice(1, nz - 1), slice(1, ny - 1), slice(1, nx - 1))
    z, y, x = I

    def stretched(d, tb, psi, m):
        lay, b, a, ik = tb
        lay = np.broadcast_to(lay, d.shape)
        p = np.where(lay, b * psi + a * d, psi)
        psi[...] = p if m is None else np.where(m, p, psi)
        return np.where(lay, d * ik + p, d), lay

    def put(dst, new, m):
        dst[I] = new if m is None else np.where(m, new, dst[I])

    Ex, Ey, Ez, Hx, Hy, Hz = Fi
    d = {"dyHz": Hz[I] - Hz[z, 0:ny - 2, x], "dzHy": Hy[I] - Hy[0:nz - 2, y, x],
         "dzHx": Hx[I] - Hx[0:nz - 2, y, x], "dxHz": Hz[I] - Hz[z, y, 0:nx - 2],
         "dxHy": Hy[I] - Hy[z, y, 0:nx - 2], "dyHx": Hx[I] - Hx[z, 0:ny - 2, x]}
    cur = []
    for (n1, t1, p1, n2, t2, p2) in (("dyHz", TE[1], psi_e[0], "dzHy", TE[2], psi_e[1]),
                                     ("dzHx", TE[2], psi_e[2], "dxHz", TE[0], psi_e[3]),
                                     ("dxHy", TE[0], psi_e[4], "dyHx", TE[1], psi_e[5])):
        s1, m1 = stretched(d[n1], t1, p1, mask_e)
        s2, m2 = stretched(d[n2], t2, p2, mask_e)
        cur.append(np.where(m1 | m2, s1 - s2, d[n1] - d[n2]))
    acc, hit = _source_terms(shape, sources, 0, t)
    for c in range(3):
        cur[c] = np.where(hit[c], cur[c] - acc[c] * dx, cur[c])
    for c in range(3):
        put(Fo[c], C[c][I] * Fi[c][I] + C[3 + c][I] * cur[c], mask_e)
    Ex, Ey, Ez = Fo[0], Fo[1], Fo[2]
    d = {"dzEy": Ey[2:nz, y, x] - Ey[I], "dyEz": Ez[z, 2:ny, x] - Ez[I],
         "dxEz": Ez[z, y, 2:nx] - Ez[I], "dzEx": Ex[2:nz, y, x] - Ex[I],
         "dyEx": Ex[z, 2:ny, x] - Ex[I], "dxEy": Ey[z, y, 2:nx] - Ey[I]}
    cur = []
    for (n1, t1, p1, n2, t2, p2) in (("dzEy", TH[2], psi_h[0], "dyEz", TH[1], psi_h[1]),
                                     ("dxEz", TH[0], psi_h[2], "dzEx", TH[2], psi_h[3]),
                                     ("dyEx", TH[1], psi_h[4], "dxEy", TH[0], psi_h[5])):
        s1, m1 = stretched(d[n1], t1, p1, mask_h)
        s2, m2 = stretched(d[n2], t2, p2, mask_h)
        cur.append(np.where(m1 | m2, s1 - s2, d[n1] - d[n2]))
    acc, hit = _source_terms(shape, sources, 3, t)
    for c in range(3):
        cur[c] = np.where(hit[c], cur[c] - acc[c] * dx, cur[c])
    for c in range(3):
        put(Fo[3 + c], C[6 + c][I] * Fi[3 + c][I] + C[9 + c][I] * cur[c], mask_h)


def run(shape, coefs, T, tables, sources=(), dx=0.1, t0=0, fields=None):
    """T steps with CPML layers.  tables[axis][kind] = (slot, b, a, inv_kappa), kind 0 = E
    positions, 1 = H positions.  sources: oracle.Source list.  Returns the 6 fields (flat)."""
    nx, ny, nz = shape
    F = [np.zeros((nz, ny, nx), F32) if fields is None else
         np.asarray(fields[c], F32).reshape(nz, ny, nx).copy() for c in range(6)]
    C = [np.asarray(c, F32).reshape(nz, ny, nx) for c in coefs]
    TE, TH = axis_tables(tables, shape)
    inner = (nz - 2, ny - 2, nx - 2)
    psi_e = [np.zeros(inner, F32) for _ in range(6)]
    psi_h = [np.zeros(inner, F32) for _ in range(6)]
    for q in range(T):
        step(shape, C, F, F, TE, TH, psi_e, psi_h, t0 + q, sources, dx)
    return [f.reshape(-1) for f in F]


def no_layers(shape):
    """Tables with every position outside any layer (the stepper is then the reference's)."""
    out = []
    for n in shape:
        z = (np.full(n, -1, np.int32), np.ones(n, F32), np.zeros(n, F32), np.ones(n, F32))
        out.append([z, z])
    return out
