"""CPU emulation of the tiled kernel's schedule (gdiamond_b200/csrc/k_tiled.cu).

Test infrastructure only.  It replays, CTA by CTA and z-iteration by z-iteration, exactly the
dataflow of ``fdtd_tiled<BLT, ROWS>``: the TMA-staged plane of each iteration (zero outside
the grid), the per-level register rotation, the warp shuffles along x (a lane at the warp edge
gets its own value), the shared-memory y-neighbour planes (clamped rows), the trapezoid output
window and the z-chunk warm-up.  Arrays of shape [ROWS, 32] stand for the CTA's threads.

It plays the role of the reference's CPU "simulations" of its GPU tile schedules
(e.g. update_FDTD_mix_mapping_sequential_ver3, gDiamond/gdiamond_gpu_mm_ver3.cuh): the
schedule is checked bit for bit against the oracle on the CPU before any GPU run, at odd
grid sizes and every (BLT, ROWS, z-chunks) the kernel is built for.
"""
from __future__ import annotations

import numpy as np


def tile_geometry(blt, rows, width=32, pairs=None):
    """(sx, xbase, sy).  One-cell kernel (fdtd_tiled): x tile starts are multiples of 4 floats
    (the TMA rule).  x-pair family (fdtd_tiled2, 64- or 32-cell rows; pairs defaults to
    width == 64): the boxes start at the tile start rounded down to 8 elements, so tile starts
    only need to be even and a tile writes width - 2*blt columns."""
    if pairs is None:
        pairs = width == 64
    if pairs:
        sx = width - 2 * blt
        xbase = -2 * ((blt + 1) // 2)
    else:
        sx = 4 * ((width - 2 * blt) // 4)
        xbase = -4 * ((blt + 3) // 4)
    sy = rows - 2 * blt
    return sx, xbase, sy


def grid_dims(shape, blt, rows, z_chunks, width=32, pairs=None):
    nx, ny, nz = shape
    sx, xbase, sy = tile_geometry(blt, rows, width, pairs)
    first = xbase + blt
    ntx = -(-(nx - first) // sx)
    nty = -(-ny // sy)
    zlen = -(-nz // z_chunks)
    nzc = -(-nz // zlen)
    return ntx, nty, nzc, zlen


def material_table(coefs):
    """uint16 map + table rows ordered Cax..Dbz (the device dedup's ids are arbitrary; the
    schedule does not depend on them)."""
    stacked = np.stack([np.asarray(c, np.float32).view(np.uint32) for c in coefs], axis=1)
    uniq, inv = np.unique(stacked, axis=0, return_inverse=True)
    return inv.reshape(-1).astype(np.int64), uniq.view(np.float32)


def _plane(F3, X, Y, z, width, rows):
    """[rows, width] box at (X, Y, z), zero outside the grid (TMA out-of-bounds fill)."""
    nz, ny, nx = F3.shape
    out = np.zeros((rows, width), F3.dtype)
    if z < 0 or z >= nz:
        return out
    y0, y1 = max(Y, 0), min(Y + rows, ny)
    x0, x1 = max(X, 0), min(X + width, nx)
    if y0 < y1 and x0 < x1:
        out[y0 - Y:y1 - Y, x0 - X:x1 - X] = F3[z, y0:y1, x0:x1]
    return out


def _shfl_up(v, width):
    """x-1 neighbour.  Width 32 (one cell per lane): lane 0 gets its own value.  Width 64 (an
    x-pair per lane): cell 0 gets cell 1, the odd cell of its own lane."""
    out = v.copy()
    out[:, 1:] = v[:, :-1]
    if width == 64:
        out[:, 0] = v[:, 1]
    return out


def _shfl_down(v, width):
    """x+1 neighbour; at the upper edge lane 31 gets its own value (width 64: cell 62)."""
    out = v.copy()
    out[:, :-1] = v[:, 1:]
    if width == 64:
        out[:, -1] = v[:, -2]
    return out


def _source_value(sources, comp, x, y, e, t, dx):
    """Per-thread sum of source waveforms of component comp at plane e (float32)."""
    acc = np.zeros(x.shape, np.float32)
    any_ = np.zeros(x.shape, bool)
    for s in sources:
        if s["comp"] != comp:
            continue
        if s["kind"] == 0:
            hit = (x == s["i"]) & (y == s["j"]) & (e == s["k"])
        else:
            hit = np.full(x.shape, e == s["k"])
        w = np.float32(s["wave"][t]) if t < len(s["wave"]) else np.float32(0)
        acc = np.where(hit, acc + w, acc).astype(np.float32)
        any_ |= hit
    return acc, any_


def tiled_pass(shape, F, mat, table, blt, rows, z_chunks, t0, dx, sources=(), monitors=(),
               width=32, pairs=None):
    """One launch: BLT steps from field set F (6 flat float32 arrays) into a new set.
    width 32 emulates fdtd_tiled (k_tiled.cu) or, with pairs, fdtd_tiled2's 32-cell rows;
    width 64 emulates fdtd_tiled2's 64-cell rows (k_tiled2.cu)."""
    nx, ny, nz = shape
    B, TY, W = blt, rows, width
    sx, xbase, sy = tile_geometry(B, TY, W, pairs)
    ntx, nty, nzc, zlen = grid_dims(shape, B, TY, z_chunks, W, pairs)
    F3 = [np.asarray(f, np.float32).reshape(nz, ny, nx) for f in F]
    M3 = mat.reshape(nz, ny, nx)
    dst = [np.full((nz, ny, nx), np.nan, np.float32) for _ in range(6)]
    dx = np.float32(dx)
    lx = np.arange(W)[None, :]
    ly = np.arange(TY)[:, None]
    f32 = np.float32
    for bz in range(nzc):
        z0 = bz * zlen
        if z0 >= nz:
            continue
        z1 = min(nz, z0 + zlen)
        ps = z0 - B
        niter = (z1 - z0) + 2 * B
        for by in range(nty):
            for bx in range(ntx):
                X = bx * sx + xbase
                Y = by * sy - B
                x = X + lx + 0 * ly
                y = Y + ly + 0 * lx
                col_int = (x >= 1) & (x <= nx - 2) & (y >= 1) & (y <= ny - 2)
                col_out = ((lx >= B) & (lx < B + sx) & (ly >= B) & (ly < TY - B) & (x >= 0)
                           & (x < nx) & (y >= 0) & (y < ny))
                Ep = np.zeros((B + 1, 3, TY, W), f32)
                Hp = np.zeros((B + 1, 3, TY, W), f32)
                mq = np.zeros((B + 1, TY, W), np.int64)
                hbuf = np.zeros((2, 2, TY, W), f32)
                ebuf = np.zeros((B, 2, TY, W), f32)
                ym = np.maximum(np.arange(TY) - 1, 0)
                yp = np.minimum(np.arange(TY) + 1, TY - 1)
                for it in range(niter):
                    p = ps + it
                    S = [_plane(F3[c], X, Y, p, W, TY) for c in range(6)]
                    mq[1:] = mq[:-1].copy()
                    mq[0] = _plane(M3, X, Y, p, W, TY)
                    Hc = [S[3], S[4], S[5]]
                    hz_ym, hx_ym = S[5][ym], S[3][ym]
                    Eo = [S[0], S[1], S[2]]
                    EnPrev = None
                    for s in range(1, B + 1):
                        e = p - s + 1
                        t = t0 + s - 1
                        hz_xm, hy_xm = _shfl_up(Hc[2], W), _shfl_up(Hc[1], W)
                        cx = (Hc[2] - hz_ym) - (Hc[1] - Hp[s - 1][1])
                        cy = (Hc[0] - Hp[s - 1][0]) - (Hc[2] - hz_xm)
                        cz = (Hc[1] - hy_xm) - (Hc[0] - hx_ym)
                        En = [Eo[0].copy(), Eo[1].copy(), Eo[2].copy()]
                        if col_int.any() and 1 <= e <= nz - 2:
                            cs = [cx, cy, cz]
                            for c in range(3):
                                v, hit = _source_value(sources, c, x, y, e, t, dx)
                                cs[c] = np.where(hit, cs[c] - v * dx, cs[c]).astype(f32)
                            tb = table[mq[s - 1]]
                            for c in range(3):
                                new = tb[..., c] * Eo[c] + tb[..., 3 + c] * cs[c]
                                En[c] = np.where(col_int, new, Eo[c]).astype(f32)
                        ez_xp, ey_xp = _shfl_down(Ep[s][2], W), _shfl_down(Ep[s][1], W)
                        ex_yp, ez_yp = ebuf[s - 1][0][yp], ebuf[s - 1][1][yp]
                        cx = (En[1] - Ep[s][1]) - (ez_yp - Ep[s][2])
                        cy = (ez_xp - Ep[s][2]) - (En[0] - Ep[s][0])
                        cz = (ex_yp - Ep[s][0]) - (ey_xp - Ep[s][1])
                        Hn = [Hp[s - 1][0].copy(), Hp[s - 1][1].copy(), Hp[s - 1][2].copy()]
                        if col_int.any() and 1 <= e - 1 <= nz - 2:
                            cs = [cx, cy, cz]
                            for c in range(3):
                                v, hit = _source_value(sources, 3 + c, x, y, e - 1, t, dx)
                                cs[c] = np.where(hit, cs[c] - v * dx, cs[c]).astype(f32)
                            tb = table[mq[s]]
                            for c in range(3):
                                new = tb[..., 6 + c] * Hp[s - 1][c] + tb[..., 9 + c] * cs[c]
                                Hn[c] = np.where(col_int, new, Hp[s - 1][c]).astype(f32)
                        for m in monitors:
                            mk = e if m["comp"] < 3 else e - 1
                            if m["k"] == mk and z0 <= mk < z1:
                                v = (En[m["comp"]] if m["comp"] < 3 else Hn[m["comp"] - 3])
                                ct, st = m["cos"][t], m["sin"][t]
                                ys, xs = np.nonzero(col_out)
                                vv = v[ys, xs].astype(np.float64)
                                gy, gx = y[ys, xs], x[ys, xs]
                                for f in range(len(ct)):
                                    m["re"][f, gy, gx] += (vv * ct[f]) * m["scale"]
                                    m["im"][f, gy, gx] -= (vv * st[f]) * m["scale"]
                        if s < B:
                            hbuf[s & 1][0] = Hn[2]
                            hbuf[s & 1][1] = Hn[0]
                        ebuf[s - 1][0] = En[0]
                        ebuf[s - 1][1] = En[2]
                        if s >= 2:
                            Ep[s - 1] = np.stack(EnPrev)
                        EnPrev = [a.copy() for a in En]
                        Hp[s - 1] = np.stack(Hc)
                        if s < B:
                            hz_ym, hx_ym = hbuf[s & 1][0][ym], hbuf[s & 1][1][ym]
                            Hc = Hn
                            Eo = [Ep[s][0].copy(), Ep[s][1].copy(), Ep[s][2].copy()]
                        else:
                            EnB, HnB = En, Hn
                    Ep[B] = np.stack(EnPrev)
                    eB, hB = p - B + 1, p - B
                    ys, xs = np.nonzero(col_out)
                    gy, gx = y[ys, xs], x[ys, xs]
                    if z0 <= eB < z1:
                        for c in range(3):
                            dst[c][eB, gy, gx] = EnB[c][ys, xs]
                    if z0 <= hB < z1:
                        for c in range(3):
                            dst[3 + c][hB, gy, gx] = HnB[c][ys, xs]
    return [d.reshape(-1) for d in dst]


def run(shape, coefs, T, blt, rows, z_chunks, dx, sources=(), monitors=(), fields=None,
        width=32, pairs=None):
    """T steps in passes of BLT (a final shorter pass for the remainder), as fdtd_step."""
    nx, ny, nz = shape
    mat, table = material_table(coefs)
    F = fields or [np.zeros(nx * ny * nz, np.float32) for _ in range(6)]
    t = 0
    while t < T:
        b = min(blt, T - t)
        F = tiled_pass(shape, F, mat, table, b, rows, z_chunks, t, dx, sources, monitors, width,
                       pairs)
        t += b
    return F
