"""CPU: the schedule of the CPML shell companion, replayed with the numpy CPML stepper.

With CPML layers the library advances the grid k steps with the plain update (the tiled
kernel) and then recomputes the cells the layers can reach (cpml_companion in fdtd_capi.cu):
step j of the block updates E on W_{e_j} and H on W_{e_j - 1}, e_j = 3k - 2(j - 1), where W_r
is every cell outside the inner box (positions whose updates involve no layer) shrunk by r on
each side with a layer; step 1 reads the block's input fields, intermediate steps run in place
in a third field set, the last writes into the tiled kernel's output; face cells are carried
from input to output.  Replayed here with oracle/cpml.step over several blocks, the result must
equal plain CPML stepping bit for bit, and the third field set (filled with NaN before each
block) must never be read outside what the schedule wrote.
"""
import numpy as np
import pytest

import oracle
from oracle import cpml
from gdiamond_b200 import workloads as W

F32 = np.float32


def inner_box(tables, shape):
    """Per axis x, y, z: (lo, hi, layer below, layer above), as fdtd_set_cpml computes it."""
    out = []
    for a, n in enumerate(shape):
        slot_e, slot_h = tables[a][0][0], tables[a][1][0]
        lo, hi = 0, n
        for p in range(n):
            if slot_e[p] >= 0 or slot_h[p] >= 0:
                if 2 * p < n:
                    lo = max(lo, p + 1)
                else:
                    hi = min(hi, p)
        out.append((lo, hi, lo > 0, hi < n))
    return out


def region(box, shape, r):
    """Interior-shaped [z][y][x] mask of W_r."""
    ins = []
    for a, n in enumerate(shape):
        lo, hi, lo_on, hi_on = box[a]
        lo_r = lo + r if lo_on else 0
        hi_r = hi - r if hi_on else n
        p = np.arange(1, n - 1)
        ins.append((p >= lo_r) & (p < hi_r))
    inside = ins[2][:, None, None] & ins[1][None, :, None] & ins[0][None, None, :]
    return ~inside


def copy_faces(dst, src):
    for d, s in zip(dst, src):
        for sl in ((0,), (-1,), (slice(None), 0), (slice(None), -1), (Ellipsis, 0), (Ellipsis, -1)):
            d[sl] = s[sl]


@pytest.mark.parametrize("k,faces", [(1, 63), (2, 63), (3, 63), (2, 16 | 32), (3, 1 | 8 | 32)])
def test_companion_schedule_equals_cpml_stepping(k, faces):
    shape, L, nblocks = (40, 36, 44), 4, 3
    nx, ny, nz = shape
    eps = W.spheres_eps(shape, n_spheres=3, r_range=(3, 5), eps_range=(2.0, 4.0), seed=3)
    coefs = W.reference_coefficients(shape, eps_re=eps, t_pml=0)
    C = [np.asarray(c, F32).reshape(nz, ny, nx) for c in coefs]
    tables = [[cpml.profile(n, L, bool(faces >> 2 * a & 1), bool(faces >> (2 * a + 1) & 1),
                            0.1, 0.05, kappa_max=1.5, half=h == 1) for h in (0, 1)]
              for a, n in enumerate(shape)]
    TE, TH = cpml.axis_tables(tables, shape)
    NE, NH = cpml.axis_tables(cpml.no_layers(shape), shape)
    box = inner_box(tables, shape)
    T = k * nblocks
    w = W.gaussian_wave(T, delay=4.0, width=2.0, period=5.0)
    src = [oracle.Source("Jx", w, k=L + 2, kind=oracle.PLANE_Z),       # near the z layer
           oracle.Source("Jy", w, i=2, j=ny // 2, k=nz // 2),           # inside the x layer
           oracle.Source("Mz", w * F32(0.5), i=nx // 3, j=ny - 4, k=nz // 2)]
    rng = np.random.default_rng(k)
    A = [(rng.standard_normal((nz, ny, nx)) * 0.1).astype(F32) for _ in range(6)]
    for f in A:
        copy_faces([f], [np.zeros_like(f)])
    inner = (nz - 2, ny - 2, nx - 2)
    zeros6 = lambda: [np.zeros(inner, F32) for _ in range(6)]

    ref = [f.copy() for f in A]
    pe, ph = zeros6(), zeros6()
    for t in range(T):
        cpml.step(shape, C, ref, ref, TE, TH, pe, ph, t, src)

    cur = [f.copy() for f in A]
    qe, qh = zeros6(), zeros6()          # psi: the companion's alone
    ne, nh = zeros6(), zeros6()          # unused by the plain update
    for blk in range(nblocks):
        t0 = blk * k
        B = [f.copy() for f in cur]
        for j in range(k):               # the tiled kernel: plain update everywhere
            cpml.step(shape, C, B, B, NE, NH, ne, nh, t0 + j, src)
        S = [np.full_like(f, np.nan) for f in cur]
        for j in range(1, k + 1):
            Fi = cur if j == 1 else S
            Fo = B if j == k else S
            re_ = 3 * k - 2 * (j - 1)
            if Fi is not Fo:
                copy_faces(Fo, Fi)
            cpml.step(shape, C, Fi, Fo, TE, TH, qe, qh, t0 + j - 1, src,
                      mask_e=region(box, shape, re_), mask_h=region(box, shape, re_ - 1))
        cur = B
    for c in range(6):
        assert not np.isnan(cur[c]).any(), c
        assert np.array_equal(cur[c].view(np.uint32), ref[c].view(np.uint32)), c
    for a, b in zip(qe + qh, pe + ph):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
