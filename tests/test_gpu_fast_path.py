"""GPU: the uniform-material fast path of the tiled x-pair kernels against the general path and
the oracle (needs a GPU).

When the material held by the most cells has Ca = Da = 1 and one Cb / Db on all axes, warps
whose cells all hold it (off the grid faces, no source in range) update E' = E + Cb*curl H and
H' = H + Db*curl E with paired FP32 instructions.  1*x == x, so the result must equal the
general per-cell path and the oracle (gDiamond/gdiamond.hpp:1193-1221 restated) bit for bit:
checked on vacuum (every interior warp fast), on dielectric spheres inside the graded PML shell
(fast and general warps mixed within a tile), with point and plane sources and DFT monitors,
for every single-grid instance family and in batches.
"""
import numpy as np
import pytest

import oracle
import gdiamond_b200 as gd
from gdiamond_b200 import workloads as W
from test_gpu_parity import assert_fields_match, osrc

pytestmark = pytest.mark.gpu


def run(shape, coefs, T, sources, mons, fast, **kw):
    sim = gd.Simulation(*shape, **kw)
    sim.set_coefficients(coefs)
    sim.set_fast_path(fast)
    sim.set_sources(sources)
    mids = [sim.add_dft_monitor(m["component"], m["k"], m["freqs"], m["scale"]) for m in mons]
    sim.step(T)
    sim.sync()
    out = (sim.fields(), [sim.get_dft(m) for m in mids], sim.fast_path, sim.config())
    sim.close()
    return out


def case(shape, T, medium):
    if medium == "vacuum":
        coefs = W.vacuum_coefficients(shape)
    else:
        eps = W.spheres_eps(shape, n_spheres=10, r_range=(3, 8), eps_range=(2.0, 9.0), seed=5)
        coefs = W.reference_coefficients(shape, eps_re=eps)  # graded PML shell too
    nx, ny, nz = shape
    w = W.gaussian_wave(T, delay=5.0, width=2.0, period=6.0)
    sources = [dict(component="Jz", wave=w, i=nx // 2, j=ny // 2, k=nz // 2),
               dict(component="Mx", wave=w * np.float32(0.25), i=nx // 3, j=ny // 4, k=nz // 3),
               dict(component="Jy", wave=w * np.float32(0.5), k=nz - 6, kind=gd.SRC_PLANE_Z)]
    freqs = W.source_band(3, period=6.0, width=2.0)
    mons = [dict(component="Ez", k=nz // 2 + 2, freqs=freqs, scale=1.0),
            dict(component="Hy", k=nz // 3, freqs=freqs, scale=0.5)]
    return coefs, sources, mons


INSTANCES = [("tiled_w32p", b, r) for r, bs in ((24, (1, 2)), (32, (1, 2, 3)), (48, (1, 2)))
             for b in bs]
INSTANCES += [("tiled_w64", b, r) for r, bs in ((16, (1, 2, 3, 4)), (24, (1, 2))) for b in bs]


@pytest.mark.parametrize("medium", ["vacuum", "spheres"])
@pytest.mark.parametrize("family,blt,rows", INSTANCES)
def test_fast_path_equals_general_path_and_oracle(family, blt, rows, medium):
    shape, T = (70, 52, 41), 13
    coefs, sources, mons = case(shape, T, medium)
    omons = [oracle.Monitor(m["component"], m["k"], m["freqs"], m["scale"]) for m in mons]
    F_ref = oracle.run(shape, coefs, T, sources=[osrc(s) for s in sources], monitors=omons)
    kw = dict(kernel=family, blt=blt, tile_rows=rows, z_chunks=2)
    Ff, Df, active, cfg = run(shape, coefs, T, sources, mons, True, **kw)
    Fg, Dg, inactive, _ = run(shape, coefs, T, sources, mons, False, **kw)
    assert active and not inactive
    assert (cfg["blt"], cfg["tile_rows"]) == (blt, rows)
    assert_fields_match(Ff, F_ref, f"fast {family} {blt} {rows} {medium}")
    assert_fields_match(Fg, F_ref, f"general {family} {blt} {rows} {medium}")
    for (re, im), (rg, ig), om in zip(Df, Dg, omons):
        assert np.abs(om.re).max() > 0
        assert np.array_equal(re, om.re) and np.array_equal(im, om.im)
        assert np.array_equal(rg, om.re) and np.array_equal(ig, om.im)


@pytest.mark.parametrize("storage", ["f16", "bf16", "f16e"])
def test_fast_path_16bit_storage_equals_general_path(storage):
    """The 16-bit storages round once per pass in both paths: fast == general bit for bit."""
    shape, T = (70, 52, 41), 12
    coefs, sources, mons = case(shape, T, "spheres")
    kw = dict(kernel="tiled", storage=storage, blt=2)
    Ff, Df, active, _ = run(shape, coefs, T, sources, mons, True, **kw)
    Fg, Dg, _, _ = run(shape, coefs, T, sources, mons, False, **kw)
    assert active
    for c in range(6):
        assert np.array_equal(Ff[c].view(np.uint32), Fg[c].view(np.uint32)), c
    for (re, im), (rg, ig) in zip(Df, Dg):
        assert np.array_equal(re, rg) and np.array_equal(im, ig)


def test_fast_path_off_for_lossy_dominant_material():
    """A dominant material with Ca != 1 (a lossy medium) does not qualify."""
    shape = (40, 30, 20)
    coefs = [c.copy() for c in W.vacuum_coefficients(shape)]
    coefs[0][:] = np.float32(0.99)  # Cax
    sim = gd.Simulation(*shape)
    sim.set_coefficients(coefs)
    assert not sim.fast_path
    sim.close()


def test_fast_path_in_batches():
    """A batch of vacuum and sphere grids: fast == general == oracle."""
    T = 10
    shapes = [(66, 40, 30), (48, 56, 36), (40, 40, 40)]
    results = {}
    refs = []
    for n, shape in enumerate(shapes):
        coefs, sources, _ = case(shape, T, "vacuum" if n % 2 else "spheres")
        refs.append((shape, coefs, sources,
                     oracle.run(shape, coefs, T, sources=[osrc(s) for s in sources])))
    for fast in (True, False):
        sims = []
        for shape, coefs, sources, _ in refs:
            s = gd.Simulation(*shape)
            s.set_coefficients(coefs)
            s.set_fast_path(fast)
            s.set_sources(sources)
            sims.append(s)
        b = gd.Batch(sims)
        b.step(T)
        for s in sims:
            s.sync()
        results[fast] = [s.fields() for s in sims]
        b.close()
        for s in sims:
            s.close()
    for n, (_, _, _, F_ref) in enumerate(refs):
        assert_fields_match(results[True][n], F_ref, f"batch fast {n}")
        assert_fields_match(results[False][n], F_ref, f"batch general {n}")
