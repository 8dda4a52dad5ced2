"""GPU: CPML absorbing layers (fdtd_set_cpml) against the numpy CPML oracle, and their absorption.

* The library's profile tables equal the formula restated in oracle/cpml.py (FP64 then FP32).
* Fields after stepping with layers on all faces, or on the z faces only, equal the oracle's
  bit for bit (point and plane sources, material map and per-cell coefficients).
* Absorption: a dipole pulse in a 64^3 box is compared at a probe near the boundary with the
  same run in a 160^3 box whose faces are too far to reflect within the window.  The CPML
  reflection error must be at least 20 dB below that of the reference's graded pseudo-PML
  (gDiamond/utils.h:585-660) of the same thickness.
"""
import numpy as np
import pytest

import oracle
from oracle import cpml
import gdiamond_b200 as gd
from gdiamond_b200 import workloads as W
from test_gpu_parity import assert_fields_match, osrc

pytestmark = pytest.mark.gpu

DX, DT = float(np.float32(0.1)), float(np.float32(0.05))


def make(shape, coefs, src, L, faces=63, kappa_max=1.5, kernel="auto", blt=0):
    sim = gd.Simulation(*shape, kernel=kernel, blt=blt)
    sim.set_coefficients(coefs)
    sim.set_cpml(thickness=L, faces=faces, kappa_max=kappa_max)
    if src:
        sim.set_sources(src)
    return sim


def test_profile_tables_match_formula():
    shape, L = (40, 36, 44), 6
    sim = make(shape, W.vacuum_coefficients(shape), [], L, faces=1 | 2 | 16 | 32)
    tabs = sim.cpml_tables()
    for axis, n in enumerate(shape):
        on = axis != 1
        for kind in (0, 1):
            want = cpml.profile(n, L, on, on, DX, DT, kappa_max=1.5, half=kind == 1)
            got = tabs[axis][kind]
            assert np.array_equal(got[0], want[0]), (axis, kind)
            for q in (1, 2, 3):
                np.testing.assert_allclose(got[q], want[q], rtol=2e-7, atol=1e-30)
    sim.close()


@pytest.mark.parametrize("faces,percell,kernel", [(63, False, "auto"), (16 | 32, False, "auto"),
                                                  (16 | 32, False, "naive"), (63, True, "auto")])
def test_cpml_fields_match_oracle(faces, percell, kernel):
    """Layers on every face (too little interior for the shell companion: per-step kernels),
    on the z faces only (the tiled kernel with the shell companion, or per-step kernels when the
    naive kernel is asked for), and with per-cell coefficients (per-step kernels)."""
    shape, T, L = ((48, 40, 44) if percell else (40, 36, 44)), 60, 6
    nx, ny, nz = shape
    eps = W.spheres_eps(shape, n_spheres=3, r_range=(3, 5), eps_range=(2.0, 4.0), seed=9)
    coefs = W.reference_coefficients(shape, eps_re=eps, t_pml=0)
    if percell:  # more distinct tuples (84480) than the material map holds: per-cell arrays
        rng = np.random.default_rng(1)
        coefs = [c.copy() for c in coefs]
        coefs[0] = (coefs[0] * rng.uniform(0.5, 1.0, coefs[0].size)).astype(np.float32)
    w = W.gaussian_wave(T, delay=15.0, width=5.0, period=8.0)
    src = [dict(component="Jz", wave=w, i=nx // 2, j=ny // 2, k=nz // 2),
           dict(component="Jx", wave=w * np.float32(0.2), k=nz - 9, kind=gd.SRC_PLANE_Z)]
    companion = faces == 16 | 32 and kernel == "auto"
    # BLT 2: the interior left beyond 3 BLT cells from the z layers is still most of this grid
    sim = make(shape, coefs, src, L, faces=faces, kernel=kernel, blt=2 if companion else 0)
    assert (sim.material_count() == 0) == percell
    sim.step(T)
    sim.sync()
    assert sim.config()["kernel"] == ("tiled" if companion else "cpml")
    F = sim.fields()
    F_ref = cpml.run(shape, coefs, T, sim.cpml_tables(), sources=[osrc(s) for s in src], dx=DX)
    assert_fields_match(F, F_ref, f"cpml faces={faces} percell={percell}")
    # reset clears the auxiliary fields too: a second run repeats the first bit for bit
    sim.reset()
    sim.step(T)
    assert_fields_match(sim.fields(), F_ref, "cpml after reset")
    sim.close()


def probe_series(shape, coefs, src_pos, probe, T, cpml_L=None):
    import torch
    nx, ny, nz = shape
    sim = gd.Simulation(*shape)
    sim.set_coefficients(coefs)
    if cpml_L:
        sim.set_cpml(thickness=cpml_L)
    w = W.gaussian_wave(T)
    sim.set_sources([dict(component="Jz", wave=w, i=src_pos[0], j=src_pos[1], k=src_pos[2])])
    buf = torch.empty(nx * ny * nz, dtype=torch.float32, device="cuda")
    out = np.empty(T)
    p = probe[0] + nx * (probe[1] + ny * probe[2])
    for t in range(T):
        sim.step(1)
        sim.get_field_device("Ez", buf.data_ptr())
        torch.cuda.synchronize()
        out[t] = float(buf[p])
    sim.close()
    return out


def test_cpml_absorbs_20db_better_than_graded_pseudo_pml():
    T, L = 200, 10
    small, big = (64, 64, 64), (160, 160, 160)
    # the 64^3 box: source at the centre, probe 16 cells away broadside, 5 cells from the layer
    ref = probe_series(big, W.vacuum_coefficients(big), (80, 80, 80), (96, 80, 80), T)
    pml = probe_series(small, W.reference_coefficients(small, t_pml=L), (32, 32, 32),
                       (48, 32, 32), T)
    cp = probe_series(small, W.vacuum_coefficients(small), (32, 32, 32), (48, 32, 32), T,
                      cpml_L=L)
    scale = np.abs(ref).max()
    assert scale > 0
    err_pml = np.abs(pml - ref).max() / scale
    err_cpml = np.abs(cp - ref).max() / scale
    print(f"reflection error: graded pseudo-PML {err_pml:.3e}, CPML {err_cpml:.3e} "
          f"({20 * np.log10(err_pml / err_cpml):.1f} dB)")
    assert err_cpml * 10 <= err_pml  # >= 20 dB less reflection


def _cpml_sim(shape, seed, L=6, flux_k=None, freqs=None):
    nx, ny, nz = shape
    eps = W.spheres_eps(shape, n_spheres=2, r_range=(3, 5), eps_range=(2.0, 5.0), seed=seed)
    sim = gd.Simulation(*shape)
    sim.set_coefficients(W.reference_coefficients(shape, eps_re=eps, t_pml=0))
    sim.set_cpml(thickness=L)
    T = 400
    w = W.gaussian_wave(T, delay=20.0 + seed, width=6.0, period=9.0)
    sim.set_sources([dict(component="Jx", wave=w, k=L + 2, kind=gd.SRC_PLANE_Z),
                     dict(component="Jz", wave=w * np.float32(0.3), i=nx // 2 - seed,
                          j=ny // 2, k=nz // 2)])
    mons = []
    if freqs is not None:
        mons.append(("flux", sim.add_flux_monitor(flux_k, freqs)))
        mons.append(("dft", sim.add_dft_monitor("Ez", nz // 2 + 1, freqs)))
    return sim, mons


def _read(sim, mons):
    out = []
    for kind, mid in mons:
        if kind == "flux":
            out.append(sim.get_flux(mid))
            for q in sim.flux_monitor_ids(mid):
                out.extend(sim.get_dft(q))
        else:
            out.extend(sim.get_dft(mid))
    return out


@pytest.mark.parametrize("use_graph", [True, False])
def test_cpml_batch_matches_single_grids(use_graph):
    """Batched CPML grids (one E and one H launch per step over all grids, staged monitors,
    deferred folds) equal the same grids stepped alone (per-step monitor accumulation) bit for
    bit: fields, DFT sums and fluxes, over two step calls that cross the staging ring's wrap."""
    shapes = [(40, 36, 44), (40, 36, 44), (48, 40, 36)]
    freqs = W.source_band(5, period=9.0, width=6.0)
    T1, T2 = 150, 110
    batch_sims, batch_mons, ref = [], [], []
    for n, shape in enumerate(shapes):
        s, m = _cpml_sim(shape, n, flux_k=shape[2] - 10, freqs=freqs)
        batch_sims.append(s)
        batch_mons.append(m)
        r, rm = _cpml_sim(shape, n, flux_k=shape[2] - 10, freqs=freqs)
        r.step(T1)
        r.step(T2)
        r.sync()
        ref.append((r.fields(), _read(r, rm)))
        r.close()
    b = gd.Batch(batch_sims)
    b.step(T1, use_graph=use_graph)
    b.step(T2, use_graph=use_graph)
    for s, m, (F_ref, R_ref) in zip(batch_sims, batch_mons, ref):
        s.sync()
        assert s.config()["kernel"] == "cpml"
        assert_fields_match(s.fields(), F_ref, "cpml batch")
        for got, want in zip(_read(s, m), R_ref):
            assert np.array_equal(got, want)
    # graph replay after a reset repeats the first call
    if use_graph:
        for s in batch_sims:
            s.reset()
        b.step(T1, use_graph=True)
        b.step(T2, use_graph=True)
        for s, m, (F_ref, R_ref) in zip(batch_sims, batch_mons, ref):
            s.sync()
            assert_fields_match(s.fields(), F_ref, "cpml batch replay")
    b.close()
    for s in batch_sims:
        s.close()


def test_cpml_batch_fields_match_oracle():
    shape, T, L = (40, 36, 44), 60, 6
    sims = [_cpml_sim(shape, n, L=L)[0] for n in range(2)]
    b = gd.Batch(sims)
    b.step(T)
    for n, s in enumerate(sims):
        s.sync()
        eps = W.spheres_eps(shape, n_spheres=2, r_range=(3, 5), eps_range=(2.0, 5.0), seed=n)
        coefs = W.reference_coefficients(shape, eps_re=eps, t_pml=0)
        w = W.gaussian_wave(400, delay=20.0 + n, width=6.0, period=9.0)
        src = [dict(component="Jx", wave=w, k=L + 2, kind=gd.SRC_PLANE_Z),
               dict(component="Jz", wave=w * np.float32(0.3), i=shape[0] // 2 - n,
                    j=shape[1] // 2, k=shape[2] // 2)]
        F_ref = cpml.run(shape, coefs, T, s.cpml_tables(), sources=[osrc(x) for x in src],
                         dx=DX)
        assert_fields_match(s.fields(), F_ref, f"cpml batch grid {n}")
    b.close()
    for s in sims:
        s.close()


def test_cpml_batch_rejects_mixed_boundaries():
    shape = (40, 36, 44)
    a, _ = _cpml_sim(shape, 0)
    c = gd.Simulation(*shape)
    c.set_coefficients(W.vacuum_coefficients(shape))
    with pytest.raises(gd.FdtdError):
        gd.Batch([a, c])
    a.close()
    c.close()


def _companion_pair(shape, L, blt, kernel):
    """A CPML grid with sources inside a layer, near the shell and in the interior, a flux
    monitor and an Ez DFT monitor on a plane that crosses the side layers."""
    nx, ny, nz = shape
    eps = W.spheres_eps(shape, n_spheres=4, r_range=(4, 8), eps_range=(2.0, 6.0), seed=4)
    sim = gd.Simulation(*shape, kernel=kernel, blt=blt if kernel != "naive" else 0)
    sim.set_coefficients(W.reference_coefficients(shape, eps_re=eps, t_pml=0))
    sim.set_cpml(thickness=L, kappa_max=1.5)
    T = 200
    w = W.gaussian_wave(T, delay=12.0, width=4.0, period=6.0)
    sim.set_sources([dict(component="Jx", wave=w, k=L + 3, kind=gd.SRC_PLANE_Z),
                     dict(component="Jz", wave=w * np.float32(0.5), i=nx // 2, j=ny // 3,
                          k=nz // 2),
                     dict(component="Jy", wave=w * np.float32(0.7), i=2, j=ny // 2, k=nz // 3),
                     dict(component="My", wave=w * np.float32(0.2), i=nx - 5, j=ny // 2,
                          k=nz // 2)])
    freqs = W.source_band(4, period=6.0, width=4.0)
    mons = [("flux", sim.add_flux_monitor(nz - L - 4, freqs)),
            ("dft", sim.add_dft_monitor("Ez", nz // 2, freqs)),
            ("dft", sim.add_dft_monitor("Hx", 3, freqs))]
    return sim, mons


@pytest.mark.parametrize("blt", [1, 2, 3])
def test_cpml_shell_companion_matches_per_step_path(blt):
    """With CPML layers on a grid large enough, the tiled kernel advances the whole grid and
    the shell companion recomputes the cells the layers reach; fields, psi (through continued
    stepping), DFT sums and fluxes equal the per-step CPML path's bit for bit, over step calls
    that are not multiples of BLT."""
    shape, L = (128, 112, 120), 6
    ref, rm = _companion_pair(shape, L, blt, "naive")
    sim, sm = _companion_pair(shape, L, blt, "auto")
    for T in (2 * blt + 1, 23, 40):
        ref.step(T)
        sim.step(T)
        ref.sync()
        sim.sync()
        assert ref.config()["kernel"] == "cpml"
        assert sim.config()["kernel"] == "tiled" and sim.config()["blt"] == blt
        assert_fields_match(sim.fields(), ref.fields(), f"companion blt={blt} T={T}")
        for got, want in zip(_read(sim, sm), _read(ref, rm)):
            assert np.array_equal(got, want)
    ref.close()
    sim.close()


@pytest.mark.parametrize("kernel", ["naive", "auto"])
def test_cpml_checkpoint_resume_continues_bit_for_bit(kernel):
    """checkpoint() carries the layers' psi arrays: a run resumed from it on a fresh handle
    equals the uninterrupted run bit for bit (per-step path and tiled kernel + companion)."""
    shape, L = ((128, 112, 120) if kernel == "auto" else (40, 36, 44)), 6
    a, am = _companion_pair(shape, L, 2, kernel)
    a.step(30)
    ck = a.checkpoint()
    assert ck["cpml_psi"] is not None and len(ck["cpml_psi"]) == 12
    assert any(np.abs(p).max() > 0 for p in ck["cpml_psi"])
    a.step(25)
    a.sync()
    b, bm = _companion_pair(shape, L, 2, kernel)
    b.restore(ck)
    b.step(25)
    b.sync()
    assert_fields_match(b.fields(), a.fields(), f"resume {kernel}")
    for got, want in zip(_read(b, bm), _read(a, am)):
        assert np.array_equal(got, want)
    # a handle without layers refuses the checkpoint
    c, _ = _companion_pair(shape, L, 2, kernel)
    c.set_cpml(thickness=None)
    with pytest.raises(ValueError):
        c.restore(ck)
    for s in (a, b, c):
        s.close()
