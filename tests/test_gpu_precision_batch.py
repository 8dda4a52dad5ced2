"""Reduced-precision storage, FP64 storage and batches, on the GPU, against the oracle.

* FP16 / BF16 / F16E storage: the tiled kernel computes each BLT-step pass in exact FP32 from
  the stored (rounded) fields and rounds once when it writes the pass's result.  The oracle
  reproduces that bit for bit: run BLT steps in FP32, then round every field to its storage
  type (value * inv_scale rounded to nearest-even, read back times scale; F16E rounds E to
  FP16 and leaves H in FP32).  Monitors sum the unrounded FP32 values in both.
* FP64 storage: the naive kernel in double against the oracle's FP64 stepper, bit for bit.
* Batches: uneven grids with their own materials, sources and monitors advanced together by
  the persistent kernel (with and without CUDA-graph replay) against the oracle.
"""
import numpy as np
import pytest

import oracle
import gdiamond_b200 as gd
from gdiamond_b200 import workloads as W

pytestmark = pytest.mark.gpu


def bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32),
                          np.asarray(b, np.float32).view(np.uint32))


def round_bf16(x):
    b = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32)


def storage_roundtrip(F, storage, scales):
    out = []
    for c, f in enumerate(F):
        if storage == "f16e" and c >= 3:  # H in FP32: no rounding, no scale
            out.append(np.asarray(f, np.float32).copy())
            continue
        sc = np.float32(scales[c])
        inv = np.float32(1.0) / sc
        v = (np.asarray(f, np.float32) * inv).astype(np.float32)
        if storage in ("f16", "f16e"):
            r = v.astype(np.float16).astype(np.float32)
        else:
            r = round_bf16(v)
        out.append((r * sc).astype(np.float32))
    return out


def oracle_stored(shape, coefs, T, blt, storage, scales, sources, monitors):
    """The oracle with the storage rounding of the tiled kernel's BLT-step passes."""
    F, t = None, 0
    while t < T:
        b = min(blt, T - t)
        F = oracle.run(shape, coefs, b, sources=sources, monitors=monitors, fields=F, t0=t)
        F = storage_roundtrip(F, storage, scales)
        t += b
    return F


def setup(shape, T, seed):
    eps = W.spheres_eps(shape, n_spheres=5, r_range=(3, 7), seed=seed)
    coefs = W.reference_coefficients(shape, eps_re=eps)
    nx, ny, nz = shape
    w = W.gaussian_wave(T, delay=6.0, width=2.5, period=5.0)
    src = [dict(component="Jz", wave=w, i=nx // 2, j=ny // 2, k=nz // 2),
           dict(component="Mx", wave=w * np.float32(0.25), i=nx // 3, j=ny // 3, k=nz // 3)]
    freqs = W.source_band(3, period=5.0, width=2.5)
    mons = [dict(component="Ez", k=nz // 2 + 2, freqs=freqs, scale=1.0)]
    return coefs, src, mons


def osrc(s):
    return oracle.Source(s["component"], s["wave"], i=s.get("i", 0), j=s.get("j", 0), k=s["k"],
                         kind=s.get("kind", 0))


@pytest.mark.parametrize("storage", ["f16", "bf16", "f16e"])
@pytest.mark.parametrize("blt,rows", [(2, 16), (3, 8), (4, 16)])
def test_16bit_storage_matches_rounded_oracle(storage, blt, rows):
    shape, T = (70, 41, 33), 14
    coefs, src, mons = setup(shape, T, 3)
    scales = [8.0, 8.0, 8.0, 2.0, 2.0, 0.5]
    omons = [oracle.Monitor(m["component"], m["k"], m["freqs"], m["scale"]) for m in mons]
    F_ref = oracle_stored(shape, coefs, T, blt, storage, scales, [osrc(s) for s in src], omons)
    sim = gd.Simulation(*shape, storage=storage, kernel="tiled", blt=blt, tile_rows=rows)
    sim.set_storage_scale(scales)
    sim.set_coefficients(coefs)
    sim.set_sources(src)
    mid = sim.add_dft_monitor(mons[0]["component"], mons[0]["k"], mons[0]["freqs"])
    sim.step(T)
    sim.sync()
    F = sim.fields()
    re, im = sim.get_dft(mid)
    cfg = sim.config()
    sim.close()
    assert (cfg["width"], cfg["blt"], cfg["tile_rows"]) == (64, blt, rows)
    for c in range(6):
        assert bits_equal(F[c], F_ref[c]), oracle.COMPONENTS[c]
    assert np.abs(omons[0].re).max() > 0
    assert np.array_equal(re, omons[0].re) and np.array_equal(im, omons[0].im)


@pytest.mark.parametrize("storage", ["f16", "bf16", "f16e"])
@pytest.mark.parametrize("blt,rows", [(1, 24), (1, 48), (2, 24), (2, 32), (2, 48), (3, 32)])
def test_16bit_pairs32_matches_rounded_oracle(storage, blt, rows):
    """The x-pair kernel with 32-cell rows (two per warp) and 16-bit storage."""
    shape, T = (70, 41, 33), 14
    coefs, src, mons = setup(shape, T, 5)
    scales = [8.0, 8.0, 8.0, 2.0, 2.0, 0.5]
    omons = [oracle.Monitor(m["component"], m["k"], m["freqs"], m["scale"]) for m in mons]
    F_ref = oracle_stored(shape, coefs, T, blt, storage, scales, [osrc(s) for s in src], omons)
    sim = gd.Simulation(*shape, storage=storage, kernel="tiled_w32p", blt=blt, tile_rows=rows)
    sim.set_storage_scale(scales)
    sim.set_coefficients(coefs)
    sim.set_sources(src)
    mid = sim.add_dft_monitor(mons[0]["component"], mons[0]["k"], mons[0]["freqs"])
    sim.step(T)
    sim.sync()
    F = sim.fields()
    re, im = sim.get_dft(mid)
    cfg = sim.config()
    sim.close()
    assert (cfg["width"], cfg["pairs"], cfg["blt"], cfg["tile_rows"]) == (32, True, blt, rows)
    for c in range(6):
        assert bits_equal(F[c], F_ref[c]), oracle.COMPONENTS[c]
    assert np.array_equal(re, omons[0].re) and np.array_equal(im, omons[0].im)


def test_16bit_rejects_naive_and_accepts_power_of_two_scales():
    for storage in ("f16", "f16e"):
        with pytest.raises(gd.FdtdError):
            gd.Simulation(20, 20, 20, storage=storage, kernel="naive")
        with pytest.raises(gd.FdtdError):
            gd.Simulation(20, 20, 20, storage=storage, kernel="tiled_w32")
    sim = gd.Simulation(40, 30, 20, storage="bf16")
    with pytest.raises(gd.FdtdError):
        sim.set_storage_scale([1, 1, 1, 1, 0, 1])
    sim.set_storage_scale([3.0, 1, 1, 1, 1, 1])  # rounded to 4
    x = np.linspace(-3, 3, 40 * 30 * 20).astype(np.float32)
    sim.set_field("Ex", x)
    got = sim.get_field("Ex")
    assert np.array_equal(got, storage_roundtrip([x] * 6, "bf16", [4.0] * 6)[0])
    sim.close()


def test_f16e_stores_e_in_fp16_and_h_in_fp32():
    shape = (40, 30, 20)
    sim = gd.Simulation(*shape, storage="f16e")
    assert sim.storage_bytes() == 2
    assert [sim.component_bytes(c) for c in range(6)] == [2, 2, 2, 4, 4, 4]
    sim.set_storage_scale([4.0] * 6)  # used by the FP16 (E) components only
    x = np.linspace(-3, 3, 40 * 30 * 20).astype(np.float32)
    for comp in gd.COMPONENTS:
        sim.set_field(comp, x)
    want = storage_roundtrip([x] * 6, "f16e", [4.0] * 6)
    assert not np.array_equal(want[0], x)
    for c, comp in enumerate(gd.COMPONENTS):
        assert bits_equal(sim.get_field(comp), want[c]), comp
    assert np.array_equal(sim.get_field_f64(5), x.astype(np.float64))
    sim.close()


def test_fp64_storage_matches_fp64_oracle():
    shape, T = (37, 29, 23), 21
    coefs, src, mons = setup(shape, T, 4)
    omons = [oracle.Monitor(m["component"], m["k"], m["freqs"], m["scale"]) for m in mons]
    F_ref = oracle.run(shape, coefs, T, sources=[osrc(s) for s in src], monitors=omons,
                       precision="f64")
    sim = gd.Simulation(*shape, storage="f64")
    sim.set_coefficients(coefs)
    sim.set_sources(src)
    mid = sim.add_dft_monitor(mons[0]["component"], mons[0]["k"], mons[0]["freqs"])
    sim.step(T)
    sim.sync()
    for c in range(6):
        assert np.array_equal(sim.get_field_f64(c), F_ref[c]), oracle.COMPONENTS[c]
    re, im = sim.get_dft(mid)
    assert np.array_equal(re, omons[0].re) and np.array_equal(im, omons[0].im)
    assert sim.config()["kernel"] == "naive"
    sim.close()


SHAPES = [(64, 40, 36), (96, 64, 48), (72, 56, 40)]


def make_batch(storage, T, scales=None):
    sims, refs = [], []
    for n, shape in enumerate(SHAPES):
        coefs, src, mons = setup(shape, T, 10 + n)
        sim = gd.Simulation(*shape, storage=storage)
        if scales:
            sim.set_storage_scale(scales)
        sim.set_coefficients(coefs)
        sim.set_sources(src)
        sim.add_dft_monitor(mons[0]["component"], mons[0]["k"], mons[0]["freqs"])
        sims.append(sim)
        refs.append((shape, coefs, src, mons))
    return sims, refs


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_fp32_matches_oracle_and_replays(use_graph):
    T = 17
    sims, refs = make_batch("f32", T)
    batch = gd.Batch(sims)
    batch.step(T, use_graph=use_graph)
    cfg = batch.config()
    assert cfg["items"] > 0 and cfg["launches"] == -(-T // cfg["blt"])
    first = []
    for sim, (shape, coefs, src, mons) in zip(sims, refs):
        omons = [oracle.Monitor(m["component"], m["k"], m["freqs"], m["scale"]) for m in mons]
        F_ref = oracle.run(shape, coefs, T, sources=[osrc(s) for s in src], monitors=omons)
        sim.sync()
        F = sim.fields()
        for c in range(6):
            assert bits_equal(F[c], F_ref[c]), (shape, oracle.COMPONENTS[c])
        re, im = sim.get_dft(0)
        assert np.array_equal(re, omons[0].re) and np.array_equal(im, omons[0].im)
        assert sim.t == T
        first.append(F)
    # reset and run again: the same graph is replayed and gives the same fields
    for sim in sims:
        sim.reset()
    batch.step(T, use_graph=use_graph)
    assert batch.config()["graph_replayed"] == use_graph
    for sim, F in zip(sims, first):
        for c, f in enumerate(sim.fields()):
            assert bits_equal(f, F[c])
    batch.close()
    for sim in sims:
        sim.close()


@pytest.mark.parametrize("storage", ["bf16", "f16e"])
def test_batch_16bit_matches_rounded_oracle(storage):
    T = 15
    scales = [8.0, 8.0, 8.0, 2.0, 2.0, 0.5]
    sims, refs = make_batch(storage, T, scales)
    batch = gd.Batch(sims)
    batch.step(T)
    blt = batch.config()["blt"]
    for sim, (shape, coefs, src, mons) in zip(sims, refs):
        omons = [oracle.Monitor(m["component"], m["k"], m["freqs"], m["scale"]) for m in mons]
        F_ref = oracle_stored(shape, coefs, T, blt, storage, scales, [osrc(s) for s in src],
                              omons)
        sim.sync()
        for c, f in enumerate(sim.fields()):
            assert bits_equal(f, F_ref[c]), (shape, oracle.COMPONENTS[c])
        re, im = sim.get_dft(0)
        assert np.array_equal(re, omons[0].re) and np.array_equal(im, omons[0].im)
    batch.close()
    for sim in sims:
        sim.close()


def test_batch_dft_folds_across_ring_wraps():
    """A batch of 260 steps folds the staged monitor values three times inside its captured
    launch sequence (two full 128-step windows and a partial one); a replay of the graph after a
    reset folds again from zero.  Sums equal the oracle's bit for bit."""
    T = 260
    sims, refs = make_batch("f32", T)
    batch = gd.Batch(sims)
    want = []
    for shape, coefs, src, mons in refs:
        omons = [oracle.Monitor(m["component"], m["k"], m["freqs"], m["scale"]) for m in mons]
        oracle.run(shape, coefs, T, sources=[osrc(s) for s in src], monitors=omons)
        assert np.abs(omons[0].re).max() > 0
        want.append((omons[0].re, omons[0].im))
    for rep in range(2):
        for sim in sims:
            sim.reset()
        batch.step(T, use_graph=True)
        cfg = batch.config()
        assert cfg["dft_folds"] == 3 and cfg["graph_replayed"] == (rep == 1)
        for sim, (re_w, im_w) in zip(sims, want):
            sim.sync()
            re, im = sim.get_dft(0)
            assert np.array_equal(re, re_w) and np.array_equal(im, im_w), (rep, sim.shape)
    batch.close()
    for sim in sims:
        sim.close()


def test_batch_rejects_mixed_storage():
    a = gd.Simulation(40, 30, 20)
    b = gd.Simulation(40, 30, 20, storage="bf16")
    for s in (a, b):
        s.set_coefficients(W.vacuum_coefficients((40, 30, 20)))
    with pytest.raises(gd.FdtdError):
        gd.Batch([a, b])
    c = gd.Simulation(40, 30, 20)  # no coefficients
    with pytest.raises(gd.FdtdError):
        gd.Batch([a, c])
    for s in (a, b, c):
        s.close()


def test_batch_back_to_back_steps_without_sync():
    """Two batch steps issued without a synchronisation between them (graph and plain): the
    second must not change the arguments the first one is still to read."""
    T = 6
    for use_graph in (True, False):
        sims, refs = make_batch("f32", 2 * T)
        batch = gd.Batch(sims)
        batch.step(T, use_graph=use_graph)
        batch.step(T, use_graph=use_graph)
        for sim, (shape, coefs, src, mons) in zip(sims, refs):
            F_ref = oracle.run(shape, coefs, 2 * T, sources=[osrc(s) for s in src])
            sim.sync()
            for c, f in enumerate(sim.fields()):
                assert bits_equal(f, F_ref[c]), (use_graph, shape, oracle.COMPONENTS[c])
        batch.close()
        for sim in sims:
            sim.close()


@pytest.mark.parametrize("storage", ["f16", "f16e"])
def test_16bit_overflow_is_reported_not_silent(storage):
    """A storage scale far too small for the field makes stored FP16 values overflow (above
    65504): fdtd_sync reports FDTD_ERR_NUMERIC instead of returning infinities silently.  After
    a reset with a sound scale the handle steps correctly.  (BF16 has FP32's exponent range, so
    it overflows only where FP32 would; the same check covers it.)"""
    shape, T = (40, 32, 24), 30
    coefs = W.reference_coefficients(shape)
    w = W.gaussian_wave(T, delay=8.0, width=3.0, period=6.0)
    src = [dict(component="Jz", wave=w, i=20, j=16, k=12)]
    sim = gd.Simulation(*shape, storage=storage, blt=2)
    sim.set_coefficients(coefs)
    sim.set_sources(src)
    sim.set_storage_scale([2.0 ** -20] * 6)
    sim.step(T)
    with pytest.raises(gd.FdtdError) as e:
        sim.sync()
    assert e.value.status == 6  # FDTD_ERR_NUMERIC
    sim.sync()  # the error word was cleared with the report
    # a sound scale: bit-exact against the oracle again
    scales = [2.0, 2.0, 2.0, 0.5, 0.5, 0.5]
    sim.set_storage_scale(scales)
    sim.reset()
    sim.step(T)
    sim.sync()
    F_ref = oracle_stored(shape, coefs, T, 2, storage, scales,
                          [oracle.Source("Jz", w, i=20, j=16, k=12)], [])
    for c, f in enumerate(sim.fields()):
        assert bits_equal(f, F_ref[c]), (storage, c)
    sim.close()
