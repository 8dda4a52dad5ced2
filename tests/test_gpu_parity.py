"""GPU parity: the CUDA kernels, called through the C-ABI, against the oracle (needs a GPU).

The bar is bit-exactness: every multiply and add in the kernels is separately rounded, as in
the reference's CPU build, so fields and FP64 monitor sums must equal the oracle's bit for bit.
The FP32 tolerance of the workload (relative L2 <= 1e-5 per component) is asserted as well, so a
failure reports both.  Cases:
  * the reference unit test (unittests/checker_gpu.cu): 100^3, 100 steps, the reference
    constructor's coefficients and its Mz source -> the golden SHA-256 of update_FDTD_seq;
  * the vacuum 100^3 Gaussian-Jz workload, 100 steps;
  * every tiled (BLT, rows, z-chunks) instance on an odd grid with PML coefficients and J/M
    point sources; plane sources with random permittivity; FP64 DFT monitors;
  * per-cell coefficients that do not compress (naive fallback; tiled refused);
  * at the full 256^3 x 1000 benchmark size: the tiled kernel against the oracle bit for bit
    (fields and the 8-frequency FP64 DFT), tiled == naive bit for bit, and linearity (doubling
    the source doubles every field to FP32 rounding);
  * state handling: split step calls, reset, set_field.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
import gdiamond_b200 as gd
from gdiamond_b200 import workloads as W

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REL_L2_TOL = 1e-5  # FP32 tolerance (relative L2 per component)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


def assert_fields_match(F, F_ref, label=""):
    for c in range(6):
        assert rel_l2(F[c], F_ref[c]) <= REL_L2_TOL, f"{label} {oracle.COMPONENTS[c]} rel-L2"
        assert np.array_equal(np.asarray(F[c], np.float32).view(np.uint32),
                              np.asarray(F_ref[c], np.float32).view(np.uint32)), \
            f"{label} {oracle.COMPONENTS[c]} not bit-identical"


def gpu_run(shape, coefs, T, sources=(), monitors=(), kernel="auto", **kw):
    sim = gd.Simulation(*shape, kernel=kernel, **kw)
    sim.set_coefficients(coefs)
    if sources:
        sim.set_sources(sources)
    mids = [sim.add_dft_monitor(m["component"], m["k"], m["freqs"], m.get("scale", 1.0))
            for m in monitors]
    sim.step(T)
    sim.sync()
    F = sim.fields()
    D = [sim.get_dft(m) for m in mids]
    cfg = sim.config()
    sim.close()
    return F, D, cfg


def osrc(s):
    return oracle.Source(s["component"], s["wave"], i=s.get("i", 0), j=s.get("j", 0), k=s["k"],
                         kind=s.get("kind", 0))


@pytest.mark.parametrize("kernel", ["naive", "tiled"])
def test_reference_unit_test_100cube(kernel):
    """unittests/checker_gpu.cu: seq vs GPU at 100^3 x 100 -- here against the golden seq."""
    g = json.load(open(os.path.join(GOLDEN, "ref_100cube_T100.json")))
    shape, T = tuple(g["shape"]), g["T"]
    nx, ny, nz = shape
    src = g["source_idx"]
    coefs = W.reference_coefficients(shape)
    sources = [dict(component="Mz", wave=W.reference_mz_wave(T), i=src % nx,
                    j=(src // nx) % ny, k=src // (nx * ny))]
    F, _, cfg = gpu_run(shape, coefs, T, sources, kernel=kernel)
    assert cfg["kernel"] == kernel
    for c, n in enumerate(oracle.COMPONENTS):
        assert np.linalg.norm(F[c].astype(np.float64)) == pytest.approx(g["seq"][n]["l2"], rel=1e-5)
        assert sha(F[c]) == g["seq"][n]["sha256"], n


def test_vacuum_gaussian_jz_100cube():
    shape, T = (100, 100, 100), 100
    coefs = W.vacuum_coefficients(shape)
    sources = [dict(component="Jz", wave=W.gaussian_wave(T), i=50, j=50, k=50)]
    F_ref = oracle.run(shape, coefs, T, sources=[osrc(s) for s in sources])
    for kernel in ("naive", "tiled"):
        F, _, _ = gpu_run(shape, coefs, T, sources, kernel=kernel)
        assert_fields_match(F, F_ref, kernel)


CONFIGS = [(b, r, z, "tiled_w32") for r, bs in ((8, (1, 2, 3)), (16, (1, 2, 3, 4, 5, 6)),
                                                (32, (1, 2, 3, 4, 5, 6)))
           for b in bs for z in (1, 3)]
CONFIGS += [(b, r, z, "tiled_w64") for r, bs in ((8, (1, 2, 3)), (16, (1, 2, 3, 4)),
                                                (20, (1, 2, 3)), (24, (1, 2)), (32, (1, 2)))
            for b in bs for z in (1, 3)]
# x-pairs in 32-wide rows, two rows per warp (FP32)
CONFIGS += [(b, r, z, "tiled_w32p") for r, bs in ((24, (1, 2)), (32, (1, 2, 3)), (48, (1, 2)))
            for b in bs for z in (1, 3)]
# register-capped x-pair variants (2 CTAs of 16 rows / 4 CTAs of 8 rows per SM)
CONFIGS += [(2, 16, 1, "tiled_w64:2"), (2, 16, 3, "tiled_w64:2"), (2, 8, 1, "tiled_w64:4"),
            (2, 8, 3, "tiled_w64:4")]


@pytest.mark.parametrize("blt,rows,zc,family", CONFIGS)
def test_tiled_instances_pml_point_sources(blt, rows, zc, family):
    family, _, mb = family.partition(":")
    mb = int(mb or 0)
    shape, T = (75 if family == "tiled_w64" else 45, 37, 29), 13
    coefs = W.reference_coefficients(shape)
    w = W.gaussian_wave(T, delay=4.0, width=2.0, period=5.0)
    sources = [dict(component="Jz", wave=w, i=22, j=18, k=14),
               dict(component="Mx", wave=w * np.float32(0.5), i=3, j=30, k=20),
               dict(component="Jy", wave=w, i=1, j=1, k=1)]
    F_ref = oracle.run(shape, coefs, T, sources=[osrc(s) for s in sources])
    F, _, cfg = gpu_run(shape, coefs, T, sources, kernel=family, blt=blt, tile_rows=rows,
                        z_chunks=zc, min_blocks=mb)
    assert (cfg["blt"], cfg["tile_rows"], cfg["z_chunks"]) == (blt, rows, zc)
    assert cfg["min_blocks"] == (mb or 1)
    assert cfg["width"] == (64 if family == "tiled_w64" else 32)
    assert_fields_match(F, F_ref, f"{family} blt={blt} rows={rows} zc={zc}")


@pytest.mark.parametrize("kernel", ["naive", "tiled_w32", "tiled_w64"])
def test_plane_source_random_eps_and_monitors(kernel):
    shape, T = (64, 48, 40), 60
    nx, ny, nz = shape
    rng = np.random.default_rng(7)
    eps = W.spheres_eps(shape, n_spheres=12, r_range=(3, 9), seed=11)
    coefs = W.reference_coefficients(shape, eps_re=eps)
    w = W.gaussian_wave(T, delay=20.0, width=6.0, period=10.0)
    sources = [dict(component="Jz", wave=w, k=12, kind=gd.SRC_PLANE_Z),
               dict(component="My", wave=w, i=30, j=20, k=25)]
    freqs = W.source_band(5, period=10.0, width=6.0)
    mons = [dict(component="Ez", k=30, freqs=freqs, scale=50.0 / T),
            dict(component="Hx", k=8, freqs=freqs[:3], scale=1.0)]
    omons = [oracle.Monitor(m["component"], m["k"], m["freqs"], m["scale"]) for m in mons]
    F_ref = oracle.run(shape, coefs, T, sources=[osrc(s) for s in sources], monitors=omons)
    F, D, _ = gpu_run(shape, coefs, T, sources, mons, kernel=kernel)
    assert_fields_match(F, F_ref, kernel)
    for (re, im), om in zip(D, omons):
        assert np.abs(om.re).max() > 0
        assert np.array_equal(re, om.re) and np.array_equal(im, om.im)
    del rng


def expected_folds(T, blt, slots=128):
    """Fold launches of one step call: before a launch that would overrun the staging ring,
    and once at the end."""
    t = t_fold = n = 0
    while t < T:
        b = min(blt, T - t)
        if t + b - t_fold > slots:
            n, t_fold = n + 1, t
        t += b
    return n + (1 if T > t_fold else 0)


@pytest.mark.parametrize("kernel,blt", [("tiled_w64", 2), ("tiled_w64", 3), ("tiled_w32", 5),
                                        ("tiled_w32p", 2)])
def test_dft_folds_across_ring_wraps(kernel, blt):
    """The tiled kernels stage monitor values in a 128-step ring that a fold kernel adds to the
    FP64 sums: 300 steps in one call (two wraps and a partial window) and in uneven calls
    (130 + 1 + 169) give the oracle's sums bit for bit."""
    shape, T = (40, 34, 26), 300
    coefs = W.reference_coefficients(shape)
    w = W.gaussian_wave(T, delay=30.0, width=10.0, period=12.0)
    src = [dict(component="Jz", wave=w, i=20, j=17, k=13)]
    freqs = W.source_band(11, period=12.0, width=10.0)
    mons = [dict(component="Ez", k=15, freqs=freqs, scale=1.0),
            dict(component="Hy", k=9, freqs=freqs[:3], scale=0.5)]
    omons = [oracle.Monitor(m["component"], m["k"], m["freqs"], m["scale"]) for m in mons]
    F_ref = oracle.run(shape, coefs, T, sources=[osrc(s) for s in src], monitors=omons)
    sim = gd.Simulation(*shape, kernel=kernel, blt=blt)
    sim.set_coefficients(coefs)
    sim.set_sources(src)
    mids = [sim.add_dft_monitor(m["component"], m["k"], m["freqs"], m["scale"]) for m in mons]
    for calls in ((T,), (130, 1, 169)):
        sim.reset()
        for n in calls:
            sim.step(n)
        assert sim.config()["dft_folds"] == expected_folds(calls[-1], blt)
        assert_fields_match(sim.fields(), F_ref, f"{kernel} {calls}")
        for mid, om in zip(mids, omons):
            re, im = sim.get_dft(mid)
            assert np.abs(om.re).max() > 0
            assert np.array_equal(re, om.re) and np.array_equal(im, om.im), (kernel, calls, mid)
    sim.close()


def test_per_cell_coefficients_fall_back_to_naive():
    shape, T = (48, 40, 44), 20  # 84480 cells, almost all with their own 12-tuple (> 65536)
    n = int(np.prod(shape))
    rng = np.random.default_rng(3)
    coefs = [c.copy() for c in W.vacuum_coefficients(shape)]
    coefs[0] = rng.uniform(0.9, 1.0, n).astype(np.float32)  # lossy Cax, distinct per cell
    sources = [dict(component="Jz", wave=W.gaussian_wave(T, delay=8, width=3, period=6),
                    i=24, j=20, k=22)]
    F_ref = oracle.run(shape, coefs, T, sources=[osrc(s) for s in sources])
    F, _, cfg = gpu_run(shape, coefs, T, sources, kernel="auto")
    assert cfg["kernel"] == "naive"
    assert_fields_match(F, F_ref, "per-cell")
    sim = gd.Simulation(*shape, kernel="tiled")
    sim.set_coefficients(coefs)
    assert sim.material_count() == 0
    with pytest.raises(gd.FdtdError) as e:
        sim.step(2)
    assert e.value.status == 4  # FDTD_ERR_UNSUPPORTED
    sim.close()


def test_material_count_of_reference_constructor():
    sim = gd.Simulation(60, 50, 40)
    sim.set_coefficients(W.reference_coefficients((60, 50, 40)))
    n = sim.material_count()
    coefs = W.reference_coefficients((60, 50, 40))
    stacked = np.stack([c.view(np.uint32) for c in coefs], 1)
    assert n == len(np.unique(stacked, axis=0))
    sim.close()


def test_full_size_benchmark_workload_against_oracle():
    """The benchmark workload itself (256^3 vacuum, Gaussian Jz at the centre, 8-frequency FP64
    DFT of Ez on z = 128, 1000 steps), autotuned tiled kernel against the oracle bit for bit."""
    shape, T = (256, 256, 256), 1000
    coefs = W.vacuum_coefficients(shape)
    w = W.gaussian_wave(T)
    freqs = W.source_band(8)
    mons = [dict(component="Ez", k=128, freqs=freqs, scale=1.0)]
    src = [dict(component="Jz", wave=w, i=128, j=128, k=128)]
    F, D, cfg = gpu_run(shape, coefs, T, src, mons, kernel="auto")
    assert cfg["kernel"] == "tiled"
    om = oracle.Monitor("Ez", 128, freqs, 1.0)
    F_ref = oracle.run(shape, coefs, T, sources=[osrc(s) for s in src], monitors=[om])
    assert_fields_match(F, F_ref, "256^3 x 1000")
    assert np.abs(om.re).max() > 0
    assert np.array_equal(D[0][0], om.re) and np.array_equal(D[0][1], om.im)


def test_full_size_tiled_equals_naive_and_is_linear():
    """256^3 x 1000 (the benchmark workload): size-independent properties."""
    shape, T = (256, 256, 256), 1000
    coefs = W.vacuum_coefficients(shape)
    w = W.gaussian_wave(T)
    freqs = W.source_band(8)
    mons = [dict(component="Ez", k=128, freqs=freqs, scale=1.0)]
    src = [dict(component="Jz", wave=w, i=128, j=128, k=128)]
    Ft, Dt, cfg = gpu_run(shape, coefs, T, src, mons, kernel="tiled")
    Fn, Dn, _ = gpu_run(shape, coefs, T, src, mons, kernel="naive")
    for c in range(6):
        assert np.array_equal(Ft[c].view(np.uint32), Fn[c].view(np.uint32)), oracle.COMPONENTS[c]
    assert np.array_equal(Dt[0][0], Dn[0][0]) and np.array_equal(Dt[0][1], Dn[0][1])
    assert np.abs(Dt[0][0]).max() > 0
    src2 = [dict(component="Jz", wave=w * np.float32(2), i=128, j=128, k=128)]
    F2, D2, _ = gpu_run(shape, coefs, T, src2, mons, kernel="tiled")
    # Scaling every input by 2 scales every IEEE operation exactly except in the subnormal
    # range (the far tail of the wavefront).  Once a bit differs the two runs round
    # differently, so over 1000 steps of a closed (PEC) box they drift apart by the FP32
    # rounding noise (~2e-6 relative): linearity holds to the FP32 tolerance.  Each
    # component's difference is measured against its whole field vector (E or H): Hz of a Jz
    # dipole in vacuum is zero by symmetry and holds only rounding noise.
    for c in range(6):
        grp = range(0, 3) if c < 3 else range(3, 6)
        ref_norm = np.sqrt(sum(np.linalg.norm(2 * Ft[q].astype(np.float64)) ** 2 for q in grp))
        err = np.linalg.norm(F2[c].astype(np.float64) - 2 * Ft[c].astype(np.float64))
        assert err / ref_norm <= REL_L2_TOL, oracle.COMPONENTS[c]
    assert rel_l2(D2[0][0], Dt[0][0] * 2) <= REL_L2_TOL
    assert rel_l2(D2[0][1], Dt[0][1] * 2) <= REL_L2_TOL
    assert np.isfinite(Ft[2]).all() and np.abs(Ft[2]).max() > 0


def test_split_steps_reset_and_set_field():
    shape = (33, 29, 31)
    coefs = W.reference_coefficients(shape)
    w = W.gaussian_wave(40, delay=10, width=4, period=8)
    src = [dict(component="Jz", wave=w, i=16, j=14, k=15)]
    rng = np.random.default_rng(5)
    init = [rng.standard_normal(int(np.prod(shape))).astype(np.float32) for _ in range(6)]
    F_ref = oracle.run(shape, coefs, 40, sources=[osrc(s) for s in src], fields=init)
    sim = gd.Simulation(*shape, kernel="tiled", blt=4)
    sim.set_coefficients(coefs)
    sim.set_sources(src)
    for c in range(6):
        sim.set_field(c, init[c])
    sim.step(7)
    sim.step(13)
    sim.step(20)
    assert sim.t == 40
    assert_fields_match(sim.fields(), F_ref, "split")
    sim.reset()
    assert sim.t == 0
    assert all(np.count_nonzero(f) == 0 for f in sim.fields())
    sim.close()


def test_step_on_external_stream():
    torch = pytest.importorskip("torch")
    shape, T = (40, 40, 40), 30
    coefs = W.vacuum_coefficients(shape)
    src = [dict(component="Jz", wave=W.gaussian_wave(T, delay=10, width=4, period=8),
                i=20, j=20, k=20)]
    F_ref = oracle.run(shape, coefs, T, sources=[osrc(s) for s in src])
    sim = gd.Simulation(*shape)
    sim.set_coefficients(coefs)
    sim.set_sources(src)
    s = torch.cuda.Stream()
    sim.step(T, stream=s)
    s.synchronize()
    assert_fields_match(sim.fields(), F_ref, "stream")
    sim.close()


def test_invalid_arguments_return_status():
    sim = gd.Simulation(20, 20, 20)
    with pytest.raises(gd.FdtdError) as e:
        sim.step(1)  # coefficients not set
    assert e.value.status == 1
    with pytest.raises(gd.FdtdError):
        sim.set_sources([dict(component="Jz", wave=np.ones(3, np.float32), i=25, j=1, k=1)])
    for _ in range(12):  # the monitor slots (a flux monitor takes six)
        sim.add_dft_monitor("Ez", 10, [1.0])
    with pytest.raises(gd.FdtdError) as e:
        sim.add_dft_monitor("Ez", 10, [1.0])
    assert e.value.status == 4
    sim.close()


@pytest.mark.parametrize("shape", [(37, 29, 23), (64, 48, 40)])
def test_gpu_coefficient_builder_matches_reference_formula(shape):
    """fdtd_set_permittivity computes gDiamond's constructor coefficients on the GPU."""
    eps = W.spheres_eps(shape, n_spheres=8, r_range=(2, 8), seed=2)
    for e in (None, eps):
        ref = oracle.coefficients(shape, eps_re=e)  # pinned to the reference constructor
        sim = gd.Simulation(*shape)
        sim.set_permittivity(e)
        got = sim.get_coefficients()
        for a in range(12):
            assert np.array_equal(got[a].view(np.uint32), ref[a].view(np.uint32)), oracle.COEFFS[a]
        sim2 = gd.Simulation(*shape)
        sim2.set_coefficients(ref)
        assert sim.material_count() == sim2.material_count() > 1
        sim.close()
        sim2.close()


@pytest.mark.parametrize("storage", ["f32", "f16", "f64", "f16e"])
def test_checkpoint_resume_continues_bit_for_bit(storage):
    """checkpoint() after 13 steps, restore() into a fresh handle, 11 more steps: the same
    fields and DFT sums as 24 uninterrupted steps.  16-bit storage rounds once per BLT-step
    pass, so there the split falls on a pass boundary (12 + 12: a multiple of every BLT the
    16-bit kernel uses); FP32 / FP64 split anywhere."""
    first = 12 if storage in ("f16", "f16e") else 13
    shape = (45, 33, 27)
    eps = W.spheres_eps(shape, n_spheres=3, r_range=(3, 6), seed=5)
    coefs = W.reference_coefficients(shape, eps_re=eps)
    w = W.gaussian_wave(24, delay=6.0, width=2.5, period=5.0)
    src = [dict(component="Jy", wave=w, i=20, j=15, k=12)]
    freqs = W.source_band(3, period=5.0, width=2.5)

    def make():
        sim = gd.Simulation(*shape, storage=storage)
        if storage in ("f16", "f16e"):
            sim.set_storage_scale([4.0] * 3 + [1.0] * 3)
        sim.set_coefficients(coefs)
        sim.set_sources(src)
        sim.add_dft_monitor("Ey", 14, freqs)
        return sim

    a = make()
    a.step(24)
    a.sync()
    want = a.checkpoint()
    b = make()
    b.step(first)
    ck = b.checkpoint()
    b.close()
    c = make()
    c.restore(ck)
    assert c.t == first
    c.step(24 - first)
    got = c.checkpoint()
    for f, g in zip(got["fields"], want["fields"]):
        assert np.array_equal(f, g)
    assert np.abs(want["dft"][0][0]).max() > 0
    assert all(np.array_equal(x, y) for x, y in zip(got["dft"][0], want["dft"][0]))
    a.close()
    c.close()
