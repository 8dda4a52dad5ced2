"""GPU: the Poynting-flux monitor (fdtd_add_flux_monitor / fdtd_get_flux) against the oracle.

The reference has no flux monitor, only the per-cell running DFT of Ex
(gDiamond/kernels.cuh:87-113); the oracle restates the flux definition (oracle.flux): six running
DFTs (Ex, Ey on the E plane k; Hx, Hy on planes k-1 and k, phased at (t + 1/2) dt), and
flux(f) = dx^2 sum Re[Ex conj(Hy) - Ey conj(Hx)] with H averaged over the two planes.  The six
monitor sums must equal the oracle's bit for bit (the half-step cos/sin tables included); the
GPU's fixed-order FP64 reduction agrees with numpy's sum to 1e-12 relative.  A physical check:
a current sheet radiates power away from itself through planes on both sides.
"""
import numpy as np
import pytest

import oracle
import gdiamond_b200 as gd
from gdiamond_b200 import workloads as W
from test_gpu_parity import assert_fields_match, osrc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernel", ["tiled", "naive"])
def test_flux_monitor_matches_oracle(kernel):
    shape, T = (48, 40, 44), 160
    nx, ny, nz = shape
    eps = W.spheres_eps(shape, n_spheres=4, r_range=(3, 6), eps_range=(2.0, 6.0), seed=3)
    coefs = W.reference_coefficients(shape, eps_re=eps)
    w = W.gaussian_wave(T, delay=30.0, width=8.0, period=10.0)
    src = [dict(component="Jx", wave=w, k=14, kind=gd.SRC_PLANE_Z),
           dict(component="Jz", wave=w * np.float32(0.1), i=20, j=18, k=22)]
    freqs = W.source_band(6, period=10.0, width=8.0)
    k_up, k_dn = 30, 8
    sim = gd.Simulation(*shape, kernel=kernel)
    sim.set_coefficients(coefs)
    sim.set_sources(src)
    f_up = sim.add_flux_monitor(k_up, freqs)
    f_dn = sim.add_flux_monitor(k_dn, freqs)
    sim.step(T)
    sim.sync()
    got_up, got_dn = sim.get_flux(f_up), sim.get_flux(f_dn)
    mons_up, mons_dn = oracle.flux_monitors(k_up, freqs), oracle.flux_monitors(k_dn, freqs)
    F_ref = oracle.run(shape, coefs, T, sources=[osrc(s) for s in src],
                       monitors=mons_up + mons_dn)
    assert_fields_match(sim.fields(), F_ref, f"flux {kernel}")
    for fid, mons in ((f_up, mons_up), (f_dn, mons_dn)):
        for mid, om in zip(sim.flux_monitor_ids(fid), mons):
            re, im = sim.get_dft(mid)
            assert np.array_equal(re, om.re) and np.array_equal(im, om.im), (fid, mid)
    dx = float(np.float32(0.1))
    want_up, want_dn = oracle.flux(mons_up, dx), oracle.flux(mons_dn, dx)
    np.testing.assert_allclose(got_up, want_up, rtol=1e-12, atol=1e-12 * np.abs(want_up).max())
    np.testing.assert_allclose(got_dn, want_dn, rtol=1e-12, atol=1e-12 * np.abs(want_dn).max())
    # the sheet radiates away from itself: +z flux above it, -z flux below, at the band centre
    mid_f = len(freqs) // 2
    assert got_up[mid_f] > 0 and got_dn[mid_f] < 0
    sim.close()


def test_flux_monitor_in_batches_and_device_output():
    import torch
    shape, T = (40, 36, 40), 120
    coefs = W.reference_coefficients(shape)
    w = W.gaussian_wave(T, delay=30.0, width=8.0, period=10.0)
    src = [dict(component="Jx", wave=w, k=10, kind=gd.SRC_PLANE_Z)]
    freqs = W.source_band(4, period=10.0, width=8.0)
    sims, fids = [], []
    for _ in range(2):
        s = gd.Simulation(*shape)
        s.set_coefficients(coefs)
        s.set_sources(src)
        fids.append(s.add_flux_monitor(26, freqs))
        sims.append(s)
    b = gd.Batch(sims)
    b.step(T)
    for s in sims:
        s.sync()
    mons = oracle.flux_monitors(26, freqs)
    oracle.run(shape, coefs, T, sources=[osrc(x) for x in src], monitors=mons)
    want = oracle.flux(mons, float(np.float32(0.1)))
    out = torch.zeros(len(freqs), dtype=torch.float64, device="cuda")
    for s, fid in zip(sims, fids):
        np.testing.assert_allclose(s.get_flux(fid), want, rtol=1e-12)
        s.get_flux_device(fid, out.data_ptr())
        torch.cuda.synchronize()
        np.testing.assert_allclose(out.cpu().numpy(), want, rtol=1e-12)
    b.close()
    for s in sims:
        s.close()


def test_flux_monitor_argument_checks():
    sim = gd.Simulation(20, 20, 20)
    sim.set_coefficients(W.vacuum_coefficients((20, 20, 20)))
    freqs = np.array([0.5, 1.0])
    for k in (0, 19):  # the flux plane needs H on both sides
        with pytest.raises(gd.FdtdError):
            sim.add_flux_monitor(k, freqs)
    sim.add_flux_monitor(5, freqs)
    sim.add_flux_monitor(10, freqs)
    with pytest.raises(gd.FdtdError):  # 12 monitor slots: two flux monitors
        sim.add_flux_monitor(12, freqs)
    sim.close()
