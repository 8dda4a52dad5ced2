"""One grid run as z-slabs on the GPU (gdiamond_b200/slabs.py ZSlabGrid): several handles on one
device, halo exchange through fdtd_get/set_planes_device after every BLT-step launch, against
the same grid run as one handle with the same BLT -- bit for bit, fields and DFT sums, for FP32,
BF16 and F16E storage (the exchange moves stored values raw; F16E's E and H components differ
in size), with a short last block.
"""
import numpy as np
import pytest

import gdiamond_b200 as gd
from gdiamond_b200 import slabs as Z
from gdiamond_b200 import workloads as W

pytestmark = pytest.mark.gpu

SHAPE = (70, 44, 61)


def problem(T):
    eps = W.spheres_eps(SHAPE, n_spheres=6, r_range=(3, 7), seed=2)
    coefs = W.reference_coefficients(SHAPE, eps_re=eps, t_pml=4)
    w = W.gaussian_wave(T, delay=8.0, width=3.0, period=6.0)
    nx, ny, nz = SHAPE
    sources = [dict(component="Jz", wave=w, i=nx // 2, j=ny // 2, k=21),
               dict(component="My", wave=w * np.float32(0.3), i=9, j=30, k=40),
               dict(component="Jx", wave=w * np.float32(0.05), k=12, kind=gd.SRC_PLANE_Z)]
    freqs = W.source_band(4, period=6.0, width=3.0)
    return coefs, sources, freqs


@pytest.mark.parametrize("storage", ["f32", "bf16", "f16e"])
@pytest.mark.parametrize("parts,halo,T", [(3, 2, 31), (2, 3, 20), (4, 1, 9)])
def test_slabs_match_single_grid(storage, parts, halo, T):
    coefs, sources, freqs = problem(T)
    mon_k = 22  # one plane above the Jz source: nonzero sums even for the short runs
    one = gd.Simulation(*SHAPE, kernel="tiled", blt=halo, storage=storage)
    one.set_coefficients(coefs)
    one.set_sources(sources)
    m1 = one.add_dft_monitor("Ez", mon_k, freqs)
    one.step(T)
    one.sync()
    ref = [one.get_field(c) for c in gd.COMPONENTS]
    ref_dft = one.get_dft(m1)
    one.close()

    grid = Z.ZSlabGrid(*SHAPE, parts=parts, halo=halo, storage=storage)
    grid.set_coefficients(coefs)
    grid.set_sources(sources)
    mid = grid.add_dft_monitor("Ez", mon_k, freqs)
    grid.step(T)
    grid.sync()
    for c, f in enumerate(grid.fields()):
        assert np.array_equal(f.view(np.uint32), ref[c].view(np.uint32)), gd.COMPONENTS[c]
    re, im = grid.get_dft(mid)
    assert np.abs(ref_dft[0]).max() > 0
    assert np.array_equal(re, ref_dft[0]) and np.array_equal(im, ref_dft[1])
    grid.close()


def test_plane_copies_round_trip():
    sim = gd.Simulation(40, 24, 16)
    x = np.arange(40 * 24 * 16, dtype=np.float32)
    sim.set_field("Hy", x)
    import torch
    buf = torch.empty((3, 24, 40), dtype=torch.int32, device="cuda")
    sim.get_planes_device("Hy", 5, 3, buf.data_ptr())
    sim.sync()
    got = buf.cpu().numpy().view(np.float32)
    assert np.array_equal(got, x.reshape(16, 24, 40)[5:8])
    sim.set_planes_device("Ex", 0, 3, buf.data_ptr())
    sim.sync()
    assert np.array_equal(sim.get_field("Ex").reshape(16, 24, 40)[:3], got)
    with pytest.raises(gd.FdtdError):
        sim.get_planes_device("Ex", 14, 3, buf.data_ptr())  # past the last plane
    sim.close()
