"""Field snapshots on the GPU (gdiamond_b200/snapshot.py): the z-plane a Simulation returns is
the oracle's plane bit for bit (FP32 storage) and the PNG written from it decodes to the
reference colour map of that plane."""
import numpy as np
import pytest

import oracle
import gdiamond_b200 as gd
from gdiamond_b200 import snapshot as P
from gdiamond_b200 import workloads as W
from test_snapshot import decode_png

pytestmark = pytest.mark.gpu


def test_plane_and_png_match_oracle(tmp_path):
    shape, T = (48, 36, 30), 24
    nx, ny, nz = shape
    coefs = W.reference_coefficients(shape)
    w = W.gaussian_wave(T, delay=8.0, width=3.0, period=6.0)
    src = [dict(component="Jz", wave=w, i=20, j=17, k=14)]
    F = oracle.run(shape, coefs, T, sources=[oracle.Source("Jz", w, i=20, j=17, k=14)])
    sim = gd.Simulation(*shape)
    sim.set_coefficients(coefs)
    sim.set_sources(src)
    sim.step(T)
    for comp, k in (("Ez", 14), ("Hx", 3)):
        c = gd.COMPONENTS.index(comp)
        want = F[c].reshape(nz, ny, nx)[k]
        got = P.plane(sim, comp, k)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), comp
        path = str(tmp_path / f"{comp}.png")
        u = P.save_field_png(sim, path, comp, k)
        vmax = float(np.abs(want).max())
        assert vmax > 0
        assert np.array_equal(decode_png(open(path, "rb").read()), P.diverging_rgb(want, vmax))
        assert np.array_equal(u, got)
    with pytest.raises(ValueError):
        P.plane(sim, "Ez", nz)
    sim.close()


@pytest.mark.parametrize("storage", ["f16", "bf16", "f16e"])
def test_plane_of_16bit_storage_equals_the_full_field(storage):
    """plane() copies one raw z-plane and widens it with the storage scale: the same values as
    the whole-field conversion of the library, for scaled FP16 / BF16 and mixed F16E storage."""
    shape, T = (40, 32, 24), 20
    nx, ny, nz = shape
    sim = gd.Simulation(*shape, storage=storage)
    sim.set_storage_scale([4.0, 4.0, 4.0, 0.25, 0.25, 0.25])
    sim.set_coefficients(W.reference_coefficients(shape))
    w = W.gaussian_wave(T, delay=8.0, width=3.0, period=6.0)
    sim.set_sources([dict(component="Jz", wave=w, i=20, j=16, k=12)])
    sim.step(T)
    for comp in ("Ex", "Ez", "Hy"):
        got = P.plane(sim, comp, 12)
        want = sim.get_field(comp).reshape(nz, ny, nx)[12]
        assert np.abs(want).max() > 0
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (storage, comp)
    sim.close()
