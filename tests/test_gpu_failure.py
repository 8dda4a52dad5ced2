"""GPU failure detection without a GPU fault: a bounded wait that runs out.

The reference's error path is CUDACHECK -> printf + exit(1) (gDiamond/gdiamond_gpu.cuh:11-20).
Here every mbarrier wait of the tiled kernels is bounded; when one gives up, the tile records
FDTD_ERR_DEVICE_TIMEOUT in the handle's device error word, waits (bounded) for its own copies in
flight, and leaves its z-march; fdtd_sync reports the status.  The test hook
fdtd_debug_fail_copy makes one tile skip issuing one plane copy, so its wait has nothing to
wait for (a flag that nothing sets) and runs out after a short limit.  Nothing faults, traps or
hangs: the context stays usable, which the test shows by resetting and stepping bit-exactly
against the oracle afterwards.
"""
import numpy as np
import pytest

import oracle
import gdiamond_b200 as gd
from gdiamond_b200 import workloads as W
from test_gpu_parity import assert_fields_match, osrc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("family,blt,rows,storage", [("tiled_w32p", 2, 24, "f32"),
                                                     ("tiled_w64", 3, 16, "f32"),
                                                     ("tiled_w32p", 2, 32, "f16e")])
def test_expired_wait_reports_timeout_and_handle_recovers(family, blt, rows, storage):
    shape, T = (70, 52, 41), 12
    coefs = W.reference_coefficients(shape)
    w = W.gaussian_wave(T, delay=4.0, width=2.0, period=5.0)
    src = [dict(component="Jz", wave=w, i=35, j=26, k=20)]
    sim = gd.Simulation(*shape, kernel=family, blt=blt, tile_rows=rows, z_chunks=2,
                        storage=storage)
    sim.set_coefficients(coefs)
    sim.set_sources(src)
    sim.step(blt)  # tunes nothing (one configuration) and runs cleanly
    sim.sync()
    sim.debug_fail_copy((1, 1, 0), iteration=5, wait_cycles=2_000_000)  # ~1 ms
    sim.step(blt)
    with pytest.raises(gd.FdtdError) as e:
        sim.sync()
    assert e.value.status == 5  # FDTD_ERR_DEVICE_TIMEOUT
    sim.sync()  # reported once, then cleared
    # the hook fired once; after a reset the handle steps correctly
    sim.reset()
    sim.step(T)
    sim.sync()
    if storage == "f32":
        F_ref = oracle.run(shape, coefs, T, sources=[osrc(s) for s in src])
        assert_fields_match(sim.fields(), F_ref, f"after timeout {family}")
    else:
        assert all(np.isfinite(f).all() for f in sim.fields())
    sim.close()
