"""The spectrum surrogate end to end on a small grid (32^3, T=300, 16 frequencies).

* the batched FDTD spectrum solver (data generator, fallback, ground truth) against the oracle: the
  plane-summed Ex DFT and the Poynting flux (the flux monitor's definition, oracle.flux) of a
  design run in a batch equal the oracle's for the same permittivity, and a box of eps 1
  transmits exactly 1;
* fallback calls of any size run on a few bucketed batch sizes;
* what the trained network gains over the method without it: on held-out designs the
  ensemble is at least twice as close to FDTD as the best constant guess (the training-set
  mean spectrum), and
  the surrogate with fallback answers many times more designs per second than the batched
  solver, returning the solver's own spectra for the designs it sends back.
"""
import numpy as np
import pytest

import oracle
from gdiamond_b200 import surrogate as S
from gdiamond_b200 import workloads as W

pytestmark = pytest.mark.gpu

SHAPE, T, NF, SRC_K, MON_K, PML = (32, 32, 32), 300, 16, 4, 27, 4


def solver(group=64, observable="flux"):
    return S.SpectrumSolver(shape=SHAPE, T=T, n_freqs=NF, group=group, source_k=SRC_K,
                            monitor_k=MON_K, t_pml=PML, observable=observable)


def test_solver_matches_oracle_and_unit_transmission():
    sol = solver(group=3, observable="amplitude")  # measures the Ex sums as well
    designs = S.sample_designs(3, seed=5, shape=SHAPE)
    designs[2, 5] = 1.0  # eps 1: the empty grid
    ex, flux = sol.measure(designs)
    for p, got_ex, got_flux in zip(designs[:2], ex[:2], flux[:2]):
        eps = S.design_eps(p, SHAPE)
        coefs = W.reference_coefficients(SHAPE, eps_re=eps, t_pml=PML)
        mons = oracle.flux_monitors(MON_K, sol.freqs)
        oracle.run(SHAPE, coefs, T, sources=[oracle.Source("Jx", sol.wave, k=SRC_K,
                                                           kind=oracle.PLANE_Z)],
                   monitors=mons)
        me = mons[0]
        want_ex = me.re.sum(axis=(1, 2)) + 1j * me.im.sum(axis=(1, 2))
        want_flux = oracle.flux(mons, float(np.float32(0.1)))
        assert np.abs(want_ex).max() > 0 and np.abs(want_flux).max() > 0
        assert np.allclose(got_ex, want_ex, rtol=1e-12, atol=1e-12 * np.abs(want_ex).max())
        assert np.allclose(got_flux, want_flux, rtol=1e-12, atol=1e-12 * np.abs(want_flux).max())
    for obs in ("flux", "amplitude"):
        sol.observable = obs
        spec = sol.to_spectra(ex, flux)
        assert np.allclose(spec[2], 1.0, rtol=0, atol=1e-12)  # up to the division
        assert np.all(np.abs(spec[:2] - 1).max(axis=1) > 1e-3)  # a real box changes it
    sol.close()


def test_cpml_solver_matches_single_grids_and_unit_transmission():
    """boundary="cpml": CPML layers on every face, vacuum coefficients, flux plane in front of
    the top layer (a plane inside a layer is refused).  The batched CPML solver's fluxes equal a single grid's (per-step monitor
    accumulation) to the reduction's rounding, and a box of eps 1 transmits exactly 1."""
    from gdiamond_b200 import SRC_PLANE_Z, Simulation
    sol = S.SpectrumSolver(shape=SHAPE, T=T, n_freqs=NF, group=3, source_k=SRC_K, t_pml=PML,
                           monitor_k=SHAPE[2] - PML - 2, boundary="cpml")
    with pytest.raises(ValueError):  # a flux plane inside the top layer
        S.SpectrumSolver(shape=SHAPE, T=T, source_k=SRC_K, t_pml=PML, monitor_k=SHAPE[2] - PML,
                         boundary="cpml")
    designs = S.sample_designs(3, seed=6, shape=SHAPE)
    designs[2, 5] = 1.0
    ex, flux = sol.measure(designs)
    for p, got in zip(designs[:2], flux[:2]):
        sim = Simulation(*SHAPE)
        sim.set_cpml(thickness=PML)
        sim.set_permittivity(S.design_eps(p, SHAPE), t_pml=0)
        sim.set_sources([dict(component="Jx", kind=SRC_PLANE_Z, k=SRC_K, wave=sol.wave)])
        fid = sim.add_flux_monitor(sol.monitor_k, sol.freqs)
        sim.step(T)
        sim.sync()
        assert sim.config()["kernel"] == "cpml"
        want = sim.get_flux(fid)
        sim.close()
        assert np.abs(want).max() > 0
        assert np.array_equal(got, want)
    spec = sol.to_spectra(ex, flux)
    assert np.allclose(spec[2], 1.0, rtol=0, atol=1e-12)
    assert np.all(np.abs(spec[:2] - 1).max(axis=1) > 1e-3)
    sol.close()


def test_surrogate_gain_over_solver():
    sol = solver()
    train = S.sample_designs(768, seed=1, shape=SHAPE)
    test = S.sample_designs(64, seed=2, shape=SHAPE)
    y_train = sol.spectra(train)
    sol.seconds = 0.0
    y_test = sol.spectra(test)
    solver_rate = len(test) / sol.seconds
    sur = S.Surrogate(dims=(6, 256, 256, 256, NF), members=4, seed=0, shape=SHAPE)
    losses = sur.fit(train, y_train, epochs=150, batch=64, lr=1e-3, seed=0)
    assert np.all(losses[-1] < 0.1 * losses[0])
    mean, sd = sur.predict(test)
    err = S.spectral_error(mean, y_test)
    base = S.spectral_error(np.broadcast_to(y_train.mean(0), y_test.shape), y_test)
    assert err.mean() < 0.5 * base.mean(), (err.mean(), base.mean())
    # surrogate with FDTD fallback: the loosest threshold sends nothing back, a threshold of
    # 0 sends everything back and reproduces the solver exactly
    out, mask, t_sur, t_fb = sur.evaluate(test, sol, threshold=np.inf)
    assert not mask.any() and np.array_equal(out, mean.astype(np.float64))
    assert len(test) / t_sur > 10 * solver_rate
    thr = float(np.median(S.Surrogate.disagreement(mean, sd)))
    out, mask, _, _ = sur.evaluate(test, sol, threshold=thr)
    assert 0 < mask.sum() < len(test)
    assert np.allclose(out[mask], y_test[mask], rtol=1e-12, atol=0)
    assert np.array_equal(out[~mask], mean[~mask].astype(np.float64))
    # designs the ensemble disagrees on are, on average, the ones it gets wrong
    assert err[mask].mean() > err[~mask].mean()
    sur.close()
    # the fallback calls above ran on bucketed batch sizes only
    assert set(sol.batches) <= {4, 8, 16, 32, 64}
    sol.close()

