"""Learned spectrum surrogate with FDTD fallback.

Design space: one axis-aligned dielectric box in a 96^3 grid with gDiamond's graded pseudo-PML
(10 cells on every face), six numbers per design:

    (cx, cy, cz)   box centre, each uniform in the central half of the grid [N/4, 3N/4]
    a              lateral side (x and y), uniform in [8, 40] cells (N/12 .. 5N/12)
    h              height along z, uniform in [8, 40] cells
    eps            relative permittivity, uniform in [2, 12]

The box is anti-aliased (a boundary cell gets eps = 1 + (eps-1) * covered volume fraction), so
the spectrum is a continuous function of the six numbers rather than a staircase in them.

Excitation and observable: a current sheet on the interior of plane z = 10 driven by the
Gaussian-modulated sinusoid of the point-source workloads launches a quasi-plane pulse along +z.
A Poynting-flux monitor on plane z = 86 at 64 frequencies across the source band
(fdtd_add_flux_monitor: Re(Ex conj(Hy) - Ey conj(Hx)) summed over the plane, H co-located with
E in z and phased half a step later) gives the transmission spectrum as that flux divided by
the same flux without the box ("flux"); the coherent normal-incidence amplitude
|Sum Ex|^2 / |Sum Ex_empty|^2, from the monitor's Ex DFT, is available as "amplitude".  The
sheet current is transverse (Jx): a z-directed current spread uniformly over a z-plane has zero
curl and launches no wave along z.

SpectrumSolver runs designs through the batched FDTD solver (the data generator, the fallback
and the ground truth).  Surrogate wraps an ensemble of MLPs 6 -> 256 -> 256 -> 256 -> 64 (GELU, BF16
tensor-core GEMMs with FP32 accumulation, Adam) trained on the GPU by gdiamond_b200.MLP; a
design whose ensemble disagreement (mean over the spectrum of the members' standard deviation,
relative to the mean over the spectrum of |ensemble mean|) exceeds a threshold (1%) is sent to
FDTD instead.
"""
from __future__ import annotations

import time

import numpy as np

from . import MLP, SRC_PLANE_Z, Batch, Simulation
from . import workloads as W

SHAPE = (96, 96, 96)
SOURCE_K = 10
MONITOR_K = 86
N_FREQS = 64
T_STEPS = 2000
DIMS = (6, 256, 256, 256, 64)
PARAM_NAMES = ("cx", "cy", "cz", "side", "height", "eps")


def param_bounds(shape=SHAPE):
    """(lo, hi) of the six design numbers; box sides span [N/12, 5N/12] of the smallest axis
    ([8, 40] cells at 96^3)."""
    nx, ny, nz = shape
    n = min(shape)
    lo = np.array([nx / 4, ny / 4, nz / 4, n / 12, n / 12, 2.0])
    hi = np.array([3 * nx / 4, 3 * ny / 4, 3 * nz / 4, 5 * n / 12, 5 * n / 12, 12.0])
    return lo, hi


def sample_designs(n, seed=0, shape=SHAPE):
    """n designs uniform in the design space (seeded)."""
    lo, hi = param_bounds(shape)
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=(int(n), 6)).astype(np.float32)


def _coverage(n, lo, hi):
    """Fraction of cell i (spanning [i-0.5, i+0.5]) inside [lo, hi]."""
    c = np.arange(n, dtype=np.float64)
    return np.clip(np.minimum(c + 0.5, hi) - np.maximum(c - 0.5, lo), 0.0, 1.0)


def design_eps(p, shape=SHAPE):
    """Per-cell relative permittivity (x-fastest, float32) of one design."""
    nx, ny, nz = shape
    cx, cy, cz, a, h, e = (float(v) for v in p)
    fx = _coverage(nx, cx - a / 2, cx + a / 2)
    fy = _coverage(ny, cy - a / 2, cy + a / 2)
    fz = _coverage(nz, cz - h / 2, cz + h / 2)
    frac = fz[:, None, None] * fy[None, :, None] * fx[None, None, :]
    return (1.0 + (e - 1.0) * frac).astype(np.float32).reshape(-1)


def bucket(n, group):
    """Batch size used for n designs: the next power of two (at least 4), at most `group`.
    Padding a call to a few fixed sizes keeps the number of batches (each created, tuned and
    graph-captured once) small, so a fallback call of any size costs a predictable time."""
    b = 4
    while b < n:
        b *= 2
    return min(b, group)


class SpectrumSolver:
    """Transmission spectra of designs by batched FDTD (FP32 fields, FP64 DFT sums).

    observable: "flux" (default) or "amplitude", as described in the module docstring.
    boundary: "pml" (default), the reference's graded pseudo-PML of t_pml cells (10) in the
    coefficients in front of never-updated faces; or "cpml", CPML layers of t_pml cells (8) on
    every face (fdtd_set_cpml) with vacuum coefficients, which reflect far less.  With 8-cell
    layers the source plane z = 10 and the flux plane z = 86 of a 96^3 grid stay outside them.

    Simulations are created once (`group` of them) and reused: each group of designs gets new
    permittivities, a reset, and one persistent batched run of T steps replayed from a CUDA
    graph.  Groups smaller than `group` are padded to a bucket size (see `bucket`) with copies
    of their last design, whose results are dropped.
    """

    def __init__(self, shape=SHAPE, T=T_STEPS, n_freqs=N_FREQS, group=256, storage="f32",
                 source_k=SOURCE_K, monitor_k=MONITOR_K, t_pml=None, observable="flux",
                 device=0, boundary="pml"):
        import torch
        if observable not in ("flux", "amplitude"):
            raise ValueError("observable is 'flux' or 'amplitude'")
        if boundary not in ("pml", "cpml"):
            raise ValueError("boundary is 'pml' (the reference's graded pseudo-PML) or 'cpml'")
        self.shape, self.T, self.group, self.storage = tuple(shape), int(T), int(group), storage
        if t_pml is None:
            t_pml = 10 if boundary == "pml" else 8
        self.t_pml, self.observable, self.boundary = int(t_pml), observable, boundary
        self.source_k, self.monitor_k, self.device = int(source_k), int(monitor_k), device
        nz = self.shape[2]
        if boundary == "cpml" and not (self.t_pml <= self.source_k and
                                       self.monitor_k <= nz - 2 - self.t_pml):
            raise ValueError("the source and flux planes must lie outside the CPML layers")
        self.freqs = W.source_band(n_freqs)
        self.wave = W.gaussian_wave(self.T)
        self.sims = []
        self.batches = {}
        self._empty = None
        nx, ny, _ = self.shape
        self._re = torch.empty((n_freqs, ny, nx), dtype=torch.float64, device=f"cuda:{device}")
        self._im = torch.empty_like(self._re)
        self._flux = torch.empty((group, n_freqs), dtype=torch.float64, device=f"cuda:{device}")
        self._ids = {}  # sim -> (flux monitor id, Ex monitor id)
        self.seconds = 0.0  # wall time in measure(): permittivities, batched runs, read-back

    def _make(self):
        sim = Simulation(*self.shape, storage=self.storage, device=self.device)
        if self.boundary == "cpml":
            sim.set_cpml(thickness=self.t_pml)
        sim.set_sources([dict(component="Jx", kind=SRC_PLANE_Z, k=self.source_k, wave=self.wave)])
        fid = sim.add_flux_monitor(self.monitor_k, self.freqs)
        self._ids[id(sim)] = (fid, sim.flux_monitor_ids(fid)[0])
        return sim

    def _measure(self, sims):
        """[n][n_freqs] complex plane sums of Ex, and the z-fluxes of the flux monitors."""
        import torch
        nf = len(self.freqs)
        ex = np.empty((len(sims), nf), np.complex128)
        stream = torch.cuda.current_stream(self.device)
        exs = torch.empty((len(sims), 2, nf), dtype=torch.float64, device=self._re.device)
        for n, sim in enumerate(sims):
            fid, exid = self._ids[id(sim)]
            sim.get_flux_device(fid, self._flux[n].data_ptr(), stream)
            sim.get_dft_device(exid, self._re.data_ptr(), self._im.data_ptr(), stream)
            exs[n, 0] = self._re.sum(dim=(1, 2))
            exs[n, 1] = self._im.sum(dim=(1, 2))
        flux = self._flux[:len(sims)].cpu().numpy().copy()
        e = exs.cpu().numpy()
        ex[:] = e[:, 0] + 1j * e[:, 1]
        return ex, flux

    def _pml_cells(self):
        """Thickness of the graded pseudo-PML in the coefficients (none under CPML layers)."""
        return self.t_pml if self.boundary == "pml" else 0

    def empty(self):
        """(Ex plane sum, flux) of the grid without a box (the normalisation)."""
        if self._empty is None:
            sim = self._make()
            sim.set_permittivity(None, t_pml=self._pml_cells())
            sim.step(self.T)
            sim.sync()
            ex, flux = self._measure([sim])
            self._empty = (ex[0], flux[0])
            sim.close()
        return self._empty

    def measure(self, designs):
        """(Ex plane sums [n][n_freqs] complex, fluxes [n][n_freqs]) of every design."""
        designs = np.asarray(designs, np.float32).reshape(-1, 6)
        nf = len(self.freqs)
        ex = np.empty((len(designs), nf), np.complex128)
        flux = np.empty((len(designs), nf), np.float64)
        t0 = time.perf_counter()
        for g0 in range(0, len(designs), self.group):
            chunk = designs[g0:g0 + self.group]
            nb = bucket(len(chunk), self.group)
            padded = np.concatenate([chunk, np.repeat(chunk[-1:], nb - len(chunk), axis=0)])
            while len(self.sims) < nb:
                self.sims.append(self._make())
            sims = self.sims[:nb]
            for sim, p in zip(sims, padded):
                sim.set_permittivity(design_eps(p, self.shape), t_pml=self._pml_cells())
                sim.reset()
            for sim in sims:
                sim.sync()
            b = self.batches.get(nb)
            if b is None:
                b = self.batches[nb] = Batch(sims)
            b.step(self.T)
            for sim in sims:
                sim.sync()
            e, f = self._measure(sims)
            ex[g0:g0 + len(chunk)], flux[g0:g0 + len(chunk)] = e[:len(chunk)], f[:len(chunk)]
        self.seconds += time.perf_counter() - t0
        return ex, flux

    def warm(self):
        """Creates, tunes and captures the batch of every bucket size once (one design per
        call), so later calls of any size run on cached graphs."""
        b = 4
        probe = sample_designs(1, seed=12345, shape=self.shape)
        while True:
            self.measure(np.repeat(probe, min(b, self.group), axis=0))
            if b >= self.group:
                break
            b *= 2

    def to_spectra(self, ex, flux):
        """Spectra [n][n_freqs] of measurements, by the solver's observable."""
        ex0, flux0 = self.empty()
        if self.observable == "flux":
            return np.asarray(flux) / flux0[None, :]
        return np.abs(np.asarray(ex) / ex0[None, :]) ** 2

    def spectra(self, designs):
        """Transmission spectra [n][n_freqs] (float64) of designs."""
        return self.to_spectra(*self.measure(designs))

    def close(self):
        for b in self.batches.values():
            b.close()
        for s in self.sims:
            s.close()
        self.batches, self.sims = {}, []


def spectral_error(pred, ref):
    """Relative L2 error of each predicted spectrum against the reference [n]."""
    pred, ref = np.asarray(pred, np.float64), np.asarray(ref, np.float64)
    return np.linalg.norm(pred - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-300)


class Surrogate:
    """Ensemble MLP surrogate of SpectrumSolver.spectra with FDTD fallback."""

    def __init__(self, dims=DIMS, members=4, seed=0, shape=SHAPE, device=0):
        self.net = MLP(dims, members=members, seed=seed, device=device)
        self.lo, self.hi = param_bounds(shape)
        self.y_mean = np.zeros(dims[-1])
        self.y_std = np.ones(dims[-1])

    def _x(self, designs):
        d = np.asarray(designs, np.float64).reshape(-1, 6)
        return (2.0 * (d - self.lo) / (self.hi - self.lo) - 1.0).astype(np.float32)

    def fit(self, designs, spectra, epochs=200, batch=64, lr=1e-3, seed=0):
        """Trains every member on standardised spectra; returns the loss per epoch."""
        y = np.asarray(spectra, np.float64)
        self.y_mean = y.mean(axis=0)
        self.y_std = np.maximum(y.std(axis=0), 1e-12)
        self.net.set_data(self._x(designs), ((y - self.y_mean) / self.y_std).astype(np.float32))
        return self.net.train(epochs, batch=batch, lr=lr, seed=seed)

    def predict(self, designs):
        """(mean, sd) of the members' spectra [n][n_freqs], in spectrum units."""
        m, s = self.net.predict(self._x(designs))
        return m * self.y_std + self.y_mean, s * self.y_std

    @staticmethod
    def disagreement(mean, sd):
        """Per design: mean over the spectrum of sd / mean over the spectrum of |mean|."""
        return np.mean(sd, axis=1) / np.maximum(np.mean(np.abs(mean), axis=1), 1e-30)

    def evaluate(self, designs, solver, threshold=0.01):
        """Spectra of `designs` from the surrogate, with designs whose disagreement exceeds
        `threshold` recomputed by `solver` (a SpectrumSolver).  Returns (spectra, fallback
        mask, seconds in the surrogate, seconds in the fallback solver)."""
        t0 = time.perf_counter()
        mean, sd = self.predict(designs)
        t1 = time.perf_counter()
        mask = self.disagreement(mean, sd) > threshold
        out = mean.astype(np.float64)
        t2 = t1
        if mask.any():
            out[mask] = solver.spectra(np.asarray(designs)[mask])
            t2 = time.perf_counter()
        return out, mask, t1 - t0, t2 - t1

    def close(self):
        self.net.close()


def active_designs(sur, pool, k):
    """The k designs of `pool` on which the ensemble `sur` disagrees most (active sampling: the
    solver's runs go where the network is uncertain, the large high-index boxes whose spectra
    vary fastest)."""
    mean, sd = sur.predict(pool)
    order = np.argsort(-Surrogate.disagreement(mean, sd))
    return np.asarray(pool)[order[:int(k)]]
