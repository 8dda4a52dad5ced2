"""Test infrastructure only: Python access to the CPU oracle for the FDTD (Yee) hot path.

Two shared libraries are wrapped here, both built by ``make -C oracle``:

* ``oracle/liboracle.so`` -- our plain-C restatement of the reference algorithm
  (``oracle/fdtd_oracle.c``): the coefficient builder of gDiamond's constructor
  (gDiamond/utils.h:542-690), the FP32 Yee stepper of ``update_FDTD_seq``
  (gDiamond/gdiamond.hpp:1193-1221) with general J/M sources, an FP64 twin, and FP64
  running-DFT monitors (the FP32 GPU monitor of gDiamond/kernels.cuh:87-113 restated in FP64).
* ``oracle/_ref/libgdref.so`` -- the reference's own ``gDiamond`` class compiled from its
  sources (``oracle/ref_harness.cpp``): constructor, ``update_FDTD_seq``, ``update_FDTD_omp``
  and ``update_FDTD_omp_dt``.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` use this
module, and only as the checker or the timed CPU baseline.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(_HERE, "liboracle.so")
REF_SO = os.path.join(_HERE, "_ref", "libgdref.so")

COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
COEFFS = ("Cax", "Cay", "Caz", "Cbx", "Cby", "Cbz", "Dax", "Day", "Daz", "Dbx", "Dby", "Dbz")
SRC_COMPONENTS = ("Jx", "Jy", "Jz", "Mx", "My", "Mz")
POINT, PLANE_Z = 0, 1


class _Source(C.Structure):
    _fields_ = [("component", C.c_int32), ("kind", C.c_int32),
                ("i", C.c_int64), ("j", C.c_int64), ("k", C.c_int64)]


class _Monitor(C.Structure):
    _fields_ = [("component", C.c_int32), ("nf", C.c_int32), ("k", C.c_int64),
                ("scale", C.c_double),
                ("cos_tab", C.POINTER(C.c_double)), ("sin_tab", C.POINTER(C.c_double)),
                ("re", C.POINTER(C.c_double)), ("im", C.POINTER(C.c_double))]


_lib = None
_ref = None


def build():
    """Compile liboracle.so (and the reference harness when its sources are present)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        P = C.POINTER
        L.oracle_coefficients.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_float, C.c_float,
                                          C.c_float, C.c_int, P(C.c_float), P(C.c_float),
                                          P(P(C.c_float))]
        L.oracle_reference_params.argtypes = [P(C.c_float), P(C.c_int)]
        L.oracle_reference_mz_wave.argtypes = [C.c_int64, P(C.c_float)]
        L.oracle_dft_tables.argtypes = [P(C.c_double), C.c_int, C.c_double, C.c_int64,
                                        P(C.c_double), P(C.c_double)]
        L.oracle_dft_tables_offset.argtypes = [P(C.c_double), C.c_int, C.c_double, C.c_double,
                                               C.c_int64, P(C.c_double), P(C.c_double)]
        for name, T in (("oracle_run_f32", C.c_float), ("oracle_run_f64", C.c_double)):
            getattr(L, name).argtypes = [C.c_int64, C.c_int64, C.c_int64, P(P(T)),
                                         P(P(C.c_float)), C.c_float, P(_Source), C.c_int,
                                         P(C.c_float), C.c_int64, C.c_int64, C.c_int64,
                                         P(_Monitor), C.c_int]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    """The reference's own solvers (oracle/_ref/libgdref.so)."""
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError("oracle/_ref/libgdref.so is not built (reference sources absent)")
        L = C.CDLL(REF_SO)
        P = C.POINTER
        L.gdref_create.restype = C.c_void_p
        L.gdref_create.argtypes = [C.c_size_t] * 3
        L.gdref_destroy.argtypes = [C.c_void_p]
        L.gdref_get_coefficients.argtypes = [C.c_void_p, P(P(C.c_float))]
        L.gdref_source_idx.restype = C.c_size_t
        L.gdref_source_idx.argtypes = [C.c_void_p]
        L.gdref_params.argtypes = [C.c_void_p, P(C.c_float)]
        for n in ("gdref_run_seq", "gdref_run_omp"):
            getattr(L, n).restype = C.c_double
            getattr(L, n).argtypes = [C.c_void_p, C.c_size_t]
        L.gdref_run_omp_dt.restype = C.c_double
        L.gdref_run_omp_dt.argtypes = [C.c_void_p] + [C.c_size_t] * 5
        L.gdref_get_fields.restype = C.c_int
        L.gdref_get_fields.argtypes = [C.c_void_p, C.c_int, P(P(C.c_float))]
        L.gdref_max_threads.restype = C.c_int
        L.gdref_last_printed_seconds.restype = C.c_double
        L.gdref_save_field_png.argtypes = [P(C.c_float), C.c_char_p, C.c_int, C.c_int,
                                           C.c_float]
        _ref = L
    return _ref


def ref_save_field_png(u, path, vmax):
    """The reference's save_field_png (gDiamond/utils.h:210-255) on a [ny][nx] float32 slice."""
    u = np.ascontiguousarray(u, np.float32)
    ny, nx = u.shape
    ref().gdref_save_field_png(_fptr(u), os.fsencode(path), nx, ny, float(vmax))


def _fptr(a: np.ndarray, T=C.c_float):
    return a.ctypes.data_as(C.POINTER(T))


def _ptr_array(arrs, T=C.c_float):
    arr = (C.POINTER(T) * len(arrs))()
    for n, a in enumerate(arrs):
        arr[n] = _fptr(a, T)
    return arr


# ----------------------------------------------------------------------------- helpers


def reference_params():
    """dict of the reference constructor's constants (gDiamond/gdiamond.hpp:893-906)."""
    out = (C.c_float * 7)()
    tp = C.c_int()
    lib().oracle_reference_params(out, C.byref(tp))
    keys = ("dx", "dt", "J_amp", "M_amp", "omega", "t_sigma", "t_peak")
    d = {k: float(np.float32(v)) for k, v in zip(keys, out)}
    d["t_pml"] = tp.value
    return d


def coefficients(shape, eps_re=None, eps_im=None, dx=None, dt=None, omega0=None, t_pml=None):
    """12 FP32 coefficient arrays (flat, x-fastest) for per-cell eps (None = vacuum)."""
    nx, ny, nz = shape
    p = reference_params()
    dx = p["dx"] if dx is None else dx
    dt = p["dt"] if dt is None else dt
    omega0 = p["omega"] if omega0 is None else omega0
    t_pml = p["t_pml"] if t_pml is None else t_pml
    n = nx * ny * nz
    out = [np.zeros(n, np.float32) for _ in range(12)]
    er = None if eps_re is None else np.ascontiguousarray(eps_re, np.float32).reshape(-1)
    ei = None if eps_im is None else np.ascontiguousarray(eps_im, np.float32).reshape(-1)
    lib().oracle_coefficients(nx, ny, nz, dx, dt, omega0, t_pml,
                              None if er is None else _fptr(er),
                              None if ei is None else _fptr(ei), _ptr_array(out))
    return out


def reference_mz_wave(T):
    out = np.zeros(T, np.float32)
    lib().oracle_reference_mz_wave(T, _fptr(out))
    return out


def dft_tables(freqs, dt, T, t_offset=0.0):
    """cos / sin of (2 pi f) * ((t + t_offset) * dt) for t < T (t_offset 1/2: a flux monitor's
    H fields)."""
    freqs = np.ascontiguousarray(freqs, np.float64)
    nf = len(freqs)
    ct = np.zeros((T, nf), np.float64)
    st = np.zeros((T, nf), np.float64)
    lib().oracle_dft_tables_offset(_fptr(freqs, C.c_double), nf, dt, float(t_offset), T,
                                   _fptr(ct, C.c_double), _fptr(st, C.c_double))
    return ct, st


@dataclass
class Source:
    component: str          # "Jx".."Mz"
    wave: np.ndarray        # FP32 samples, sample t used at step t
    i: int = 0
    j: int = 0
    k: int = 0
    kind: int = POINT       # POINT or PLANE_Z (every interior cell of plane k)


@dataclass
class Monitor:
    component: str          # "Ex".."Hz"
    k: int                  # z-plane index
    freqs: np.ndarray       # FP64 frequencies
    scale: float = 1.0
    re: np.ndarray = field(default=None)
    im: np.ndarray = field(default=None)
    t_offset: float = 0.0   # step t phased at (t + t_offset) dt


def flux_monitors(k, freqs):
    """The six running DFTs of a Poynting-flux monitor on the E plane z = k: Ex(k), Ey(k),
    Hx(k-1), Hx(k), Hy(k-1), Hy(k), the H ones phased half a step later."""
    return [Monitor("Ex", k, freqs), Monitor("Ey", k, freqs),
            Monitor("Hx", k - 1, freqs, t_offset=0.5), Monitor("Hx", k, freqs, t_offset=0.5),
            Monitor("Hy", k - 1, freqs, t_offset=0.5), Monitor("Hy", k, freqs, t_offset=0.5)]


def flux(mons, dx):
    """Flux spectrum from flux_monitors() after a run: per frequency
    dx^2 * sum over the plane of Re[Ex conj(Hy) - Ey conj(Hx)], H averaged over the two planes
    (k -+ 1/2 average to the E plane k); X = re + i im is the monitor's sum_t x(t) e^{-i w t'}.
    There is no reference counterpart (the reference keeps a per-cell DFT of Ex only,
    gDiamond/kernels.cuh:87-113); this is the definition the GPU reduction is checked against."""
    ex, ey, hx0, hx1, hy0, hy1 = [m.re + 1j * m.im for m in mons]
    hx, hy = 0.5 * (hx0 + hx1), 0.5 * (hy0 + hy1)
    s = np.real(ex * np.conj(hy) - ey * np.conj(hx))
    return float(dx) ** 2 * s.sum(axis=(1, 2))


def run(shape, coefs, T, sources=(), monitors=(), dx=None, dt=None, fields=None, t0=0,
        precision="f32"):
    """Run T Yee steps from global step t0 on the CPU oracle.

    Returns the 6 field arrays (flat, x-fastest); each Monitor gets .re/.im ([nf, Ny, Nx]) filled.
    """
    nx, ny, nz = shape
    n = nx * ny * nz
    p = reference_params()
    dx = p["dx"] if dx is None else dx
    dt = p["dt"] if dt is None else dt
    T_ = np.float32 if precision == "f32" else np.float64
    CT = C.c_float if precision == "f32" else C.c_double
    if fields is None:
        F = [np.zeros(n, T_) for _ in range(6)]
    else:
        F = [np.ascontiguousarray(f, T_).reshape(-1).copy() for f in fields]
    Cs = [np.ascontiguousarray(c, np.float32).reshape(-1) for c in coefs]
    nsrc = len(sources)
    Tw = max([len(s.wave) for s in sources] + [1])
    waves = np.zeros((max(nsrc, 1), Tw), np.float32)
    src_arr = (_Source * max(nsrc, 1))()
    for s_i, s in enumerate(sources):
        waves[s_i, :len(s.wave)] = s.wave
        src_arr[s_i] = _Source(SRC_COMPONENTS.index(s.component), s.kind, s.i, s.j, s.k)
    keep = []
    mon_arr = (_Monitor * max(len(monitors), 1))()
    for m_i, m in enumerate(monitors):
        freqs = np.asarray(m.freqs, np.float64)
        ct, st = dft_tables(freqs, float(np.float32(dt)), t0 + T, m.t_offset)
        if m.re is None:
            m.re = np.zeros((len(freqs), ny, nx), np.float64)
            m.im = np.zeros((len(freqs), ny, nx), np.float64)
        keep += [ct, st]
        mon_arr[m_i] = _Monitor(COMPONENTS.index(m.component), len(freqs), m.k, m.scale,
                                _fptr(ct, C.c_double), _fptr(st, C.c_double),
                                _fptr(m.re, C.c_double), _fptr(m.im, C.c_double))
    fn = lib().oracle_run_f32 if precision == "f32" else lib().oracle_run_f64
    fn(nx, ny, nz, _ptr_array(F, CT), _ptr_array(Cs), dx, src_arr, nsrc, _fptr(waves), Tw,
       t0, T, mon_arr, len(monitors))
    return F


# ------------------------------------------------------------- the reference's own class


class Reference:
    """The reference gDiamond object (its constructor, seq / omp / omp_dt solvers)."""

    def __init__(self, nx, ny, nz):
        self.shape = (nx, ny, nz)
        self.h = ref().gdref_create(nx, ny, nz)

    def close(self):
        if self.h:
            ref().gdref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n(self):
        nx, ny, nz = self.shape
        return nx * ny * nz

    def coefficients(self):
        out = [np.zeros(self.n, np.float32) for _ in range(12)]
        ref().gdref_get_coefficients(self.h, _ptr_array(out))
        return out

    def source_idx(self):
        return ref().gdref_source_idx(self.h)

    def params(self):
        out = (C.c_float * 7)()
        ref().gdref_params(self.h, out)
        keys = ("dx", "dt", "J_amp", "M_amp", "omega", "t_sigma", "t_peak")
        return {k: float(np.float32(v)) for k, v in zip(keys, out)}

    def run_seq(self, T):
        return ref().gdref_run_seq(self.h, T)

    def run_omp(self, T):
        return ref().gdref_run_omp(self.h, T)

    def run_omp_dt(self, blx, bly, blz, blt, T):
        return ref().gdref_run_omp_dt(self.h, blx, bly, blz, blt, T)

    @staticmethod
    def last_printed_seconds():
        """The time the reference printed for its own loop in the last run (-1: none)."""
        return ref().gdref_last_printed_seconds()

    def fields(self, variant="seq"):
        v = {"seq": 0, "omp": 1, "omp_dt": 2}[variant]
        out = [np.zeros(self.n, np.float32) for _ in range(6)]
        rc = ref().gdref_get_fields(self.h, v, _ptr_array(out))
        if rc != 0:
            raise RuntimeError(f"gdref_get_fields({variant}) failed: {rc}")
        return out
