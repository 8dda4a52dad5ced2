"""gdiamond_b200 -- B200-native 3D FDTD (Yee) solver.

Python binding of the C-ABI in ``include/fdtd_capi.h`` (``libgdiamond_b200.so``, built
in-tree by ``python -m gdiamond_b200.build``).  Every step runs a CUDA kernel through the
C-ABI; there is no CPU path here, and importing the binding fails loudly when the library
is missing.

Reference surface mirrored: gdiamond::gDiamond (gDiamond/gdiamond.hpp:17-907) -- a grid of
Nx x Ny x Nz cells with 12 per-cell coefficient arrays, J/M current sources and
``update_FDTD_gpu*(num_timesteps)``; results read back per field component.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgdiamond_b200.so")

COMPONENTS = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")
SOURCE_COMPONENTS = ("Jx", "Jy", "Jz", "Mx", "My", "Mz")
COEFFS = ("Cax", "Cay", "Caz", "Cbx", "Cby", "Cbz", "Dax", "Day", "Daz", "Dbx", "Dby", "Dbz")
KERNELS = {"auto": 0, "naive": 1, "tiled": 2, "tiled_w32": 3, "tiled_w64": 4, "tiled_w32p": 5}
STORAGE = {"f32": 0, "f16": 1, "bf16": 2, "f64": 3, "f16e": 4}  # f16e: FP16 E, FP32 H
SRC_POINT, SRC_PLANE_Z = 0, 1

# Every symbol declared in include/fdtd_capi.h.
EXPORTS = (
    "fdtd_version", "fdtd_status_string", "fdtd_last_error", "fdtd_create", "fdtd_destroy",
    "fdtd_set_coefficients", "fdtd_set_coefficients_device", "fdtd_material_count",
    "fdtd_set_sources", "fdtd_add_dft_monitor", "fdtd_reset", "fdtd_step", "fdtd_sync",
    "fdtd_get_step", "fdtd_get_field", "fdtd_set_field", "fdtd_get_dft",
    "fdtd_get_field_device", "fdtd_set_storage_scale", "fdtd_get_config",
    "fdtd_build_material_map_noalloc", "fdtd_get_field_f64",
    "fdtd_batch_create", "fdtd_batch_destroy", "fdtd_batch_step", "fdtd_batch_get_config",
    "fdtd_batch_last_error", "fdtd_set_permittivity", "fdtd_get_coefficients",
    "fdtd_mlp_create", "fdtd_mlp_destroy", "fdtd_mlp_last_error", "fdtd_mlp_layout",
    "fdtd_mlp_get_params", "fdtd_mlp_set_params", "fdtd_mlp_set_data", "fdtd_mlp_grad",
    "fdtd_mlp_train", "fdtd_mlp_predict", "fdtd_mlp_predict_device", "fdtd_get_dft_device",
    "fdtd_mlp_set_gemm", "fdtd_get_planes_device", "fdtd_set_planes_device",
    "fdtd_storage_bytes", "fdtd_set_step", "fdtd_set_dft", "fdtd_component_bytes",
    "fdtd_dft_folds", "fdtd_set_fast_path", "fdtd_fast_path", "fdtd_add_flux_monitor",
    "fdtd_get_flux", "fdtd_get_flux_device", "fdtd_flux_monitor_ids", "fdtd_debug_fail_copy",
    "fdtd_set_cpml", "fdtd_get_cpml_profile", "fdtd_cpml_psi_bytes", "fdtd_get_cpml_psi",
    "fdtd_set_cpml_psi",
)


class FdtdError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{msg} (status {status})")
        self.status = status


class _Desc(C.Structure):
    _fields_ = [("nx", C.c_int64), ("ny", C.c_int64), ("nz", C.c_int64), ("dx", C.c_float),
                ("device", C.c_int32), ("storage", C.c_int32), ("kernel", C.c_int32),
                ("blt", C.c_int32), ("tile_rows", C.c_int32), ("z_chunks", C.c_int32),
                ("min_blocks", C.c_int32)]


class _Cpml(C.Structure):
    _fields_ = [("thickness", C.c_int32), ("faces", C.c_int32), ("order", C.c_float),
                ("reflection", C.c_float), ("kappa_max", C.c_float), ("alpha_max", C.c_float),
                ("dt", C.c_float)]


class _Source(C.Structure):
    _fields_ = [("component", C.c_int32), ("kind", C.c_int32),
                ("i", C.c_int64), ("j", C.c_int64), ("k", C.c_int64)]


_lib = None


def library():
    """The loaded C-ABI library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m gdiamond_b200.build`")
        L = C.CDLL(LIB_PATH)
        P, V = C.POINTER, C.c_void_p
        sig = {
            "fdtd_version": ([], C.c_char_p),
            "fdtd_status_string": ([C.c_int], C.c_char_p),
            "fdtd_last_error": ([V], C.c_char_p),
            "fdtd_create": ([P(_Desc), P(V)], C.c_int),
            "fdtd_destroy": ([V], C.c_int),
            "fdtd_set_coefficients": ([V, P(P(C.c_float))], C.c_int),
            "fdtd_set_coefficients_device": ([V, P(V)], C.c_int),
            "fdtd_material_count": ([V, P(C.c_int32)], C.c_int),
            "fdtd_set_sources": ([V, P(_Source), C.c_int32, P(C.c_float), C.c_int64], C.c_int),
            "fdtd_add_dft_monitor": ([V, C.c_int32, C.c_int64, P(C.c_double), C.c_int32,
                                      C.c_double, C.c_double, P(C.c_int32)], C.c_int),
            "fdtd_reset": ([V], C.c_int),
            "fdtd_step": ([V, C.c_int64, V], C.c_int),
            "fdtd_sync": ([V], C.c_int),
            "fdtd_get_step": ([V, P(C.c_int64)], C.c_int),
            "fdtd_get_field": ([V, C.c_int32, P(C.c_float)], C.c_int),
            "fdtd_set_field": ([V, C.c_int32, P(C.c_float)], C.c_int),
            "fdtd_get_dft": ([V, C.c_int32, P(C.c_double), P(C.c_double)], C.c_int),
            "fdtd_get_field_device": ([V, C.c_int32, V, V], C.c_int),
            "fdtd_set_storage_scale": ([V, P(C.c_float)], C.c_int),
            "fdtd_get_config": ([V, P(C.c_int32)], C.c_int),
            "fdtd_get_field_f64": ([V, C.c_int32, P(C.c_double)], C.c_int),
            "fdtd_get_dft_device": ([V, C.c_int32, V, V, V], C.c_int),
            "fdtd_get_planes_device": ([V, C.c_int32, C.c_int64, C.c_int64, V, V], C.c_int),
            "fdtd_set_planes_device": ([V, C.c_int32, C.c_int64, C.c_int64, V, V], C.c_int),
            "fdtd_storage_bytes": ([V, P(C.c_int32)], C.c_int),
            "fdtd_component_bytes": ([V, C.c_int32, P(C.c_int32)], C.c_int),
            "fdtd_dft_folds": ([V, P(C.c_int32)], C.c_int),
            "fdtd_set_fast_path": ([V, C.c_int32], C.c_int),
            "fdtd_set_cpml": ([V, P(_Cpml)], C.c_int),
            "fdtd_cpml_psi_bytes": ([V, C.c_int32, P(C.c_int64)], C.c_int),
            "fdtd_get_cpml_psi": ([V, C.c_int32, V], C.c_int),
            "fdtd_set_cpml_psi": ([V, C.c_int32, V], C.c_int),
            "fdtd_get_cpml_profile": ([V, C.c_int32, C.c_int32, P(C.c_float), P(C.c_float),
                                       P(C.c_float), P(C.c_int32)], C.c_int),
            "fdtd_debug_fail_copy": ([V, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int64],
                                     C.c_int),
            "fdtd_add_flux_monitor": ([V, C.c_int64, P(C.c_double), C.c_int32, C.c_double,
                                       P(C.c_int32)], C.c_int),
            "fdtd_get_flux": ([V, C.c_int32, P(C.c_double)], C.c_int),
            "fdtd_get_flux_device": ([V, C.c_int32, V, V], C.c_int),
            "fdtd_flux_monitor_ids": ([V, C.c_int32, P(C.c_int32)], C.c_int),
            "fdtd_fast_path": ([V, P(C.c_int32)], C.c_int),
            "fdtd_set_step": ([V, C.c_int64], C.c_int),
            "fdtd_set_dft": ([V, C.c_int32, P(C.c_double), P(C.c_double)], C.c_int),
            "fdtd_batch_create": ([P(V), C.c_int32, P(V)], C.c_int),
            "fdtd_batch_destroy": ([V], C.c_int),
            "fdtd_batch_step": ([V, C.c_int64, C.c_int32, V], C.c_int),
            "fdtd_batch_get_config": ([V, P(C.c_int32)], C.c_int),
            "fdtd_batch_last_error": ([V], C.c_char_p),
            "fdtd_set_permittivity": ([V, P(C.c_float), C.c_int32, C.c_float, C.c_float], C.c_int),
            "fdtd_get_coefficients": ([V, P(P(C.c_float))], C.c_int),
            "fdtd_mlp_create": ([P(C.c_int32), C.c_int32, C.c_int32, C.c_uint64, C.c_int32,
                                 P(V)], C.c_int),
            "fdtd_mlp_destroy": ([V], C.c_int),
            "fdtd_mlp_last_error": ([V], C.c_char_p),
            "fdtd_mlp_layout": ([V, P(C.c_int64), P(C.c_int64), P(C.c_int64)], C.c_int),
            "fdtd_mlp_get_params": ([V, P(C.c_float)], C.c_int),
            "fdtd_mlp_set_params": ([V, P(C.c_float)], C.c_int),
            "fdtd_mlp_set_data": ([V, P(C.c_float), P(C.c_float), C.c_int64], C.c_int),
            "fdtd_mlp_grad": ([V, P(C.c_float), P(C.c_float), C.c_int64, P(C.c_float),
                               P(C.c_float)], C.c_int),
            "fdtd_mlp_train": ([V, C.c_int32, C.c_int32, C.c_float, C.c_uint64, P(C.c_float)],
                               C.c_int),
            "fdtd_mlp_predict": ([V, P(C.c_float), C.c_int64, P(C.c_float), P(C.c_float),
                                  P(C.c_float)], C.c_int),
            "fdtd_mlp_predict_device": ([V, V, C.c_int64, V, V, V], C.c_int),
            "fdtd_mlp_set_gemm": ([V, C.c_int32], C.c_int),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _fp(a, T=C.c_float):
    return a.ctypes.data_as(C.POINTER(T))


def _stream(stream):
    """A torch.cuda.Stream, an int handle or None as a cudaStream_t argument."""
    if stream is None:
        return None
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


class Simulation:
    """One FDTD grid resident on a GPU (a handle of the C-ABI).

    Parameters mirror the reference constructor ``gDiamond(Nx, Ny, Nz)``; ``dx`` is the
    spacing used in the -J*dx / -M*dx source terms (reference default 0.1,
    gDiamond/gdiamond.hpp:899).
    """

    def __init__(self, nx, ny, nz, dx=np.float32(0.1), device=0, kernel="auto", blt=0,
                 tile_rows=0, z_chunks=0, storage="f32", min_blocks=0):
        self.shape = (int(nx), int(ny), int(nz))
        self._L = library()
        d = _Desc(nx, ny, nz, float(np.float32(dx)), device, STORAGE[storage], KERNELS[kernel],
                  blt, tile_rows, z_chunks, min_blocks)
        h = C.c_void_p()
        st = self._L.fdtd_create(C.byref(d), C.byref(h))
        if st != 0:
            raise FdtdError(st, self._L.fdtd_last_error(None).decode())
        self._h = h
        self._device = int(device)
        self.storage = storage
        self.storage_scale = [1.0] * 6  # value = stored * scale (16-bit components)
        self._keep = []
        self.n_monitors = 0
        self._monitor_nf = []
        self._flux_nf = []

    # ---------------------------------------------------------------- plumbing
    def _check(self, st):
        if st != 0:
            raise FdtdError(st, self._L.fdtd_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            self._L.fdtd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def ncells(self):
        nx, ny, nz = self.shape
        return nx * ny * nz

    # ---------------------------------------------------------------- set-up
    def set_coefficients(self, coefs):
        """12 arrays (Cax..Dbz) of Nx*Ny*Nz float32, host numpy or device torch tensors."""
        if len(coefs) != 12:
            raise ValueError("need 12 coefficient arrays")
        if hasattr(coefs[0], "data_ptr"):  # device tensors
            arr = (C.c_void_p * 12)(*[int(c.data_ptr()) for c in coefs])
            self._check(self._L.fdtd_set_coefficients_device(self._h, arr))
            return
        cs = [np.ascontiguousarray(c, np.float32).reshape(-1) for c in coefs]
        for c in cs:
            if c.size != self.ncells:
                raise ValueError("coefficient array size mismatch")
        arr = (C.POINTER(C.c_float) * 12)(*[_fp(c) for c in cs])
        self._check(self._L.fdtd_set_coefficients(self._h, arr))

    def set_permittivity(self, eps_re=None, t_pml=10, dt=np.float32(0.05),
                         omega0=np.float32(2) * np.float32(3.14159265359)):
        """gDiamond's constructor coefficients (graded pseudo-PML) for a per-cell relative
        permittivity (None = vacuum), computed on the GPU."""
        e = None
        if eps_re is not None:
            e = np.ascontiguousarray(eps_re, np.float32).reshape(-1)
            if e.size != self.ncells:
                raise ValueError("permittivity size mismatch")
            self._keep_eps = e
        self._check(self._L.fdtd_set_permittivity(self._h, None if e is None else _fp(e),
                                                   int(t_pml), float(np.float32(dt)),
                                                   float(np.float32(omega0))))

    def get_coefficients(self):
        out = [np.empty(self.ncells, np.float32) for _ in range(12)]
        arr = (C.POINTER(C.c_float) * 12)(*[_fp(c) for c in out])
        self._check(self._L.fdtd_get_coefficients(self._h, arr))
        return out

    def material_count(self):
        n = C.c_int32()
        self._check(self._L.fdtd_material_count(self._h, C.byref(n)))
        return n.value

    def set_sources(self, sources):
        """sources: iterable of dicts {component: "Jz", wave: float32[T], i, j, k, kind}."""
        sources = list(sources)
        n = len(sources)
        arr = (_Source * max(n, 1))()
        tw = max([len(s["wave"]) for s in sources] + [1])
        waves = np.zeros((max(n, 1), tw), np.float32)
        for q, s in enumerate(sources):
            comp = s["component"]
            comp = SOURCE_COMPONENTS.index(comp) if isinstance(comp, str) else int(comp)
            arr[q] = _Source(comp, s.get("kind", SRC_POINT), s.get("i", 0), s.get("j", 0), s["k"])
            waves[q, :len(s["wave"])] = s["wave"]
        self._keep = [arr, waves]
        self._check(self._L.fdtd_set_sources(self._h, arr, n, _fp(waves), tw))

    def add_dft_monitor(self, component, k, freqs, scale=1.0, dt=np.float32(0.05)):
        comp = COMPONENTS.index(component) if isinstance(component, str) else int(component)
        f = np.ascontiguousarray(freqs, np.float64)
        mid = C.c_int32()
        self._check(self._L.fdtd_add_dft_monitor(self._h, comp, k, _fp(f, C.c_double), len(f),
                                                  float(scale), float(np.float32(dt)),
                                                  C.byref(mid)))
        self.n_monitors += 1
        self._monitor_nf.append(len(f))
        return mid.value

    def add_flux_monitor(self, k, freqs, dt=np.float32(0.05)):
        """Poynting flux through the E plane z = k at each frequency (fdtd_add_flux_monitor):
        six running DFTs (Ex, Ey at k; Hx, Hy at k-1 and k, phased half a step later)."""
        f = np.ascontiguousarray(freqs, np.float64)
        fid = C.c_int32()
        self._check(self._L.fdtd_add_flux_monitor(self._h, int(k), _fp(f, C.c_double), len(f),
                                                   float(np.float32(dt)), C.byref(fid)))
        self.n_monitors += 6
        self._monitor_nf += [len(f)] * 6
        self._flux_nf.append(len(f))
        return fid.value

    def get_flux(self, flux_id):
        out = np.empty(self._flux_nf[flux_id], np.float64)
        self._check(self._L.fdtd_get_flux(self._h, int(flux_id), _fp(out, C.c_double)))
        return out

    def get_flux_device(self, flux_id, out_ptr, stream=None):
        self._check(self._L.fdtd_get_flux_device(self._h, int(flux_id), C.c_void_p(out_ptr),
                                                  _stream(stream)))

    def flux_monitor_ids(self, flux_id):
        """Monitor ids of Ex(k), Ey(k), Hx(k-1), Hx(k), Hy(k-1), Hy(k)."""
        ids = (C.c_int32 * 6)()
        self._check(self._L.fdtd_flux_monitor_ids(self._h, int(flux_id), ids))
        return list(ids)

    # ---------------------------------------------------------------- running
    def reset(self):
        self._check(self._L.fdtd_reset(self._h))

    def step(self, T, stream=None):
        """Run T steps asynchronously on `stream` (a torch.cuda.Stream, an int handle or None)."""
        s = None
        if stream is not None:
            s = C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        self._check(self._L.fdtd_step(self._h, int(T), s))

    def sync(self):
        self._check(self._L.fdtd_sync(self._h))

    @property
    def t(self):
        v = C.c_int64()
        self._check(self._L.fdtd_get_step(self._h, C.byref(v)))
        return v.value

    def config(self):
        out = (C.c_int32 * 6)()
        self._check(self._L.fdtd_get_config(self._h, out))
        kernel = {1: "naive", 3: "tiled", 4: "tiled", 5: "tiled", 6: "cpml"}.get(out[0], "none")
        width = {3: 32, 4: 64, 5: 32}.get(out[0], 0)
        folds = C.c_int32()
        self._check(self._L.fdtd_dft_folds(self._h, C.byref(folds)))
        return {"kernel": kernel, "width": width, "pairs": out[0] in (4, 5), "blt": out[1],
                "tile_rows": out[2], "z_chunks": out[3], "launches": out[4],
                "min_blocks": out[5], "dft_folds": folds.value}

    def set_fast_path(self, enable):
        """Uniform-material fast path of the tiled x-pair kernels (on by default); off forces
        the general per-cell path, which gives the same bits."""
        self._check(self._L.fdtd_set_fast_path(self._h, 1 if enable else 0))

    def set_cpml(self, thickness=10, faces=63, order=3.0, reflection=1e-6, kappa_max=1.0,
                 alpha_max=0.05, dt=np.float32(0.05)):
        """CPML absorbing layers (fdtd_set_cpml); thickness=None turns them off."""
        if thickness is None:
            self._check(self._L.fdtd_set_cpml(self._h, None))
            return
        d = _Cpml(int(thickness), int(faces), float(order), float(reflection), float(kappa_max),
                  float(alpha_max), float(np.float32(dt)))
        self._check(self._L.fdtd_set_cpml(self._h, C.byref(d)))

    def cpml_state(self):
        """The twelve CPML psi arrays (float32, flat; None without layers)."""
        out = []
        for q in range(12):
            n = C.c_int64()
            if self._L.fdtd_cpml_psi_bytes(self._h, q, C.byref(n)) != 0:
                return None
            a = np.empty(n.value // 4, np.float32)
            self._check(self._L.fdtd_get_cpml_psi(self._h, q, a.ctypes.data_as(C.c_void_p)))
            out.append(a)
        return out

    def set_cpml_state(self, psi):
        for q, a in enumerate(psi):
            a = np.ascontiguousarray(a, np.float32)
            n = C.c_int64()
            self._check(self._L.fdtd_cpml_psi_bytes(self._h, q, C.byref(n)))
            if a.nbytes != n.value:
                raise ValueError("CPML state of other layers")
            self._check(self._L.fdtd_set_cpml_psi(self._h, q, a.ctypes.data_as(C.c_void_p)))

    def cpml_tables(self):
        """[axis][kind] = (slot, b, a, inv_kappa) of the layers (kind 0: E positions, 1: H)."""
        out = []
        for axis, n in enumerate(self.shape):
            row = []
            for kind in (0, 1):
                b, a, ik = (np.empty(n, np.float32) for _ in range(3))
                slot = np.empty(n, np.int32)
                self._check(self._L.fdtd_get_cpml_profile(self._h, axis, kind, _fp(b), _fp(a),
                                                           _fp(ik), _fp(slot, C.c_int32)))
                row.append((slot, b, a, ik))
            out.append(row)
        return out

    def debug_fail_copy(self, tile, iteration, wait_cycles):
        """Failure-path test hook (fdtd_debug_fail_copy): in the next tiled launch, tile
        (bx, by, bz) skips the copy of one z-iteration and waits at most wait_cycles."""
        bx, by, bz = (int(v) for v in tile)
        self._check(self._L.fdtd_debug_fail_copy(self._h, bx, by, bz, int(iteration),
                                                  int(wait_cycles)))

    @property
    def fast_path(self):
        v = C.c_int32()
        self._check(self._L.fdtd_fast_path(self._h, C.byref(v)))
        return bool(v.value)

    # ---------------------------------------------------------------- results
    def get_field(self, component, out=None):
        comp = COMPONENTS.index(component) if isinstance(component, str) else int(component)
        if out is None:
            out = np.empty(self.ncells, np.float32)
        self._check(self._L.fdtd_get_field(self._h, comp, _fp(out)))
        return out

    def fields(self):
        return [self.get_field(c) for c in range(6)]

    def get_field_f64(self, component, out=None):
        comp = COMPONENTS.index(component) if isinstance(component, str) else int(component)
        if out is None:
            out = np.empty(self.ncells, np.float64)
        self._check(self._L.fdtd_get_field_f64(self._h, comp, _fp(out, C.c_double)))
        return out

    def set_storage_scale(self, scale6):
        s = (C.c_float * 6)(*[float(v) for v in scale6])
        self._check(self._L.fdtd_set_storage_scale(self._h, s))
        # the library keeps the nearest power of two of each (16-bit components only)
        def p2(v):  # lround(log2 v): halves away from zero, as the library rounds
            e = float(np.log2(float(v)))
            return float(2.0 ** (np.floor(e + 0.5) if e >= 0 else -np.floor(-e + 0.5)))
        self.storage_scale = [p2(v) if self.component_bytes(c) == 2 else 1.0
                              for c, v in enumerate(scale6)]

    def set_field(self, component, values):
        comp = COMPONENTS.index(component) if isinstance(component, str) else int(component)
        v = np.ascontiguousarray(values, np.float32).reshape(-1)
        if v.size != self.ncells:
            raise ValueError("field size mismatch")
        self._check(self._L.fdtd_set_field(self._h, comp, _fp(v)))

    def get_field_device(self, component, out_ptr, stream=None):
        comp = COMPONENTS.index(component) if isinstance(component, str) else int(component)
        s = None
        if stream is not None:
            s = C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        self._check(self._L.fdtd_get_field_device(self._h, comp, C.c_void_p(out_ptr), s))

    def get_dft(self, monitor_id):
        nx, ny, _ = self.shape
        nf = self._monitor_nf[monitor_id]
        re = np.empty((nf, ny, nx), np.float64)
        im = np.empty((nf, ny, nx), np.float64)
        self._check(self._L.fdtd_get_dft(self._h, monitor_id, _fp(re, C.c_double),
                                          _fp(im, C.c_double)))
        return re, im

    def storage_bytes(self):
        n = C.c_int32()
        self._check(self._L.fdtd_storage_bytes(self._h, C.byref(n)))
        return n.value

    def component_bytes(self, component):
        """Bytes per stored value of one component (differs between E and H for f16e)."""
        comp = COMPONENTS.index(component) if isinstance(component, str) else int(component)
        n = C.c_int32()
        self._check(self._L.fdtd_component_bytes(self._h, comp, C.byref(n)))
        return n.value

    def get_planes_device(self, component, k0, nk, ptr, stream=None):
        """Raw copy of z-planes [k0, k0+nk) of a component (current set) to a device buffer."""
        comp = COMPONENTS.index(component) if isinstance(component, str) else int(component)
        self._check(self._L.fdtd_get_planes_device(self._h, comp, int(k0), int(nk),
                                                    C.c_void_p(ptr), _stream(stream)))

    def set_planes_device(self, component, k0, nk, ptr, stream=None):
        """Raw copy of a device buffer into z-planes [k0, k0+nk) of a component (current set)."""
        comp = COMPONENTS.index(component) if isinstance(component, str) else int(component)
        self._check(self._L.fdtd_set_planes_device(self._h, comp, int(k0), int(nk),
                                                    C.c_void_p(ptr), _stream(stream)))

    def set_dft(self, monitor_id, re, im):
        re = np.ascontiguousarray(re, np.float64)
        im = np.ascontiguousarray(im, np.float64)
        nx, ny, _ = self.shape
        if re.size != self._monitor_nf[monitor_id] * nx * ny or im.size != re.size:
            raise ValueError("DFT sums of the wrong size")
        self._check(self._L.fdtd_set_dft(self._h, int(monitor_id), _fp(re, C.c_double),
                                          _fp(im, C.c_double)))

    def checkpoint(self):
        """The whole state as host arrays: step counter, the current field set in its storage
        format (raw), every monitor's sums, the CPML psi arrays when layers are on.  restore() on a handle with the same shape,
        storage, sources and monitors continues bit for bit."""
        import torch
        self.sync()
        nx, ny, nz = self.shape
        esz = [self.component_bytes(c) for c in range(6)]
        dev = torch.device("cuda", self._device)
        fields = []
        for c in range(6):
            raw = {2: torch.int16, 4: torch.int32, 8: torch.int64}[esz[c]]
            buf = torch.empty((nz, ny, nx), dtype=raw, device=dev)
            self.get_planes_device(c, 0, nz, buf.data_ptr())
            self.sync()
            fields.append(buf.cpu().numpy().copy())
        return {"t": self.t, "shape": self.shape, "esz": esz, "fields": fields,
                "dft": [self.get_dft(m) for m in range(self.n_monitors)],
                "cpml_psi": self.cpml_state()}

    def restore(self, ckpt):
        import torch
        if (tuple(ckpt["shape"]) != self.shape
                or list(ckpt["esz"]) != [self.component_bytes(c) for c in range(6)]):
            raise ValueError("checkpoint of another shape or storage")
        if len(ckpt["dft"]) != self.n_monitors:
            raise ValueError("checkpoint with another set of monitors")
        psi = ckpt.get("cpml_psi")
        if (psi is None) != (self.cpml_state() is None):
            raise ValueError("checkpoint and handle differ in CPML layers")
        nz = self.shape[2]
        self.sync()
        for c, f in enumerate(ckpt["fields"]):
            t = torch.from_numpy(np.ascontiguousarray(f)).to(torch.device("cuda", self._device))
            self.set_planes_device(c, 0, nz, t.data_ptr())
            self.sync()
        for m, (re, im) in enumerate(ckpt["dft"]):
            self.set_dft(m, re, im)
        if psi is not None:
            self.set_cpml_state(psi)
        self._check(self._L.fdtd_set_step(self._h, int(ckpt["t"])))

    def get_dft_device(self, monitor_id, re_ptr, im_ptr, stream=None):
        """Copy a monitor's running sums into device arrays (float64 [nf][ny][nx] pointers)."""
        s = None
        if stream is not None:
            s = C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        self._check(self._L.fdtd_get_dft_device(self._h, int(monitor_id), C.c_void_p(re_ptr),
                                                 C.c_void_p(im_ptr), s))


class Batch:
    """Independent simulations advanced together by persistent launches (fdtd_batch_*).

    All simulations must live on one device with one storage type and have their
    coefficients set (compressed to a material map).  Each keeps its own fields, sources,
    monitors and step counter; results are read from the Simulation objects as usual.
    """

    def __init__(self, sims):
        self.sims = list(sims)
        self._L = library()
        arr = (C.c_void_p * len(self.sims))(*[s._h.value for s in self.sims])
        h = C.c_void_p()
        st = self._L.fdtd_batch_create(arr, len(self.sims), C.byref(h))
        if st != 0:
            raise FdtdError(st, self._L.fdtd_batch_last_error(None).decode())
        self._h = h

    def _check(self, st):
        if st != 0:
            raise FdtdError(st, self._L.fdtd_batch_last_error(self._h).decode())

    def step(self, T, use_graph=True, stream=None):
        s = None
        if stream is not None:
            s = C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        self._check(self._L.fdtd_batch_step(self._h, int(T), 1 if use_graph else 0, s))

    def config(self):
        out = (C.c_int32 * 6)()
        self._check(self._L.fdtd_batch_get_config(self._h, out))
        folds = C.c_int32()
        self._check(self._L.fdtd_dft_folds(self.sims[0]._h, C.byref(folds)))
        return {"blt": out[0], "tile_rows": out[1], "ctas": out[2], "items": out[3],
                "launches": out[4], "graph_replayed": bool(out[5]), "dft_folds": folds.value}

    def close(self):
        if getattr(self, "_h", None):
            self._L.fdtd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MLP:
    """An ensemble of MLPs trained and evaluated on the GPU (fdtd_mlp_*).

    dims = (inputs, hidden..., outputs); GELU between layers; BF16 tensor-core GEMMs with FP32
    accumulation and FP32 master weights; Adam.  Parameters of all members as one array
    [members][n_params]; ``layout()`` gives each layer's weight and bias offsets.
    """

    GEMMS = {"tcgen05": 0, "mma_sync": 1, "auto": 2}

    def __init__(self, dims, members=4, seed=0, device=0, gemm="auto"):
        self.dims = tuple(int(d) for d in dims)
        self.members = int(members)
        self._L = library()
        d = (C.c_int32 * len(self.dims))(*self.dims)
        h = C.c_void_p()
        st = self._L.fdtd_mlp_create(d, len(self.dims), self.members, int(seed), int(device),
                                     C.byref(h))
        if st != 0:
            raise FdtdError(st, "fdtd_mlp_create failed")
        self._h = h
        n = C.c_int64()
        w = (C.c_int64 * (len(self.dims) - 1))()
        b = (C.c_int64 * (len(self.dims) - 1))()
        self._check(self._L.fdtd_mlp_layout(self._h, C.byref(n), w, b))
        self.n_params = n.value
        self.w_off, self.b_off = list(w), list(b)
        self.set_gemm(gemm)

    def set_gemm(self, gemm):
        """GEMM path: "tcgen05" (tensor-memory accumulator), "mma_sync" (warp-level) or "auto"
        (tcgen05 for products of >= 1024 rows, mma_sync for training minibatches)."""
        self._check(self._L.fdtd_mlp_set_gemm(self._h, self.GEMMS[gemm]))
        self.gemm = gemm

    def _check(self, st):
        if st != 0:
            raise FdtdError(st, self._L.fdtd_mlp_last_error(self._h).decode())

    def layout(self):
        """[(W offset, W shape (out, in), b offset)] per layer, within one member."""
        return [(self.w_off[l], (self.dims[l + 1], self.dims[l]), self.b_off[l])
                for l in range(len(self.dims) - 1)]

    def unpack(self, flat):
        """One member's flat parameters -> [(W, b)] per layer (views)."""
        return [(flat[w:w + o * i].reshape(o, i), flat[b:b + o])
                for w, (o, i), b in self.layout()]

    def get_params(self):
        out = np.empty((self.members, self.n_params), np.float32)
        self._check(self._L.fdtd_mlp_get_params(self._h, _fp(out)))
        return out

    def set_params(self, params):
        p = np.ascontiguousarray(params, np.float32).reshape(self.members, self.n_params)
        self._check(self._L.fdtd_mlp_set_params(self._h, _fp(p)))

    def set_data(self, x, y):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.dims[0])
        y = np.ascontiguousarray(y, np.float32).reshape(-1, self.dims[-1])
        if len(x) != len(y):
            raise ValueError("x and y differ in length")
        self._check(self._L.fdtd_mlp_set_data(self._h, _fp(x), _fp(y), len(x)))

    def grad(self, x, y):
        """(loss [members], grads [members][n_params]) of every member on one batch."""
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.dims[0])
        y = np.ascontiguousarray(y, np.float32).reshape(-1, self.dims[-1])
        loss = np.empty(self.members, np.float32)
        g = np.empty((self.members, self.n_params), np.float32)
        self._check(self._L.fdtd_mlp_grad(self._h, _fp(x), _fp(y), len(x), _fp(loss), _fp(g)))
        return loss, g

    def train(self, epochs, batch=256, lr=1e-3, seed=0):
        """Adam over the data of set_data(); returns the loss per epoch [epochs][members]."""
        loss = np.empty((int(epochs), self.members), np.float32)
        self._check(self._L.fdtd_mlp_train(self._h, int(epochs), int(batch), float(lr),
                                           int(seed), _fp(loss)))
        return loss

    def predict(self, x, members=False):
        """(mean, sd) over the ensemble, and every member's output when members=True."""
        x = np.ascontiguousarray(x, np.float32).reshape(-1, self.dims[0])
        n, o = len(x), self.dims[-1]
        mean = np.empty((n, o), np.float32)
        sd = np.empty((n, o), np.float32)
        per = np.empty((self.members, n, o), np.float32) if members else None
        self._check(self._L.fdtd_mlp_predict(self._h, _fp(x), n, _fp(mean), _fp(sd),
                                              None if per is None else _fp(per)))
        return (mean, sd, per) if members else (mean, sd)

    def predict_device(self, x_ptr, n, mean_ptr, sd_ptr, stream=None):
        """predict() on device buffers (float32 pointers) ordered on `stream`."""
        s = None
        if stream is not None:
            s = C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        self._check(self._L.fdtd_mlp_predict_device(self._h, C.c_void_p(x_ptr), int(n),
                                                     C.c_void_p(mean_ptr), C.c_void_p(sd_ptr), s))

    def close(self):
        if getattr(self, "_h", None):
            self._L.fdtd_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


from . import workloads  # noqa: E402,F401
