"""Field snapshots: a z-plane of one component as an array or a PNG image.

The image follows the reference's save_field_png (gDiamond/utils.h:210-255): width Nx, height
Ny (row j of the image is y = j), value / vmax clipped to [-1, 1], white at zero, towards red
(255, 255(1-v), 255(1-v)) for positive and towards blue (255(1+v), 255(1+v), 255) for
negative values, channels truncated to 8 bits.  The reference writes the file with
stb_image_write; here a small PNG encoder (8-bit RGB, zlib from the standard library) writes
the same pixels.  The plane is converted and sliced on the GPU; only Nx*Ny values cross to the
host.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

from . import COMPONENTS


def plane(sim, component="Ez", k=None):
    """z-plane k (default Nz/2) of a component of the current field set: float32 [ny][nx].

    Only that plane is copied out of the grid (raw storage values, Nx*Ny of them); 16-bit
    values are widened and multiplied by their power-of-two storage scale, which is exact."""
    import torch
    nx, ny, nz = sim.shape
    k = nz // 2 if k is None else int(k)
    if not 0 <= k < nz:
        raise ValueError(f"plane {k} outside 0..{nz - 1}")
    comp = COMPONENTS.index(component) if isinstance(component, str) else int(component)
    esz = sim.component_bytes(comp)
    dtype = {4: torch.float32, 8: torch.float64}.get(esz)
    if dtype is None:
        dtype = torch.bfloat16 if sim.storage == "bf16" else torch.float16
    raw = torch.empty((ny, nx), dtype=dtype, device=f"cuda:{sim._device}")
    sim.get_planes_device(comp, k, 1, raw.data_ptr())
    sim.sync()
    out = raw.float()
    if esz == 2:
        out = out * sim.storage_scale[comp]
    return out.cpu().numpy()


def diverging_rgb(u, vmax):
    """uint8 [ny][nx][3] image of a [ny][nx] slice, the reference's colour map."""
    u = np.asarray(u, np.float32)
    v = u / np.float32(vmax)
    pos = v >= 0
    v = np.clip(v, np.float32(-1), np.float32(1))
    fade_pos = (np.float32(255) * (np.float32(1) - v)).astype(np.uint8)  # positive branch
    fade_neg = (np.float32(255) * (np.float32(1) + v)).astype(np.uint8)  # negative branch
    full = np.uint8(255)
    rgb = np.empty(u.shape + (3,), np.uint8)
    rgb[..., 0] = np.where(pos, full, fade_neg)
    rgb[..., 1] = np.where(pos, fade_pos, fade_neg)
    rgb[..., 2] = np.where(pos, fade_pos, full)
    return rgb


def _chunk(tag, data):
    return (struct.pack(">I", len(data)) + tag + data +
            struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF))


def encode_png(rgb):
    """PNG bytes of a uint8 [h][w][3] image (filter 0 on every row)."""
    rgb = np.ascontiguousarray(rgb, np.uint8)
    h, w, ch = rgb.shape
    if ch != 3:
        raise ValueError("RGB image expected")
    raw = np.concatenate([np.zeros((h, 1), np.uint8), rgb.reshape(h, w * 3)], axis=1)
    return (b"\x89PNG\r\n\x1a\n" +
            _chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)) +
            _chunk(b"IDAT", zlib.compress(raw.tobytes(), 6)) +
            _chunk(b"IEND", b""))


def save_field_png(sim, path, component="Ez", k=None, vmax=None):
    """Writes z-plane k of a component as a PNG (vmax: colour scale; default the plane's
    largest magnitude).  Returns the float32 plane."""
    u = plane(sim, component, k)
    if vmax is None:
        vmax = float(np.abs(u).max()) or 1.0
    with open(path, "wb") as f:
        f.write(encode_png(diverging_rgb(u, vmax)))
    return u
