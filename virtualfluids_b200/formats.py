"""Host-side view of the E3M12 storage format (csrc/storage.cuh, Codec<e3m12_t>).

E3M12 stores the 1/w-scaled populations g = (f - w)/w in 16 bits: 1 sign, 3 exponent and 12
significand bits, exponent bias 7, no infinity and no NaN. Normal values (e = 1..7) are
(-1)^s 2^(e-7) (1 + m/4096), magnitudes in [2^-6, 2); subnormals (e = 0) are (-1)^s 2^-6 m/4096.
The bits are those of the float g 2^-120 shifted right by 11, so decoding is a shift and a
multiplication by 2^120; encoding adds r in [0, 2048) to the float's magnitude bits before the
shift (stochastic rounding when r is random, truncation when r = 0) and saturates at 2 - 2^-12.
These numpy functions restate the device codec for reading population arrays and restart files.
"""
from __future__ import annotations

import numpy as np

MAX = 2.0 - 2.0 ** -12


def decode(bits) -> np.ndarray:
    """g (float64) from E3M12 bit patterns (uint16 or int16 arrays)."""
    b = np.asarray(bits).astype(np.uint32) & 0xFFFF
    f = (((b & 0x8000) << 16) | ((b & 0x7FFF) << 11)).astype(np.uint32).view(np.float32)
    return f.astype(np.float64) * 2.0 ** 120


def encode(g, r=0) -> np.ndarray:
    """E3M12 bit patterns (uint16) of float32 values g; r: the added bits, scalar or array in
    [0, 2048) (0 truncates toward zero)."""
    t = (np.asarray(g, dtype=np.float32) * np.float32(2.0 ** -120)).astype(np.float32)
    b = t.view(np.uint32).astype(np.uint64)
    mag = np.minimum(((b & 0x7FFFFFFF) + np.asarray(r, dtype=np.uint64)) >> 11, 0x7FFF)
    return (((b >> 16) & 0x8000) | mag).astype(np.uint16)
