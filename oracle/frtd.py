"""ORACLE TEST INFRASTRUCTURE -- reader for the FRTD state dumps (layout in oracle/frtd.h)."""
from __future__ import annotations

import struct
from typing import Dict

import numpy as np

_DT = {0: np.float32, 1: np.float64, 2: np.int32, 3: np.int64, 4: np.uint8, 5: np.int16, 6: np.uint16}


def read(path: str) -> Dict[str, np.ndarray]:
    out: Dict[str, np.ndarray] = {}
    with open(path, "rb") as f:
        if f.read(4) != b"FRTD":
            raise ValueError(f"{path}: not an FRTD file")
        _version, count = struct.unpack("<ii", f.read(8))
        for _ in range(count):
            name = f.read(32).split(b"\0", 1)[0].decode()
            dtype, ndim = struct.unpack("<ii", f.read(8))
            dims = struct.unpack("<4q", f.read(32))[:ndim]
            dt = np.dtype(_DT[dtype])
            n = int(np.prod(dims)) if ndim else 1
            arr = np.frombuffer(f.read(n * dt.itemsize), dtype=dt).reshape(dims)
            out[name] = arr.copy()
    return out
