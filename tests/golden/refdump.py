"""Reader for the tagged binary records written by oracle/ref_dump.cpp."""
import struct

import numpy as np

_DT = {0: np.float64, 1: np.int32, 2: np.int64}


def read_dump(path):
    out = {}
    with open(path, "rb") as f:
        if f.read(4) != b"TDBD":
            raise ValueError(f"{path}: not a reference dump")
        while True:
            h = f.read(4)
            if len(h) < 4:
                break
            (n,) = struct.unpack("<I", h)
            name = f.read(n).decode()
            (dt,) = struct.unpack("<B", f.read(1))
            (nd,) = struct.unpack("<I", f.read(4))
            dims = struct.unpack(f"<{nd}Q", f.read(8 * nd))
            count = int(np.prod(dims)) if nd else 1
            dtype = _DT[dt]
            arr = np.frombuffer(f.read(count * np.dtype(dtype).itemsize), dtype=dtype).reshape(dims)
            out[name] = arr.copy()
    return out
