"""Reader/writer for the CPBIN01 record container (see oracle/cpbin.h).

TEST INFRASTRUCTURE ONLY: used by tests/, the golden-fixture script and the
CPU-baseline leg of bench.py to talk to the oracle programs.
"""
import struct

import numpy as np

_MAGIC = b"CPBIN01\n"
_DT = {"d": np.float64, "i": np.int32, "b": np.uint8}
_CODE = {np.dtype(np.float64): "d", np.dtype(np.int32): "i", np.dtype(np.uint8): "b"}


def read(path):
    """Returns {name: np.ndarray} (scalars come back as 1-element arrays)."""
    out = {}
    with open(path, "rb") as f:
        if f.read(8) != _MAGIC:
            raise ValueError(f"{path}: not a CPBIN01 file")
        while True:
            hdr = f.read(40)
            if len(hdr) < 40:
                break
            name = hdr[:32].split(b"\0", 1)[0].decode()
            code = chr(hdr[32])
            (count,) = struct.unpack("<q", f.read(8))
            dt = np.dtype(_DT[code])
            out[name] = np.frombuffer(f.read(count * dt.itemsize), dtype=dt).copy()
    return out


def write(path, arrays):
    """arrays: {name: array-like}; float -> f64, int -> i32, bool/uint8 -> u8."""
    with open(path, "wb") as f:
        f.write(_MAGIC)
        for name, a in arrays.items():
            a = np.asarray(a)
            if a.dtype == np.bool_:
                a = a.astype(np.uint8)
            elif np.issubdtype(a.dtype, np.floating):
                a = a.astype(np.float64)
            elif np.issubdtype(a.dtype, np.integer) and a.dtype != np.uint8:
                a = a.astype(np.int32)
            a = np.ascontiguousarray(a).ravel()
            hdr = bytearray(40)
            nb = name.encode()[:31]
            hdr[: len(nb)] = nb
            hdr[32] = ord(_CODE[a.dtype])
            f.write(bytes(hdr))
            f.write(struct.pack("<q", a.size))
            f.write(a.tobytes())
