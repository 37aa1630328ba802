"""Reader for the PDB1 record files written by oracle/ref_harness.cpp."""
import struct

import numpy as np

_DT = {"d": np.float64, "i": np.int32, "q": np.int64}


def read_pdb(path):
    out = {}
    with open(path, "rb") as f:
        if f.read(4) != b"PDB1":
            raise ValueError(f"{path}: not a PDB1 file")
        while True:
            h = f.read(4)
            if not h:
                break
            (nl,) = struct.unpack("<I", h)
            name = f.read(nl).decode()
            t = f.read(1).decode()
            (cnt,) = struct.unpack("<Q", f.read(8))
            dt = _DT[t]
            out[name] = np.frombuffer(f.read(cnt * np.dtype(dt).itemsize), dtype=dt).copy()
    return out
