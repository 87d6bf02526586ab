"""Reader of the flat record files written by the reference dump drivers
(oracle/ref_setup_dump.cu, oracle/ref_hybrid_amg_dump.cu): magic NDSDUMP1,
then records of (48-byte name, 8-byte dtype tag, int64 count, data).
Test infrastructure only."""
from __future__ import annotations

import numpy as np


def read_dump(path) -> dict:
    """Reader of the flat record files written by oracle/ref_setup_dump."""
    dt = {"f64": np.float64, "i32": np.int32, "i64": np.int64, "u8": np.uint8, "u32": np.uint32}
    out = {}
    with open(path, "rb") as f:
        if f.read(8) != b"NDSDUMP1":
            raise ValueError("not an NDSDUMP1 file")
        while True:
            nm = f.read(48)
            if len(nm) < 48:
                break
            name = nm.split(b"\0", 1)[0].decode()
            d = f.read(8).split(b"\0", 1)[0].decode()
            n = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
            t = np.dtype(dt[d])
            out[name] = np.frombuffer(f.read(n * t.itemsize), dtype=t).copy()
    return out
