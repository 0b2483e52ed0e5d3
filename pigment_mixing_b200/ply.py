"""Reader for the binary little-endian PLY files the library writes (the reference's
save_data.cpp format: one `vertex` element of float32 properties)."""
from __future__ import annotations

import numpy as np


def read_ply(path: str) -> dict:
    """Property name -> float32 array of the `vertex` element."""
    with open(path, "rb") as f:
        if f.readline().strip() != b"ply":
            raise ValueError(f"{path}: not a PLY file")
        fmt = f.readline().split()
        if fmt[:2] != [b"format", b"binary_little_endian"]:
            raise ValueError(f"{path}: unsupported PLY format {fmt!r}")
        n, names = 0, []
        while True:
            line = f.readline()
            if not line:
                raise ValueError(f"{path}: no end_header")
            tok = line.split()
            if tok[0] == b"end_header":
                break
            if tok[0] == b"element":
                if tok[1] != b"vertex":
                    raise ValueError(f"{path}: unexpected element {tok[1]!r}")
                n = int(tok[2])
            elif tok[0] == b"property":
                if tok[1] != b"float":
                    raise ValueError(f"{path}: only float properties are written")
                names.append(tok[2].decode())
        data = np.frombuffer(f.read(), dtype="<f4")
    if data.size != n * len(names):
        raise ValueError(f"{path}: {data.size} values for {n} x {len(names)}")
    rows = data.reshape(n, len(names))
    return {name: rows[:, k].copy() for k, name in enumerate(names)}
