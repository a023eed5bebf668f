"""A small DCD writer for the tests (CHARMM, NAMD 2.5 and X-PLOR variants), written
from the file-format description, independent of the library's reader."""
import struct

import numpy as np


def _rec(payload: bytes, end: str, marker: int) -> bytes:
    fmt = end + ("i" if marker == 4 else "q")
    return struct.pack(fmt, len(payload)) + payload + struct.pack(fmt, len(payload))


def cell_record(a, b, c, alpha, beta, gamma, cosines=True):
    """A, gamma, B, beta, alpha, C; angles in degrees, stored as cosines (CHARMM / NAMD >= 2.5)
    or as degrees (NAMD 2.5)."""
    if cosines:
        g, bt, al = (np.cos(np.radians(x)) for x in (gamma, beta, alpha))
    else:
        g, bt, al = gamma, beta, alpha
    return [a, g, b, bt, al, c]


def write_dcd(path, frames, cells=None, end="<", marker=4, charmm=True, dim4=False, fixed=0, nframes=None,
              ntitle=2, truncate=0):
    """frames: list of [natoms, 3] arrays; cells: list of 6-value unit-cell records or None."""
    natoms = len(frames[0])
    ic = [0] * 20
    ic[0] = len(frames) if nframes is None else nframes
    ic[1], ic[2], ic[3] = 1, 1, len(frames)
    ic[8] = fixed
    if charmm:
        ic[10] = 1 if cells is not None else 0
        ic[11] = 1 if dim4 else 0
        ic[19] = 24
    hdr = b"CORD" + struct.pack(end + "20i", *ic)
    if charmm:   # CHARMM stores DELTA as a float in word 9
        hdr = hdr[:4 + 36] + struct.pack(end + "f", 0.002) + hdr[4 + 40:]
    out = _rec(hdr, end, marker)
    title = struct.pack(end + "i", ntitle) + b"".join(f"title line {i}".ljust(80).encode() for i in range(ntitle))
    out += _rec(title, end, marker)
    out += _rec(struct.pack(end + "i", natoms), end, marker)
    for k, x in enumerate(frames):
        x = np.asarray(x, dtype=np.float64)
        if cells is not None:
            out += _rec(struct.pack(end + "6d", *cells[k]), end, marker)
        for ax in range(3):
            out += _rec(np.asarray(x[:, ax], dtype=end + "f4").tobytes(), end, marker)
        if dim4:
            out += _rec(np.zeros(natoms, dtype=end + "f4").tobytes(), end, marker)
    if truncate:
        out = out[:-truncate]
    with open(path, "wb") as f:
        f.write(out)


def vmd_cell(a, b, c, alpha, beta, gamma):
    """The cell matrix built from A, B, C and the angles as the molfile path does, in FP64."""
    x, y = np.cos(np.radians(gamma)), np.sin(np.radians(gamma))
    u = np.cos(np.radians(beta))
    v = (np.cos(np.radians(alpha)) - x * u) / y
    w = np.sqrt(1 - u * u - v * v)
    m = np.zeros(9)
    m[0] = a
    m[3], m[4] = b * x, b * y
    m[6], m[7], m[8] = c * u, c * v, c * w
    return m
