"""Reader and writer of the reference's binary .H files.

Format of binWrite/binRead (nmbader/fwi3d src/include/IO.hpp:181-430): a text
header of `key=value` words -- n1..n6 (default 1), o1..o6 (0), d1..d6 (1),
label1..label6, esize (4), in=<path of the binary> (quotes allowed); lines
starting with '#' are comments -- and a raw binary of n1*...*n6 elements,
axis 1 fastest, in native byte order (esize 4: float32, 8: float64).  The
writer puts the binary at <datapath>/<header path>@, datapath from the
DATAPATH environment variable, else PWD, else ".", as binWrite does.  Headers
that declare data_format=xdr_* (SEPlib files) are read big-endian.

Arrays are returned C-ordered with the slowest axis first (shape
(nk, ..., n1)), i.e. the reference's [ny][nx][nz] model layout for a
(n1=nz, n2=nx, n3=ny) cube.  Trailing axes of length 1 are dropped down to
`ndim0` axes, as binRead does.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np


@dataclass
class Axis:
    n: int
    o: float = 0.0
    d: float = 1.0
    label: str = ""


def read_header(path: str) -> dict:
    h: dict = {}
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                continue
            for word in line.split():
                if "=" not in word:
                    continue
                k, v = word.split("=", 1)
                if k == "in" and len(v) >= 2 and v[0] == '"':
                    v = v[1:-1]
                h[k] = v
    return h


def read(path: str, ndim0: int = 1) -> Tuple[np.ndarray, List[Axis]]:
    """binRead: returns (array, axes)."""
    h = read_header(path)
    axes = []
    for i in range(1, 7):
        axes.append(Axis(int(h.get(f"n{i}", 1)), float(h.get(f"o{i}", 0.0)), float(h.get(f"d{i}", 1.0)),
                         h.get(f"label{i}", "")))
    ndim = 6
    while ndim > 1 and axes[ndim - 1].n == 1 and ndim0 != ndim:
        ndim -= 1
    axes = axes[:ndim]
    esize = int(h.get("esize", 4))
    if esize not in (4, 8):
        raise ValueError(f"{path}: esize {esize} is not 4 or 8")
    big = "xdr" in h.get("data_format", "")
    dt = np.dtype((">" if big else "<") + ("f4" if esize == 4 else "f8"))
    binp = h.get("in", "")
    if not binp:
        raise ValueError(f"{path}: no in= entry")
    if not os.path.isabs(binp) and not os.path.exists(binp):
        alt = os.path.join(os.path.dirname(os.path.abspath(path)), os.path.basename(binp))
        if os.path.exists(alt):
            binp = alt
    n123 = int(np.prod([a.n for a in axes]))
    size = os.path.getsize(binp)
    if size != n123 * esize:
        raise ValueError(f"The binary file contains {size} bytes whereas the description file suggests "
                         f"{n123 * esize} bytes")
    data = np.fromfile(binp, dtype=dt, count=n123)
    shape = tuple(a.n for a in reversed(axes))
    return data.reshape(shape).astype(dt.newbyteorder("=")), axes


def write(path: str, array: np.ndarray, axes: Optional[Sequence[Axis]] = None,
          datapath: Optional[str] = None) -> str:
    """binWrite: header at `path`, binary at <datapath>/<path>@; returns the binary path."""
    a = np.ascontiguousarray(array)
    if a.dtype not in (np.float32, np.float64):
        a = a.astype(np.float32)
    if axes is None:
        axes = [Axis(n) for n in reversed(a.shape)]
    if int(np.prod([ax.n for ax in axes])) != a.size:
        raise ValueError("axes do not match the array size")
    if datapath is None:
        datapath = os.environ.get("DATAPATH") or os.environ.get("PWD") or "."
    binp = datapath + "/" + path + "@"
    with open(path, "w") as f:
        for i, ax in enumerate(axes, start=1):
            f.write(f"n{i}={ax.n}\no{i}={_num(ax.o)}\nd{i}={_num(ax.d)}\n")
        f.write(f"esize={a.dtype.itemsize}\n")
        f.write(f"in={binp}\n")
    os.makedirs(os.path.dirname(os.path.abspath(binp)), exist_ok=True)
    a.astype(a.dtype.newbyteorder("<")).tofile(binp)
    return binp


def _num(v: float) -> str:
    # the C++ stream default: up to 6 significant digits
    return f"{v:.6g}"


def model_axes(sv) -> List[Axis]:
    """Axes of a model cube (z, x, y, parameter) as the reference writes them."""
    return [Axis(sv.nz, sv.oz, sv.dz), Axis(sv.nx, sv.ox, sv.dx), Axis(sv.ny, sv.oy, sv.dy), Axis(sv.nmodels, 0, 1)]
