"""Post-processing reader of this library's snapshot files, with the interface of the reference's
``ext/python/read_cruna_data.py`` (``read_cruna_data(fname, **kwargs)`` :37-160 and
``read_cruna_params(fname)`` :164-236), so that a post-processing script switches by changing its
import.  The reference reads HDF5 files through h5py; this library stores the same content (the 4-D
FP64 dataset in Fortran order and the "key = value" parameter lines) in the flat binary container of
``public_b200/csrc/restart.cu``, which this module parses in plain Python (no CUDA library, no h5py).

Container: a 64-byte header -- magic "CRUNAB2D", int32 version 1, int32 element size (8 = float64,
4 = int32), int64 dims[4] (the Fortran shape), int64 length of the params text, int64 0 -- then the
params text, then the data.

Kept from the reference:
* file names ``<type>__BB_IIIII<idents>.<ext>``: ``images`` selects the block images to assemble
  (default: all i1*i2*i3 of ``parallelism``), each placed by its ``geom.xi{1,2,3}{0,1}i`` global index
  range; a single image without such keys fills the whole grid;
* ``component`` reads one of the five variables (0 density, 1-3 velocity components, 4 pressure in
  the reference's naming; here the stored conservative or adjoint variable of that index);
* ``read_params = [False, params]`` reuses a parameter dict instead of reading it;
* the result is squeezed: (n1, n2, n3, 5) for all components, (n1, n2, n3) for one;
* parameters become a nested dict by the dots of their keys (at most three levels), values are floats
  where they parse (lists split at ';', one value unwrapped), strings otherwise;
* ASCII parameter files (any other extension) are read with '%' starting a comment.
"""
from __future__ import annotations

import os
import struct
from typing import Dict, Tuple

import numpy as np

_MAGIC = b"CRUNAB2D"
_HEADER = struct.Struct("<8sii4qqq")     # 64 bytes


def _read_header(fh) -> Tuple[int, Tuple[int, int, int, int], int]:
    raw = fh.read(_HEADER.size)
    if len(raw) != _HEADER.size:
        raise ValueError("not a snapshot file of this library (short header)")
    magic, version, elem, d0, d1, d2, d3, plen, _ = _HEADER.unpack(raw)
    if magic != _MAGIC or version != 1:
        raise ValueError("not a snapshot file of this library")
    if elem not in (4, 8) or min(d0, d1, d2, d3) < 1 or plen < 0:
        raise ValueError("corrupt snapshot header")
    return elem, (d0, d1, d2, d3), plen


def _params_text(fname: str) -> str:
    with open(fname, "rb") as fh:
        _, _, plen = _read_header(fh)
        txt = fh.read(plen)
    if len(txt) != plen:
        raise ValueError(f"{fname}: truncated params")
    return txt.decode()


def _parse_value(v: str):
    parts = [p for p in v.split(";") if p]
    try:
        vals = [float(p) for p in parts]
    except ValueError:
        vals = parts
    return vals[0] if len(vals) == 1 else vals


def _nest(pairs) -> Dict:
    params: Dict = {}
    for key, value in pairs:
        levels = key.split(".")
        if len(levels) > 3:
            break                                   # the reference stops at the first deeper key
        node = params
        for k in levels[:-1]:
            node = node.setdefault(k, {})
        node[levels[-1]] = value
    return params


def read_cruna_params(fname: str) -> Dict:
    """Parameters of a snapshot file (its params text) or of an ASCII parameter file, as a dict nested
    by the dots of the keys."""
    if os.path.splitext(fname)[1] == ".bin":
        lines = _params_text(fname).splitlines()
    else:
        with open(fname) as fh:
            lines = fh.readlines()
    pairs = []
    for line in lines:
        line = line.split("%", 1)[0].replace(" ", "").replace("\t", "").strip()
        if not line or "=" not in line:
            continue
        key, value = line.split("=", 1)
        if key:
            pairs.append((key, _parse_value(value)))
    return _nest(pairs)


def _read_data(fname: str, component) -> np.ndarray:
    with open(fname, "rb") as fh:
        elem, dims, plen = _read_header(fh)
        fh.seek(_HEADER.size + plen)
        count = int(np.prod(dims))
        dt = np.float64 if elem == 8 else np.int32
        a = np.fromfile(fh, dtype=dt, count=count)
    if a.size != count:
        raise ValueError(f"{fname}: truncated data")
    a = a.reshape(dims, order="F")
    if component != "all":
        c = int(component)
        a = a[:, :, :, c:c + 1]
    return a


def _image_names(fname: str, images) -> list:
    folder, base = os.path.split(fname)
    root, ext = os.path.splitext(base)
    head, sep, tail = root.partition("__")
    if not sep:
        return [fname]
    fields = tail.split("_")
    block, idents = fields[0], "".join("_" + f for f in fields[2:])
    return [os.path.join(folder, f"{head}__{block}_{int(n):05d}{idents}{ext}") for n in images]


def read_cruna_data(fname: str, **kwargs):
    """(data, params) of the snapshot fname and, by the image number in its name, of the other block
    images; keyword arguments ``component`` ('all' or 0-4), ``images`` ('all' or a list of image
    numbers) and ``read_params`` ([True, None] or [False, params])."""
    component = kwargs.get("component", "all")
    images = kwargs.get("images", "all")
    read_params = kwargs.get("read_params", [True, False])
    params = read_cruna_params(fname) if read_params[0] else read_params[1]
    if images == "all":
        par = params.get("parallelism", {})
        nimg = int(par.get("i1", 1)) * int(par.get("i2", 1)) * int(par.get("i3", 1))
        images = list(range(1, nimg + 1))
    names = _image_names(fname, images)
    first = _read_data(names[0], component)
    geom = params.get("geom", {})
    n = [int(geom[k]) for k in ("n1", "n2", "n3")] if all(k in geom for k in ("n1", "n2", "n3")) \
        else list(first.shape[:3])
    data = np.zeros(n + [first.shape[3]], dtype=first.dtype, order="F")
    for name in names:
        part = first if name == names[0] else _read_data(name, component)
        g = read_cruna_params(name).get("geom", {})
        if "xi10i" in g:
            lo = [int(g[f"xi{d}0i"]) - 1 for d in (1, 2, 3)]
            hi = [int(g[f"xi{d}1i"]) for d in (1, 2, 3)]
        elif len(names) == 1:
            lo, hi = [0, 0, 0], n
        else:
            raise NotImplementedError(f"{name}: no global index range (geom.xi10i ...) to place the image")
        data[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2], :] = part
    return np.squeeze(data), params
