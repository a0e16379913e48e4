"""Grid snapshots for a renderer.

The reference announces a binary file of grid data for its renderer
(data.hpp:8-9, "the structures necessary for writing grid data to a binary
file to be read by the renderer"; the data_write switch, main.cpp:40-43)
but defines neither the structures nor the writer.  This module is that
hand-off: the interior primitives of the leaf patches with the geometry a
reader needs to place them, in one self-describing little-endian file.

File layout::

    8 bytes   magic b"BHSNAP01"
    8 bytes   uint64 n: length of the header
    n bytes   header, UTF-8 JSON, padded with spaces to a multiple of 16
    arrays    each at header["arrays"][name]["offset"] (bytes from the start
              of the file, 16-byte aligned), C order, dtype and shape as given

Header: ``version``, ``t``, ``step``, ``metric`` {M, a, Q}, ``gamma``,
``block`` (16: interior cells per patch edge), ``fields`` (the primitive
names, the reference's prim order rho, eps, v0..v2, B0..B2), ``arrays``.
Arrays: ``W`` [npatch][8][16][16][16] float64 (patch, field, i, j, k; i
slowest as in the reference's patch index, grid.cpp:51-53), ``origin``
[npatch][3] (edge of the patch's cell 0 along x, y, z), ``spacing``
[npatch][3] (cell widths, patch::dx), ``level`` [npatch] int32, and with
``derived`` also ``Wd`` [npatch][4][16][16][16] (Lorentz factor, pressure,
enthalpy, b^2 as floors and regrid record them).
"""
from __future__ import annotations

import json
import struct

import numpy as np

MAGIC = b"BHSNAP01"
VERSION = 1
FIELDS = ["rho", "eps", "v0", "v1", "v2", "B0", "B1", "B2"]
DERIVED = ["lor", "p", "h", "b2"]
BLOCK, GHOST, CPN = 16, 2, 20


def _align(n: int, a: int = 16) -> int:
    return (n + a - 1) // a * a


def write(path: str, arrays: dict, t: float = 0.0, step: int = 0, metric=(0.0, 0.0, 0.0), gamma: float = 4.0 / 3.0):
    """Write a snapshot from host arrays (numpy): W, origin, spacing, level
    and optionally Wd, shaped as in the module docstring."""
    n = arrays["W"].shape[0]
    want = {"W": ((n, 8, BLOCK, BLOCK, BLOCK), "<f8"), "origin": ((n, 3), "<f8"), "spacing": ((n, 3), "<f8"),
            "level": ((n,), "<i4")}
    if "Wd" in arrays:
        want["Wd"] = ((n, 4, BLOCK, BLOCK, BLOCK), "<f8")
    data = {}
    for name, (shape, dt) in want.items():
        a = np.ascontiguousarray(arrays[name], dtype=np.dtype(dt))
        if a.shape != shape:
            raise ValueError(f"snapshot array {name}: shape {a.shape}, expected {shape}")
        data[name] = a
    header = {"version": VERSION, "t": float(t), "step": int(step),
              "metric": {"M": float(metric[0]), "a": float(metric[1]), "Q": float(metric[2])},
              "gamma": float(gamma), "block": BLOCK, "fields": FIELDS,
              "derived_fields": DERIVED if "Wd" in data else [], "arrays": {}}
    # offsets depend on the header's length, which depends on the offsets'
    # digits: fix the header length first with generous placeholders
    for name, a in data.items():
        header["arrays"][name] = {"dtype": a.dtype.str, "shape": list(a.shape), "offset": 10 ** 15}
    hlen = _align(16 + len(json.dumps(header).encode())) - 16
    off = 16 + hlen
    for name, a in data.items():
        header["arrays"][name]["offset"] = off
        off = _align(off + a.nbytes)
    text = json.dumps(header).encode()
    assert len(text) <= hlen
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<Q", hlen))
        f.write(text + b" " * (hlen - len(text)))
        for name, a in data.items():
            pos = f.tell()
            f.write(b"\0" * (header["arrays"][name]["offset"] - pos))
            f.write(a.tobytes())


def read(path: str):
    """(header, {name: numpy array}) of a snapshot file."""
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise ValueError(f"{path}: not a snapshot (magic)")
        (hlen,) = struct.unpack("<Q", f.read(8))
        header = json.loads(f.read(hlen).decode())
        if header.get("version") != VERSION:
            raise ValueError(f"{path}: snapshot version {header.get('version')}")
        out = {}
        for name, d in header["arrays"].items():
            f.seek(d["offset"])
            dt = np.dtype(d["dtype"])
            cnt = int(np.prod(d["shape"]))
            out[name] = np.frombuffer(f.read(cnt * dt.itemsize), dtype=dt).reshape(d["shape"])
    return header, out


def from_tree(tree, path: str, t: float = 0.0, step: int = 0, derived: bool = False):
    """data_write for an AmrTree: gather the leaf patches' interior cells on
    the device, copy them to the host once, write the snapshot."""
    import torch
    leaves = tree.leaves.long()
    n = int(leaves.numel())
    s = slice(GHOST, GHOST + BLOCK)
    W = tree.W.index_select(0, leaves).view(n, 8, CPN, CPN, CPN)[:, :, s, s, s].contiguous().cpu().numpy()
    arrays = {"W": W, "origin": tree.tables["pgeo"][leaves.cpu().numpy(), :3],
              "spacing": tree.tables["pgeo"][leaves.cpu().numpy(), 3:], "level": tree.tables["lvl"][leaves.cpu().numpy()]}
    if derived:
        arrays["Wd"] = tree.Wd.index_select(0, leaves).view(n, 4, CPN, CPN, CPN)[:, :, s, s, s].contiguous().cpu().numpy()
    torch.cuda.synchronize()
    write(path, arrays, t=t, step=step, metric=(tree.mtr.M, tree.mtr.a, tree.mtr.Q), gamma=tree.stt.gamma)
