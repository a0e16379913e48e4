"""Launch-bound autotuner for the heaviest kernels (bh_tune_* in bhgpu.h).

The flux, update, con2prim (interior and ghost) and floors kernels are
compiled for several numbers of resident 128-thread CTAs per SM; more CTAs
per SM hide more latency but cap the registers a thread may use (spills).
Which count is fastest depends on the GPU, the arithmetic variant and the
state being stepped (con2prim's iteration counts), so ``autotune`` measures
it: it times whole RK2 steps of the caller's tree, restarted from the same
state each time, for every candidate of one kernel at a time (the others
held at their current choice), keeps the fastest, and moves on to the next
kernel.  The tree's state is restored afterwards.  The choices can be kept
in a JSON file keyed by GPU name and variant and applied again with
``load_tuning``.

The choice is per process and per arithmetic variant; CUDA graphs captured
before a change keep the kernels they recorded.  In the reference-faithful
variant every choice gives the same bits; in the contracted variants ptxas
may fuse a different set of multiply-add pairs under another register
budget, which moves results by ulps.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import torch

from ._lib import check, lib

KERNELS = ("flux", "update", "prims_interior", "prims_ghost", "floors")
PRECISION = {"fp64": 0, "fp64-fma": 1, "mixed": 2}


def _sig():
    i32 = C.c_int32
    lib.bh_tune_candidates.argtypes = [i32, C.POINTER(i32), i32]
    lib.bh_tune_set.argtypes = [i32, i32, i32]
    lib.bh_tune_get.argtypes = [i32, i32, C.POINTER(i32)]
    for f in ("bh_tune_candidates", "bh_tune_set", "bh_tune_get"):
        getattr(lib, f).restype = C.c_int


_sig()


def candidates(kernel: str) -> list[int]:
    buf = (C.c_int32 * 8)()
    n = lib.bh_tune_candidates(KERNELS.index(kernel), buf, 8)
    if n < 0:
        raise ValueError(kernel)
    return list(buf[:n])


def get(precision: str, kernel: str) -> int:
    v = C.c_int32()
    check(lib.bh_tune_get(PRECISION[precision], KERNELS.index(kernel), C.byref(v)), "bh_tune_get")
    return int(v.value)


def set(precision: str, kernel: str, ctas_per_sm: int) -> None:  # noqa: A001 (mirrors bh_tune_set)
    check(lib.bh_tune_set(PRECISION[precision], KERNELS.index(kernel), int(ctas_per_sm)), "bh_tune_set")


def current(precision: str) -> dict:
    return {k: get(precision, k) for k in KERNELS}


def _cache_path(path: str | None) -> str:
    if path:
        return path
    return os.environ.get("BHGPU_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "bhgpu", "tune.json"))


def _key(precision: str) -> str:
    return f"{torch.cuda.get_device_name()}|{precision}"


def autotune(tree, integrator, reps: int = 3, cache: str | None = None, save: bool = False) -> dict:
    """Time every candidate of every tuned kernel on ``tree`` (whole RK2
    steps through ``integrator``, each from the same saved state), set the
    fastest, restore the state and return ``{"choice": {...}, "ms": {...}}``
    (per kernel, the best step time of each candidate).  ``save`` writes the
    choice to the cache file."""
    prec = tree.precision
    names = ("U", "W", "dU", "Bf", "F", "EMF", "Wd", "aux", "status", "dt", "err")
    snap = {n: getattr(tree, n).clone() for n in names}

    def restore():
        for n in names:
            getattr(tree, n).copy_(snap[n])

    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    timings = {}
    for k in KERNELS:
        best, best_ms, per = None, None, {}
        for c in candidates(k):
            set(prec, k, c)
            ms = []
            for _ in range(reps + 1):          # the first step of each candidate is a warm-up
                restore()
                a.record()
                integrator.step(tree, sync=False, check_domain=False)
                b.record()
                torch.cuda.synchronize()
                ms.append(a.elapsed_time(b))
            per[c] = min(ms[1:])
            if best_ms is None or per[c] < best_ms:
                best, best_ms = c, per[c]
        set(prec, k, best)
        timings[k] = per
    restore()
    torch.cuda.synchronize()
    choice = current(prec)
    if save:
        _save(_cache_path(cache), _key(prec), choice)
    return {"choice": choice, "ms": timings}


def _save(path: str, key: str, choice: dict) -> None:
    """Merge one choice into the cache file; the file is replaced whole
    (write to a temporary name, then rename), so a reader never sees half
    of it, and an unreadable old file is started afresh."""
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    data = {}
    try:
        with open(path) as f:
            data = json.load(f)
    except (OSError, ValueError):
        data = {}
    data[key] = choice
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def load_tuning(precision: str, cache: str | None = None) -> dict | None:
    """Apply the cached choice for this GPU and variant, if there is one."""
    path = _cache_path(cache)
    try:
        with open(path) as f:
            choice = json.load(f).get(_key(precision))
    except (OSError, ValueError):
        return None
    if not choice:
        return None
    for k, c in choice.items():
        set(precision, k, c)
    return choice
