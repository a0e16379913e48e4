"""CPU-only checks of the boundary and the host logic: the C ABI library
loads and exports every function include/bhgpu.h declares (no GPU call is
made), and the host-side patch quilt behaves like amrtree's bookkeeping."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from bhgpu import mesh

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(REPO, "include", "bhgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\bint\s+(bh_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import bhgpu
    lib = C.CDLL(bhgpu.LIB_PATH)
    names = declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.bh_abi_version() == 1


def test_header_has_no_torch_types():
    src = open(os.path.join(REPO, "include", "bhgpu.h")).read()
    assert "torch" not in src.lower().replace("pytorch", "") or "Tensor" not in src
    assert "at::" not in src and "Tensor" not in src


def test_periodic_quilt_neighbours():
    q = mesh.Quilt([0.0] * 3, [1.0] * 3, 3, periodic=True)
    T = q.tables()
    assert (T["nbr"][:, :, 1] == mesh.NB_COPY).all()
    # patch (0,0,0) wraps to (2,0,0) on its lower x side
    p = 0
    assert q.patches[T["nbr"][p, 0, 0]].ijk == (2, 0, 0)
    assert q.patches[T["nbr"][p, 1, 0]].ijk == (1, 0, 0)
    waves = q.ghost_waves(T["nbr"], T["leaf"])
    assert len(waves) == 1 and len(waves[0]) == 27


def test_outflow_quilt_and_refinement_tables():
    q = mesh.Quilt([0.0] * 3, [1.0] * 3, 2)
    T = q.tables()
    kinds = T["nbr"][:, :, 1]
    assert (kinds == mesh.NB_BNDY).sum() == 8 * 3 and (kinds == mesh.NB_COPY).sum() == 8 * 3
    kids = q.refine(0)
    assert len(kids) == 8 and not q.patches[0].leaf
    T = q.tables()
    assert T["leaf"].sum() == 7 + 8
    # a child on the outer face of patch 0 sees a coarse neighbour
    assert (T["nbr"][kids, :, 1] == mesh.NB_PROLONG).any()
    # child spacing is half the parent's
    assert np.allclose(T["pgeo"][kids[0], 3:], T["pgeo"][0, 3:] / 2)


def test_ghost_waves_order_prolongation_sources_first():
    q = mesh.Quilt([0.0] * 3, [1.0] * 3, 2)
    q.refine(0)
    q.refine(9)
    T = q.tables()
    waves = q.ghost_waves(T["nbr"], T["leaf"])
    where = {}
    for w, lst in enumerate(waves):
        for p in lst:
            where[int(p)] = w
    for p in where:
        for s in range(6):
            nb, kind = T["nbr"][p, s]
            if kind == mesh.NB_PROLONG and nb in where:
                # whichever comes first in quilt order is filled first
                if nb < p:
                    assert where[nb] < where[p]
                else:
                    assert where[p] < where[nb]


def test_pool_lists_longer_than_the_pool_are_rejected():
    """A pool whose `all` or `leaves` list claims more entries than it has
    patches is refused before anything is launched (no device needed)."""
    import ctypes as C
    import numpy as np
    from bhgpu._lib import BhParams, BhPool, lib
    idx = np.arange(4, dtype=np.int32)
    p = C.c_void_p(idx.ctypes.data)
    P = BhParams(0.0, 0.0, 0.0, 4.0 / 3.0, 0, 500, 1e-10, 1.0, 0.0, 0.0, 0, 0)
    too_many_all = BhPool(2, *([None] * 9), p, p, 0, *([None] * 5), 3)
    too_many_leaves = BhPool(2, *([None] * 9), p, p, 3, *([None] * 5), 0)
    for pool in (too_many_all, too_many_leaves):
        assert lib.bh_fluxcomp(C.byref(P), C.byref(pool), None) == -1
        assert lib.bh_floors(C.byref(P), C.byref(pool), None) == -1


def test_tuning_table_host_side():
    """The autotuner's launch-bound table: candidates per kernel, the
    compiled-in defaults among them, settable per variant, invalid values
    refused (host calls only, no device needed)."""
    from bhgpu import tune, BhError
    assert tune.candidates("flux") == [3, 4, 5, 6]
    assert tune.candidates("floors") == [4, 6, 8]
    for prec in ("fp64", "fp64-fma", "mixed"):
        for k, c in tune.current(prec).items():
            assert c in tune.candidates(k)
    assert tune.get("mixed", "flux") == 6 and tune.get("fp64", "flux") == 4
    tune.set("fp64", "update", 5)
    assert tune.get("fp64", "update") == 5 and tune.get("fp64-fma", "update") == 4
    tune.set("fp64", "update", 4)
    with pytest.raises(BhError):
        tune.set("fp64", "update", 7)
    assert tune.get("fp64", "update") == 4


def test_tuning_cache_file(tmp_path):
    """The tuner's cache: merged per key, replaced whole, a damaged file
    started afresh and read as absent (host only)."""
    import json
    from bhgpu import tune
    path = str(tmp_path / "t.json")
    tune._save(path, "GPU|fp64", {"flux": 4})
    tune._save(path, "GPU|mixed", {"flux": 6})
    with open(path) as f:
        assert json.load(f) == {"GPU|fp64": {"flux": 4}, "GPU|mixed": {"flux": 6}}
    with open(path, "w") as f:
        f.write("{not json")
    assert tune.load_tuning("fp64", cache=path) is None
    tune._save(path, "GPU|fp64", {"flux": 5})
    with open(path) as f:
        assert json.load(f) == {"GPU|fp64": {"flux": 5}}
