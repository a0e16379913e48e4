"""The renderer hand-off snapshot (bhgpu.snapshot): a written file reads
back bit for bit with its header; wrong shapes and foreign files are
refused.  Host arrays only (no device needed)."""
import numpy as np
import pytest

from bhgpu import snapshot


def arrays(n, rng, derived=False):
    a = {"W": rng.normal(size=(n, 8, 16, 16, 16)), "origin": rng.normal(size=(n, 3)),
         "spacing": rng.uniform(0.1, 1.0, size=(n, 3)), "level": rng.integers(0, 4, size=n).astype(np.int32)}
    if derived:
        a["Wd"] = rng.normal(size=(n, 4, 16, 16, 16))
    return a


@pytest.mark.parametrize("derived", [False, True])
def test_round_trip(tmp_path, derived):
    rng = np.random.default_rng(1)
    a = arrays(5, rng, derived)
    a["W"][0, 0, 0, 0, 0] = np.nan
    path = str(tmp_path / "s.bhsnap")
    snapshot.write(path, a, t=1.25, step=7, metric=(1.0, 0.9375, 0.0), gamma=4.0 / 3.0)
    h, b = snapshot.read(path)
    assert h["t"] == 1.25 and h["step"] == 7 and h["metric"]["a"] == 0.9375 and h["block"] == 16
    assert h["fields"] == snapshot.FIELDS
    assert set(b) == set(a)
    for k in a:
        assert b[k].dtype == np.dtype(h["arrays"][k]["dtype"])
        assert np.array_equal(b[k].view(np.uint8), np.ascontiguousarray(a[k], b[k].dtype).view(np.uint8)), k
        assert h["arrays"][k]["offset"] % 16 == 0


def test_refusals(tmp_path):
    rng = np.random.default_rng(2)
    a = arrays(2, rng)
    a["W"] = a["W"][:, :7]
    with pytest.raises(ValueError):
        snapshot.write(str(tmp_path / "bad"), a)
    p = tmp_path / "other"
    p.write_bytes(b"NOTASNAP" + b"\0" * 64)
    with pytest.raises(ValueError):
        snapshot.read(str(p))
