"""The boundary from plain C: tests/capi/capi_roundtrip.c includes only
include/bhgpu.h (and the CUDA runtime's C API), is compiled as C99 with
every warning an error and linked against libbhgpu.so.  On the CPU it makes
the host-only calls; on a B200 it round-trips static states through
bh_ptoc and bh_ctop."""
import os
import re
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIBDIR = os.path.join(REPO, "black-hole-simulator_b200", "bhgpu")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build(tmp_path):
    exe = str(tmp_path / "capi_roundtrip")
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-O2", "-I" + os.path.join(REPO, "include"),
           "-I" + os.path.join(CUDA, "include"), os.path.join(HERE, "capi", "capi_roundtrip.c"), "-o", exe,
           "-L" + LIBDIR, "-lbhgpu", "-Wl,-rpath," + LIBDIR, "-L" + os.path.join(CUDA, "lib64"), "-lcudart",
           "-Wl,-rpath," + os.path.join(CUDA, "lib64"), "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_header_compiles_as_c99_and_links(tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert re.search(r"abi 1 flux_candidates 4 first 3", r.stdout), r.stdout


@pytest.mark.gpu
def test_c_caller_round_trips_static_states(tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([exe, "gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    m = re.search(r"rho_max_rel_err (\S+) not_recovered (\d+)", r.stdout)
    assert m, r.stdout
    assert float(m.group(1)) <= 1e-12 and int(m.group(2)) == 0, r.stdout
