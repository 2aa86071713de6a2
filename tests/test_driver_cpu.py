"""The standalone driver (gpuimogen_b200/imogen_run): argument handling and input checks, which
run before any CUDA call, so no GPU is needed."""
import os
import subprocess

import numpy as np
import pytest

from gpuimogen_b200 import build as bld


@pytest.fixture(scope="module")
def exe():
    return bld.build_driver()


def run(exe, *args):
    return subprocess.run([exe, *args], capture_output=True, text=True, timeout=60)


def test_help_and_bad_arguments(exe):
    r = run(exe, "--help")
    assert r.returncode == 0 and "usage: imogen_run" in r.stdout
    for bad in (["--bogus", "1"], ["--grid", "64,64"], ["--grid", "0,4,4"], ["--method", "roe"],
                ["--limiter", "koren"], ["--drag", "euler"], ["--cfl", "-1"], ["--problem", "blast"],
                ["--steps"]):
        r = run(exe, *bad)
        assert r.returncode == 2, (bad, r.returncode, r.stderr)
        assert "usage" in r.stderr


def test_input_state_size_checked(exe, tmp_path):
    # a 16 x 8 x 4 grid has a 512-double slab pitch: the file must hold exactly 5 x 512 doubles
    f = tmp_path / "short.bin"
    np.zeros(5 * 512 - 1).tofile(f)
    r = run(exe, "--grid", "16,8,4", "--input", str(f))
    assert r.returncode == 2 and "is not a" in r.stderr
    r = run(exe, "--grid", "16,8,4", "--input", str(tmp_path / "missing.bin"))
    assert r.returncode == 2
