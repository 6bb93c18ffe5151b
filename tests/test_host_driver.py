"""The C++ host layer (polystring_b200/host): config parsing of the
reference's own example param.ini files and the MAT-v5 field reader, on the
CPU; the full driver run is in test_gpu_host_driver.py."""
import os
import shutil
import subprocess

import numpy as np
import pytest
import scipy.io

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def exe():
    from polystring_b200 import build
    build.build()
    return build.HOST_EXE


def _case(tmp_path, golden, dim):
    """Copy the unchanged example config and write its field file."""
    d = tmp_path / ("lam%s" % dim)
    d.mkdir()
    shutil.copy(os.path.join(GOLD, "lam%s_param.ini" % dim), d / "param.ini")
    wA, wB = golden["lam%s_wA" % dim], golden["lam%s_wB" % dim]
    fname = "field_in_64.mat" if dim == "1d" else "field_in_32x32.mat"
    scipy.io.savemat(str(d / fname), {"wA": wA, "wB": wB})
    return d, wA, wB


def _parse(out):
    """key -> tokens of the last line starting with that key"""
    vals = {}
    for line in out.splitlines():
        f = line.split()
        if f:
            vals[f[0]] = f[1:]
    return vals


def test_check_parses_example_configs(exe, tmp_path, golden):
    for dim, mde, scft, grid, thresh in (("1d", "0", "0", ["64", "1", "1"], 1e-8),
                                         ("2d", "1", "1", ["32", "32", "1"], 1e-6)):
        d, wA, wB = _case(tmp_path, golden, dim)
        r = subprocess.run([exe, "--check", str(d / "param.ini")], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        v = _parse(r.stdout)
        assert v["dim"][2:5] == grid
        assert v["Ms"][:2] == ["51", "51"] and float(v["Ms"][3]) == 30.0
        assert [float(x) for x in v["lam"]] == [0.05, 0.05, 5.0]
        assert v["mde"][0] == mde and v["mde"][2] == scft        # OS2/RQM4, EM/Anderson
        assert v["mde"][4] == "1"                                # Simpson
        assert float(v["n_anderson"][10]) == thresh
        # MAT-v5 reader: the same values scipy wrote (column-major on disk)
        assert abs(float(v["wA"][1]) - wA.mean()) < 1e-15 * max(1.0, abs(wA.mean())) + 1e-15
        assert float(v["wA"][3]) == wA.ravel()[0] and float(v["wB"][5]) == wB.ravel()[-1]


def test_driver_without_gpu_fails_cleanly(exe, tmp_path, golden):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    d, _, _ = _case(tmp_path, golden, "1d")
    r = subprocess.run([exe, str(d / "param.ini")], capture_output=True, text=True)
    assert r.returncode == 1 and "error" in r.stderr
