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


def _mat_values(exe, path, name):
    r = subprocess.run([exe, "--mat", path, name], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    v = _parse(r.stdout)
    return [int(x) for x in v["dims"]], np.array([float(x) for x in v.get("values", [])])


def test_mat_reader_on_the_reference_string_file_excerpt(exe):
    """tests/golden/defect_excerpt.mat holds, byte for byte, the header and
    four variables of the reference's string/defect.mat, among them the double
    arrays MATLAB stored as miUINT8 (z, incomp) and miUINT16 (t): the reader
    returns the values scipy reads, in file (column-major) order."""
    path = os.path.join(GOLD, "defect_excerpt.mat")
    ref = scipy.io.loadmat(path)
    for name in ("Q", "z", "t", "incomp"):
        dims, vals = _mat_values(exe, path, name)
        want = np.asarray(ref[name], dtype=np.float64)
        assert dims == list(want.shape), name
        assert np.array_equal(vals, want.ravel(order="F")), name
    r = subprocess.run([exe, "--mat", path, "wA"], capture_output=True, text=True)
    assert r.returncode == 1 and "not found" in r.stderr


@pytest.mark.skipif(not os.environ.get("POLYSTRING_REFERENCE"), reason="POLYSTRING_REFERENCE not set")
def test_mat_reader_on_the_whole_reference_string_files(exe):
    """Every variable of the reference's string/defect.mat and string/vLam.mat
    (the end states of its string example), unchanged, against scipy."""
    for f in ("defect.mat", "vLam.mat"):
        path = os.path.join(os.environ["POLYSTRING_REFERENCE"], "string", f)
        ref = scipy.io.loadmat(path)
        for name in [k for k in ref if not k.startswith("__")]:
            dims, vals = _mat_values(exe, path, name)
            want = np.asarray(ref[name], dtype=np.float64)
            assert dims == list(want.shape), (f, name)
            assert np.array_equal(vals, want.ravel(order="F")), (f, name)


def test_string_driver_without_gpu_fails_cleanly(tmp_path):
    """The string application reads the reference's paramString.ini and its
    end-state files, then needs a device."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from polystring_b200 import build
    build.build()
    shutil.copy(os.path.join(GOLD, "paramString.ini"), tmp_path / "paramString.ini")
    rng = np.random.default_rng(0)
    for f in ("defect.mat", "vLam.mat"):
        scipy.io.savemat(str(tmp_path / f), {k: rng.uniform(size=(128, 352)) for k in ("wA", "wB", "phiA", "phiB")})
    r = subprocess.run([build.STRING_EXE, str(tmp_path / "paramString.ini")], capture_output=True, text=True)
    assert r.returncode == 1 and "error" in r.stderr
    assert "Initializing string by two ends" in r.stdout


@pytest.mark.parametrize("m_value,expect", [("", "0"), ("16", "16")])
def test_check_reads_etdrk4_keys(exe, tmp_path, golden, m_value, expect):
    """algorithm = ETDRK4 in [Algorithm_MDE] selects Etdrk4_PBC (enum value 2:
    OS2, RQM4, ETDRK4) and etdrk4_M is passed through (empty: the default)."""
    d, _, _ = _case(tmp_path, golden, "1d")
    text = (d / "param.ini").read_text()
    text = text.replace("algorithm = OS2", "algorithm = ETDRK4", 1).replace("etdrk4_M =", "etdrk4_M = " + m_value, 1)
    (d / "param.ini").write_text(text)
    r = subprocess.run([exe, "--check", str(d / "param.ini")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    v = _parse(r.stdout)
    assert v["mde"][0] == "2" and v["mde"][10] == expect
