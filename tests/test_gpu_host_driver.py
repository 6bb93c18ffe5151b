"""polyorder_b200 (the C++ host driver over the C ABI) runs the reference's
own example param.ini files unchanged, including their Brent cell
optimisation, and reproduces the optimum the reference published."""
import os
import subprocess

import numpy as np

import pytest

from test_host_driver import _case, _parse

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def exe():
    from polystring_b200 import build
    build.build()
    return build.HOST_EXE


# tolerances: the reference's Brent stops on a bracket of about 4 tol_cell a
# (tol_cell 1e-4), so its optimum a is known to ~2e-3 and F(a) to ~2e-7 near
# the flat minimum; the 2D fields are converged only to 1e-6
@pytest.mark.parametrize("dim,tag,ftol,atol,tol0", [("1d", "1d_os2", 3e-7, 3e-3, 3e-8),
                                                    ("2d", "2d_rqm4_anderson", 2e-6, 4e-3, 1e-6)])
def test_example_config_runs_brent_to_published_optimum(exe, tmp_path, golden, dim, tag, ftol, atol, tol0):
    """The example configs ask for a Brent cell optimisation from a = 3.0
    with step 1.0 (2D: stress-driven root of dF/da; 1D OS2: F only)."""
    import scipy.io
    d, _, _ = _case(tmp_path, golden, dim)
    r = subprocess.run([exe, str(d / "param.ini")], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    v = _parse(r.stdout)
    H, amin = float(v["H"][1]), float(v["amin"][1])
    assert abs(H - golden[tag + "_F"][-1]) < ftol, (H, golden[tag + "_F"][-1])
    assert abs(amin - golden[tag + "_a"][-1]) < atol, (amin, golden[tag + "_a"][-1])
    assert abs(float(v["Fmin"][1]) - H) < 1e-12   # printed with different formats
    assert float(v["residual"][1]) < (1e-8 if dim == "1d" else 1e-6)
    # the cell record (scft::save_cell): its first solve is the configured a = 3.0,
    # whose free energy is the first entry the reference wrote
    cell = scipy.io.loadmat(str(d / "scft_out_cell.mat"))
    assert cell["a"].ravel()[0] == 3.0 == golden[tag + "_a"][0]
    assert abs(cell["F"].ravel()[0] - golden[tag + "_F"][0]) < tol0
    assert cell["F"].ravel().min() >= H - 1e-12 or abs(cell["F"].ravel().min() - H) < ftol


def _string_case(tmp_path, beads, iters, thresh, shape=(32, 64), cell=(4.0, 8.0)):
    """The reference's string config with its [string] run shortened and,
    unless shape is the reference's own 128 x 352, its grid and cell shrunk;
    the other sections unchanged (compressible AB, chiN 30, RQM4, Ms [21, 21],
    3 SCFT iterations per image, lam [0.015, 0.015, 100]); end states written
    as the reference's defect.mat / vLam.mat are."""
    import re
    import scipy.io
    from test_host_driver import GOLD
    lines = open(os.path.join(GOLD, "paramString.ini")).read().splitlines()
    edits = {("string", "num_of_beads"): beads, ("string", "string_iteration"): iters,
             ("string", "save_string_interval"): 1, ("string", "thresh_string_H"): thresh}
    if shape != (128, 352):
        edits.update({("Grid", "Lx"): shape[0], ("Grid", "Ly"): shape[1], ("UnitCell", "a"): cell[0],
                      ("UnitCell", "b"): cell[1]})
    section, done = None, set()
    for i, line in enumerate(lines):
        sec = re.match(r"\s*\[(\w+)\]", line)
        if sec:
            section = sec.group(1)
            continue
        kv = re.match(r"\s*(\w+)\s*=", line)
        if kv and (section, kv.group(1)) in edits:
            lines[i] = "%s = %s" % (kv.group(1), edits[(section, kv.group(1))])
            done.add((section, kv.group(1)))
    assert done == set(edits), set(edits) - done
    (tmp_path / "paramString.ini").write_text("\n".join(lines) + "\n")
    from polystring_b200 import workloads
    wa, wb = workloads.string_images(m=2, shape=shape + (1,), L=cell[0], seed=12)
    rng = np.random.default_rng(3)
    ends = []
    for k, f in enumerate(("defect.mat", "vLam.mat")):
        d = {"wA": wa[k][..., 0], "wB": wb[k][..., 0], "phiA": rng.uniform(size=shape), "phiB": rng.uniform(size=shape),
             "Q": np.ones((1, 1))}
        scipy.io.savemat(str(tmp_path / f), d)
        ends.append(d)
    return ends


@pytest.mark.parametrize("m,iters,shape,cell", [(5, 3, (32, 64), (4.0, 8.0)),
                                                 (61, 2, (128, 352), (26.3145, 70.1720))])
def test_string_driver_matches_oracle_string_iterations(tmp_path, m, iters, shape, cell):
    """polystring_ab_b200 on the reference's paramString.ini, with only the
    run length shortened (and, in the first case, the grid reduced; the
    second keeps the reference's 61 beads on its 128 x 352 grid, whose
    352-point lines take the radix-11 Stockham plan): the initial string
    interpolated from the end-state files, the string iterations, the records
    and the string in result.mat against the oracle's composition of
    polystring_AB's steps."""
    import scipy.io
    import oracle
    from polystring_b200 import build
    build.build()
    oracle.build()
    oracle.set_threads(oracle.max_threads())
    ends = _string_case(tmp_path, m, iters, 1e-12, shape, cell)
    r = subprocess.run([build.STRING_EXE, str(tmp_path / "paramString.ini")], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    res = scipy.io.loadmat(str(tmp_path / "result.mat"))
    # the oracle: same initial interpolation, same model
    wa = np.stack([ends[0]["wA"] + i / (m - 1) * (ends[1]["wA"] - ends[0]["wA"]) for i in range(m)])[..., None]
    wb = np.stack([ends[0]["wB"] + i / (m - 1) * (ends[1]["wB"] - ends[0]["wB"]) for i in range(m)])[..., None]
    o = oracle.ModelAB(2, shape + (1,), cell, (21, 21), 30.0, lam=(0.015, 0.015, 100.0), compressible=True)
    end_a, end_b = (wa[0].copy(), wa[-1].copy()), (wb[0].copy(), wb[-1].copy())
    H_prev = None
    for st in range(iters):
        H, S = oracle.string_iteration(o, wa, wb, end_a, end_b, 3)
        np.testing.assert_allclose(res["H"][st], H, rtol=1e-10, atol=0)
        np.testing.assert_allclose(res["S"][st], S, rtol=1e-10, atol=1e-12)
        assert abs(res["F"].ravel()[st] - H.mean()) <= 1e-10 * abs(H.mean())
        if H_prev is not None:
            np.testing.assert_allclose(res["dH"][st], np.abs(H - H_prev), rtol=1e-6, atol=1e-12)
        H_prev = H
    assert np.abs(res["wa"].reshape(m, shape[0], shape[1], 1) - wa).max() < 1e-10
    assert np.abs(res["wb"].reshape(m, shape[0], shape[1], 1) - wb).max() < 1e-10
    # the ends' densities are the input files' (restored, as the reference does)
    assert np.array_equal(res["phia"][0].reshape(shape), ends[0]["phiA"])
    assert np.array_equal(res["phib"][m - 1].reshape(shape), ends[1]["phiB"])


def test_string_driver_stops_on_thresh_string_H(tmp_path):
    """max |dH| <= thresh_string_H ends the run (the first iteration's dH is
    the reference's initial 10)."""
    import scipy.io
    from polystring_b200 import build
    build.build()
    _string_case(tmp_path, 4, 50, 20.0)
    r = subprocess.run([build.STRING_EXE, str(tmp_path / "paramString.ini")], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "string iterations = 1" in r.stdout
    res = scipy.io.loadmat(str(tmp_path / "result.mat"))
    assert res["F"].ravel()[0] != 0.0 and np.all(res["F"].ravel()[1:] == 0.0)
