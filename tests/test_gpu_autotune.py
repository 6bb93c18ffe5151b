"""The line-pass autotuner chooses, per axis, the FFT schedule (Stockham
passes or the register-resident four-step) and the Stockham tile height.
The tile never changes a line's arithmetic: with the schedule pinned
(PS_B200_REG_FFT=0) tuned and untuned models agree bit for bit.  A different
schedule only reorders roundings: free energies and densities agree to 1e-12."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, sys
import numpy as np
sys.path.insert(0, %(root)r)
import polystring_b200 as ps
from polystring_b200 import capi
out = {}
for dim, shape, cell in ((2, (128, 128, 1), ("SQUARE", (8.0,))), (3, (48, 32, 24), ("ORTHORHOMBIC", (4.0, 3.6, 3.2)))):
    rng = np.random.default_rng(5)
    wA = 0.5 * rng.standard_normal(shape)
    wB = -wA + 0.1 * rng.standard_normal(shape)
    m = ps.ModelAB(dim, shape, ps.make_cell(dim, cell[0], *cell[1]), (21, 33), 16.0)
    m.set_fields(wA, wB)
    m.update(2)
    out[str(shape)] = {"H": m.H()[0], "phiA": m.get("phiA").ravel()[::97].tolist()}
out["log"] = capi.load().ps_tuning_log().decode()
print(json.dumps(out))
"""


def _run(tune, sched=None):
    env = dict(os.environ)
    env["PS_B200_AUTOTUNE"] = "1" if tune else "0"
    if sched is not None:
        env["PS_B200_REG_FFT"] = sched
    r = subprocess.run([sys.executable, "-c", CHILD % {"root": ROOT}], capture_output=True, text=True, env=env,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_tuned_and_default_schedules_agree():
    tuned, plain = _run(True), _run(False)
    assert plain["log"] == ""
    assert "grid 128x128x1 RQM4 batch 1: schedule [" in tuned["log"]
    for key in ("(128, 128, 1)", "(48, 32, 24)"):
        assert abs(tuned[key]["H"] - plain[key]["H"]) <= 1e-12 * abs(plain[key]["H"])
        a, b = np.array(tuned[key]["phiA"]), np.array(plain[key]["phiA"])
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_tiles_alone_change_nothing():
    # Stockham everywhere: only tile heights are tuned, results are identical
    tuned, plain = _run(True, "0"), _run(False, "0")
    for key in ("(128, 128, 1)", "(48, 32, 24)"):
        assert tuned[key]["H"] == plain[key]["H"]
        assert np.array_equal(np.array(tuned[key]["phiA"]), np.array(plain[key]["phiA"]))


@pytest.fixture(scope="module")
def ps():
    import polystring_b200
    return polystring_b200


@pytest.mark.parametrize("shape,L", [((32, 32, 32), 3.9), ((48, 48, 48), 4.3)])
def test_sweep_tile_variants_are_bit_identical(ps, monkeypatch, shape, L):
    """The x-tile variants of the generic persistent sweep (the autotuner's
    choices for 32^3 and 48^3) give bit-identical iterations; the tuner logs
    its timings and choice."""
    rng = np.random.default_rng(5)
    wA = 0.5 * rng.uniform(-1, 1, shape)
    wB = -wA + 0.1 * rng.uniform(-1, 1, shape)
    out = []
    for v in ("0", "1", "2"):
        monkeypatch.setenv("PS_B200_SWEEP_VARIANT", v)
        m = ps.ModelAB(3, shape, ps.make_cell(3, "CUBIC", L), (13, 21), 20.0, scft="Anderson", n_anderson=3)
        assert m.launches_per_propagate() == 1
        m.set_fields(wA, wB)
        m.update(3)
        out.append((m.H(), m.get("phiA"), m.get("wB")))
    for H, phi, w in out[1:]:
        assert H == out[0][0]
        assert np.array_equal(phi, out[0][1]) and np.array_equal(w, out[0][2])
    monkeypatch.delenv("PS_B200_SWEEP_VARIANT")
    monkeypatch.setenv("PS_B200_AUTOTUNE", "1")
    ps.ModelAB(3, shape, ps.make_cell(3, "CUBIC", L), (13, 21), 20.0)
    log = ps.lib().ps_tuning_log().decode()
    assert "grid %dx%dx%d persistent sweep, x-tile columns" % shape in log
