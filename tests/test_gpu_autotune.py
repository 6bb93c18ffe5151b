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
