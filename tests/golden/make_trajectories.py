"""Long oracle trajectories of the benchmark workloads, for the GPU tests.

    python tests/golden/make_trajectories.py C2 [iterations]

Runs the CPU oracle (oracle/scft_oracle.c) on the seeded inputs of a
workload for many SCFT iterations and writes tests/golden/<name>_trajectory.npz
with, after every iteration k = 1..n:

* H, Hw, Hs, Q and the residual error (Model_AB.cc:263-371);

and every `every` iterations (k = every, 2 every, ...):

* wA, wB, phiA, phiB at `n_sample` fixed grid points (seeded choice), and the
  max-abs of each field over the whole grid.

The GPU test replays the same iterations through the C ABI and compares.
The oracle's reductions are sequential and only its FFTs are threaded (each
thread owns whole lines), so the fixture does not depend on the thread count.
C2 (64^3, Ns 200, Anderson 20) costs about 9 s per iteration on 8 cores.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from polystring_b200 import workloads  # noqa: E402

FIELDS = ("wA", "wB", "phiA", "phiB")


def sample_index(M, n_sample, seed=99):
    return np.sort(np.random.default_rng(seed).choice(M, size=n_sample, replace=False))


def lengths(cfg):
    system, a = cfg["cell"]
    if system in ("SQUARE", "CUBIC"):
        return tuple([a[0]] * cfg["dim"])
    return tuple(a)


def run(name, n_iter, every=50, n_sample=512, suffix=""):
    cfg = workloads.config(name)
    oracle.set_threads(oracle.max_threads())
    o = oracle.ModelAB(cfg["dim"], cfg["shape"], lengths(cfg), cfg["Ms"], cfg["chiN"], lam=cfg["lam"],
                       mde=cfg["mde"], scft=cfg["scft"], n_anderson=cfg["n_anderson"])
    o.init_fields(cfg["wA"], cfg["wB"])
    M = int(np.prod(cfg["shape"]))
    idx = sample_index(M, n_sample)
    scal = np.zeros((n_iter, 5))
    snaps = {f: [] for f in FIELDS}
    maxabs = {f: [] for f in FIELDS}
    t0 = time.time()
    for k in range(1, n_iter + 1):
        o.update(1)
        H, Hw, Hs = o.H()
        scal[k - 1] = (H, Hw, Hs, o.Q(), o.residual())
        if k % every == 0:
            for f in FIELDS:
                a = o.get(f).ravel()
                snaps[f].append(a[idx])
                maxabs[f].append(np.abs(a).max())
            print("%s it %d H %.15f res %.3e (%.0f s)" % (name, k, H, scal[k - 1, 4], time.time() - t0), flush=True)
            save(name + suffix, scal[:k], idx, every, snaps, maxabs)
    print("done in %.0f s" % (time.time() - t0))


def save(name, scal, idx, every, snaps, maxabs):
    """Written after every checkpoint, so a run cut short still leaves a
    fixture of the iterations it finished."""
    out = dict(scalars=scal, sample_index=idx, every=np.int64(every))
    for f in FIELDS:
        out[f + "_sample"] = np.array(snaps[f])
        out[f + "_maxabs"] = np.array(maxabs[f])
    dst = os.path.join(HERE, "%s_trajectory.npz" % name.lower())
    np.savez_compressed(dst + ".tmp.npz", **out)
    os.replace(dst + ".tmp.npz", dst)


if __name__ == "__main__":
    # make_trajectories.py NAME [ITERATIONS [EVERY [SUFFIX]]]: the fixture is
    # tests/golden/<name><suffix>_trajectory.npz
    name = sys.argv[1] if len(sys.argv) > 1 else "C2"
    n = int(sys.argv[2]) if len(sys.argv) > 2 else dict(C1=500, C2=1000).get(name, 100)
    every = int(sys.argv[3]) if len(sys.argv) > 3 else (50 if name == "C1" else 100)
    suffix = sys.argv[4] if len(sys.argv) > 4 else ""
    run(name, n, every=every, suffix=suffix)
