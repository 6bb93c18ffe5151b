"""Oracle parity at the full sizes of the benchmark workloads.

Every case compares the CUDA path (through the C ABI) with the CPU oracle on
the same seeded inputs, at the parity bar: 1e-10 relative on Q and H,
1e-10 max-abs on the densities and fields (FP64).

* C1: 2D 64x64, Ms [31, 71], simple mixing lambda 0.1, the whole 500-iteration
  trajectory, compared every 50 iterations (oracle run live).
* C2: 3D 64^3, Ms [71, 131], Anderson (history 20): the first 5 iterations
  live (histories too), and the long trajectory against the oracle's
  committed fixtures (tests/golden/make_trajectories.py): parity through
  iteration 50, then a divergence that a 1e-15 perturbation reproduces.
* C3: one string iteration of 40 images of 128x128, Ms [46, 84]
  (Quad4_Closed on both blocks), three SCFT iterations per image.
* C5: every member of the 27-solve uneven sample (32^3 / 48^3 / 64^3, Ns
  64 / 128 / 256) for 2 Anderson iterations.
"""
import os

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def ps():
    oracle.build()
    oracle.set_threads(oracle.max_threads())
    import polystring_b200
    return polystring_b200


def _lengths(cfg):
    system, a = cfg["cell"]
    return tuple([a[0]] * cfg["dim"]) if system in ("SQUARE", "CUBIC") else tuple(a)


def _pair(ps, cfg):
    """(oracle model, GPU model) of a workload configuration, fields set."""
    system, a = cfg["cell"]
    cell = ps.make_cell(cfg["dim"], system, *a)
    kw = dict(lam=cfg["lam"], mde=cfg["mde"], scft=cfg["scft"], n_anderson=cfg["n_anderson"])
    o = oracle.ModelAB(cfg["dim"], cfg["shape"], _lengths(cfg), cfg["Ms"], cfg["chiN"], **kw)
    m = ps.ModelAB(cfg["dim"], cfg["shape"], cell, cfg["Ms"], cfg["chiN"], **kw)
    o.init_fields(cfg["wA"], cfg["wB"])
    m.set_fields(cfg["wA"], cfg["wB"])
    return o, m


def _compare(o, m, tag, fields=("phiA", "phiB", "wA", "wB")):
    assert abs(m.Q() - o.Q()) / o.Q() < 1e-10, (tag, m.Q(), o.Q())
    Ho, Hg = o.H()[0], m.H()[0]
    assert abs(Hg - Ho) / abs(Ho) < 1e-10, (tag, Hg, Ho)
    for f in fields:
        d = np.abs(m.get(f) - o.get(f)).max()
        assert d < 1e-10, (tag, f, d)
    assert abs(m.residual_error() - o.residual()) <= 1e-8 * o.residual(), (tag, m.residual_error(), o.residual())


def test_c1_em_trajectory_matches_oracle(ps):
    """C1: the whole 500-iteration simple-mixing trajectory."""
    from polystring_b200 import workloads
    cfg = workloads.config("C1")
    o, m = _pair(ps, cfg)
    for it in range(50, cfg["iters"] + 1, 50):
        o.update(50)
        m.update(50)
        _compare(o, m, "C1 iteration %d" % it)


def test_c2_first_iterations_match_oracle(ps):
    """C2 at full size: Ns 200 on 64^3 with Anderson (history 20); H, Q,
    densities and fields every iteration, the four histories after the first."""
    from polystring_b200 import workloads
    cfg = workloads.config("C2")
    o, m = _pair(ps, cfg)
    for it in range(1, 6):
        o.update(1)
        m.update(1)
        _compare(o, m, "C2 iteration %d" % it)
        if it == 1:
            for f in ("qA", "qB", "qAc", "qBc"):
                a, b = m.get(f), o.get(f)
                assert np.abs(a - b).max() / np.abs(b).max() < 1e-12, f


def _trajectory_fixture(name):
    path = os.path.join(HERE, "golden", "%s_trajectory.npz" % name)
    if not os.path.exists(path):
        pytest.skip("no trajectory fixture %s" % path)
    return np.load(path)


def _c2_run(ps, cfg, n, perturb=0.0, sample=None, every=10):
    """H, Q after each of n C2 iterations on the GPU (wA scaled point by point
    by 1 + perturb N(0, 1)), and fields at `sample` every `every` iterations."""
    from polystring_b200 import workloads
    m = workloads.model_of(ps, cfg)
    wA = cfg["wA"] * (1.0 + perturb * np.random.default_rng(5).standard_normal(cfg["shape"]))
    m.set_fields(wA, cfg["wB"])
    HQ, fields = np.zeros((n, 2)), []
    for k in range(1, n + 1):
        m.update(1)
        HQ[k - 1] = (m.H()[0], m.Q())
        if sample is not None and k % every == 0:
            fields.append(np.stack([m.get(f).ravel()[sample] for f in ("wA", "wB", "phiA", "phiB")]))
    return HQ, fields


def test_c2_trajectory_parity_and_where_it_diverges(ps):
    """C2's Anderson trajectory (history 20) against the oracle's recorded one.

    * Through iteration 50: H and Q at 1e-10 after every iteration; wA, wB,
      phiA, phiB at 512 sampled points (fixture c2_start, every 10
      iterations) at 1e-10 of each field's max-abs at iteration 10, and within
      100 times the perturbed run's spread up to 50 (the fields move off by
      about 6e-11 relative by iteration 10, before H and Q do).
    * Beyond, the iteration itself amplifies rounding: a GPU run started from
      the same fields with a 1e-15 relative perturbation of wA leaves the
      unperturbed run by about 1e-11 at iteration 60 and 1e-8 at 100 (H), the
      way the GPU and the oracle (two FFT orders) leave each other.  Along the
      whole recorded trajectory (fixture c2, up to the workload's 1000
      iterations) the GPU-oracle difference of H stays within 100 times that
      perturbation's spread (floor 1e-12), the spread at iteration k being the
      largest perturbed-run difference within 10 iterations of k (the
      difference of two such runs changes sign now and then, so its value at
      a single iteration can be arbitrarily small).  The first iteration where
      H leaves 1e-10 is printed."""
    from polystring_b200 import workloads
    fx, fs = _trajectory_fixture("c2"), _trajectory_fixture("c2_start")
    cfg = workloads.config("C2")
    n = fx["scalars"].shape[0]
    assert n >= 60
    every = int(fs["every"])
    HQ, fields = _c2_run(ps, cfg, n, sample=fs["sample_index"], every=every)
    HQp, fields_p = _c2_run(ps, cfg, n, perturb=1e-15, sample=fs["sample_index"], every=every)
    ref = fx["scalars"][:, [0, 3]]
    e_or = np.abs(HQ - ref).max(axis=1) / np.abs(ref).max(axis=1)
    e_pt = np.abs(HQ - HQp).max(axis=1) / np.abs(HQ).max(axis=1)
    assert e_or[:50].max() < 1e-10, e_or[:50].max()
    # sampled fields, relative to each field's max-abs over the grid: 1e-10 at
    # iteration 10; through 50 within 100 times the perturbed run's spread
    for j in range(min(50 // every, len(fs["wA_sample"]))):
        for i, f in enumerate(("wA", "wB", "phiA", "phiB")):
            scale = fs[f + "_maxabs"][j]
            d = np.abs(fields[j][i] - fs[f + "_sample"][j]).max() / scale
            dp = np.abs(fields[j][i] - fields_p[j][i]).max() / scale
            if j == 0:
                assert d < 1e-10, ((j + 1) * every, f, d)
            assert d <= 100.0 * max(dp, 1e-12), ((j + 1) * every, f, d, dp)
    win = 10
    spread = np.array([e_pt[max(0, k - win):k + win + 1].max() for k in range(n)])
    ratio = e_or / np.maximum(spread, 1e-12)
    k = int(np.argmax(ratio))
    assert ratio[k] <= 100.0, (k + 1, e_or[k], spread[k])
    over = np.nonzero(e_or > 1e-10)[0]
    print("C2 trajectory: H/Q within 1e-10 of the oracle through iteration %d of %d; at 100: oracle %.1e, "
          "1e-15 perturbation %.1e" % (over[0] if len(over) else n, n, e_or[min(99, n - 1)], e_pt[min(99, n - 1)]))


def test_c3_string_iteration_matches_oracle(ps):
    """C3 at full size: one string iteration of 40 images of 128x128 (three
    SCFT iterations per image, arc length, spline re-sampling), against the
    oracle's composition of polystring_AB's steps."""
    from polystring_b200 import workloads
    m_img, shape, L = 40, (128, 128, 1), 8.0
    Ms, chiN, lam = workloads.ms_from(0.35, 128), 18.0, (0.05, 0.05, 5.0)
    wa, wb = workloads.string_images(m=m_img, shape=shape, L=L)
    g = ps.StringAB(m_img, 2, shape, ps.make_cell(2, "SQUARE", L), Ms, chiN, lam=lam, max_iter=3)
    g.set_images(wa, wb)
    g.iterate(1)
    o = oracle.ModelAB(2, shape, (L, L), Ms, chiN, lam=lam)
    wa_o, wb_o = wa.copy(), wb.copy()
    H = np.zeros(m_img)
    phiA = np.zeros_like(wa)
    for s in range(m_img):
        o.init_fields(wa_o[s], wb_o[s])
        o.update(3)
        H[s] = o.H()[0]
        phiA[s] = o.get("phiA")
        wa_o[s], wb_o[s] = o.get("wA"), o.get("wB")
    S = oracle.string_arclength(wa_o)
    oracle.string_redistribute(wa_o, S, wa[0], wa[-1])
    oracle.string_redistribute(wb_o, S, wb[0], wb[-1])
    np.testing.assert_allclose(g.H(), H, rtol=1e-10, atol=0)
    np.testing.assert_allclose(g.S(), S, rtol=1e-10, atol=1e-12)
    assert np.abs(g.get("phiA") - phiA).max() < 1e-10
    assert np.abs(g.get("wa") - wa_o).max() < 1e-10
    assert np.abs(g.get("wb") - wb_o).max() < 1e-10


def test_c5_sample_members_match_oracle(ps):
    """Every member of the 27-solve uneven sample, advanced as one batch for
    two Anderson iterations, against its own oracle solve."""
    from polystring_b200 import workloads
    specs = workloads.uneven_solves(27)
    b = ps.BatchAB([dict(dim=3, shape=sp["shape"], cell=ps.make_cell(3, "CUBIC", sp["cell"][1][0]), Ms=sp["Ms"],
                         chiN=sp["chiN"], lam=sp["lam"], scft=sp["scft"], n_anderson=sp["n_anderson"])
                    for sp in specs])
    for k, sp in enumerate(specs):
        b.set_fields(k, sp["wA"], sp["wB"])
    b.update(2)
    for k, sp in enumerate(specs):
        a = sp["cell"][1][0]
        o = oracle.ModelAB(3, sp["shape"], (a, a, a), sp["Ms"], sp["chiN"], lam=sp["lam"], scft=sp["scft"],
                           n_anderson=sp["n_anderson"])
        o.init_fields(sp["wA"], sp["wB"])
        o.update(2)
        Ho, Hg = o.H()[0], b.H(k)[0]
        assert abs(Hg - Ho) / abs(Ho) < 1e-10, (k, Hg, Ho)
        for f in ("phiA", "phiB", "wA", "wB"):
            d = np.abs(b.get(k, f) - o.get(f)).max()
            assert d < 1e-10, (k, f, d)
        del o
