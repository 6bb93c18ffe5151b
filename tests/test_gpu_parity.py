"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Tolerances (FP64 throughout; the parity bar is 1e-10 relative on Q and H
and max-abs on the densities):
* single propagator solves: 1e-12 relative to max |q|;
* one SCFT iteration and short trajectories: 1e-10;
* converged free energies against the reference's published values: the
  reference's own convergence threshold (3e-8 in 1D, 1e-8 in 2D).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ps():
    oracle.build()
    import polystring_b200
    return polystring_b200


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _cell(ps, dim, L):
    if dim == 1:
        return ps.make_cell(1, "LAMELLAR", L[0])
    if dim == 2:
        return ps.make_cell(2, "RECTANGULAR", L[0], L[1])
    return ps.make_cell(3, "ORTHORHOMBIC", L[0], L[1], L[2])


SHAPES = [(1, (64, 1, 1), (4.0,)), (1, (48, 1, 1), (3.3,)), (2, (32, 32, 1), (4.0, 4.0)),
          (2, (64, 48, 1), (4.2, 3.9)), (2, (12, 128, 1), (3.0, 8.0)), (3, (16, 16, 16), (3.5, 3.5, 3.5)),
          (3, (24, 32, 12), (3.8, 4.0, 4.2)), (3, (32, 32, 32), (4.0, 4.0, 4.0))]


@pytest.mark.parametrize("dim,shape,L", SHAPES)
@pytest.mark.parametrize("scheme", ["RQM4", "OS2"])
def test_updater_solve_matches_oracle(ps, dim, shape, L, scheme):
    rng = np.random.default_rng(7)
    ds = 0.01
    w = 0.5 * rng.standard_normal(shape)
    qs = np.zeros((31,) + shape)
    qs[0] = 1.0 + 0.2 * rng.standard_normal(shape)
    cell = _cell(ps, dim, L)
    g, l = oracle.unit_cell(dim, cell.system, cell.a, cell.b, cell.c)
    if scheme == "RQM4":
        ref = oracle.Updater("RQM4", oracle.k2_orthogonal(dim, l, shape), shape, ds).solve(w, qs.copy())
        up = ps.RQM4(cell, *shape, ds)
    else:
        ref = oracle.Updater("OS2", oracle.k_laplacian(g, shape, ds), shape, ds).solve(w, qs.copy())
        up = ps.PseudoSpectral(cell, *shape, ds)
    out = up.solve(qs.copy(), w)
    assert _rel(out, ref) < 1e-12


@pytest.mark.parametrize("rule,n", [("simpson", 30), ("quad4_closed", 45), ("trapezoid", 20), ("quad4_open", 40),
                                    ("quad4_semiopen_left", 33), ("quad4_semiopen_right", 33)])
def test_density_matches_oracle(ps, rule, n):
    rng = np.random.default_rng(3)
    shape = (12, 8, 6)
    q = 1 + 0.1 * rng.standard_normal((n + 1,) + shape)
    qc = 1 + 0.1 * rng.standard_normal((n + 1,) + shape)
    r = {"trapezoid": 0, "simpson": 1, "quad4_closed": 2, "quad4_open": 3,
         "quad4_semiopen_left": 4, "quad4_semiopen_right": 5}[rule]
    ref = oracle.density(r, q, qc, 0.01, 0.7)
    out = ps.density(rule, q, qc, 0.01, 0.7)
    assert np.abs(out - ref).max() < 1e-13


def test_density_precondition_is_an_error(ps):
    q = np.ones((36,) + (4, 1, 1))     # n = 35: Simpson needs even n
    with pytest.raises(ps.PSError) as e:
        ps.density("simpson", q, q, 0.01, 1.0)
    assert e.value.code == -4


def test_unsupported_size_is_an_error(ps):
    with pytest.raises(ps.PSError) as e:
        ps.RQM4(ps.make_cell(1, "LAMELLAR", 4.0), 7, 1, 1, 0.01)
    assert e.value.code == -2


def _models(ps, dim, shape, L, Ms, chiN, **kw):
    cell = _cell(ps, dim, L)
    g, l = oracle.unit_cell(dim, cell.system, cell.a, cell.b, cell.c)
    o = oracle.ModelAB(dim, shape, tuple(l[:dim]), Ms, chiN, g=g, **kw)
    m = ps.ModelAB(dim, shape, cell, Ms, chiN, **kw)
    return o, m


def _seed_fields(shape, seed, amp=0.5):
    rng = np.random.default_rng(seed)
    wA = amp * rng.uniform(-1, 1, shape)
    wB = -wA + 0.1 * rng.uniform(-1, 1, shape)
    return wA, wB


MODEL_CASES = [
    (1, (64, 1, 1), (4.0,), (51, 51), 30.0),
    (2, (32, 32, 1), (4.0, 4.0), (31, 71), 20.0),
    (2, (24, 48, 1), (3.7, 4.4), (46, 84), 18.0),      # Quad4_Closed on both blocks
    (3, (16, 16, 16), (3.8, 4.0, 4.2), (39, 91), 22.0),
]


@pytest.mark.parametrize("dim,shape,L,Ms,chiN", MODEL_CASES)
@pytest.mark.parametrize("scft", ["EM", "Anderson"])
@pytest.mark.parametrize("mde", ["RQM4", "OS2"])
def test_model_trajectory_matches_oracle(ps, dim, shape, L, Ms, chiN, scft, mde):
    o, m = _models(ps, dim, shape, L, Ms, chiN, mde=mde, scft=scft, n_anderson=5)
    wA, wB = _seed_fields(shape, 11)
    o.init_fields(wA, wB)
    m.set_fields(wA, wB)
    for it, n in enumerate((1, 4, 15)):
        o.update(n)
        m.update(n)
        Ho, Hg = o.H()[0], m.H()[0]
        assert abs(m.Q() - o.Q()) / o.Q() < 1e-10, (it, m.Q(), o.Q())
        assert abs(Hg - Ho) / abs(Ho) < 1e-10, (it, Hg, Ho)
        for f in ("phiA", "phiB", "wA", "wB"):
            assert np.abs(m.get(f) - o.get(f)).max() < 1e-10, (it, f)
        assert abs(m.residual_error() - o.residual()) / o.residual() < 1e-8


def test_model_histories_match_oracle(ps):
    o, m = _models(ps, 2, (32, 32, 1), (4.0, 4.0), (31, 71), 20.0)
    wA, wB = _seed_fields((32, 32, 1), 5)
    o.init_fields(wA, wB)
    m.set_fields(wA, wB)
    o.update(1)
    m.update(1)
    for f in ("qA", "qB", "qAc", "qBc"):
        assert _rel(m.get(f), o.get(f)) < 1e-12, f


@pytest.mark.parametrize("mde", ["RQM4", "OS2"])
def test_uniform_field_is_exact(ps, mde):
    shape = (16, 12, 8)
    cell = ps.make_cell(3, "ORTHORHOMBIC", 3.0, 3.5, 4.0)
    m = ps.ModelAB(3, shape, cell, (31, 71), 20.0, mde=mde)
    m.set_fields(np.full(shape, 0.1), np.full(shape, 0.3))
    m.update(1)
    assert abs(m.Q() - np.exp(-0.1 * 0.3 - 0.3 * 0.7)) < 5e-14
    assert np.abs(m.get("phiA") - 0.3).max() < 5e-14
    assert np.abs(m.get("phiB") - 0.7).max() < 5e-14


def _converge(m, thresh, max_iter=20000):
    r = None
    for it in range(10, max_iter + 1, 10):
        m.update(10)
        if it > 10:
            r = m.residual_error()
            if r < thresh:
                break
    return r


@pytest.mark.parametrize("mde,scft,tag", [("RQM4", "EM", "1d_rqm4"), ("RQM4", "Anderson", "1d_rqm4_anderson"),
                                          ("OS2", "EM", "1d_os2"), ("OS2", "Anderson", "1d_os2_anderson")])
def test_published_free_energy_1d(ps, golden, mde, scft, tag):
    """Converged H on the reference's own 1D LAM input equals the F(a) the
    reference wrote, to the reference's convergence threshold."""
    a_tab, F_tab = golden[tag + "_a"], golden[tag + "_F"]
    for i in range(len(a_tab)):
        m = ps.ModelAB(1, (64, 1, 1), ps.make_cell(1, "LAMELLAR", a_tab[i]), (51, 51), 30.0,
                       lam=(0.05, 0.05, 5.0), mde=mde, scft=scft, n_anderson=5)
        m.set_fields(golden["lam1d_wA"], golden["lam1d_wB"])
        r = _converge(m, 1e-8)
        assert r < 1e-8
        assert abs(m.H()[0] - F_tab[i]) < 3e-8, (a_tab[i], m.H()[0], F_tab[i])


@pytest.mark.parametrize("mde,scft,tag", [("RQM4", "Anderson", "2d_rqm4_anderson"), ("OS2", "Anderson", "2d_os2_anderson")])
def test_published_free_energy_2d(ps, golden, mde, scft, tag):
    a_tab, F_tab = golden[tag + "_a"], golden[tag + "_F"]
    i = 1   # a = 4.0
    m = ps.ModelAB(2, (32, 32, 1), ps.make_cell(2, "SQUARE", a_tab[i]), (51, 51), 30.0,
                   lam=(0.05, 0.05, 5.0), mde=mde, scft=scft, n_anderson=5)
    m.set_fields(golden["lam2d_wA"], golden["lam2d_wB"])
    r = _converge(m, 1e-6)
    assert r < 1e-6
    # the 2D runs stopped at residual 1e-6: H is pinned to that level
    assert abs(m.H()[0] - F_tab[i]) < 1e-6, (m.H()[0], F_tab[i])


@pytest.mark.parametrize("shape,L", [((32, 32, 32), (3.6, 3.8, 4.0)), ((48, 48, 48), (3.8, 4.0, 4.2)),
                                     ((64, 64, 64), (4.2, 4.2, 4.2))])
@pytest.mark.parametrize("scft", ["EM", "Anderson"])
def test_persistent_sweep_matches_oracle(ps, shape, L, scft):
    """3D grids that run the persistent cooperative sweep (one launch per
    propagator sweep) against the oracle, short chains."""
    oracle.set_threads(oracle.max_threads())
    o, m = _models(ps, 3, shape, L, (9, 13), 20.0, scft=scft, n_anderson=3)
    assert m.launches_per_propagate() == 1
    wA, wB = _seed_fields(shape, 21)
    o.init_fields(wA, wB)
    m.set_fields(wA, wB)
    for n in (1, 2):
        o.update(n)
        m.update(n)
        assert abs(m.Q() - o.Q()) / o.Q() < 1e-10
        assert abs(m.H()[0] - o.H()[0]) / abs(o.H()[0]) < 1e-10
        for f in ("phiA", "phiB", "wA", "wB"):
            assert np.abs(m.get(f) - o.get(f)).max() < 1e-10, f
    for f in ("qA", "qB", "qAc", "qBc"):
        assert _rel(m.get(f), o.get(f)) < 1e-12, f


def test_full_size_chain_symmetry(ps):
    """At the full 64^3, Ns = 200 size: the RQM4 step operator is symmetric,
    so mean(q_N) of the forward chain equals mean(q^dagger_N) of the
    complementary chain; and densities integrate to fA, fB within the
    contour quadrature error."""
    from polystring_b200 import workloads
    cfg = workloads.config("C2")
    cell = ps.make_cell(3, "CUBIC", cfg["cell"][1][0])
    m = ps.ModelAB(3, cfg["shape"], cell, cfg["Ms"], cfg["chiN"], lam=cfg["lam"], scft="Anderson", n_anderson=20)
    m.set_fields(cfg["wA"], cfg["wB"])
    for _ in range(3):
        m.update(1)
        qB = m.get("qB")[-1]
        qAc = m.get("qAc")[-1]
        assert abs(qB.mean() - qAc.mean()) / qB.mean() < 1e-12
        fa = m.get("phiA").mean()
        fb = m.get("phiB").mean()
        assert abs(fa + fb - 1.0) < 1e-6
        assert abs(fa - 70.0 / 200.0) < 1e-3


@pytest.mark.parametrize("engine", ["sweep64", "generic", "line_passes"])
def test_64cube_engines_agree_with_oracle(ps, engine, monkeypatch):
    """The three GPU code paths for a 64^3 grid (specialised persistent sweep,
    generic persistent sweep, per-pass launches) against the oracle."""
    if engine == "generic":
        monkeypatch.setenv("PS_B200_GENERIC_SWEEP", "1")
    if engine == "line_passes":
        monkeypatch.setenv("PS_B200_LINE_PASSES", "1")
    oracle.set_threads(oracle.max_threads())
    shape = (64, 64, 64)
    o, m = _models(ps, 3, shape, (4.2, 4.2, 4.2), (11, 17), 25.0, scft="Anderson", n_anderson=4)
    assert (m.launches_per_propagate() == 1) == (engine != "line_passes")
    wA, wB = _seed_fields(shape, 8)
    o.init_fields(wA, wB)
    m.set_fields(wA, wB)
    o.update(2)
    m.update(2)
    assert abs(m.Q() - o.Q()) / o.Q() < 1e-10
    assert abs(m.H()[0] - o.H()[0]) / abs(o.H()[0]) < 1e-10
    for f in ("phiA", "phiB", "wA", "wB"):
        assert np.abs(m.get(f) - o.get(f)).max() < 1e-10, f
    for f in ("qA", "qB", "qAc", "qBc"):
        assert _rel(m.get(f), o.get(f)) < 1e-12, f
