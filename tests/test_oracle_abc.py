"""The oracle's linear ABC triblock (scft_oracle.c, Model_ABC block): the
model is defined in this project (the reference has no periodic ABC melt),
so its restatement is checked against identities instead of reference
outputs ("parity unpinned"):

* uniform fields: Q = exp(-sum_X fX wX), phiX = fX exactly;
* an A-B-C chain whose C block is chemically B (chiAC = chiAB, chiBC = 0,
  wC = wB, lamC = lamB) is an AB diblock with a B block of LB + LC steps:
  with the trapezoid rule (whose weights add across the B/C junction) its
  simple-mixing trajectory equals the oracle's Model_AB's to rounding.
"""
import numpy as np
import pytest

import oracle


@pytest.fixture(scope="module", autouse=True)
def built():
    oracle.build()


@pytest.mark.parametrize("scft", ["EM", "Anderson"])
def test_uniform_fields_are_exact(scft):
    shape, L = (8, 6, 4), (3.0, 3.5, 4.0)
    Ms = (21, 31, 11)
    m = oracle.ModelABC(3, shape, L, Ms, (15.0, 12.0, 20.0), scft=scft, n_anderson=4)
    m.init_fields(np.full(shape, 0.1), np.full(shape, 0.2), np.full(shape, 0.3))
    m.update(1)
    Lx = [s - 1 for s in Ms]
    f = [l / sum(Lx) for l in Lx]
    assert abs(m.Q() - np.exp(-(0.1 * f[0] + 0.2 * f[1] + 0.3 * f[2]))) < 1e-14
    for name, fx in zip(("phiA", "phiB", "phiC"), f):
        assert np.abs(m.get(name) - fx).max() < 1e-14


def test_c_block_of_b_chemistry_is_the_ab_diblock():
    shape, L = (32, 1, 1), (4.0,)
    x = np.arange(32) / 32
    wA = (2.0 * np.cos(2 * np.pi * x)).reshape(shape)
    wB = -wA + 0.1 * np.sin(4 * np.pi * x).reshape(shape)
    chiN = 16.0
    abc = oracle.ModelABC(1, shape, L, (21, 17, 15), (chiN, 0.0, chiN), lam=(0.05, 0.05, 0.05, 2.0),
                          scft="EM", contour="trapezoid")
    ab = oracle.ModelAB(1, shape, L, (21, 31), chiN, lam=(0.05, 0.05, 2.0), scft="EM", contour="trapezoid")
    abc.init_fields(wA, wB, wB)
    ab.init_fields(wA, wB)
    for _ in range(4):
        abc.update(10)
        ab.update(10)
        assert abs(abc.H()[0] - ab.H()[0]) < 1e-12 * abs(ab.H()[0])
        assert abs(abc.Q() - ab.Q()) < 1e-12 * ab.Q()
        assert np.abs(abc.get("phiA") - ab.get("phiA")).max() < 1e-12
        assert np.abs(abc.get("phiB") + abc.get("phiC") - ab.get("phiB")).max() < 1e-12
        assert np.abs(abc.get("wB") - abc.get("wC")).max() < 1e-12
        assert np.abs(abc.get("wA") - ab.get("wA")).max() < 1e-12


def test_anderson_converges_and_eta_balances_the_targets():
    """Three-field Anderson from seeded noise reaches a small residual, and
    eta makes the targets sum to the current fields."""
    shape, L = (12, 12, 12), (4.0, 4.0, 4.0)
    w = 0.1 * np.random.default_rng(1).standard_normal((3,) + shape)
    chi = (18.0, 14.0, 25.0)
    m = oracle.ModelABC(3, shape, L, (21, 21, 23), chi, scft="Anderson", n_anderson=10).init_fields(*w)
    m.update(1)
    a, b, c = (m.get(n) for n in ("phiA", "phiB", "phiC"))
    eta = m.get("yita")
    tgt = (chi[0] * b + chi[2] * c + eta) + (chi[0] * a + chi[1] * c + eta) + (chi[2] * a + chi[1] * b + eta)
    np.testing.assert_allclose(tgt, w[0] + w[1] + w[2], atol=1e-12)
    m.update(149)
    assert m.residual() < 1e-4
