"""The linear ABC triblock on the device (csrc/model_abc.cu) against the
oracle's restatement (oracle/scft_oracle.c, Model_ABC block) at the parity
bar: 1e-10 relative on Q and H, 1e-10 max-abs on densities and relative to
max |w| on the fields, every 5 of 20 iterations of simple and Anderson
mixing; and the AB-reduction identity
(C block of B chemistry, trapezoid rule) against the device Model_AB."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ps():
    oracle.build()
    import polystring_b200
    return polystring_b200


def _cell(ps, dim, L):
    if dim == 1:
        return ps.make_cell(1, "LAMELLAR", L[0])
    if dim == 2:
        return ps.make_cell(2, "RECTANGULAR", L[0], L[1])
    return ps.make_cell(3, "ORTHORHOMBIC", L[0], L[1], L[2])


def test_uniform_fields_are_exact(ps):
    shape = (16, 12, 8)
    Ms = (21, 31, 11)
    m = ps.ModelABC(3, shape, _cell(ps, 3, (3.0, 3.5, 4.0)), Ms, (15.0, 12.0, 20.0))
    m.set_fields(np.full(shape, 0.1), np.full(shape, 0.2), np.full(shape, 0.3))
    m.update(1)
    Lx = [s - 1 for s in Ms]
    f = [l / sum(Lx) for l in Lx]
    assert abs(m.Q() - np.exp(-(0.1 * f[0] + 0.2 * f[1] + 0.3 * f[2]))) < 5e-14
    for name, fx in zip(("phiA", "phiB", "phiC"), f):
        assert np.abs(m.get(name) - fx).max() < 5e-14


# the 64^3 case runs on the 64^3 sweep (three factor sets), the 32^3 one on
# the generic sweep, the others on line passes
CASES = [(2, (32, 32, 1), (4.0, 4.0), (21, 31, 11), "EM"), (2, (24, 48, 1), (3.6, 4.4), (20, 24, 17), "Anderson"),
         (3, (16, 24, 32), (3.5, 3.8, 4.1), (21, 22, 23), "Anderson"), (3, (32, 32, 32), (4.2, 4.2, 4.2),
                                                                          (41, 45, 43), "Anderson"),
         (3, (64, 64, 64), (4.2, 4.4, 4.6), (21, 16, 25), "Anderson")]


@pytest.mark.parametrize("dim,shape,L,Ms,scft", CASES)
def test_abc_iterations_match_oracle(ps, dim, shape, L, Ms, scft):
    rng = np.random.default_rng(5)
    X = np.meshgrid(*[np.arange(n) / n for n in shape], indexing="ij")
    base = np.cos(2 * np.pi * X[0]) + (np.cos(2 * np.pi * X[1]) if dim > 1 else 0)
    w = [2.0 * base + 0.2 * rng.standard_normal(shape), -1.5 * base + 0.2 * rng.standard_normal(shape),
         0.3 * rng.standard_normal(shape)]
    chi = (18.0, 14.0, 25.0)
    lam = (0.05, 0.05, 0.05, 5.0)
    o = oracle.ModelABC(dim, shape, L, Ms, chi, lam=lam, scft=scft, n_anderson=10).init_fields(*w)
    m = ps.ModelABC(dim, shape, _cell(ps, dim, L), Ms, chi, lam=lam, scft=scft, n_anderson=10).set_fields(*w)
    for it in range(5, 21, 5):
        o.update(5)
        m.update(5)
        assert abs(m.Q() - o.Q()) / o.Q() < 1e-10, (it, m.Q(), o.Q())
        Ho, Hg = o.H()[0], m.H()[0]
        assert abs(Hg - Ho) / abs(Ho) < 1e-10, (it, Hg, Ho)
        for f in ("phiA", "phiB", "phiC", "wA", "wB", "wC"):
            ref = o.get(f)
            # densities max-abs; fields relative to their max-abs (Anderson
            # mixing amplifies rounding into the fields first: about 2e-10 of
            # max |w| by iteration 25 in 3D, so the comparison stops at 20)
            scale = 1.0 if f.startswith("phi") else np.abs(ref).max()
            d = np.abs(m.get(f) - ref).max() / scale
            assert d < 1e-10, (it, f, d)
        assert abs(m.residual_error() - o.residual()) <= 1e-8 * o.residual()


def test_c_block_of_b_chemistry_is_the_device_ab_diblock(ps):
    shape, L = (32, 48, 1), (4.0, 4.4)
    X = np.meshgrid(*[np.arange(n) / n for n in shape], indexing="ij")
    wA = 2.0 * np.cos(2 * np.pi * X[0])
    wB = -wA + 0.1 * np.sin(4 * np.pi * X[1])
    chiN = 16.0
    cell = _cell(ps, 2, L)
    abc = ps.ModelABC(2, shape, cell, (21, 17, 15), (chiN, 0.0, chiN), lam=(0.05, 0.05, 0.05, 2.0), scft="EM",
                      contour="trapezoid").set_fields(wA, wB, wB)
    ab = ps.ModelAB(2, shape, cell, (21, 31), chiN, lam=(0.05, 0.05, 2.0), scft="EM", contour="trapezoid")
    ab.set_fields(wA, wB)
    abc.update(20)
    ab.update(20)
    assert abs(abc.H()[0] - ab.H()[0]) < 1e-11 * abs(ab.H()[0])
    assert np.abs(abc.get("phiB") + abc.get("phiC") - ab.get("phiB")).max() < 1e-11
    assert np.abs(abc.get("wA") - ab.get("wA")).max() < 1e-11


def test_mixed_batch_members_equal_their_single_solves(ps):
    """AB and ABC solves in one batch (ps_batch_ab_create_mixed): the ABC
    members run in shared generic-sweep launches (32^3, 48^3), their own
    64^3 sweep (64^3) or grouped line-pass launches (64^2), and equal their
    single solves bit for bit; the AB members likewise."""
    rng = np.random.default_rng(9)
    ab = [dict(dim=3, shape=(32, 32, 32), cell=ps.make_cell(3, "CUBIC", 4.0), Ms=(21, 45), chiN=16.0,
               scft="Anderson", n_anderson=10),
          dict(dim=3, shape=(24, 32, 16), cell=ps.make_cell(3, "ORTHORHOMBIC", 3.6, 4.0, 3.2), Ms=(17, 31),
               chiN=20.0, scft="Anderson", n_anderson=10)]
    abc = [dict(dim=3, shape=(32, 32, 32), cell=ps.make_cell(3, "CUBIC", 4.4), Ms=(21, 22, 23),
                chi=(18.0, 14.0, 25.0), scft="Anderson", n_anderson=10),
           dict(dim=3, shape=(48, 48, 48), cell=ps.make_cell(3, "CUBIC", 4.8), Ms=(33, 30, 31),
                chi=(15.0, 20.0, 12.0), scft="Anderson", n_anderson=10),
           dict(dim=2, shape=(64, 64, 1), cell=ps.make_cell(2, "SQUARE", 4.0), Ms=(21, 21, 21),
                chi=(20.0, 20.0, 20.0), scft="EM"),
           dict(dim=3, shape=(64, 64, 64), cell=ps.make_cell(3, "CUBIC", 4.6), Ms=(17, 26, 21),
                chi=(16.0, 19.0, 22.0), scft="Anderson", n_anderson=10)]
    b = ps.BatchAB(ab, abc)
    fields = []
    for k, sv in enumerate(ab + abc):
        w = 0.1 * rng.standard_normal((3,) + sv["shape"])
        fields.append(w)
        if k < len(ab):
            b.set_fields(k, w[0], w[1])
        else:
            b.set_fields(k, w[0], w[1], w[2])
    b.update(3)
    for k, sv in enumerate(ab):
        m = ps.ModelAB(**sv)
        m.set_fields(fields[k][0], fields[k][1])
        m.update(3)
        assert b.H(k)[0] == m.H()[0]
        assert np.array_equal(b.get(k, "phiA"), m.get("phiA"))
    for j, sv in enumerate(abc):
        k = len(ab) + j
        m = ps.ModelABC(**sv).set_fields(*fields[k])
        m.update(3)
        assert b.H(k)[0] == m.H()[0], (k, b.H(k)[0], m.H()[0])
        for f in ("phiA", "phiC", "wB"):
            assert np.array_equal(b.get(k, f), m.get(f)), (k, f)
        assert b.residual_error(k) == m.residual_error()


@pytest.mark.parametrize("n", [32, 64])
def test_sweep_and_line_passes_agree(ps, monkeypatch, n):
    """A 32^3 triblock on the generic persistent sweep and a 64^3 one on the
    64^3 sweep (three factor sets a lane), against the packed line passes
    (PS_B200_LINE_PASSES=1 at creation)."""
    shape = (n, n, n)
    w = 0.1 * np.random.default_rng(4).standard_normal((3,) + shape)
    args = dict(dim=3, shape=shape, cell=ps.make_cell(3, "CUBIC", 4.2), Ms=(31, 25, 29), chi=(16.0, 22.0, 13.0),
                scft="Anderson", n_anderson=10)
    a = ps.ModelABC(**args).set_fields(*w)
    monkeypatch.setenv("PS_B200_LINE_PASSES", "1")
    b = ps.ModelABC(**args).set_fields(*w)
    monkeypatch.delenv("PS_B200_LINE_PASSES")
    a.update(4)
    b.update(4)
    assert abs(a.H()[0] - b.H()[0]) < 1e-12 * abs(b.H()[0])
    for f in ("phiA", "phiB", "phiC"):
        assert np.abs(a.get(f) - b.get(f)).max() < 1e-12
