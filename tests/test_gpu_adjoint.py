"""Adjoint of the RQM4 chain on the GPU: w-gradients of a density-target loss
and the cell stress, against central finite differences of the GPU forward
map, and against the density identity d(-ln Q)/dw_A = phi_A / M."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ps():
    import polystring_b200
    return polystring_b200


def _fields(shape, seed, amp=0.8):
    rng = np.random.default_rng(seed)
    wA = amp * rng.uniform(-1, 1, shape)
    wB = -wA + 0.2 * rng.uniform(-1, 1, shape)
    return wA, wB


def _loss(m, wA, wB, target):
    m.set_fields(wA, wB)
    m.forward()
    return float(((m.get("phiA") - target) ** 2).sum())


CASES = [(2, (32, 32, 1), ("RECTANGULAR", (3.9, 4.3)), (17, 25)),
         (3, (16, 12, 8), ("ORTHORHOMBIC", (3.8, 4.0, 4.2)), (13, 21))]


@pytest.mark.parametrize("dim,shape,cell,Ms", CASES)
def test_loss_gradient_matches_finite_differences(ps, dim, shape, cell, Ms):
    c = ps.make_cell(dim, cell[0], *cell[1])
    m = ps.ModelAB(dim, shape, c, Ms, 20.0)
    wA, wB = _fields(shape, 4)
    rng = np.random.default_rng(9)
    target = rng.uniform(0, 1, shape)
    m.set_fields(wA, wB)
    m.forward()
    phiA = m.get("phiA")
    gA, gB = m.grad_w(2.0 * (phiA - target), np.zeros(shape), 0.0)
    # fourth-order central stencil at h = 1e-4: truncation ~h^4, rounding
    # ~eps * loss / h ~ 2e-10 for a loss summed over ~10^3 points
    h = 1e-4
    for trial in range(3):
        dA = rng.standard_normal(shape)
        dB = rng.standard_normal(shape)
        f = {k: _loss(m, wA + k * h * dA, wB + k * h * dB, target) for k in (-2, -1, 1, 2)}
        fd = (f[-2] - 8.0 * f[-1] + 8.0 * f[1] - f[2]) / (12.0 * h)
        an = float((gA * dA).sum() + (gB * dB).sum())
        assert abs(fd - an) <= 1e-8 * abs(an) + 1e-9, (trial, fd, an)


@pytest.mark.parametrize("dim,shape,cell,Ms", CASES)
def test_lnQ_gradient_is_the_density(ps, dim, shape, cell, Ms):
    """d(-ln Q)/dw_A(r) = phi_A(r)/M up to the contour discretisation."""
    c = ps.make_cell(dim, cell[0], *cell[1])
    m = ps.ModelAB(dim, shape, c, Ms, 20.0)
    wA, wB = _fields(shape, 5)
    m.set_fields(wA, wB)
    m.forward()
    Q = m.Q()
    M = np.prod(shape)
    gA, gB = m.grad_w(np.zeros(shape), np.zeros(shape), -1.0 / Q)
    assert np.abs(gA * M - m.get("phiA")).max() < 2e-3
    assert np.abs(gB * M - m.get("phiB")).max() < 2e-3


@pytest.mark.parametrize("dim,shape,cell,Ms", CASES)
def test_stress_matches_finite_differences_at_fixed_fields(ps, dim, shape, cell, Ms):
    wA, wB = _fields(shape, 6)
    L = list(cell[1])
    c = ps.make_cell(dim, cell[0], *L)
    m = ps.ModelAB(dim, shape, c, Ms, 20.0)
    m.set_fields(wA, wB)
    st = m.stress()
    # fourth-order central stencil at h = 1e-4 (rounding ~eps |ln Q| / h)
    h = 1e-4
    for i in range(dim):
        vals = {}
        for k in (-2, -1, 1, 2):
            Lp = list(L)
            Lp[i] += k * h
            mm = ps.ModelAB(dim, shape, ps.make_cell(dim, cell[0], *Lp), Ms, 20.0)
            mm.set_fields(wA, wB)
            mm.forward()
            vals[k] = -np.log(mm.Q())
        fd = (vals[-2] - 8.0 * vals[-1] + 8.0 * vals[1] - vals[2]) / (12.0 * h)
        assert abs(fd - st[i]) <= 1e-7 * abs(st[i]) + 1e-11, (i, fd, st[i])
    assert np.all(st[dim:] == 0.0)


def test_autograd_harness(ps):
    import torch
    from polystring_b200.autograd import DensityMap
    shape = (16, 16, 1)
    m = ps.ModelAB(2, shape, ps.make_cell(2, "SQUARE", 4.0), (13, 21), 18.0)
    wA, wB = _fields(shape, 7)
    tA = torch.tensor(wA, requires_grad=True)
    tB = torch.tensor(wB, requires_grad=True)
    target = torch.from_numpy(np.random.default_rng(1).uniform(0, 1, shape))
    phiA, phiB, Q = DensityMap.apply(tA, tB, m)
    loss = ((phiA - target) ** 2).sum() + 0.3 * torch.log(Q)
    loss.backward()
    gA, gB = m.grad_w(2.0 * (phiA.detach().numpy() - target.numpy()), np.zeros(shape), 0.3 / Q.item())
    assert np.abs(tA.grad.numpy() - gA).max() == 0.0
    assert np.abs(tB.grad.numpy() - gB).max() == 0.0


def test_saddle_point_stress_matches_converged_free_energy(ps):
    """2D LAM (32x32, Ms [51, 51], chiN 30, the reference's example): the
    adjoint stress at the converged fields against the central difference of
    converged F(a).  The two differ by the contour-quadrature mismatch between
    the Simpson densities and the exact derivative of the discrete ln Q
    (bounded at 2e-3 pointwise above), so the check is relative 1e-3."""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "lam_pins.npz"))

    def converge(a):
        m = ps.ModelAB(2, (32, 32, 1), ps.make_cell(2, "SQUARE", a), (51, 51), 30.0, scft="Anderson", n_anderson=5)
        m.set_fields(g["lam2d_wA"], g["lam2d_wB"])
        for it in range(800):
            m.update(20)
            if m.residual_error() < 1e-11:
                break
        return m

    a, h = 4.0, 1e-4
    m0 = converge(a)
    st = m0.stress()
    dFda = st[0] + st[1]
    Fp = converge(a + h).H()[0]
    Fm = converge(a - h).H()[0]
    fd = (Fp - Fm) / (2 * h)
    assert abs(fd - dFda) <= 1e-3 * abs(dFda), (fd, dFda)


@pytest.mark.parametrize("dim,shape,cell,Ms", CASES)
def test_checkpointed_stress_equals_full_history_stress(ps, dim, shape, cell, Ms):
    """sqrt(Ns) checkpoints (and other segment lengths): the forward chain is
    recomputed segment by segment during the reverse sweep; the stress agrees
    with the full-history one to rounding (the recomputation runs the chain
    without its packed partner, which changes roundings only)."""
    c = ps.make_cell(dim, cell[0], *cell[1])
    m = ps.ModelAB(dim, shape, c, Ms, 20.0)
    m.set_fields(*_fields(shape, 6))
    full = m.stress()
    Ns = sum(Ms) - 2
    for k in (0, 1, 5, Ns - 1, Ns):
        ck = m.stress(checkpoints=k)
        for i in range(dim):
            assert abs(ck[i] - full[i]) <= 1e-10 * abs(full[i]), (k, i, ck[i], full[i])


def test_c4_full_size_adjoint(ps):
    """The adjoint at the full C4 size: 48^3 orthorhombic (3.8, 4.0, 4.2),
    fA 0.30, chiN 22, Ns 128 (Ms [39, 91]), fields converged by Anderson
    mixing (residual 1e-9) from the seeded start (noise plus an ordered
    seed), an ordered structure whose stress is 5e-4..7e-3 in every axis.

    * stress with the full history and with sqrt(Ns) checkpoints agree to
      1e-8 of the largest component;
    * the stress agrees with fourth-order central differences of -ln Q
      (h = 1e-4) to 1e-7 relative per component, and with second-order ones
      at h = 1e-6 to their rounding floor (~1e-15 |ln Q| / h ~ 1e-9);
    * dLoss/dw for Loss = ||phiA - phi_target||^2 agrees with fourth-order
      central differences (h = 1e-3) to 1e-8 relative, along the gradient and
      along the gradient modulated by a smooth seeded field (directions with
      a large projection on the gradient, so the check is not a cancellation);
    * d(-ln Q)/dwA = phiA / M to the contour rule's accuracy."""
    from polystring_b200 import workloads as wl
    cfg = wl.config("C4")
    m = wl.model_of(ps, cfg)
    m.set_fields(cfg["wA"], cfg["wB"])
    it, res = wl.converge(m, 1e-9, 2000)
    assert res < 1e-8, (it, res)
    wA, wB = m.get("wA"), m.get("wB")
    assert np.ptp(m.get("phiA")) > 0.5          # ordered, not the disordered saddle
    m.set_fields(wA, wB)
    st = m.stress()
    ck = m.stress(checkpoints=0)
    assert np.abs(st).min() > 1e-4, st
    for i in range(3):
        # the checkpointed sweep recomputes q without its packed partner: a
        # rounding difference, 1e-8 of the largest component at most
        assert abs(ck[i] - st[i]) <= 1e-8 * np.abs(st).max(), (i, ck[i], st[i])
        fd4 = wl.stress_fd(ps, cfg, wA, wB, i, 1e-4, order=4)
        assert abs(fd4 - st[i]) <= 1e-7 * abs(st[i]), (i, fd4, st[i])
        fd2 = wl.stress_fd(ps, cfg, wA, wB, i, 1e-6, order=2)
        assert abs(fd2 - st[i]) <= 1e-6 * np.abs(st).max(), (i, fd2, st[i])
    tgt = wl.smoothed_target(cfg["shape"])
    m.forward()
    phiA, Q = m.get("phiA"), m.Q()
    gA, gB = m.grad_w(2.0 * (phiA - tgt), np.zeros(cfg["shape"]), 0.0)
    sc = max(np.abs(gA).max(), np.abs(gB).max())
    mod = 1.0 + wl.smoothed_target(cfg["shape"], seed=21)
    for dA, dB in ((gA / sc, gB / sc), (gA * mod / sc, gB * mod / sc)):
        fd = wl.loss_fd(m, wA, wB, dA, dB, tgt, 1e-3)
        an = float((gA * dA).sum() + (gB * dB).sum())
        assert abs(fd - an) <= 1e-8 * abs(an), (fd, an)
    m.forward()
    M = np.prod(cfg["shape"])
    lA, lB = m.grad_w(np.zeros(cfg["shape"]), np.zeros(cfg["shape"]), -1.0 / Q)
    assert np.abs(lA * M - m.get("phiA")).max() < 1e-3
    assert np.abs(lB * M - m.get("phiB")).max() < 1e-3
