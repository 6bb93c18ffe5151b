"""String method on the GPU (all images batched) against the CPU oracle."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ps():
    oracle.build()
    import polystring_b200
    return polystring_b200


def _images(m, shape, L, seed):
    from polystring_b200 import workloads
    return workloads.string_images(m=m, shape=shape, L=L, seed=seed)


@pytest.mark.parametrize("mde", ["RQM4", "OS2"])
def test_string_iterations_match_oracle(ps, mde):
    m, shape, L, Ms, chiN = 6, (32, 32, 1), 4.0, (17, 25), 18.0
    wa, wb = _images(m, shape, L, 3)
    end_a = (wa[0].copy(), wa[-1].copy())
    end_b = (wb[0].copy(), wb[-1].copy())
    o = oracle.ModelAB(2, shape, (L, L), Ms, chiN, lam=(0.05, 0.05, 5.0), mde=mde)
    g = ps.StringAB(m, 2, shape, ps.make_cell(2, "SQUARE", L), Ms, chiN, lam=(0.05, 0.05, 5.0), mde=mde, max_iter=3)
    g.set_images(wa, wb)
    wa_o, wb_o = wa.copy(), wb.copy()
    for it in range(3):
        Ho, So = oracle.string_iteration(o, wa_o, wb_o, end_a, end_b, 3)
        g.iterate(1)
        np.testing.assert_allclose(g.H(), Ho, rtol=1e-10, atol=0)
        np.testing.assert_allclose(g.S(), So, rtol=1e-10, atol=1e-12)
        assert np.abs(g.get("wa") - wa_o).max() < 1e-9
        assert np.abs(g.get("wb") - wb_o).max() < 1e-9


def test_full_string_properties(ps):
    """The 40-image 128x128 string: ends are restored bit-exactly, S runs from
    0 to 1 monotonically, H is finite for every image, and the batched run
    matches a sequential per-image run of the same model on the GPU."""
    from polystring_b200 import workloads
    m, shape, L = 40, (128, 128, 1), 8.0
    Ms = workloads.ms_from(0.35, 128)
    wa, wb = workloads.string_images(m=m, shape=shape, L=L)
    g = ps.StringAB(m, 2, shape, ps.make_cell(2, "SQUARE", L), Ms, 18.0, max_iter=3)
    g.set_images(wa, wb)
    g.iterate(2)
    H, S = g.H(), g.S()
    assert np.all(np.isfinite(H))
    assert S[0] == 0.0 and S[-1] == 1.0 and np.all(np.diff(S) > 0)
    ga = g.get("wa")
    assert np.array_equal(ga[0], wa[0]) and np.array_equal(ga[-1], wa[-1])
    # the first image's first string iteration equals a plain single-model run
    g2 = ps.StringAB(m, 2, shape, ps.make_cell(2, "SQUARE", L), Ms, 18.0, max_iter=3)
    g2.set_images(wa, wb)
    g2.iterate(1)
    single = ps.ModelAB(2, shape, ps.make_cell(2, "SQUARE", L), Ms, 18.0)
    for s in (0, 17, 39):
        single.set_fields(wa[s], wb[s])
        single.update(3)
        assert abs(single.H()[0] - g2.H()[s]) < 1e-11 * abs(single.H()[0])
