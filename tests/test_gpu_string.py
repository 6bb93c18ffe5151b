"""String method on the GPU (all images batched) against the CPU oracle."""
import os

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


@pytest.mark.parametrize("mde,path", [("RQM4", "cluster"), ("RQM4", "line_passes"), ("OS2", "line_passes")])
def test_string_iterations_match_oracle(ps, mde, path, monkeypatch):
    """RQM4 on 32x32 runs the cluster-resident sweep (one launch per SCFT
    iteration: 2 + 3 * (1 + 5) + 7 launches per string iteration) unless
    PS_B200_LINE_PASSES=1 selects the batched line passes."""
    if path == "line_passes":
        monkeypatch.setenv("PS_B200_LINE_PASSES", "1")
    m, shape, L, Ms, chiN = 6, (32, 32, 1), 4.0, (17, 25), 18.0
    wa, wb = _images(m, shape, L, 3)
    end_a = (wa[0].copy(), wa[-1].copy())
    end_b = (wb[0].copy(), wb[-1].copy())
    o = oracle.ModelAB(2, shape, (L, L), Ms, chiN, lam=(0.05, 0.05, 5.0), mde=mde)
    g = ps.StringAB(m, 2, shape, ps.make_cell(2, "SQUARE", L), Ms, chiN, lam=(0.05, 0.05, 5.0), mde=mde, max_iter=3)
    assert (g.launches_per_iteration() == 27) == (path == "cluster")
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


@pytest.mark.parametrize("shape,L", [((64, 64, 1), 6.0), ((128, 128, 1), 8.0)])
def test_cluster_sweep_matches_line_passes(ps, shape, L, monkeypatch):
    """The cluster-resident sweep and the batched line passes give the same
    string iteration (two FFT orders, so equal to rounding)."""
    from polystring_b200 import workloads
    m = 9
    Ms = workloads.ms_from(0.35, 128)
    wa, wb = workloads.string_images(m=m, shape=shape, L=L, seed=5)
    out = {}
    for path in ("cluster", "line_passes"):
        if path == "line_passes":
            monkeypatch.setenv("PS_B200_LINE_PASSES", "1")
        g = ps.StringAB(m, 2, shape, ps.make_cell(2, "SQUARE", L), Ms, 18.0, max_iter=3)
        assert (g.launches_per_iteration() == 27) == (path == "cluster")
        g.set_images(wa, wb)
        g.iterate(2)
        out[path] = (g.H(), g.get("wa"), g.get("phiA"))
        del g
    Hc, wc, pc = out["cluster"]
    Hl, wl, pl = out["line_passes"]
    np.testing.assert_allclose(Hc, Hl, rtol=1e-12, atol=0)
    assert np.abs(wc - wl).max() < 1e-11 * np.abs(wl).max()
    assert np.abs(pc - pl).max() < 1e-11


def test_cluster_sweep_more_images_than_fit(ps, monkeypatch):
    """64 images of 128^2 need 512 CTAs, more than are resident at once (48
    clusters of 8): the clusters beyond run in later waves, with the same
    results as the batched line passes; the tuning log reports the fit."""
    from polystring_b200 import workloads
    m, shape, L = 64, (128, 128, 1), 8.0
    Ms = workloads.ms_from(0.35, 128)
    wa, wb = workloads.string_images(m=m, shape=shape, L=L, seed=9)
    out = {}
    for path in ("cluster", "line_passes"):
        if path == "line_passes":
            monkeypatch.setenv("PS_B200_LINE_PASSES", "1")
        g = ps.StringAB(m, 2, shape, ps.make_cell(2, "SQUARE", L), Ms, 18.0, max_iter=2)
        g.set_images(wa, wb)
        g.iterate(1)
        out[path] = (g.H(), g.get("phiA"))
        del g
    log = ps.lib().ps_tuning_log().decode()
    assert "cluster sweep: 8 CTAs per problem" in log and "batch 64" in log
    np.testing.assert_allclose(out["cluster"][0], out["line_passes"][0], rtol=1e-12, atol=0)
    assert np.abs(out["cluster"][1] - out["line_passes"][1]).max() < 1e-11


def test_sharded_contexts_equal_the_whole_string(ps):
    """Two contexts on one GPU, each relaxing part of the images
    (ps_string_ab_create_shard), exchanging the relaxed blocks of wa and wb
    as the ranks' all-gather would, then re-parameterising the whole string:
    H, S and fields bit-identical to one context running the whole string;
    and the rank orchestration (string_dist.ShardedString) on one rank equals
    it too."""
    import torch
    from polystring_b200 import workloads
    from polystring_b200.dist import Ranks
    from polystring_b200.string_dist import CudaStringBackend, ShardedString
    m, shape, L = 12, (128, 128, 1), 8.0
    Ms = workloads.ms_from(0.35, 128)
    cell = ps.make_cell(2, "SQUARE", L)
    wa, wb = workloads.string_images(m=m, shape=shape, L=L, seed=6)
    whole = ps.StringAB(m, 2, shape, cell, Ms, 18.0, max_iter=2)
    whole.set_images(wa, wb)
    halves = [CudaStringBackend(ps, m, lo, hi, 2, shape, cell, Ms, 18.0, max_iter=2) for lo, hi in ((0, 5), (5, m))]
    for h in halves:
        h.set_images(wa, wb)
    for it in range(2):
        whole.iterate(1)
        for h in halves:
            h.relax()
        for h in halves:
            h.sync()
        full = {f: torch.cat([h.block(f) for h in halves]).clone() for f in ("wa", "wb")}
        H = torch.cat([h.H_local() for h in halves]).cpu().numpy()
        for h in halves:
            for f in ("wa", "wb"):
                h.set_all(f, full[f])
            h.reparameterize()
            h.sync()
        assert np.array_equal(H, whole.H()), it
        for h in halves:
            assert np.array_equal(h.S(), whole.S()), it
            assert np.array_equal(h.get("wa"), whole.get("wa")), it
            assert np.array_equal(h.get("wb"), whole.get("wb")), it
    for k in ("RANK", "WORLD_SIZE"):
        os.environ.pop(k, None)
    st = ShardedString(Ranks(), m, lambda lo, hi: CudaStringBackend(ps, m, lo, hi, 2, shape, cell, Ms, 18.0,
                                                                      max_iter=2))
    st.backend.set_images(wa, wb)
    ref = ps.StringAB(m, 2, shape, cell, Ms, 18.0, max_iter=2)
    ref.set_images(wa, wb)
    for it in range(2):
        H = st.iterate(1)
        ref.iterate(1)
        assert np.array_equal(H, ref.H()), it
        assert np.array_equal(st.S(), ref.S()), it
        assert np.array_equal(st.backend.get("wa"), ref.get("wa")), it
