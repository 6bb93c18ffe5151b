"""Independent solves of uneven grids, contour lengths and parameters in one
batch (grouped line passes, one graph per batch iteration): every member
follows exactly the trajectory of the same solve run alone, and matches the
oracle."""
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
    if dim == 2:
        return ps.make_cell(2, "RECTANGULAR", L[0], L[1])
    return ps.make_cell(3, "ORTHORHOMBIC", L[0], L[1], L[2])


# (dim, shape, lengths, Ms, chiN, scft): uneven grids, Ns from 18 to 72, both
# mixing schemes; 2D and 3D members run in separate groups of the same batch
SOLVES = [
    (3, (16, 16, 16), (3.8, 4.0, 4.2), (13, 21), 20.0, "EM"),
    (3, (24, 16, 32), (4.1, 3.6, 4.4), (31, 43), 16.0, "Anderson"),
    (3, (32, 24, 16), (4.4, 4.0, 3.9), (7, 13), 24.0, "EM"),
    (3, (16, 48, 16), (3.9, 4.6, 4.0), (21, 33), 18.0, "Anderson"),
    (2, (64, 32, 1), (4.2, 3.9), (17, 29), 22.0, "EM"),
    (2, (32, 32, 1), (4.0, 4.0), (31, 71), 20.0, "Anderson"),
]


def _fields(shape, seed):
    rng = np.random.default_rng(seed)
    wA = 0.5 * rng.uniform(-1, 1, shape)
    wB = -wA + 0.1 * rng.uniform(-1, 1, shape)
    return wA, wB


def _spec(ps, s):
    dim, shape, L, Ms, chiN, scft = s
    return dict(dim=dim, shape=shape, cell=_cell(ps, dim, L), Ms=Ms, chiN=chiN, scft=scft, n_anderson=4)


def test_batch_members_follow_their_single_solves_exactly(ps, monkeypatch):
    # batch members run the default FFT schedules; untuned single solves do too
    monkeypatch.setenv("PS_B200_AUTOTUNE", "0")
    b = ps.BatchAB([_spec(ps, s) for s in SOLVES])
    singles = []
    for k, s in enumerate(SOLVES):
        wA, wB = _fields(s[1], 100 + k)
        b.set_fields(k, wA, wB)
        m = ps.ModelAB(**_spec(ps, s))
        m.set_fields(wA, wB)
        singles.append(m)
    for n in (1, 3):
        b.update(n)
        for k, m in enumerate(singles):
            m.update(n)
            assert b.H(k) == m.H(), (k, b.H(k), m.H())
            for f in ("phiA", "phiB", "wA", "wB"):
                assert np.array_equal(b.get(k, f), m.get(f)), (k, f)
            assert b.residual_error(k) == m.residual_error()
    assert b.launches_per_iteration() > 0


def test_batch_member_matches_oracle(ps):
    dim, shape, L, Ms, chiN, scft = SOLVES[1]
    b = ps.BatchAB([_spec(ps, s) for s in SOLVES[:3]])
    cell = _cell(ps, dim, L)
    g, l = oracle.unit_cell(dim, cell.system, cell.a, cell.b, cell.c)
    o = oracle.ModelAB(dim, shape, tuple(l[:dim]), Ms, chiN, g=g, scft=scft, n_anderson=4)
    for k, s in enumerate(SOLVES[:3]):
        b.set_fields(k, *_fields(s[1], 7 + k))
    o.init_fields(*_fields(shape, 8))
    b.update(4)
    o.update(4)
    assert abs(b.H(1)[0] - o.H()[0]) / abs(o.H()[0]) < 1e-10
    for f in ("phiA", "phiB", "wA", "wB"):
        assert np.abs(b.get(1, f) - o.get(f)).max() < 1e-10, f


def test_batch_rejects_what_it_cannot_run(ps):
    good = _spec(ps, SOLVES[0])
    with pytest.raises(ps.PSError) as e:
        ps.BatchAB([good, dict(good, mde="OS2")])
    assert e.value.code == -2
    with pytest.raises(ps.PSError) as e:
        ps.BatchAB([dict(good, shape=(12, 16, 16))])
    assert e.value.code == -2
    b = ps.BatchAB([good, good])
    b.set_fields(0, *_fields(good["shape"], 1))
    with pytest.raises(ps.PSError) as e:
        b.update(1)
    assert e.value.code == -6


# cubic members take persistent sweeps: 32^3 and 48^3 solves of one shape share
# one cooperative launch (uneven Ns), 64^3 runs its own 64^3 sweep; a 16^3
# member stays on grouped line passes
CUBIC = [
    (3, (32, 32, 32), (3.8, 3.8, 3.8), (13, 21), 20.0, "Anderson"),
    (3, (32, 32, 32), (4.1, 4.1, 4.1), (31, 43), 16.0, "EM"),
    (3, (48, 48, 48), (4.4, 4.4, 4.4), (7, 13), 24.0, "EM"),
    (3, (64, 64, 64), (4.2, 4.2, 4.2), (9, 17), 18.0, "Anderson"),
    (3, (48, 48, 48), (3.9, 3.9, 3.9), (21, 33), 18.0, "Anderson"),
    (3, (16, 16, 16), (3.6, 3.6, 3.6), (11, 15), 20.0, "EM"),
]


def _cubic(ps, s):
    dim, shape, L, Ms, chiN, scft = s
    return dict(dim=dim, shape=shape, cell=ps.make_cell(3, "CUBIC", L[0]), Ms=Ms, chiN=chiN, scft=scft,
                n_anderson=4)


def test_batch_sweep_members_follow_their_single_solves_exactly(ps, monkeypatch):
    monkeypatch.setenv("PS_B200_AUTOTUNE", "0")
    b = ps.BatchAB([_cubic(ps, s) for s in CUBIC])
    singles = []
    for k, s in enumerate(CUBIC):
        wA, wB = _fields(s[1], 200 + k)
        b.set_fields(k, wA, wB)
        m = ps.ModelAB(**_cubic(ps, s))
        m.set_fields(wA, wB)
        singles.append(m)
    for n in (1, 2):
        b.update(n)
        # 2 shared sweep launches (32^3, 48^3), one 64^3 sweep, grouped passes
        # for the 16^3 member (Ns 24): fewer launches than the longest member
        # (Ns 72) would need alone on per-step passes
        assert 0 < b.launches_per_iteration() < 8 * 72
        for k, m in enumerate(singles):
            m.update(n)
            assert b.H(k) == m.H(), (k, b.H(k), m.H())
            for f in ("phiA", "phiB", "wA", "wB"):
                assert np.array_equal(b.get(k, f), m.get(f)), (k, f)


def test_batch_sweep_chunks_beyond_resident_ctas(ps, monkeypatch):
    """149 solves of 32^3 split into several cooperative launches (as many
    solves a launch as can each have the 16 CTAs a 32^3 sweep keeps busy,
    taken in order of Ns) and still follow their single solves exactly."""
    monkeypatch.setenv("PS_B200_AUTOTUNE", "0")
    n = 149
    spec = lambda k: dict(dim=3, shape=(32, 32, 32), cell=ps.make_cell(3, "CUBIC", 3.8 + 0.01 * (k % 7)),
                          Ms=(5, 7 + (k % 3)), chiN=18.0 + 0.1 * (k % 5), scft="EM")
    b = ps.BatchAB([spec(k) for k in range(n)])
    fields = [_fields((32, 32, 32), 300 + k) for k in range(n)]
    for k in range(n):
        b.set_fields(k, *fields[k])
    b.update(2)
    for k in (0, 147, 148):
        m = ps.ModelAB(**spec(k))
        m.set_fields(*fields[k])
        m.update(2)
        assert b.H(k) == m.H(), (k, b.H(k), m.H())
        assert np.array_equal(b.get(k, "phiA"), m.get("phiA")), k
