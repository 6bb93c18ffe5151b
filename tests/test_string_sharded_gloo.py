"""The string method with its images partitioned over ranks
(polystring_b200/string_dist.py), on gloo ranks on the CPU.

The per-rank work runs on a CPU backend built on the oracle (the SCFT of an
image, arc length and spline re-sampling restated from polystring_AB.cc);
what is under test is the partition of the images, the all-gather of the
relaxed fields and of H, and the replicated re-parameterisation: H, S and the
fields after every string iteration must be bit-identical to a single-rank
run.  On hardware the same orchestration drives CudaStringBackend with NCCL;
that multi-GPU run is not measured here (one GPU per run)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import oracle

SHAPE, L, MS, CHIN, LAM, MAX_ITER, M_IMAGES = (16, 16, 1), 4.0, (9, 13), 18.0, (0.05, 0.05, 5.0), 2, 7


class OracleStringBackend:
    """Backend of ShardedString on the CPU: images [lo, hi) relaxed by the
    oracle's Model_AB, the whole string kept as numpy arrays."""

    device = torch.device("cpu")

    def __init__(self, lo, hi, wa, wb):
        oracle.build()
        self.lo, self.hi = lo, hi
        self.wa, self.wb = wa.copy(), wb.copy()
        self.ends_a = (wa[0].copy(), wa[-1].copy())
        self.ends_b = (wb[0].copy(), wb[-1].copy())
        self.model = oracle.ModelAB(2, SHAPE, (L, L), MS, CHIN, lam=LAM)
        self.H = np.full(wa.shape[0], np.nan)
        self._S = None

    def relax(self):
        for s in range(self.lo, self.hi):
            self.model.init_fields(self.wa[s], self.wb[s])
            self.model.update(MAX_ITER)
            self.H[s] = self.model.H()[0]
            self.wa[s] = self.model.get("wA")
            self.wb[s] = self.model.get("wB")

    def sync(self):
        pass

    def block(self, name):
        a = getattr(self, name)[self.lo:self.hi]
        return torch.from_numpy(a.reshape(a.shape[0], -1).copy())

    def set_all(self, name, full):
        getattr(self, name)[...] = full.numpy().reshape(getattr(self, name).shape)

    def reparameterize(self):
        self._S = oracle.string_arclength(self.wa)
        oracle.string_redistribute(self.wa, self._S, *self.ends_a)
        oracle.string_redistribute(self.wb, self._S, *self.ends_b)

    def H_local(self):
        return torch.from_numpy(self.H[self.lo:self.hi].copy())

    def S(self):
        return self._S


def _initial():
    from polystring_b200 import workloads
    return workloads.string_images(m=M_IMAGES, shape=SHAPE, L=L, seed=4)


def _run(ranks, iters):
    from polystring_b200.string_dist import ShardedString
    wa, wb = _initial()
    backends = {}

    def make(lo, hi):
        backends["b"] = OracleStringBackend(lo, hi, wa, wb)
        return backends["b"]
    st = ShardedString(ranks, M_IMAGES, make)
    out = []
    for _ in range(iters):
        H = st.iterate(1)
        b = backends["b"]
        out.append((H.copy(), st.S().copy(), b.wa.copy(), b.wb.copy()))
    return out, (st.lo, st.hi)


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from polystring_b200.dist import Ranks
    r = Ranks("gloo", timeout_s=60)
    out, rng = _run(r, 2)
    r.close()
    q.put((rank, rng, out))


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_string_is_bit_identical_to_one_rank(world):
    from polystring_b200.dist import Ranks
    for k in ("RANK", "WORLD_SIZE"):
        os.environ.pop(k, None)
    single, _ = _run(Ranks(), 2)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(k, world, port, q)) for k in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in range(world)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # the shards cover every image once, in order
    assert [i for _, rng, _ in res for i in range(*rng)] == list(range(M_IMAGES))
    for rank, _, out in res:
        for it, ((H, S, wa, wb), (H1, S1, wa1, wb1)) in enumerate(zip(out, single)):
            assert np.array_equal(H, H1), (rank, it)
            assert np.array_equal(S, S1), (rank, it)
            assert np.array_equal(wa, wa1), (rank, it)
            assert np.array_equal(wb, wb1), (rank, it)
