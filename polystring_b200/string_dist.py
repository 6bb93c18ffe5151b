"""The string method with its images partitioned over ranks (one process per
GPU, torchrun environment).

The reference's string driver runs the SCFT of every image one after another
(scft/polystring_AB.cc:256-281); its archived threaded driver gives each
image a std::thread (scft/polystring_AB_back/polystring_AB_backThread.cc:
256-258, 412-423).  Here each rank relaxes a contiguous block of images
(dist.shard) on its own GPU; the images are independent inside an SCFT
relaxation, so the only exchange is one all-gather of the relaxed wa and wb
(and of H) per string iteration.  Every rank then runs the arc-length and
spline re-sampling step over the whole string itself (polystring_AB.cc:
283-329); that step is deterministic, so the ranks keep bit-identical
strings, equal to the single-rank run.

The exchange goes through torch.distributed (NCCL on GPUs, device tensors; gloo
on the CPU for the tests); the kernels read only their own GPU's memory.

A backend supplies the per-rank work:

    relax()                  SCFT of this rank's images (run_scftInString)
    block(name) -> tensor    this rank's images of "wa" / "wb", (n_local, M)
    set_all(name, tensor)    the whole string's field, (m, M)
    reparameterize()         arc length, re-sampling, ends, over all m images
    H_local() -> tensor      H of this rank's images, (n_local,)
    S() -> numpy             normalised arc length, (m,)
    sync()                   wait for the backend's queued device work
    device                   torch device of the tensors

CudaStringBackend is the GPU one (a ps_string_ab context created for the
rank's shard); the tests add a CPU one built on the oracle.
"""
import numpy as np

from .dist import shard


class _DeviceArray:
    """A CUDA array interface over device memory owned by the library, so that
    torch can view it without a copy."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class CudaStringBackend:
    """A sharded ps_string_ab context: the string fields of all m images live
    in the context's device memory; the rank relaxes images [lo, hi)."""

    def __init__(self, ps, m, lo, hi, dim, shape, cell, Ms, chiN, **kw):
        import torch
        self.torch = torch
        self.ctx = ps.StringAB(m, dim, shape, cell, Ms, chiN, shard=(lo, hi), **kw)
        self.m, self.lo, self.hi = m, lo, hi
        self.M = self.ctx.M
        self.device = torch.device("cuda", torch.cuda.current_device())

    def _view(self, name):
        return self.torch.as_tensor(_DeviceArray(self.ctx.device_ptr(name), (self.m, self.M)), device=self.device)

    def set_images(self, wa, wb):
        self.ctx.set_images(wa, wb)

    def relax(self):
        self.ctx.relax()

    def sync(self):
        self.ctx.synchronize()

    def block(self, name):
        return self._view(name)[self.lo:self.hi]

    def set_all(self, name, full):
        v = self._view(name)
        if full.data_ptr() != v.data_ptr():
            v.copy_(full)
        self.torch.cuda.current_stream(self.device).synchronize()

    def reparameterize(self):
        self.ctx.reparameterize()

    def H_local(self):
        return self.torch.from_numpy(self.ctx.H()[self.lo:self.hi].copy()).to(self.device)

    def S(self):
        return self.ctx.S()

    def get(self, name):
        return self.ctx.get(name)


class ShardedString:
    """polystring_AB's string iteration over the ranks of `ranks`
    (dist.Ranks); `make_backend(lo, hi)` builds this rank's backend for
    images [lo, hi)."""

    def __init__(self, ranks, m, make_backend):
        self.ranks = ranks
        self.m = m
        rng = shard(m, ranks.rank, ranks.world)
        self.lo, self.hi = rng.start, rng.stop
        if self.hi <= self.lo:
            raise ValueError("every rank needs at least one image (m >= world size)")
        self.sizes = [len(shard(m, r, ranks.world)) for r in range(ranks.world)]
        self.chunk = max(self.sizes)
        self.backend = make_backend(self.lo, self.hi)
        self.H = np.full(m, np.nan)

    def _gather(self, local):
        """Concatenate every rank's (n_r, ...) block in rank (= image) order."""
        import torch
        if self.ranks.world == 1:
            return local
        pad = torch.zeros((self.chunk,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
        pad[:local.shape[0]] = local
        parts = [torch.empty_like(pad) for _ in range(self.ranks.world)]
        self.ranks.dist.all_gather(parts, pad)
        return torch.cat([p[:n] for p, n in zip(parts, self.sizes)])

    def iterate(self, n=1):
        b = self.backend
        for _ in range(n):
            b.relax()
            b.sync()
            for name in ("wa", "wb"):
                b.set_all(name, self._gather(b.block(name)))
            self.H = self._gather(b.H_local()).cpu().numpy()
            b.reparameterize()
        b.sync()
        return self.H

    def S(self):
        return self.backend.S()
