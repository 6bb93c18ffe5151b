"""polystring_b200 -- B200 (sm_100a, FP64) implementation of PolyOrder's
periodic pseudospectral SCFT path behind the reference's Updater / Model
interface.

The compute path is libpolystring_b200.so (hand-written CUDA, C ABI in
include/polystring_b200.h); this module is a thin Python mirror of the
reference's classes over that ABI:

    RQM4(cell, Lx, Ly, Lz, ds).solve(qs, w)        src/RQM4.cc:9-93
    PseudoSpectral(cell, Lx, Ly, Lz, ds).solve(..)  src/PseudoSpectral.cc:190-261
    density(rule, q, qc, ds, cc)                    src/Simpson.cc, src/Quadrature4.cc
    ModelAB(...).update(), H(), residual_error()    src/Model_AB.cc:85-371

Host numpy arrays go through the host entry points; torch CUDA tensors go
through the "_device" entry points without copies.  There is no CPU
fallback: without the built library every entry point raises ImportError.
"""
import ctypes

import numpy as np

from . import capi
from .capi import PSError, make_cell, FIELDS, RULES

__all__ = ["RQM4", "PseudoSpectral", "ModelAB", "BatchAB", "density", "grid_mean", "make_cell", "PSError", "lib"]


def lib():
    """The loaded CUDA library; raises ImportError when it is not built."""
    return capi.load()


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class _Updater:
    scheme = None

    def __init__(self, cell, Lx, Ly, Lz, ds):
        h = ctypes.c_void_p()
        capi.check(lib().ps_updater_create(self.scheme, ctypes.byref(cell), Lx, Ly, Lz, ds, ctypes.byref(h)))
        self._h = h
        self.shape = (Lx, Ly, Lz)
        self.M = Lx * Ly * Lz

    def clone(self):
        h = ctypes.c_void_p()
        capi.check(lib().ps_updater_clone(self._h, ctypes.byref(h)))
        c = object.__new__(type(self))
        c._h, c.shape, c.M = h, self.shape, self.M
        return c

    def solve(self, qs, w, stream=None):
        """Updater::solve(Propagator& q, const Grid& w): qs (len, Lx, Ly, Lz),
        qs[0] is the head; slices 1.. are overwritten in place."""
        if _is_torch(qs):
            assert qs.is_cuda and w.is_cuda and qs.is_contiguous() and w.is_contiguous()
            capi.check(lib().ps_updater_solve_device(self._h, w.data_ptr(), qs.data_ptr(), qs.shape[0],
                                                     stream if stream is not None else None))
            return qs
        assert qs.dtype == np.float64 and qs.flags.c_contiguous
        w = _f64(w)
        capi.check(lib().ps_updater_solve(self._h, capi.dptr(w), capi.dptr(qs), qs.shape[0]))
        return qs

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().ps_updater_destroy(h)
            self._h = None


class RQM4(_Updater):
    """4th-order Richardson-extrapolated operator splitting (src/RQM4.cc)."""
    scheme = 0


class PseudoSpectral(_Updater):
    """2nd-order operator splitting, general-cell Laplacian (src/PseudoSpectral.cc)."""
    scheme = 1


class Etdrk4_PBC(_Updater):
    """Cox-Matthews ETDRK4 with contour-integral coefficients (src/Etdrk4_PBC.cc),
    M contour points (include/Etdrk4_PBC.h:47-51, default 32)."""
    scheme = 2

    def __init__(self, cell, Lx, Ly, Lz, ds, M=32):
        h = ctypes.c_void_p()
        capi.check(lib().ps_updater_create_etdrk4(ctypes.byref(cell), Lx, Ly, Lz, ds, M, ctypes.byref(h)))
        self._h = h
        self.shape = (Lx, Ly, Lz)
        self.M = Lx * Ly * Lz


def density(rule, q, qc, ds, cc):
    """phi = cc ds sum_s c_s q[s] qc[n-s] (Simpson / Quad4 / trapezoid)."""
    r = RULES[rule] if isinstance(rule, str) else int(rule)
    q = _f64(q)
    qc = _f64(qc)
    M = int(np.prod(q.shape[1:]))
    phi = np.zeros(q.shape[1:])
    capi.check(lib().ps_density_solve(r, capi.dptr(q), capi.dptr(qc), q.shape[0], M, ds, cc, capi.dptr(phi)))
    return phi


def grid_mean(x_cuda):
    """Grid::quadrature of a CUDA tensor (deterministic device reduction)."""
    out = ctypes.c_double()
    capi.check(lib().ps_grid_mean_device(x_cuda.data_ptr(), x_cuda.numel(), ctypes.byref(out), None))
    return out.value


def _params(dim, shape, cell, Ms, chiN, lam=(0.05, 0.05, 5.0), mde="RQM4", scft="EM", n_anderson=5,
            compressible=False, contour="Simpson", etdrk4_M=0):
    """ps_model_ab_params of one Model_AB (the [Model] / [Grid] / [Algorithm_*] values of a config)."""
    Lx, Ly, Lz = shape
    p = capi.ModelABParamsC()
    p.dim, p.Lx, p.Ly, p.Lz = dim, Lx, Ly, Lz
    p.cell = cell
    p.sA, p.sB = Ms
    p.chiN = chiN
    p.lamA, p.lamB, p.lamYita = lam
    p.mde = capi.MDE[mde.upper()]
    p.scft = capi.SCFT[scft.upper()]
    p.n_anderson = n_anderson
    p.compressible = 1 if compressible else 0
    p.contour = capi.CONTOUR[contour.upper()]
    p.etdrk4_M = etdrk4_M
    return p


class ModelAB:
    """Model_AB on the device: one SCFT iteration is one replay of a captured
    CUDA graph (propagators, Q, densities, field update)."""

    def __init__(self, dim, shape, cell, Ms, chiN, lam=(0.05, 0.05, 5.0), mde="RQM4", scft="EM",
                 n_anderson=5, compressible=False, contour="Simpson", etdrk4_M=0):
        Lx, Ly, Lz = shape
        p = _params(dim, shape, cell, Ms, chiN, lam, mde, scft, n_anderson, compressible, contour, etdrk4_M)
        h = ctypes.c_void_p()
        capi.check(lib().ps_model_ab_create(ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self.shape = tuple(shape)
        self.M = Lx * Ly * Lz
        self.Ms = tuple(Ms)

    def set_fields(self, wA, wB):
        if _is_torch(wA):
            capi.check(lib().ps_model_ab_set_fields_device(self._h, wA.data_ptr(), wB.data_ptr()))
        else:
            wA, wB = _f64(wA), _f64(wB)
            capi.check(lib().ps_model_ab_set_fields(self._h, capi.dptr(wA), capi.dptr(wB)))
        return self

    def update(self, n=1):
        capi.check(lib().ps_model_ab_update(self._h, int(n)))

    def update_timed(self, n):
        """update(n) timed with CUDA events on the context stream; returns
        (total_ms, propagator_ms) after synchronising."""
        tot, prop = ctypes.c_double(), ctypes.c_double()
        capi.check(lib().ps_model_ab_update_timed(self._h, int(n), ctypes.byref(tot), ctypes.byref(prop)))
        return tot.value, prop.value

    def propagate(self, n=1):
        capi.check(lib().ps_model_ab_propagate(self._h, int(n)))

    def synchronize(self):
        capi.check(lib().ps_model_ab_synchronize(self._h))

    def H(self):
        H, Hw, Hs = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        capi.check(lib().ps_model_ab_H(self._h, ctypes.byref(H), ctypes.byref(Hw), ctypes.byref(Hs)))
        return H.value, Hw.value, Hs.value

    def residual_error(self):
        r = ctypes.c_double()
        capi.check(lib().ps_model_ab_residual(self._h, ctypes.byref(r)))
        return r.value

    def Q(self):
        q = ctypes.c_double()
        capi.check(lib().ps_model_ab_Q(self._h, ctypes.byref(q)))
        return q.value

    def forward(self):
        """Evaluate (wA, wB) -> (phiA, phiB, Q) at the current fields, no field update."""
        capi.check(lib().ps_model_ab_forward(self._h))
        return self

    def grad_w(self, dL_dphiA, dL_dphiB, dL_dQ=0.0):
        """Gradient of sum(dL_dphiA*phiA + dL_dphiB*phiB) + dL_dQ*Q with respect
        to (wA, wB) at the current fields (RQM4, 2D/3D grids)."""
        a, b = _f64(dL_dphiA), _f64(dL_dphiB)
        gA, gB = np.zeros(self.shape), np.zeros(self.shape)
        capi.check(lib().ps_model_ab_grad_w(self._h, capi.dptr(a), capi.dptr(b), float(dL_dQ),
                                            capi.dptr(gA), capi.dptr(gB)))
        return gA, gB

    def stress(self, checkpoints=None):
        """d(-ln Q)/dl for the three cell lengths at the current fields.
        checkpoints=k keeps the forward chain only every k slices (0: sqrt(Ns))
        and recomputes it segment by segment in the reverse sweep."""
        out = np.zeros(3)
        if checkpoints is None:
            capi.check(lib().ps_model_ab_stress(self._h, capi.dptr(out)))
        else:
            capi.check(lib().ps_model_ab_stress_checkpointed(self._h, int(checkpoints), capi.dptr(out)))
        return out

    def get(self, name):
        idx = FIELDS[name]
        if name in ("qA", "qAc"):
            out = np.zeros((self.Ms[0],) + self.shape)
        elif name in ("qB", "qBc"):
            out = np.zeros((self.Ms[1],) + self.shape)
        else:
            out = np.zeros(self.shape)
        capi.check(lib().ps_model_ab_get(self._h, idx, capi.dptr(out)))
        return out

    def device_ptr(self, name):
        p = ctypes.c_void_p()
        capi.check(lib().ps_model_ab_device_ptr(self._h, FIELDS[name], ctypes.byref(p)))
        return p.value

    def launches_per_iteration(self):
        return lib().ps_model_ab_launches_per_iteration(self._h)

    def launches_per_propagate(self):
        return lib().ps_model_ab_launches_per_propagate(self._h)

    def stream(self):
        return lib().ps_model_ab_stream(self._h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().ps_model_ab_destroy(h)
            self._h = None


ABC_FIELDS = {"wA": 0, "wB": 1, "wC": 2, "phiA": 3, "phiB": 4, "phiC": 5, "yita": 6}


def _abc_params(dim, shape, cell, Ms, chi, lam=(0.05, 0.05, 0.05, 5.0), scft="EM", n_anderson=5,
                contour="Simpson"):
    """ps_model_abc_params: Ms = (sA, sB, sC), chi = (chiAB, chiBC, chiAC) N,
    lam = (lamA, lamB, lamC, lamYita)."""
    p = capi.ModelABCParamsC()
    p.dim, (p.Lx, p.Ly, p.Lz) = dim, shape
    p.cell = cell
    p.sA, p.sB, p.sC = Ms
    p.chiAB, p.chiBC, p.chiAC = chi
    p.lamA, p.lamB, p.lamC, p.lamYita = lam
    p.scft = capi.SCFT[scft.upper()]
    p.n_anderson = n_anderson
    p.contour = capi.CONTOUR[contour.upper()]
    return p


class ModelABC:
    """A linear A-B-C triblock melt on the device (no counterpart in the
    reference): Model_AB's SCFT iteration with a third block and field,
    incompressible, RQM4; one iteration is one CUDA graph replay."""

    def __init__(self, dim, shape, cell, Ms, chi, lam=(0.05, 0.05, 0.05, 5.0), scft="EM", n_anderson=5,
                 contour="Simpson"):
        p = _abc_params(dim, shape, cell, Ms, chi, lam, scft, n_anderson, contour)
        h = ctypes.c_void_p()
        capi.check(lib().ps_model_abc_create(ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self.shape = tuple(shape)
        self.Ms = tuple(Ms)

    def set_fields(self, wA, wB, wC):
        w = [_f64(x) for x in (wA, wB, wC)]
        capi.check(lib().ps_model_abc_set_fields(self._h, *[capi.dptr(x) for x in w]))
        return self

    def update(self, n=1):
        capi.check(lib().ps_model_abc_update(self._h, int(n)))

    def synchronize(self):
        capi.check(lib().ps_model_abc_synchronize(self._h))

    def Q(self):
        q = ctypes.c_double()
        capi.check(lib().ps_model_abc_Q(self._h, ctypes.byref(q)))
        return q.value

    def H(self):
        H, Hw, Hs = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        capi.check(lib().ps_model_abc_H(self._h, ctypes.byref(H), ctypes.byref(Hw), ctypes.byref(Hs)))
        return H.value, Hw.value, Hs.value

    def residual_error(self):
        r = ctypes.c_double()
        capi.check(lib().ps_model_abc_residual(self._h, ctypes.byref(r)))
        return r.value

    def get(self, name):
        out = np.zeros(self.shape)
        capi.check(lib().ps_model_abc_get(self._h, ABC_FIELDS[name], capi.dptr(out)))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().ps_model_abc_destroy(h)
            self._h = None


class StringAB:
    """polystring_AB on the device: m images advanced together, one captured
    graph per string iteration (SCFT of every image, arc length, spline
    re-sampling, ends restored)."""

    def __init__(self, m, dim, shape, cell, Ms, chiN, lam=(0.05, 0.05, 5.0), mde="RQM4", max_iter=3,
                 compressible=False, contour="Simpson", shard=None):
        Lx, Ly, Lz = shape
        p = capi.ModelABParamsC()
        p.dim, p.Lx, p.Ly, p.Lz = dim, Lx, Ly, Lz
        p.cell = cell
        p.sA, p.sB = Ms
        p.chiN = chiN
        p.lamA, p.lamB, p.lamYita = lam
        p.mde = capi.MDE[mde.upper()]
        p.scft = 0
        p.n_anderson = 1
        p.compressible = 1 if compressible else 0
        p.contour = capi.CONTOUR[contour.upper()]
        h = ctypes.c_void_p()
        if shard is None:
            capi.check(lib().ps_string_ab_create(ctypes.byref(p), int(m), int(max_iter), ctypes.byref(h)))
            self.shard = (0, m)
        else:
            lo, hi = shard
            capi.check(lib().ps_string_ab_create_shard(ctypes.byref(p), int(m), int(max_iter), int(lo), int(hi),
                                                       ctypes.byref(h)))
            self.shard = (int(lo), int(hi))
        self._h = h
        self.m = m
        self.shape = tuple(shape)
        self.M = Lx * Ly * Lz

    def set_images(self, wa, wb):
        wa, wb = _f64(wa), _f64(wb)
        capi.check(lib().ps_string_ab_set_images(self._h, capi.dptr(wa), capi.dptr(wb)))
        return self

    def iterate(self, n=1):
        capi.check(lib().ps_string_ab_iterate(self._h, int(n)))

    def relax(self):
        """run_scftInString for the images of this context's shard."""
        capi.check(lib().ps_string_ab_relax(self._h))

    def reparameterize(self):
        """Arc length, spline re-sampling and ends over all images."""
        capi.check(lib().ps_string_ab_reparameterize(self._h))

    def device_ptr(self, name):
        p = ctypes.c_void_p()
        capi.check(lib().ps_string_ab_device_ptr(self._h, {"wa": 0, "wb": 1, "phiA": 2, "phiB": 3}[name],
                                                 ctypes.byref(p)))
        return p.value

    def stream(self):
        return lib().ps_string_ab_stream(self._h)

    def synchronize(self):
        capi.check(lib().ps_string_ab_synchronize(self._h))

    def H(self):
        out = np.zeros(self.m)
        capi.check(lib().ps_string_ab_H(self._h, capi.dptr(out)))
        return out

    def S(self):
        out = np.zeros(self.m)
        capi.check(lib().ps_string_ab_S(self._h, capi.dptr(out)))
        return out

    def get(self, name):
        idx = {"wa": 0, "wb": 1, "phiA": 2, "phiB": 3}[name]
        out = np.zeros((self.m,) + self.shape)
        capi.check(lib().ps_string_ab_get(self._h, idx, capi.dptr(out)))
        return out

    def launches_per_iteration(self):
        return lib().ps_string_ab_launches_per_iteration(self._h)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().ps_string_ab_destroy(h)
            self._h = None


class BatchAB:
    """Independent Model_AB solves of uneven grids, contour lengths and
    parameters advanced together (the reference runs such solves one per host
    thread, scft/polystring_AB_backThread.cc).  `solves` is a list of dicts of
    ModelAB's constructor arguments (dim, shape, cell, Ms, chiN, lam, scft,
    n_anderson, compressible, contour; RQM4 only).  `triblocks` adds linear
    ABC solves (dicts of ModelABC's constructor arguments), numbered after
    the AB solves.  update(n) runs n SCFT iterations of every solve; each line
    pass of a contour step is one launch over all solves still running."""

    def __init__(self, solves, triblocks=()):
        n, nq = len(solves), len(triblocks)
        arr = (capi.ModelABParamsC * max(n, 1))()
        arq = (capi.ModelABCParamsC * max(nq, 1))()
        self.shapes, self.Ms = [], []
        for i, sv in enumerate(solves):
            arr[i] = _params(**sv)
            self.shapes.append(tuple(sv["shape"]))
            self.Ms.append(tuple(sv["Ms"]))
        for i, sv in enumerate(triblocks):
            arq[i] = _abc_params(**sv)
            self.shapes.append(tuple(sv["shape"]))
            self.Ms.append(tuple(sv["Ms"]))
        h = ctypes.c_void_p()
        if nq:
            capi.check(lib().ps_batch_ab_create_mixed(arr, n, arq, nq, ctypes.byref(h)))
        else:
            capi.check(lib().ps_batch_ab_create(arr, n, ctypes.byref(h)))
        self._h = h
        self.n = n + nq
        self.n_ab = n

    def set_fields(self, k, wA, wB, wC=None):
        """Fields of solve k: (wA, wB) for an AB solve, (wA, wB, wC) for a triblock."""
        if k >= self.n_ab:
            w = [_f64(x) for x in (wA, wB, wC)]
            capi.check(lib().ps_batch_ab_set_fields_abc(self._h, int(k), *[capi.dptr(x) for x in w]))
            return
        wA, wB = _f64(wA), _f64(wB)
        capi.check(lib().ps_batch_ab_set_fields(self._h, int(k), capi.dptr(wA), capi.dptr(wB)))

    def update(self, n=1):
        capi.check(lib().ps_batch_ab_update(self._h, int(n)))

    def update_timed(self, n):
        """update(n) between CUDA events on the batch stream; device ms."""
        ms = ctypes.c_double()
        capi.check(lib().ps_batch_ab_update_timed(self._h, int(n), ctypes.byref(ms)))
        return ms.value

    def synchronize(self):
        capi.check(lib().ps_batch_ab_synchronize(self._h))

    def H(self, k):
        H, Hw, Hs = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        capi.check(lib().ps_batch_ab_H(self._h, int(k), ctypes.byref(H), ctypes.byref(Hw), ctypes.byref(Hs)))
        return H.value, Hw.value, Hs.value

    def residual_error(self, k):
        r = ctypes.c_double()
        capi.check(lib().ps_batch_ab_residual(self._h, int(k), ctypes.byref(r)))
        return r.value

    def get(self, k, name):
        shape, Ms = self.shapes[k], self.Ms[k]
        if k >= self.n_ab:
            out = np.zeros(shape)
            capi.check(lib().ps_batch_ab_get(self._h, int(k), ABC_FIELDS[name], capi.dptr(out)))
            return out
        if name in ("qA", "qAc"):
            out = np.zeros((Ms[0],) + shape)
        elif name in ("qB", "qBc"):
            out = np.zeros((Ms[1],) + shape)
        else:
            out = np.zeros(shape)
        capi.check(lib().ps_batch_ab_get(self._h, int(k), FIELDS[name], capi.dptr(out)))
        return out

    def launches_per_iteration(self):
        return lib().ps_batch_ab_launches_per_iteration(self._h)

    def launches_per_propagate(self):
        """Propagator launches of one batch iteration (the rest are the
        members' Q, density and field-update kernels)."""
        return lib().ps_batch_ab_launches_per_propagate(self._h)

    def gridpoint_steps(self):
        v = ctypes.c_double()
        capi.check(lib().ps_batch_ab_gridpoint_steps(self._h, ctypes.byref(v)))
        return v.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().ps_batch_ab_destroy(h)
            self._h = None
