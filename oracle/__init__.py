"""CPU FP64 oracle for the periodic pseudospectral SCFT path.

TEST INFRASTRUCTURE ONLY: the parity tests, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` use this package as the checker.  The
product (``polystring_b200``) never imports it.

Two restatements live here:

* ``scft_oracle.c`` -- the C restatement (own mixed-radix FFT, RQM4/OS2,
  quadratures, Model_AB with EM and Anderson mixing, string reparam), loaded
  through ctypes.  It is also the timed CPU baseline.
* ``numpy_ref.py`` -- an independent NumPy restatement (numpy.fft) used to
  cross-check the C one at small sizes.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_SO = os.path.join(_BUILD, "liboracle.so")
_SRC = os.path.join(_HERE, "scft_oracle.c")

# crystal systems (same numbering as include/polystring_b200.h)
LAMELLAR, SQUARE, RECTANGULAR, HEXAGONAL2, OBLIQUE = 0, 1, 2, 3, 4
CUBIC, TETRAGONAL, ORTHORHOMBIC, HEXAGONAL3, TRIGONAL, MONOCLINIC, TRICLINIC = 5, 6, 7, 8, 9, 10, 11
# contour rules
TRAPEZOID, SIMPSON, QUAD4_CLOSED, QUAD4_OPEN, QUAD4_SEMIOPEN_LEFT, QUAD4_SEMIOPEN_RIGHT = range(6)
RQM4, OS2, ETDRK4 = 0, 1, 2
EM, ANDERSON = 0, 1


def build(force=False):
    """Compile scft_oracle.c into oracle/_build/liboracle.so (gcc, -O3, OpenMP)."""
    os.makedirs(_BUILD, exist_ok=True)
    if not force and os.path.exists(_SO) and os.path.getmtime(_SO) >= os.path.getmtime(_SRC):
        return _SO
    cmd = ["gcc", "-O3", "-std=c11", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-o", _SO + ".tmp", _SRC, "-lm"]
    subprocess.check_call(cmd)
    os.replace(_SO + ".tmp", _SO)
    return _SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = ctypes.CDLL(_SO)
        dp = ctypes.POINTER(ctypes.c_double)
        vp = ctypes.c_void_p
        L.orc_fft3.argtypes = [ctypes.c_int] * 3 + [dp, ctypes.c_int]
        L.orc_unit_cell.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 6 + [dp, dp]
        L.orc_k2_orthogonal.argtypes = [ctypes.c_int] + [ctypes.c_double] * 3 + [ctypes.c_int] * 3 + [dp]
        L.orc_k_laplacian.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, dp]
        L.orc_rqm4_create.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.orc_rqm4_create.restype = vp
        L.orc_os2_create.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        L.orc_os2_create.restype = vp
        L.orc_etdrk4_create.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.orc_etdrk4_create.restype = vp
        L.orc_updater_destroy.argtypes = [vp]
        L.orc_updater_solve.argtypes = [vp, dp, dp, ctypes.c_int]
        L.orc_mean.argtypes = [dp, ctypes.c_size_t]
        L.orc_mean.restype = ctypes.c_double
        L.orc_contour_weights.argtypes = [ctypes.c_int, ctypes.c_int, dp]
        L.orc_density.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_size_t,
                                  ctypes.c_double, ctypes.c_double, dp]
        L.orc_solve_small.argtypes = [ctypes.c_int, dp, dp, dp]
        L.orc_model_ab_create.argtypes = [ctypes.POINTER(_ABParams), dp, dp]
        L.orc_model_ab_create.restype = vp
        L.orc_model_ab_destroy.argtypes = [vp]
        L.orc_model_ab_update.argtypes = [vp]
        L.orc_model_ab_H.argtypes = [vp, dp, dp, dp]
        L.orc_model_ab_residual.argtypes = [vp]
        L.orc_model_ab_residual.restype = ctypes.c_double
        L.orc_model_ab_Q.argtypes = [vp]
        L.orc_model_ab_Q.restype = ctypes.c_double
        L.orc_model_ab_last_rc.argtypes = [vp]
        L.orc_model_ab_get.argtypes = [vp, ctypes.c_int, dp]
        L.orc_model_abc_create.argtypes = [ctypes.POINTER(_ABCParams), dp, dp, dp]
        L.orc_model_abc_create.restype = vp
        L.orc_model_abc_destroy.argtypes = [vp]
        L.orc_model_abc_update.argtypes = [vp]
        L.orc_model_abc_H.argtypes = [vp, dp, dp, dp]
        L.orc_model_abc_residual.argtypes = [vp]
        L.orc_model_abc_residual.restype = ctypes.c_double
        L.orc_model_abc_Q.argtypes = [vp]
        L.orc_model_abc_Q.restype = ctypes.c_double
        L.orc_model_abc_get.argtypes = [vp, ctypes.c_int, dp]
        L.orc_string_arclength.argtypes = [dp, ctypes.c_int, ctypes.c_size_t, dp]
        L.orc_string_redistribute.argtypes = [dp, dp, ctypes.c_int, ctypes.c_size_t, dp, dp]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class _ABParams(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int), ("Lx", ctypes.c_int), ("Ly", ctypes.c_int), ("Lz", ctypes.c_int),
        ("sA", ctypes.c_int), ("sB", ctypes.c_int),
        ("chiN", ctypes.c_double),
        ("lamA", ctypes.c_double), ("lamB", ctypes.c_double), ("lamYita", ctypes.c_double),
        ("mde", ctypes.c_int), ("scft", ctypes.c_int), ("n_anderson", ctypes.c_int),
        ("compressible", ctypes.c_int), ("contour", ctypes.c_int),
        ("k2", ctypes.POINTER(ctypes.c_double)),
        ("lapA", ctypes.POINTER(ctypes.c_double)),
        ("lapB", ctypes.POINTER(ctypes.c_double)),
    ]


def set_threads(n):
    lib().orc_set_threads(int(n))


def max_threads():
    return lib().orc_max_threads()


def fft3(a, sign=-1):
    """Unnormalised c2c FFT over the 3 axes of a complex (Lx, Ly, Lz) array."""
    a = np.ascontiguousarray(a, dtype=np.complex128).copy()
    Lx, Ly, Lz = a.shape
    rc = lib().orc_fft3(Lx, Ly, Lz, a.view(np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double)), sign)
    assert rc == 0
    return a


def unit_cell(dim, system, a, b=0.0, c=0.0, alpha=0.0, beta=0.0, gamma=0.0):
    """Reciprocal shape matrix g (3x3) and lengths l (3,) as UnitCell builds them."""
    g = np.zeros(9)
    l = np.zeros(3)
    rc = lib().orc_unit_cell(dim, system, a, b, c, alpha, beta, gamma, _p(g), _p(l))
    if rc != 0:
        raise ValueError("bad cell parameters")
    return g.reshape(3, 3), l


def k2_orthogonal(dim, lengths, shape):
    Lx, Ly, Lz = shape
    out = np.zeros(shape)
    lx, ly, lz = (list(lengths) + [0.0, 0.0, 0.0])[:3]
    lib().orc_k2_orthogonal(dim, lx, ly, lz, Lx, Ly, Lz, _p(out))
    return out


def k_laplacian(g, shape, ds):
    out = np.zeros(shape)
    gg = _f64(np.asarray(g).reshape(9))
    lib().orc_k_laplacian(_p(gg), shape[0], shape[1], shape[2], ds, _p(out))
    return out


class Updater:
    """RQM4 (scheme 'RQM4', table = -k^2), OS2 (scheme 'OS2', table = exp(-ds q^2))
    or ETDRK4 (scheme 'ETDRK4', table = -k^2, contour points Mc)."""

    def __init__(self, scheme, table, shape, ds, Mc=32):
        t = _f64(table)
        self.shape = tuple(shape)
        self.M = int(np.prod(shape))
        if scheme == "RQM4":
            self.h = lib().orc_rqm4_create(_p(t), *self.shape, ds)
        elif scheme == "ETDRK4":
            self.h = lib().orc_etdrk4_create(_p(t), *self.shape, ds, Mc)
        else:
            self.h = lib().orc_os2_create(_p(t), *self.shape, ds)

    def solve(self, w, qs):
        """In place: qs (len, Lx, Ly, Lz) with qs[0] the head."""
        assert qs.dtype == np.float64 and qs.flags.c_contiguous
        w = _f64(w)
        lib().orc_updater_solve(self.h, _p(w), _p(qs), qs.shape[0])
        return qs

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_updater_destroy(self.h)
            self.h = None


def contour_weights(rule, n):
    c = np.zeros(n + 1)
    rc = lib().orc_contour_weights(rule, n, _p(c))
    if rc != 0:
        raise ValueError("quadrature precondition failed")
    return c


def density(rule, q, qc, ds, cc):
    q = _f64(q)
    qc = _f64(qc)
    M = int(np.prod(q.shape[1:]))
    phi = np.zeros(q.shape[1:])
    rc = lib().orc_density(rule, _p(q), _p(qc), q.shape[0], M, ds, cc, _p(phi))
    if rc != 0:
        raise ValueError("quadrature precondition failed")
    return phi


def solve_small(U, V):
    U = _f64(U)
    V = _f64(V)
    n = V.shape[0]
    C = np.zeros(n)
    rc = lib().orc_solve_small(n, _p(U), _p(V), _p(C))
    if rc != 0:
        raise ValueError("singular")
    return C


class ModelAB:
    """Model_AB restated on the CPU (periodic cell, DATA_INIT fields)."""

    def __init__(self, dim, shape, lengths, Ms, chiN, lam=(0.05, 0.05, 5.0), mde="RQM4",
                 scft="EM", n_anderson=5, compressible=False, contour="Simpson", g=None):
        self.shape = tuple(shape)
        self.M = int(np.prod(shape))
        self.Ms = tuple(Ms)
        sA, sB = Ms
        LA, LB = sA - 1, sB - 1
        fA = 1.0 * LA / (LA + LB)
        fB = 1.0 * LB / (LA + LB)
        self.dsA, self.dsB = fA / LA, fB / LB
        self._k2 = k2_orthogonal(dim, lengths, shape)
        if mde == "OS2":
            if g is None:
                g = np.diag([2 * np.pi / lengths[0],
                             2 * np.pi / (lengths[1] if dim >= 2 else 1.0),
                             2 * np.pi / (lengths[2] if dim >= 3 else 1.0)])
            self._lapA = k_laplacian(g, shape, self.dsA)
            self._lapB = k_laplacian(g, shape, self.dsB)
        else:
            self._lapA = np.zeros(1)
            self._lapB = np.zeros(1)
        self.params = _ABParams(
            dim, shape[0], shape[1], shape[2], sA, sB, chiN, lam[0], lam[1], lam[2],
            {"RQM4": RQM4, "OS2": OS2, "ETDRK4": ETDRK4}[mde], ANDERSON if scft == "Anderson" else EM,
            n_anderson, 1 if compressible else 0, 1 if contour == "Simpson" else 0,
            _p(self._k2), _p(self._lapA), _p(self._lapB))
        self.h = None

    def init_fields(self, wA, wB):
        if self.h:
            lib().orc_model_ab_destroy(self.h)
        wA = _f64(wA)
        wB = _f64(wB)
        self.h = lib().orc_model_ab_create(ctypes.byref(self.params), _p(wA), _p(wB))
        return self

    def update(self, n=1):
        rc = 0
        for _ in range(n):
            rc |= lib().orc_model_ab_update(self.h)
        return rc

    def H(self):
        H, Hw, Hs = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        lib().orc_model_ab_H(self.h, ctypes.byref(H), ctypes.byref(Hw), ctypes.byref(Hs))
        return H.value, Hw.value, Hs.value

    def residual(self):
        return lib().orc_model_ab_residual(self.h)

    def Q(self):
        return lib().orc_model_ab_Q(self.h)

    def get(self, name):
        idx = {"wA": 0, "wB": 1, "phiA": 2, "phiB": 3, "yita": 4,
               "qA": 5, "qB": 6, "qAc": 7, "qBc": 8}[name]
        if idx in (5, 7):
            out = np.zeros((self.Ms[0],) + self.shape)
        elif idx in (6, 8):
            out = np.zeros((self.Ms[1],) + self.shape)
        else:
            out = np.zeros(self.shape)
        rc = lib().orc_model_ab_get(self.h, idx, _p(out))
        if rc != 0:
            raise KeyError(name)
        return out

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_model_ab_destroy(self.h)
            self.h = None


class _ABCParams(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int), ("Lx", ctypes.c_int), ("Ly", ctypes.c_int), ("Lz", ctypes.c_int),
        ("s", ctypes.c_int * 3), ("chi", ctypes.c_double * 3), ("lam", ctypes.c_double * 4),
        ("scft", ctypes.c_int), ("n_anderson", ctypes.c_int), ("contour", ctypes.c_int),
        ("k2", ctypes.POINTER(ctypes.c_double))]


class ModelABC:
    """Linear A-B-C triblock melt (defined in scft_oracle.c's Model_ABC block:
    Model_AB's steps with a third block and field; incompressible, RQM4).
    chi = (chiAB N, chiBC N, chiAC N); lam = (lamA, lamB, lamC, lamYita)."""

    def __init__(self, dim, shape, lengths, Ms, chi, lam=(0.05, 0.05, 0.05, 5.0), scft="EM", n_anderson=5,
                 contour="Simpson"):
        self.shape = tuple(shape)
        self.M = int(np.prod(shape))
        self.Ms = tuple(Ms)
        self._k2 = k2_orthogonal(dim, lengths, shape)
        self.params = _ABCParams(dim, shape[0], shape[1], shape[2], (ctypes.c_int * 3)(*Ms),
                                 (ctypes.c_double * 3)(*chi), (ctypes.c_double * 4)(*lam),
                                 ANDERSON if scft == "Anderson" else EM, n_anderson,
                                 1 if contour == "Simpson" else 0, _p(self._k2))
        self.h = None

    def init_fields(self, wA, wB, wC):
        if self.h:
            lib().orc_model_abc_destroy(self.h)
        self._w = [_f64(wA), _f64(wB), _f64(wC)]
        self.h = lib().orc_model_abc_create(ctypes.byref(self.params), *[_p(w) for w in self._w])
        return self

    def update(self, n=1):
        rc = 0
        for _ in range(n):
            rc |= lib().orc_model_abc_update(self.h)
        return rc

    def H(self):
        H, Hw, Hs = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        lib().orc_model_abc_H(self.h, ctypes.byref(H), ctypes.byref(Hw), ctypes.byref(Hs))
        return H.value, Hw.value, Hs.value

    def residual(self):
        return lib().orc_model_abc_residual(self.h)

    def Q(self):
        return lib().orc_model_abc_Q(self.h)

    def get(self, name):
        idx = {"wA": 0, "wB": 1, "wC": 2, "phiA": 3, "phiB": 4, "phiC": 5, "yita": 6}[name]
        out = np.zeros(self.shape)
        if lib().orc_model_abc_get(self.h, idx, _p(out)) != 0:
            raise KeyError(name)
        return out

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_model_abc_destroy(self.h)
            self.h = None


def string_arclength(wa):
    wa = _f64(wa)
    m = wa.shape[0]
    M = int(np.prod(wa.shape[1:]))
    S = np.zeros(m)
    lib().orc_string_arclength(_p(wa), m, M, _p(S))
    return S


def string_redistribute(f, S, end0, end1):
    """In place on f (m, ...): per-point natural cubic spline re-sampling."""
    assert f.dtype == np.float64 and f.flags.c_contiguous
    m = f.shape[0]
    M = int(np.prod(f.shape[1:]))
    S = _f64(S)
    e0 = _f64(end0)
    e1 = _f64(end1)
    rc = lib().orc_string_redistribute(_p(f), _p(S), m, M, _p(e0), _p(e1))
    assert rc == 0
    return f


def string_iteration(model, wa, wb, end_a, end_b, max_iter):
    """One iteration of polystring_AB (scft/polystring_AB.cc:125-150) on the
    CPU: every image restarts from its fields (fresh Yita, resetInString) and
    runs max_iter updates; then arc length from wa, per-point natural spline
    re-sampling of wa and wb, ends restored.  wa, wb (m, ...) are updated in
    place; returns (H per image, S)."""
    m = wa.shape[0]
    H = np.zeros(m)
    for s in range(m):
        model.init_fields(wa[s], wb[s])
        model.update(max_iter)
        H[s] = model.H()[0]
        wa[s] = model.get("wA")
        wb[s] = model.get("wB")
    S = string_arclength(wa)
    string_redistribute(wa, S, end_a[0], end_a[1])
    string_redistribute(wb, S, end_b[0], end_b[1])
    return H, S
