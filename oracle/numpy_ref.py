"""Independent NumPy restatement of the propagator and density steps.

TEST INFRASTRUCTURE ONLY (a second oracle that cross-checks the C one at
small sizes).  Uses numpy.fft (pocketfft, FP64) for the c2c transforms.

References (paths relative to the reference project root):
  RQM4::solve            src/RQM4.cc:41-93
  PseudoSpectral::solve  src/PseudoSpectral.cc:226-261
  calc_k2_orthogonal     src/UnitCell.cc:368-418
  Simpson / Quad4        src/Simpson.cc:14-45, src/Quadrature4.cc:17-53
"""
import numpy as np


def k2_orthogonal(dim, lengths, shape):
    """-|k|^2 with the reference's index folding i < L/2+1 ? i : L-i."""
    out = np.zeros(shape)
    cc = [0.0, 0.0, 0.0]
    for d in range(dim):
        cc[d] = -4.0 * np.pi * np.pi / (lengths[d] * lengths[d])
    r = []
    for L in shape:
        i = np.arange(L)
        r.append(np.where(i < L // 2 + 1, i, L - i).astype(np.float64))
    # same operation order as the reference: ccx*ri*ri + ccy*rj*rj + ccz*rk*rk
    tx = (cc[0] * r[0]) * r[0]
    ty = (cc[1] * r[1]) * r[1]
    tz = (cc[2] * r[2]) * r[2]
    out = (tx[:, None, None] + ty[None, :, None]) + tz[None, None, :]
    return out


def _split(q, e, L):
    b = np.fft.fftn(e * q)
    b *= L
    return np.real(np.fft.ifftn(b)) * e   # ifftn already divides by M


def rqm4_solve(w, qs, k2, ds):
    expq = np.exp(-0.5 * ds * w)
    expq2 = np.exp(-0.25 * ds * w)
    L1 = np.exp(ds * k2)
    L2 = np.exp(0.5 * ds * k2)
    for s in range(qs.shape[0] - 1):
        full = _split(qs[s], expq, L1)
        qt = _split(qs[s], expq2, L2)
        qt = _split(qt, expq2, L2)
        qs[s + 1] = (4.0 * qt - full) / 3.0
    return qs


def os2_solve(w, qs, lap, ds):
    expq = np.exp(-0.5 * ds * w)
    for s in range(qs.shape[0] - 1):
        qs[s + 1] = _split(qs[s], expq, lap)
    return qs


def simpson_weights(n):
    c = np.zeros(n + 1)
    c[1:n:2] = 4.0
    c[2:n - 1:2] = 2.0
    c[0] = c[n] = 1.0
    return c / 3.0


def quad4_closed_weights(n):
    c = np.ones(n + 1)
    c[0] = c[n] = 9.0 / 24.0
    c[1] = c[n - 1] = 28.0 / 24.0
    c[2] = c[n - 2] = 23.0 / 24.0
    return c


def density(c, q, qc, ds, cc):
    n = q.shape[0] - 1
    acc = np.zeros(q.shape[1:])
    for s in range(n + 1):
        acc += c[s] * (q[s] * qc[n - s])
    return acc * (cc * ds)


def etdrk4_solve(w, qs, k2, ds, Mc=32):
    """Etdrk4_PBC::solve (src/Etdrk4_PBC.cc:110-184) with the contour
    coefficients of init_coefficient (:43-99), numpy.fft: the spectrum v of q
    is carried from step to step."""
    L = k2.astype(complex)
    r = np.exp(1j * np.pi * (np.arange(Mc) + 0.5) / Mc)
    x = ds * L[..., None] + r
    ex = np.exp(x)
    Q = ds * np.real(np.mean((np.exp(x / 2.0) - 1.0) / x, -1))
    f1 = ds * np.real(np.mean((ex * (x * x - 3.0 * x + 4.0) - x - 4.0) / x ** 3, -1))
    f2 = ds * np.real(np.mean((ex * (x - 2.0) + x + 2.0) / x ** 3, -1))
    f3 = ds * np.real(np.mean((ex * (4.0 - x) - x * x - 3.0 * x - 4.0) / x ** 3, -1))
    E, E2 = np.exp(ds * k2), np.exp(ds * k2 / 2.0)
    F, IF = np.fft.fftn, np.fft.ifftn
    v = F(qs[0])
    for s in range(qs.shape[0] - 1):
        Nv = F(-w * qs[s])
        a = E2 * v + Q * Nv
        Na = F(-w * np.real(IF(a)))
        b = E2 * v + Q * Na
        Nb = F(-w * np.real(IF(b)))
        c = E2 * a + Q * (2.0 * Nb - Nv)
        Nc = F(-w * np.real(IF(c)))
        v = E * v + f1 * Nv + 2.0 * f2 * (Na + Nb) + f3 * Nc
        qs[s + 1] = np.real(IF(v))
    return qs
