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
