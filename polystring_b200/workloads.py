"""Seeded synthetic inputs of the benchmark configurations.

There is no public dataset on this path; every configuration is an AB
diblock melt on a periodic cell with fields generated from a seed on the
host and handed identically to the CUDA path and to the CPU oracle.

  C1  2D 64x64, square 4.0 Rg, fA 0.30, chiN 20, Ns 100 (Ms [31, 71]), RQM4,
      simple mixing lambda 0.1; w = 0.1 U(-1,1) +/- 0.5 x (6-fold cosine)
  C2  3D 64^3, cubic 4.2 Rg, fA 0.35, chiN 25, Ns 200 (Ms [71, 131]), RQM4,
      Anderson (history 20); w = 0.1 N(0,1) +/- 1.0 x (gyroid level set)
  C3  40 images, 2D 128x128, square 8.0 Rg, fA 0.35, chiN 18, Ns 128
      (Ms [46, 84], Quad4_Closed on both blocks); images interpolate between
      a lamellar field (cos x, amp 2.0) and a hexagonal field (3 waves, amp
      2.0), each plus 0.05 N(0,1)
  C4  3D 48^3, orthorhombic (3.8, 4.0, 4.2), fA 0.30, chiN 22, Ns 128
      (Ms [39, 91]); w = 0.1 N(0,1) +/- 2.0 x (cos x + cos y + cos z)
  C5  independent solves of uneven grids and Ns (uneven_solves)

Ms follows from fA and Ns as LA = round(fA Ns), LB = Ns - LA, Ms = [LA+1, LB+1]
(the reference reads Ms and recomputes f = LA/(LA+LB), src/Model_AB.cc:100-111).
"""
import numpy as np


def ms_from(fA, Ns):
    LA = int(round(fA * Ns))
    return (LA + 1, Ns - LA + 1)


def _coords(shape, lengths):
    axes = []
    for n, L in zip(shape, lengths):
        axes.append(np.arange(n) * (L / n))
    return np.meshgrid(*axes, indexing="ij")


def six_fold(shape, L):
    """Sum of three plane waves at 60 degrees with wavevector 2 pi / L."""
    x, y = _coords(shape[:2], (L, L))
    k = 2 * np.pi / L
    s = np.zeros(shape[:2])
    for ang in (0.0, np.pi / 3, 2 * np.pi / 3):
        s += np.cos(k * (np.cos(ang) * x + np.sin(ang) * y))
    return (s / 3.0).reshape(shape)


def gyroid(shape, L):
    """Gyroid level set sin x cos y + sin y cos z + sin z cos x with one period
    per cell axis; L is one length (cubic) or three."""
    Ls = (L, L, L) if np.isscalar(L) else tuple(L)
    x, y, z = _coords(shape, Ls)
    kx, ky, kz = (2 * np.pi / l for l in Ls)
    return (np.sin(kx * x) * np.cos(ky * y) + np.sin(ky * y) * np.cos(kz * z) + np.sin(kz * z) * np.cos(kx * x))


def cosine_sum(shape, L):
    """cos x + cos y + cos z with one period per cell axis (L: three lengths)."""
    x, y, z = _coords(shape, tuple(L))
    kx, ky, kz = (2 * np.pi / l for l in L)
    return np.cos(kx * x) + np.cos(ky * y) + np.cos(kz * z)


def config(name, seed=2024):
    """Parameters and initial fields of a configuration (C1, C2, C4)."""
    rng = np.random.default_rng(seed)
    if name == "C1":
        shape, L = (64, 64, 1), 4.0
        base = 0.1 * rng.uniform(-1, 1, (2,) + shape)
        c6 = six_fold(shape, L)
        return dict(dim=2, shape=shape, cell=("SQUARE", (L,)), Ms=ms_from(0.30, 100), chiN=20.0,
                    lam=(0.1, 0.1, 5.0), mde="RQM4", scft="EM", n_anderson=5, iters=500,
                    wA=base[0] + 0.5 * c6, wB=base[1] - 0.5 * c6)
    if name == "C2":
        shape, L = (64, 64, 64), 4.2
        base = 0.1 * rng.standard_normal((2,) + shape)
        g = gyroid(shape, L)
        return dict(dim=3, shape=shape, cell=("CUBIC", (L,)), Ms=ms_from(0.35, 200), chiN=25.0,
                    lam=(0.05, 0.05, 5.0), mde="RQM4", scft="Anderson", n_anderson=20, iters=1000,
                    wA=base[0] + 1.0 * g, wB=base[1] - 1.0 * g)
    if name == "C4":
        # seeded noise plus an ordered seed, the simple-cubic wave sum
        # cos x + cos y + cos z (one period per cell axis, amplitude 2): from
        # noise alone, or from a gyroid seed of amplitude 1, the Anderson
        # iteration settles on the disordered saddle point, whose cell stress
        # vanishes; this seed converges (residual 1e-9 in ~200 iterations) to
        # an ordered structure with a stress of 5e-4..7e-3 in every axis
        shape, L = (48, 48, 48), (3.8, 4.0, 4.2)
        base = 0.1 * rng.standard_normal((2,) + shape)
        g = 2.0 * cosine_sum(shape, L)
        return dict(dim=3, shape=shape, cell=("ORTHORHOMBIC", L), Ms=ms_from(0.30, 128), chiN=22.0,
                    lam=(0.05, 0.05, 5.0), mde="RQM4", scft="Anderson", n_anderson=20, iters=300,
                    wA=base[0] + 1.0 * g, wB=base[1] - 1.0 * g)
    raise KeyError(name)


def uneven_solves(n=27, seed=2024):
    """C5: independent solves on cubic grids {32^3, 48^3, 64^3} with Ns in
    {64, 128, 256} (cycled, so every pairing occurs), fA ~ U(0.2, 0.5),
    chiN ~ U(12, 30), cell ~ U(3.5, 5.0) Rg, Anderson mixing, fields
    0.1 N(0, 1).  Ms follows from fA and Ns, so block lengths, and with them
    Simpson or Quad4 rules, differ between solves."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        L = (32, 48, 64)[k % 3]
        Ns = (64, 128, 256)[(k // 3) % 3]
        fA = rng.uniform(0.2, 0.5)
        chiN = rng.uniform(12.0, 30.0)
        a = rng.uniform(3.5, 5.0)
        shape = (L, L, L)
        w = 0.1 * rng.standard_normal((2,) + shape)
        out.append(dict(dim=3, shape=shape, cell=("CUBIC", (a,)), Ms=ms_from(fA, Ns), chiN=chiN,
                        lam=(0.05, 0.05, 5.0), scft="Anderson", n_anderson=10, wA=w[0], wB=w[1]))
    return out


def uneven_triblocks(n=64, seed=2025):
    """The ABC share of C5: linear A-B-C triblock solves on cubic grids
    {32^3, 48^3, 64^3} with Ns in {64, 128, 256} (cycled like the AB solves),
    fA ~ U(0.2, 0.5), fB ~ U(0.2, min(0.5, 0.9 - fA)), fC = 1 - fA - fB,
    chiAB, chiBC, chiAC N ~ U(12, 30), cell ~ U(3.5, 5.0) Rg, Anderson(10),
    fields 0.1 N(0, 1)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        L = (32, 48, 64)[k % 3]
        Ns = (64, 128, 256)[(k // 3) % 3]
        fA = rng.uniform(0.2, 0.5)
        fB = rng.uniform(0.2, min(0.5, 0.9 - fA))
        chi = tuple(rng.uniform(12.0, 30.0, 3))
        a = rng.uniform(3.5, 5.0)
        shape = (L, L, L)
        LA, LB = int(round(fA * Ns)), int(round(fB * Ns))
        Ms = (LA + 1, LB + 1, Ns - LA - LB + 1)
        w = 0.1 * rng.standard_normal((3,) + shape)
        out.append(dict(dim=3, shape=shape, cell=("CUBIC", (a,)), Ms=Ms, chi=chi, lam=(0.05, 0.05, 0.05, 5.0),
                        scft="Anderson", n_anderson=10, w=w))
    return out


def string_images(m=40, shape=(128, 128, 1), L=8.0, seed=2024):
    """C3 initial string: m images linearly interpolated between a lamellar
    and a hexagonal field (polystring_AB.cc:207-214 interpolation)."""
    rng = np.random.default_rng(seed)
    x, y = _coords(shape[:2], (L, L))
    k = 2 * np.pi / L
    lam = (2.0 * np.cos(k * x)).reshape(shape)
    hexa = (2.0 * sum(np.cos(k * (np.cos(a) * x + np.sin(a) * y)) for a in (0.0, np.pi / 3, 2 * np.pi / 3)) / 3.0)
    hexa = hexa.reshape(shape)
    e0A = lam + 0.05 * rng.standard_normal(shape)
    e0B = -lam + 0.05 * rng.standard_normal(shape)
    e1A = hexa + 0.05 * rng.standard_normal(shape)
    e1B = -hexa + 0.05 * rng.standard_normal(shape)
    wa = np.stack([e0A + i / (m - 1) * (e1A - e0A) for i in range(m)])
    wb = np.stack([e0B + i / (m - 1) * (e1B - e0B) for i in range(m)])
    return wa, wb


def model_of(ps, cfg, cell_lengths=None, **over):
    """A ps.ModelAB of a configuration dict (fields not set)."""
    system, a = cfg["cell"]
    a = tuple(cell_lengths) if cell_lengths is not None else a
    kw = dict(lam=cfg["lam"], mde=cfg["mde"], scft=cfg["scft"], n_anderson=cfg["n_anderson"])
    kw.update(over)
    return ps.ModelAB(cfg["dim"], cfg["shape"], ps.make_cell(cfg["dim"], system, *a), cfg["Ms"], cfg["chiN"], **kw)


def converge(m, thresh, max_iter, chunk=50):
    """Run m.update in chunks until residual_error() < thresh or max_iter
    iterations; returns (iterations, residual)."""
    it, r = 0, float("inf")
    while it < max_iter:
        m.update(chunk)
        it += chunk
        r = m.residual_error()
        if r < thresh or not np.isfinite(r):
            break
    return it, r


def smoothed_target(shape, seed=7, passes=2):
    """A seeded field in [0, 1] smoothed by periodic 3-point means per axis."""
    t = np.random.default_rng(seed).uniform(0, 1, shape)
    for _ in range(passes):
        t = sum(np.roll(t, s, ax) for ax in range(len(shape)) for s in (-1, 0, 1)) / (3.0 * len(shape))
    return t


def neg_lnQ(ps, cfg, lengths, wA, wB):
    """-ln Q of the forward map at fixed fields for the given cell lengths."""
    m = model_of(ps, cfg, lengths)
    m.set_fields(wA, wB)
    m.forward()
    return -np.log(m.Q())


def stress_fd(ps, cfg, wA, wB, i, h, order=4):
    """Central difference of -ln Q in cell length i: fourth order (points
    +-h, +-2h) or second order (+-h)."""
    L = list(cfg["cell"][1])
    v = {}
    for k in ((-2, -1, 1, 2) if order == 4 else (-1, 1)):
        Lp = list(L)
        Lp[i] += k * h
        v[k] = neg_lnQ(ps, cfg, Lp, wA, wB)
    if order == 4:
        return (v[-2] - 8 * v[-1] + 8 * v[1] - v[2]) / (12 * h)
    return (v[1] - v[-1]) / (2 * h)


def loss_fd(m, wA, wB, dA, dB, target, h, order=4):
    """Central difference of Loss = sum (phiA - target)^2 along (dA, dB).
    Loss differences are formed point by point before the sum,
    Loss(k) - Loss(0) = sum (phi_k - phi_0)(phi_k + phi_0 - 2 target),
    so the rounding of the ~10^5-term sums does not enter the difference."""
    m.set_fields(wA, wB)
    m.forward()
    p0 = m.get("phiA")
    dl = {}
    for k in ((-2, -1, 1, 2) if order == 4 else (-1, 1)):
        m.set_fields(wA + k * h * dA, wB + k * h * dB)
        m.forward()
        pk = m.get("phiA")
        dl[k] = float(((pk - p0) * (pk + p0 - 2.0 * target)).sum())
    m.set_fields(wA, wB)
    if order == 4:
        return (dl[-2] - 8 * dl[-1] + 8 * dl[1] - dl[2]) / (12 * h)
    return (dl[1] - dl[-1]) / (2 * h)


def run_once(name):
    """One pass of a case through the library, for profilers and smoke runs:
    'string' (C3: 40 images of 128^2, one string iteration with one SCFT
    iteration per image), 'batch' (nine C5 solves, one batch iteration),
    'adjoint' (48^3 C4 shape, one stress evaluation); and two small cases
    for kernel captures, with inputs above the 126 MB L2 but few GB on the
    device: 'sweep64' (the C2 64^3 model with Ms [21, 41], 244 MB of
    histories, three iterations: one 64^3 sweep launch each) and 'string12'
    (12 images of 128^2, Ns 128, three string iterations of one SCFT
    iteration each: one cluster-sweep launch each)."""
    import polystring_b200 as ps
    if name == "sweep64":
        c = config("C2")
        m = ps.ModelAB(3, c["shape"], ps.make_cell(3, "CUBIC", 4.2), (21, 41), c["chiN"], scft="Anderson",
                       n_anderson=5)
        m.set_fields(c["wA"], c["wB"])
        m.update(3)
        m.synchronize()
        return m.H()
    if name == "string12":
        g = ps.StringAB(12, 2, (128, 128, 1), ps.make_cell(2, "SQUARE", 8.0), ms_from(0.35, 128), 18.0, max_iter=1)
        wa, wb = string_images(m=12)
        g.set_images(wa, wb)
        g.iterate(3)
        g.synchronize()
        return g.H()
    if name == "string":
        g = ps.StringAB(40, 2, (128, 128, 1), ps.make_cell(2, "SQUARE", 8.0), ms_from(0.35, 128), 18.0, max_iter=1)
        wa, wb = string_images(m=40)
        g.set_images(wa, wb)
        g.iterate(1)
        g.synchronize()
        return g.H()
    if name == "batch":
        specs = uneven_solves(9)
        b = ps.BatchAB([dict(dim=3, shape=s["shape"], cell=ps.make_cell(3, "CUBIC", s["cell"][1][0]), Ms=s["Ms"],
                             chiN=s["chiN"], lam=s["lam"], scft="Anderson", n_anderson=10) for s in specs])
        for k, s in enumerate(specs):
            b.set_fields(k, s["wA"], s["wB"])
        b.update(1)
        b.synchronize()
        return [b.H(k)[0] for k in range(len(specs))]
    if name == "adjoint":
        c = config("C4")
        m = ps.ModelAB(3, c["shape"], ps.make_cell(3, "ORTHORHOMBIC", *c["cell"][1]), c["Ms"], c["chiN"])
        m.set_fields(c["wA"], c["wB"])
        return m.stress()
    raise KeyError(name)


if __name__ == "__main__":
    import sys
    print(run_once(sys.argv[1] if len(sys.argv) > 1 else "string"))
