"""Benchmark of the periodic pseudospectral SCFT hot path on B200.

Workload (one GPU): the 3D configuration -- AB diblock melt on a 64^3
periodic cubic cell of 4.2 Rg, fA 0.35, chiN 25, Ns 200 (Ms [71, 131]),
RQM4 propagators, Simpson contour integration, Anderson mixing with history
20, FP64, seeded gyroid-plus-noise fields.  A step is one SCFT iteration
(Model_AB::update: four propagators over 2 Ns contour steps, Q, densities,
Anderson update).  Metric: gridpoint x contour-steps per second, 2 Ns M per
step.  Inputs (the 0.8 GB propagator histories) exceed the 126 MB L2, so no
explicit flush is done between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank runs an independent replica (a single solve
does not shard); value = total gridpoint-steps of all ranks / max time.
--impl reference times the CPU restatement of the reference algorithm on the
host cores (rank 0 only).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "gridpt_contour_steps_per_s"
UNIT = "gridpt*contour-steps/s"
BYTES_PER_GRIDPT_STEP = 24.0       # read q_s, read w, write q_{s+1}
WORKLOAD = "C2 Model_AB 3D 64^3 RQM4 Anderson(20) Ns=200 FP64"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--profile", action="store_true",
                    help="only warm-up and timed iterations (for ncu captures); prints a short line")
    return ap.parse_args()


def config():
    from polystring_b200 import workloads
    return workloads.config("C2")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def fp64_peak_tflops(ps):
    """FP64 FMA throughput of this GPU measured live (ps_measure_fp64_peak:
    CUDA events around launches of independent FMA chains on every SM);
    the nominal 37 TFLOP/s only if the measurement fails."""
    import ctypes
    v = ctypes.c_double()
    try:
        if ps.lib().ps_measure_fp64_peak(ctypes.byref(v)) == 0 and v.value > 0:
            return v.value, "measured (ps_measure_fp64_peak, DFMA chains, CUDA events)"
    except Exception:
        pass
    return 37.0, "nominal"


def traffic_per_gridpt_step():
    """DRAM bytes per gridpoint-step of the propagator line passes from the
    committed ncu summary (None until one exists)."""
    path = os.path.join(ROOT, "profiles", "propagator_sweep64_c2_64cube.txt")
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_gridpt_step:"):
                    return float(line.split(":")[1])
    except OSError:
        pass
    return None


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_propagation_rate(dim, shape, lengths, Ms, w, seconds, threads):
    """Gridpoint contour steps per second of the CPU oracle's RQM4 propagator
    (the restatement of the reference's step sequence) on one field of the
    given grid: as many steps as fit in about `seconds`."""
    import oracle
    oracle.build()
    oracle.set_threads(threads)
    M = int(np.prod(shape))
    Ns = Ms[0] + Ms[1] - 2
    k2 = oracle.k2_orthogonal(dim, tuple(lengths), shape)
    u = oracle.Updater("RQM4", k2, shape, 1.0 / Ns)
    qs = np.ones((2,) + tuple(shape))
    t0 = time.perf_counter()
    u.solve(w, qs)
    one = time.perf_counter() - t0
    nsteps = max(1, int(seconds / max(one, 1e-6)))
    qs = np.ones((nsteps + 1,) + tuple(shape))
    t0 = time.perf_counter()
    u.solve(w, qs)
    dt = time.perf_counter() - t0
    return nsteps * M / dt, nsteps, dt


def cpu_iteration_rate(cfg, threads, iters, warm=1):
    """Gridpoint contour steps per second of whole SCFT iterations of the CPU
    oracle (Model_AB::update restated: four RQM4 propagators, Q, Simpson
    densities, Anderson mixing) on the workload's seeded fields, `warm`
    untimed iterations then `iters` timed ones; the same unit the GPU arm
    times.  Only the oracle's FFTs use the threads."""
    import oracle
    oracle.build()
    oracle.set_threads(threads)
    L = cfg["cell"][1][0]
    o = oracle.ModelAB(3, cfg["shape"], (L, L, L), cfg["Ms"], cfg["chiN"], lam=cfg["lam"], mde=cfg["mde"],
                       scft=cfg["scft"], n_anderson=cfg["n_anderson"])
    o.init_fields(cfg["wA"], cfg["wB"])
    o.update(warm)
    t0 = time.perf_counter()
    o.update(iters)
    dt = time.perf_counter() - t0
    units = 2 * (sum(cfg["Ms"]) - 2) * int(np.prod(cfg["shape"]))
    return units * iters / dt, dt


def cpu_baseline(cfg, threads, iters=2, one_thread_iters=1):
    """Time the CPU oracle on a bounded sample of the workload: `iters` whole
    SCFT iterations of the 64^3 model on all host threads, and
    `one_thread_iters` on one thread (the reference itself is single-threaded)."""
    rate, dt = cpu_iteration_rate(cfg, threads, iters)
    out = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": "%d whole SCFT iterations (Model_AB::update: propagators, densities, Anderson) of the 64^3 "
                     "workload by oracle/scft_oracle.c (own FFT, %d OpenMP threads), %.1f s" % (iters, threads, dt)}
    if one_thread_iters:
        r1, dt1 = cpu_iteration_rate(cfg, 1, one_thread_iters)
        out["one_thread"] = {"value": r1, "unit": UNIT, "cores": 1,
                             "sample": "%d whole SCFT iteration(s) on one thread, %.1f s" % (one_thread_iters, dt1)}
    return out


def bench_config(cfg, world):
    """The `config` object both arms print."""
    return {"workload": WORKLOAD, "grid": list(cfg["shape"]), "Ns": sum(cfg["Ms"]) - 2, "Ms": list(cfg["Ms"]),
            "step": "one SCFT iteration (Model_AB::update)", "l2_flush": "inputs > L2 (0.8 GB histories)",
            "parallelism": "replicas" if world > 1 else "single"}


def cpu_string_baseline(seconds, threads, m=40, max_iter=3):
    """The string section's CPU leg: the oracle's RQM4 steps on one 128^2
    image, converted to string iterations per second of the 40-image C3
    string (2 Ns steps per image per SCFT iteration).  Propagation only, about
    95% of the work, so the CPU rate is if anything overstated."""
    from polystring_b200 import workloads
    shape, L = (128, 128, 1), 8.0
    Ms = workloads.ms_from(0.35, 128)
    wa, _ = workloads.string_images(m=m, shape=shape, L=L)
    rate, nsteps, dt = cpu_propagation_rate(2, shape, (L, L), Ms, wa[m // 2], seconds, threads)
    work = m * max_iter * 2 * (Ms[0] + Ms[1] - 2) * int(np.prod(shape))
    return {"string_iters_per_s": rate / work, "gridpt_steps_per_s": rate, "cores": threads, "kind": "port",
            "sample": "%d RQM4 steps of one 128^2 image propagator (oracle, %d OpenMP threads), %.1f s; "
                      "propagation only" % (nsteps, threads, dt)}


def cpu_batch_baseline(seconds, threads, n=256):
    """The uneven batch's CPU leg: the oracle's RQM4 rate on each grid of the
    sample (seconds split between them), applied to every solve's 2 Ns M
    steps, as one host process running the solves one after another would."""
    from polystring_b200 import workloads
    n_ab, n_abc = c5_split(n)
    specs = workloads.uneven_solves(n_ab)
    tri = workloads.uneven_triblocks(n_abc)
    rates, samples = {}, []
    shapes = sorted({tuple(sp["shape"]) for sp in specs})
    for shp in shapes:
        sp = next(x for x in specs if tuple(x["shape"]) == shp)
        L = sp["cell"][1][0]
        r, nsteps, dt = cpu_propagation_rate(3, shp, (L, L, L), sp["Ms"], sp["wA"], seconds / len(shapes), threads)
        rates[shp] = r
        samples.append("%d steps at %d^3 in %.1f s" % (nsteps, shp[0], dt))
    specs = specs + tri
    work = [2 * (sum(sp["Ms"]) - len(sp["Ms"])) * int(np.prod(sp["shape"])) for sp in specs]
    t = sum(w / rates[tuple(sp["shape"])] for w, sp in zip(work, specs))
    return {"gridpt_steps_per_s": sum(work) / t, "cores": threads, "kind": "port",
            "sample": "oracle RQM4 propagators, %d OpenMP threads: %s; propagation only"
                      % (threads, ", ".join(samples))}


def string_method(ps, fp64=(37.0, "nominal"), iters=200, seq_reps=3):
    """Secondary result: the batched string method (40 images, 2D 128x128,
    Ns 128, 3 SCFT iterations per image per string iteration; the config's
    200 string iterations timed) against the same SCFT work run image by image
    through the plain single-model path (seq_reps string iterations' worth,
    averaged)."""
    from polystring_b200 import workloads
    m, shape, L = 40, (128, 128, 1), 8.0
    Ms = workloads.ms_from(0.35, 128)
    wa, wb = workloads.string_images(m=m, shape=shape, L=L)
    cell = ps.make_cell(2, "SQUARE", L)
    g = ps.StringAB(m, 2, shape, cell, Ms, 18.0, max_iter=3)
    g.set_images(wa, wb)
    g.iterate(2)
    g.synchronize()
    t0 = time.perf_counter()
    g.iterate(iters)
    g.synchronize()
    tb = (time.perf_counter() - t0) / iters
    single = ps.ModelAB(2, shape, cell, Ms, 18.0)
    single.set_fields(wa[0], wb[0])
    single.update(3)
    single.synchronize()
    t0 = time.perf_counter()
    for rep in range(seq_reps):
        for s in range(m):
            single.set_fields(wa[s], wb[s])
            single.update(3)
            single.H()
    ts = (time.perf_counter() - t0) / seq_reps
    # the whole string iteration as propagator work: 2 Ns steps of M points
    # per image and SCFT iteration, 15 log2(M) + 20 FP64 flops each
    import math
    M = int(np.prod(shape))
    rate = m * 3 * 2 * (Ms[0] + Ms[1] - 2) * M / tb
    flop = 15.0 * math.log2(M) + 20.0
    return {"config": "C3 string, 40 images 128x128, Ms %s, 3 SCFT iterations per image" % list(Ms),
            "batched_string_iters_per_s": 1.0 / tb, "sequential_plain_gpu_iters_per_s": 1.0 / ts,
            "gridpt_steps_per_s": rate,
            "fp64": {"flop_per_gridpt_step": flop, "achieved_tflops": rate * flop / 1e12, "peak_tflops": fp64[0],
                     "peak_kind": fp64[1], "frac": rate * flop / (fp64[0] * 1e12),
                     "note": "whole string iteration (densities, mixing, spline included) counted as propagation"},
            "speedup_vs_sequential": ts / tb, "launches_per_string_iteration": g.launches_per_iteration(),
            "propagator_path": [l for l in ps.lib().ps_tuning_log().decode().split("\ngrid ") if "128x128x1" in l],
            "string_iterations_timed": iters, "sequential_string_iterations_timed": seq_reps,
            "timing": "host wall clock around synchronised replays"}


def c5_split(n):
    """C5's n solves: three quarters AB diblocks, one quarter ABC triblocks."""
    return n - n // 4, n // 4


def uneven_batch(ps, n=256, iters=2):
    """Secondary result: the C5 workload -- n = 256 independent solves of
    uneven grids (32^3, 48^3, 64^3) and Ns (64, 128, 256), 192 AB diblocks
    and 64 linear ABC triblocks -- advanced as one batch for `iters` Anderson
    iterations (of the 300 the workload runs), against the same solves run
    one after another, each on its own fastest single path (persistent sweeps
    for the AB solves on these cubic grids, line passes for the triblocks).
    Device time by CUDA events."""
    from polystring_b200 import workloads
    n_ab, n_abc = c5_split(n)
    specs = workloads.uneven_solves(n_ab)
    tri = workloads.uneven_triblocks(n_abc)

    def model_args(sp):
        return dict(dim=sp["dim"], shape=sp["shape"], cell=ps.make_cell(3, "CUBIC", sp["cell"][1][0]), Ms=sp["Ms"],
                    chiN=sp["chiN"], lam=sp["lam"], scft=sp["scft"], n_anderson=sp["n_anderson"])

    def abc_args(sp):
        return dict(dim=sp["dim"], shape=sp["shape"], cell=ps.make_cell(3, "CUBIC", sp["cell"][1][0]), Ms=sp["Ms"],
                    chi=sp["chi"], lam=sp["lam"], scft=sp["scft"], n_anderson=sp["n_anderson"])
    b = ps.BatchAB([model_args(sp) for sp in specs], [abc_args(sp) for sp in tri])
    for k, sp in enumerate(specs):
        b.set_fields(k, sp["wA"], sp["wB"])
    for j, sp in enumerate(tri):
        b.set_fields(n_ab + j, *sp["w"])
    b.update(1)
    tb = b.update_timed(iters) / 1e3
    work = b.gridpoint_steps() * iters
    launches = b.launches_per_iteration()
    launches_prop = b.launches_per_propagate()
    del b
    ts = ts_abc = 0.0
    for sp in specs:
        m = ps.ModelAB(**model_args(sp))
        m.set_fields(sp["wA"], sp["wB"])
        m.update(1)
        ts += m.update_timed(iters)[0] / 1e3
        del m
    for sp in tri:
        m = ps.ModelABC(**abc_args(sp)).set_fields(*sp["w"])
        m.update(1)
        m.synchronize()
        t0 = time.perf_counter()
        m.update(iters)
        m.synchronize()
        ts_abc += time.perf_counter() - t0
        del m
    sizes = sorted({sp["shape"][0] for sp in specs})
    return {"config": "C5: %d solves (%d AB, %d linear ABC), grids %s^3, Ns 64/128/256, Anderson(10), "
                      "%d of 300 iterations timed" % (n, n_ab, n_abc, sizes, iters),
            "batch_gridpt_steps_per_s": work / tb, "sequential_gridpt_steps_per_s": work / (ts + ts_abc),
            "speedup_vs_sequential": (ts + ts_abc) / tb, "launches_per_batch_iteration": launches,
            "launches_split": {"propagators": launches_prop, "q_density_field_update": launches - launches_prop,
                               "note": "one persistent sweep launch covers all contour steps of the solves it "
                                       "carries; the rest are each member's own small Q, density and Anderson "
                                       "kernels, replayed in the same graph"},
            "sequential_s": {"ab": ts, "abc": ts_abc},
            "timing": "CUDA events on the batch stream and each AB solve's stream; host clock around "
                      "synchronised runs for each ABC solve"}


def adjoint_c4(ps, thresh=1e-9, max_iter=2000):
    """Secondary result: the adjoint on C4 (48^3 orthorhombic (3.8, 4.0, 4.2),
    fA 0.30, chiN 22, Ns 128, seeded noise plus an ordered seed, converged by
    Anderson mixing to residual `thresh`): time of one stress evaluation
    (dF/dL_cell) and of one loss gradient (Loss = ||phiA - phi_target||^2,
    phi_target a smoothed seeded field in [0, 1]), each including its forward
    map, and their agreement with central differences of the forward map:
    fourth order at h = 1e-4 (stress) or 1e-3 (loss) and second order at
    h = 1e-6."""
    from polystring_b200 import workloads as wl
    cfg = wl.config("C4")
    m = wl.model_of(ps, cfg)
    m.set_fields(cfg["wA"], cfg["wB"])
    t0 = time.perf_counter()
    iters, res = wl.converge(m, thresh, max_iter)
    t_conv = time.perf_counter() - t0
    wA, wB = m.get("wA"), m.get("wB")
    tgt = wl.smoothed_target(cfg["shape"])
    m.set_fields(wA, wB)
    st = m.stress()
    t0 = time.perf_counter()
    for _ in range(3):
        st = m.stress()
    t_stress = (time.perf_counter() - t0) / 3
    st_ck = m.stress(checkpoints=0)
    m.forward()
    phi = m.get("phiA")
    t0 = time.perf_counter()
    for _ in range(3):
        gA, gB = m.grad_w(2.0 * (phi - tgt), np.zeros(cfg["shape"]), 0.0)
    t_grad = (time.perf_counter() - t0) / 3
    fd4 = [wl.stress_fd(ps, cfg, wA, wB, i, 1e-4, order=4) for i in range(3)]
    fd2 = [wl.stress_fd(ps, cfg, wA, wB, i, 1e-6, order=2) for i in range(3)]
    rel = lambda a, b: max(abs(x - y) / abs(y) for x, y in zip(a, b))
    # direction: the gradient modulated by a smooth seeded field (a large
    # projection on the gradient, so the check is not a cancellation)
    sc = max(np.abs(gA).max(), np.abs(gB).max())
    mod = 1.0 + wl.smoothed_target(cfg["shape"], seed=21)
    dA, dB = gA * mod / sc, gB * mod / sc
    an = float((gA * dA).sum() + (gB * dB).sum())
    gfd4 = wl.loss_fd(m, wA, wB, dA, dB, tgt, 1e-3, order=4)
    gfd2 = wl.loss_fd(m, wA, wB, dA, dB, tgt, 1e-6, order=2)
    Ns = sum(cfg["Ms"]) - 2
    M = int(np.prod(cfg["shape"]))
    return {"config": "C4 48^3 orthorhombic (3.8, 4.0, 4.2), Ms %s, seeded noise + ordered seed, %d Anderson(20) "
                      "iterations to residual %.1e (%.1f s)" % (list(cfg["Ms"]), iters, res, t_conv),
            "stress": list(st), "stress_checkpointed": list(st_ck), "checkpointed_rel_diff": rel(st_ck, st),
            "stress_ms": t_stress * 1e3, "loss_gradient_ms": t_grad * 1e3,
            "stress_fd4_h1e-4_rel_err_max": rel(st, fd4), "stress_fd2_h1e-6_rel_err_max": rel(st, fd2),
            "gradient_fd4_h1e-3_rel_err": abs(gfd4 - an) / abs(an),
            "gradient_fd2_h1e-6_rel_err": abs(gfd2 - an) / abs(an),
            "fd_note": "central differences of the GPU forward map; loss differences formed point by point",
            "adjoint_gridpt_steps_per_s": Ns * M / t_stress,
            "timing": "host wall clock around synchronised calls (forward map included)"}


def cufft_comparison(ps, cfg, m, reps=3):
    """Comparison only (never the product): the same packed RQM4 chain sweep of
    C2 (both chains of one SCFT iteration, Ns contour steps, histories kept)
    written with torch.fft (cuFFT, complex128) and torch elementwise kernels,
    captured in one CUDA graph.  Checked against this library's sweep on the
    same fields; device time by CUDA events."""
    import torch
    dev = torch.device("cuda")
    shape = cfg["shape"]
    M = int(np.prod(shape))
    LA, LB = cfg["Ms"][0] - 1, cfg["Ms"][1] - 1
    Ns = LA + LB
    ds = 1.0 / Ns
    L = cfg["cell"][1][0]
    r = [np.minimum(np.arange(n), n - np.arange(n)) for n in shape]
    k2 = -(2 * np.pi / L) ** 2 * (r[0][:, None, None] ** 2 + r[1][None, :, None] ** 2 + r[2][None, None, :] ** 2)
    L1 = torch.from_numpy(np.exp(ds * k2)).to(dev)
    L2 = torch.from_numpy(np.exp(0.5 * ds * k2)).to(dev)
    wA = torch.from_numpy(np.ascontiguousarray(cfg["wA"])).to(dev)
    wB = torch.from_numpy(np.ascontiguousarray(cfg["wB"])).to(dev)
    eF = {0: torch.exp(-wA * ds / 2), 1: torch.exp(-wB * ds / 2)}
    eH = {0: torch.exp(-wA * ds / 4), 1: torch.exp(-wB * ds / 4)}
    hist = torch.zeros((Ns + 1,) + tuple(shape), dtype=torch.complex128, device=dev)
    hist[0] = torch.complex(torch.ones(shape, dtype=torch.float64, device=dev),
                            torch.ones(shape, dtype=torch.float64, device=dev))

    def lanes(z, a, b):                   # lane f (real) times a, lane c (imag) times b
        return torch.complex(z.real * a, z.imag * b)

    def sweep():
        for t in range(Ns):
            bf, bc = (0 if t < LA else 1), (1 if t < LB else 0)
            q = hist[t]
            u = lanes(torch.fft.ifftn(torch.fft.fftn(lanes(q, eF[bf], eF[bc])) * L1), eF[bf], eF[bc])
            qt = lanes(torch.fft.ifftn(torch.fft.fftn(lanes(q, eH[bf], eH[bc])) * L2), eH[bf], eH[bc])
            qt2 = lanes(torch.fft.ifftn(torch.fft.fftn(lanes(qt, eH[bf], eH[bc])) * L2), eH[bf], eH[bc])
            hist[t + 1] = (4.0 * qt2 - u) / 3.0

    st = torch.cuda.Stream()
    st.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(st):
        sweep()                           # plans and allocations outside the capture
    torch.cuda.current_stream().wait_stream(st)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        sweep()
    g.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        g.replay()
    e1.record()
    torch.cuda.synchronize()
    t_cufft = e0.elapsed_time(e1) / 1e3 / reps
    # this library on the same fields: one propagator sweep of a fresh model
    mm = ps.ModelAB(3, shape, ps.make_cell(3, "CUBIC", L), cfg["Ms"], cfg["chiN"], lam=cfg["lam"])
    mm.set_fields(cfg["wA"], cfg["wB"])
    mm.propagate(1)
    qB = mm.get("qB")[-1]
    ref = hist[Ns].real.cpu().numpy()
    rel = float(np.abs(qB - ref).max() / np.abs(ref).max())
    tot, prop = mm.update_timed(reps)
    ours = prop / 1e3 / reps
    units = 2 * Ns * M
    del mm, hist, g
    torch.cuda.empty_cache()
    return {"what": "C2 propagator sweep (2 x Ns RQM4 steps, packed chains, histories) with torch.fft / cuFFT "
                    "complex128 in one CUDA graph",
            "cufft_gridpt_steps_per_s": units / t_cufft, "ours_gridpt_steps_per_s": units / ours,
            "ours_over_cufft": t_cufft / ours, "max_rel_diff_qB_tail": rel}


def run_reference(args, rank, world):
    """The reference algorithm's CPU restatement on all host threads (rank 0):
    each step is one whole SCFT iteration of the same workload, the unit the
    GPU arm times; then one iteration on one thread."""
    if rank != 0:
        return
    cfg = config()
    import oracle
    oracle.build()
    threads = oracle.max_threads()
    oracle.set_threads(threads)
    L = cfg["cell"][1][0]
    o = oracle.ModelAB(3, cfg["shape"], (L, L, L), cfg["Ms"], cfg["chiN"], lam=cfg["lam"], mde=cfg["mde"],
                       scft=cfg["scft"], n_anderson=cfg["n_anderson"])
    o.init_fields(cfg["wA"], cfg["wB"])
    o.update(max(1, args.warmup))
    t0 = time.perf_counter()
    o.update(args.steps)
    dt = time.perf_counter() - t0
    del o
    Ns = sum(cfg["Ms"]) - 2
    M = int(np.prod(cfg["shape"]))
    v = 2 * Ns * M * args.steps / dt
    r1, dt1 = cpu_iteration_rate(cfg, 1, 1)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded gyroid + noise fields)", "config": bench_config(cfg, world),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": "%d whole SCFT iterations (Model_AB::update) of the 64^3 workload by "
                                       "oracle/scft_oracle.c (own FFT, %d OpenMP threads) after %d untimed, %.1f s"
                                       % (args.steps, threads, max(1, args.warmup), dt),
                             "one_thread": {"value": r1, "unit": UNIT, "cores": 1,
                                            "sample": "1 whole SCFT iteration on one thread, %.1f s" % dt1}},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import torch
    torch.cuda.set_device(local)
    from polystring_b200.dist import Ranks
    ranks = Ranks("nccl")
    dist = ranks.dist
    barrier = ranks.barrier
    allmax = ranks.allmax

    import polystring_b200 as ps
    cfg = config()
    shape = cfg["shape"]
    M = int(np.prod(shape))
    Ns = sum(cfg["Ms"]) - 2
    units_per_step = 2 * Ns * M
    cell = ps.make_cell(3, cfg["cell"][0], cfg["cell"][1][0])
    m = ps.ModelAB(3, shape, cell, cfg["Ms"], cfg["chiN"], lam=cfg["lam"], mde=cfg["mde"], scft=cfg["scft"],
                   n_anderson=cfg["n_anderson"])
    m.set_fields(cfg["wA"], cfg["wB"])
    fp64_meas = fp64_peak_tflops(ps)
    m.update(args.warmup)
    m.synchronize()

    # ---- device-resident timed region --------------------------------------
    barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        # CUDA events on the model's stream around the K replays and around
        # every propagator sweep inside them
        total_ms, prop_ms = m.update_timed(args.steps)
    barrier()
    torch.cuda.synchronize()
    total_s = allmax(total_ms / 1e3)
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile": True, "ms_per_step": total_s / args.steps * 1e3,
                              "propagator_ms_per_step": prop_ms / args.steps,
                              "launches_per_step": m.launches_per_iteration()}), flush=True)
        ranks.close()
        return
    value = ranks.allsum(units_per_step * args.steps) / total_s
    launches = m.launches_per_iteration() * args.steps
    H = m.H()[0]
    if not np.isfinite(H):
        raise RuntimeError("non-finite H after the timed region")

    # ---- end to end through the C ABI with host buffers --------------------
    wA_h = torch.from_numpy(np.ascontiguousarray(cfg["wA"])).pin_memory()
    wB_h = torch.from_numpy(np.ascontiguousarray(cfg["wB"])).pin_memory()
    outs = [torch.empty(shape, dtype=torch.float64).pin_memory() for _ in range(4)]
    K = args.steps
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    m.set_fields(wA_h.numpy(), wB_h.numpy())               # H2D of the inputs
    for _ in range(K):
        m.update(1)
        m.H()                                              # D2H scalars each step (record_interval 1)
        m.residual_error()
    for o, name in zip(outs, ("wA", "wB", "phiA", "phiB")):
        o.numpy()[...] = m.get(name)                       # D2H of the result fields
    e2e_s = allmax(time.perf_counter() - t0)
    e2e = {"value": world * units_per_step * K / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": 2 * M * 8 / K, "d2h_bytes_per_step": (4 * M * 8 + 5 * 8 * K) / K}

    # ---- roofline of the dominant kernel family (propagator line passes) ---
    peak, peak_kind = peaks()
    prop_s = allmax(prop_ms / 1e3)
    achieved = BYTES_PER_GRIDPT_STEP * units_per_step * args.steps / prop_s / 1e9
    tr = traffic_per_gridpt_step()
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": tr * units_per_step if tr else None, "peak_kind": peak_kind,
            "kernel": "propagator sweep (persistent RQM4 kernel), %d launch(es) per iteration" % m.launches_per_propagate(),
            "propagator_share_of_step": prop_s / total_s}
    # the FP64 side of the same kernel: 6 FFTs of M points per RQM4 step at
    # 2.5 log2(M) flops per point each, plus ~20 elementwise flops; at 64^3
    # the FP64 floor is above the HBM floor, so report both and the fraction
    # of the attainable (larger) floor
    import math
    flop = 15.0 * math.log2(M) + 20.0
    rate = units_per_step * args.steps / prop_s
    fp64_peak, fp64_kind = fp64_meas
    fp64_peak *= 1e12
    roof["fp64"] = {"flop_per_gridpt_step": flop, "achieved_tflops": rate * flop / 1e12,
                    "peak_tflops": fp64_peak / 1e12, "peak_kind": fp64_kind, "frac": rate * flop / fp64_peak}
    roof["attainable_frac"] = rate * max(BYTES_PER_GRIDPT_STEP / (peak * 1e9), flop / fp64_peak)

    string = string_method(ps, fp64_meas) if rank == 0 and world == 1 else None
    batch = uneven_batch(ps) if rank == 0 and world == 1 else None
    adj = adjoint_c4(ps) if rank == 0 and world == 1 else None
    cuf = cufft_comparison(ps, cfg, m) if rank == 0 and world == 1 else None

    cpu = None
    if rank == 0 and world == 1:
        import oracle
        cpu = cpu_baseline(cfg, oracle.max_threads())
        if string is not None:
            string["cpu_baseline"] = cpu_string_baseline(0.5 * args.cpu_seconds, oracle.max_threads())
        if batch is not None:
            batch["cpu_baseline"] = cpu_batch_baseline(0.5 * args.cpu_seconds, oracle.max_threads())

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_s / args.steps * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded gyroid + noise fields)",
                "config": bench_config(cfg, world),
                "e2e": e2e, "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu,
                "clocks": clk.summary(), "H_after": H, "string_method": string, "uneven_batch": batch, "adjoint": adj,
                "cufft_comparison": cuf}
        print(json.dumps(line), flush=True)
    ranks.close()


if __name__ == "__main__":
    main()
