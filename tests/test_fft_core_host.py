"""The radix butterflies and Stockham index arithmetic of the CUDA FFT core
(polystring_b200/csrc/fft_core.cuh), compiled for the host with g++ and
checked against a long-double DFT for every supported line length."""
import os
import subprocess
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_fft_core_all_lengths():
    src = os.path.join(ROOT, "tests", "native", "fft_core_check.cpp")
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "fft_core_check")
        subprocess.check_call(["g++", "-O2", "-std=c++17", "-o", exe, src])
        r = subprocess.run([exe], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
        lines = [l.split() for l in r.stdout.splitlines()]
        assert len(lines) >= 21
        assert max(float(l[2]) for l in lines) < 1e-14


def test_lane_factor_sets():
    """engine.h LaneFactors: the factor set of a packed lane at each step
    (two-block chains, ranges past the junction, triblock chains)."""
    src = os.path.join(ROOT, "tests", "native", "lane_factors_check.cpp")
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "lane_factors_check")
        import shutil
        nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
        inc = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc))), "include")
        subprocess.check_call(["g++", "-O1", "-std=c++17", "-I" + inc, "-o", exe, src])
        r = subprocess.run([exe], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
