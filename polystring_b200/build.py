"""Build libpolystring_b200.so in-tree with nvcc for sm_100a.

    python -m polystring_b200.build          # incremental
    python -m polystring_b200.build --force  # rebuild everything

Objects and the shared library go to polystring_b200/_build/.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "libpolystring_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I", os.path.join(HERE, "..", "include")]

SOURCES = ["line_pass.cu", "sweep.cu", "sweep64.cu", "cluster_sweep.cu", "twiddles.cu", "field_kernels.cu", "anderson.cu", "engine.cu", "adjoint.cu", "string_ab.cu", "capi.cu", "density_noalloc.cu", "autotune.cu", "grouped_pass.cu", "batch_ab.cu", "fp64_peak.cu", "etdrk4.cu", "model_abc.cu"]


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))] + \
        [os.path.join(HERE, "..", "include", "polystring_b200.h")]


def _needs(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, obj, verbose):
    cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
    return r.stderr


def build(force=False, verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers()
    todo = []
    objs = []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s.replace(".cu", ".o"))
        objs.append(obj)
        if force or _needs(obj, [src] + hdrs):
            todo.append((src, obj))
    logs = []
    if todo:
        with concurrent.futures.ThreadPoolExecutor(max_workers=jobs or min(8, len(todo))) as ex:
            for log in ex.map(lambda a: _compile(a[0], a[1], verbose), todo):
                logs.append(log)
    if force or todo or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB + ".tmp"] + objs
        subprocess.check_call(cmd)
        os.replace(LIB + ".tmp", LIB)
    build_host(force)
    if verbose:
        print("".join(logs))
    return LIB


# host executables: name -> their own source (each links polyorder.cc too)
HOST_APPS = {"polyorder_b200": "polyorder_b200.cc", "polystring_ab_b200": "polystring_ab_b200.cc"}
HOST_EXE = os.path.join(BUILD, "polyorder_b200")
STRING_EXE = os.path.join(BUILD, "polystring_ab_b200")


def build_host(force=False):
    """The C++ host classes and the two drivers (plain SCFT, string method),
    linked against libpolystring_b200.so (g++, rpath to the library's directory)."""
    host = os.path.join(HERE, "host")
    for name, main in HOST_APPS.items():
        exe = os.path.join(BUILD, name)
        srcs = [os.path.join(host, "polyorder.cc"), os.path.join(host, main)]
        deps = srcs + [os.path.join(host, "polyorder.h"), LIB] + _headers()
        if not force and not _needs(exe, deps):
            continue
        cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(HERE, "..", "include"), "-o", exe + ".tmp"] + srcs + \
            ["-L", BUILD, "-lpolystring_b200", "-Wl,-rpath,$ORIGIN"]
        subprocess.check_call(cmd)
        os.replace(exe + ".tmp", exe)
    return HOST_EXE


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
