"""Build recipe for the engine's shared library (sm_100a only).

    python -m molecular2_b200.build            # incremental
    python -m molecular2_b200.build --force

Compiles every ``csrc/*.cu`` with nvcc for ``arch=compute_100a,code=sm_100a``
into objects under ``_build/`` (git-ignored) and links ``libm2jk.so`` beside
this file, against cuBLAS and cuSOLVER from the CUDA toolkit.  nvcc
cross-compiles here without a GPU; the .so travels with the repository
snapshot to the GPU host.
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(os.path.dirname(HERE), "_build")
LIB = os.path.join(HERE, "libm2jk.so")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-Xptxas", "-warn-spills"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def deps(src, seen=None):
    """Transitive local #include "..." dependencies of a source file."""
    import re
    seen = set() if seen is None else seen
    for m in re.finditer(r'#include\s+"([^"]+)"', open(src).read()):
        p = os.path.normpath(os.path.join(os.path.dirname(src), m.group(1)))
        if os.path.exists(p) and p not in seen:
            seen.add(p)
            deps(p, seen)
    return seen


def _obj(src):
    return os.path.join(BUILD, os.path.basename(src) + ".o")


def _compile(src, verbose):
    cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", _obj(src)]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, r.stdout + r.stderr


def build(force=False, verbose=False, jobs=None):
    os.makedirs(BUILD, exist_ok=True)
    todo = []
    for s in sources():
        o = _obj(s)
        newest = max([os.path.getmtime(s)] + [os.path.getmtime(h) for h in deps(s)])
        if force or not os.path.exists(o) or os.path.getmtime(o) < newest:
            todo.append(s)
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
        for src, rc, out in ex.map(lambda s: _compile(s, verbose), todo):
            if out.strip() and (verbose or rc):
                print(f"== {os.path.basename(src)}\n{out}", file=sys.stderr)
            if rc:
                raise RuntimeError(f"nvcc failed on {src}")
    objs = [_obj(s) for s in sources()]
    if todo or not os.path.exists(LIB):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcublas", "-lcusolver"]
        subprocess.check_call(cmd)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
