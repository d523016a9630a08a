"""Build the in-tree CUDA library libugks_b200.so for sm_100a with nvcc (no JIT, no torch extension).

The shared library sits next to this file so that it travels with the repository snapshot.  Each
translation unit is compiled to an object in _build/ on its own nvcc process (they run in parallel),
then the objects are linked; no device code crosses translation units, so this is the same program
as one nvcc call over all sources.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(ROOT, "_build", "ugks_b200")
LIB = os.path.join(HERE, "libugks_b200.so")
SOURCES = ["ugks_lo.cu", "ugks_implicit.cu", "ugks_s2.cu", "ugks_s2cn2.cu", "ugks_batch.cu", "ugks_capi.cu",
           "ugks_noalloc.cu", "ugks_s2_adjoint.cu", "ugks_s2_walls.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                "-I" + os.path.join(ROOT, "include")]


def _sources():
    return [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "ugks_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False, extra=()):
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    objs, cmds = [], []
    for s in _sources():
        o = os.path.join(OBJ, s.replace(".cu", ".o"))
        objs.append(o)
        cmds.append([NVCC] + FLAGS + list(extra) + ["-c", os.path.join(CSRC, s), "-o", o])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        return subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        results = list(ex.map(run, cmds))
    for cmd, r in zip(cmds, results):
        if r.stdout or r.stderr:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise subprocess.CalledProcessError(r.returncode, cmd)
    link = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.run(link, check=True)
    return LIB


if __name__ == "__main__":
    build(force=True, verbose=True, extra=sys.argv[1:])
