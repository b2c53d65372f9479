"""Build recipe of the CUDA library ``fmm2d_b200/libfmm2d_b200.so``.

Every ``csrc/*.cu`` is compiled for sm_100a with nvcc (objects under
``fmm2d_b200/_build/``) and linked into one shared library exporting the C ABI
of ``include/fmm2d_b200.h``.  ``csrc/fortran_abi.c`` becomes
``fmm2d_b200/libfmm2d.so``: the reference library's own Fortran and C entry
points (``include/fmm2d_f77.h``), linked against the first.  Run
``python -m fmm2d_b200.build`` or call ``build()``; ``verbose_ptxas=True``
adds ``-Xptxas -v`` (registers, spills).
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfmm2d_b200.so")
F77_SRC = os.path.join(CSRC, "fortran_abi.c")
F77_LIB = os.path.join(HERE, "libfmm2d.so")
INCLUDE = os.path.join(HERE, "..", "include")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xcompiler", "-Wno-unused-function", "-diag-suppress", "177,550"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + [
        os.path.join(HERE, "..", "include", "fmm2d_b200.h")]


def _stale(obj, src, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + deps if os.path.exists(p))


def build(force=False, verbose_ptxas=False, jobs=None):
    os.makedirs(OUT, exist_ok=True)
    nvcc = _nvcc()
    deps = _headers()
    srcs = _sources()
    objs = []
    todo = []
    for s in srcs:
        o = os.path.join(OUT, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, s, deps):
            cmd = [nvcc] + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose_ptxas else []) + [
                "-c", s, "-o", o]
            todo.append(cmd)

    def run(cmd):
        p = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, p

    failed = []
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        for cmd, p in ex.map(run, todo):
            if p.returncode != 0 or verbose_ptxas:
                sys.stderr.write(p.stdout + p.stderr)
            if p.returncode != 0:
                failed.append(cmd[-3])
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(failed))
    if todo or force or not os.path.exists(LIB) or any(
            os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            sys.stderr.write(p.stdout + p.stderr)
            raise RuntimeError("link failed")
    _build_f77(force)
    return LIB


def _build_f77(force):
    """libfmm2d.so from csrc/fortran_abi.c (gcc), resolving the B200 library
    beside it at run time."""
    deps = [LIB, os.path.join(INCLUDE, "fmm2d_f77.h"), os.path.join(INCLUDE, "fmm2d_b200.h")]
    if not force and not _stale(F77_LIB, F77_SRC, deps):
        return
    cmd = [os.environ.get("CC", "gcc"), "-std=c11", "-O2", "-fPIC", "-shared", "-Wall",
           "-Werror", "-I", INCLUDE, F77_SRC, "-o", F77_LIB, "-L", HERE, "-l:libfmm2d_b200.so",
           "-Wl,-rpath,$ORIGIN", "-Wl,--no-undefined"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError("libfmm2d.so failed to build")


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
    print(LIB)
