"""Build the sm_100a shared library ``libnozzle_b200.so`` in-tree.

    python -m <package>.build            (or: python 2d_nozzle_b200/build.py)

Every ``csrc/*.cu`` translation unit (the C ABI with the forward kernels, and
the adjoint kernels per element kind) is compiled by nvcc for ``sm_100a``
only, with ``-lineinfo`` for profiler source mapping, in parallel; the objects
are linked into one library with the CUDA runtime linked statically, so
loading it needs nothing but the driver.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libnozzle_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    return "nvcc"


def sources() -> list[str]:
    d = os.path.join(HERE, "csrc")
    return [os.path.join(d, f) for f in sorted(os.listdir(d)) if f.endswith((".cu", ".cuh"))] + [
        os.path.join(ROOT, "include", "nozzle_b200.h")
    ]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources())


def units() -> list[str]:
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith(".cu")]


def build(force: bool = False, verbose: bool = False, defines=(), out: str | None = None) -> str:
    """Build the library (``out``: another path, ``defines``: extra -D macros, e.g. launch bounds)."""
    lib = out or LIB
    if not force and not defines and out is None and up_to_date():
        return LIB
    os.makedirs(os.path.dirname(lib), exist_ok=True)
    tag = f"tmp{os.getpid()}"
    flags = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
             "-I", os.path.join(ROOT, "include"), "-I", CSRC, *[f"-D{d}" for d in defines]]
    if verbose:
        flags.insert(0, "-Xptxas=-v")
    objs, procs = [], []
    for src in units():
        obj = os.path.join(os.path.dirname(lib), os.path.basename(src)[:-3] + f".{tag}.o")
        objs.append(obj)
        procs.append((src, subprocess.Popen([nvcc(), *flags, "-c", src, "-o", obj], stdout=subprocess.PIPE,
                                            stderr=subprocess.PIPE, text=True)))
    errors = []
    for src, pr in procs:
        out, err = pr.communicate()
        if pr.returncode != 0:
            errors.append(f"{os.path.basename(src)}: nvcc failed ({pr.returncode}):\n{err[-6000:]}")
        elif verbose:
            sys.stderr.write(err)
    try:
        if errors:
            raise RuntimeError("\n".join(errors))
        tmp = lib + f".{tag}"
        res = subprocess.run([nvcc(), *ARCH, "-shared", "-cudart", "static", *objs, "-o", tmp], capture_output=True,
                             text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed ({res.returncode}):\n{res.stderr[-6000:]}")
        os.replace(tmp, lib)
    finally:
        for o in objs:
            if os.path.exists(o):
                os.remove(o)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
