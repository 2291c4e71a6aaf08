"""Build the engine library ``libdoe_b200.so`` in-tree with nvcc for sm_100a.

    python -m diffractiveopticalelement_b200.build      (or build() from Python)

Every translation unit under ``csrc/`` is compiled with
``-gencode arch=compute_100a,code=sm_100a`` and linked into one shared library
next to this file, so the library travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdoe_b200.so")
OBJ_DIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the engine needs the CUDA toolkit to build")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _includes(path: str, seen: set) -> set:
    """Every file reachable through #include "..." from `path` (quoted includes only)."""
    import re
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    for name in re.findall(r'^\s*#\s*include\s+"([^"]+)"', open(path).read(), re.M):
        _includes(os.path.normpath(os.path.join(os.path.dirname(path), name)), seen)
    return seen


def _fingerprint(src: str, flags: list[str]) -> str:
    """SHA-256 of the source, every file it includes and the compile flags."""
    import hashlib
    h = hashlib.sha256(" ".join(flags).encode())
    for path in sorted(_includes(src, set())):
        h.update(path.encode())
        with open(path, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def _stale(obj: str, src: str, flags: list[str]) -> bool:
    """An object is rebuilt unless it exists and was compiled from exactly the
    current contents of its source and includes (a stamp beside it holds their
    fingerprint; modification times alone miss an edit made during a build)."""
    stamp = obj + ".sha256"
    if not os.path.exists(obj) or not os.path.exists(stamp):
        return True
    with open(stamp) as f:
        return f.read().strip() != _fingerprint(src, flags)


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    nvcc = _nvcc()
    os.makedirs(OBJ_DIR, exist_ok=True)
    extra = list(extra or [])

    def compile_one(src):
        obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
        flags = [*ARCH, *FLAGS, *extra]
        if _stale(obj, src, flags):
            fp = _fingerprint(src, flags)  # taken before compiling: a later edit leaves the object stale
            cmd = [nvcc, *flags, "-c", src, "-o", obj]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
            if verbose and r.stderr:
                sys.stderr.write(r.stderr)
            with open(obj + ".sha256", "w") as f:
                f.write(fp)
            return obj, True
        return obj, False

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        done = list(ex.map(compile_one, sources()))
    objs = [o for o, _ in done]
    newest = max(os.path.getmtime(o) for o in objs)
    if any(r for _, r in done) or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc, *ARCH, "-shared", "-Xlinker", "-z,defs", "-o", LIB, *objs, "-lcudart"]  # no unresolved symbols
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
