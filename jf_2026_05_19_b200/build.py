"""Build recipe for the in-tree CUDA library ``libjfemgpu.so`` (sm_100a).

The library is a plain C-ABI shared object (include/jfem_gpu.h) compiled
with nvcc for sm_100a only; it is built in-tree so it travels with the
repository snapshot.
"""
from __future__ import annotations

import hashlib
import os
import re
import shutil
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libjfemgpu.so")
SOURCES = ["jfg_api.cu", "jfg_server.cu", "jfg_host.cpp"]
_INCLUDE = re.compile(r'^\s*#\s*include\s*"([^"]+)"', re.M)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_compiler() -> list:
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def deps() -> list:
    """Every file the library is compiled from: the SOURCES and, transitively,
    every quoted #include they reach (resolved against the including file's
    folder, as the preprocessor does).  Sorted, so the hash is stable."""
    seen, todo = set(), [os.path.join(CSRC, f) for f in SOURCES]
    while todo:
        p = os.path.normpath(todo.pop())
        if p in seen:
            continue
        seen.add(p)
        with open(p) as f:
            for inc in _INCLUDE.findall(f.read()):
                q = os.path.join(os.path.dirname(p), inc)
                if not os.path.exists(q):
                    raise FileNotFoundError(f"{p} includes {inc}, which does not exist")
                todo.append(q)
    return sorted(seen)


def source_hash() -> str:
    """Content hash of every source and header the library is built from.

    It is compiled into the library (reported by jfg_version) so that a
    library built from other sources -- whose entry points may have other
    signatures -- is never loaded by mistake, whatever the file times are."""
    h = hashlib.sha256()
    for p in deps():
        h.update(os.path.relpath(p, ROOT).encode())
        with open(p, "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def built_hash() -> str:
    """Source hash recorded beside the built library, or '' when absent."""
    try:
        with open(LIB + ".srchash") as f:
            return f.read().strip()
    except OSError:
        return ""


def needs_build() -> bool:
    return not os.path.exists(LIB) or built_hash() != source_hash()


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    if not force and not needs_build():
        return LIB
    sh = source_hash()
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "--expt-relaxed-constexpr", *host_compiler(), "-I", os.path.join(ROOT, "include"),
           f"-DJFG_SRC_HASH=\"{sh}\"", *(extra or []), "-o", LIB + ".tmp", *[os.path.join(CSRC, s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    with open(LIB + ".srchash", "w") as f:
        f.write(sh + "\n")
    return LIB


if __name__ == "__main__":
    import sys
    print(build(force="--force" in sys.argv, verbose=True,
                extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None))
