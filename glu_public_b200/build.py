"""In-tree build of ``libglu_b200.so`` (CUDA kernels + C ABI) for sm_100a with nvcc.

The library is built next to this file so it travels with the repository; it is loaded with
ctypes by :mod:`glu_public_b200._lib`.  Run ``python -m glu_public_b200.build``.
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libglu_b200.so")
STAMP = LIB + ".srchash"

SOURCES = ["api.cu", "kernels.cu", "dense.cu", "noalloc.cu", "plan_host.cpp", "symbolic.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _src_hash() -> str:
    h = hashlib.sha256()
    names = sorted(os.listdir(CSRC))
    for name in names:
        with open(os.path.join(CSRC, name), "rb") as f:
            h.update(name.encode())
            h.update(f.read())
    with open(os.path.join(INCLUDE, "glu_b200.h"), "rb") as f:
        h.update(f.read())
    h.update(" ".join(ARCH).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles the library unless an up-to-date build exists; returns its path."""
    digest = _src_hash()
    if not force and os.path.exists(LIB) and os.path.exists(STAMP):
        with open(STAMP) as f:
            if f.read().strip() == digest:
                return LIB
    cmd = [_nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
           "-Xptxas", "-v" if verbose else "-O3", f"-I{INCLUDE}", f"-I{CSRC}",
           "-Xlinker", "--exclude-libs,ALL", "-o", LIB + ".tmp"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libglu_b200.so")
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(LIB + ".tmp", LIB)
    with open(STAMP, "w") as f:
        f.write(digest)
    return LIB


CMD_SRC = os.path.join(HERE, "cmd", "glu_cmd.cpp")
CMD = os.path.join(HERE, "glu_cmd")


def build_cmd(force: bool = False) -> str:
    """Compiles the C++ driver glu_cmd against the library and the CUDA runtime (host code only;
    it finds libglu_b200.so next to itself)."""
    lib = build()
    if (not force and os.path.exists(CMD) and os.path.getmtime(CMD) >= os.path.getmtime(lib)
            and os.path.getmtime(CMD) >= os.path.getmtime(CMD_SRC)):
        return CMD
    cuda = os.path.dirname(os.path.dirname(_nvcc()))
    cmd = ["g++", "-O2", "-std=c++17", f"-I{INCLUDE}", f"-I{os.path.join(cuda, 'include')}",
           CMD_SRC, "-o", CMD + ".tmp", f"-L{HERE}", "-lglu_b200",
           f"-L{os.path.join(cuda, 'lib64')}", "-lcudart", "-Wl,-rpath,$ORIGIN",
           f"-Wl,-rpath,{os.path.join(cuda, 'lib64')}"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("g++ failed building glu_cmd")
    os.replace(CMD + ".tmp", CMD)
    return CMD


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
    print(build_cmd(force="--force" in sys.argv))
