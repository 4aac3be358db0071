"""Build recipes for the in-tree native libraries.

``build_engine()`` compiles the sm_100a CUDA engine (samos_b200/csrc) into
samos_b200/libsamos_gpu.so with nvcc; ``build_host()`` compiles the C++
conf-file host (samos_b200/host) against it.  Both are plain command lines so
that the built files sit in the source tree and travel with it.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
INCLUDE = os.path.join(ROOT, "include")
ENGINE_SO = os.path.join(PKG, "libsamos_gpu.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: no a*b+c contraction, so device arithmetic follows the
# reference's evaluation order term by term.
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-shared"]


def _run(cmd: list[str]) -> None:
    print("+", " ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _sources(d: str, exts: tuple[str, ...]) -> list[str]:
    return sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(exts))


def build_engine(force: bool = False) -> str:
    srcs = _sources(CSRC, (".cu", ".cuh")) + [os.path.join(INCLUDE, "samos_gpu.h")]
    if force or _stale(ENGINE_SO, srcs):
        _run([NVCC, *NVCC_FLAGS, *ARCH, f"-I{INCLUDE}", "-o", ENGINE_SO,
              os.path.join(CSRC, "sg_engine.cu"), os.path.join(CSRC, "sg_static.cu"),
              os.path.join(CSRC, "sg_ml.cu")])
    return ENGINE_SO


def build_host(force: bool = False) -> str | None:
    if not os.path.isdir(HOST):
        return None
    cpp = _sources(HOST, (".cpp",))
    if not cpp:
        return None
    target = os.path.join(PKG, "samos-gpu")
    srcs = cpp + _sources(HOST, (".hpp",)) + [ENGINE_SO]
    if force or _stale(target, srcs):
        _run(["g++", "-std=c++17", "-O2", f"-I{INCLUDE}", "-o", target, *cpp,
              f"-L{PKG}", "-lsamos_gpu", "-Wl,-rpath,$ORIGIN"])
    return target


def build_all(force: bool = False) -> None:
    build_engine(force)
    build_host(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
