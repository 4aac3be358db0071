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
NVCC_COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC"]
# The FP64 particle path (engine, allocation-free entry point) is compiled
# with -fmad=false: no a*b+c contraction, so device arithmetic follows the
# reference's evaluation order term by term.  The FP32/BF16 network kernels of
# the learned warm start have no bit-parity requirement and keep FMA.
PARITY_UNITS = ("sg_engine.cu", "sg_static.cu")
FREE_UNITS = ("sg_ml.cu",)
OBJ_DIR = os.path.join(PKG, "_build")


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
        os.makedirs(OBJ_DIR, exist_ok=True)
        objs, procs = [], []
        for unit in PARITY_UNITS + FREE_UNITS:  # independent units, compiled side by side
            obj = os.path.join(OBJ_DIR, unit.replace(".cu", ".o"))
            fmad = ["-fmad=false"] if unit in PARITY_UNITS else []
            cmd = [NVCC, *NVCC_COMMON, *fmad, *ARCH, f"-I{INCLUDE}", "-c", os.path.join(CSRC, unit), "-o", obj]
            print("+", " ".join(cmd), file=sys.stderr)
            procs.append((cmd, subprocess.Popen(cmd)))
            objs.append(obj)
        for cmd, p in procs:
            if p.wait() != 0:
                raise subprocess.CalledProcessError(p.returncode, cmd)
        _run([NVCC, "-shared", *ARCH, "-o", ENGINE_SO, *objs])
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
