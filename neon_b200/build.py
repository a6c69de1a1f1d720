"""Build libneon_b200.so in-tree with nvcc for sm_100a.

    python -m neon_b200.build [--verbose-ptxas]

Output: neon_b200/_lib/libneon_b200.so (plus the C++ adapter test driver when requested).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libneon_b200.so")
SOURCES = ["api.cu", "batch.cu", "elements.cu", "loads.cu", "pattern.cu", "pcg.cu", "post.cu",
           "probe.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    headers = sorted(f for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h")))
    deps = [os.path.join(CSRC, s) for s in SOURCES] + [os.path.join(CSRC, h) for h in headers] + [
        os.path.join(ROOT, "include", "neon_b200.h"),
        os.path.join(ROOT, "include", "neon_b200_probe.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = os.path.join(LIBDIR, "obj")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                    "--expt-relaxed-constexpr", "-ccbin", shutil.which("g++") or "g++"]
    if verbose_ptxas:
        flags += ["-Xptxas", "-v"]
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(objdir, s.replace(".cu", ".o"))
        if force or _stale(obj, [src] + deps[len(SOURCES):]):
            cmd = [nvcc()] + flags + ["-c", src, "-o", obj]
            subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-ccbin", shutil.which("g++") or "g++"]
    subprocess.run(cmd, check=True)
    return LIB


DRIVER = os.path.join(LIBDIR, "adapter_driver")


def build_adapter_driver(force: bool = False) -> str:
    """C++ consumer of include/neon_b200.hpp (tests/cpp/adapter_driver.cpp), linked against the
    library with an $ORIGIN rpath so it runs from the tree."""
    lib = build()
    src = os.path.join(ROOT, "tests", "cpp", "adapter_driver.cpp")
    deps = [src, lib, os.path.join(ROOT, "include", "neon_b200.hpp"),
            os.path.join(ROOT, "include", "neon_b200_json.hpp")]
    if force or _stale(DRIVER, deps):
        cmd = [shutil.which("g++") or "g++", "-std=c++17", "-O2", src, "-o", DRIVER,
               "-I" + os.path.join(ROOT, "include"), "-L" + LIBDIR, "-lneon_b200",
               "-Wl,-rpath,$ORIGIN"]
        inc = nlohmann_include()
        if inc:
            cmd += ["-DNB2_DRIVER_JSON", "-I" + inc]
        subprocess.run(cmd, check=True)
    return DRIVER


def nlohmann_include() -> str | None:
    """A directory holding nlohmann/json.hpp (the JSON library neon uses), for the driver's deck
    mode: $NLOHMANN_JSON_INCLUDE, the system include paths, or a copy that a Python package in
    this environment vendors.  None when there is none."""
    cands = [os.environ.get("NLOHMANN_JSON_INCLUDE", ""), "/usr/include", "/usr/local/include"]
    import site
    import sysconfig
    roots = {sysconfig.get_paths()["purelib"], *site.getsitepackages()}
    for r in sorted(roots):
        cands += [os.path.join(r, "include", "cudnn_frontend", "thirdparty"),
                  os.path.join(r, "include")]
    for c in cands:
        if c and os.path.isfile(os.path.join(c, "nlohmann", "json.hpp")):
            return c
    return None


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--verbose-ptxas" in sys.argv)
    build_adapter_driver(force="--force" in sys.argv)
    print(LIB)
