"""Builds halloc-b200 for sm_100a, in-tree.

Outputs (all git-ignored, all travel with the source tree):

* ``halloc_b200/libhalloc.a``       -- relocatable-device-code static library
  with hamalloc/hafree/ha_init/...: the drop-in for halloc's libhalloc.a.
  Users compile with ``-rdc=true`` and link it (include/halloc.h).
* ``halloc_b200/libhalloc_b200.so`` -- the same allocator plus the batch
  kernels, device-linked, exporting the C ABI of include/halloc_c.h.
* ``halloc_b200/libhalloc_b200_stamps.so`` -- an instrumented copy (latency
  stamps, -DHA_STAMPS) for halloc_b200/stamps.py only.

Run ``python -m halloc_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
SO = os.path.join(PKG, "libhalloc_b200.so")
LIB_A = os.path.join(PKG, "libhalloc.a")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-rdc=true", "-Xcompiler", "-fPIC",
                  "-I" + INCLUDE, "-I" + CSRC]

HEADERS = [os.path.join(CSRC, f) for f in ("ha_core.cuh", "ha_types.h", "ha_hist.cuh",
                                           "ha_stamp.cuh")] + [
    os.path.join(INCLUDE, f) for f in ("halloc.h", "halloc_c.h")]
# The allocator's device functions are capped at 64 registers: every kernel
# that calls hamalloc/hafree inherits the callee's register count at device
# link time, so this bounds the occupancy cost for user kernels (the
# reference built with the same cap).
SOURCES = {"halloc.cu": ["-maxrregcount=64"], "ha_kernels.cu": [],
           "ha_serve.cu": ["-maxrregcount=64"], "ha_samples.cu": []}


def nvcc() -> str:
    env = os.environ.get("NVCC")
    if env:
        return env
    for cand in ("/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


STAMPS_SO = os.path.join(PKG, "libhalloc_b200_stamps.so")
STAMPS_BUILD = os.path.join(PKG, "_build_stamps")


def build_stamps(verbose: bool = False, defines=()) -> str:
    """The instrumented library (-DHA_STAMPS): the allocator and the batch
    kernels with latency stamps after every dependent round trip of
    hamalloc / hafree (see csrc/ha_stamp.cuh).  Used only by
    halloc_b200/stamps.py, never by the product path."""
    os.makedirs(STAMPS_BUILD, exist_ok=True)
    cc = nvcc()
    objs = []
    dflags = ["-D" + d for d in defines]
    for src in ("halloc.cu", "ha_kernels.cu"):
        s = os.path.join(CSRC, src)
        o = os.path.join(STAMPS_BUILD, src.replace(".cu", ".o"))
        if _stale(o, [s, __file__] + HEADERS) or dflags:
            _run([cc] + CUFLAGS + SOURCES[src] + dflags + ["-DHA_STAMPS", "-c", s, "-o", o],
                 verbose)
        objs.append(o)
    dlink = os.path.join(STAMPS_BUILD, "dlink.o")
    if _stale(STAMPS_SO, objs) or dflags:
        _run([cc] + ARCH + ["-Xcompiler", "-fPIC", "-dlink"] + objs + ["-o", dlink], verbose)
        _run([cc] + ARCH + ["-shared", "-Xcompiler", "-fPIC"] + objs + [dlink, "-o", STAMPS_SO,
                                                                         "-lcudadevrt"],
             verbose)
    return STAMPS_SO


def build(verbose: bool = False, ptxas_info: bool = False, defines=()) -> str:
    """Compiles what is out of date; returns the path of the shared library.
    `defines` (e.g. ["HA_L2_HINTS=0"]) rebuilds everything with those macros:
    a variant build for a measurement, replacing the default one in place."""
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    objs = []
    dflags = ["-D" + d for d in defines]
    for src, flags in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        if _stale(o, [s, __file__] + HEADERS) or ptxas_info or dflags:
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            _run([cc] + CUFLAGS + flags + dflags + extra + ["-c", s, "-o", o], verbose)
        objs.append(o)
    halloc_o = objs[0]
    if _stale(LIB_A, [halloc_o]) or dflags:
        _run([cc] + ARCH + ["-lib", halloc_o, "-o", LIB_A], verbose)
    dlink = os.path.join(BUILD, "dlink.o")
    if _stale(SO, objs) or dflags:
        _run([cc] + ARCH + ["-Xcompiler", "-fPIC", "-dlink"] + objs + ["-o", dlink], verbose)
        _run([cc] + ARCH + ["-shared", "-Xcompiler", "-fPIC"] + objs + [dlink, "-o", SO,
                                                                         "-lcudadevrt"],
             verbose)
    _build_pyfast(verbose)
    build_stamps(verbose, defines)
    return SO


def _build_pyfast(verbose: bool) -> None:
    """The CPython fast path of the host-buffer loop (csrc/ha_pyfast.c), linked
    against the shared library beside it."""
    import sysconfig
    src = os.path.join(CSRC, "ha_pyfast.c")
    out = os.path.join(PKG, "_pyfast" + sysconfig.get_config_var("EXT_SUFFIX"))
    if not _stale(out, [src, SO, os.path.join(INCLUDE, "halloc_c.h")]):
        return
    _run(["gcc", "-O2", "-shared", "-fPIC", "-Wall", "-I" + sysconfig.get_paths()["include"],
          "-I" + INCLUDE, src, "-o", out, "-L" + PKG, "-l:" + os.path.basename(SO),
          "-Wl,-rpath,$ORIGIN"], verbose)


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv,
          defines=[a[2:] for a in sys.argv[1:] if a.startswith("-D")])
    print(SO)
