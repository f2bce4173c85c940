"""Build the native libraries in-tree (gap_b200/lib/).

    python -m gap_b200.csrc.build          # or gap_b200.csrc.build.build()

Everything is compiled for sm_100a only (-gencode arch=compute_100a,code=sm_100a).  nvcc
cross-compiles without a GPU.  Rebuilds a target only when one of its sources is newer.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
LIB = os.path.join(PKG, "lib")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++20", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I" + INCLUDE] + ARCH


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r


CORE_SOURCES = ["symbolic.cpp", "nr.cu", "ybus.cu"]
HEADERS = ["internal.h", "blocks.cuh", "nr_kernels.cuh", "dense_lu_tc.cuh"]


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile libgapk.so; returns its path."""
    os.makedirs(LIB, exist_ok=True)
    nvcc = _nvcc()
    objdir = os.path.join(LIB, "obj")
    os.makedirs(objdir, exist_ok=True)
    hdrs = [os.path.join(HERE, h) for h in HEADERS] + [os.path.join(INCLUDE, "gapk.h")]
    objs = []
    for src in CORE_SOURCES:
        s = os.path.join(HERE, src)
        o = os.path.join(objdir, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + hdrs):
            cmd = [nvcc] + NVCC_FLAGS + ["-c", s, "-o", o]
            if src.endswith(".cpp"):
                cmd = [nvcc] + NVCC_FLAGS + ["-x", "c++", "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)
    so = os.path.join(LIB, "libgapk.so")
    if force or _stale(so, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", so] + objs
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    build_plugins(so, verbose=verbose, force=force)
    build_io_and_cli(verbose=verbose, force=force)
    return so


PLUGINS = {"libgap_admittance_gpu.so": "admittance_gpu.cpp", "libgap_lu_gpu.so": "lu_gpu.cpp",
           "libgap_powerflow_gpu.so": "powerflow_gpu.cpp"}


def build_plugins(core_so, verbose=False, force=False):
    """The reference-ABI plugin libraries (dlopen'ed by name by the reference's
    BackendFactory), linked against libgapk.so with an $ORIGIN rpath."""
    nvcc = _nvcc()
    pdir = os.path.join(HERE, "plugins")
    deps = [os.path.join(pdir, "common.hpp"), os.path.join(INCLUDE, "gap_b200", "gap_interfaces.hpp"),
            os.path.join(INCLUDE, "gapk.h"), core_so]
    for lib, src in PLUGINS.items():
        s = os.path.join(pdir, src)
        out = os.path.join(LIB, lib)
        if force or _stale(out, [s] + deps):
            cmd = [nvcc] + ARCH + ["-x", "c++", "-std=c++20", "-O2", "-Xcompiler", "-fPIC",
                                   "-I" + INCLUDE, "-shared", "-cudart", "static", "-o", out, s,
                                   "-L" + LIB, "-lgapk", "-Xlinker", "-rpath=$ORIGIN"]
            if verbose:
                print(" ".join(cmd))
            _run(cmd)


def build_io_and_cli(verbose=False, force=False):
    """libgap_io_pgm.so (the PGM reader behind the reference's IIOModule; host code only) and
    gap_b200_main (the reference's command-line flow over the B200 libraries, which it loads
    with dlopen through an $ORIGIN rpath)."""
    pdir = os.path.join(HERE, "plugins")
    iface = os.path.join(INCLUDE, "gap_b200", "gap_interfaces.hpp")
    # nvcc's host compiler, as for the plugin libraries (one C++ runtime for every library)
    cxx = [_nvcc(), "-x", "c++", "-cudart", "none"]
    io_src = os.path.join(pdir, "pgm_io.cpp")
    io_so = os.path.join(LIB, "libgap_io_pgm.so")
    if force or _stale(io_so, [io_src, iface, os.path.join(pdir, "json_min.hpp")]):
        cmd = cxx + ["-std=c++20", "-O2", "-Xcompiler", "-fPIC", "-shared", "-I" + INCLUDE, "-o",
                     io_so, io_src]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
    cli_src = os.path.join(pdir, "gap_b200_main.cpp")
    cli = os.path.join(LIB, "gap_b200_main")
    if force or _stale(cli, [cli_src, iface]):
        cmd = cxx + ["-std=c++20", "-O2", "-I" + INCLUDE, "-o", cli, cli_src, "-ldl",
                     "-Xlinker", "-rpath=$ORIGIN"]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)


if __name__ == "__main__":
    p = build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(p)
