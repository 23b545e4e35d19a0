"""Builds the native parts in-tree (no GPU needed: nvcc cross-compiles sm_100a).

Outputs (flysim_b200/_build/):
  libflysim_b200.so   device engine (CUDA, sm_100a) + host model (parser,
                      builder, protocol driver) behind the C ABI of
                      include/flysim_b200.h
  flysim              the drop-in command line
  fs_gen_tables       generator of the glibc expf/logf exception tables
  expf_glibc.bin, logf_glibc.bin   the tables (generated by calling glibc)

The compat kernels are compiled with -fmad=false so that no multiply-add is
contracted (the reference's x86-64 build has no FMA); nothing is compiled
with fast-math, and host code is compiled without -march so libm and the
arithmetic match the reference build.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
INC = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

HOST_SRC = ["host/fs_parse.cpp", "host/fs_build.cpp", "host/fs_driver.cpp", "host/fs_model_api.cpp",
            "host/fs_tables.cpp", "host/fs_cache.cpp", "host/fs_netlog.cpp"]
CU_SRC = {"fs_engine.cu": [], "fs_prod.cu": [], "fs_compat.cu": ["-fmad=false"], "fs_mlp.cu": []}
HDRS = ["fs_device.cuh", "fs_prod.cuh", "host/fs_host.hpp"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    return r


def build(verbose: bool = False, tables: bool = True) -> str:
    os.makedirs(OUT, exist_ok=True)
    hdr = [os.path.join(CSRC, h) for h in HDRS] + [os.path.join(INC, "flysim_b200.h")]
    objs = []
    for src in HOST_SRC:
        s = os.path.join(CSRC, src)
        o = os.path.join(OUT, os.path.basename(src) + ".o")
        if _newer(o, [s] + hdr):
            _run(["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-Wno-unused-function", "-I", INC,
                  "-I", os.path.join(CSRC, "host"), "-c", s, "-o", o], verbose)
        objs.append(o)
    for src, extra in CU_SRC.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(OUT, src + ".o")
        if _newer(o, [s] + hdr):
            _run([NVCC, "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", "-I", INC,
                  "-I", CSRC, "-I", os.path.join(CSRC, "host"), *extra, "-c", s, "-o", o], verbose)
        objs.append(o)
    lib = os.path.join(OUT, "libflysim_b200.so")
    if _newer(lib, objs):
        _run([NVCC, "-shared", *ARCH, "-o", lib, *objs, "-cudart", "static", "-ldl", "-lpthread"], verbose)
    cli = os.path.join(OUT, "flysim")
    cli_src = os.path.join(CSRC, "host", "fs_cli.cpp")
    if _newer(cli, [cli_src, lib] + hdr):
        _run(["g++", "-std=c++17", "-O2", "-I", INC, "-I", os.path.join(CSRC, "host"), cli_src, "-o", cli,
              "-L", OUT, "-lflysim_b200", "-Wl,-rpath,$ORIGIN"], verbose)
    gen = os.path.join(OUT, "fs_gen_tables")
    gen_src = os.path.join(CSRC, "host", "fs_tables.cpp")
    if _newer(gen, [gen_src]):
        _run(["g++", "-std=c++17", "-O2", "-DFS_TABLES_MAIN", gen_src, "-o", gen, "-pthread"], verbose)
    if tables:
        tab = os.path.join(OUT, "expf_glibc.bin")
        if _newer(tab, [gen]):
            _run([gen, OUT], verbose)
    return lib


def build_oracle(verbose: bool = False, ref_src: str | None = None) -> str:
    """Test infrastructure: the CPU oracle (oracle/fs_oracle.cpp,
    oracle/fs_philox.c) and, when the reference's sources are given, the
    reference itself (oracle/_ref).  ref_src is the reference's code/
    directory; without it the environment variable FLYSIM_REF_SRC is used,
    and with neither the reference is not built."""
    odir = os.path.join(ROOT, "oracle", "_build")
    os.makedirs(odir, exist_ok=True)
    src = os.path.join(ROOT, "oracle", "fs_oracle.cpp")
    csrc = os.path.join(ROOT, "oracle", "fs_philox.c")
    cobj = os.path.join(odir, "fs_philox.o")
    lib = os.path.join(odir, "liboracle.so")
    if _newer(cobj, [csrc]):
        _run(["gcc", "-std=c11", "-O2", "-fPIC", "-ffp-contract=off", "-c", csrc, "-o", cobj], verbose)
    if _newer(lib, [src, cobj, os.path.join(INC, "flysim_b200.h")]):
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I", INC, src, cobj, "-o", lib, "-lm"], verbose)
    ref_src = ref_src or os.environ.get("FLYSIM_REF_SRC")
    if ref_src and os.path.isdir(ref_src):
        _run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "Makefile.ref"), "-j8", "REF=" + ref_src,
              "OUT=" + os.path.join(ROOT, "oracle", "_ref")], verbose)
    return lib


if __name__ == "__main__":
    print(build(verbose=True))
    print(build_oracle(verbose=True, ref_src=sys.argv[1] if len(sys.argv) > 1 else None))
