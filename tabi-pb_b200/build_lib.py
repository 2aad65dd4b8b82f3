"""Builds libtabi_gpu.so (sm_100a) in-tree with nvcc.

    python tabi-pb_b200/build_lib.py [--force] [-j N]

Each .cu under csrc/ is compiled to an object (in parallel), then linked into
tabi-pb_b200/_build/libtabi_gpu.so.  csrc/taylor_gen.cuh is regenerated from
csrc/gen_taylor.py when the generator is newer.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "_build")
LIB = os.path.join(OUT, "libtabi_gpu.so")
SOURCES = ["tree.cu", "matvec.cu", "precond.cu", "gmres.cu", "rhs_energy.cu", "tabi_api.cu",
           "warmstart.cu", "potential.cu", "noalloc.cu"]
HEADERS = ["tabi_impl.cuh", "taylor_gen.cuh", "bie_kernels.cuh", "reduce.cuh", "warmstart.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def gen_header(force=False):
    gen = os.path.join(CSRC, "gen_taylor.py")
    hdr = os.path.join(CSRC, "taylor_gen.cuh")
    if force or _mtime(hdr) < _mtime(gen):
        subprocess.run([sys.executable, gen, "8"], check=True)


def compile_one(src, force, extra):
    obj = os.path.join(OUT, os.path.splitext(src)[0] + ".o")
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(PKG, "..", "include", "tabi_gpu.h")]
    if not force and _mtime(obj) >= max(_mtime(d) for d in deps):
        return obj, None
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
           "--expt-relaxed-constexpr", "-c", os.path.join(CSRC, src), "-o", obj, *extra]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, jobs: int = 6, verbose_ptxas: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    gen_header(force)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        res = list(ex.map(lambda s: compile_one(s, force, extra), SOURCES))
    objs = [o for o, _ in res]
    if verbose_ptxas:
        for o, log in res:
            if log:
                print(log)
    if force or not os.path.exists(LIB) or _mtime(LIB) < max(_mtime(o) for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        subprocess.run(cmd, check=True)
    build_driver(force)
    return LIB


def build_driver(force: bool = False) -> str:
    """tabipb (host driver mirroring main.f90) and tabi_msms next to the library."""
    src = os.path.join(PKG, "host", "tabipb_main.cpp")
    exe = os.path.join(OUT, "tabipb")
    hdr = os.path.join(PKG, "..", "include", "tabi_gpu.h")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    if force or _mtime(exe) < max(_mtime(src), _mtime(hdr), _mtime(LIB)):
        subprocess.run([cxx, "-O2", "-std=c++17", "-o", exe, src, "-L" + OUT, "-ltabi_gpu",
                        "-Wl,-rpath,$ORIGIN"], check=True)
    sg = os.path.join(PKG, "surfgen")
    msms = os.path.join(OUT, "tabi_msms")
    srcs = [os.path.join(sg, f) for f in ("tabi_msms.c", "surfgen.c", "surfgen.h")]
    if force or _mtime(msms) < max(map(_mtime, srcs)):
        cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
        subprocess.run([cc, "-O2", "-o", msms, srcs[0], srcs[1], "-lm"], check=True)
    return exe


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=6)
    ap.add_argument("--ptxas", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.j, a.ptxas))
