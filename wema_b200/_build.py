"""In-tree build of the native libraries (no JIT cache: the built .so files
live in ``wema_b200/lib`` and travel with the repository snapshot).

* ``libwema_cuda.so`` - the C-ABI library (CUDA kernels for sm_100a plus the
  host runtime), compiled by nvcc straight from ``csrc/``.
* ``libwema_synth.so`` - the seeded synthetic video generator (gcc).
* ``wema-cuda-cli`` - the reference CLI's command line over raw RGB24 frames,
  linked against libwema_cuda (gcc).
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_DIR = os.path.join(PKG, "lib")
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def cuda_lib_path() -> str:
    return os.path.join(LIB_DIR, "libwema_cuda.so")


def synth_lib_path() -> str:
    return os.path.join(LIB_DIR, "libwema_synth.so")


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_synth(force: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    out = synth_lib_path()
    src = [os.path.join(PKG, "synth", "synth.c"), os.path.join(PKG, "synth", "synth.h")]
    if force or _stale(out, src):
        subprocess.run(["gcc", "-std=c11", "-O2", "-fPIC", "-shared", "-fopenmp",
                        "-ffp-contract=off", src[0], "-o", out, "-lm"], check=True)
    return out


def build_cuda(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIB_DIR, exist_ok=True)
    out = cuda_lib_path()
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cpp = sorted(glob.glob(os.path.join(CSRC, "*.cpp")))
    deps = cu + cpp + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) \
        + glob.glob(os.path.join(INCLUDE, "*.h"))
    if not (force or _stale(out, deps)):
        return out
    objdir = os.path.join(ROOT, "_build", "wema_cuda")
    os.makedirs(objdir, exist_ok=True)
    nvcc = _nvcc()
    common = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "-Xcompiler", "-ffp-contract=off", "-I", INCLUDE, "-I", CSRC, "-lineinfo"]
    objs = []
    for src in cu + cpp:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [src] + deps):
            continue
        cmd = [nvcc, *NVCC_ARCH, *common, "-c", src, "-o", obj]
        if src.endswith(".cu"):
            cmd += ["--expt-relaxed-constexpr", "-Xptxas", "-O3"]
            if verbose:
                cmd += ["-Xptxas", "-v"]
        subprocess.run(cmd, check=True)
    subprocess.run([nvcc, *NVCC_ARCH, "-shared", *objs, "-o", out, "-lcudart", "-lpthread"],
                   check=True)
    return out


def cli_path() -> str:
    return os.path.join(LIB_DIR, "wema-cuda-cli")


def build_cli(force: bool = False) -> str:
    lib = build_cuda()
    out = cli_path()
    src = os.path.join(PKG, "cli", "wema_cuda_cli.c")
    if force or _stale(out, [src, lib, os.path.join(INCLUDE, "wema_cuda.h")]):
        subprocess.run(["gcc", "-std=c11", "-O2", "-Wall", "-Wextra", "-I", INCLUDE, src, "-o", out,
                        "-L", LIB_DIR, "-lwema_cuda", "-Wl,-rpath,$ORIGIN"], check=True)
    return out


def build_all(force: bool = False) -> None:
    build_synth(force)
    build_cuda(force)
    build_cli(force)
