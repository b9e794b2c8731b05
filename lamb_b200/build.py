"""Builds the package's native libraries in-tree.

* lamb_b200/liblamb_b200.so -- the CUDA library behind include/lamb_gpu.h,
  compiled for sm_100a only;
* lamb_b200/liblamb_gen.so  -- the synthetic water-box generator (include/lamb_gen.h).

Run as ``python -m lamb_b200.build``.  nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
INC = os.path.join(REPO, "include")
CSRC = os.path.join(PKG, "csrc")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "-Xptxas", "-warn-spills"]


def _nvcc() -> str:
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target: str, sources) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_gen(force: bool = False) -> str:
    out = os.path.join(PKG, "liblamb_gen.so")
    srcs = [os.path.join(CSRC, "water_gen.cpp"), os.path.join(INC, "lamb_gen.h")]
    if force or _stale(out, srcs):
        subprocess.check_call(["g++", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared", "-std=c++17",
                               "-I", INC, srcs[0], "-o", out], env=_host_env())
    return out


def build_cuda(force: bool = False, verbose: bool = False) -> str:
    out = os.path.join(PKG, "liblamb_b200.so")
    cus = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    deps = cus + glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(INC, "lamb_gpu.h")]
    if force or _stale(out, deps):
        objdir = os.path.join(PKG, "_build")
        os.makedirs(objdir, exist_ok=True)
        objs = []
        procs = []
        for cu in cus:
            obj = os.path.join(objdir, os.path.basename(cu) + ".o")
            objs.append(obj)
            cmd = [_nvcc()] + NVCC_FLAGS + ["-I", INC, "-I", CSRC, "-c", cu, "-o", obj]
            if verbose:
                cmd += ["-Xptxas", "-v"]
            procs.append((cu, subprocess.Popen(cmd, env=_host_env(), stdout=subprocess.PIPE,
                                               stderr=subprocess.STDOUT, text=True)))
        failed = False
        for cu, p in procs:
            txt, _ = p.communicate()
            if p.returncode != 0 or verbose:
                sys.stderr.write(f"--- {os.path.basename(cu)}\n{txt}")
            failed |= p.returncode != 0
        if failed:
            raise RuntimeError("nvcc failed")
        subprocess.check_call([_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler",
                               "-fPIC", "-o", out] + objs + ["-lcudart"],
                              env=_host_env())
    return out


def _host_env():
    env = dict(os.environ)
    # Use the system toolchain (its OpenMP runtime and specs) for host code.
    env["CC"] = "gcc"
    env["CXX"] = "g++"
    env["PATH"] = "/usr/bin:" + env.get("PATH", "")
    return env


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_gen(force)
    build_cuda(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print("built", os.path.join(PKG, "liblamb_b200.so"), os.path.join(PKG, "liblamb_gen.so"))
