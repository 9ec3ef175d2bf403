"""Builds libtffb200.so (sm_100a) from torchff-lib_b200/csrc with nvcc, in-tree.

    python torchff-lib_b200/torchff_b200/_build.py [-f] [-v]

Run as a script (not ``-m``): importing the package first would try to load the library.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)                       # torchff-lib_b200/
CSRC = os.path.join(ROOT, "csrc")
INCLUDE = os.path.join(os.path.dirname(ROOT), "include")
BUILD = os.path.join(ROOT, "_build")
LIB_NAME = "libtffb200.so"
SOURCES = ["tff_common.cu", "pairs.cu", "nblist.cu", "cpairs.cu", "bonded.cu", "pme.cu", "fused.cu", "batch.cu", "server.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -ftz=true: FP32 subnormals flush to zero (none arise on this path); FP64 is unaffected
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
              "-ftz=true", "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = os.path.join(cuda, "bin", "nvcc")
    return p if os.path.exists(p) else (shutil.which("nvcc") or "nvcc")


def lib_path() -> str:
    return os.path.join(PKG_DIR, LIB_NAME)


# libtorch binding for C++ hosts and the Python package alike, linked against libtffb200.so
# and libtorch, built with the host C++ compiler: the drop-in torch.ops.torchff.* operators
# (torch_ops.cpp) and the TorchScript class torch.classes.torchff_b200.System (torch_shim.cpp).
TORCH_LIB_NAME = "libtffb200_torch.so"
TORCH_SOURCES = ["torch_ops.cpp", "torch_shim.cpp"]


def torch_lib_path() -> str:
    return os.path.join(PKG_DIR, TORCH_LIB_NAME)


def build_torch_shim(force: bool = False) -> str:
    import torch.utils.cpp_extension as ce

    srcs = [os.path.join(CSRC, f) for f in TORCH_SOURCES]
    out = torch_lib_path()
    deps = [*srcs, os.path.join(INCLUDE, "tffb200.h"), lib_path()]
    if not force and os.path.exists(out) and not _needs_rebuild(out, deps):
        return out
    import torch

    cuda = os.path.dirname(os.path.dirname(nvcc()))
    tlib = ce.library_paths()[0]
    cmd = [shutil.which("g++") or "g++", "-O2", "-std=c++17", "-fPIC", "-shared",
           f"-D_GLIBCXX_USE_CXX11_ABI={int(torch._C._GLIBCXX_USE_CXX11_ABI)}",
           *[f"-I{p}" for p in ce.include_paths()], f"-I{os.path.join(cuda, 'include')}", f"-I{INCLUDE}",
           *srcs, "-o", out, f"-L{tlib}", "-ltorch", "-ltorch_cpu", "-lc10", "-lc10_cuda", f"-L{PKG_DIR}", "-ltffb200",
           "-Wl,-rpath,$ORIGIN", f"-Wl,-rpath,{tlib}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return out


def _needs_rebuild(obj: str, deps: list[str]) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "tffb200.h"))
    objs = []
    jobs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _needs_rebuild(o, [s] + headers):
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", s, "-o", o]
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr, file=sys.stderr)
        return r

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    out = lib_path()
    if jobs or not os.path.exists(out) or force:
        cuda = os.path.dirname(os.path.dirname(nvcc()))
        link = [nvcc(), *ARCH, "-shared", "-o", out, *objs, "-cudart", "static", "-lcufft",
                "-L", os.path.join(cuda, "lib64"), "-Xlinker", f"-rpath,{os.path.join(cuda, 'lib64')}"]
        run(link)
    build_torch_shim(force)
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
