"""In-tree build of the native libraries (sm_100a only).

* ``liblpc_b200.so``: the CUDA kernels and the C ABI (include/lpc_b200.h),
  compiled by nvcc with ``-gencode arch=compute_100a,code=sm_100a`` and the CUDA
  runtime linked statically.  No torch dependency.
* ``_C.so``: the torch operator layer (namespace ``torchlpc_b200``) that
  validates tensors, allocates outputs/workspaces with the caching allocator,
  takes the current CUDA stream and calls the C ABI.

Both land next to this file so that they travel with the source tree.
Run ``python -m torchlpc_b200.build`` (``--force`` rebuilds everything).
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "liblpc_b200.so"
EXT = PKG / "_C.so"

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = str(Path(CUDA_HOME) / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                     "--expt-relaxed-constexpr", f"-I{INCLUDE}"]

CU_SOURCES = ["lpc_plain.cu", "lpc_chunked.cu", "lpc_ti.cu", "lpc_capi.cu", "lpc_noalloc.cu"]
HEADERS = ["lpc_common.cuh", "lpc_plain.cuh", "lpc_chunked.cuh", "lpc_ti.cuh"]


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r


def build_lib(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    hdrs = [CSRC / h for h in HEADERS] + [INCLUDE / "lpc_b200.h"]
    objs, jobs = [], []
    for src in CU_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            jobs.append([NVCC, *NVCC_FLAGS, *(["-Xptxas", "-v"] if verbose else []),
                         "-c", str(s), "-o", str(o)])
    if jobs:
        with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            for r in ex.map(_run, jobs):
                if verbose:
                    sys.stderr.write(r.stderr)
    if force or jobs or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)])
    return LIB


def build_ext(force: bool = False) -> Path:
    src = CSRC / "torch_ops.cpp"
    if not force and not _newer(EXT, [src, LIB, INCLUDE / "lpc_b200.h"]):
        return EXT
    import torch
    from torch.utils import cpp_extension

    inc = [f"-I{p}" for p in cpp_extension.include_paths()] + [
        f"-I{sysconfig.get_paths()['include']}", f"-I{CUDA_HOME}/include", f"-I{INCLUDE}"]
    tlib = os.path.join(os.path.dirname(torch.__file__), "lib")
    gxx = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
    _run([gxx, "-O2", "-shared", "-fPIC", "-std=c++17",
          f"-D_GLIBCXX_USE_CXX11_ABI={int(torch._C._GLIBCXX_USE_CXX11_ABI)}", *inc, str(src),
          f"-L{PKG}", "-llpc_b200", f"-L{tlib}", "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu",
          "-ltorch_cuda", "-ltorch_python", "-Wl,-rpath,$ORIGIN", f"-Wl,-rpath,{tlib}",
          "-o", str(EXT)])
    return EXT


def build(force: bool = False, verbose: bool = False) -> None:
    build_lib(force=force, verbose=verbose)
    build_ext(force=force)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
    print(EXT)
