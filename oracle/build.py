"""Build recipes for the checker (TEST INFRASTRUCTURE ONLY).

* ``build_oracle()`` compiles ``oracle/lpc_oracle.c`` (the FP64 C restatement)
  into ``oracle/liblpc_oracle.so`` with gcc + OpenMP.
* ``build_reference_cuda()`` compiles the reference's CPU operator together
  with its CUDA kernels (``torchlpc/csrc/cuda/lpc.cu``,
  ``linear_recurrence.cu``, unmodified, nvcc for sm_100a) into
  ``oracle/_ref_cuda/`` with the reference's Python package: the same-GPU
  comparator of the benchmark (the reference's own CUDA path).
* ``build_reference()`` compiles the reference's own CPU operator
  (``torchlpc/csrc/scan_cpu.cpp`` of DiffAPF/torchlpc, read where it lies under
  /root/reference) with g++ against the installed torch, and lays out the
  reference's Python package next to it, all under ``oracle/_ref/`` (git-ignored;
  the built files travel with the working tree to a GPU host, the sources do not
  need to).  It does not run the reference's own build system.  Nothing here is
  imported by the product package ``torchlpc_b200``.

Run ``python -m oracle.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import sysconfig
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_SRC = Path("/root/reference")
REF_OUT = HERE / "_ref"
REF_CUDA_OUT = HERE / "_ref_cuda"
ORACLE_SO = HERE / "liblpc_oracle.so"


def _gcc() -> str:
    # /usr/bin/gcc ships libgomp; other gcc installs in this image may not.
    return "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc"


def _gxx() -> str:
    return "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"


def build_oracle(force: bool = False) -> Path:
    src = HERE / "lpc_oracle.c"
    if not force and ORACLE_SO.exists() and ORACLE_SO.stat().st_mtime >= src.stat().st_mtime:
        return ORACLE_SO
    cmd = [_gcc(), "-O2", "-fopenmp", "-shared", "-fPIC", "-o", str(ORACLE_SO), str(src)]
    subprocess.run(cmd, check=True)
    return ORACLE_SO


def build_reference(force: bool = False) -> Path | None:
    """Compile the reference CPU op and stage its Python package in oracle/_ref.

    Returns the package directory (``oracle/_ref``, to be put on sys.path), or
    None when the reference tree is not present (e.g. on a GPU host, which only
    uses the files built here).
    """
    pkg = REF_OUT / "torchlpc"
    so = pkg / "_C.so"
    if so.exists() and not force:
        return REF_OUT
    if not (REF_SRC / "torchlpc" / "csrc" / "scan_cpu.cpp").exists():
        return REF_OUT if so.exists() else None
    import torch
    from torch.utils import cpp_extension

    pkg.mkdir(parents=True, exist_ok=True)
    for py in (REF_SRC / "torchlpc").glob("*.py"):
        shutil.copyfile(py, pkg / py.name)
    inc = [f"-I{p}" for p in cpp_extension.include_paths()] + [
        f"-I{sysconfig.get_paths()['include']}"
    ]
    libdir = os.path.join(os.path.dirname(torch.__file__), "lib")
    cmd = [
        _gxx(), "-O3", "-fopenmp", "-shared", "-fPIC", "-std=c++17",
        "-D_GLIBCXX_USE_CXX11_ABI=" + str(int(torch._C._GLIBCXX_USE_CXX11_ABI)),
        *inc,
        str(REF_SRC / "torchlpc" / "csrc" / "scan_cpu.cpp"),
        f"-L{libdir}", "-lc10", "-ltorch", "-ltorch_cpu", "-ltorch_python",
        f"-Wl,-rpath,{libdir}", "-o", str(so),
    ]
    subprocess.run(cmd, check=True)
    return REF_OUT


def build_reference_cuda(force: bool = False) -> Path | None:
    """Compile the reference's CPU operator and CUDA kernels (sm_100a) into
    oracle/_ref_cuda with the reference's Python package beside them.

    Returns the directory to put on sys.path, or None when neither the
    sources nor a previous build are present.
    """
    pkg = REF_CUDA_OUT / "torchlpc"
    so = pkg / "_C.so"
    if so.exists() and not force:
        return REF_CUDA_OUT
    src = REF_SRC / "torchlpc" / "csrc"
    if not (src / "cuda" / "lpc.cu").exists():
        return REF_CUDA_OUT if so.exists() else None
    import torch
    from torch.utils import cpp_extension

    pkg.mkdir(parents=True, exist_ok=True)
    for py in (REF_SRC / "torchlpc").glob("*.py"):
        shutil.copyfile(py, pkg / py.name)
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    abi = "-D_GLIBCXX_USE_CXX11_ABI=" + str(int(torch._C._GLIBCXX_USE_CXX11_ABI))
    inc = [f"-I{p}" for p in cpp_extension.include_paths()] + [
        f"-I{sysconfig.get_paths()['include']}", f"-I{cuda_home}/include"]
    objs = []
    for cu in ("lpc.cu", "linear_recurrence.cu"):
        o = pkg / (cu + ".o")
        subprocess.run([f"{cuda_home}/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                        "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", abi, *inc, "-c", str(src / "cuda" / cu),
                        "-o", str(o)], check=True)
        objs.append(str(o))
    o = pkg / "scan_cpu.o"
    subprocess.run([_gxx(), "-O3", "-fopenmp", "-fPIC", "-std=c++17", abi, *inc, "-c", str(src / "scan_cpu.cpp"),
                    "-o", str(o)], check=True)
    objs.append(str(o))
    libdir = os.path.join(os.path.dirname(torch.__file__), "lib")
    subprocess.run([_gxx(), "-shared", "-fopenmp", *objs, f"-L{libdir}", "-lc10", "-lc10_cuda", "-ltorch",
                    "-ltorch_cpu", "-ltorch_cuda", "-ltorch_python", f"-L{cuda_home}/lib64", "-lcudart",
                    f"-Wl,-rpath,{libdir}", "-o", str(so)], check=True)
    for ob in objs:
        os.unlink(ob)
    return REF_CUDA_OUT


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_reference(force="--force" in sys.argv))
    print(build_reference_cuda(force="--force" in sys.argv))
