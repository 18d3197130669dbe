"""Build recipe of the native libraries, in-tree, for sm_100a only.

* ``libnabladyn_b200.so``: every CUDA kernel and the C-ABI of ``include/nabladyn_b200.h``,
  compiled by nvcc for ``sm_100a`` with the CUDA runtime linked statically. No torch inside.
* ``_nabladyn_neighbors_ops.so``: the ``torch.library`` registration of the reference's
  ``nabladyn_neighbors`` schemas, a thin C++ layer over the C-ABI.

Both land in ``nabladyn_b200/_lib``. A file is rebuilt only when a source or header is newer.
Run as ``python -m nabladyn_b200.csrc.build``.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

CSRC = Path(__file__).resolve().parent
PACKAGE = CSRC.parent
ROOT = PACKAGE.parent
INCLUDE = ROOT / "include"
LIB = PACKAGE / "_lib"
OBJ = LIB / "obj"

CUDA_SOURCES = ("neighbors.cu", "lj.cu", "md.cu", "serve.cu", "schnet.cu", "schnet_tangent.cu",
                "schnet_atoms.cu",
                "integrate.cu")
CXX_SOURCES = ("abi.cpp",)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# IEEE arithmetic as in the reference build: no fast math, no flush-to-zero.
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--ftz=false", "-Xcompiler", "-fPIC"]

CORE = LIB / "libnabladyn_b200.so"
TORCH_OPS = LIB / "_nabladyn_neighbors_ops.so"


def _nvcc() -> str:
    home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    return str(Path(home) / "bin" / "nvcc")


def _headers() -> list[Path]:
    return [*CSRC.glob("*.cuh"), *INCLUDE.glob("*.h")]


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    built = target.stat().st_mtime
    return any(source.stat().st_mtime > built for source in sources)


def _run(command: list[str]) -> None:
    print(" ".join(command), flush=True)
    subprocess.run(command, check=True)


def build_core(verbose_ptxas: bool = False) -> Path:
    """Compile the CUDA sources and link libnabladyn_b200.so."""
    OBJ.mkdir(parents=True, exist_ok=True)
    objects = []
    for name in CUDA_SOURCES:
        source = CSRC / name
        obj = OBJ / (source.stem + ".o")
        if _stale(obj, [source, *_headers()]):
            flags = ["-Xptxas", "-v"] if verbose_ptxas else []
            _run([_nvcc(), *ARCH, *NVCC_FLAGS, *flags, f"-I{INCLUDE}", f"-I{CSRC}",
                  "-c", str(source), "-o", str(obj)])
        objects.append(obj)
    for name in CXX_SOURCES:
        source = CSRC / name
        obj = OBJ / (source.stem + ".o")
        if _stale(obj, [source, *_headers()]):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", f"-I{INCLUDE}", f"-I{CSRC}",
                  "-c", str(source), "-o", str(obj)])
        objects.append(obj)
    if _stale(CORE, objects):
        _run([_nvcc(), *ARCH, "-shared", "-o", str(CORE), *map(str, objects)])
    return CORE


def build_torch_ops() -> Path:
    """Compile the torch.library layer against the installed torch and link it to the core."""
    source = CSRC / "torch_ops.cpp"
    if not _stale(TORCH_OPS, [source, CORE, *INCLUDE.glob("*.h")]):
        return TORCH_OPS
    import torch
    from torch.utils import cpp_extension

    includes = [*cpp_extension.include_paths(device_type="cuda"), str(INCLUDE)]
    cuda_home = cpp_extension.CUDA_HOME or "/usr/local/cuda"
    torch_lib = Path(torch.__file__).resolve().parent / "lib"
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    command = [
        "g++", "-O2", "-std=c++17", "-fPIC", "-shared",
        f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
        *[f"-I{path}" for path in includes],
        f"-I{Path(cuda_home) / 'include'}",
        str(source),
        "-o", str(TORCH_OPS),
        f"-L{torch_lib}", "-lc10", "-lc10_cuda", "-ltorch_cpu", "-ltorch",
        f"-L{LIB}", "-lnabladyn_b200",
        f"-Wl,-rpath,{torch_lib}", "-Wl,-rpath,$ORIGIN",
    ]
    _run(command)
    return TORCH_OPS


def build(verbose_ptxas: bool = False) -> None:
    build_core(verbose_ptxas)
    build_torch_ops()


if __name__ == "__main__":
    build(verbose_ptxas="-v" in sys.argv)
