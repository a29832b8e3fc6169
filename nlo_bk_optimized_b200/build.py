"""Build ``libnlo_b200.so`` (sm_100a) in-tree with nvcc.

The library is plain C-ABI (include/nlo_b200.h); it links only the CUDA runtime.
``python -m nlo_bk_optimized_b200.build`` rebuilds it; ``build()`` is what
``__graft_entry__.build()`` calls.  nvcc cross-compiles without a GPU.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
LIBDIR = PACKAGE / "lib"
LIBRARY = LIBDIR / "libnlo_b200.so"
HEADERS = [ROOT / "include" / "nlo_b200.h"]

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _nvcc() -> str:
    candidate = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(candidate).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libnlo_b200.so")
    return candidate


def _stale() -> bool:
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    inputs = sources() + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + HEADERS + [Path(__file__)]
    return any(path.stat().st_mtime > built for path in inputs)


# Per-file flags.  The DIS kernels' FP32 bodies use approximate single-precision
# division and square root (about 2 ulp) and flush FP32 denormals; their FP64 template
# instances and every other file keep IEEE arithmetic.
FILE_FLAGS = {name: ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"] for name in ("dis.cu", "dis_fixed.cu")}
# The tabulated initial condition reproduces the reference's FP64 spline coefficients bit
# for bit: no fused multiply-adds there.
FILE_FLAGS["ic.cu"] = ["-fmad=false"]


def _compile(source: Path, obj: Path, verbose: bool) -> tuple[int, str]:
    command = [
        _nvcc(),
        *ARCH_FLAGS,
        "-O3",
        "-lineinfo",
        "-std=c++17",
        "-Xcompiler",
        "-fPIC",
        "--expt-relaxed-constexpr",
        *FILE_FLAGS.get(source.name, []),
        "-c",
        str(source),
        "-o",
        str(obj),
    ]
    if verbose or os.environ.get("NLO_PTXAS_VERBOSE"):
        command.insert(1, "-Xptxas=-v")
    result = subprocess.run(command, capture_output=True, text=True)
    return result.returncode, result.stdout + result.stderr


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile every csrc/*.cu for sm_100a (in parallel, one nvcc per file) and link
    libnlo_b200.so."""
    if not force and not _stale():
        return LIBRARY
    LIBDIR.mkdir(parents=True, exist_ok=True)
    objdir = PACKAGE / "_build"
    objdir.mkdir(parents=True, exist_ok=True)
    srcs = sources()
    objs = [objdir / (src.stem + ".o") for src in srcs]
    workers = max(1, min(len(srcs), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as pool:
        results = list(pool.map(lambda pair: _compile(pair[0], pair[1], verbose), zip(srcs, objs)))
    failed = [(src, out) for src, (code, out) in zip(srcs, results) if code != 0]
    if verbose:
        for src, (_, out) in zip(srcs, results):
            sys.stderr.write(f"== {src.name}\n{out}")
    if failed:
        for src, out in failed:
            sys.stderr.write(f"== {src.name}\n{out}")
        raise RuntimeError("nvcc failed to build libnlo_b200.so")
    tmp = LIBRARY.with_suffix(".so.tmp")
    link = [_nvcc(), *ARCH_FLAGS, "-shared", "-o", str(tmp), *[str(o) for o in objs], "-lcudart"]
    result = subprocess.run(link, capture_output=True, text=True)
    if result.returncode != 0:
        sys.stderr.write(result.stdout + result.stderr)
        raise RuntimeError("nvcc failed to link libnlo_b200.so")
    tmp.replace(LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build(force=True, verbose="-v" in sys.argv))
