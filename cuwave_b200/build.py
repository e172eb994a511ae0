"""Build libcuwave_b200.so in-tree for sm_100a with nvcc.

Each (precision, dimension, radius) of the stencil kernels is its own translation unit
(csrc/unit.cu compiled with -D flags), so the 32 units build in parallel; objects land
in cuwave_b200/_build/ and are rebuilt only when a source or the flags change.

    python -m cuwave_b200.build [-j JOBS]
"""

from __future__ import annotations

import argparse
import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
CSRC = PACKAGE / "csrc"
BUILD = PACKAGE / "_build"
INCLUDE = PACKAGE.parent / "include"
LIBRARY = PACKAGE / "libcuwave_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: no product is fused into a sum unless the source asks for it, the
# rounding the reference's host build (g++ -ffp-contract=off) keeps
NVFLAGS = [
    "-std=c++17",
    "-O3",
    "--fmad=false",
    "-lineinfo",
    "-diag-suppress",
    "177",
    "-Xcompiler",
    "-fPIC,-ffp-contract=off",
    f"-I{INCLUDE}",
    f"-I{CSRC}",
]
PRECISIONS = {"f32": "float", "f64": "double"}
RADII = range(1, 9)
DIMS = (2, 3)


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build")
    return path


def _sources_digest() -> str:
    digest = hashlib.sha256()
    for path in sorted(CSRC.glob("*")) + [INCLUDE / "cuwave_b200.h"]:
        digest.update(path.name.encode())
        digest.update(path.read_bytes())
    digest.update(" ".join(ARCH + NVFLAGS).encode())
    return digest.hexdigest()[:16]


def _jobs() -> list[tuple[Path, list[str]]]:
    jobs = []
    for tag, real in PRECISIONS.items():
        for ndim in DIMS:
            for radius in RADII:
                obj = BUILD / f"unit_{tag}_{ndim}d_r{radius}.o"
                defines = [f"-DCWB_REAL={real}", f"-DCWB_NDIM={ndim}", f"-DCWB_RADIUS={radius}"]
                jobs.append((obj, [str(CSRC / "unit.cu"), *defines]))
    jobs.append((BUILD / "transfer.o", [str(CSRC / "transfer.cu")]))
    jobs.append((BUILD / "conv.o", [str(CSRC / "conv.cu")]))
    jobs.append((BUILD / "api.o", [str(CSRC / "api.cu")]))
    return jobs


def build(jobs: int | None = None, verbose: bool = False) -> Path:
    """Compile every unit that is out of date and link the library; returns its path."""
    BUILD.mkdir(exist_ok=True)
    digest = _sources_digest()
    stamp = BUILD / "digest"
    stale = not stamp.exists() or stamp.read_text() != digest
    compiler = nvcc()
    todo = [(obj, args) for obj, args in _jobs() if stale or not obj.exists()]

    def compile_one(item):
        obj, args = item
        cmd = [compiler, *ARCH, *NVFLAGS, "-c", *args, "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        done = subprocess.run(cmd, capture_output=True, text=True)
        if done.returncode:
            raise RuntimeError(f"{' '.join(cmd)} failed:\n{done.stderr}")
        return obj

    if todo:
        workers = jobs or max(1, os.cpu_count() or 1)
        with ThreadPoolExecutor(max_workers=workers) as pool:
            list(pool.map(compile_one, todo))
    objects = [str(obj) for obj, _ in _jobs()]
    if todo or not LIBRARY.exists():
        tmp = LIBRARY.with_suffix(".so.tmp")
        cmd = [compiler, *ARCH, "-shared", "-Xcompiler", "-fPIC", *objects, "-o", str(tmp)]
        done = subprocess.run(cmd, capture_output=True, text=True)
        if done.returncode:
            raise RuntimeError(f"link failed:\n{done.stderr}")
        os.replace(tmp, LIBRARY)
    stamp.write_text(digest)
    return LIBRARY


def main(argv=None) -> int:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("-j", "--jobs", type=int, default=None)
    parser.add_argument("-v", "--verbose", action="store_true")
    args = parser.parse_args(argv)
    print(build(args.jobs, args.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
