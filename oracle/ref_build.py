"""Build the reference's own scalar kernels for the host, into oracle/_ref/.

CPU ORACLE -- baseline infrastructure, not the product. Compiles ref_driver.cpp, which
includes the reference's cuwave/kernels/cpu.hpp, common.cuh and scalar.cu where they lie
in the reference tree, with the preamble the reference's Python would generate
(STENCIL_RADIUS and the OP_COEFFS table of cuwave/stencils.py:186-213; the staggered
table only the elastic kernels read is left zero).

Flags: the reference's own host build (cuwave/cpu.py:22, applied at cpu.py:175-178) is
`-O3 -march=native -fopenmp -ffp-contract=off`. The library is built here and run on
another host, so `-march=native` of this machine is not that host's; instead each
configuration is built for three instruction-set levels -- x86-64-v4 (AVX-512, what
`-march=native` gives on an AVX-512 Xeon or EPYC), x86-64-v3 (AVX2) and baseline x86-64 --
and `library()` picks the highest level the running host's CPU flags allow.
`-ffp-contract=off` keeps every level bit-identical to the others.

    python oracle/ref_build.py [--reference PATH]

Outputs oracle/_ref/libref{2,3}d_r4_optimized_{f32,f64}.{v4,v3,v1}.so: the 3D job of the
bench and the 2D forward of the parity tests, in float32 and float64. The reference tree
is read at build time only (REFERENCE_TREE overrides its location).
"""

from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
DEFAULT_TREE = os.environ.get("REFERENCE_TREE", "/root/reference")

# instruction-set levels, highest first: (tag, -march value or None, CPU flags it needs)
LEVELS = (
    ("v4", "x86-64-v4", ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl")),
    ("v3", "x86-64-v3", ("avx2", "fma", "bmi2")),
    ("v1", None, ()),
)
CONFIGS = ((3, 4, "optimized", "float32"), (3, 4, "optimized", "float64"),
           (2, 4, "optimized", "float32"), (2, 4, "optimized", "float64"))


def library_name(ndim: int, radius: int, stencil: str, precision: str, level: str) -> Path:
    tag = "f32" if precision == "float32" else "f64"
    return OUT / f"libref{ndim}d_r{radius}_{stencil}_{tag}.{level}.so"


def host_flags() -> set[str]:
    try:
        text = Path("/proc/cpuinfo").read_text()
    except OSError:
        return set()
    for line in text.splitlines():
        if line.startswith("flags"):
            return set(line.split(":", 1)[1].split())
    return set()


def library(ndim: int, radius: int, stencil: str, precision: str) -> tuple[Path, str]:
    """(path, level) of the built library for this host: the highest instruction-set
    level its CPU supports and that was built. The path of the baseline level when none
    is built."""
    flags = host_flags()
    for tag, _, need in LEVELS:
        path = library_name(ndim, radius, stencil, precision, tag)
        if all(f in flags for f in need) and path.exists():
            return path, tag
    return library_name(ndim, radius, stencil, precision, "v1"), "v1"


def preamble(radius: int, stencil: str) -> str:
    import importlib.util

    spec = importlib.util.spec_from_file_location("_oracle_tables", HERE / "oracle.py")
    module = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = module
    spec.loader.exec_module(module)
    cell_coefficients = module.cell_coefficients

    rows = []
    for r in range(1, radius + 1):
        row = cell_coefficients(r, stencil if r == radius else "taylor")
        rows.append("{" + ", ".join(repr(float(v)) for v in list(row) + [0.0] * (radius - r)) + "}")
    zero = "{" + ", ".join("{" + ", ".join(["0.0"] * radius) + "}" for _ in range(radius)) + "}"
    return (
        f"#define STENCIL_RADIUS {radius}\n"
        f"#define OP_COEFFS {{ {', '.join(rows)} }}\n"
        f"#define STAG_COEFFS {zero}\n"
    )


def _compile(kernels: Path, head: Path, ndim: int, precision: str, march: str | None,
             lib: Path) -> Path:
    cxx = os.environ.get("REF_CXX", "/usr/bin/g++")
    cmd = [cxx, "-O3", "-fopenmp", "-ffp-contract=off", "-std=c++17", "-shared", "-fPIC", "-w"]
    if march:
        cmd.append(f"-march={march}")
    cmd += [f"-DNDIM={ndim}", "-DDIRICHLET_FACES=0", f'-DREF_PREAMBLE="{head}"']
    if precision == "float32":
        cmd.append("-DUSE_FLOAT")
    tmp = lib.with_suffix(".tmp.so")
    cmd += [f"-I{kernels}", str(HERE / "ref_driver.cpp"), "-o", str(tmp)]
    done = subprocess.run(cmd, capture_output=True, text=True)
    if done.returncode:
        raise RuntimeError(f"{' '.join(cmd)} failed:\n{done.stderr}")
    os.replace(tmp, lib)
    return lib


def build(reference: str = DEFAULT_TREE) -> list[Path]:
    """Every configuration at every level, skipping libraries newer than their inputs."""
    kernels = Path(reference) / "cuwave" / "kernels"
    if not (kernels / "scalar.cu").exists():
        raise FileNotFoundError(f"the reference kernels are not at {kernels}")
    OUT.mkdir(exist_ok=True)
    inputs = [HERE / "ref_driver.cpp", Path(__file__).resolve(),
              *(kernels / n for n in ("scalar.cu", "common.cuh", "cpu.hpp"))]
    newest = max(p.stat().st_mtime for p in inputs)
    jobs = []
    for ndim, radius, stencil, precision in CONFIGS:
        head = OUT / f"preamble_r{radius}_{stencil}.h"
        text = preamble(radius, stencil)
        if not head.exists() or head.read_text() != text:
            head.write_text(text)
        for tag, march, _ in LEVELS:
            lib = library_name(ndim, radius, stencil, precision, tag)
            if lib.exists() and lib.stat().st_mtime >= max(newest, head.stat().st_mtime):
                continue
            jobs.append((kernels, head, ndim, precision, march, lib))
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        list(pool.map(lambda j: _compile(*j), jobs))
    return [library_name(*c, tag) for c in CONFIGS for tag, _, _ in LEVELS]


def main(argv=None) -> int:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--reference", default=DEFAULT_TREE)
    args = parser.parse_args(argv)
    for path in build(args.reference):
        print(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
