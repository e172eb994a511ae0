"""Build the reference's own scalar kernels for the host, into oracle/_ref/.

CPU ORACLE -- baseline infrastructure, not the product. Compiles ref_driver.cpp, which
includes the reference's cuwave/kernels/cpu.hpp, common.cuh and scalar.cu where they lie
in the reference tree, with the preamble the reference's Python would generate
(STENCIL_RADIUS and the OP_COEFFS table of cuwave/stencils.py:186-213; the staggered
table only the elastic kernels read is left zero). g++ -O3 -fopenmp -ffp-contract=off,
as the reference's own host build (cuwave/cpu.py) compiles them, without -march=native
so the library runs on any x86-64 host.

    python oracle/ref_build.py [--reference PATH]

Outputs oracle/_ref/libref3d_r4_optimized_f32.so (3D, radius 4, the bench workload),
which bench.py's reference arm and cpu_baseline load. The reference tree is read at
build time only.
"""

from __future__ import annotations

import argparse
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"


def library_name(ndim: int, radius: int, stencil: str, precision: str) -> Path:
    tag = "f32" if precision == "float32" else "f64"
    return OUT / f"libref{ndim}d_r{radius}_{stencil}_{tag}.so"


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


def build(reference: str = "/root/reference", ndim: int = 3, radius: int = 4,
          stencil: str = "optimized", precision: str = "float32") -> Path:
    kernels = Path(reference) / "cuwave" / "kernels"
    if not (kernels / "scalar.cu").exists():
        raise FileNotFoundError(f"the reference kernels are not at {kernels}")
    OUT.mkdir(exist_ok=True)
    lib = library_name(ndim, radius, stencil, precision)
    head = OUT / f"preamble_r{radius}_{stencil}.h"
    head.write_text(preamble(radius, stencil))
    cxx = os.environ.get("REF_CXX", "/usr/bin/g++")
    cmd = [
        cxx, "-O3", "-fopenmp", "-ffp-contract=off", "-std=c++17", "-shared", "-fPIC", "-w",
        f"-DNDIM={ndim}", "-DDIRICHLET_FACES=0", f'-DREF_PREAMBLE="{head}"',
        f"-I{kernels}", str(HERE / "ref_driver.cpp"), "-o", str(lib),
    ]
    if precision == "float32":
        cmd.insert(-3, "-DUSE_FLOAT")
    done = subprocess.run(cmd, capture_output=True, text=True)
    if done.returncode:
        raise RuntimeError(f"{' '.join(cmd)} failed:\n{done.stderr}")
    return lib


def main(argv=None) -> int:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--reference", default="/root/reference")
    args = parser.parse_args(argv)
    print(build(args.reference))
    return 0


if __name__ == "__main__":
    sys.exit(main())
