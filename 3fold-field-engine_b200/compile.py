"""Build recipe of the CUDA library ``libfield_b200.so`` (sm_100a only), in-tree.

    python -c "import field_b200.compile as c; c.build()"

nvcc cross-compiles without a GPU.  The shared library is written next to this file so that it
travels with the source tree; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUTPUT = HERE / "libfield_b200.so"
INCLUDE = HERE.parent / "include"

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-Xcompiler", "-fPIC", "-shared", "--threads", "0", "-Xptxas", "-v",
]


def sources():
    return sorted(str(p) for p in CSRC.glob("*.cu"))


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile every CUDA source into libfield_b200.so; returns its path."""
    srcs = sources()
    deps = srcs + [str(p) for p in CSRC.glob("*.cuh")] + [str(p) for p in INCLUDE.glob("*.h")]
    if not force and OUTPUT.exists():
        newest = max(os.path.getmtime(p) for p in deps)
        if os.path.getmtime(OUTPUT) >= newest:
            return OUTPUT
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *NVCC_FLAGS, "-I", str(INCLUDE), *srcs, "-o", str(OUTPUT) + ".tmp"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + proc.stdout[-4000:] + proc.stderr[-8000:])
    os.replace(str(OUTPUT) + ".tmp", OUTPUT)
    if verbose:
        print(proc.stderr)
    (HERE / "ptxas_report.txt").write_text(proc.stderr)
    return OUTPUT
