"""Recipe that builds the reference's own CUDA sources (sajidanis/GV) with the
test harness oracle/ref_harness.cu into oracle/_ref/gv_ref_harness.

The reference is compiled where it lies (read-only); nothing is copied into
this repository and the output stays in oracle/_ref/ (git-ignored, shipped to
the GPU box with the working tree).  The file list is the reference's own
build list (CMakeLists.txt:20-37) minus src/main.cu, whose role the harness
takes.  Needs nvcc only; the reference's CMake build is not used.

    python -m oracle.ref_build [/path/to/reference]

The reference's location comes from the argument, else from the
GV_REFERENCE_DIR environment variable, else DEFAULT_REFERENCE_DIR (where the
build container mounts it); when none holds the sources nothing is built.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_DIR = HERE / "_ref"
BIN = OUT_DIR / "gv_ref_harness"
SOURCES = [
    "src/reader/marketReader.cu", "src/util/profiler.cu", "src/dynamicStructure/graphvine.cu",
    "src/dynamicStructure/csr.cu", "src/util/util.cu", "src/dynamicStructure/kernels/init_kernels.cu",
    "src/dynamicStructure/kernels/insert_kernels.cu", "src/dynamicStructure/kernels/delete_kernels.cu",
    "src/dynamicStructure/kernels/util_kernels.cu", "src/util/device_functions.cu",
    "src/algorithm/pagerank/pagerank.cu", "src/algorithm/pagerank/pr_kernel.cu", "src/algorithm/tc/tc.cu",
    "src/algorithm/tc/tc_kernel.cu", "src/util/gpu.cu", "src/algorithm/bc/bc_kernel.cu", "src/algorithm/bc/bc.cu",
]
INCLUDES = ["include", "include/algorithm/pagerank", "include/algorithm/tc", "include/algorithm/bc",
            "include/dynamicStructure", "include/dynamicStructure/kernels", "include/reader", "include/util", "src"]


DEFAULT_REFERENCE_DIR = "/root/reference"


def reference_dir() -> Path:
    """The reference checkout: GV_REFERENCE_DIR, else DEFAULT_REFERENCE_DIR."""
    return Path(os.environ.get("GV_REFERENCE_DIR") or DEFAULT_REFERENCE_DIR)


def build(ref: Path | None = None, force: bool = False) -> Path | None:
    ref = Path(ref) if ref is not None else reference_dir()
    if not (ref / "src").exists():
        return None
    harness = HERE / "ref_harness.cu"
    if BIN.exists() and not force and BIN.stat().st_mtime >= harness.stat().st_mtime:
        return BIN
    OUT_DIR.mkdir(exist_ok=True)
    objs = []
    procs = []
    flags = ["-gencode", "arch=compute_100a,code=sm_100a", "-rdc=true", "-O2", "-std=c++17",
             *[f"-I{ref / i}" for i in INCLUDES]]
    for src in [*(ref / s for s in SOURCES), harness]:
        obj = OUT_DIR / (src.stem + ".o")
        objs.append(obj)
        procs.append((src, subprocess.Popen(["nvcc", *flags, "-c", str(src), "-o", str(obj)],
                                            stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    ok = True
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode:
            ok = False
            print(f"--- {src}\n{out}", file=sys.stderr)
    if not ok:
        raise RuntimeError("reference build failed")
    subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-rdc=true", *map(str, objs),
                    "-o", str(BIN)], check=True)
    for o in objs:
        o.unlink()
    return BIN


if __name__ == "__main__":
    print(build(Path(sys.argv[1]) if len(sys.argv) > 1 else None, force=True))
