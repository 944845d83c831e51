"""Build the engine in-tree with nvcc for sm_100a.

Outputs (git-ignored, they travel with the repository snapshot):
  matrix-permanent-calculator_b200/libperman_b200.so   C ABI (include/perman_b200.h)
  matrix-permanent-calculator_b200/bin/perman          drop-in command line

Usage: python matrix-permanent-calculator_b200/build.py [--force] [-j N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libperman_b200.so"
CLI = PKG / "bin" / "perman"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
              "--expt-relaxed-constexpr", f"-I{INCLUDE}"]
HOST_CXX = os.environ.get("PERM_HOST_CXX", "/usr/bin/g++")

LIB_SOURCES = [
    "engine.cu", "ryser_skipper.cu", "mc.cu", "mc_sparse.cu", "batch.cu", "serve.cu", "noalloc.cu", "multi_device.cpp",
    "ryser_dense_inst_0.cu", "ryser_dense_inst_1.cu", "ryser_dense_inst_2.cu",
    "ryser_dense_inst_3.cu", "ryser_dense_inst_4.cu", "ryser_dense_2l_inst_0.cu", "ryser_dense_2l_inst_1.cu", "ryser_dense_int_g3.cu", "ryser_dense_int_g4.cu",
    "ryser_dense_int_g5.cu", "ryser_dense_int_g6.cu", "ryser_dense_int_sparse_g4.cu", "ryser_dense_int_sparse_g5.cu",
    "ryser_dense_int_sparse_g6.cu", "ryser_dense_int_3l_g4.cu", "ryser_dense_int_3l_g5.cu", "ryser_dense_int_3l_g6.cu", "ryser_dense_intc_sparse_g4p.cu", "ryser_dense_intc_sparse_g5.cu",
    "ryser_dense_intc_sparse_g6p.cu", "ryser_dense_intc_3l_g4p.cu", "ryser_dense_intc_3l_g5.cu",
    "ryser_dense_intc_3l_g6p.cu", "ryser_dense_dd_inst.cu", "matrix_io.cpp",
    "ryser_dense_tc_g3.cu", "ryser_dense_tc_g4.cu", "ryser_dense_tc_g5.cu", "ryser_dense_tc_g6.cu",
    "ryser_dense_split_inst.cu", "ryser_dense_intc_g3.cu", "ryser_dense_intc_g4.cu", "ryser_dense_intc_g5.cu",
    "ryser_dense_intc_g6.cu", "ryser_dense_intc_p4.cu", "ryser_dense_intc_p5.cu", "ryser_dense_intc_p6.cu",
    "ryser_dense_sdd_inst.cu", "ryser_sparse_sdd_r6.cu", "ryser_sparse_sdd_r8.cu",
    "ryser_sparse_sdd_r12.cu", "ryser_sparse_sdd_r16.cu", "ryser_sparse_sdd_r20.cu", "ryser_sparse_sdd_r24.cu",
    "ryser_sparse_sdd_r28.cu", "ryser_sdd_3l_r16.cu", "ryser_sdd_3l_r20.cu", "ryser_sdd_3l_r24.cu",
    "ryser_sdd_3l_r28.cu", "ryser_dense_3l_r20.cu", "ryser_dense_3l_r24.cu", "ryser_dense_3l_r28.cu",
    "ryser_dense_3l_r32.cu", "ryser_dense_3l_r36.cu",
]
CLI_SOURCES = ["perman_cli.cpp"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(path).exists():
        raise RuntimeError("nvcc not found (CUDA 12.9 toolkit required)")
    return path


def _deps(src: Path) -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "perman_b200.h", src]


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def _compile(src: Path, force: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if not force and not _stale(obj, _deps(src)):
        return obj
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, f"-ccbin={HOST_CXX}", "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cpp":
        cmd = [nvcc(), "-x", "cu", *cmd[1:]]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stderr[-4000:]}")
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    (PKG / "bin").mkdir(exist_ok=True)
    srcs = [CSRC / s for s in LIB_SOURCES if (CSRC / s).exists()]
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, f"-ccbin={HOST_CXX}", "-shared", "-o", str(LIB), *map(str, objs)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr[-4000:]}")
        if verbose:
            print(f"linked {LIB}")
    cli_srcs = [CSRC / s for s in CLI_SOURCES if (CSRC / s).exists()]
    if cli_srcs and (force or _stale(CLI, [LIB, *cli_srcs])):
        cmd = [HOST_CXX, "-O2", "-std=c++17", f"-I{INCLUDE}", *map(str, cli_srcs), "-o", str(CLI),
               f"-L{PKG}", "-lperman_b200", "-Wl,-rpath,$ORIGIN/.."]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"CLI build failed:\n{res.stderr[-4000:]}")
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    args = ap.parse_args()
    build(force=args.force, jobs=args.j, verbose=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
