"""Build the in-tree CUDA library ``libnrldpc_b200.so`` for sm_100a.

The library is compiled straight with nvcc (no torch extension machinery):
every source under ``csrc/`` is compiled for ``arch=compute_100a,code=sm_100a``
and linked with the static CUDA runtime into one shared object that exposes
the plain C ABI declared in ``include/nrldpc_b200.h``.

    python -m deeplearning_5g_ldpc_decoder_b200.build [--force] [--verbose]
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
INCLUDE = os.path.join(REPO_DIR, "include")
LIB_NAME = "libnrldpc_b200.so"
LIB_PATH = os.path.join(PKG_DIR, LIB_NAME)
# Debug build: the same sources with device-side index checks on every gather
# and scatter of the decode kernels (-DNRLDPC_BOUNDS_CHECK); never on the product path.
DEBUG_LIB_PATH = os.path.join(PKG_DIR, "libnrldpc_b200_debug.so")

SOURCES = [
    "nrldpc_api.cu",
    "nrldpc_channel.cu",
    "nrldpc_encode.cu",
    "nrldpc_fixed.cu",
    "nrldpc_float.cu",
    "nrldpc_mixed.cu",
    "nrldpc_mixed_api.cu",
    "nrldpc_noalloc.cu",
    "nrldpc_tb.cu",
    "nrldpc_train.cu",
    "nrldpc_tables.cpp",
]
HEADERS = [
    "nrldpc_internal.h",
    "nrldpc_decode_common.cuh",
    "nrldpc_fixed_row.cuh",
    "nrldpc_bounds.cuh",
    "nrldpc_tb.cuh",
    "nr_base_graphs.inc",
]

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libnrldpc_b200.so")
    return cand


def _inputs():
    files = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    files.append(os.path.join(INCLUDE, "nrldpc_b200.h"))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date(path: str = LIB_PATH) -> bool:
    if not os.path.exists(path):
        return False
    t = os.path.getmtime(path)
    return all(os.path.getmtime(f) <= t for f in _inputs())


def build_library(force: bool = False, verbose: bool = False, extra_flags=None, debug: bool = False) -> str:
    """Compile the library (or, with debug, the bounds-checked debug library) if
    any input is newer than it; return its path."""
    out = DEBUG_LIB_PATH if debug else LIB_PATH
    if not force and up_to_date(out):
        return out
    cmd = [
        nvcc_path(),
        *ARCH_FLAGS,
        "-lineinfo",
        "-O3",
        "-std=c++17",
        "-Xcompiler", "-fPIC,-O3,-Wall",
        "-shared",
        "-cudart", "static",
        "-I", INCLUDE,
        "-I", CSRC,
    ]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    if extra_flags:
        cmd += list(extra_flags)
    if debug:
        cmd += ["-DNRLDPC_BOUNDS_CHECK"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    tmp = out + ".tmp"
    cmd += ["-o", tmp, "-lpthread", "-ldl", "-lrt"]
    proc = subprocess.run(cmd, cwd=PKG_DIR, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout)
        sys.stderr.write(proc.stderr)
        raise RuntimeError(f"nvcc failed with exit code {proc.returncode}")
    if verbose:
        sys.stderr.write(proc.stderr)
    os.replace(tmp, out)
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--debug", action="store_true", help="the bounds-checked debug library")
    args = ap.parse_args()
    print(build_library(force=args.force, verbose=args.verbose, debug=args.debug))


if __name__ == "__main__":
    main()
