"""Builds the library's native code in-tree.

``build_library()`` compiles ``csrc/*.cu`` for sm_100a into
``fmm2d_c_translation_b200/libfmm2d_b200.so`` (one nvcc invocation, static
CUDA runtime, only libcuda needed at run time).  ``build_oracle()`` runs
``make -C oracle``: the checkers used by the tests and by bench.py's CPU
baseline (the reference's own C translation is rebuilt only where its
sources exist).
"""
import glob
import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
LIB_PATH = os.path.join(PKG_DIR, "libfmm2d_b200.so")

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "--extended-lambda",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-fvisibility=hidden,-O3",
    "-Xptxas", "-warn-spills",
    "-shared",
]


def _nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build")
    return cand


def build_library(verbose=False, extra_flags=()):
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    cmd = [_nvcc()] + NVCC_FLAGS + list(extra_flags) + ["-o", LIB_PATH] + srcs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=CSRC)
    return LIB_PATH


def build_oracle(verbose=False):
    odir = os.path.join(REPO_DIR, "oracle")
    targets = ["_ref/liboracle.so"]
    ref = os.environ.get("FMM2D_REFERENCE", "/root/reference")
    if os.path.isdir(os.path.join(ref, "c_translation", "src")):
        targets.append("ref")
    cmd = ["make", "-C", odir, "REF=" + ref] + targets
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build_library(verbose=True, extra_flags=sys.argv[1:])
    build_oracle(verbose=True)
