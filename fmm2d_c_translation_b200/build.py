"""Builds the library's native code in-tree.

``build_library()`` compiles ``csrc/*.cu`` for sm_100a into
``fmm2d_c_translation_b200/libfmm2d_b200.so`` (one object per source,
compiled in parallel under ``_build/`` and only when the source or a header
changed; static CUDA runtime, only libcuda needed at run time).  ``build_oracle()`` runs
``make -C oracle``: the checkers used by the tests and by bench.py's CPU
baseline (the reference's own C translation is rebuilt only where its
sources exist).
"""
import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
LIB_PATH = os.path.join(PKG_DIR, "libfmm2d_b200.so")
OBJ_DIR = os.path.join(REPO_DIR, "_build")

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "--extended-lambda",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-fvisibility=hidden,-O3",
    "-Xptxas", "-warn-spills",
]


def _nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build")
    return cand


def build_library(verbose=False, extra_flags=()):
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = glob.glob(os.path.join(CSRC, "*.cuh"))
    newest_header = max((os.path.getmtime(h) for h in headers), default=0.0)
    os.makedirs(OBJ_DIR, exist_ok=True)
    nvcc = _nvcc()
    flags = NVCC_FLAGS + list(extra_flags)
    stamp = os.path.join(OBJ_DIR, "flags.txt")
    same_flags = os.path.exists(stamp) and open(stamp).read() == " ".join(flags)

    def compile_one(src):
        obj = os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + ".o")
        if (same_flags and os.path.exists(obj) and
                os.path.getmtime(obj) >= max(os.path.getmtime(src), newest_header)):
            return obj
        cmd = [nvcc] + flags + ["-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=CSRC)
        return obj

    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, srcs))
    with open(stamp, "w") as f:
        f.write(" ".join(flags))
    cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB_PATH] + objs
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
