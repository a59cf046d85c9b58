"""Build recipe for the sm_100a CUDA library behind the C ABI.

``build()`` compiles every ``csrc/*.cu`` file with nvcc for sm_100a only (and
the host-only ``csrc/*.cpp`` files with nvcc's host compiler, ``-pthread``)
(``-gencode arch=compute_100a,code=sm_100a``) into
``flagsparse_public_b200/libflagsparse_b200.so``, in-tree, so the library
travels with the source tree.  It needs nvcc but no GPU.
"""

import concurrent.futures
import os
import shutil
import subprocess
import sys

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG_DIR, "csrc")
ROOT = os.path.dirname(PKG_DIR)
LIB_NAME = "libflagsparse_b200.so"
LIB_PATH = os.path.join(PKG_DIR, LIB_NAME)
OBJ_DIR = os.path.join(PKG_DIR, "_build")

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC,-O3,-pthread",
    "-DNDEBUG",
    "-I" + os.path.join(ROOT, "include"),
]


def _nvcc():
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build flagsparse_public_b200")
    return nvcc


def _sources():
    return sorted(
        os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp"))
    )


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "flagsparse_b200.h"))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose):
    obj = os.path.join(OBJ_DIR, os.path.splitext(os.path.basename(src))[0] + ".o")
    if not _stale(obj, [src] + _headers()):
        return obj
    cmd = [_nvcc()] + ARCH_FLAGS + NVCC_FLAGS + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        print(res.stderr, flush=True)
    return obj


def build(verbose=False, jobs=None):
    """Compile (incrementally) and link libflagsparse_b200.so; returns its path."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _stale(LIB_PATH, objs):
        cmd = [_nvcc()] + ARCH_FLAGS + ["-shared", "-o", LIB_PATH] + objs + ["-lpthread"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
