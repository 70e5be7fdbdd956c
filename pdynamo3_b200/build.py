"""Build the in-tree CUDA library ``pdynamo3_b200/lib/libpdgpu.so`` for sm_100a.

Each ``csrc/*.cu`` is compiled separately (in parallel) with nvcc and linked with cuBLAS
and cuSOLVER.  Objects go to ``pdynamo3_b200/_build``; a file is recompiled when it or
any header in ``csrc`` or ``include`` is newer than its object.
"""
import concurrent.futures
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libpdgpu.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]


def _newest_header():
    files = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(CSRC, "*.inc")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(f) for f in files), default=0.0)


def _compile(src, verbose):
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), _newest_header()):
        return obj, None
    cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        return obj, "compile failed: %s\n%s%s" % (" ".join(cmd), p.stdout, p.stderr)
    return obj, (p.stderr if verbose else None)


def build(verbose=False, jobs=None):
    """Compile every CUDA source and link the shared library; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    objs = []
    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
        for obj, msg in ex.map(lambda s: _compile(s, verbose), srcs):
            if msg and msg.startswith("compile failed"):
                raise RuntimeError(msg)
            if msg:
                sys.stderr.write(msg)
            objs.append(obj)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcublas", "-lcusolver"]
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError("link failed: %s\n%s%s" % (" ".join(cmd), p.stdout, p.stderr))
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
