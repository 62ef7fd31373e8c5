"""Build the engine library in-tree: mpdpft_b200/libmpdpft_b200.so (sm_100a).

Usage: python -m mpdpft_b200.build [--debug]
The library is plain C ABI (include/mpdpft_gpu.h); it links only the CUDA
runtime.  nvcc cross-compiles for sm_100a without a GPU.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libmpdpft_b200.so")
SOURCES = ["engine.cu", "fft.cu", "capi.cu", "noalloc.cu", "batch.cu", "adjoint.cu", "refio.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def host_compiler():
    # /usr/bin/g++ is the system compiler CUDA 12.9 supports
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def flags(debug=False):
    f = ARCH + ["-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", host_compiler(),
                "-I", os.path.join(ROOT, "include")]
    f += ["-O0", "-G"] if debug else ["-O3"]
    if os.environ.get("MPDPFT_PTXAS_VERBOSE"):
        f += ["-Xptxas", "-v"]
    return f


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, x) for x in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "mpdpft_gpu.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(debug=False, force=False, verbose=False):
    if not force and not stale():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    cc = nvcc()
    fl = flags(debug)

    def compile_one(src):
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        cmd = [cc] + fl + ["-c", os.path.join(CSRC, src), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, r.stdout, r.stderr))
        if verbose and (r.stderr or r.stdout):
            print(r.stdout + r.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    tmp = LIB + ".tmp"
    cmd = [cc] + ARCH + ["-shared", "-ccbin", host_compiler(), "-o", tmp] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(debug="--debug" in sys.argv, force=True, verbose="-v" in sys.argv)
    print(LIB)
