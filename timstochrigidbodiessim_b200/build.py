"""Build recipe of the B200 FCM library: every CUDA source in csrc/ is compiled
for sm_100a and linked, with cuFFT, into timstochrigidbodiessim_b200/libfcm_b200.so
(in-tree, so it ships with the repository snapshot).  Run
``python -m timstochrigidbodiessim_b200.build``.
"""
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "libfcm_b200.so")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = GENCODE + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                    "-ccbin", "/usr/bin/g++", "--expt-relaxed-constexpr",
                    "-I" + os.path.join(ROOT, "include")]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _compile(src, extra):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if (os.path.exists(obj) and os.path.getmtime(obj) > os.path.getmtime(src)
            and all(os.path.getmtime(obj) > os.path.getmtime(h)
                    for h in glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(ROOT, "include", "fcm_b200.h")])):
        return obj, ""
    cmd = [NVCC] + CFLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return obj, r.stderr


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, extra), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                sys.stderr.write(log)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [NVCC] + GENCODE + ["-shared", "-o", LIB] + objs + [
            "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcufft", "-lcudart",
            "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return LIB


def clean():
    shutil.rmtree(BUILD, ignore_errors=True)
    if os.path.exists(LIB):
        os.remove(LIB)


if __name__ == "__main__":
    if "--clean" in sys.argv:
        clean()
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv))
