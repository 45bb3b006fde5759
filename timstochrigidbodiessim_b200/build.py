"""Build recipe of the B200 FCM library: every CUDA source in csrc/ is compiled
for sm_100a and linked, with cuFFT, into timstochrigidbodiessim_b200/libfcm_b200.so
(in-tree, so it ships with the repository snapshot), and a second time with
-DFCM_BOUNDS_CHECK (every device index checked, violations counted and skipped)
into libfcm_b200_debug.so.  Run ``python -m timstochrigidbodiessim_b200.build``.
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
DEBUG_LIB = os.path.join(PKG, "libfcm_b200_debug.so")
DEBUG_BUILD = os.path.join(BUILD, "bounds_check")
HOST_LIB = os.path.join(PKG, "libfcm_b200_host.so")
DRIVER = os.path.join(PKG, "rigid_bodies_sim")
HOST_DIR = os.path.join(CSRC, "host")
CXX = "/usr/bin/g++"

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = GENCODE + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                    "-ccbin", "/usr/bin/g++", "--expt-relaxed-constexpr",
                    "-I" + os.path.join(ROOT, "include")]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _compile(src, extra, out_dir=BUILD):
    obj = os.path.join(out_dir, os.path.basename(src) + ".o")
    if (os.path.exists(obj) and os.path.getmtime(obj) > os.path.getmtime(src)
            and all(os.path.getmtime(obj) > os.path.getmtime(h)
                    for h in glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(ROOT, "include", "fcm_b200.h")])):
        return obj, ""
    cmd = [NVCC] + CFLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return obj, r.stderr


def _build_lib(lib, out_dir, extra, verbose):
    os.makedirs(out_dir, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, extra, out_dir), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                sys.stderr.write(log)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(lib) or os.path.getmtime(lib) < newest:
        cmd = [NVCC] + GENCODE + ["-shared", "-o", lib] + objs + [
            "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcufft", "-lcudart",
            "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))


def build(verbose=False, ptxas_info=False, bounds_check=True):
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    _build_lib(LIB, BUILD, extra, verbose)
    if bounds_check:
        _build_lib(DEBUG_LIB, DEBUG_BUILD, extra + ["-DFCM_BOUNDS_CHECK"], verbose)
    _build_host()
    return LIB


def _build_host():
    """The reference-named C++ classes (libfcm_b200_host.so) and the driver."""
    hsrc = os.path.join(HOST_DIR, "fcm_host.cpp")
    hdr = os.path.join(HOST_DIR, "fcm_host.hpp")
    main = os.path.join(HOST_DIR, "rigid_bodies_main.cpp")
    flags = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-I" + os.path.join(ROOT, "include")]
    newest = max(os.path.getmtime(x) for x in (hsrc, hdr, LIB))
    if not os.path.exists(HOST_LIB) or os.path.getmtime(HOST_LIB) < newest:
        cmd = [CXX] + flags + ["-shared", "-o", HOST_LIB, hsrc, "-L" + PKG, "-lfcm_b200", "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("host library build failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    newest = max(newest, os.path.getmtime(main), os.path.getmtime(HOST_LIB))
    if not os.path.exists(DRIVER) or os.path.getmtime(DRIVER) < newest:
        cmd = [CXX] + flags + ["-o", DRIVER, main, "-L" + PKG, "-lfcm_b200_host", "-lfcm_b200", "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("driver build failed:\n%s\n%s" % (" ".join(cmd), r.stderr))


def clean():
    shutil.rmtree(BUILD, ignore_errors=True)
    for f in (LIB, DEBUG_LIB, HOST_LIB, DRIVER):
        if os.path.exists(f):
            os.remove(f)


if __name__ == "__main__":
    if "--clean" in sys.argv:
        clean()
    print(build(verbose=True, ptxas_info="--ptxas" in sys.argv, bounds_check="--no-bounds-check" not in sys.argv))
