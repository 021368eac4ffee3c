"""Build of the sm_100a shared library (libblgpu.so) from csrc/*.cu.

nvcc cross-compiles for sm_100a without a GPU.  stencil64.cu and
dynsgs.cu are compiled with -fmad=false so that the FP64 stencil kernels evaluate each expression with the
rounding of the Fortran source; the transform kernels keep fused multiply-adds.
The library is written in-tree (lib/libblgpu.so) so that it ships with the
source tree to the GPU host.
"""
import os
import subprocess
import concurrent.futures as cf

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(PKG_ROOT, "csrc")
LIB_DIR = os.path.join(PKG_ROOT, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libblgpu.so")
OBJ_DIR = os.path.join(PKG_ROOT, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + ARCH
SOURCES = {
    "stencil64.cu": ["-fmad=false"],
    "dynsgs.cu": ["-fmad=false"],
    "stencil32.cu": [],
    "spectral.cu": [],
    "capi.cu": [],
    "noalloc.cu": [],
    "mlp.cu": [],
    "capi_mlp.cu": [],
    "zdft_tc.cu": [],
    "zdft_umma.cu": [],
    "snapshot.cpp": [],
    "thomas_tma.cu": [],
    "cufft_path.cu": [],
}


def _newest_input():
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    paths.append(os.path.join(PKG_ROOT, "..", "include", "blgpu.h"))
    paths.append(os.path.abspath(__file__))
    return max(os.path.getmtime(p) for p in paths if os.path.exists(p))


def needs_build():
    return (not os.path.exists(LIB_PATH)) or os.path.getmtime(LIB_PATH) < _newest_input()


def build(force=False, verbose=False):
    """Compile every .cu in csrc for sm_100a and link lib/libblgpu.so."""
    if not force and not needs_build():
        return LIB_PATH
    os.makedirs(OBJ_DIR, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)

    def compile_one(name):
        src = os.path.join(CSRC, name)
        obj = os.path.join(OBJ_DIR, os.path.splitext(name)[0] + ".o")
        cmd = [NVCC] + COMMON + SOURCES[name] + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (name, " ".join(cmd), r.stderr))
        if verbose and r.stderr:
            print(r.stderr)
        return obj

    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, sorted(SOURCES)))
    tmp = LIB_PATH + ".tmp"
    cmd = [NVCC, "-shared"] + ARCH + ["-o", tmp] + objs + ["-lcufft"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build(force=True, verbose=True))
