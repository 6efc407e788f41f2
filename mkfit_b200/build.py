"""Builds the CUDA extension library in-tree for sm_100a.

    python -m mkfit_b200.build            # -> mkfit_b200/_lib/libmkfit_b200.so

The library is a plain shared object with a C ABI (include/mkfit_b200.h);
Python loads it with ctypes. Incremental: objects are rebuilt when their
source or any header in csrc/ is newer.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIB = os.path.join(OUT_DIR, "libmkfit_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills"]


def _newer(dst, srcs):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(s) > t for s in srcs)


def build(verbose=False, extra_flags=(), out_dir=None):
    """Compiles csrc/ into OUT_DIR (or out_dir, for variant builds)."""
    lib = LIB if out_dir is None else os.path.join(out_dir, "libmkfit_b200.so")
    obj_dir = OBJ_DIR if out_dir is None else os.path.join(out_dir, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    gen = os.path.join(CSRC, "generated_ops.cuh")
    if _newer(gen, [os.path.join(CSRC, "gen_ops.py")]):
        subprocess.check_call([sys.executable, os.path.join(CSRC, "gen_ops.py")])
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(HERE, "..", "include", "*.h"))
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cc"))):
        obj = os.path.join(obj_dir, os.path.basename(src)[:-3] + "_host.o")
        objs.append(obj)
        if _newer(obj, [src] + headers):
            cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-fPIC", "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(obj_dir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if _newer(obj, [src] + headers):
            cmd = [NVCC] + ARCH + FLAGS + list(extra_flags) + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    if _newer(lib, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart"]
        subprocess.check_call(cmd)
    return lib


EXT_SRC = os.path.join(CSRC, "torch_ext", "align_ext.cc")
EXT_NAME = "_align_ext"


def ext_path(out_dir=None):
    import sysconfig
    return os.path.join(out_dir or OUT_DIR, EXT_NAME + sysconfig.get_config_var("EXT_SUFFIX"))


def build_torch_ext(verbose=False, out_dir=None):
    """Compiles the PyTorch binding of the differentiable fit (an autograd
    Function in C++ over the C ABI) next to the library."""
    import sysconfig
    import torch
    lib = build(verbose=verbose, out_dir=out_dir)
    out = ext_path(out_dir)
    header = os.path.join(HERE, "..", "include", "mkfit_b200.h")
    if not _newer(out, [EXT_SRC, header]):
        return out
    tdir = os.path.dirname(torch.__file__)
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    cmd = [os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-fPIC", "-shared", "-Wno-interference-size",
           "-DTORCH_EXTENSION_NAME=" + EXT_NAME, "-DTORCH_API_INCLUDE_EXTENSION_H",
           "-D_GLIBCXX_USE_CXX11_ABI=%d" % abi,
           "-I" + os.path.join(tdir, "include"),
           "-I" + os.path.join(tdir, "include", "torch", "csrc", "api", "include"),
           "-I/usr/local/cuda/include", "-I" + sysconfig.get_paths()["include"],
           EXT_SRC, "-o", out,
           "-L" + os.path.join(tdir, "lib"), "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu",
           "-ltorch_python", "-L" + os.path.dirname(lib), "-lmkfit_b200",
           "-Wl,-rpath," + os.path.join(tdir, "lib"), "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return out


if __name__ == "__main__":
    print(build(verbose=True))
    print(build_torch_ext(verbose=True))
