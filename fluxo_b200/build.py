"""Builds the in-tree CUDA library ``fluxo_b200/libfluxo_gpu.so`` for sm_100a.

nvcc cross-compiles without a GPU, so this runs in any container with CUDA 12.9.
Each translation unit compiles in parallel; objects go to ``fluxo_b200/_build/``.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfluxo_gpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
                     "--expt-relaxed-constexpr", "-I" + CSRC]
CU_SOURCES = (["fluxo_gpu.cu", "launch_misc.cu", "lift_impl.cu", "noalloc.cu", "analyze.cu", "host_copy.cu"] +
              ["vol_vf%d.cu" % v for v in (0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 32)] +
              ["mhd_launch.cu", "mhd_vol_ec.cu", "mhd_vol_std.cu", "nfvse_launch.cu", "nfvse_ns.cu", "batch.cu",
               "gauss_launch.cu", "gauss_surf.cu", "gauss_mhd.cu"])
CPP_SOURCES = ["host_setup.cpp"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(HERE, "..", "include", "fluxo_gpu.h"))
    return hs


def build(verbose=False, jobs=None, extra_flags=(), build_dir=None, lib_path=None):
    """Compiles (incrementally) and links the library; extra_flags go to nvcc."""
    BUILD_ = build_dir or BUILD
    LIB_ = lib_path or LIB
    os.makedirs(BUILD_, exist_ok=True)
    nvcc = _nvcc()
    hdrs = _headers()
    cmds = []
    objs = []
    for src in CU_SOURCES + CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD_, src + ".o")
        objs.append(o)
        if not _stale(o, [s] + hdrs):
            continue
        if src.endswith(".cu"):
            cmd = [nvcc] + NVCC_FLAGS + list(extra_flags) + ["-c", s, "-o", o]
        else:
            cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-I" + CSRC, "-c", s, "-o", o]
        cmds.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for cmd, r in ex.map(run, cmds):
            if verbose:
                print(" ".join(cmd))
                print(r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError("compile failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    if cmds or not os.path.exists(LIB_):
        link = [nvcc] + ARCH + ["-shared", "-o", LIB_] + objs + ["-Xcompiler", "-fopenmp", "-lgomp", "-lcudart"]
        r = subprocess.run(link, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return LIB_


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
