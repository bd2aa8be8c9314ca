"""Builds the sm_100a shared library of the DEM step in-tree.

    python -m pacific_b200.build          # -> pacific_b200/lib/libgrains_gpu.so

Both kernel units are compiled with -fmad=false.  In the plain-FP64 kernels
every double expression then rounds like the reference's x86-64 build.  The
mixed-precision kernels run the same double narrowphase for every contact
(GJK witness points on flat faces hinge on the last bit of near-equal support
values), so they must round it the same way as the FP64 kernels.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libgrains_gpu.so")
EXAMPLE = os.path.join(LIBDIR, "grains_host_example")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "nvcc")

UNITS = [
    ("kernels_fp64.cu", ["-fmad=false"]),
    ("kernels_mixed.cu", ["-fmad=false"]),
    ("adjoint_fp64.cu", ["-fmad=false"]),
    ("adjoint_mixed.cu", ["-fmad=false"]),
    ("adjoint_api.cu", []),
    ("api.cu", []),
    ("noalloc.cu", []),
    ("io.cu", ["-fmad=false"]),
]
HEADERS = ["common.cuh", "sphere_contact.cuh", "contact_law.cuh", "gjk.cuh", "kernels.cuh", "device_state.h",
           "dual.cuh", "adjoint.cuh", "adjoint.h", "format.cuh", "io.h"]


def _newer(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(verbose=False, force=False):
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS]
    hdrs.append(os.path.join(HERE, "..", "include", "grains_gpu.h"))
    hdrs.append(os.path.abspath(__file__))  # compiler flags live here
    objs = []
    procs = []
    for src, extra in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            cmd = [NVCC, "-std=c++17", "-O3", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v" if verbose else "-O3",
                   *extra, "-c", s, "-o", o]
            procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if verbose and out:
            print(out)
        if p.returncode != 0:
            raise RuntimeError("nvcc failed: %s\n%s" % (" ".join(cmd), out))
    if force or _newer(LIB, objs):
        cmd = [NVCC, "-shared", *ARCH, "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: %s\n%s" % (" ".join(cmd), r.stdout))
    # C++ caller of the adaptor in include/grains_gpu.hpp
    src = os.path.join(CSRC, "host_example.cpp")
    hpp = os.path.join(HERE, "..", "include", "grains_gpu.hpp")
    if force or _newer(EXAMPLE, [src, hpp, LIB]):
        cmd = ["g++", "-O2", "-std=c++17", src, "-o", EXAMPLE, "-L" + LIBDIR, "-lgrains_gpu",
               "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError("example build failed: %s\n%s" % (" ".join(cmd), r.stdout))
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
