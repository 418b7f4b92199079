"""Build of the B200 NEGF solver and its host layer (in-tree, sm_100a only).

    python quichotte-and-sancho_b200/build.py

produces, under quichotte-and-sancho_b200/_build/:
    libqs_host.so    host layer: input.dat reader, model builders, output files, program flow
    libqsb200.so     the CUDA library (include/qsb200.h), compiled for sm_100a
    quichotte_b200   the QUICHOTTE program over libqsb200.so (drop-in for bin/quichotte.x)
    sancho_b200      the SANCHO program over libqsb200.so (drop-in for SANCHO's bin/sancho.x)
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_build")
INC = os.path.join(ROOT, "include")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def run(cmd, verbose=False):
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("build failed: " + os.path.basename(cmd[-1]))
    return r.stdout + r.stderr


def newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def build_host(verbose=False):
    os.makedirs(OUT, exist_ok=True)
    srcs = [os.path.join(HERE, "host", f) for f in ("qs_host.cpp", "qs_main.cpp", "sancho_host.cpp")]
    lib = os.path.join(OUT, "libqs_host.so")
    hdrs = [os.path.join(HERE, "host", "host_common.hpp")] + [os.path.join(INC, h) for h in
                                                               ("qs_host.h", "qsb200.h", "qsa200.h", "qsa_host.h")]
    if not newer(lib, srcs + hdrs):
        run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-I" + INC] + srcs + ["-o", lib], verbose)
    return lib


def build_cuda(verbose=False, ptxas_verbose=False):
    os.makedirs(OUT, exist_ok=True)
    cu = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
    hdr = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + [os.path.join(INC, "qsb200.h"),
                                                                      os.path.join(INC, "qsa200.h")]
    lib = os.path.join(OUT, "libqsb200.so")
    if newer(lib, cu + hdr):
        return lib
    objs = []
    log = ""
    for src in cu:
        obj = os.path.join(OUT, os.path.basename(src)[:-3] + ".o")
        cmd = [NVCC] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INC,
                               "-I" + os.path.join(HERE, "csrc"), "--expt-relaxed-constexpr", "-c", src, "-o", obj]
        if ptxas_verbose:
            cmd.insert(1, "-Xptxas=-v")
        if not newer(obj, [src] + hdr):
            log += run(cmd, verbose)
        objs.append(obj)
    run([NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart"], verbose)
    if ptxas_verbose:
        print(log)
    return lib


def build_program(verbose=False):
    for name, main in (("quichotte_b200", "qs_gpu_main.cpp"), ("sancho_b200", "sancho_gpu_main.cpp")):
        exe = os.path.join(OUT, name)
        src = os.path.join(HERE, "host", main)
        deps = [src, os.path.join(OUT, "libqs_host.so"), os.path.join(OUT, "libqsb200.so")]
        if not newer(exe, deps):
            run(["g++", "-O2", "-std=c++17", "-I" + INC, src, "-o", exe, "-L" + OUT, "-lqsb200", "-lqs_host",
                 "-Wl,-rpath," + OUT], verbose)
    return os.path.join(OUT, "quichotte_b200")


def build(verbose=False):
    build_host(verbose)
    build_cuda(verbose)
    build_program(verbose)


if __name__ == "__main__":
    if "--host-only" in sys.argv:
        build_host(True)
    else:
        build_host(True)
        build_cuda(True, ptxas_verbose="--ptxas" in sys.argv)
        build_program(True)
