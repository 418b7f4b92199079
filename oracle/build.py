"""Build recipe of the CPU oracle (TEST INFRASTRUCTURE; see oracle.cpp).

    python oracle/build.py        -> oracle/_build/liboracle.so, oracle/_build/quichotte_oracle,
                                     oracle/_build/sancho_oracle

The oracle links LAPACK/BLAS from the OpenBLAS inside the numpy wheel (ILP64 symbols
scipy_*_64_), the only LAPACK in this image. It also links the host layer of the product
(libqs_host.so: input.dat reader, model builders, output files), which must be built first.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_build")
HOSTLIB = os.path.join(ROOT, "quichotte-and-sancho_b200", "_build")


def openblas_lib():
    import numpy
    libs = glob.glob(os.path.join(os.path.dirname(numpy.__file__) + ".libs", "libscipy_openblas64_*.so"))
    if not libs:
        raise RuntimeError("numpy's bundled OpenBLAS (libscipy_openblas64_*.so) not found")
    return libs[0]


def run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("oracle build failed")


def build(verbose=False):
    os.makedirs(OUT, exist_ok=True)
    ob = openblas_lib()
    obdir, obname = os.path.dirname(ob), os.path.basename(ob)
    lib = os.path.join(OUT, "liboracle.so")
    run(["g++", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=c++17",
         os.path.join(HERE, "oracle.cpp"), "-o", lib,
         "-L" + obdir, "-l:" + obname, "-Wl,-rpath," + obdir])
    for name, main in (("quichotte_oracle", "oracle_main.cpp"), ("sancho_oracle", "sancho_oracle_main.cpp")):
        exe = os.path.join(OUT, name)
        run(["g++", "-O2", "-std=c++17", os.path.join(HERE, main), "-o", exe,
             "-I" + os.path.join(ROOT, "include"),
             "-L" + OUT, "-loracle", "-L" + HOSTLIB, "-lqs_host", "-fopenmp",
             "-Wl,-rpath," + OUT, "-Wl,-rpath," + HOSTLIB, "-Wl,-rpath," + obdir])
    exe = os.path.join(OUT, "quichotte_oracle")
    if verbose:
        print("built", lib, exe)
    return lib, exe


if __name__ == "__main__":
    build(verbose=True)
