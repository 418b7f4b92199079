"""Copy the reference's regression cases into tests/golden/cases (run once, in the
container that has the reference checked out; the copies are committed so the GPU
tests can use them where the reference is absent).

    python tests/golden/make_fixtures.py /path/to/reference

Copied: tests/cases.txt and every tests/cases/<case>/ (inputs such as input.dat,
DFTB+ matrices, xyz and U files, and the golden outputs under reference/), and the same of
SANCHO's suite (SANCHO/tests) into tests/golden/sancho/. These files
are the reference's golden vectors for the NEGF path: outputs of its Fortran FP64 build,
compared field by field at |new - ref| <= 1e-6 + 1e-5 |ref| (tests/run_tests.f90:14).
"""
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def copy_suite(src, dst_root):
    dst = os.path.join(dst_root, "cases")
    if os.path.isdir(dst):
        shutil.rmtree(dst)
    os.makedirs(dst_root, exist_ok=True)
    shutil.copytree(os.path.join(src, "cases"), dst)
    shutil.copy(os.path.join(src, "cases.txt"), os.path.join(dst_root, "cases.txt"))
    n = sum(len(f) for _, _, f in os.walk(dst))
    print(f"copied {n} files into {dst}")


def main(ref):
    copy_suite(os.path.join(ref, "tests"), HERE)                                   # QUICHOTTE
    copy_suite(os.path.join(ref, "SANCHO", "tests"), os.path.join(HERE, "sancho"))  # SANCHO


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py /path/to/reference")
    main(sys.argv[1])
