"""Compile tests/dropin/cdi_program.cpp against the drop-in headers
(include/nadia) and libnadia_b200.so, as a caller of the reference's C++
classes would: float build by default, DOUBLE_PRECISION for the double build."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
SRC = os.path.join(ROOT, "tests", "dropin", "cdi_program.cpp")
LIBDIR = os.path.join(ROOT, "nadia-coecxs_b200")


def build(out, double=False):
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror",
           "-I", os.path.join(ROOT, "include", "nadia"), "-I", os.path.join(ROOT, "include"),
           SRC, "-L", LIBDIR, "-lnadia_b200", "-Wl,-rpath," + LIBDIR, "-o", out]
    if double:
        cmd.insert(1, "-DDOUBLE_PRECISION")
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out
