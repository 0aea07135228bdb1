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


IO_SHIM = os.path.join(ROOT, "tests", "dropin", "io_shim.cpp")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def build_io_shim(out, reference=False):
    """io_shim.cpp as a shared library: over the drop-in io.h / Config.h
    (double build), or -- reference=True -- over the reference's own headers
    and oracle/_ref/libnadia_ref_io.a.  Returns None when the reference
    variant is asked for and oracle/_ref was not built."""
    if reference:
        lib = os.path.join(REF_DIR, "libnadia_ref_io.a")
        if not os.path.exists(lib):
            return None
        cmd = ["g++", "-std=c++17", "-O2", "-w", "-shared", "-fPIC", "-DDOUBLE_PRECISION",
               "-I", os.path.join(ROOT, "oracle", "shim"), "-I", os.path.join(REF_DIR, "include"),
               IO_SHIM, "-Wl,--whole-archive", lib, "-Wl,--no-whole-archive", "-o", out]
    else:
        cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-shared", "-fPIC",
               "-DDOUBLE_PRECISION", "-I", os.path.join(ROOT, "include", "nadia"),
               "-I", os.path.join(ROOT, "include"), IO_SHIM, "-L", LIBDIR, "-lnadia_b200",
               "-Wl,-rpath," + LIBDIR, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stdout + r.stderr)
    return out
