"""Build recipe for the oracle -- TEST INFRASTRUCTURE, not part of the product.

Builds
  oracle/liboracle.so           the C restatement (nadia_oracle.c) + canonical FFT
and, when the reference sources are present ($NADIA_REFERENCE, else a
checkout named `reference` beside this repository), the reference's own
hot-path sources compiled unmodified
against the FFTW shim:
  oracle/_ref/libnadia_ref64.so       -DDOUBLE_PRECISION, -O2 -fno-fast-math  (parity)
  oracle/_ref/libnadia_ref64_fast.so  -DDOUBLE_PRECISION, -O3 -ffast-math     (timing)
  oracle/_ref/libnadia_ref32_fast.so  float build,        -O3 -ffast-math     (timing)
  oracle/_ref/libnadia_ref_io.a       io_*.c + Config.c++ (+ Complex_2D.c++), double build
  oracle/_ref/CDI_reconstruction_ref  NADIA/tools/CDI_reconstruction.c, double build
(libtiff, libhdf4 and LAPACK are not linked: ref_stubs.cpp stands in for them).
The reference flags are those of NADIA/configure.in:11 (-O3 -fPIC -ffast-math).

The reference headers are copied into oracle/_ref/include and three
assignment operators that fall off the end without `return *this;` are fixed
(NADIA/include/Complex_2D.h:117,151 and NADIA/include/Double_2D.h:348; without
the fix the optimised build crashes).  Only oracle/_ref/ is written; nothing
from the reference is committed.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")

REF_SOURCES = [
    "src/Complex_2D.c++",
    "src/BaseCDI.c++",
    "src/PlanarCDI.c++",
    "src/FresnelCDI.c++",
    "src/FresnelCDI_WF.c++",
    "src/PolyCDI.c++",
    "src/TransmissionConstraint.c++",
    "src/PhaseDiverseCDI.c++",
    "src/utils.c",
    "src/io_spec.c",
    "src/io_cplx.c",
    "src/io_dbin.c",
    "src/io_ppm.c",
]

# (file, 1-based line that closes an assignment operator without a return)
HEADER_FIXES = [
    ("Complex_2D.h", 117),
    ("Complex_2D.h", 151),
    ("Double_2D.h", 348),
]

PARITY_FLAGS = ["-O2", "-fno-fast-math", "-ffp-contract=off"]


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s" % (" ".join(cmd), r.stdout))
    return r.stdout


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build_oracle(force=False):
    """Compile oracle/liboracle.so (the C restatement)."""
    out = os.path.join(HERE, "liboracle.so")
    deps = [os.path.join(HERE, f) for f in ("nadia_oracle.c", "canon_fft.h")]
    if force or _stale(out, deps):
        _run(["gcc", "-shared", "-fPIC", *PARITY_FLAGS, "-Wall", "-Wno-maybe-uninitialized",
              "-o", out, os.path.join(HERE, "nadia_oracle.c"), "-lm"])
    return out


def reference_root():
    """The reference checkout: $NADIA_REFERENCE, else `reference` beside the
    repository; None when its sources are absent (the prebuilt oracle/_ref
    files are used as they are)."""
    root = os.environ.get("NADIA_REFERENCE") or os.path.join(
        os.path.dirname(os.path.dirname(HERE)), "reference")
    nadia = os.path.join(root, "NADIA")
    return nadia if os.path.isdir(os.path.join(nadia, "src")) else None


def _copy_headers(nadia):
    inc = os.path.join(REF_OUT, "include")
    os.makedirs(inc, exist_ok=True)
    src_inc = os.path.join(nadia, "include")
    for f in os.listdir(src_inc):
        if f.endswith(".h"):
            shutil.copyfile(os.path.join(src_inc, f), os.path.join(inc, f))
    for fname in sorted({f for f, _ in HEADER_FIXES}):
        p = os.path.join(inc, fname)
        lines = open(p).read().split("\n")
        for f, line in HEADER_FIXES:
            if f != fname:
                continue
            assert lines[line - 1].strip() == "};", (fname, line, lines[line - 1])
            lines[line - 1] = "    return *this;\n  };"
        open(p, "w").write("\n".join(lines))
    return inc


def build_reference(force=False):
    """Compile the reference's own sources into oracle/_ref (needs the sources)."""
    nadia = reference_root()
    if nadia is None:
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    inc = _copy_headers(nadia)
    variants = {
        "libnadia_ref64.so": ["-DDOUBLE_PRECISION", *PARITY_FLAGS],
        "libnadia_ref64_fast.so": ["-DDOUBLE_PRECISION", "-O3", "-ffast-math"],
        "libnadia_ref32_fast.so": ["-O3", "-ffast-math"],
        # the reference's MULTI_THREADED float build (Complex_2D.c++:465-467):
        # FFTs on NADIA_REF_FFT_THREADS threads, the rest of the loop serial
        "libnadia_ref32_fast_mt.so": ["-O3", "-ffast-math", "-DMULTI_THREADED",
                                      "-DNUM_THREADS=nadia_shim_env_threads()"],
    }
    srcs = [os.path.join(nadia, s) for s in REF_SOURCES]
    own = [os.path.join(HERE, f) for f in ("fftw_shim.c", "canon_fft.h", "ref_driver.cpp",
                                           "ref_stubs.cpp", "shim/fftw3.h")]
    outs = {}
    for name, flags in variants.items():
        out = os.path.join(REF_OUT, name)
        outs[name] = out
        if not (force or _stale(out, srcs + own)):
            continue
        objdir = os.path.join(REF_OUT, "obj_" + name.split(".")[0])
        os.makedirs(objdir, exist_ok=True)
        objs = []
        common = ["-fPIC", "-w", "-I", os.path.join(HERE, "shim"), "-I", inc, *flags]
        for s in srcs:
            o = os.path.join(objdir, os.path.basename(s).replace(".", "_") + ".o")
            _run(["g++", "-x", "c++", "-c", *common, s, "-o", o])
            objs.append(o)
        o = os.path.join(objdir, "ref_driver.o")
        _run(["g++", "-c", *common, os.path.join(HERE, "ref_driver.cpp"), "-o", o])
        objs.append(o)
        o = os.path.join(objdir, "ref_stubs.o")
        _run(["g++", "-c", *common, os.path.join(HERE, "ref_stubs.cpp"), "-o", o])
        objs.append(o)
        o = os.path.join(objdir, "fftw_shim.o")
        _run(["gcc", "-c", "-fPIC", "-w", *flags, os.path.join(HERE, "fftw_shim.c"), "-o", o])
        objs.append(o)
        _run(["g++", "-shared", "-o", out, *objs, "-lm", "-lpthread"])
    return outs


# the file helpers and configuration reader (test of include/nadia/io.h and
# Config.h) and the reconstruction tool (test of the CLI)
IO_SOURCES = [
    "src/Complex_2D.c++",
    "src/io_cplx.c",
    "src/io_dbin.c",
    "src/io_ppm.c",
    "src/io_spec.c",
    "src/Config.c++",
]
CLI_SOURCES = REF_SOURCES + [s for s in IO_SOURCES if s not in REF_SOURCES] + [
    "src/PartialCDI.c++",
    "src/PartialCharCDI.c++",
    "tools/CDI_reconstruction.c",
]


def _objects(nadia, inc, sources, objdir, flags, extra_own=()):
    os.makedirs(objdir, exist_ok=True)
    common = ["-fPIC", "-w", "-I", os.path.join(HERE, "shim"), "-I", inc, *flags]
    objs = []
    for s in sources:
        o = os.path.join(objdir, s.replace("/", "_").replace(".", "_") + ".o")
        _run(["g++", "-x", "c++", "-c", *common, os.path.join(nadia, s), "-o", o])
        objs.append(o)
    for f in extra_own:
        o = os.path.join(objdir, os.path.basename(f).replace(".", "_") + ".o")
        if f.endswith(".c"):
            _run(["gcc", "-c", "-fPIC", "-w", *flags, f, "-o", o])
        else:
            _run(["g++", "-c", *common, f, "-o", o])
        objs.append(o)
    return objs


def build_reference_tools(force=False):
    """oracle/_ref/libnadia_ref_io.a (the reference's io_*.c, Config.c++ and
    Complex_2D.c++, double build) and oracle/_ref/CDI_reconstruction_ref (the
    reference's tool, double build, parity flags).  Needs the sources."""
    nadia = reference_root()
    if nadia is None:
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    inc = _copy_headers(nadia)
    flags = ["-DDOUBLE_PRECISION", *PARITY_FLAGS]
    stubs = os.path.join(HERE, "ref_stubs.cpp")
    lib = os.path.join(REF_OUT, "libnadia_ref_io.a")
    cli = os.path.join(REF_OUT, "CDI_reconstruction_ref")
    own = [stubs, os.path.join(HERE, "fftw_shim.c")]
    if force or _stale(lib, [os.path.join(nadia, s) for s in IO_SOURCES] + own):
        objs = _objects(nadia, inc, IO_SOURCES, os.path.join(REF_OUT, "obj_io"), flags, own)
        if os.path.exists(lib):
            os.remove(lib)
        _run(["ar", "rcs", lib, *objs])
    if force or _stale(cli, [os.path.join(nadia, s) for s in CLI_SOURCES] + own):
        objs = _objects(nadia, inc, CLI_SOURCES, os.path.join(REF_OUT, "obj_cli"), flags, own)
        _run(["g++", "-o", cli, *objs, "-lm", "-lpthread"])
    return {"io": lib, "cli": cli, "include": inc}


def main():
    force = "--force" in sys.argv
    print(build_oracle(force))
    print(build_reference(force))
    print(build_reference_tools(force))


if __name__ == "__main__":
    main()
