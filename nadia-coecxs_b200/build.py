"""Build libnadia_b200.so in place (sm_100a).

Usage: python nadia-coecxs_b200/build.py [--force]

Every .cu file is compiled by nvcc for sm_100a only; plain64.cu additionally
with --fmad=false so the FP64 path performs no contracted multiply-adds.  The
shared library lands next to this file and is what the Python binding and the
C++ drop-in headers load.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnadia_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off",
                 "-I", os.path.join(ROOT, "include"), "-I", CSRC]
PER_FILE = {
    "plain64.cu": ["--fmad=false"],
    "phase_diverse.cu": ["--fmad=false"],
}


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs += [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
           if f.endswith(".h")]
    return hs


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s" % (" ".join(cmd), r.stdout))
    return r.stdout


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    hdr_time = max(os.path.getmtime(h) for h in headers())
    objs, jobs = [], []
    for src in sources():
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(path)
                and os.path.getmtime(obj) >= hdr_time):
            continue
        lang = [] if src.endswith(".cu") else ["-x", "cu"]
        jobs.append([NVCC, *COMMON, *PER_FILE.get(src, []), *lang, "-c", path, "-o", obj])
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        for out in pool.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB)
                                                for o in objs):
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs])
    return LIB


CLI_SRC = os.path.join(HERE, "cli", "CDI_reconstruction.cpp")
BIN = os.path.join(HERE, "bin")


def build_cli(force=False):
    """Compile the reconstruction tool twice (float and DOUBLE_PRECISION
    builds) against the drop-in headers and libnadia_b200.so; returns the
    paths of bin/CDI_reconstruction and bin/CDI_reconstruction_double."""
    lib = build(force)
    os.makedirs(BIN, exist_ok=True)
    deps = [CLI_SRC, lib] + [os.path.join(ROOT, "include", "nadia", f)
                             for f in os.listdir(os.path.join(ROOT, "include", "nadia"))]
    outs = []
    for name, flags in (("CDI_reconstruction", []), ("CDI_reconstruction_double", ["-DDOUBLE_PRECISION"])):
        out = os.path.join(BIN, name)
        outs.append(out)
        if not force and os.path.exists(out) and all(os.path.getmtime(d) <= os.path.getmtime(out)
                                                     for d in deps):
            continue
        _run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", *flags,
              "-I", os.path.join(ROOT, "include", "nadia"), "-I", os.path.join(ROOT, "include"),
              CLI_SRC, "-L", HERE, "-lnadia_b200", "-Wl,-rpath,$ORIGIN/..", "-o", out])
    return outs


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
    print(build_cli(force="--force" in sys.argv))
