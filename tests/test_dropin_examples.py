"""Callers of the reference compile unchanged against the drop-in headers.

* The reference's own example programs (NADIA/examples: PlanarCDI,
  FresnelCDI, FresnelCDI_WF, PolyCDI, ComplexConstraints and the Planar and
  Poly simulations), unmodified, compile and link against include/nadia and
  libnadia_b200.so in the float and the double build.  The PhaseDiverse
  example and the Fresnel simulation include two headers this library does
  not provide -- the reference's image utilities (utils.h, from which they
  call nothing) and gperftools' google/profiler.h -- so they are compiled
  with test-only stand-ins for those two.  The partially coherent examples
  are out of scope.
* PolyCDI's public expand_wl / get_intensity, used by the Poly simulation and
  computed on the host by the drop-in class, equal the reference's
  (PolyCDI.c++:66-89, 296-334; double build, oracle/_ref) bit for bit.

Compile-and-compare only: nothing runs on a GPU.  Needs the reference sources
(skipped without them)."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "nadia-coecxs_b200")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import build_oracle  # noqa: E402

NADIA = build_oracle.reference_root()
EXAMPLES = ["PlanarCDI_example", "FresnelCDI_example", "FresnelCDI_WF_example", "PolyCDI_example",
            "ComplexConstraints_example", "PlanarCDI_simulation_example",
            "PolyCDI_simulation_example"]

needs_ref = pytest.mark.skipif(NADIA is None, reason="reference sources not present")
needs_lib = pytest.mark.skipif(not os.path.exists(os.path.join(LIBDIR, "libnadia_b200.so")),
                               reason="libnadia_b200.so not built")


@needs_ref
@needs_lib
@pytest.mark.parametrize("double", [False, True], ids=["float", "double"])
@pytest.mark.parametrize("name", EXAMPLES)
def test_reference_example_compiles_unchanged(tmp_path, name, double):
    src = os.path.join(NADIA, "examples", name + ".c")
    cmd = ["g++", "-std=c++17", "-O1", "-x", "c++", "-I", os.path.join(ROOT, "include", "nadia"),
           "-I", os.path.join(ROOT, "include"), src, "-L", LIBDIR, "-lnadia_b200",
           "-Wl,-rpath," + LIBDIR, "-o", str(tmp_path / name)]
    if double:
        cmd.insert(1, "-DDOUBLE_PRECISION")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


@needs_ref
@needs_lib
@pytest.mark.parametrize("double", [False, True], ids=["float", "double"])
@pytest.mark.parametrize("name", ["PhaseDiverse_example", "FresnelCDI_simulation_example"])
def test_reference_example_with_stand_in_headers(tmp_path, name, double):
    inc = tmp_path / "stand_in"
    (inc / "google").mkdir(parents=True)
    (inc / "utils.h").write_text("// stand-in: the example includes it and calls nothing from it\n")
    (inc / "google" / "profiler.h").write_text(
        "// stand-in for gperftools\n"
        "inline int ProfilerStart(const char *) { return 1; }\n"
        "inline void ProfilerStop() {}\n")
    src = os.path.join(NADIA, "examples", name + ".c")
    cmd = ["g++", "-std=c++17", "-O1", "-x", "c++", "-I", os.path.join(ROOT, "include", "nadia"),
           "-I", os.path.join(ROOT, "include"), "-I", str(inc), src, "-L", LIBDIR,
           "-lnadia_b200", "-Wl,-rpath," + LIBDIR, "-o", str(tmp_path / name)]
    if double:
        cmd.insert(1, "-DDOUBLE_PRECISION")
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("shim") / "libexpand_shim.so")
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-shared", "-fPIC",
           "-DDOUBLE_PRECISION", "-I", os.path.join(ROOT, "include", "nadia"),
           "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "dropin",
                                                             "expand_wl_shim.cpp"),
           "-L", LIBDIR, "-lnadia_b200", "-Wl,-rpath," + LIBDIR, "-o", out]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    lib = ctypes.CDLL(out)
    D = ctypes.POINTER(ctypes.c_double)
    lib.shim_expand_wl.argtypes = [ctypes.c_int, ctypes.c_int, D, ctypes.c_int, D, ctypes.c_int,
                                   ctypes.c_int, D, ctypes.POINTER(ctypes.c_int)]
    lib.shim_expand_wl.restype = ctypes.c_int
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def reference_expand(nx, ny, spec, field):
    ref = po.Reference("poly", nx, ny, variant="64")
    ref.set_spectrum(spec)
    f = ref.L.lib.ref_poly_expand_wl
    f.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                  ctypes.POINTER(ctypes.c_double)]
    f.restype = None
    out = np.zeros((nx, ny))
    fld = np.ascontiguousarray(field, dtype=np.complex128)
    f(ref.h, _p(fld), fld.shape[0], fld.shape[1], _p(out))
    return out


def gaussian_spectrum(nl, lc, fwhm, seed):
    # longest wavelength first, as PolyCDI's padding needs
    g = np.random.default_rng(seed)
    sig = fwhm * lc / 2.3548
    wl = np.linspace(lc + 2 * sig, lc - 2 * sig, nl)
    w = np.exp(-0.5 * ((wl - lc) / sig) ** 2) * (1 + 0.01 * g.random(nl))
    return np.stack([wl, w], axis=1)


@needs_ref
@pytest.mark.skipif(not po.reference_available("64"), reason="oracle/_ref not built")
@pytest.mark.parametrize("nx,ny,nl,fwhm,padded", [(64, 64, 10, 0.05, True),
                                                  (64, 64, 10, 0.05, False),
                                                  (48, 40, 7, 0.12, True),
                                                  (32, 32, 1, 0.05, False)])
def test_expand_wl_matches_reference(shim, nx, ny, nl, fwhm, padded):
    spec = gaussian_spectrum(nl, 1.0e-10, fwhm, seed=nx + nl)
    if nl > 2:
        spec[nl // 2 + 1, 1] = spec[:, 1].max()  # a tie: the first maximum is the centre
    pad = np.zeros(2, dtype=np.int32)
    # the padding the reference would use, from the shim's own bookkeeping
    probe = np.zeros((nx, ny))
    g = np.random.default_rng(7)
    f0 = g.standard_normal((nx, ny)) + 1j * g.standard_normal((nx, ny))
    assert shim.shim_expand_wl(nx, ny, _p(np.ascontiguousarray(spec)), nl, _p(f0), nx, ny,
                               _p(probe), pad.ctypes.data_as(ctypes.POINTER(ctypes.c_int))) == 0
    fx, fy = (nx + 2 * pad[0], ny + 2 * pad[1]) if padded else (nx, ny)
    field = g.standard_normal((fx, fy)) + 1j * g.standard_normal((fx, fy))
    ours = np.zeros((nx, ny))
    assert shim.shim_expand_wl(nx, ny, _p(np.ascontiguousarray(spec)), nl, _p(field), fx, fy,
                               _p(ours), pad.ctypes.data_as(ctypes.POINTER(ctypes.c_int))) == 0
    if padded and nl > 1:
        assert pad[0] > 0
    ref = reference_expand(nx, ny, spec, field)
    assert np.array_equal(ours, ref)
    assert np.isfinite(ours).all() and ours.max() > 0
