"""The reconstruction tool's sequence of calls (tests/cli_cases.py) on the
oracle reproduces the reference's own tool (NADIA/tools/CDI_reconstruction.c
built into oracle/_ref) bit for bit: final estimate, magnitude images and the
Fresnel transmission function.  This pins the expected outputs that the GPU
tool is checked against (tests/test_gpu_cli.py).  CPU only; skipped when
oracle/_ref was not built."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

import cli_cases as cc

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "dropin"))
import build_program  # noqa: E402

REF_CLI = os.path.join(build_program.REF_DIR, "CDI_reconstruction_ref")

pytestmark = pytest.mark.skipif(not os.path.exists(REF_CLI), reason="oracle/_ref not built")


@pytest.fixture(scope="module")
def ppm_writer(tmp_path_factory):
    """write_ppm of include/nadia/io.h (byte-identical to the reference's,
    tests/test_io_formats.py) for the expected images."""
    if not os.path.exists(os.path.join(build_program.LIBDIR, "libnadia_b200.so")):
        pytest.skip("libnadia_b200.so not built")
    so = build_program.build_io_shim(str(tmp_path_factory.mktemp("shim") / "io.so"))
    L = ctypes.CDLL(so)
    D = ctypes.POINTER(ctypes.c_double)
    L.shim_write_ppm.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, D, ctypes.c_int,
                                 ctypes.c_double, ctypes.c_double]

    def write(directory, name, img, log_scale=False):
        os.makedirs(directory, exist_ok=True)
        a = np.ascontiguousarray(img, dtype=np.float64)
        cwd = os.getcwd()
        os.chdir(directory)
        try:
            assert L.shim_write_ppm(name.encode(), a.shape[0], a.shape[1], a.ctypes.data_as(D),
                                    1 if log_scale else 0, 0.0, 0.0) == 1
        finally:
            os.chdir(cwd)
        with open(os.path.join(directory, name), "rb") as fh:
            return fh.read()
    return write


def run_tool(exe, case, seed, timeout=600, env=None):
    r = subprocess.run([exe, os.path.basename(case.config), case.kind, str(seed)], cwd=case.dir,
                       capture_output=True, text=True, timeout=timeout, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def check_outputs(case, seed, ppm_writer, exp=None):
    exp = exp or case.expected(seed)
    n = case.n
    got = cc.read_cplx(case.path(case.output_file), n, n)
    assert np.array_equal(got, exp["final"])
    names = case.image_names()
    assert sorted(names) == sorted(exp["images"])
    for i, name in names.items():
        want = ppm_writer(case.path("expected"), name, exp["images"][i])
        with open(case.path(name), "rb") as fh:
            assert fh.read() == want, name
    if case.kind == "fresnel":
        t = cc.read_cplx(case.path("transmission_function.cplx"), n, n)
        assert np.array_equal(t, exp["transmission"])
    if case.diffraction:
        for i, name in case.diffraction_names().items():
            want = ppm_writer(case.path("expected"), name, exp["diffraction"][i], True)
            with open(case.path(name), "rb") as fh:
                assert fh.read() == want, name


@pytest.mark.parametrize("kind,n", [("planar", 64), ("planar", 40), ("fresnel_wf", 32),
                                    ("fresnel", 32), ("poly", 32)])
def test_reference_tool_matches_oracle_sequence(tmp_path, ppm_writer, kind, n):
    case = cc.CliCase(kind, n, tmp_path / kind)
    run_tool(REF_CLI, case, seed=3)
    check_outputs(case, 3, ppm_writer)
