"""The drop-in C++ headers (include/nadia: BaseCDI, PlanarCDI, FresnelCDI,
PolyCDI, Complex_2D, Double_2D, types) compile and link a caller written
against the reference's classes, in both the float and the double build.
Runs nothing on a GPU; tests/test_gpu_dropin.py runs the program."""
import os
import sys

import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "dropin"))
import build_program  # noqa: E402


@pytest.mark.parametrize("double", [False, True])
def test_caller_compiles_and_links(tmp_path, double):
    if not os.path.exists(os.path.join(build_program.LIBDIR, "libnadia_b200.so")):
        pytest.skip("libnadia_b200.so not built")
    out = build_program.build(str(tmp_path / "cdi_program"), double=double)
    assert os.path.getsize(out) > 0
