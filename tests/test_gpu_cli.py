"""The reconstruction tool (nadia-coecxs_b200/cli/CDI_reconstruction.cpp) on
the GPU: the double build writes exactly the files the reference's tool
writes (the oracle sequence of tests/cli_cases.py, itself pinned to the
reference tool by tests/test_cli_reference.py); a run restarted from a
checkpoint it wrote ends where the uninterrupted run ends; the float build
runs the fused FP32 form and its printed error metric follows the oracle's."""
import importlib.util
import os
import re

import numpy as np
import pytest

import cli_cases as cc
from test_cli_reference import check_outputs, ppm_writer, run_tool  # noqa: F401

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def tools():
    spec = importlib.util.spec_from_file_location(
        "nadia_build", os.path.join(ROOT, "nadia-coecxs_b200", "build.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    single, double = m.build_cli()
    return {"float": single, "double": double}


@pytest.mark.parametrize("kind,n", [("planar", 64), ("planar", 40), ("fresnel_wf", 32),
                                    ("fresnel", 32), ("poly", 32)])
def test_double_build_matches_oracle(tmp_path, tools, ppm_writer, kind, n):
    case = cc.CliCase(kind, n, tmp_path / kind)
    run_tool(tools["double"], case, seed=3)
    check_outputs(case, 3, ppm_writer)


@pytest.mark.parametrize("kind", ["planar", "fresnel"])
def test_double_build_diffraction_images(tmp_path, tools, ppm_writer, kind):
    """output_diffraction_estimate: |propagate_to_detector(estimate)|^2 on a
    log scale every output_iterations, bit for bit."""
    case = cc.CliCase(kind, 32, tmp_path / kind, diffraction=True, output_iterations=7)
    run_tool(tools["double"], case, seed=4)
    check_outputs(case, 4, ppm_writer)


def test_double_build_iteration_by_iteration(tmp_path, tools, ppm_writer):
    """info_level 2 runs and prints every iteration on its own; the files are
    the same as those of the chunked run."""
    case = cc.CliCase("planar", 64, tmp_path / "p", info_level=2)
    out = run_tool(tools["double"], case, seed=5)
    check_outputs(case, 5, ppm_writer)
    assert out.count("Error for iteration") == sum(k for _, k in case.stages) - 1
    assert "Applying shrink-wrap at iteration 11" in out


@pytest.mark.parametrize("build,n", [("double", 64), ("float", 256)])
def test_restart_from_checkpoint(tmp_path, tools, build, n):
    """The three runs are separate processes: the FP32 form's tile choice is
    pinned (NADIA_TUNE=0) so that all three run the same kernels -- a timed
    choice may differ between processes, and with it the rounding."""
    env = dict(os.environ, NADIA_TUNE="0")
    whole = cc.CliCase("planar", n, tmp_path, stages=[("HIO", 40)], shrinkwrap_iterations=0,
                       prefix="whole", output_iterations=100)
    run_tool(tools[build], whole, seed=2, env=env)
    first = cc.CliCase("planar", n, tmp_path, stages=[("HIO", 20)], shrinkwrap_iterations=0,
                       prefix="first", output_iterations=100)
    run_tool(tools[build], first, seed=2, env=env)
    rest = cc.CliCase("planar", n, tmp_path, stages=[("HIO", 20)], shrinkwrap_iterations=0,
                      prefix="rest", output_iterations=100, starting_point="first.cplx")
    run_tool(tools[build], rest, seed=99, env=env)  # the seed is unused after a restart
    a = cc.read_cplx(whole.path("whole.cplx"), n, n)
    b = cc.read_cplx(rest.path("rest.cplx"), n, n)
    assert np.array_equal(a, b)
    if build == "double":
        assert np.array_equal(a, whole.expected(2)["final"])


def test_float_build_runs_fused_form(tmp_path, tools):
    case = cc.CliCase("planar", 256, tmp_path, stages=[("HIO", 16)], shrinkwrap_iterations=0,
                      info_level=2, output_iterations=5)
    out = run_tool(tools["float"], case, seed=1)
    printed = [float(v) for v in re.findall(r"Error for iteration \d+ is (\S+)", out)]
    assert len(printed) == 15
    s = cc.po.Oracle("planar", 256, 256)
    s.set_support(case.support)
    s.set_intensity(case.data)
    s.initialise_estimate(1)
    s.set_algorithm(cc.ALG["HIO"])
    errs = []
    for _ in range(16):
        s.iterate()
        errs.append(s.get_error())
    # FP32 against FP64: the tracks agree closely over the first iterations
    np.testing.assert_allclose(printed[:10], errs[1:11], rtol=2e-3)
    final = cc.read_cplx(case.path(case.output_file), 256, 256)
    assert np.isfinite(final).all()
    assert sorted(os.path.basename(p) for p in case.image_names().values()) == \
        sorted(f for f in os.listdir(case.dir) if f.endswith(".ppm"))
