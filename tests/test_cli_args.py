"""The reconstruction tool's argument and configuration errors (no GPU is
touched before they are found): the messages and exit codes of the
reference's tool (NADIA/tools/CDI_reconstruction.c:94-170)."""
import importlib.util
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def tool():
    if not os.path.exists(os.path.join(ROOT, "nadia-coecxs_b200", "libnadia_b200.so")):
        pytest.skip("libnadia_b200.so not built")
    spec = importlib.util.spec_from_file_location(
        "nadia_build", os.path.join(ROOT, "nadia-coecxs_b200", "build.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m.build_cli()[0]


def run(tool, cwd, *args):
    r = subprocess.run([tool, *args], cwd=str(cwd), capture_output=True, text=True, timeout=60)
    return r.returncode, r.stdout


CONFIG = """pixels_x = 32
pixels_y = 32
output_iterations = 5
algorithm = HIO ER
iterations = 10 5
data_file_name = data.dbin
support_file_name = support.dbin
output_file_name_prefix = out
"""


def test_usage_without_arguments(tool, tmp_path):
    rc, out = run(tool, tmp_path)
    assert rc == 0 and "No config file given" in out and "Usage" in out


def test_missing_config_file(tool, tmp_path):
    rc, out = run(tool, tmp_path, "none.config", "planar", "0")
    assert rc == 0 and "Could not open the file none.config" in out


def test_too_many_arguments(tool, tmp_path):
    rc, out = run(tool, tmp_path, "a", "planar", "0", "extra")
    assert rc == 0 and "Wrong number of arguments given" in out


def test_missing_required_key(tool, tmp_path):
    (tmp_path / "c.config").write_text(CONFIG.replace("pixels_y = 32\n", ""))
    rc, out = run(tool, tmp_path, "c.config", "planar")
    assert rc == 0 and "Key:pixels_y not found in config file" in out
    assert "Problem reading the configuration file" in out


def test_list_lengths_differ(tool, tmp_path):
    (tmp_path / "c.config").write_text(CONFIG.replace("iterations = 10 5", "iterations = 10"))
    rc, out = run(tool, tmp_path, "c.config", "planar", "1")
    assert rc == 0 and "do not match" in out


@pytest.mark.parametrize("kind", ["partial", "partchar", "bogus"])
def test_unsupported_types(tool, tmp_path, kind):
    (tmp_path / "c.config").write_text(CONFIG)
    rc, out = run(tool, tmp_path, "c.config", kind, "1")
    assert rc == 1
    assert ("not part of this library" in out) if kind != "bogus" else ("unrecognised" in out)


def test_unreadable_starting_point(tool, tmp_path):
    (tmp_path / "c.config").write_text(CONFIG + "starting_point_file_name = nothing.cplx\n")
    rc, out = run(tool, tmp_path, "c.config", "planar", "1")
    assert rc == 1 and "Can not process the file nothing.cplx" in out
