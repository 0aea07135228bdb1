"""The persistent passes' bounded device waits: a wait that runs out is
reported through the C ABI as NADIA_ERR_CUDA, and the GPU context stays
usable for the next reconstruction.

The case runs in a child process so that its environment applies from the
start: NADIA_TUNE_FILE pins the persistent, TMA-pipelined column and row
variants of the 1024^2 grid (the ones with mbarrier waits), and
NADIA_FAULT_WAIT=<polls>, set while one handle is created, arms that handle's
test hook: each CTA's first tile is expected on its barrier but its copy is
never issued, and waits give up after <polls> polls.  Every copy that is
issued lands before the CTA leaves, so nothing is left in flight; no fault,
trap or endless wait is involved."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import os, sys
import numpy as np
import pynadia
from pynadia import synth

n = 1024
c = synth.PlanarCase(n, 160, 2, 1e8, seed=5, support_side=400, beam_stop=4)


def make(prec):
    s = pynadia.Solver("planar", n, n, precision=prec)
    s.set_support(c.support)
    s.set_intensity(c.intensity)
    s.set_beam_stop(c.beam_stop)
    s.initialise_estimate(3)
    s.set_algorithm("HIO")
    return s


os.environ["NADIA_FAULT_WAIT"] = "2048"
bad = make(pynadia.FP32)
del os.environ["NADIA_FAULT_WAIT"]
bad.iterate(1)
try:
    bad.get_error()
except pynadia.NadiaError as e:
    assert e.code == 4 and "timed out" in str(e), str(e)
else:
    print("the wait did not run out")
    sys.exit(3)
bad.close()
good, ref = make(pynadia.FP32), make(pynadia.FP64)
for s in (good, ref):
    s.iterate(5)
eg, er = good.get_error_history(5), ref.get_error_history(5)
assert np.max(np.abs(eg - er) / er) <= 1e-4, (eg, er)
print("timeout reported; context usable")
'''


@pytest.mark.gpu
def test_wait_that_runs_out_is_reported(tmp_path):
    tune = tmp_path / "tune.txt"
    # variants(1024)[4]: persistent column and row passes, 256 threads, 16.16.4
    tune.write_text("1024 1024 0 1 4 4\n")
    env = dict(os.environ, NADIA_TUNE_FILE=str(tune),
               PYTHONPATH=os.pathsep.join([os.path.join(ROOT, "nadia-coecxs_b200"),
                                           os.environ.get("PYTHONPATH", "")]))
    env.pop("NADIA_FAULT_WAIT", None)
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, cwd=ROOT, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "timeout reported; context usable" in r.stdout


def test_tune_file_index_is_a_persistent_variant():
    """The index pinned above names a persistent 1024-point variant."""
    src = open(os.path.join(ROOT, "nadia-coecxs_b200", "csrc", "fused32_v1024.cu")).read()
    lines = [ln.strip() for ln in src.splitlines() if ln.strip().startswith("v.push_back(")]
    assert lines[4].startswith("v.push_back(make_persistent<1024,")
