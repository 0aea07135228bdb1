"""PhaseDiverseCDI on the GPU (nadia_pd_*) against the oracle and against the
golden fixtures the reference itself produced: the object, the frames'
estimates and the positions found by both position searches agree bit for
bit (the frames' error metrics, sums in a different order, to 1e-12
relative; with a transmission constraint, whose logarithms and arctangents
come from the device maths library, to the FP64 path's 1e-10)."""
import os

import numpy as np
import pytest

import pynadia
import pyoracle as po
import scenarios as sc

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def gpu(kind, nx, ny, **kw):
    return pynadia.Solver(kind, nx, ny, precision=pynadia.FP64, **kw)


def gpu_pd(**kw):
    return pynadia.PhaseDiverse(**kw)


def check(got, want, tol=0.0):
    for k in want:
        if k == "input_digest":
            continue
        a, b = np.asarray(got[k]), np.asarray(want[k])
        assert a.shape == b.shape, k
        if k == "errors":
            assert np.all(np.abs(a - b) <= 1e-12 * np.abs(b)), k
        elif tol == 0.0:
            assert np.array_equal(a, b), (k, np.max(np.abs(a - b)))
        else:
            assert np.max(np.abs(a - b)) <= tol * max(1.0, np.max(np.abs(b))), k


CASES = [dict(), dict(parallel=True), dict(granularity=2), dict(parallel=True, granularity=3),
         dict(parallel=True, beta=0.7, gamma=2.0, alphas=[1.0, 0.5, 2.0]), dict(adjust="cc"),
         dict(adjust="me"), dict(adjust="cc", forward=False), dict(adjust="me", granularity=2),
         dict(n=40, adjust="cc", granularity=2, parallel=True), dict(n=64, cycles=2)]


@pytest.mark.parametrize("kw", CASES,
                         ids=lambda kw: "-".join("%s=%s" % i for i in kw.items()) or "series")
def test_matches_oracle(kw):
    kw = dict(kw)
    n = kw.pop("n", 32)
    check(sc.phase_diverse_mixed(gpu, gpu_pd, n=n, **kw), sc.phase_diverse_mixed(po.Oracle, n=n, **kw))


def test_with_transmission_constraint():
    got = sc.phase_diverse_mixed(gpu, gpu_pd, constraint=True)
    want = sc.phase_diverse_mixed(po.Oracle, constraint=True)
    check(got, want, tol=1e-10)


@pytest.mark.parametrize("name", ["phase_diverse_series_32", "phase_diverse_parallel_g2_32",
                                  "phase_diverse_align_32", "phase_diverse_minerr_32"])
def test_matches_reference_golden(name):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    assert str(g["input_digest"]) == mg.input_digest(name)
    fn, kw = mg.CASES[name]
    check(fn(gpu, gpu_pd, **kw), {k: g[k] for k in g.files})


def test_fractional_positions_run_in_reference_order():
    """Positions whose truncation maps two local pixels onto one object pixel
    (a frame reaching past the object's left edge at a fractional offset) are
    blended in the reference's loop order."""
    out = []
    for make, make_pd in ((gpu, gpu_pd), (po.Oracle, None)):
        c = sc.phase_diverse_inputs(32)
        frames = sc.phase_diverse_frames(make, c)
        pd = make_pd(beta=0.8) if make_pd else po._PhaseDiverse(frames[0].L, beta=0.8)
        pd.add_new_position(frames[0], 0.0, 0.0)
        pd.add_new_position(frames[1], 3.5, -2.25)
        pd.add_new_position(frames[2], -2.75, 1.5)
        pd.initialise_estimate()
        pd.iterate()
        pd.iterate()
        out.append((pd.get_transmission(), frames[1].get_exit_surface_wave()))
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


def test_refusals():
    c = sc.phase_diverse_inputs(32)
    frames = sc.phase_diverse_frames(gpu, c)
    pd = pynadia.PhaseDiverse()
    with pytest.raises(pynadia.NadiaError):
        pd.set_probe_scaling(0, 2.0)  # before any position
    pd.add_new_position(frames[0], *c.positions[0])
    pd.set_probe_scaling(0, 2.0)
    with pytest.raises(pynadia.NadiaError):
        pd.adjust_positions(7)
    with pytest.raises(pynadia.NadiaError):
        pd.set_transmission(np.ones((5, 5), dtype=complex))
    # a frame in use can not be destroyed
    rc = frames[0].lib.nadia_destroy(frames[0].h)
    assert rc != 0
    pd.close()
    frames[0].close()  # released by the phase-diverse object
    assert frames[0].h is None
