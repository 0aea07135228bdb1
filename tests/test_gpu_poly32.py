"""The FP32 PolyCDI form against the FP64 form (which matches the oracle to
1e-10, tests/test_gpu_plain64.py), on padded grids of 256 (240 padded by 8),
512 (480 by 16) and 1080 (1024 by 28, the 10-line 5% FWHM spectrum).

Tolerances as for the other FP32 passes: one iteration from the same state
agrees to 2e-5 relative in the estimate (L2) and in the error metric; runs of
up to 20 iterations keep every error metric within 1e-4 relative."""
import numpy as np
import pytest

import pynadia
from pynadia import synth

pytestmark = pytest.mark.gpu

STEP_TOL = 2e-5
RUN_TOL = 1e-4
CASES = [(240, 8), (480, 16), (1024, 28)]


def l2rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def poly_pair(n, padding, beam_stop=True):
    p = synth.PolyCase(n, seed=3, padding=padding, photons=1e8)
    bs = np.ones((n, n))
    if beam_stop:
        c = n // 2
        bs[c - 3:c + 3, c - 3:c + 3] = 0
    out = []
    for prec in (pynadia.FP64, pynadia.FP32):
        s = pynadia.Solver("poly", n, n, precision=prec)
        s.set_support(p.support)
        s.set_intensity(p.intensity)
        s.set_beam_stop(bs)
        s.set_spectrum(p.spectrum)
        assert s.get_padding() == (padding, padding)
        s.initialise_estimate(5)
        out.append(s)
    return out


@pytest.mark.parametrize("n,padding", CASES)
@pytest.mark.parametrize("alg", ["ER", "HIO", "RAAR"])
def test_one_iteration_matches_fp64(n, padding, alg):
    a, b = poly_pair(n, padding)
    for s in (a, b):
        s.set_algorithm(alg)
        s.iterate(1)
    ea, eb = a.get_error(), b.get_error()
    assert abs(eb - ea) <= STEP_TOL * abs(ea)
    assert l2rel(b.get_exit_surface_wave(), a.get_exit_surface_wave()) <= STEP_TOL


@pytest.mark.parametrize("n,padding", CASES)
def test_short_run_error_track(n, padding):
    a, b = poly_pair(n, padding)
    hist = []
    for s in (a, b):
        s.set_relaxation_parameter(0.9)
        s.set_algorithm("ER")
        s.iterate(4)
        s.set_algorithm("HIO")
        s.iterate(16)      # replays the captured 16-iteration graph on FP32
        hist.append(s.get_error_history(20))
    assert np.max(np.abs(hist[1] - hist[0]) / hist[0]) <= RUN_TOL


def test_teacher_forced_steps_with_shrinkwrap():
    a, b = poly_pair(480, 16)
    for s in (a, b):
        s.set_algorithm("HIO")
    for it in range(6):
        b.set_exit_surface_wave(a.get_exit_surface_wave())
        a.iterate(1)
        b.iterate(1)
        assert abs(b.get_error() - a.get_error()) <= STEP_TOL * a.get_error()
        assert l2rel(b.get_exit_surface_wave(), a.get_exit_surface_wave()) <= STEP_TOL
    a.apply_shrinkwrap(1.5, 0.1)
    b.apply_shrinkwrap(1.5, 0.1)
    sa, sb = a.get_support(), b.get_support()
    assert np.mean(np.abs(sa - sb) > 1e-5) < 1e-3


def test_unsupported_padded_size_is_refused():
    p = synth.PolyCase(200, seed=3, padding=8, photons=1e8)   # 216: no FP32 tiles
    s = pynadia.Solver("poly", 200, 200, precision=pynadia.FP32)
    with pytest.raises(pynadia.NadiaError) as e:
        s.set_spectrum(p.spectrum)
    assert e.value.code == 3


def test_batched_equals_alone_and_pass_times():
    """PolyCDI handles of one padded size step as one batch in
    nadia_iterate_many; each ends bit for bit where it ends alone."""
    p = synth.PolyCase(480, seed=3, padding=16, photons=1e8)

    def make(seed):
        s = pynadia.Solver("poly", 480, 480, precision=pynadia.FP32)
        s.set_support(p.support)
        s.set_intensity(p.intensity)
        s.set_spectrum(p.spectrum)
        s.initialise_estimate(seed)
        s.set_algorithm("HIO")
        return s

    batch = [make(k) for k in range(3)]
    alone = [make(k) for k in range(3)]
    pynadia.iterate_many(batch, 21)
    for s in alone:
        s.iterate(21)
    for a, b in zip(alone, batch):
        assert np.array_equal(a.get_error_history(21), b.get_error_history(21))
        assert np.array_equal(a.get_exit_surface_wave(), b.get_exit_surface_wave())
    c1, c2, r = pynadia.pass_times(batch, reps=3)
    assert c1 > 0 and c2 > 0 and r > 0


@pytest.mark.parametrize("alg", ["ER", "HIO"])
def test_1080_tile_shapes_agree(alg, monkeypatch):
    """The three 1080-point tile shapes (two 144-thread CTAs per SM with the
    row pass's x and support staged by cp.async, the same without staging,
    one 288-thread CTA; NADIA_POLY_TILE selects the first shape tried) run
    the same radix passes; the compiler may contract their multiply-adds
    differently, so after five iterations they agree to FP32 rounding (the
    per-step bar), not bit for bit."""
    p = synth.PolyCase(1024, seed=3, padding=28, photons=1e8)
    out = []
    for k in ("0", "1", "2"):
        monkeypatch.setenv("NADIA_POLY_TILE", k)
        s = pynadia.Solver("poly", 1024, 1024, precision=pynadia.FP32)
        s.set_support(p.support)
        s.set_intensity(p.intensity)
        s.set_spectrum(p.spectrum)
        s.initialise_estimate(7)
        s.set_algorithm(alg)
        s.iterate(5)
        out.append((s.get_error_history(5), s.get_exit_surface_wave()))
        s.close()
    for h, x in out[1:]:
        assert np.allclose(h, out[0][0], rtol=STEP_TOL, atol=0)
        assert l2rel(x, out[0][1]) <= STEP_TOL
