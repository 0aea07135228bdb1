"""nadia_convert_to_fp64: an FP32 reconstruction moved to the FP64 form in
place continues exactly as an FP64 reconstruction given the same inputs and
the estimate the FP32 form had reached."""
import numpy as np
import pytest

import pynadia
import scenarios as sc
from pynadia import synth

pytestmark = pytest.mark.gpu


def _planar(prec, c):
    s = pynadia.Solver("planar", 256, 256, precision=prec, n_best=2)
    s.set_support(c.support)
    s.set_intensity(c.intensity)
    s.set_beam_stop(c.beam_stop)
    return s


def test_planar_continues_as_fp64():
    c = synth.PlanarCase(256, 40, 2, 1e8, seed=3, support_side=100, beam_stop=6)
    a = _planar(pynadia.FP32, c)
    a.initialise_estimate(1)
    a.set_algorithm(sc.HIO)
    for _ in range(5):
        a.iterate()
    esw = a.get_exit_surface_wave()
    sup = a.get_support()
    a.convert_to_fp64()
    assert a.get_precision() == pynadia.FP64
    assert np.array_equal(a.get_exit_surface_wave(), esw)
    assert np.array_equal(a.get_support(), sup)
    b = _planar(pynadia.FP64, c)
    b.set_exit_surface_wave(esw)
    b.set_algorithm(sc.HIO)
    for _ in range(6):
        a.iterate()
        b.iterate()
        assert a.get_error() == b.get_error()
    a.apply_shrinkwrap(1.5, 0.1)
    b.apply_shrinkwrap(1.5, 0.1)
    a.iterate()
    b.iterate()
    assert np.array_equal(a.get_exit_surface_wave(), b.get_exit_surface_wave())
    assert np.array_equal(a.get_support(), b.get_support())
    # n-best results and the error history carry over
    err, best = a.get_best_result(0)
    assert np.isfinite(best).all() and err <= 1
    assert len(a.get_error_history(12)) == 12


def test_fresnel_continues_as_fp64():
    f = synth.FresnelCase(256, seed=4)
    kw = dict(white_field=f.white_field, wavelength=f.wavelength, focal_detector_length=f.zfd,
              focal_sample_length=f.zfs, pixel_size=f.pixel, normalisation=0.97)
    a = pynadia.Solver("fresnel", 256, 256, precision=pynadia.FP32, **kw)
    b = pynadia.Solver("fresnel", 256, 256, precision=pynadia.FP64, **kw)
    for s in (a, b):
        s.set_support(f.support)
        s.set_intensity(f.intensity)
    a.initialise_estimate(2)
    for _ in range(4):
        a.iterate()
    esw = a.get_exit_surface_wave()
    a.convert_to_fp64()
    b.set_exit_surface_wave(esw)
    assert np.array_equal(a.get_illumination_at_sample(), b.get_illumination_at_sample())
    for _ in range(5):
        a.iterate()
        b.iterate()
    assert np.array_equal(a.get_exit_surface_wave(), b.get_exit_surface_wave())
    assert np.array_equal(a.get_transmission(), b.get_transmission())
    # the constraint and phase-diverse paths accept it now
    a.set_transmission_constraint(True, True)
    pd = pynadia.PhaseDiverse()
    pd.add_new_position(a, 0, 0)
    pd.initialise_estimate()
    pd.iterate()
    pd.close()
