"""FresnelCDI_WF in the FP32 form (FresnelCDI_WF.c++:122-182) against the
FP64 form, which equals the oracle and the reference bit for bit
(test_gpu_plain64.py::test_fresnel_wf_vs_oracle).

The FP32 iteration is one column pass and one row pass (eight FP32
transforms, the zone-plate factors per axis, the quadrant swaps as signs),
so it is compared with FP64 per step (teacher-forced: both forms take the
same estimate), over short error tracks, and on the operations around the
iteration (set_support's projected disk and soften, initialise_estimate,
shrinkwrap)."""
import numpy as np
import pytest

import pynadia
from pynadia import synth

pytestmark = pytest.mark.gpu

# One FP32 iteration from the FP64 state.  The modulus keeps the phase of
# the propagated field c9 and sets the magnitude to sqrt(I), so a rounding
# error e in c9 moves the estimate by about e sqrt(I)/|c9|: where |c9| is far
# below sqrt(I) (up to 1e5 times in the first iterations) that ratio
# amplifies FP32 rounding by as much.  Each pixel's difference is therefore
# divided by max(1, sqrt(I)/|c9|) (c9 from the FP64 form's single
# operators) before it is compared with the largest value (and in the L2
# norm); without that the first step at 256^2 differs by 3.4e-4 at the worst
# pixel and 1.6e-5 in the L2 norm, with it by 1.8e-7.
STEP_TOL = 2e-6
L2_TOL = 2e-6
ERR_TOL = 2e-5


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def step(d, s, x0, isqrt, measured):
    """Both forms iterate once from x0; returns the amplification-normalised
    difference of the estimates, its largest value and its L2 norm, each
    relative to the estimate's."""
    c9 = d.propagate_to_detector(d.apply_support(d.propagate_from_detector(x0)))
    for h in (d, s):
        h.set_exit_surface_wave(x0)
        h.iterate(1)
    xd, xs = d.get_exit_surface_wave(), s.get_exit_surface_wave()
    with np.errstate(divide="ignore"):
        amp = np.where(measured, isqrt / np.abs(c9), 1.0)
    amp = np.maximum(np.nan_to_num(amp, posinf=np.inf), 1.0)
    dn = np.abs(xs - xd) / amp
    return float(dn.max() / np.abs(xd).max()), float(np.linalg.norm(dn) / np.linalg.norm(xd))


def make(prec, f, nx, ny=None):
    ny = ny or nx
    s = pynadia.Solver("fresnel_wf", nx, ny, precision=prec, wavelength=f.wavelength,
                       zone_focal_length=f.z12, focal_detector_length=f.z23, pixel_size=f.pixel)
    return s


def setup(s, f, intensity):
    s.set_wf_support(f.z_diameter)
    s.set_intensity(intensity)
    s.initialise_estimate(0)
    return s


@pytest.mark.parametrize("n", [256, 512, 768, 1024, 1536, 2048])
def test_wf_fp32_steps_match_fp64(n):
    f = synth.FresnelWFCase(n, seed=7)
    d = setup(make(pynadia.FP64, f, n), f, f.intensity)
    s = setup(make(pynadia.FP32, f, n), f, f.intensity)
    assert rel(s.get_support(), d.get_support()) < 1e-6
    assert rel(s.get_exit_surface_wave(), d.get_exit_surface_wave()) < 1e-6
    isqrt, measured = np.sqrt(f.intensity), np.ones((n, n), bool)
    for k in range(4):
        norm, l2 = step(d, s, d.get_exit_surface_wave(), isqrt, measured)
        assert norm < STEP_TOL and l2 < L2_TOL, (k, norm, l2)
        assert abs(s.get_error() - d.get_error()) <= ERR_TOL * d.get_error(), (k, s.get_error(),
                                                                              d.get_error())


@pytest.mark.parametrize("nx,ny", [(256, 512), (512, 256)])
def test_wf_fp32_non_square(nx, ny):
    f = synth.FresnelWFCase(max(nx, ny), seed=9)
    sl = (slice(0, nx), slice(0, ny))
    inten = f.intensity[sl]
    d = setup(make(pynadia.FP64, f, nx, ny), f, inten)
    s = setup(make(pynadia.FP32, f, nx, ny), f, inten)
    assert rel(s.get_support(), d.get_support()) < 1e-6
    isqrt, measured = np.sqrt(inten), np.ones((nx, ny), bool)
    for _ in range(3):
        norm, l2 = step(d, s, d.get_exit_surface_wave(), isqrt, measured)
        assert norm < STEP_TOL and l2 < L2_TOL, (norm, l2)
        assert abs(s.get_error() - d.get_error()) <= ERR_TOL * d.get_error()


def test_wf_fp32_error_track_and_shrinkwrap():
    n = 512
    f = synth.FresnelWFCase(n, seed=11)
    d = setup(make(pynadia.FP64, f, n), f, f.intensity)
    s = setup(make(pynadia.FP32, f, n), f, f.intensity)
    ed, es = [], []
    for it in range(20):
        d.iterate(1)
        s.iterate(1)
        ed.append(d.get_error())
        es.append(s.get_error())
    ed, es = np.array(ed), np.array(es)
    assert np.max(np.abs(es - ed) / ed) < 1e-4, (es, ed)
    # the error history of a chunked call equals the per-iteration values
    s2 = setup(make(pynadia.FP32, f, n), f, f.intensity)
    s2.iterate(20)
    np.testing.assert_array_equal(s2.get_error_history(20), es)
    # shrinkwrap on the estimate (the detector-plane field, as the reference)
    d.apply_shrinkwrap(1.5, 0.1)
    s.apply_shrinkwrap(1.5, 0.1)
    a, b = s.get_support(), d.get_support()
    assert np.mean((a > 0) != (b > 0)) < 1e-3
    d.iterate(2)
    s.iterate(2)
    assert abs(s.get_error() - d.get_error()) < 1e-3 * d.get_error()


def test_wf_fp32_unmeasured_pixels():
    """A beam stop: unmeasured pixels keep the propagated field and stay out
    of the error metric."""
    n = 256
    f = synth.FresnelWFCase(n, seed=13)
    bs = np.ones((n, n))
    bs[n // 2 - 6:n // 2 + 6, n // 2 - 6:n // 2 + 6] = 0
    d = make(pynadia.FP64, f, n)
    s = make(pynadia.FP32, f, n)
    for h in (d, s):
        h.set_wf_support(f.z_diameter)
        h.set_intensity(f.intensity)
        h.set_beam_stop(bs)
        h.initialise_estimate(0)
    isqrt, measured = np.sqrt(f.intensity), bs > 0
    for _ in range(3):
        x0 = d.get_exit_surface_wave()
        norm, l2 = step(d, s, x0, isqrt, measured)
        assert norm < STEP_TOL and l2 < L2_TOL, (norm, l2)
        assert abs(s.get_error() - d.get_error()) <= ERR_TOL * d.get_error()
    # unmeasured pixels are not set to sqrt(I)
    x = s.get_exit_surface_wave()
    assert not np.allclose(np.abs(x[~measured]), isqrt[~measured], rtol=1e-3)
    np.testing.assert_allclose(np.abs(x[measured]), isqrt[measured], rtol=1e-5, atol=1e-6 * isqrt.max())


def test_wf_fp32_fixed_algorithm():
    f = synth.FresnelWFCase(256, seed=3)
    s = make(pynadia.FP32, f, 256)
    for call in (lambda: s.set_algorithm("HIO"), lambda: s.set_relaxation_parameter(0.5)):
        with pytest.raises(pynadia.NadiaError) as e:
            call()
        assert e.value.code == 3
