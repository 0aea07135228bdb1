"""The transmission constraint in the FP32 form -- its per-pixel part (unit
magnitude, charge flipping) inside the fused row pass, its complex-constraint
regions in the row pass split around the region sums -- and FP32
phase-diverse frames: each step matches the FP64 form (itself the oracle's
arithmetic) to the FP32 per-step bar, 2e-5 relative; short runs follow it."""
import numpy as np
import pytest

import pynadia
import pyoracle as po
import scenarios as sc
from pynadia import synth

pytestmark = pytest.mark.gpu

STEP_TOL = 2e-5


def l2rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def planar_pair(n=256):
    c = synth.PlanarCase(n, n // 6, 2, 1e8, seed=3, support_side=int(0.42 * n), beam_stop=6)
    out = []
    for prec in (pynadia.FP64, pynadia.FP32):
        s = pynadia.Solver("planar", n, n, precision=prec)
        s.set_support(c.support)
        s.set_intensity(c.intensity)
        s.set_beam_stop(c.beam_stop)
        s.initialise_estimate(4)
        out.append(s)
    return out


def fresnel_pair(n=256):
    f = synth.FresnelCase(n, seed=4)
    kw = dict(white_field=f.white_field, wavelength=f.wavelength, focal_detector_length=f.zfd,
              focal_sample_length=f.zfs, pixel_size=f.pixel, normalisation=0.97)
    out = []
    for prec in (pynadia.FP64, pynadia.FP32):
        s = pynadia.Solver("fresnel", n, n, precision=prec, **kw)
        s.set_support(f.support)
        s.set_intensity(f.intensity)
        s.initialise_estimate(2)
        out.append(s)
    return out


@pytest.mark.parametrize("kind", ["planar", "fresnel"])
@pytest.mark.parametrize("alg", ["ER", "HIO"])
@pytest.mark.parametrize("unity,flip,sign", [(True, True, 1), (True, True, -1), (True, False, 1),
                                             (False, True, -1)])
def test_teacher_forced_steps(kind, alg, unity, flip, sign):
    a, b = planar_pair() if kind == "planar" else fresnel_pair()
    for s in (a, b):
        s.set_algorithm(alg)
        s.set_transmission_constraint(unity, flip, sign)
    assert b.get_precision() == pynadia.FP32
    for _ in range(4):
        b.set_exit_surface_wave(a.get_exit_surface_wave())
        a.iterate(1)
        b.iterate(1)
        assert abs(b.get_error() - a.get_error()) <= STEP_TOL * a.get_error()
        assert l2rel(b.get_exit_surface_wave(), a.get_exit_surface_wave()) <= STEP_TOL
    if kind == "fresnel":  # get_transmission applies the constraint too
        assert l2rel(b.get_transmission(), a.get_transmission()) <= STEP_TOL


def test_constraint_changes_the_iterate():
    """The constraint is really applied: with it the FP32 step differs from
    the unconstrained one by far more than the FP32 bar."""
    a, b = planar_pair()
    for s in (a, b):
        s.set_algorithm("HIO")
    a.convert_to_fp64()  # both in step, one FP64
    b.set_transmission_constraint(True, True, 1)
    x0 = a.get_exit_surface_wave()
    b.set_exit_surface_wave(x0)
    a.iterate(1)
    b.iterate(1)
    assert l2rel(b.get_exit_surface_wave(), a.get_exit_surface_wave()) > 1e-3
    b.clear_transmission_constraint()
    a.set_exit_surface_wave(x0)
    b.set_exit_surface_wave(x0)
    a.iterate(1)
    b.iterate(1)
    assert l2rel(b.get_exit_surface_wave(), a.get_exit_surface_wave()) <= STEP_TOL


@pytest.mark.parametrize("kind", ["planar", "fresnel"])
@pytest.mark.parametrize("alg", ["ER", "HIO"])
def test_regions_teacher_forced_steps(kind, alg):
    """Three complex-constraint regions (one with a fixed c_mean, one
    overlapping another) with charge flipping and unit magnitude: the FP32
    row pass in two halves around the region sums against the FP64 form."""
    n = 256
    a, b = planar_pair(n) if kind == "planar" else fresnel_pair(n)
    regions, alphas, fixed = synth.constraint_regions(n)
    for s in (a, b):
        s.set_algorithm(alg)
        s.set_transmission_constraint(True, True, 1, regions, alphas, fixed)
    assert b.get_precision() == pynadia.FP32
    # FresnelCDI's initial transmission function is real (1 - 0.2 rand), so
    # sum |arg T| over a region is a sum of rounding errors and c_mean their
    # ratio to sum |ln|T||: any two arithmetics disagree there (the FP32 step
    # from it differs by 0.47, the next one by 1e-6).  The comparison starts
    # after two FP64 iterations have given T its phase.
    if kind == "fresnel":
        a.iterate(2)
    for _ in range(4):
        b.set_exit_surface_wave(a.get_exit_surface_wave())
        a.iterate(1)
        b.iterate(1)
        assert abs(b.get_error() - a.get_error()) <= STEP_TOL * a.get_error()
        assert l2rel(b.get_exit_surface_wave(), a.get_exit_surface_wave()) <= STEP_TOL
    if kind == "fresnel":  # get_transmission applies the constraint, regions included
        assert l2rel(b.get_transmission(), a.get_transmission()) <= STEP_TOL


def test_regions_change_the_iterate():
    """The regions are really applied: with them the FP32 step differs from
    the step with the per-pixel part alone by far more than the FP32 bar."""
    n = 256
    a, b = planar_pair(n)
    regions, alphas, fixed = synth.constraint_regions(n)
    for s in (a, b):
        s.set_algorithm("HIO")
    a.set_transmission_constraint(True, True, 1)
    b.set_transmission_constraint(True, True, 1, regions, alphas, fixed)
    b.set_exit_surface_wave(a.get_exit_surface_wave())
    a.iterate(1)
    b.iterate(1)
    assert l2rel(b.get_exit_surface_wave(), a.get_exit_surface_wave()) > 1e-3


def test_refusals_and_conversion():
    n = 256
    a, b = planar_pair(n)
    b.set_transmission_constraint(True, True, -1)
    with pytest.raises(pynadia.NadiaError):
        b.set_transmission_custom(lambda t, nx, ny: None)
    # converted, the constraint carries over and the FP64 steps are exact
    for s in (a, b):
        s.set_algorithm("HIO")
    a.set_transmission_constraint(True, True, -1)
    b.iterate(2)
    b.convert_to_fp64()
    a.set_exit_surface_wave(b.get_exit_surface_wave())
    a.iterate(3)
    b.iterate(3)
    assert np.array_equal(a.get_exit_surface_wave(), b.get_exit_surface_wave())
    p = synth.PolyCase(1024, seed=300, padding=28)  # padded to 1080^2
    s = pynadia.Solver("poly", 1024, 1024, precision=pynadia.FP32)
    s.set_support(p.support)
    s.set_intensity(p.intensity)
    s.set_spectrum(p.spectrum)
    with pytest.raises(pynadia.NadiaError):
        s.set_transmission_constraint(True, True, 1)
    with pytest.raises(pynadia.NadiaError):
        pynadia.PhaseDiverse().add_new_position(s, 0, 0)


@pytest.mark.parametrize("parallel", [False, True])
def test_phase_diverse_fp32_frames(parallel):
    """Three FP32 Fresnel frames (256^2, default constraint) against the same
    run on FP64 frames: the object follows to 1e-4 over three cycles."""
    n = 256
    c = sc.phase_diverse_inputs(n, positions=((0, 0), (20, -12), (-16, 24)))
    objs = []
    for prec in (pynadia.FP64, pynadia.FP32):
        frames = sc.phase_diverse_frames(
            lambda kind, nx, ny, **kw: pynadia.Solver(kind, nx, ny, precision=prec, **kw), c,
            constraint=True)
        pd = pynadia.PhaseDiverse(beta=0.9, parallel=parallel)
        for k, f in enumerate(frames):
            pd.add_new_position(f, *c.positions[k])
        pd.set_iterations_per_cycle(2)
        pd.initialise_estimate()
        pd.iterate(3)
        objs.append(pd.get_transmission())
        assert frames[0].get_precision() == prec
    assert l2rel(objs[1], objs[0]) <= 1e-4
    # and the FP64 run is the oracle's
    frames = sc.phase_diverse_frames(po.Oracle, c, constraint=True)
    pd = po._PhaseDiverse(frames[0].L, beta=0.9, parallel=parallel)
    for k, f in enumerate(frames):
        pd.add_new_position(f, *c.positions[k])
    pd.set_iterations_per_cycle(2)
    pd.initialise_estimate()
    for _ in range(3):
        pd.iterate()
    assert l2rel(objs[0], pd.get_transmission()) <= 1e-10
