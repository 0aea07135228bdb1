"""Reconstruction scenarios run identically on the reference (oracle/_ref), the
oracle restatement and the CUDA library.  A scenario takes a factory
``make(kind, nx, ny, **kw)`` and returns a dict of results."""
import numpy as np

from pynadia import synth

ER, BIO, BOO, HIO, DM, SF, ASR, HPR, RAAR, CUSTOM = range(10)


def planar_inputs(n, seed=5, beam_stop=4, ny=None):
    ny = ny or n
    c = synth.PlanarCase(n, max(3, n // 6), 2, 1e6, seed=seed, support_side=max(4, int(n * 0.42)),
                         beam_stop=beam_stop, ny=ny)
    return c


def planar_mixed(make, n=32, n_best=2, ny=None, hio=24, raar=10, er=6, seed=3):
    """ER/HIO/RAAR with shrinkwrap, a beam stop, the relaxation quirk and n-best."""
    ny = ny or n
    c = planar_inputs(n, ny=ny)
    s = make("planar", n, ny, n_best=n_best)
    s.set_support(c.support)
    s.set_intensity(c.intensity)
    s.set_beam_stop(c.beam_stop)
    s.initialise_estimate(seed)
    out = {"init": s.get_exit_surface_wave()}
    errs = []
    for _ in range(3):
        s.iterate()
        errs.append(s.get_error())
    s.set_relaxation_parameter(0.7)  # no effect until the algorithm changes
    s.set_algorithm(HIO)
    for it in range(hio):
        s.iterate()
        errs.append(s.get_error())
        if it % 8 == 7:
            s.apply_shrinkwrap(1.5, 0.1)
    s.set_relaxation_parameter(0.8)
    s.set_algorithm(RAAR)
    for _ in range(raar):
        s.iterate()
        errs.append(s.get_error())
    s.set_algorithm(ER)
    for _ in range(er):
        s.iterate()
        errs.append(s.get_error())
    out["errors"] = np.array(errs)
    out["esw"] = s.get_exit_surface_wave()
    out["support"] = s.get_support()
    out["transmission"] = s.get_transmission()
    if n_best:
        out["best_err"], out["best"] = s.get_best_result(n_best - 1)
    return out


def planar_custom(make, n=32, seed=4):
    """DM and a custom algorithm (both use the PfPs term: two projections)."""
    c = planar_inputs(n, beam_stop=0)
    s = make("planar", n, n)
    s.set_support(c.support, True)
    s.set_intensity(c.intensity)
    s.initialise_estimate(seed)
    errs = []
    s.set_algorithm(DM)
    for _ in range(6):
        s.iterate()
        errs.append(s.get_error())
    s.set_custom_algorithm(np.array([0.3, 0.5, 1.0, 0.1, 0.2, 0.05, 0.1, 0.2, 0.3, 0.1]))
    for _ in range(6):
        s.iterate()
        errs.append(s.get_error())
    return {"errors": np.array(errs), "esw": s.get_exit_surface_wave(),
            "support": s.get_support()}


def fresnel_inputs(n, seed=4, ny=None):
    return synth.FresnelCase(n, seed=seed, ny=ny)


def fresnel_mixed(make, n=32, seed=2, ny=None):
    f = fresnel_inputs(n, ny=ny)
    s = make("fresnel", n, ny or n, white_field=f.white_field, wavelength=f.wavelength,
             focal_detector_length=f.zfd, focal_sample_length=f.zfs, pixel_size=f.pixel,
             normalisation=0.97)
    s.set_support(f.support)
    s.set_intensity(f.intensity)
    s.auto_set_norm()
    s.initialise_estimate(seed)
    out = {"init": s.get_exit_surface_wave(), "illum": s.get_illumination_at_sample()}
    errs = []
    for _ in range(8):
        s.iterate()
        errs.append(s.get_error())
    s.set_algorithm(HIO)
    for it in range(12):
        s.iterate()
        errs.append(s.get_error())
        if it == 6:
            s.apply_shrinkwrap(2, 0.1)
    out["errors"] = np.array(errs)
    out["esw"] = s.get_exit_surface_wave()
    out["transmission"] = s.get_transmission()
    out["support"] = s.get_support()
    return out


def poly_inputs(n, padding, seed=9):
    return synth.PolyCase(n, seed=seed, padding=padding, photons=1e7)


def poly_mixed(make, n=32, padding=2, seed=7):
    p = poly_inputs(n, padding)
    s = make("poly", n, n, n_best=1)
    s.set_support(p.support)
    s.set_intensity(p.intensity)
    s.set_spectrum(p.spectrum)
    s.initialise_estimate(seed)
    errs = []
    for _ in range(3):
        s.iterate()
        errs.append(s.get_error())
    s.set_algorithm(HIO)
    for it in range(8):
        s.iterate()
        errs.append(s.get_error())
        if it == 4:
            s.apply_shrinkwrap(1.5, 0.1)
    return {"errors": np.array(errs), "esw": s.get_exit_surface_wave(),
            "support": s.get_support()}


def config1(make, iterations=200, seed=0, start="reference"):
    """PlanarCDI HIO FP64 at 256^2: disk R=40, sigma 2, 1e8 photons, 100x100
    initial support, beta 0.9, shrinkwrap every 20 (sigma 1.5, threshold
    0.1).  start="reference": initialise_estimate(seed); start="random_phase":
    the seeded random-phase estimate of synth.random_phase_start, set through
    set_exit_surface_wave."""
    c = synth.planar_case("c1")
    s = make("planar", 256, 256)
    s.set_support(c.support)
    s.set_intensity(c.intensity)
    if start == "random_phase":
        s.set_exit_surface_wave(synth.random_phase_start(c.intensity, c.support, seed))
    else:
        s.initialise_estimate(seed)
    s.set_algorithm(HIO)
    errs = []
    for it in range(iterations):
        s.iterate()
        errs.append(s.get_error())
        if it % 20 == 19:
            s.apply_shrinkwrap(1.5, 0.1)
    return {"errors": np.array(errs), "esw": s.get_exit_surface_wave(),
            "support": s.get_support()}


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    d = np.abs(a - b).max()
    m = np.abs(b).max()
    return d / m if m else d


def fresnel_wf_inputs(n, seed=6):
    return synth.FresnelWFCase(n, seed=seed)


def fresnel_wf_mixed(make, n=32, seed=6, iterations=12):
    """FresnelCDI_WF: the projected zone-plate support, sqrt(I) initial
    estimate, the fixed algorithm, a shrinkwrap, and the single operators."""
    f = fresnel_wf_inputs(n, seed)
    s = make("fresnel_wf", n, n, wavelength=f.wavelength, zone_focal_length=f.z12,
             focal_detector_length=f.z23, pixel_size=f.pixel)
    s.set_wf_support(f.z_diameter)
    s.set_intensity(f.intensity)
    s.initialise_estimate(0)
    out = {"init": s.get_exit_surface_wave(), "support0": s.get_support()}
    errs = []
    for it in range(iterations):
        s.iterate()
        errs.append(s.get_error())
        if it == iterations // 2:
            s.apply_shrinkwrap(1.5, 0.1)
    out["errors"] = np.array(errs)
    out["esw"] = s.get_exit_surface_wave()
    out["support"] = s.get_support()
    g = np.random.default_rng(seed)
    field = g.standard_normal((n, n)) + 1j * g.standard_normal((n, n))
    out["to_detector"] = s.propagate_to_detector(field)
    out["from_detector"] = s.propagate_from_detector(field)
    return out


def constraint_regions(n, ny=None):
    """Three ComplexConstraint regions (pynadia.synth.constraint_regions)."""
    return synth.constraint_regions(n, ny)


def planar_constrained(make, n=32, seed=3, iterations=12, hio_from=3):
    """PlanarCDI with a transmission constraint on the exit-surface wave:
    unit magnitude, charge flipping (sign -1) and three complex-constraint
    regions, through ER and (from iteration hio_from; None = never) HIO."""
    c = planar_inputs(n, beam_stop=0)
    s = make("planar", n, n)
    s.set_support(c.support)
    s.set_intensity(c.intensity)
    regions, alphas, fixed = constraint_regions(n)
    s.set_transmission_constraint(True, True, -1, regions, alphas, fixed)
    s.initialise_estimate(seed)
    errs = []
    for it in range(iterations):
        if it == hio_from:
            s.set_algorithm(HIO)
        s.iterate()
        errs.append(s.get_error())
    return {"errors": np.array(errs), "esw": s.get_exit_surface_wave()}


def fresnel_constrained(make, n=32, seed=2, iterations=12, hio_from=4):
    """FresnelCDI with a transmission constraint on the transmission function
    (FresnelCDI::apply_support and get_transmission_function)."""
    f = fresnel_inputs(n)
    s = make("fresnel", n, n, white_field=f.white_field, wavelength=f.wavelength,
             focal_detector_length=f.zfd, focal_sample_length=f.zfs, pixel_size=f.pixel,
             normalisation=0.97)
    s.set_support(f.support)
    s.set_intensity(f.intensity)
    regions, alphas, fixed = constraint_regions(n)
    s.set_transmission_constraint(True, True, 1, regions[:2], alphas[:2], fixed[:2])
    s.initialise_estimate(seed)
    errs = []
    for it in range(iterations):
        if it == hio_from:
            s.set_algorithm(HIO)
        s.iterate()
        errs.append(s.get_error())
    return {"errors": np.array(errs), "esw": s.get_exit_surface_wave(),
            "transmission": s.get_transmission()}


def phase_diverse_inputs(n, positions=((0, 0), (5, -3), (-4, 6)), seed=11):
    return synth.PhaseDiverseCase(n, positions=positions, seed=seed)


def phase_diverse_frames(make, c, offsets=None, constraint=False):
    """FresnelCDI frames of a PhaseDiverseCase, each initialised with its own
    seed; `offsets` perturbs the positions handed to add_new_position."""
    frames = []
    for k in range(len(c.positions)):
        s = make("fresnel", c.n, c.n, white_field=c.white_fields[k], wavelength=c.wavelength,
                 focal_detector_length=c.zfd, focal_sample_length=c.zfs[k], pixel_size=c.pixel,
                 normalisation=1.0)
        s.set_support(c.support)
        s.set_intensity(c.intensities[k])
        s.initialise_estimate(k + 1)
        if constraint:
            s.set_transmission_constraint(True, True)
        frames.append(s)
    return frames


def phase_diverse_mixed(make, make_pd=None, n=32, parallel=False, granularity=1, cycles=3,
                        per_cycle=2, beta=1.0, gamma=1.0, alphas=None, adjust=None,
                        offsets=((0, 0), (1, -2), (2, 1)), constraint=False, forward=True):
    """PhaseDiverseCDI over three Fresnel frames: optional position search
    (adjust = 'cc' CROSS_CORRELATION or 'me' MINIMUM_ERROR, from positions
    off by `offsets`), then `cycles` iterations in series or parallel mode."""
    c = phase_diverse_inputs(n)
    frames = phase_diverse_frames(make, c, constraint=constraint)
    if make_pd is None:  # the CPU libraries: PhaseDiverseCDI of the frames' own library
        import pyoracle
        make_pd = lambda **k: pyoracle._PhaseDiverse(frames[0].L, **k)  # noqa: E731
    pd = make_pd(beta=beta, gamma=gamma, parallel=parallel, granularity=granularity)
    for k, f in enumerate(frames):
        x, y = c.positions[k]
        dx, dy = offsets[k] if adjust else (0, 0)
        pd.add_new_position(f, x + dx, y + dy, alphas[k] if alphas else 1.0)
    pd.set_iterations_per_cycle(per_cycle)
    pd.initialise_estimate()
    out = {"init": pd.get_transmission()}
    if adjust == "cc":
        pd.adjust_positions(0, forward, -6, 6, -6, 6)
    elif adjust == "me":
        pd.adjust_positions(1, forward, -6, 6, -6, 6, 2.0)
    for _ in range(cycles):
        pd.iterate()
    out["object"] = pd.get_transmission()
    out["positions"] = np.array([[pd.get_final_x_position(k), pd.get_final_y_position(k)]
                                 for k in range(len(frames))])
    out["frames"] = np.array([f.get_exit_surface_wave() for f in frames])
    out["errors"] = np.array([f.get_error() for f in frames])
    return out
