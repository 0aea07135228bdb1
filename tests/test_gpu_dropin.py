"""A caller written against the reference's C++ classes, compiled against
the drop-in headers (include/nadia) and run on the GPU, gives the oracle's
results.

Double build (-DDOUBLE_PRECISION): the FP64 form; estimate, support, initial
estimate and n-best result equal the oracle bit for bit, error metrics to
1e-12 relative (summation order).  Float build at grid sizes the FP32 form
does not cover: the FP64 form behind float host arrays, so the oracle fed the
same float-rounded inputs gives the same results once its outputs are rounded
to float (bit for bit; 1e-12 for error metrics).  Float build at 256x256:
the FP32 form: bit for bit the results of the same calls on an FP32 handle
through the C ABI in another process with the same tile choice; against the FP64 oracle, the error metrics up to the
first shrinkwrap within 1e-4 and all 43 within 2e-2 (the FP32 shrinkwrap
flips pixels that sit on the threshold, after which HIO trajectories part)."""
import os
import subprocess
import sys

import numpy as np
import pytest

import pyoracle as po
import scenarios as sc

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "dropin"))
import build_program  # noqa: E402

pytestmark = pytest.mark.gpu

ERR_TOL = 1e-12
F32_TRACK_TOL = 1e-4
F32_RUN_TOL = 2e-2


@pytest.fixture(scope="module")
def programs(tmp_path_factory):
    d = tmp_path_factory.mktemp("dropin")
    return {False: build_program.build(str(d / "cdi_float")),
            True: build_program.build(str(d / "cdi_double"), double=True)}


def put(d, name, a):
    a = np.asarray(a)
    if np.iscomplexobj(a):
        a = np.stack([a.real, a.imag], axis=-1)
    np.ascontiguousarray(a, dtype=np.float64).tofile(os.path.join(d, name))


def get(d, name, shape=None, cplx=False):
    a = np.fromfile(os.path.join(d, name), dtype=np.float64)
    if cplx:
        a = a[0::2] + 1j * a[1::2]
    return a.reshape(shape) if shape else a


def run(prog, mode, nx, ny, d, *extra, env=None):
    r = subprocess.run([prog, mode, str(nx), str(ny), str(d)] + [str(e) for e in extra],
                       capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr


def f32(a):
    a = np.asarray(a)
    if np.iscomplexobj(a):
        return a.real.astype(np.float32).astype(np.float64) + \
            1j * a.imag.astype(np.float32).astype(np.float64)
    return a.astype(np.float32).astype(np.float64)


class RoundedOracle:
    """The oracle with every array input rounded to float first, as a float
    build's Double_2D / Complex_2D hold them."""

    def __init__(self, kind, nx, ny, **kw):
        if "white_field" in kw:
            kw["white_field"] = f32(kw["white_field"])
        self.o = po.Oracle(kind, nx, ny, **kw)

    def __getattr__(self, name):
        fn = getattr(self.o, name)
        if name in ("set_support", "set_intensity", "set_beam_stop", "set_spectrum"):
            return lambda a, *r: fn(f32(a), *r)
        return fn


def oracle_factory(double):
    if double:
        return lambda kind, nx, ny, **kw: po.Oracle(kind, nx, ny, **kw)
    return lambda kind, nx, ny, **kw: RoundedOracle(kind, nx, ny, **kw)


def out_round(double, a):
    return np.asarray(a) if double else f32(a)


def assert_errors(got, ref, tol=ERR_TOL):
    assert got.shape == ref.shape
    assert sc.rel_err(got, ref) <= tol, sc.rel_err(got, ref)


@pytest.mark.parametrize("double", [True, False])
@pytest.mark.parametrize("nx,ny", [(32, 32), (40, 56)])
def test_planar(programs, tmp_path, double, nx, ny):
    c = sc.planar_inputs(nx, ny=ny)
    put(tmp_path, "support.bin", c.support)
    put(tmp_path, "intensity.bin", c.intensity)
    put(tmp_path, "beam_stop.bin", c.beam_stop)
    run(programs[double], "planar", nx, ny, tmp_path)
    ref = sc.planar_mixed(oracle_factory(double), n=nx, ny=ny)
    assert_errors(get(tmp_path, "errors.bin"), ref["errors"])
    for key, name in (("init", "init.bin"), ("esw", "esw.bin"), ("best", "best.bin")):
        got = get(tmp_path, name, (nx, ny), cplx=True)
        assert np.array_equal(got, out_round(double, ref[key])), key
    got = get(tmp_path, "support_out.bin", (nx, ny))
    assert np.array_equal(got, out_round(double, ref["support"]))
    assert abs(get(tmp_path, "best_err.bin")[0] - ref["best_err"]) <= ERR_TOL * ref["best_err"]


@pytest.mark.parametrize("double", [True, False])
def test_fresnel(programs, tmp_path, double):
    n = 64
    f = sc.fresnel_inputs(n)
    put(tmp_path, "support.bin", f.support)
    put(tmp_path, "intensity.bin", f.intensity)
    put(tmp_path, "white_field.bin", f.white_field)
    put(tmp_path, "params.bin", [f.wavelength, f.zfd, f.zfs, f.pixel])
    run(programs[double], "fresnel", n, n, tmp_path)
    ref = sc.fresnel_mixed(oracle_factory(double), n=n)
    assert_errors(get(tmp_path, "errors.bin"), ref["errors"])
    for key in ("init", "esw", "transmission", "illum"):
        got = get(tmp_path, key + ".bin", (n, n), cplx=True)
        assert np.array_equal(got, out_round(double, ref[key])), key
    assert np.array_equal(get(tmp_path, "support_out.bin", (n, n)),
                          out_round(double, ref["support"]))
    # the host formula on a caller's estimate: the GPU result to rounding
    host = get(tmp_path, "transmission_host.bin", (n, n), cplx=True)
    tol = 1e-12 if double else 1e-5
    assert sc.rel_err(host, ref["transmission"]) <= tol


@pytest.mark.parametrize("double", [True, False])
def test_poly(programs, tmp_path, double):
    n, padding = 48, 3
    p = sc.poly_inputs(n, padding)
    put(tmp_path, "support.bin", p.support)
    put(tmp_path, "intensity.bin", p.intensity)
    put(tmp_path, "spectrum.bin", p.spectrum)
    put(tmp_path, "spectrum_n.bin", [p.spectrum.shape[0]])
    run(programs[double], "poly", n, n, tmp_path, padding)
    ref = sc.poly_mixed(oracle_factory(double), n=n, padding=padding)
    # PolyCDI squares magnitudes with pow() in the oracle and m*m on the GPU
    assert_errors(get(tmp_path, "errors.bin"), ref["errors"], tol=1e-10)
    got = get(tmp_path, "esw.bin", (n, n), cplx=True)
    assert sc.rel_err(got, out_round(double, ref["esw"])) <= (1e-10 if double else 1e-6)


@pytest.mark.parametrize("double", [True, False])
def test_fresnel_wf(programs, tmp_path, double):
    n = 64
    f = sc.fresnel_wf_inputs(n)
    put(tmp_path, "intensity.bin", f.intensity)
    put(tmp_path, "params.bin", [f.wavelength, f.z12, f.z23, f.pixel, f.z_diameter])
    run(programs[double], "wf", n, n, tmp_path)
    ref = sc.fresnel_wf_mixed(oracle_factory(double), n=n)
    assert_errors(get(tmp_path, "errors.bin"), ref["errors"])
    for key in ("init", "esw"):
        got = get(tmp_path, key + ".bin", (n, n), cplx=True)
        assert np.array_equal(got, out_round(double, ref[key])), key
    assert np.array_equal(get(tmp_path, "support0.bin", (n, n)), out_round(double, ref["support0"]))
    assert np.array_equal(get(tmp_path, "support_out.bin", (n, n)),
                          out_round(double, ref["support"]))


def test_transmission_constraint(programs, tmp_path):
    """Double build: a PlanarCDI with a TransmissionConstraint (unit
    magnitude, charge flipping, three complex-constraint regions) over ER
    iterations, against the oracle to the 1e-10 bar (the constraint's maths
    functions come from the device library)."""
    n = 32
    c = sc.planar_inputs(n, beam_stop=0)
    regions, alphas, fixed = sc.constraint_regions(n)
    put(tmp_path, "support.bin", c.support)
    put(tmp_path, "intensity.bin", c.intensity)
    for r in range(3):
        put(tmp_path, "region%d.bin" % r, regions[r])
    put(tmp_path, "tc_params.bin", [v for (a1, a2), fc in zip(alphas, fixed) for v in (a1, a2, fc)])
    run(programs[True], "tc", n, n, tmp_path)
    ref = sc.planar_constrained(oracle_factory(True), n=n, hio_from=None)
    assert sc.rel_err(get(tmp_path, "errors.bin"), ref["errors"]) <= 1e-10
    assert sc.rel_err(get(tmp_path, "esw.bin", (n, n), cplx=True), ref["esw"]) <= 1e-10


def example_oracle(make, nx, ny, intensity, support):
    s = make("planar", nx, ny, n_best=4)
    s.set_support(support)
    s.set_intensity(intensity)
    s.initialise_estimate(0)
    errs, mags = [], []
    s.set_algorithm(sc.ER)
    for _ in range(2):
        for i in range(10):
            s.iterate()
            errs.append(s.get_error())
            if i % 10 == 0:
                mags.append(np.abs(s.get_exit_surface_wave()).sum())
            if i % 10 == 9:
                s.apply_shrinkwrap(1.5, 0.1)
        s.set_relaxation_parameter(0.5)
        s.set_algorithm(sc.HIO)
        for i in range(10, 30):
            s.iterate()
            errs.append(s.get_error())
            if i % 10 == 0:
                mags.append(np.abs(s.get_exit_surface_wave()).sum())
            if i % 10 == 9:
                s.apply_shrinkwrap(2.0, 0.1)
        s.set_algorithm(sc.ER)
        for i in range(30, 40):
            s.iterate()
            errs.append(s.get_error())
            if i % 10 == 9:
                s.apply_shrinkwrap(2.0, 0.1)
    return np.array(errs), np.array(mags), s.get_exit_surface_wave()


def test_example_flow_double(programs, tmp_path):
    n = 64
    c = sc.planar_inputs(n, beam_stop=0)
    put(tmp_path, "support.bin", c.support)
    put(tmp_path, "intensity.bin", c.intensity)
    run(programs[True], "example", n, n, tmp_path)
    errs, mags, esw = example_oracle(lambda k, x, y, **kw: po.Oracle(k, x, y, **kw), n, n,
                                     c.intensity, c.support)
    assert_errors(get(tmp_path, "errors.bin"), errs)
    assert sc.rel_err(get(tmp_path, "mags.bin"), mags) <= 1e-12
    assert np.array_equal(get(tmp_path, "esw.bin", (n, n), cplx=True), esw)


def test_planar_fp32_form(programs, tmp_path):
    """Float build at 256x256: the fused FP32 form (with n-best).  The
    program's results are those of the same calls made through the C ABI on
    an FP32 handle (bit for bit), and track the FP64 oracle."""
    n = 256
    c = sc.planar_inputs(n)
    put(tmp_path, "support.bin", c.support)
    put(tmp_path, "intensity.bin", c.intensity)
    put(tmp_path, "beam_stop.bin", c.beam_stop)
    # the first tile variant per axis in both processes (no timing-based choice)
    env = dict(os.environ, NADIA_TUNE="0")
    run(programs[False], "planar", n, n, tmp_path, env=env)
    ref = sc.planar_mixed(oracle_factory(False), n=n)
    got = get(tmp_path, "errors.bin")
    assert got.shape == ref["errors"].shape and np.all(np.isfinite(got))
    first_shrinkwrap = 3 + 8  # 3 ER, then shrinkwrap after the 8th HIO iteration
    assert sc.rel_err(got[:first_shrinkwrap], ref["errors"][:first_shrinkwrap]) <= F32_TRACK_TOL
    assert sc.rel_err(got, ref["errors"]) <= F32_RUN_TOL
    helper = os.path.join(os.path.dirname(os.path.abspath(__file__)), "dropin",
                          "fp32_handle_run.py")
    r = subprocess.run([sys.executable, helper, str(n), str(tmp_path / "same.npz")], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    same = np.load(tmp_path / "same.npz")
    assert np.array_equal(got, same["errors"])
    assert np.array_equal(get(tmp_path, "esw.bin", (n, n), cplx=True), f32(same["esw"]))
    sup = get(tmp_path, "support_out.bin", (n, n))
    assert np.array_equal(sup, f32(same["support"]))
    assert sup.min() >= 0 and sup.max() <= 1.0


def _phase_diverse_inputs(d, n):
    c = sc.phase_diverse_inputs(n)
    offsets = ((0, 0), (1, -2), (2, 1))
    put(d, "support.bin", c.support)
    params = [c.wavelength, c.zfd, c.pixel]
    for k in range(3):
        put(d, "white_field%d.bin" % k, c.white_fields[k])
        put(d, "intensity%d.bin" % k, c.intensities[k])
        params += [c.zfs[k], c.positions[k][0], c.positions[k][1], offsets[k][0], offsets[k][1]]
    put(d, "params.bin", params)


def test_phase_diverse_double_build(programs, tmp_path):
    """PhaseDiverseCDI (three FresnelCDI frames, cross-correlation position
    search, series iterations) from a caller of the reference's classes:
    double build bit-identical to the oracle."""
    n = 32
    _phase_diverse_inputs(tmp_path, n)
    run(programs[True], "pd", n, n, tmp_path)
    ref = sc.phase_diverse_mixed(po.Oracle, n=n, adjust="cc")
    obj = ref["object"]
    assert np.array_equal(get(tmp_path, "object.bin", obj.shape, cplx=True), obj)
    assert np.array_equal(get(tmp_path, "positions.bin", (3, 2)), ref["positions"])
    for k in range(3):
        assert np.array_equal(get(tmp_path, "frame%d.bin" % k, (n, n), cplx=True), ref["frames"][k])


def test_phase_diverse_float_build_moves_frames_to_fp64(programs, tmp_path):
    """Float build at 256^2: the frames start in the FP32 form (their
    initial estimates are made there) and move to the FP64 form when added;
    the run completes and its position search lands within a pixel of the
    double build's."""
    n = 256
    _phase_diverse_inputs(tmp_path, n)
    run(programs[False], "pd", n, n, tmp_path)
    ref = sc.phase_diverse_mixed(oracle_factory(False), n=n, adjust="cc")
    got = get(tmp_path, "object.bin", ref["object"].shape, cplx=True)
    assert np.isfinite(got).all()
    assert np.max(np.abs(get(tmp_path, "positions.bin", (3, 2)) - ref["positions"])) <= 1
