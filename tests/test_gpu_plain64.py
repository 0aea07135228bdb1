"""Parity of the plain FP64 CUDA path with the oracle and with the golden
fixtures made by the reference itself.

The FP64 path performs the reference's per-element operations in the same
order with the same transform schedule, so the estimate, support and
transmission agree bit for bit with the oracle; the error metric is a sum
whose order differs on the GPU, so it is compared to 1e-12 relative.  The
bar set for this path is 1e-10 relative on every iterate."""
import os

import numpy as np
import pytest

import pynadia
import pyoracle as po
import scenarios as sc
from pynadia import synth

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-10          # the parity bar for the FP64 path, per iterate
ERR_TOL = 1e-12      # error-metric sums (different summation order)


def gpu(kind, nx, ny, **kw):
    return pynadia.Solver(kind, nx, ny, precision=pynadia.FP64, **kw)


def orc(kind, nx, ny, **kw):
    return po.Oracle(kind, nx, ny, **kw)


def compare(a, b, exact_keys=(), tol=TOL):
    for k in b:
        if k in ("input_digest",) or b[k] is None or (k in a and a[k] is None):
            continue
        x, y = np.asarray(a[k]), np.asarray(b[k])
        if k == "errors" or k == "best_err":
            assert sc.rel_err(x, y) <= ERR_TOL if k == "errors" else abs(x - y) <= ERR_TOL * abs(y), k
            continue
        if k in exact_keys:
            assert np.array_equal(x, y), (k, sc.rel_err(x, y))
        else:
            assert sc.rel_err(x, y) <= tol, (k, sc.rel_err(x, y))


@pytest.mark.parametrize("name", ["planar_mixed_32", "planar_mixed_32x48", "planar_custom_32",
                                  "fresnel_mixed_32", "poly_mixed_32", "fresnel_wf_mixed_32"])
def test_golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden",
                                                  os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    fn, kw = mg.CASES[name]
    res = fn(gpu, **kw)
    exact = () if name.startswith("poly") else ("esw", "support", "init", "transmission", "best",
                                                 "illum", "support0", "to_detector",
                                                 "from_detector")
    compare(res, g, exact_keys=exact)


@pytest.mark.parametrize("n,ny", [(64, 64), (48, 32), (40, 56)])
def test_planar_vs_oracle(n, ny):
    compare(sc.planar_mixed(gpu, n=n, ny=ny), sc.planar_mixed(orc, n=n, ny=ny),
            exact_keys=("esw", "support", "init", "best"))


@pytest.mark.parametrize("n", [64, 128])
def test_fresnel_wf_vs_oracle(n):
    compare(sc.fresnel_wf_mixed(gpu, n=n), sc.fresnel_wf_mixed(orc, n=n),
            exact_keys=("esw", "support", "init", "support0", "to_detector", "from_detector"))


@pytest.mark.parametrize("n", [32, 64])
def test_transmission_constraint_vs_oracle(n):
    """Charge flipping, unit magnitude and complex-constraint regions after
    every support projection (Planar: on the estimate; Fresnel: on the
    transmission function), over ER iterations, and the constrained support
    projection alone.  The constraint's log/exp/atan2/cos/sin come from the
    device's maths library and its region sums are reduced in another order,
    so agreement is to the 1e-10 bar (1e-14 for one projection) rather than
    bit for bit.  Under HIO the region update's phase, arg(T), jumps by 2*pi
    across the negative real axis, so last-bit differences in T can take
    different sides of that cut: the HIO sequences are checked against the
    reference on the CPU (tests/test_oracle_vs_reference.py), not here."""
    compare(sc.planar_constrained(gpu, n=n, hio_from=None),
            sc.planar_constrained(orc, n=n, hio_from=None))
    compare(sc.fresnel_constrained(gpu, n=n, hio_from=None),
            sc.fresnel_constrained(orc, n=n, hio_from=None))
    c = sc.planar_inputs(n, beam_stop=0)
    regions, alphas, fixed = sc.constraint_regions(n)
    g = np.random.default_rng(1)
    field = (g.standard_normal((n, n)) + 1j * g.standard_normal((n, n))) * 0.8
    out = []
    for make in (gpu, orc):
        s = make("planar", n, n)
        s.set_support(c.support)
        s.set_intensity(c.intensity)
        s.set_transmission_constraint(True, True, -1, regions, alphas, fixed)
        out.append(s.apply_support(field))
    assert sc.rel_err(out[0], out[1]) <= 1e-14


def test_transmission_custom_function():
    def clamp(t):
        t.real = np.clip(t.real, -0.5, 1.5)

    def run(make):
        c = sc.planar_inputs(32, beam_stop=0)
        s = make("planar", 32, 32)
        s.set_support(c.support)
        s.set_intensity(c.intensity)
        s.set_transmission_constraint(False, True, 1)
        s.set_transmission_custom(clamp)
        s.initialise_estimate(1)
        errs = []
        for _ in range(6):
            s.iterate()
            errs.append(s.get_error())
        return {"errors": np.array(errs), "esw": s.get_exit_surface_wave()}

    compare(run(gpu), run(orc))


def test_transmission_constraint_refusals():
    # the FP32 form takes regions but not a custom host function
    s = pynadia.Solver("planar", 256, 256, precision=pynadia.FP32)
    regions, alphas, fixed = sc.constraint_regions(256)
    s.set_transmission_constraint(True, True, 1, regions, alphas, fixed)
    with pytest.raises(pynadia.NadiaError) as e:
        s.set_transmission_custom(lambda t: None)
    assert e.value.code == 3
    with pytest.raises(pynadia.NadiaError) as e:   # at most 16 regions
        s.set_transmission_constraint(True, True, 1, [regions[0]] * 17, [alphas[0]] * 17)
    assert e.value.code == 1   # NADIA_ERR_INVALID: a bad argument
    s = gpu("planar", 32, 32)
    with pytest.raises(pynadia.NadiaError) as e:   # a custom function needs a constraint
        s.set_transmission_custom(lambda t: None)
    assert e.value.code == 2


def test_fresnel_wf_fixed_algorithm():
    f = sc.fresnel_wf_inputs(32)
    kw = dict(wavelength=f.wavelength, zone_focal_length=f.z12, focal_detector_length=f.z23,
              pixel_size=f.pixel)
    s = gpu("fresnel_wf", 32, 32, **kw)
    for call in (lambda: s.set_algorithm("HIO"), lambda: s.set_relaxation_parameter(0.5)):
        with pytest.raises(pynadia.NadiaError) as e:
            call()
        assert e.value.code == 3
    with pytest.raises(pynadia.NadiaError) as e:  # no FP32 tiles for 32-point transforms
        pynadia.Solver("fresnel_wf", 32, 32, precision=pynadia.FP32, **kw)
    assert e.value.code == 3


def test_fresnel_vs_oracle():
    compare(sc.fresnel_mixed(gpu, n=64), sc.fresnel_mixed(orc, n=64),
            exact_keys=("esw", "support", "init", "transmission", "illum"))


@pytest.mark.parametrize("n,padding", [(48, 3), (64, 4)])
def test_poly_vs_oracle(n, padding):
    compare(sc.poly_mixed(gpu, n=n, padding=padding), sc.poly_mixed(orc, n=n, padding=padding))


def test_large_prime_lengths_vs_oracle():
    """Transform lengths with prime factors above 64 (134 = 2 x 67, 2 x 131):
    the prime butterflies' direct sums formed from shared memory."""
    compare(sc.planar_mixed(gpu, n=134, ny=262, hio=6, raar=3, er=2),
            sc.planar_mixed(orc, n=134, ny=262, hio=6, raar=3, er=2),
            exact_keys=("esw", "support", "init"))


@pytest.mark.parametrize("n,ny", [(35, 35), (33, 45), (30, 45)])
def test_planar_odd_sizes_vs_oracle(n, ny):
    """Odd grids (PlanarCDI, FP64 form): the reference's quadrant swap on odd
    sizes replayed exactly; the rest of the loop as on even grids."""
    compare(sc.planar_mixed(gpu, n=n, ny=ny), sc.planar_mixed(orc, n=n, ny=ny),
            exact_keys=("esw", "support", "init"))


def test_odd_sizes_refused_elsewhere():
    for kind, prec in (("planar", pynadia.FP32), ("fresnel", pynadia.FP64)):
        with pytest.raises(pynadia.NadiaError) as e:
            if kind == "fresnel":
                pynadia.Solver(kind, 33, 33, precision=prec, white_field=np.ones((33, 33)),
                               wavelength=1.5e-10, focal_detector_length=1.0,
                               focal_sample_length=1e-3, pixel_size=13.5e-6)
            else:
                pynadia.Solver(kind, 33, 33, precision=prec)
        assert e.value.code in (1, 3)


def test_config1_256_hio_200_shrinkwrap():
    """PlanarCDI HIO FP64, 256^2, 200 iterations, shrinkwrap every 20."""
    a = sc.config1(gpu)
    b = sc.config1(orc)
    assert sc.rel_err(a["errors"], b["errors"]) <= ERR_TOL
    assert np.array_equal(a["esw"], b["esw"])
    assert np.array_equal(a["support"], b["support"])


def test_config1_random_phase_start():
    """Config 1 from its seeded random-phase start estimate (the same array
    given to both through set_exit_surface_wave)."""
    a = sc.config1(gpu, seed=17, start="random_phase")
    b = sc.config1(orc, seed=17, start="random_phase")
    assert sc.rel_err(a["errors"], b["errors"]) <= ERR_TOL
    assert np.array_equal(a["esw"], b["esw"])
    assert np.array_equal(a["support"], b["support"])
    # the start differs from the reference initialisation's
    c = sc.config1(orc, iterations=1, seed=17)
    assert not np.array_equal(c["esw"], b["esw"])


def config2(make, alg2=sc.HIO, beta2=0.9, iters=(50, 400, 50)):
    c = synth.planar_case("c2")
    s = make("planar", 1024, 1024)
    s.set_support(c.support)
    s.set_intensity(c.intensity)
    s.initialise_estimate(2)
    s.set_relaxation_parameter(beta2)
    errs = []
    for alg, n in zip((sc.ER, alg2, sc.ER), iters):
        s.set_algorithm(alg)
        for _ in range(n):
            s.iterate()
            errs.append(s.get_error())
    return np.array(errs), s.get_exit_surface_wave()


@pytest.mark.parametrize("alg,beta", [(sc.HIO, 0.9), (sc.RAAR, 0.8)])
def test_config2_1024_er_hio_er(alg, beta):
    """1024^2 FP64: ER 50 / HIO 400 (beta 0.9) / ER 50, then the same with RAAR
    at beta 0.8, compared with the oracle on every iterate."""
    ea, xa = config2(gpu, alg, beta)
    eb, xb = config2(orc, alg, beta)
    per_iter = np.abs(ea - eb) / np.abs(eb)
    assert per_iter.max() <= TOL
    assert sc.rel_err(xa, xb) <= TOL


def test_single_operators_and_autocorrelation():
    c = sc.planar_inputs(64)
    a, b = gpu("planar", 64, 64), orc("planar", 64, 64)
    for s in (a, b):
        s.set_support(c.support)
        s.set_intensity(c.intensity)
        s.set_beam_stop(c.beam_stop)
    f = np.random.default_rng(0).standard_normal((64, 64, 2)) @ np.array([1, 1j])
    for op in ("propagate_to_detector", "propagate_from_detector", "scale_intensity",
               "apply_support", "project_intensity"):
        assert np.array_equal(getattr(a, op)(f), getattr(b, op)(f)), op
    assert np.array_equal(a.get_intensity_autocorrelation(), b.get_intensity_autocorrelation())


def test_projection_properties():
    """Pf(Pf x) = Pf x on measured pixels; Ps(Ps x) = Ps x; beam-stop pixels
    are left free by the modulus step."""
    c = sc.planar_inputs(64)
    s = gpu("planar", 64, 64)
    s.set_support(c.support)
    s.set_intensity(c.intensity)
    s.set_beam_stop(c.beam_stop)
    f = np.random.default_rng(1).standard_normal((64, 64, 2)) @ np.array([1, 1j])
    p1 = s.project_intensity(f)
    p2 = s.project_intensity(p1)
    assert sc.rel_err(p2, p1) < 1e-12
    s1 = s.apply_support(f)
    assert np.array_equal(s.apply_support(s1), s1)
    d = s.propagate_to_detector(f)
    m = s.scale_intensity(d)
    free = c.beam_stop == 0
    assert np.array_equal(m[free], d[free])
    assert np.allclose(np.abs(m[~free]), np.sqrt(c.intensity[~free]), rtol=1e-12, atol=1e-12)
    back = s.propagate_from_detector(d)
    assert sc.rel_err(back, f) < 1e-12


def test_error_history_matches_get_error():
    c = sc.planar_inputs(32)
    s = gpu("planar", 32, 32)
    s.set_support(c.support)
    s.set_intensity(c.intensity)
    s.initialise_estimate(1)
    s.set_algorithm("HIO")
    errs = []
    for _ in range(7):
        s.iterate()
        errs.append(s.get_error())
    assert np.array_equal(s.get_error_history(7), np.array(errs))
    s.iterate(5)
    assert s.get_error_history(1)[0] == s.get_error()


def test_errors_are_status_codes():
    with pytest.raises(pynadia.NadiaError) as e:   # odd sizes: PlanarCDI only
        gpu("fresnel", 33, 32, white_field=np.ones((33, 32)), wavelength=1.5e-10,
            focal_detector_length=1.0, focal_sample_length=1e-3, pixel_size=13.5e-6)
    assert e.value.code == 1
    with pytest.raises(pynadia.NadiaError) as e:
        gpu("planar", 2 * 1031, 64)  # 1031 is a prime above 1021
    assert e.value.code == 1
    p = gpu("poly", 32, 32)
    with pytest.raises(pynadia.NadiaError) as e:
        p.iterate()
    assert e.value.code == 2
    with pytest.raises(pynadia.NadiaError):
        p.set_spectrum(np.array([[1.0, 1.0], [2.0, 3.0]]))  # shortest first: negative padding
    s = gpu("planar", 32, 32, n_best=1)
    assert s.get_best_result(1) == (None, None)


def test_spectrum_file_matches_reference_semantics(tmp_path):
    p = tmp_path / "spec.txt"
    p.write_text("Energy\tF.Density\n1200\t1.336e+15\n1250\t3e+15\n1300\t1.2e+15\n")
    s = gpu("poly", 64, 64)
    s.set_spectrum(str(p))
    o = orc("poly", 64, 64)
    o.set_spectrum(po.read_spec(str(p)))
    px, py = s.get_padding()
    q = po.ctypes.c_int(), po.ctypes.c_int()
    po.oracle_lib().lib.orc_padding(o.h, po.ctypes.byref(q[0]), po.ctypes.byref(q[1]))
    assert (px, py) == (q[0].value, q[1].value) and px > 0


def test_handles_of_different_sizes_coexist():
    """A smaller FP64 handle made after a larger one leaves the larger one's
    transforms working (the kernels' shared-memory limit is shared by all
    handles)."""
    big = sc.planar_inputs(256)
    a = gpu("planar", 256, 256)
    a.set_support(big.support)
    a.set_intensity(big.intensity)
    a.initialise_estimate(1)
    b = gpu("planar", 64, 64)
    small = sc.planar_inputs(64)
    b.set_support(small.support)
    b.set_intensity(small.intensity)
    b.initialise_estimate(1)
    a.set_algorithm(sc.HIO)
    a.iterate(2)
    b.iterate(2)
    o = orc("planar", 256, 256)
    o.set_support(big.support)
    o.set_intensity(big.intensity)
    o.initialise_estimate(1)
    o.set_algorithm(sc.HIO)
    o.iterate(2)
    assert np.array_equal(a.get_exit_surface_wave(), o.get_exit_surface_wave())
