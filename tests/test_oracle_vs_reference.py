"""The oracle restatement against the reference's own sources compiled here
(oracle/_ref).  Skipped when the reference was not available to build."""
import os

import numpy as np
import pytest

import pyoracle as po
import scenarios as sc

pytestmark = pytest.mark.skipif(not po.reference_available("64"),
                                reason="oracle/_ref not built")


def orc(kind, nx, ny, **kw):
    return po.Oracle(kind, nx, ny, **kw)


def ref(kind, nx, ny, **kw):
    return po.Reference(kind, nx, ny, variant="64", **kw)


def same(a, b):
    for k in a:
        if a[k] is None:
            continue
        assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k


# ny < nx is left out: the reference's apply_threshold loops j < nx
# (NADIA/src/BaseCDI.c++:485) and writes past the end of its array there,
# which corrupts its heap; the restatement and the CUDA path skip those writes.
@pytest.mark.parametrize("n,ny", [(64, 64), (40, 56)])
def test_planar(n, ny):
    same(sc.planar_mixed(orc, n=n, ny=ny), sc.planar_mixed(ref, n=n, ny=ny))


# odd sizes: Complex_2D::invert's swap loop then visits some elements twice
# and leaves the last column alone (Complex_2D.c++:318-353; the reference
# warns and runs), reproduced loop for loop
@pytest.mark.parametrize("n,ny", [(35, 35), (33, 45), (30, 45)])
def test_planar_odd_sizes(n, ny):
    same(sc.planar_mixed(orc, n=n, ny=ny), sc.planar_mixed(ref, n=n, ny=ny))


def test_planar_custom():
    same(sc.planar_custom(orc, n=48), sc.planar_custom(ref, n=48))


def test_fresnel():
    same(sc.fresnel_mixed(orc, n=64), sc.fresnel_mixed(ref, n=64))


def test_fresnel_non_square():
    # the phase-factor table is (nx/2) x (ny/2) with separate x and y centres
    # (FresnelCDI.c++:57-126); ny > nx (see test_planar for ny < nx)
    same(sc.fresnel_mixed(orc, n=40, ny=56), sc.fresnel_mixed(ref, n=40, ny=56))


@pytest.mark.parametrize("n", [32, 64])
def test_planar_transmission_constraint(n):
    same(sc.planar_constrained(orc, n=n), sc.planar_constrained(ref, n=n))


@pytest.mark.parametrize("n", [32, 64])
def test_fresnel_transmission_constraint(n):
    same(sc.fresnel_constrained(orc, n=n), sc.fresnel_constrained(ref, n=n))


@pytest.mark.parametrize("n", [32, 64])
def test_fresnel_wf(n):
    same(sc.fresnel_wf_mixed(orc, n=n), sc.fresnel_wf_mixed(ref, n=n))


@pytest.mark.parametrize("kw", [dict(), dict(parallel=True), dict(granularity=2),
                                dict(parallel=True, granularity=3),
                                dict(parallel=True, beta=0.7, gamma=2.0, alphas=[1.0, 0.5, 2.0]),
                                dict(constraint=True), dict(adjust="cc"), dict(adjust="me"),
                                dict(adjust="cc", forward=False), dict(adjust="me", granularity=2),
                                dict(n=40, adjust="cc", granularity=2, parallel=True)],
                         ids=lambda kw: "-".join("%s=%s" % i for i in kw.items()) or "series")
def test_phase_diverse(kw):
    kw = dict(kw)
    n = kw.pop("n", 32)
    same(sc.phase_diverse_mixed(orc, n=n, **kw), sc.phase_diverse_mixed(ref, n=n, **kw))


def test_phase_diverse_remove_positions():
    """remove_positions forgets the frames only: frames added afterwards
    reuse the earlier positions, scalings and results by index."""
    out = []
    for make in (orc, ref):
        c = sc.phase_diverse_inputs(32)
        frames = sc.phase_diverse_frames(make, c)
        import pyoracle
        pd = pyoracle._PhaseDiverse(frames[0].L, beta=0.9)
        for k, f in enumerate(frames[:2]):
            pd.add_new_position(f, *c.positions[k])
        pd.initialise_estimate()
        pd.iterate()
        pd.remove_positions()
        pd.add_new_position(frames[2], *c.positions[2])
        pd.iterate()
        out.append((pd.get_transmission(), pd.get_final_x_position(2), frames[2].get_exit_surface_wave()))
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][2], out[1][2])


@pytest.mark.parametrize("n,padding", [(48, 3), (64, 4)])
def test_poly(n, padding):
    same(sc.poly_mixed(orc, n=n, padding=padding), sc.poly_mixed(ref, n=n, padding=padding))


def test_single_operators():
    c = sc.planar_inputs(32)
    a, b = orc("planar", 32, 32), ref("planar", 32, 32)
    for s in (a, b):
        s.set_support(c.support)
        s.set_intensity(c.intensity)
    g = np.random.default_rng(0)
    f = g.standard_normal((32, 32)) + 1j * g.standard_normal((32, 32))
    for op in ("propagate_to_detector", "propagate_from_detector", "scale_intensity",
               "apply_support", "project_intensity"):
        assert np.array_equal(getattr(a, op)(f), getattr(b, op)(f)), op
    assert np.array_equal(a.get_intensity_autocorrelation(), b.get_intensity_autocorrelation())


def test_read_spec(tmp_path):
    p = tmp_path / "spec.txt"
    p.write_text("Energy\tF.Density\n1200\t1.336e+15\n1208\t1.439e+15\n1216\t2e+15\n")
    got = po.read_spec(str(p))
    s = ref("poly", 16, 16)
    s.L.lib.ref_poly_set_spectrum_file.argtypes = [po._V, po.ctypes.c_char_p]
    s.L.lib.ref_poly_set_spectrum_file(s.h, str(p).encode())
    assert got.shape == (3, 2)
    assert np.float32(got[0, 0]) == np.float32(1.0 / np.float32(1200))
    assert got[2, 1] == np.float32(2e15)


@pytest.mark.skipif(not (po.reference_available("32_fast") and
                         po.reference_available("32_fast_mt")),
                    reason="timing builds of the reference not built")
def test_threaded_fft_build_matches_serial_build(monkeypatch):
    """The reference's MULTI_THREADED float build, whose FFTs the shim splits
    over NADIA_REF_FFT_THREADS threads (the CPU baseline's --enable-threads
    leg), gives the serial float build's results bit for bit: 40 rows over 5
    threads, 56 columns in 4 blocks (the last one ragged) over 4 of them."""
    monkeypatch.setenv("NADIA_REF_FFT_THREADS", "5")

    def make(variant):
        return lambda kind, nx, ny, **kw: po.Reference(kind, nx, ny, variant=variant, **kw)

    same(sc.planar_mixed(make("32_fast"), n=40, ny=56, n_best=0),
         sc.planar_mixed(make("32_fast_mt"), n=40, ny=56, n_best=0))


def every_algorithm(make, n=32, ny=40):
    """Each named algorithm of BaseCDI::set_algorithm (BaseCDI.c++:192-275)
    for a few iterations from the same start, with the relaxation parameter
    changed before each switch (it takes effect at the switch)."""
    c = sc.planar_inputs(n, ny=ny)
    s = make("planar", n, ny)
    s.set_support(c.support)
    s.set_intensity(c.intensity)
    s.set_beam_stop(c.beam_stop)
    s.initialise_estimate(2)
    out = {}
    for k, alg in enumerate([sc.BIO, sc.BOO, sc.HIO, sc.DM, sc.SF, sc.ASR, sc.HPR, sc.RAAR,
                             sc.ER]):
        s.set_relaxation_parameter(0.6 + 0.04 * k)
        s.set_algorithm(alg)
        errs = []
        for _ in range(4):
            s.iterate()
            errs.append(s.get_error())
        out["errors_%d" % alg] = np.array(errs)
        out["esw_%d" % alg] = s.get_exit_surface_wave()
    return out


def test_every_named_algorithm():
    same(every_algorithm(orc), every_algorithm(ref))


def poly_non_square(make, nx=40, ny=56, seed=8):
    """PolyCDI on a non-square grid: the padding differs per axis
    ((lambda_0/lambda_c - 1) * n / 2 for n = nx and ny, PolyCDI.c++:86-87) and
    the wavelength expansion resamples each axis about its own centre."""
    from pynadia import synth
    g = np.random.default_rng(seed)
    spec = synth.gaussian_spectrum(6, 0.1, 1.0e-10, 2, nx)
    intensity = g.uniform(0.0, 50.0, (nx, ny)) * (g.random((nx, ny)) > 0.1)
    support = np.zeros((nx, ny))
    support[nx // 4:3 * nx // 4, ny // 4:3 * ny // 4] = 1.0
    s = make("poly", nx, ny, n_best=1)
    s.set_support(support)
    s.set_intensity(intensity)
    s.set_spectrum(spec)
    s.initialise_estimate(seed)
    errs = []
    for alg, its in ((sc.ER, 3), (sc.HIO, 5)):
        s.set_algorithm(alg)
        for _ in range(its):
            s.iterate()
            errs.append(s.get_error())
    s.apply_shrinkwrap(1.5, 0.1)
    s.iterate()
    errs.append(s.get_error())
    return {"errors": np.array(errs), "esw": s.get_exit_surface_wave(),
            "support": s.get_support()}


def test_poly_non_square():
    same(poly_non_square(orc), poly_non_square(ref))
