"""The request loop (nadia_server_*): admission by HBM budget and slot limit,
continuous batching, and results that are the same alone and in the mix.

* Admission charge: a reconstruction's device bytes, measured after it has
  run every operation that allocates (inputs, HIO, shrinkwrap, readback),
  never exceed nadia_estimate_device_bytes.
* Same alone and in the mix: a request's estimate, support and error are
  bit-identical whether it ran alone or among requests of other sizes,
  kinds and precisions admitted while it was on the GPU (tolerance: exact).
* Parity: an FP64 request gives the oracle's result for the same call
  sequence bit for bit (error metric to 1e-12); an FP32 request's error
  metrics before the first shrinkwrap stay within 1e-4 of the oracle's.
* Errors: invalid requests are refused at submit, a request that fails on
  the device side fails alone, and destroying a busy server ends cleanly."""
import gc
import time

import numpy as np
import pytest

import pynadia
import pyoracle as po
import scenarios as sc
from pynadia import synth

pytestmark = pytest.mark.gpu

GB = 1 << 30


def planar(n, seed):
    return synth.PlanarCase(n, n * 0.16, 2, 1e8, seed=seed, support_side=int(n * 0.42),
                            beam_stop=4)


def submit_planar(srv, n, seed, precision=pynadia.FP32, iterations=60, every=20):
    c = planar(n, seed)
    return srv.submit("planar", c.intensity, c.support, precision=precision,
                      beam_stop=c.beam_stop, algorithm="HIO", beta=0.9, iterations=iterations,
                      shrinkwrap_every=every, seed=seed)


def run_alone(request):
    srv = pynadia.Server(8 * GB, max_active=4, chunk=25)
    rid = request(srv)
    assert srv.wait(rid, 300)
    out = srv.result(rid)
    srv.close()
    return out


@pytest.mark.parametrize("kind,prec,n", [("planar", pynadia.FP64, 256),
                                         ("planar", pynadia.FP32, 512),
                                         ("fresnel", pynadia.FP64, 128),
                                         ("fresnel", pynadia.FP32, 256),
                                         ("poly", pynadia.FP64, 96),
                                         ("poly", pynadia.FP32, 240),
                                         ("fresnel_wf", pynadia.FP64, 128),
                                         ("fresnel_wf", pynadia.FP32, 256)])
def test_admission_charge_covers_device_bytes(kind, prec, n):
    # handles of earlier tests that are still unreferenced release their
    # buffers when collected; collect them before the count is taken
    gc.collect()
    before = pynadia.device_bytes()
    kw = {}
    if kind == "fresnel":
        f = synth.FresnelCase(n, seed=3)
        kw = dict(white_field=f.white_field, wavelength=f.wavelength,
                  focal_detector_length=f.zfd, focal_sample_length=f.zfs, pixel_size=f.pixel)
        inten, sup = f.intensity, f.support
    elif kind == "poly":
        p = synth.PolyCase(n, seed=3, padding=8 if prec == pynadia.FP32 else 4, photons=1e7)
        inten, sup = p.intensity, p.support
    elif kind == "fresnel_wf":
        w = synth.FresnelWFCase(n, seed=3)
        kw = dict(wavelength=w.wavelength, zone_focal_length=w.z12, focal_detector_length=w.z23,
                  pixel_size=w.pixel)
        inten, sup = w.intensity, None
    else:
        c = planar(n, 3)
        inten, sup = c.intensity, c.support
    s = pynadia.Solver(kind, n, n, precision=prec, **kw)
    if kind == "fresnel_wf":
        s.set_wf_support(w.z_diameter)
    else:
        s.set_support(sup, True)
    s.set_intensity(inten)
    s.set_beam_stop(np.ones((n, n)))
    pad = (0, 0)
    nl = 0
    if kind == "poly":
        s.set_spectrum(p.spectrum)
        pad = s.get_padding()
        nl = p.spectrum.shape[0]
    s.initialise_estimate(1)
    for alg in ("HIO", "RAAR", "ER"):
        if kind != "fresnel_wf":  # its algorithm is fixed
            s.set_algorithm(alg)
        s.iterate(3)
    s.apply_shrinkwrap(1.5, 0.1)
    s.get_exit_surface_wave()
    s.get_support()
    used = pynadia.device_bytes() - before
    est = pynadia.estimate_device_bytes(kind, n, n, prec, 0, pad, nl)
    assert 0 < used <= est, (used, est)
    assert used >= 0.55 * est, (used, est)  # and not grossly above it
    s.close()


def test_same_alone_and_in_the_mix():
    # the probes: an FP32 planar, an FP32 Fresnel and an FP64 planar request
    f = synth.FresnelCase(256, seed=8)

    def fresnel_req(srv):
        return srv.submit("fresnel", f.intensity, f.support, precision=pynadia.FP32,
                          white_field=f.white_field, wavelength=f.wavelength,
                          focal_detector_length=f.zfd, focal_sample_length=f.zfs,
                          pixel_size=f.pixel, auto_norm=True, algorithm="HIO", iterations=50,
                          shrinkwrap_every=20, seed=8)

    probes = [lambda srv: submit_planar(srv, 512, 11, iterations=70, every=20),
              fresnel_req,
              lambda srv: submit_planar(srv, 64, 12, precision=pynadia.FP64, iterations=45,
                                        every=15)]
    alone = [run_alone(p) for p in probes]

    # the mix: a small budget and slot limit so that requests queue, probes
    # submitted while others are on the device, sizes that share batches
    budget = 3 * pynadia.estimate_device_bytes("planar", 512, 512, pynadia.FP32) + \
        4 * pynadia.estimate_device_bytes("planar", 256, 256, pynadia.FP32)
    srv = pynadia.Server(budget, max_active=5, chunk=10)
    ids = [submit_planar(srv, 256, 20 + i, iterations=40 + 10 * i) for i in range(3)]
    ids.append(submit_planar(srv, 512, 30, iterations=90, every=30))
    time.sleep(0.05)
    probe_ids = [probes[0](srv)]
    ids.append(submit_planar(srv, 256, 31, iterations=33, every=11))
    time.sleep(0.02)
    probe_ids.append(probes[1](srv))
    ids.append(submit_planar(srv, 128, 32, precision=pynadia.FP64, iterations=30))
    probe_ids.append(probes[2](srv))
    ids.append(submit_planar(srv, 512, 33, iterations=50))
    for rid in ids + probe_ids:
        assert srv.wait(rid, 600)
    st = srv.stats()
    res, errors = {}, []
    for rid in ids + probe_ids:
        try:
            res[rid] = srv.result(rid)
        except pynadia.NadiaError as e:
            errors.append((rid, str(e)))
    srv.close()
    assert not errors, errors
    assert st["completed"] == len(ids) + len(probe_ids) and st["failed"] == 0, st
    assert st["peak_bytes"] <= budget
    mixed = [res[rid] for rid in probe_ids]
    for (ea, sa, erra, _), (eb, sb, errb, _) in zip(alone, mixed):
        assert np.array_equal(ea, eb)
        assert np.array_equal(sa, sb)
        assert erra == errb


def test_serving_request_types_same_alone_and_in_the_mix():
    """The serving workload's own request types -- PlanarCDI FP32 at 1024^2
    (radius 160) and 2048^2 (radius 320, 8x8 beam stop) and PolyCDI FP32 at
    1024^2 padded to 1080^2 with the 10-line, 5% FWHM spectrum -- give the
    same estimate, support and error alone and admitted among one another
    under a budget that makes them queue (tolerance: exact).  100 HIO
    iterations each, shrinkwrap every 50."""
    p1 = synth.PlanarCase(1024, 160, 2, 1e8, seed=100, support_side=400)
    p2 = synth.PlanarCase(2048, 320, 4, 1e9, seed=200, support_side=800, beam_stop=8)
    pp = synth.PolyCase(1024, seed=300, padding=28)
    common = dict(algorithm="HIO", beta=0.9, iterations=100, shrinkwrap_every=50,
                  shrinkwrap_sigma=1.5, shrinkwrap_threshold=0.1)

    def req(c, kind, seed):
        def submit(srv):
            if kind == "poly":
                return srv.submit("poly", c.intensity, c.support, precision=pynadia.FP32,
                                  spectrum=c.spectrum, seed=seed, **common)
            return srv.submit("planar", c.intensity, c.support, precision=pynadia.FP32,
                              beam_stop=c.beam_stop, seed=seed, **common)
        return submit

    probes = [req(p1, "planar", 1), req(p2, "planar", 2), req(pp, "poly", 3)]
    alone = [run_alone(p) for p in probes]

    est = pynadia.estimate_device_bytes
    budget = (2 * est("planar", 2048, 2048, pynadia.FP32) + est("planar", 1024, 1024, pynadia.FP32)
              + est("poly", 1024, 1024, pynadia.FP32, 0, (28, 28), 10))
    srv = pynadia.Server(budget, max_active=4, chunk=25)
    ids = [req(p2, "planar", 10)(srv), req(pp, "poly", 11)(srv), req(p1, "planar", 12)(srv)]
    time.sleep(0.02)
    probe_ids = [probes[0](srv)]
    ids.append(req(pp, "poly", 13)(srv))
    probe_ids.append(probes[1](srv))
    ids.append(req(p1, "planar", 14)(srv))
    probe_ids.append(probes[2](srv))
    ids.append(req(p2, "planar", 15)(srv))
    for rid in ids + probe_ids:
        assert srv.wait(rid, 600)
    st = srv.stats()
    res, errors = {}, []
    for rid in ids + probe_ids:
        try:
            res[rid] = srv.result(rid)
        except pynadia.NadiaError as e:
            errors.append((rid, str(e)))
    srv.close()
    assert not errors, errors
    assert st["completed"] == len(ids) + len(probe_ids) and st["failed"] == 0, st
    assert st["peak_bytes"] <= budget
    for (ea, sa, erra, _), (eb, sb, errb, _) in zip(alone, [res[r] for r in probe_ids]):
        assert np.array_equal(ea, eb)
        assert np.array_equal(sa, sb)
        assert erra == errb


def oracle_sequence(c, n, seed, iterations, every, beta=0.9):
    o = po.Oracle("planar", n, n)
    o.set_support(c.support)
    o.set_intensity(c.intensity)
    o.set_beam_stop(c.beam_stop)
    o.initialise_estimate(seed)
    o.set_relaxation_parameter(beta)
    o.set_algorithm(sc.HIO)
    errs = []
    for it in range(iterations):
        o.iterate()
        errs.append(o.get_error())
        if every and (it + 1) % every == 0:
            o.apply_shrinkwrap(1.5, 0.1)
    return o.get_exit_surface_wave(), o.get_support(), np.array(errs)


def test_fp64_request_matches_oracle():
    n, seed = 64, 41
    srv = pynadia.Server(GB, max_active=2, chunk=7)
    rid = submit_planar(srv, n, seed, precision=pynadia.FP64, iterations=50, every=20)
    assert srv.wait(rid, 300)
    esw, sup, err, _ = srv.result(rid)
    srv.close()
    e, s, errs = oracle_sequence(planar(n, seed), n, seed, 50, 20)
    assert np.array_equal(esw, e)
    assert np.array_equal(sup, s)
    assert abs(err - errs[-1]) <= 1e-12 * errs[-1]


def test_fp32_request_tracks_oracle():
    n, seed = 256, 42
    srv = pynadia.Server(GB, max_active=2, chunk=25)
    rid = submit_planar(srv, n, seed, iterations=20, every=0)
    assert srv.wait(rid, 300)
    _, _, err, _ = srv.result(rid)
    srv.close()
    _, _, errs = oracle_sequence(planar(n, seed), n, seed, 20, 0)
    assert abs(err - errs[-1]) <= 1e-4 * errs[-1]


def test_refusals_and_failures():
    srv = pynadia.Server(GB, max_active=2, chunk=5)
    c = planar(256, 1)
    with pytest.raises(pynadia.NadiaError) as e:  # more than the whole budget
        pynadia.Server(1 << 20).submit("planar", c.intensity, c.support)
    assert e.value.code == 5
    with pytest.raises(pynadia.NadiaError) as e:  # PolyCDI without a spectrum
        srv.submit("poly", c.intensity, c.support, precision=pynadia.FP64)
    assert e.value.code == 1
    # the FP32 form has no PolyCDI: this request fails when it starts, alone
    p = synth.PolyCase(256, seed=2, padding=4, photons=1e7)
    bad = srv.submit("poly", p.intensity, p.support, precision=pynadia.FP32,
                     spectrum=p.spectrum, iterations=5)
    good = submit_planar(srv, 256, 3, iterations=10, every=0)
    assert srv.wait(bad, 300) and srv.wait(good, 300)
    with pytest.raises(pynadia.NadiaError) as e:
        srv.result(bad)
    assert e.value.code == 3
    esw, _, err, _ = srv.result(good)
    assert np.isfinite(err) and np.abs(esw).max() > 0
    # destroying a server with work queued and on the device ends cleanly
    for i in range(4):
        submit_planar(srv, 512, 50 + i, iterations=400)
    srv.close()
