"""The FP32 fused form against the FP64 form (the oracle's arithmetic, bit
for bit) beyond one step, on an ensemble of seeded PlanarCDI problems at
256^2 (config 1's generator: disk radius 40, sigma 2, 1e8 photons, 100x100
initial support; problem k has data seed 1000+k and initialise_estimate(k)).

* Same state, contractive steps: the FP64 state after 150 HIO iterations
  (shrinkwrap every 20) given to an FP64 and an FP32 reconstruction; 50 ER
  iterations keep every iterate's error metric within RUN_TOL (1e-4,
  relative) in both.  ER is a composition of projections, so rounding does
  not grow along the track.
* Ensemble, chaotic schedule: 200 HIO iterations with shrinkwrap every 20 in
  three forms -- FP64, FP32, and FP64 from a start perturbed by 1e-12
  (relative).  Over 16 problems the FP32 final errors are drawn from the same
  distribution as the FP64 ones (two-sample Kolmogorov-Smirnov p >= 0.01),
  and the median per-problem distance of FP32 from FP64 is no larger than
  that of the 1e-12-perturbed FP64 control (times 3), or 1e-4 where neither
  run parts."""
import numpy as np
import pytest

import pynadia
from pynadia import synth

pytestmark = pytest.mark.gpu

RUN_TOL = 1e-4
SEEDS = 16
N = 256


def case(k):
    return synth.PlanarCase(N, 40, 2, 1e8, seed=1000 + k, support_side=100)


def make(c, prec, k):
    s = pynadia.Solver("planar", N, N, precision=prec)
    s.set_support(c.support)
    s.set_intensity(c.intensity)
    s.initialise_estimate(k)
    s.set_algorithm("HIO")
    return s


def hio(solvers, iters, every=20):
    for _ in range(iters // every):
        pynadia.iterate_many(solvers, every)
        for s in solvers:
            s.apply_shrinkwrap(1.5, 0.1)


def test_same_state_contractive_steps_agree():
    worst = 0.0
    for k in range(4):
        c = case(k)
        a = make(c, pynadia.FP64, k)
        hio([a], 140)
        a.iterate(10)
        x, sup = a.get_exit_surface_wave(), a.get_support()
        b = make(c, pynadia.FP32, k)
        for s in (a, b):
            s.set_exit_surface_wave(x)
            s.set_support(sup)
            s.set_algorithm("ER")
            s.iterate(50)
        ha, hb = a.get_error_history(50), b.get_error_history(50)
        d = np.max(np.abs(hb - ha) / ha)
        worst = max(worst, d)
        assert d <= RUN_TOL, (k, d)
        a.close()
        b.close()
    print("same state, 50 ER: worst per-iterate relative difference %.3g" % worst)


def test_ensemble_final_errors():
    from scipy import stats

    finals = []
    for k in range(SEEDS):
        c = case(k)
        a, b, p = make(c, pynadia.FP64, k), make(c, pynadia.FP32, k), make(c, pynadia.FP64, k)
        x0 = p.get_exit_surface_wave()
        g = np.random.default_rng(1000 + k)
        p.set_exit_surface_wave(x0 * (1 + 1e-12 * g.standard_normal(x0.shape)))
        hio([a, b, p], 200)
        finals.append([s.get_error() for s in (a, b, p)])
        for s in (a, b, p):
            s.close()
    F = np.array(finals)
    ks = stats.ks_2samp(F[:, 1], F[:, 0]).pvalue
    d32 = np.median(np.abs(F[:, 1] - F[:, 0]) / F[:, 0])
    dctl = np.median(np.abs(F[:, 2] - F[:, 0]) / F[:, 0])
    print("ensemble of %d: FP64 mean %.4g sd %.3g, FP32 mean %.4g sd %.3g, KS p %.3g, "
          "median distance FP32 %.3g, perturbed FP64 %.3g"
          % (SEEDS, F[:, 0].mean(), F[:, 0].std(ddof=1), F[:, 1].mean(), F[:, 1].std(ddof=1),
             ks, d32, dctl))
    assert ks >= 0.01
    assert d32 <= max(3 * dctl, RUN_TOL)
