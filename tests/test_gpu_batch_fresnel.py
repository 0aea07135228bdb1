"""Batching FresnelCDI reconstructions of uneven sizes (grids drawn from
{512, 768, 1024, 1536, 2048}^2, disk objects of radius 30% of the grid, own
seeds, HIO) in one nadia_iterate_many call: each member ends exactly where it
ends when stepped alone through the same entry point (tolerance: bit for bit),
with one launch per size and pass or one launch per pass over every size,
and the library reports the tiles it runs for every size."""
import numpy as np
import pytest

import pynadia
from pynadia import synth

pytestmark = pytest.mark.gpu

SIZES = (512, 768, 1024, 1536, 2048)


def make(n, seed):
    f = synth.FresnelCase(n, seed=seed)
    s = pynadia.Solver("fresnel", n, n, precision=pynadia.FP32, white_field=f.white_field,
                       wavelength=f.wavelength, focal_detector_length=f.zfd,
                       focal_sample_length=f.zfs, pixel_size=f.pixel)
    s.set_support(f.support)
    s.set_intensity(f.intensity)
    s.auto_set_norm()
    s.initialise_estimate(seed)
    s.set_relaxation_parameter(0.9)
    s.set_algorithm("HIO")
    return s


@pytest.mark.parametrize("mixed", ["0", "1"], ids=["per-size launches", "one launch per pass"])
def test_uneven_sizes_batch_equals_alone(mixed, monkeypatch):
    # NADIA_MIXED=1: one launch per pass over a work list of every size
    monkeypatch.setenv("NADIA_MIXED", mixed)
    rng = np.random.default_rng(4)
    sizes = [int(x) for x in rng.choice(SIZES, 7)] + [512]
    batch = [make(n, 10 + i) for i, n in enumerate(sizes)]
    alone = [make(n, 10 + i) for i, n in enumerate(sizes)]
    pynadia.iterate_many(batch, 20)
    for s in alone:
        pynadia.iterate_many([s], 20)
    for s in batch + alone:
        s.apply_shrinkwrap(2.0, 0.1)
    pynadia.iterate_many(batch, 17)
    for s in alone:
        pynadia.iterate_many([s], 17)
    for a, b in zip(alone, batch):
        assert np.array_equal(a.get_error_history(37), b.get_error_history(37))
        assert np.array_equal(a.get_exit_surface_wave(), b.get_exit_surface_wave())
        assert np.array_equal(a.get_transmission(), b.get_transmission())
    for n in sorted(set(sizes)):
        desc = pynadia.tuned_tiles(n, n, fresnel=True, batched=True)
        assert "column pass: n=%d" % n in desc and "row pass: n=%d" % n in desc
