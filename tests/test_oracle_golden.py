"""The oracle restatement against fixtures produced by the reference itself
(tests/golden/make_golden.py).  The restatement follows the reference's
operation order, so agreement is exact."""
import os

import numpy as np
import pytest

import pyoracle as po
import scenarios as sc

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    assert str(g["input_digest"]) == mg.input_digest(name), "synthetic inputs changed"
    fn, kw = mg.CASES[name]
    return g, fn, kw


def oracle_factory(kind, nx, ny, **kw):
    return po.Oracle(kind, nx, ny, **kw)


@pytest.mark.parametrize("name", ["planar_mixed_32", "planar_mixed_32x48", "planar_custom_32",
                                  "fresnel_mixed_32", "poly_mixed_32", "fresnel_wf_mixed_32",
                                  "phase_diverse_series_32", "phase_diverse_parallel_g2_32",
                                  "phase_diverse_align_32", "phase_diverse_minerr_32"])
def test_oracle_matches_golden(name):
    g, fn, kw = load_golden(name)
    res = fn(oracle_factory, **kw)
    for key in res:
        if res[key] is None:
            continue
        assert np.array_equal(np.asarray(res[key]), g[key]), key


@pytest.mark.skipif(not po.reference_available("64"), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", ["planar_mixed_32", "planar_mixed_32x48", "planar_custom_32",
                                  "fresnel_mixed_32", "poly_mixed_32", "fresnel_wf_mixed_32",
                                  "phase_diverse_series_32", "phase_diverse_parallel_g2_32",
                                  "phase_diverse_align_32", "phase_diverse_minerr_32"])
def test_reference_reproduces_golden(name):
    """The committed fixtures are what the reference build here produces
    (make_golden.py's own recipe, run again): the fixtures are reproducible."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    g, fn, kw = load_golden(name)
    res = fn(mg.reference_factory, **kw)
    for key in res:
        if res[key] is None:
            continue
        assert np.array_equal(np.asarray(res[key]), g[key]), key
