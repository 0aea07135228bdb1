"""The C-ABI library: it loads, and exports every entry point that
include/nadia_b200.h declares (no GPU needed)."""
import os
import re

import numpy as np

import pynadia

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "nadia_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(nadia_[a-z0-9_]+)\s*\(", txt)))


def test_library_loads_and_exports_everything():
    lib = pynadia.load()
    names = declared_symbols()
    assert len(names) >= 40
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(pynadia.exported_symbols())


def test_version_string():
    assert b"sm_100a" in pynadia.load().nadia_version()


def test_custom_weights_host_only():
    # BaseCDI.c++:245-249; HIO = set_custom_algorithm(0,beta,1,0,...)
    w = pynadia.custom_weights([0, 0.9, 1, 0, 0, 0, 0, 0, 0, 0])
    assert np.allclose(w, [1.9, 0, -1, -0.9, 0])
    w = pynadia.custom_weights([0, 1, 0.8, 0, 0, 0, 0, 0, 0.2, 0])
    assert np.allclose(w, [1.8, 0, -0.8, -0.8, -0.2])


def test_read_spec_host_only(tmp_path):
    import pyoracle
    p = tmp_path / "spec.txt"
    p.write_text("Energy\tF.Density\n1200\t1.336e+15\n1208\t1.439e+15\n1216\t2e+15\n")
    got = pynadia.read_spec(str(p))
    assert np.array_equal(got, pyoracle.read_spec(str(p)))
    assert got.shape == (3, 2)
    import pytest
    with pytest.raises(pynadia.NadiaError):
        pynadia.read_spec(str(tmp_path / "missing.txt"))
