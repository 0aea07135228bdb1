"""The file helpers (include/nadia/io.h) and the configuration reader
(include/nadia/Config.h) against the reference's own (NADIA/src/io_cplx.c,
io_dbin.c, io_ppm.c, io_spec.c, Config.c++ compiled into oracle/_ref) -- the
same C entry points (tests/dropin/io_shim.cpp) built over both header sets
write identical bytes and read identical values.  The raw formats are also
checked against numpy's reading of them, which needs no reference.  CPU only."""
import ctypes
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "dropin"))
import build_program  # noqa: E402

D = ctypes.POINTER(ctypes.c_double)


def _bind(path):
    L = ctypes.CDLL(path)
    i, d, s = ctypes.c_int, ctypes.c_double, ctypes.c_char_p
    for name, args in {
        "shim_write_cplx": [s, i, i, D], "shim_read_cplx": [s, i, i, D],
        "shim_write_dbin": [s, i, i, D], "shim_read_dbin": [s, i, i, D],
        "shim_write_ppm": [s, i, i, D, i, d, d],
        "shim_read_ppm": [s, i, D, ctypes.POINTER(i), ctypes.POINTER(i)],
        "shim_write_spec": [s, i, i, D],
        "shim_read_spec": [s, i, D, ctypes.POINTER(i), ctypes.POINTER(i)],
        "shim_config": [s, s, i, ctypes.c_char_p, i],
        "shim_tokenise": [s, ctypes.c_char_p, i],
    }.items():
        getattr(L, name).argtypes = args
        getattr(L, name).restype = i
    L.shim_scale_value.argtypes = [d, d, i, d, i]
    L.shim_scale_value.restype = ctypes.c_uint
    return L


@pytest.fixture(scope="module")
def libs(tmp_path_factory):
    if not os.path.exists(os.path.join(build_program.LIBDIR, "libnadia_b200.so")):
        pytest.skip("libnadia_b200.so not built")
    t = tmp_path_factory.mktemp("io")
    own = _bind(build_program.build_io_shim(str(t / "own_io.so")))
    r = build_program.build_io_shim(str(t / "ref_io.so"), reference=True)
    return own, (_bind(r) if r else None)


def _ref(libs):
    if libs[1] is None:
        pytest.skip("oracle/_ref not built")
    return libs[1]


def _p(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(D)


def _field(nx, ny, seed):
    g = np.random.default_rng(seed)
    return g.standard_normal((nx, ny)) + 1j * g.standard_normal((nx, ny))


def _interleave(c):
    return np.ascontiguousarray(np.stack([c.real, c.imag], -1))


@pytest.mark.parametrize("nx,ny", [(24, 17), (1, 5), (16, 16)])
def test_cplx_layout_and_round_trip(libs, tmp_path, nx, ny):
    own = libs[0]
    c = _field(nx, ny, nx * 100 + ny)
    f = str(tmp_path / "a.cplx").encode()
    assert own.shim_write_cplx(f, nx, ny, _p(_interleave(c))) == 1
    raw = np.fromfile(f.decode(), dtype=np.float64)
    # column-major: element (x, y) at y*nx + x, (re, im) pairs
    assert np.array_equal(raw, _interleave(c.T).ravel())
    got = np.zeros((nx, ny, 2))
    assert own.shim_read_cplx(f, nx, ny, got.ctypes.data_as(D)) == 1
    assert np.array_equal(got[..., 0] + 1j * got[..., 1], c)


@pytest.mark.parametrize("nx,ny", [(24, 17), (16, 16)])
def test_dbin_layout_and_round_trip(libs, tmp_path, nx, ny):
    own = libs[0]
    v = np.random.default_rng(nx + ny).standard_normal((nx, ny))
    f = str(tmp_path / "a.dbin").encode()
    assert own.shim_write_dbin(f, nx, ny, _p(v)) == 1
    assert np.array_equal(np.fromfile(f.decode(), dtype=np.float64), v.T.ravel())
    got = np.zeros((nx, ny))
    assert own.shim_read_dbin(f, nx, ny, got.ctypes.data_as(D)) == 1
    assert np.array_equal(got, v)


def test_short_files_fail(libs, tmp_path):
    own = libs[0]
    f = tmp_path / "short.bin"
    np.zeros(10).tofile(str(f))
    out = np.zeros(64)
    assert own.shim_read_cplx(str(f).encode(), 4, 4, out.ctypes.data_as(D)) == 0
    assert own.shim_read_dbin(str(f).encode(), 4, 4, out.ctypes.data_as(D)) == 0
    assert own.shim_read_dbin(str(tmp_path / "missing").encode(), 4, 4, out.ctypes.data_as(D)) == 0


@pytest.mark.parametrize("nx,ny", [(24, 17), (16, 16)])
def test_binary_formats_match_reference(libs, tmp_path, nx, ny):
    own, ref = libs[0], _ref(libs)
    c = _field(nx, ny, 7)
    for L, name in ((own, "own"), (ref, "ref")):
        L.shim_write_cplx(str(tmp_path / (name + ".cplx")).encode(), nx, ny, _p(_interleave(c)))
        L.shim_write_dbin(str(tmp_path / (name + ".dbin")).encode(), nx, ny, _p(c.real))
    for ext in ("cplx", "dbin"):
        assert (tmp_path / ("own." + ext)).read_bytes() == (tmp_path / ("ref." + ext)).read_bytes()
    a, b = np.zeros((nx, ny, 2)), np.zeros((nx, ny, 2))
    own.shim_read_cplx(str(tmp_path / "ref.cplx").encode(), nx, ny, a.ctypes.data_as(D))
    ref.shim_read_cplx(str(tmp_path / "own.cplx").encode(), nx, ny, b.ctypes.data_as(D))
    assert np.array_equal(a, b)


def _images():
    g = np.random.default_rng(3)
    yield "normal", g.standard_normal((24, 17)), 0, 0.0, 0.0
    yield "positive_log", np.abs(g.standard_normal((24, 17))) * 1e4, 1, 0.0, 0.0
    yield "range", g.standard_normal((16, 9)), 0, -0.5, 0.7
    yield "range_log", np.abs(g.standard_normal((16, 9))), 1, 0.1, 2.0
    yield "constant", np.full((5, 4), 3.25), 0, 0.0, 0.0


@pytest.mark.parametrize("case", list(_images()), ids=lambda c: c[0])
def test_ppm_matches_reference(libs, tmp_path, case):
    own, ref = libs[0], _ref(libs)
    _, v, log, lo, hi = case
    nx, ny = v.shape
    # the comment line carries the file name: write both under the same name
    outs = []
    for L, sub in ((own, "own"), (ref, "ref")):
        d = tmp_path / sub
        d.mkdir()
        cwd = os.getcwd()
        os.chdir(str(d))
        try:
            assert L.shim_write_ppm(b"img.ppm", nx, ny, _p(v), log, lo, hi) == 1
        finally:
            os.chdir(cwd)
        outs.append((d / "img.ppm").read_bytes())
    assert outs[0] == outs[1]
    assert outs[0].startswith(b"P2\n#img.ppm\n")


def test_scale_value_matches_reference(libs):
    own, ref = libs[0], _ref(libs)
    g = np.random.default_rng(5)
    for lo, hi in ((0.0, 1.0), (-3.0, 7.5), (2.0, 2.0), (1e-9, 1e9)):
        for v in np.concatenate([g.uniform(lo - 1, hi + 1, 50), [lo, hi]]):
            for log in (0, 1):
                assert own.shim_scale_value(lo, hi, 65535, v, log) == \
                    ref.shim_scale_value(lo, hi, 65535, v, log)


def test_read_ppm_matches_reference(libs, tmp_path):
    own, ref = libs[0], _ref(libs)
    # tab-separated P2 (the reference's tokeniser splits on tabs only)
    g = np.random.default_rng(9)
    img = g.integers(0, 65536, size=(7, 5))  # (ny, nx) rows of y
    lines = ["P2", "#comment", "5\t7", "65535"] + ["\t".join(str(x) for x in row) for row in img]
    f = tmp_path / "in.ppm"
    f.write_text("\n".join(lines) + "\n")
    res = []
    for L in (own, ref):
        out = np.zeros(64)
        nx, ny = ctypes.c_int(), ctypes.c_int()
        assert L.shim_read_ppm(str(f).encode(), 64, out.ctypes.data_as(D), ctypes.byref(nx),
                               ctypes.byref(ny)) == 1
        res.append(out[:nx.value * ny.value].reshape(nx.value, ny.value))
    assert np.array_equal(res[0], res[1])
    assert np.array_equal(res[0], img.T)
    # P5 is refused by both
    f.write_text("P5\n5 7\n255\n")
    for L in (own, ref):
        assert L.shim_read_ppm(str(f).encode(), 64, np.zeros(64).ctypes.data_as(D),
                               ctypes.byref(ctypes.c_int()), ctypes.byref(ctypes.c_int())) == 0


def test_spec_matches_reference(libs, tmp_path):
    own, ref = libs[0], _ref(libs)
    f = tmp_path / "spec.txt"
    f.write_text("Energy\tF.Density\n1200\t1.336e+15\n1208\t1.439e+15\n1216\t2e+15\n1224.5\t3\n")
    res = []
    for L in (own, ref):
        out = np.zeros(64)
        nx, ny = ctypes.c_int(), ctypes.c_int()
        assert L.shim_read_spec(str(f).encode(), 64, out.ctypes.data_as(D), ctypes.byref(nx),
                                ctypes.byref(ny)) == 1
        res.append(out[:nx.value * ny.value].reshape(nx.value, ny.value))
    assert res[0].shape == (4, 2)
    assert np.array_equal(res[0], res[1])
    v = np.random.default_rng(1).standard_normal((6, 2))
    for L, name in ((own, "own.txt"), (ref, "ref.txt")):
        assert L.shim_write_spec(str(tmp_path / name).encode(), 6, 2, _p(v)) == 1
    assert (tmp_path / "own.txt").read_bytes() == (tmp_path / "ref.txt").read_bytes()


CONFIG = """# a configuration file
output_iterations = 10   # every ten
algorithm = HIO ER  HIO
iterations = 30 10 5
pixels_x = 64
pixels_y=48
beam_wavelength = 4.892e-10
data_file_name  data.dbin extra
spaced_key value_after_space
empty_list =
pixels_x = 128
  indented = 7.5
"""

KEYS = [("output_iterations", "d"), ("output_iterations", "i"), ("algorithm", "S"),
        ("iterations", "I"), ("pixels_x", "i"), ("pixels_y", "i"), ("beam_wavelength", "d"),
        ("data_file_name", "s"), ("spaced_key", "s"), ("empty_list", "S"), ("empty_list", "I"),
        ("indented", "d"), ("missing", "s"), ("missing", "d"), ("missing", "I"),
        ("algorithm", "s"), ("iterations", "i")]


def test_config_matches_reference(libs, tmp_path):
    own, ref = libs[0], _ref(libs)
    f = tmp_path / "c.config"
    f.write_text(CONFIG)
    for key, kind in KEYS:
        got = []
        for L in (own, ref):
            buf = ctypes.create_string_buffer(4096)
            st = L.shim_config(str(f).encode(), key.encode(), ord(kind), buf, 4096)
            got.append((st, buf.value))
        assert got[0] == got[1], (key, kind, got)


def test_config_values(libs, tmp_path):
    own = libs[0]
    f = tmp_path / "c.config"
    f.write_text(CONFIG)

    def q(key, kind):
        buf = ctypes.create_string_buffer(4096)
        st = own.shim_config(str(f).encode(), key.encode(), ord(kind), buf, 4096)
        return st, buf.value.decode()

    assert q("algorithm", "S") == (1, "HIO\nER\nHIO\n")
    assert q("iterations", "I") == (1, "30\n10\n5\n")
    assert q("pixels_x", "i") == (1, "64")  # the first line of a key wins
    assert q("pixels_y", "i") == (1, "48")
    assert q("data_file_name", "s") == (1, "data.dbin")
    assert q("missing", "s") == (0, "")
    assert q("empty_list", "S")[0] == 0
    assert own.shim_config(str(tmp_path / "none").encode(), b"x", ord("s"),
                           ctypes.create_string_buffer(16), 16) == 0


def test_line_tokeniser_matches_reference(libs):
    # io.h's line_tokeniser splits on tabs only (NADIA/include/io.h:289-299)
    own, ref = libs[0], _ref(libs)
    for line in [b"1\t2\t3", b"a b\tc", b"", b"\t", b"x\t\ty\t", b"no tabs here", b"\t\tz"]:
        got = []
        for L in (own, ref):
            buf = ctypes.create_string_buffer(256)
            n = L.shim_tokenise(line, buf, 256)
            got.append((n, buf.value))
        assert got[0] == got[1], (line, got)
