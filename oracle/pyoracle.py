"""ctypes wrappers for the oracle libraries -- TEST INFRASTRUCTURE.

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module.

``Oracle``     drives oracle/liboracle.so (the C restatement, always built).
``Reference``  drives oracle/_ref/libnadia_ref*.so (the reference's own sources
               compiled against the FFTW shim), when that directory was built.
Both expose the same methods, named after the reference API
(NADIA/include/BaseCDI.h, PlanarCDI.h, FresnelCDI.h, PolyCDI.h).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_D = ctypes.POINTER(ctypes.c_double)
_V = ctypes.c_void_p


def _ptr(a):
    return a.ctypes.data_as(_D)


def _cplx_in(a, nx, ny):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    assert a.shape == (nx, ny), a.shape
    return a


def _real_in(a, nx, ny):
    a = np.ascontiguousarray(a, dtype=np.float64)
    assert a.shape == (nx, ny), a.shape
    return a


_PROTOS = {
    "planar_create": (_V, [ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "fresnel_create": (_V, [ctypes.c_int, ctypes.c_int, _D, ctypes.c_double, ctypes.c_double,
                            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]),
    "poly_create": (_V, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int]),
    "fresnel_wf_create": (_V, [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                               ctypes.c_double, ctypes.c_double, ctypes.c_int]),
    "fresnel_wf_set_support": (None, [_V, ctypes.c_double, ctypes.c_double]),
    "set_transmission_constraint": (None, [_V, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, _D, _D, _D]),
    "destroy": (None, [_V]),
    "set_support": (None, [_V, _D, ctypes.c_int]),
    "set_intensity": (None, [_V, _D]),
    "set_beam_stop": (None, [_V, _D]),
    "set_algorithm": (None, [_V, ctypes.c_int]),
    "set_custom_algorithm": (None, [_V, _D]),
    "set_relaxation_parameter": (None, [_V, ctypes.c_double]),
    "initialise_estimate": (None, [_V, ctypes.c_int]),
    "set_esw": (None, [_V, _D]),
    "get_esw": (None, [_V, _D]),
    "iterate": (None, [_V]),
    "get_error": (ctypes.c_double, [_V]),
    "apply_shrinkwrap": (None, [_V, ctypes.c_double, ctypes.c_double]),
    "get_support": (None, [_V, _D]),
    "get_transmission": (None, [_V, _D]),
    "set_transmission": (None, [_V, _D]),
    "get_illumination_at_sample": (None, [_V, _D]),
    "fresnel_auto_set_norm": (None, [_V]),
    "fresnel_set_norm": (None, [_V, ctypes.c_double]),
    "poly_set_spectrum": (None, [_V, _D, ctypes.c_int]),
    "get_best_result": (ctypes.c_int, [_V, ctypes.c_int, _D, _D]),
    "reset_best": (None, [_V]),
    "propagate_to_detector": (None, [_V, _D]),
    "propagate_from_detector": (None, [_V, _D]),
    "scale_intensity": (None, [_V, _D]),
    "apply_support": (None, [_V, _D]),
    "project_intensity": (None, [_V, _D]),
    "get_intensity_autocorrelation": (None, [_V, _D]),
}


class _Lib:
    def __init__(self, path, prefix):
        self.lib = ctypes.CDLL(path)
        self.prefix = prefix
        for name, (res, args) in _PROTOS.items():
            f = getattr(self.lib, prefix + name)
            f.restype = res
            f.argtypes = args
            setattr(self, name, f)


def oracle_lib_path():
    return os.path.join(HERE, "liboracle.so")


_ORACLE = None
_REFS = {}


def oracle_lib():
    global _ORACLE
    if _ORACLE is None:
        path = oracle_lib_path()
        if not os.path.exists(path):
            import importlib.util
            spec = importlib.util.spec_from_file_location(
                "build_oracle", os.path.join(HERE, "build_oracle.py"))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build_oracle()
        _ORACLE = _Lib(path, "orc_")
        _ORACLE.lib.orc_fft2d.argtypes = [_D, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _ORACLE.lib.orc_fft2d.restype = ctypes.c_int
        _ORACLE.lib.orc_read_spec.argtypes = [ctypes.c_char_p, _D, ctypes.c_int]
        _ORACLE.lib.orc_read_spec.restype = ctypes.c_int
        _ORACLE.lib.orc_padding.argtypes = [_V, ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)]
    return _ORACLE


def reference_available(variant="64"):
    return os.path.exists(os.path.join(REF_DIR, "libnadia_ref%s.so" % variant))


def reference_lib(variant="64"):
    """variant: '64' (parity build), '64_fast' or '32_fast' (timing builds)."""
    if variant not in _REFS:
        _REFS[variant] = _Lib(os.path.join(REF_DIR, "libnadia_ref%s.so" % variant), "ref_")
    return _REFS[variant]


def canon_fft2d(a, forward=True):
    """The oracle's canonical unnormalised 2-D DFT of a complex array."""
    a = np.array(a, dtype=np.complex128, order="C", copy=True)
    rc = oracle_lib().lib.orc_fft2d(_ptr(a), a.shape[0], a.shape[1], 1 if forward else 0)
    if rc != 0:
        raise ValueError("unsupported FFT size %s" % (a.shape,))
    return a


def read_spec(path, capacity=4096):
    out = np.zeros((capacity, 2), dtype=np.float64)
    n = oracle_lib().lib.orc_read_spec(path.encode(), _ptr(out), capacity)
    if n < 0:
        raise IOError(path)
    return out[:n].copy()


class _Solver:
    """One reconstruction (PlanarCDI / FresnelCDI / PolyCDI / FresnelCDI_WF) on a
    CPU library."""

    def __init__(self, lib, kind, nx, ny, n_best=0, white_field=None, wavelength=None,
                 focal_detector_length=None, focal_sample_length=None, pixel_size=None,
                 normalisation=1.0, beta=0.9, zone_focal_length=None):
        self.L = lib
        self.kind = kind
        self.nx, self.ny = nx, ny
        if kind == "planar":
            self.h = lib.planar_create(nx, ny, n_best)
        elif kind == "fresnel":
            wf = _cplx_in(white_field, nx, ny)
            self.h = lib.fresnel_create(nx, ny, _ptr(wf), wavelength, focal_detector_length,
                                        focal_sample_length, pixel_size, normalisation, n_best)
        elif kind == "poly":
            self.h = lib.poly_create(nx, ny, beta, n_best)
        elif kind == "fresnel_wf":
            self.h = lib.fresnel_wf_create(nx, ny, wavelength, zone_focal_length,
                                           focal_detector_length, pixel_size, n_best)
        else:
            raise ValueError(kind)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.destroy(self.h)
            self.h = None

    def set_support(self, s, soften=False):
        s = _real_in(s, self.nx, self.ny)
        self.L.set_support(self.h, _ptr(s), int(bool(soften)))

    def set_intensity(self, i):
        i = _real_in(i, self.nx, self.ny)
        self.L.set_intensity(self.h, _ptr(i))

    def set_beam_stop(self, b):
        b = _real_in(b, self.nx, self.ny)
        self.L.set_beam_stop(self.h, _ptr(b))

    def set_algorithm(self, alg):
        self.L.set_algorithm(self.h, int(alg))

    def set_custom_algorithm(self, m):
        m = np.ascontiguousarray(m, dtype=np.float64)
        assert m.shape == (10,)
        self.L.set_custom_algorithm(self.h, _ptr(m))

    def set_relaxation_parameter(self, b):
        self.L.set_relaxation_parameter(self.h, float(b))

    def initialise_estimate(self, seed=0):
        self.L.initialise_estimate(self.h, int(seed))

    def set_exit_surface_wave(self, e):
        e = _cplx_in(e, self.nx, self.ny)
        self.L.set_esw(self.h, _ptr(e))

    def get_exit_surface_wave(self):
        out = np.empty((self.nx, self.ny), dtype=np.complex128)
        self.L.get_esw(self.h, _ptr(out))
        return out

    def iterate(self, n=1):
        for _ in range(n):
            self.L.iterate(self.h)

    def get_error(self):
        return self.L.get_error(self.h)

    def apply_shrinkwrap(self, gauss_width=1.5, threshold=0.1):
        self.L.apply_shrinkwrap(self.h, gauss_width, threshold)

    def get_support(self):
        out = np.empty((self.nx, self.ny), dtype=np.float64)
        self.L.get_support(self.h, _ptr(out))
        return out

    def get_transmission(self):
        out = np.empty((self.nx, self.ny), dtype=np.complex128)
        self.L.get_transmission(self.h, _ptr(out))
        return out

    def set_transmission(self, t):
        t = _cplx_in(t, self.nx, self.ny)
        self.L.set_transmission(self.h, _ptr(t))

    def get_illumination_at_sample(self):
        out = np.zeros((self.nx, self.ny), dtype=np.complex128)
        self.L.get_illumination_at_sample(self.h, _ptr(out))
        return out

    def set_wf_support(self, z_diameter, size=1.01):
        """FresnelCDI_WF::set_support(z_diameter, size)."""
        self.L.fresnel_wf_set_support(self.h, z_diameter, size)

    def set_transmission_constraint(self, enforce_unity=True, charge_flip=True, flip_sign=1,
                                    regions=(), alphas=(), fixed_c=None):
        """BaseCDI::set_complex_constraint with a TransmissionConstraint: the
        unit-magnitude and charge-flipping switches and ComplexConstraint
        regions (masks, (alpha1, alpha2) each, optional fixed c; NaN = free)."""
        nr = len(regions)
        reg = np.ascontiguousarray(np.array(regions, dtype=np.float64).reshape(nr, self.nx, self.ny)
                                   if nr else np.zeros(1))
        al = np.ascontiguousarray(np.array(alphas, dtype=np.float64).reshape(-1)
                                  if nr else np.zeros(2))
        fc = None if fixed_c is None else np.ascontiguousarray(fixed_c, dtype=np.float64)
        self.L.set_transmission_constraint(self.h, int(enforce_unity), int(charge_flip),
                                           int(flip_sign), nr, _ptr(reg), _ptr(al),
                                           _ptr(fc) if fc is not None else None)

    def set_transmission_custom(self, fn):
        """Oracle only: a Python function changing the transmission in place."""
        proto = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                 ctypes.c_int, ctypes.c_void_p)

        def tramp(p, nx, ny, user):
            a = np.ctypeslib.as_array(p, shape=(nx * ny * 2,)).view(np.complex128)
            fn(a.reshape(nx, ny))

        self._custom = proto(tramp)
        f = self.L.lib.orc_set_transmission_custom
        f.argtypes = [_V, ctypes.c_void_p, ctypes.c_void_p]
        f.restype = None
        f(self.h, ctypes.cast(self._custom, ctypes.c_void_p), None)

    def auto_set_norm(self):
        self.L.fresnel_auto_set_norm(self.h)

    def set_norm(self, n):
        self.L.fresnel_set_norm(self.h, float(n))

    def set_spectrum(self, spec):
        spec = np.ascontiguousarray(spec, dtype=np.float64)
        assert spec.ndim == 2 and spec.shape[1] == 2
        self.L.poly_set_spectrum(self.h, _ptr(spec), spec.shape[0])

    def get_best_result(self, index=0):
        err = ctypes.c_double(0)
        out = np.empty((self.nx, self.ny), dtype=np.complex128)
        ok = self.L.get_best_result(self.h, index, ctypes.byref(err), _ptr(out))
        return (err.value, out) if ok else (None, None)

    def reset_best(self):
        self.L.reset_best(self.h)

    def _op(self, f, c):
        c = np.array(c, dtype=np.complex128, order="C", copy=True)
        assert c.shape == (self.nx, self.ny)
        f(self.h, _ptr(c))
        return c

    def propagate_to_detector(self, c):
        return self._op(self.L.propagate_to_detector, c)

    def propagate_from_detector(self, c):
        return self._op(self.L.propagate_from_detector, c)

    def scale_intensity(self, c):
        return self._op(self.L.scale_intensity, c)

    def apply_support(self, c):
        return self._op(self.L.apply_support, c)

    def project_intensity(self, c):
        return self._op(self.L.project_intensity, c)

    def get_intensity_autocorrelation(self):
        out = np.empty((self.nx, self.ny), dtype=np.float64)
        self.L.get_intensity_autocorrelation(self.h, _ptr(out))
        return out


def Oracle(kind, nx, ny, **kw):
    return _Solver(oracle_lib(), kind, nx, ny, **kw)


def Reference(kind, nx, ny, variant="64", **kw):
    return _Solver(reference_lib(variant), kind, nx, ny, **kw)


_PD_PROTOS = {
    "pd_create": (_V, [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int]),
    "pd_destroy": (None, [_V]),
    "pd_add_position": (None, [_V, _V, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    "pd_remove_positions": (None, [_V]),
    "pd_initialise_estimate": (None, [_V]),
    "pd_iterate": (None, [_V]),
    "pd_set_iterations_per_cycle": (None, [_V, ctypes.c_int]),
    "pd_set_feedback_parameter": (None, [_V, ctypes.c_double]),
    "pd_set_amplification_factor": (None, [_V, ctypes.c_double]),
    "pd_set_probe_scaling": (None, [_V, ctypes.c_int, ctypes.c_double]),
    "pd_get_size": (None, [_V, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "pd_get_transmission": (None, [_V, _D]),
    "pd_set_transmission": (None, [_V, ctypes.c_int, ctypes.c_int, _D]),
    "pd_adjust_positions": (None, [_V, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_double]),
    "pd_get_x": (ctypes.c_double, [_V, ctypes.c_int]),
    "pd_get_y": (ctypes.c_double, [_V, ctypes.c_int]),
}


class _PhaseDiverse:
    """PhaseDiverseCDI (NADIA/include/PhaseDiverseCDI.h) over frames made by
    the same library's Oracle / Reference factory."""

    CROSS_CORRELATION, MINIMUM_ERROR = 0, 1

    def __init__(self, L, beta=1.0, gamma=1.0, parallel=False, granularity=1):
        self.L = L
        self.f = {}
        for name, (res, args) in _PD_PROTOS.items():
            fn = getattr(L.lib, L.prefix + name)
            fn.restype = res
            fn.argtypes = args
            self.f[name] = fn
        self.h = self.f["pd_create"](beta, gamma, int(bool(parallel)), granularity)
        self.frames = []

    def __del__(self):
        if getattr(self, "h", None):
            self.f["pd_destroy"](self.h)
            self.h = None

    def add_new_position(self, frame, x=0.0, y=0.0, alpha=1.0):
        assert frame.L is self.L
        self.frames.append(frame)
        self.f["pd_add_position"](self.h, frame.h, x, y, alpha)

    def remove_positions(self):
        self.f["pd_remove_positions"](self.h)

    def initialise_estimate(self):
        self.f["pd_initialise_estimate"](self.h)

    def iterate(self):
        self.f["pd_iterate"](self.h)

    def set_iterations_per_cycle(self, n):
        self.f["pd_set_iterations_per_cycle"](self.h, n)

    def set_feedback_parameter(self, b):
        self.f["pd_set_feedback_parameter"](self.h, b)

    def set_amplification_factor(self, g):
        self.f["pd_set_amplification_factor"](self.h, g)

    def set_probe_scaling(self, n, alpha):
        self.f["pd_set_probe_scaling"](self.h, n, alpha)

    def size(self):
        nx, ny = ctypes.c_int(), ctypes.c_int()
        self.f["pd_get_size"](self.h, ctypes.byref(nx), ctypes.byref(ny))
        return nx.value, ny.value

    def get_transmission(self):
        nx, ny = self.size()
        out = np.empty((nx, ny), dtype=np.complex128)
        self.f["pd_get_transmission"](self.h, _ptr(out))
        return out

    def set_transmission(self, t):
        t = np.ascontiguousarray(t, dtype=np.complex128)
        self.f["pd_set_transmission"](self.h, t.shape[0], t.shape[1], _ptr(t))

    def adjust_positions(self, type=0, forward=True, x_min=-50, x_max=50, y_min=-50, y_max=50,
                         step_size=4.0):
        self.f["pd_adjust_positions"](self.h, type, int(bool(forward)), x_min, x_max, y_min,
                                      y_max, step_size)

    def get_final_x_position(self, n):
        return self.f["pd_get_x"](self.h, n)

    def get_final_y_position(self, n):
        return self.f["pd_get_y"](self.h, n)


def OraclePD(**kw):
    return _PhaseDiverse(oracle_lib(), **kw)


def ReferencePD(variant="64", **kw):
    return _PhaseDiverse(reference_lib(variant), **kw)
