"""Python binding of libnadia_b200 (the C ABI in include/nadia_b200.h).

``Solver`` mirrors the reference's class API (NADIA/include/BaseCDI.h,
PlanarCDI.h, FresnelCDI.h, PolyCDI.h): set_support, set_intensity,
set_beam_stop, set_algorithm, set_relaxation_parameter, initialise_estimate,
iterate, get_error, apply_shrinkwrap, get_transmission, ... with numpy arrays
(complex128 for complex fields, float64 for real ones, shape (nx, ny),
element (x, y) as in the reference's x*ny+y layout).

There is no fallback: if the CUDA library is missing or fails to load, the
import raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "libnadia_b200.so")

ER, BIO, BOO, HIO, DM, SF, ASR, HPR, RAAR, CUSTOM = range(10)
ALGORITHMS = {"ER": ER, "BIO": BIO, "BOO": BOO, "HIO": HIO, "DM": DM, "SF": SF, "ASR": ASR,
              "HPR": HPR, "RAAR": RAAR}
PLANAR, FRESNEL, POLY, FRESNEL_WF = 0, 1, 2, 3
FP64, FP32 = 0, 1
KINDS = {"planar": PLANAR, "fresnel": FRESNEL, "poly": POLY, "fresnel_wf": FRESNEL_WF}

STATUS = {0: "OK", 1: "INVALID", 2: "STATE", 3: "UNSUPPORTED", 4: "CUDA", 5: "NOMEM",
          6: "RANGE"}


class NadiaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (STATUS.get(code, "?"), code, msg))
        self.code = code


_D = ctypes.POINTER(ctypes.c_double)
_F = ctypes.POINTER(ctypes.c_float)
_H = ctypes.c_void_p
_I = ctypes.c_int

class _Request(ctypes.Structure):
    """struct nadia_request (include/nadia_b200.h)."""
    _fields_ = [("kind", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("precision", ctypes.c_int),
                ("intensity", _D), ("support", _D), ("beam_stop", _D),
                ("spectrum", _D), ("nlambda", ctypes.c_int),
                ("white_field", _D),
                ("wavelength", ctypes.c_double), ("focal_detector_length", ctypes.c_double),
                ("focal_sample_length", ctypes.c_double), ("pixel_size", ctypes.c_double),
                ("normalisation", ctypes.c_double), ("fresnel_auto_norm", ctypes.c_int),
                ("algorithm", ctypes.c_int), ("beta", ctypes.c_double),
                ("iterations", ctypes.c_int), ("shrinkwrap_every", ctypes.c_int),
                ("shrinkwrap_sigma", ctypes.c_double), ("shrinkwrap_threshold", ctypes.c_double),
                ("seed", ctypes.c_int)]


_LL = ctypes.c_longlong

_PROTOS = {
    "nadia_last_error": (ctypes.c_char_p, []),
    "nadia_version": (ctypes.c_char_p, []),
    "nadia_planar_create": (_I, [_I, _I, _I, _I, ctypes.POINTER(_H)]),
    "nadia_fresnel_create": (_I, [_I, _I, _I, _D, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double, _I,
                                  ctypes.POINTER(_H)]),
    "nadia_poly_create": (_I, [_I, _I, _I, ctypes.c_double, _I, ctypes.POINTER(_H)]),
    "nadia_fresnel_wf_create": (_I, [_I, _I, _I, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, _I, ctypes.POINTER(_H)]),
    "nadia_fresnel_wf_set_support": (_I, [_H, ctypes.c_double, ctypes.c_double]),
    "nadia_set_transmission_constraint": (_I, [_H, _I, _I, _I, _I, _D, _D, _D]),
    "nadia_set_transmission_custom": (_I, [_H, ctypes.c_void_p, ctypes.c_void_p]),
    "nadia_clear_transmission_constraint": (_I, [_H]),
    "nadia_destroy": (_I, [_H]),
    "nadia_get_size": (_I, [_H, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "nadia_set_support": (_I, [_H, _D, _I]),
    "nadia_set_intensity": (_I, [_H, _D]),
    "nadia_set_beam_stop": (_I, [_H, _D]),
    "nadia_poly_set_spectrum": (_I, [_H, _D, _I]),
    "nadia_poly_set_spectrum_file": (_I, [_H, ctypes.c_char_p]),
    "nadia_read_spec": (_I, [ctypes.c_char_p, _D, _I, ctypes.POINTER(_I)]),
    "nadia_poly_get_padding": (_I, [_H, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "nadia_set_algorithm": (_I, [_H, _I]),
    "nadia_set_custom_algorithm": (_I, [_H, _D]),
    "nadia_set_relaxation_parameter": (_I, [_H, ctypes.c_double]),
    "nadia_get_algorithm_structure": (_I, [_H, _D, ctypes.POINTER(_I)]),
    "nadia_custom_weights": (None, [_D, _D]),
    "nadia_initialise_estimate": (_I, [_H, _I]),
    "nadia_set_exit_surface_wave": (_I, [_H, _D]),
    "nadia_get_exit_surface_wave": (_I, [_H, _D]),
    "nadia_set_exit_surface_wave_f32": (_I, [_H, _F]),
    "nadia_get_exit_surface_wave_f32": (_I, [_H, _F]),
    "nadia_iterate": (_I, [_H, _I]),
    "nadia_get_error": (_I, [_H, _D]),
    "nadia_get_error_history": (_I, [_H, _D, _I]),
    "nadia_apply_shrinkwrap": (_I, [_H, ctypes.c_double, ctypes.c_double]),
    "nadia_get_support": (_I, [_H, _D]),
    "nadia_get_best_result": (_I, [_H, _I, _D, _D]),
    "nadia_reset_best": (_I, [_H]),
    "nadia_get_transmission": (_I, [_H, _D]),
    "nadia_set_transmission": (_I, [_H, _D]),
    "nadia_fresnel_auto_set_norm": (_I, [_H]),
    "nadia_fresnel_set_norm": (_I, [_H, ctypes.c_double]),
    "nadia_fresnel_get_illumination_at_sample": (_I, [_H, _D]),
    "nadia_fresnel_set_experimental_parameters": (_I, [_H, ctypes.c_double, ctypes.c_double,
                                                      ctypes.c_double, ctypes.c_double]),
    "nadia_fresnel_set_normalisation": (_I, [_H, ctypes.c_double]),
    "nadia_propagate_to_detector": (_I, [_H, _D]),
    "nadia_propagate_from_detector": (_I, [_H, _D]),
    "nadia_scale_intensity": (_I, [_H, _D]),
    "nadia_apply_support": (_I, [_H, _D]),
    "nadia_project_intensity": (_I, [_H, _D]),
    "nadia_get_intensity_autocorrelation": (_I, [_H, _D]),
    "nadia_synchronize": (_I, [_H]),
    "nadia_fft2d": (_I, [_D, _I, _I, _I]),
    "nadia_iterate_many": (_I, [ctypes.POINTER(_H), _I, _I]),
    "nadia_get_stream": (_I, [_H, ctypes.POINTER(ctypes.c_void_p)]),
    "nadia_pass_times": (_I, [ctypes.POINTER(_H), _I, _I, _D]),
    "nadia_launch_count": (ctypes.c_longlong, []),
    "nadia_shrinkwrap_noalloc_f32": (_I, [ctypes.c_void_p, ctypes.c_void_p, _I, _I,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_void_p]),
    "nadia_server_create": (_I, [ctypes.c_ulonglong, _I, _I, ctypes.POINTER(_H)]),
    "nadia_server_submit": (_I, [_H, ctypes.POINTER(_Request), ctypes.POINTER(_LL)]),
    "nadia_server_wait": (_I, [_H, _LL, ctypes.c_double, ctypes.POINTER(_I)]),
    "nadia_server_result": (_I, [_H, _LL, _D, _D, _D, _D]),
    "nadia_server_stats": (_I, [_H, ctypes.POINTER(_LL)]),
    "nadia_server_destroy": (_I, [_H]),
    "nadia_estimate_device_bytes": (_I, [_I, _I, _I, _I, _I, _I, _I, _I,
                                         ctypes.POINTER(ctypes.c_ulonglong)]),
    "nadia_device_bytes": (_LL, []),
    "nadia_tuned_tiles": (_I, [_I, _I, _I, _I, ctypes.c_char_p, _I]),
    "nadia_convert_to_fp64": (_I, [_H]),
    "nadia_get_precision": (_I, [_H, ctypes.POINTER(_I)]),
    "nadia_pd_create": (_I, [ctypes.c_double, ctypes.c_double, _I, _I, ctypes.POINTER(_H)]),
    "nadia_pd_destroy": (_I, [_H]),
    "nadia_pd_add_position": (_I, [_H, _H, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    "nadia_pd_remove_positions": (_I, [_H]),
    "nadia_pd_initialise_estimate": (_I, [_H]),
    "nadia_pd_iterate": (_I, [_H, _I]),
    "nadia_pd_set_iterations_per_cycle": (_I, [_H, _I]),
    "nadia_pd_set_feedback_parameter": (_I, [_H, ctypes.c_double]),
    "nadia_pd_set_amplification_factor": (_I, [_H, ctypes.c_double]),
    "nadia_pd_set_probe_scaling": (_I, [_H, _I, ctypes.c_double]),
    "nadia_pd_get_size": (_I, [_H, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "nadia_pd_get_transmission": (_I, [_H, _D]),
    "nadia_pd_set_transmission": (_I, [_H, _I, _I, _D]),
    "nadia_pd_adjust_positions": (_I, [_H, _I, _I, _I, _I, _I, _I, ctypes.c_double]),
    "nadia_pd_get_position": (_I, [_H, _I, _D, _D]),
}

_LIB = None


def load(path=LIB_PATH):
    """Load the CUDA library (raises if it is missing)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(path):
            raise ImportError("libnadia_b200.so not built (run __graft_entry__.build() or "
                              "python nadia-coecxs_b200/build.py): %s" % path)
        lib = ctypes.CDLL(path)
        for name, (res, args) in _PROTOS.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _LIB = lib
    return _LIB


def exported_symbols():
    return sorted(_PROTOS)


def _check(rc):
    if rc != 0:
        raise NadiaError(rc, _LIB.nadia_last_error().decode())


def _ptr(a):
    return a.ctypes.data_as(_D)


def read_spec(path):
    """read_spec (NADIA/src/io_spec.c:61-133): the file's rows of
    (1/energy, weight) as an (n, 2) array.  Needs no GPU."""
    lib = load()
    n = ctypes.c_int()
    _check(lib.nadia_read_spec(path.encode(), None, 0, ctypes.byref(n)))
    out = np.zeros((n.value, 2))
    _check(lib.nadia_read_spec(path.encode(), _ptr(out), n.value, ctypes.byref(n)))
    return out


def custom_weights(m):
    """Weights [PsPf, PfPs, Ps, Pf, I] of set_custom_algorithm(m1..m10) (BaseCDI.c++:245-249)."""
    lib = load()
    m = np.ascontiguousarray(m, dtype=np.float64)
    w = np.zeros(5)
    lib.nadia_custom_weights(_ptr(m), _ptr(w))
    return w


class Solver:
    """One reconstruction on the GPU (PlanarCDI / FresnelCDI / PolyCDI /
    FresnelCDI_WF)."""

    def __init__(self, kind, nx, ny, precision=FP64, n_best=0, white_field=None,
                 wavelength=None, focal_detector_length=None, focal_sample_length=None,
                 pixel_size=None, normalisation=1.0, beta=0.9, zone_focal_length=None):
        self.lib = load()
        self.kind = kind
        self.nx, self.ny = int(nx), int(ny)
        self.precision = precision
        h = _H()
        if kind == "planar":
            _check(self.lib.nadia_planar_create(nx, ny, precision, n_best, ctypes.byref(h)))
        elif kind == "fresnel":
            wf = np.ascontiguousarray(white_field, dtype=np.complex128)
            assert wf.shape == (nx, ny)
            _check(self.lib.nadia_fresnel_create(nx, ny, precision, _ptr(wf), wavelength,
                                                 focal_detector_length, focal_sample_length,
                                                 pixel_size, normalisation, n_best,
                                                 ctypes.byref(h)))
        elif kind == "poly":
            _check(self.lib.nadia_poly_create(nx, ny, precision, beta, n_best, ctypes.byref(h)))
        elif kind == "fresnel_wf":
            _check(self.lib.nadia_fresnel_wf_create(nx, ny, precision, wavelength,
                                                    zone_focal_length, focal_detector_length,
                                                    pixel_size, n_best, ctypes.byref(h)))
        else:
            raise ValueError(kind)
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.nadia_destroy(self.h)
            self.h = None

    def convert_to_fp64(self):
        """Move an FP32 reconstruction to the FP64 form in place."""
        _check(self.lib.nadia_convert_to_fp64(self.h))
        self.precision = FP64

    def get_precision(self):
        p = _I()
        _check(self.lib.nadia_get_precision(self.h, ctypes.byref(p)))
        return p.value

    __del__ = close

    def _real(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == (self.nx, self.ny), a.shape
        return a

    def _cplx(self, a):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        assert a.shape == (self.nx, self.ny), a.shape
        return a

    def set_support(self, s, soften=False):
        _check(self.lib.nadia_set_support(self.h, _ptr(self._real(s)), int(bool(soften))))

    def set_intensity(self, i):
        _check(self.lib.nadia_set_intensity(self.h, _ptr(self._real(i))))

    def set_transmission_constraint(self, enforce_unity=True, charge_flip=True, flip_sign=1,
                                    regions=(), alphas=(), fixed_c=None):
        """BaseCDI::set_complex_constraint with a TransmissionConstraint
        (nadia_set_transmission_constraint)."""
        nr = len(regions)
        reg = np.ascontiguousarray(np.array(regions, dtype=np.float64).reshape(nr, self.nx, self.ny)
                                   if nr else np.zeros(1))
        al = np.ascontiguousarray(np.array(alphas, dtype=np.float64).reshape(-1)
                                  if nr else np.zeros(2))
        fc = None if fixed_c is None else np.ascontiguousarray(fixed_c, dtype=np.float64)
        _check(self.lib.nadia_set_transmission_constraint(
            self.h, int(enforce_unity), int(charge_flip), int(flip_sign), nr, _ptr(reg), _ptr(al),
            _ptr(fc) if fc is not None else None))

    def set_transmission_custom(self, fn):
        """A Python function f(transmission) changing the (nx, ny) complex128
        array in place, called after the built-in constraint steps."""
        if fn is None:
            self._custom = None
            _check(self.lib.nadia_set_transmission_custom(self.h, None, None))
            return
        proto = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                                 ctypes.c_int, ctypes.c_void_p)

        def tramp(p, nx, ny, user):
            a = np.ctypeslib.as_array(p, shape=(nx * ny * 2,)).view(np.complex128)
            fn(a.reshape(nx, ny))

        self._custom = proto(tramp)   # kept alive with the handle
        _check(self.lib.nadia_set_transmission_custom(
            self.h, ctypes.cast(self._custom, ctypes.c_void_p), None))

    def clear_transmission_constraint(self):
        _check(self.lib.nadia_clear_transmission_constraint(self.h))

    def set_wf_support(self, z_diameter, size=1.01):
        """FresnelCDI_WF::set_support(z_diameter, size)."""
        _check(self.lib.nadia_fresnel_wf_set_support(self.h, float(z_diameter), float(size)))

    def set_beam_stop(self, b):
        _check(self.lib.nadia_set_beam_stop(self.h, _ptr(self._real(b))))

    def set_spectrum(self, spec):
        if isinstance(spec, str):
            _check(self.lib.nadia_poly_set_spectrum_file(self.h, spec.encode()))
            return
        spec = np.ascontiguousarray(spec, dtype=np.float64)
        assert spec.ndim == 2 and spec.shape[1] == 2
        _check(self.lib.nadia_poly_set_spectrum(self.h, _ptr(spec), spec.shape[0]))

    def get_padding(self):
        a, b = _I(), _I()
        _check(self.lib.nadia_poly_get_padding(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def set_algorithm(self, alg):
        if isinstance(alg, str):
            alg = ALGORITHMS[alg]
        _check(self.lib.nadia_set_algorithm(self.h, int(alg)))

    def set_custom_algorithm(self, m):
        m = np.ascontiguousarray(m, dtype=np.float64)
        assert m.shape == (10,)
        _check(self.lib.nadia_set_custom_algorithm(self.h, _ptr(m)))

    def set_relaxation_parameter(self, b):
        _check(self.lib.nadia_set_relaxation_parameter(self.h, float(b)))

    def algorithm_structure(self):
        w = np.zeros(5)
        a = _I()
        _check(self.lib.nadia_get_algorithm_structure(self.h, _ptr(w), ctypes.byref(a)))
        return w, a.value

    def initialise_estimate(self, seed=0):
        _check(self.lib.nadia_initialise_estimate(self.h, int(seed)))

    def set_exit_surface_wave(self, e):
        _check(self.lib.nadia_set_exit_surface_wave(self.h, _ptr(self._cplx(e))))

    def get_exit_surface_wave(self):
        out = np.empty((self.nx, self.ny), dtype=np.complex128)
        _check(self.lib.nadia_get_exit_surface_wave(self.h, _ptr(out)))
        return out

    def set_exit_surface_wave_f32(self, e):
        e = np.ascontiguousarray(e, dtype=np.complex64)
        _check(self.lib.nadia_set_exit_surface_wave_f32(self.h, e.ctypes.data_as(_F)))

    def get_exit_surface_wave_f32(self):
        out = np.empty((self.nx, self.ny), dtype=np.complex64)
        _check(self.lib.nadia_get_exit_surface_wave_f32(self.h, out.ctypes.data_as(_F)))
        return out

    def iterate(self, n=1):
        _check(self.lib.nadia_iterate(self.h, int(n)))

    def get_error(self):
        e = ctypes.c_double()
        _check(self.lib.nadia_get_error(self.h, ctypes.byref(e)))
        return e.value

    def get_error_history(self, count):
        out = np.empty(count)
        _check(self.lib.nadia_get_error_history(self.h, _ptr(out), int(count)))
        return out

    def apply_shrinkwrap(self, gauss_width=1.5, threshold=0.1):
        _check(self.lib.nadia_apply_shrinkwrap(self.h, gauss_width, threshold))

    def get_support(self):
        out = np.empty((self.nx, self.ny))
        _check(self.lib.nadia_get_support(self.h, _ptr(out)))
        return out

    def get_best_result(self, index=0):
        e = ctypes.c_double()
        out = np.empty((self.nx, self.ny), dtype=np.complex128)
        rc = self.lib.nadia_get_best_result(self.h, int(index), ctypes.byref(e), _ptr(out))
        if rc == 6:
            return None, None
        _check(rc)
        return e.value, out

    def reset_best(self):
        _check(self.lib.nadia_reset_best(self.h))

    def get_transmission(self):
        out = np.empty((self.nx, self.ny), dtype=np.complex128)
        _check(self.lib.nadia_get_transmission(self.h, _ptr(out)))
        return out

    def set_transmission(self, t):
        _check(self.lib.nadia_set_transmission(self.h, _ptr(self._cplx(t))))

    def auto_set_norm(self):
        _check(self.lib.nadia_fresnel_auto_set_norm(self.h))

    def set_norm(self, n):
        _check(self.lib.nadia_fresnel_set_norm(self.h, float(n)))

    def get_illumination_at_sample(self):
        out = np.empty((self.nx, self.ny), dtype=np.complex128)
        _check(self.lib.nadia_fresnel_get_illumination_at_sample(self.h, _ptr(out)))
        return out

    def _op(self, f, c):
        c = np.array(c, dtype=np.complex128, order="C", copy=True)
        assert c.shape == (self.nx, self.ny)
        _check(f(self.h, _ptr(c)))
        return c

    def propagate_to_detector(self, c):
        return self._op(self.lib.nadia_propagate_to_detector, c)

    def propagate_from_detector(self, c):
        return self._op(self.lib.nadia_propagate_from_detector, c)

    def scale_intensity(self, c):
        return self._op(self.lib.nadia_scale_intensity, c)

    def apply_support(self, c):
        return self._op(self.lib.nadia_apply_support, c)

    def project_intensity(self, c):
        return self._op(self.lib.nadia_project_intensity, c)

    def get_intensity_autocorrelation(self):
        out = np.empty((self.nx, self.ny))
        _check(self.lib.nadia_get_intensity_autocorrelation(self.h, _ptr(out)))
        return out

    def synchronize(self):
        _check(self.lib.nadia_synchronize(self.h))

    def stream(self):
        """The cudaStream_t (as an int) this handle's work is queued on."""
        p = ctypes.c_void_p()
        _check(self.lib.nadia_get_stream(self.h, ctypes.byref(p)))
        return p.value or 0


class PhaseDiverse:
    """PhaseDiverseCDI (NADIA/include/PhaseDiverseCDI.h) on the GPU over FP64
    Solver frames: the reference's method names and defaults."""

    CROSS_CORRELATION, MINIMUM_ERROR = 0, 1

    def __init__(self, beta=1.0, gamma=1.0, parallel=False, granularity=1):
        self.lib = load()
        h = _H()
        _check(self.lib.nadia_pd_create(beta, gamma, int(bool(parallel)), granularity,
                                        ctypes.byref(h)))
        self.h = h
        self.frames = []  # the frames must outlive this object

    def close(self):
        if getattr(self, "h", None):
            self.lib.nadia_pd_destroy(self.h)
            self.h = None

    __del__ = close

    def add_new_position(self, frame, x=0.0, y=0.0, alpha=1.0):
        _check(self.lib.nadia_pd_add_position(self.h, frame.h, x, y, alpha))
        self.frames.append(frame)

    def remove_positions(self):
        _check(self.lib.nadia_pd_remove_positions(self.h))

    def initialise_estimate(self):
        _check(self.lib.nadia_pd_initialise_estimate(self.h))

    def iterate(self, cycles=1):
        _check(self.lib.nadia_pd_iterate(self.h, cycles))

    def set_iterations_per_cycle(self, n):
        _check(self.lib.nadia_pd_set_iterations_per_cycle(self.h, n))

    def set_feedback_parameter(self, beta):
        _check(self.lib.nadia_pd_set_feedback_parameter(self.h, beta))

    def set_amplification_factor(self, gamma):
        _check(self.lib.nadia_pd_set_amplification_factor(self.h, gamma))

    def set_probe_scaling(self, n, alpha):
        _check(self.lib.nadia_pd_set_probe_scaling(self.h, n, alpha))

    def size(self):
        nx, ny = _I(), _I()
        _check(self.lib.nadia_pd_get_size(self.h, ctypes.byref(nx), ctypes.byref(ny)))
        return nx.value, ny.value

    def get_transmission(self):
        nx, ny = self.size()
        out = np.empty((nx, ny), dtype=np.complex128)
        _check(self.lib.nadia_pd_get_transmission(self.h, _ptr(out)))
        return out

    def set_transmission(self, t):
        t = np.ascontiguousarray(t, dtype=np.complex128)
        _check(self.lib.nadia_pd_set_transmission(self.h, t.shape[0], t.shape[1], _ptr(t)))

    def adjust_positions(self, type=0, forward=True, x_min=-50, x_max=50, y_min=-50, y_max=50,
                         step_size=4.0):
        _check(self.lib.nadia_pd_adjust_positions(self.h, type, int(bool(forward)), x_min, x_max,
                                                  y_min, y_max, step_size))

    def _position(self, n):
        x, y = ctypes.c_double(), ctypes.c_double()
        _check(self.lib.nadia_pd_get_position(self.h, n, ctypes.byref(x), ctypes.byref(y)))
        return x.value, y.value

    def get_final_x_position(self, n):
        return self._position(n)[0]

    def get_final_y_position(self, n):
        return self._position(n)[1]


def iterate_many(solvers, iterations):
    """Step several reconstructions together (nadia_iterate_many)."""
    lib = load()
    arr = (_H * len(solvers))(*[s.h for s in solvers])
    _check(lib.nadia_iterate_many(arr, len(solvers), int(iterations)))


def pass_times(solvers, reps=5):
    """Device microseconds of each pass for a batch: (column, second column
    (PolyCDI only, else 0), row)."""
    lib = load()
    arr = (_H * len(solvers))(*[s.h for s in solvers])
    out = np.zeros(3)
    _check(lib.nadia_pass_times(arr, len(solvers), int(reps), _ptr(out)))
    return float(out[0]), float(out[1]), float(out[2])


def launch_count():
    return int(load().nadia_launch_count())


def shrinkwrap_noalloc_f32(esw_ptr, support_ptr, nx, ny, gauss_width=1.5, threshold=0.1,
                           stream=0):
    """nadia_shrinkwrap_noalloc_f32 on device pointers (ints); queued on `stream`."""
    _check(load().nadia_shrinkwrap_noalloc_f32(esw_ptr, support_ptr, int(nx), int(ny),
                                               float(gauss_width), float(threshold), stream))


def estimate_device_bytes(kind, nx, ny, precision=FP32, n_best=0, poly_padding=(0, 0),
                          nlambda=0):
    """Admission charge of one reconstruction (nadia_estimate_device_bytes)."""
    out = ctypes.c_ulonglong()
    k = KINDS[kind] if isinstance(kind, str) else kind
    _check(load().nadia_estimate_device_bytes(k, nx, ny, precision, n_best, poly_padding[0],
                                              poly_padding[1], nlambda, ctypes.byref(out)))
    return int(out.value)


def device_bytes():
    """Device bytes the library's reconstructions hold now."""
    return int(load().nadia_device_bytes())


class Server:
    """The request loop of nadia_server_* : submit patterns at any time,
    collect each reconstruction when it is done."""

    STATS = ("queued", "active", "completed", "failed", "bytes", "peak_bytes", "steps",
             "admitted", "us_step", "us_idle", "us_prepare", "us_readback")

    def __init__(self, budget_bytes, max_active=64, chunk=25):
        self.lib = load()
        self.h = _H()
        _check(self.lib.nadia_server_create(int(budget_bytes), int(max_active), int(chunk),
                                            ctypes.byref(self.h)))
        self.sizes = {}

    def close(self):
        if self.h:
            self.lib.nadia_server_destroy(self.h)
            self.h = _H()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, kind, intensity, support, precision=FP32, beam_stop=None, spectrum=None,
               white_field=None, wavelength=0.0, focal_detector_length=0.0,
               focal_sample_length=0.0, pixel_size=0.0, normalisation=1.0,
               auto_norm=False, algorithm="HIO", beta=0.9, iterations=500,
               shrinkwrap_every=0, shrinkwrap_sigma=1.5, shrinkwrap_threshold=0.1, seed=0):
        k = KINDS[kind] if isinstance(kind, str) else kind
        intensity = np.ascontiguousarray(intensity, dtype=np.float64)
        nx, ny = intensity.shape
        support = np.ascontiguousarray(support, dtype=np.float64)
        assert support.shape == (nx, ny)
        keep = [intensity, support]
        r = _Request()
        r.kind, r.nx, r.ny, r.precision = k, nx, ny, precision
        r.intensity, r.support = _ptr(intensity), _ptr(support)
        if beam_stop is not None:
            b = np.ascontiguousarray(beam_stop, dtype=np.float64)
            keep.append(b)
            r.beam_stop = _ptr(b)
        if spectrum is not None:
            sp = np.ascontiguousarray(spectrum, dtype=np.float64)
            keep.append(sp)
            r.spectrum, r.nlambda = _ptr(sp), sp.shape[0]
        if white_field is not None:
            w = np.ascontiguousarray(white_field, dtype=np.complex128)
            keep.append(w)
            r.white_field = w.ctypes.data_as(_D)
        r.wavelength, r.focal_detector_length = wavelength, focal_detector_length
        r.focal_sample_length, r.pixel_size = focal_sample_length, pixel_size
        r.normalisation, r.fresnel_auto_norm = normalisation, int(bool(auto_norm))
        r.algorithm = ALGORITHMS[algorithm] if isinstance(algorithm, str) else algorithm
        r.beta, r.iterations, r.shrinkwrap_every = beta, iterations, shrinkwrap_every
        r.shrinkwrap_sigma, r.shrinkwrap_threshold, r.seed = (shrinkwrap_sigma,
                                                              shrinkwrap_threshold, seed)
        rid = _LL()
        _check(self.lib.nadia_server_submit(self.h, ctypes.byref(r), ctypes.byref(rid)))
        self.sizes[rid.value] = (nx, ny)
        return rid.value

    def wait(self, rid, timeout=-1.0):
        done = _I()
        _check(self.lib.nadia_server_wait(self.h, rid, float(timeout), ctypes.byref(done)))
        return bool(done.value)

    def result(self, rid):
        """(esw, support, final_error, times) of a finished request; times =
        (queued, on the device, arrival to result) in seconds."""
        nx, ny = self.sizes.pop(rid)
        esw = np.empty((nx, ny), dtype=np.complex128)
        sup = np.empty((nx, ny))
        err = np.zeros(1)
        t = np.zeros(3)
        _check(self.lib.nadia_server_result(self.h, rid, esw.ctypes.data_as(_D), _ptr(sup),
                                            _ptr(err), _ptr(t)))
        return esw, sup, float(err[0]), tuple(t)

    def stats(self):
        out = (_LL * 12)()
        _check(self.lib.nadia_server_stats(self.h, out))
        return dict(zip(self.STATS, list(out)))


def tuned_tiles(nx, ny, fresnel=False, batched=True):
    """The autotuner's column- and row-pass variants for an FP32 grid."""
    buf = ctypes.create_string_buffer(512)
    _check(load().nadia_tuned_tiles(int(nx), int(ny), int(bool(fresnel)), int(bool(batched)),
                                    buf, 512))
    return buf.value.decode()
