"""Seeded synthetic diffraction data for PlanarCDI, FresnelCDI and PolyCDI.

The reference ships no usable test data (its example images need libtiff and
several are missing), so the benchmarks and parity tests run on synthetic
objects with the shapes and value distributions of the benchmark workloads:

* object: complex transmission inside a centred disk of radius R; amplitude
  uniform in [0.5, 1]; phase uniform in [-pi/2, pi/2], Gaussian-smoothed with
  sigma px (periodic boundary); zero outside the disk;
* Planar intensity: |F|^2 with F the centred, unitary transform that
  PlanarCDI::propagate_to_detector applies (NADIA/src/PlanarCDI.c++:65-68:
  forward FFT, quadrant swap, 1/sqrt(nx*ny)), scaled to a photon total and
  Poisson-sampled;
* Fresnel: a white field W (smooth disk footprint with a gentle quadratic
  phase -- our reading of a defocused pinhole image), the sample-plane
  illumination L = propagate_from_detector(W) and the recorded intensity
  |propagate_to_detector((T-1) L) + W|^2 (FresnelCDI.c++:217-250, 253-283);
* Poly: a Gaussian spectrum of lines listed longest wavelength first, and
  the polychromatic intensity sum_l w_l |Psi(lf*(i-n/2)+n/2, ...)|^2 of
  PolyCDI::expand_wl (NADIA/src/PolyCDI.c++:296-334);
* FresnelCDI_WF: a zone-plate-plane field (a disk with a smooth phase
  aberration) carried to the detector by FresnelCDI_WF::propagate_to_detector
  (NADIA/src/FresnelCDI_WF.c++:176-182), whose intensity is the white-field
  measurement.

Random numbers come from numpy's Philox counter-based generator (Philox4x64-10,
Salmon et al. SC'11) and its Poisson sampler (PTRS for large means); every
array is generated on the host once and the same bytes feed the oracle and
the GPU.
"""
import math

import numpy as np
from scipy.ndimage import gaussian_filter


def rng(seed):
    return np.random.Generator(np.random.Philox(int(seed)))


def centred_unitary_fft(x):
    """PlanarCDI::propagate_to_detector for even sizes: fftshift(fft2(x))/sqrt(N)."""
    nx, ny = x.shape
    return np.fft.fftshift(np.fft.fft2(x)) / math.sqrt(nx * ny)


def disk_mask(nx, ny, radius):
    i = np.arange(nx)[:, None] - nx / 2.0
    j = np.arange(ny)[None, :] - ny / 2.0
    return (i * i + j * j) <= radius * radius


def disk_object(nx, ny, radius, sigma, seed):
    g = rng(seed)
    amp = g.uniform(0.5, 1.0, (nx, ny))
    ph = g.uniform(-np.pi / 2, np.pi / 2, (nx, ny))
    if sigma > 0:
        ph = gaussian_filter(ph, sigma, mode="wrap")
    obj = amp * np.exp(1j * ph)
    obj[~disk_mask(nx, ny, radius)] = 0
    return obj


def poisson_scale(I, photons, seed):
    I = I * (photons / I.sum())
    return rng(seed + 7919).poisson(I).astype(np.float64)


def square_support(nx, ny, side):
    s = np.zeros((nx, ny))
    x0, y0 = nx // 2 - side // 2, ny // 2 - side // 2
    s[x0:x0 + side, y0:y0 + side] = 1.0
    return s


def centre_beam_stop(nx, ny, side):
    """Mask with 0 = unmeasured over a centred side x side block (BaseCDI.c++:112-116,173)."""
    b = np.ones((nx, ny))
    if side > 0:
        x0, y0 = nx // 2 - side // 2, ny // 2 - side // 2
        b[x0:x0 + side, y0:y0 + side] = 0.0
    return b


class PlanarCase:
    """A PlanarCDI problem: object, intensity, initial support, optional beam stop."""

    def __init__(self, n, radius, sigma, photons, seed, support_side=None, beam_stop=0, ny=None):
        ny = ny or n
        self.nx, self.ny = n, ny
        self.obj = disk_object(n, ny, radius, sigma, seed)
        I = np.abs(centred_unitary_fft(self.obj)) ** 2
        self.intensity = poisson_scale(I, photons, seed) if photons else I
        side = support_side or int(2.5 * radius)
        self.support = square_support(n, ny, side)
        self.beam_stop = centre_beam_stop(n, ny, beam_stop) if beam_stop else None


def random_phase_start(intensity, support, seed):
    """The random-phase start estimate of the PlanarCDI workloads: inside the
    support (> 0) a seeded phase uniform in [-pi, pi) with the constant
    amplitude sqrt(sum(I) / pixels in the support), so that the estimate
    carries the measured total intensity (the planar propagators are
    unitary); zero outside the support.  Complex128, shape of `intensity`."""
    inside = np.asarray(support) > 0
    amp = math.sqrt(float(np.sum(intensity)) / max(int(inside.sum()), 1))
    ph = rng(seed).uniform(-math.pi, math.pi, np.shape(intensity))
    return np.where(inside, amp * np.exp(1j * ph), 0.0 + 0.0j)


def planar_case(cfg):
    """Named workloads: 'c1' (256^2), 'c2' (1024^2), 'c3' (2048^2) and small 'tN' tests."""
    if cfg == "c1":
        return PlanarCase(256, 40, 2, 1e8, seed=1, support_side=100)
    if cfg == "c2":
        return PlanarCase(1024, 160, 2, 1e8, seed=2, support_side=400)
    if cfg == "c3":
        return PlanarCase(2048, 320, 4, 1e9, seed=3, support_side=800, beam_stop=8)
    raise ValueError(cfg)


# ------------------------------------------------------------------ Fresnel

def fresnel_factor(nx, ny, wavelength, zfd, zfs, pixel):
    """The quadratic-phase coefficient of FresnelCDI.c++:67-87 on the full grid,
    evaluated at the folded indices of multiply_factors (FresnelCDI.c++:113-117)."""
    x_mid, y_mid = (nx - 1) / 2.0, (ny - 1) / 2.0
    zsd = zfd - zfs
    factor = pixel * pixel * math.pi / wavelength * ((1 / zfd) - (1 / zsd))
    i = np.arange(nx)
    j = np.arange(ny)
    i_ = np.trunc(x_mid - np.abs(x_mid - i)).astype(int)
    j_ = np.trunc(y_mid - np.abs(y_mid - j)).astype(int)
    a = (x_mid - i_)[:, None]
    b = (y_mid - j_)[None, :]
    phi = factor * (a * a + b * b)
    return np.cos(phi) + 1j * np.sin(phi)


def fresnel_to_detector(x, coef):
    """FresnelCDI::propagate_to_detector: swap+scale, FFT, multiply by conj(coef)."""
    nx, ny = x.shape
    y = np.fft.fft2(np.fft.fftshift(x) / math.sqrt(nx * ny))
    return y * np.conj(coef)


def fresnel_from_detector(x, coef):
    """FresnelCDI::propagate_from_detector: multiply by coef, inverse FFT, swap+scale."""
    nx, ny = x.shape
    y = np.fft.ifft2(x * coef) * (nx * ny)
    return np.fft.fftshift(y) / math.sqrt(nx * ny)


class FresnelCase:
    """A FresnelCDI problem (8 keV, zfs 1 mm, zfd 1 m, 13.5 um pixels by default)."""

    HC_KEV_M = 1.23984198e-9  # h*c in keV*m

    def __init__(self, n, seed, energy_kev=8.0, zfs=1e-3, zfd=1.0, pixel=13.5e-6,
                 radius_frac=0.3, footprint_frac=0.42, photons=None, ny=None):
        ny = ny or n
        self.nx, self.ny = n, ny
        self.wavelength = self.HC_KEV_M / energy_kev
        self.zfd, self.zfs, self.pixel = zfd, zfs, pixel
        # white field at the detector: defocused pinhole image, a disk footprint
        # with a soft edge and a gentle quadratic phase (max gradient pi/8 per pixel)
        i = np.arange(n)[:, None] - n / 2.0
        j = np.arange(ny)[None, :] - ny / 2.0
        r2 = i * i + j * j
        rf = footprint_frac * min(n, ny)
        amp = gaussian_filter((r2 <= rf * rf).astype(float), 2.0)
        alpha = (math.pi / 8) / (2 * rf)
        self.white_field = amp * np.exp(1j * alpha * r2) * 100.0
        coef = fresnel_factor(n, ny, self.wavelength, zfd, zfs, pixel)
        self.illum_sample = fresnel_from_detector(self.white_field, coef)
        R = radius_frac * min(n, ny)
        g = rng(seed)
        amp_t = g.uniform(0.8, 1.0, (n, ny))
        ph_t = gaussian_filter(g.uniform(-np.pi / 4, np.pi / 4, (n, ny)), 2.0, mode="wrap")
        T = amp_t * np.exp(1j * ph_t)
        T[~disk_mask(n, ny, R)] = 1.0
        self.transmission = T
        esw = (T - 1) * self.illum_sample
        I = np.abs(fresnel_to_detector(esw, coef) + self.white_field) ** 2
        self.intensity = poisson_scale(I, photons, seed) if photons else I
        self.support = disk_mask(n, ny, R * 1.1).astype(float)



class PhaseDiverseCase:
    """Phase-diverse Fresnel frames of one extended object: frame k sees the
    n x n window of a global transmission function at its position
    (positions[k]: the x, y given to PhaseDiverseCDI::add_new_position; the
    window starts at global index -position - x_min with x_min = -position of
    frame 0, PhaseDiverseCDI.h:380-397) under its own illumination -- a
    different focus-to-sample distance per frame (the phase diversity)."""

    def __init__(self, n, positions=((0, 0), (5, -3), (-4, 6)), seed=11, energy_kev=8.0,
                 zfd=1.0, zfs=(1.0e-3, 0.97e-3, 1.04e-3), pixel=13.5e-6, photons=None,
                 wavelength=None):
        self.n = n
        self.positions = [tuple(float(v) for v in p) for p in positions]
        self.wavelength = wavelength or FresnelCase.HC_KEV_M / energy_kev
        self.pixel = pixel
        # one focus-to-detector distance for all frames (zfd), or one per frame
        zl = list(zfd) if hasattr(zfd, "__len__") else [zfd]
        self.zfd = zl[0]
        self.zfds = [zl[k % len(zl)] for k in range(len(positions))]
        self.zfs = [zfs[k % len(zfs)] for k in range(len(positions))]
        xmin = int(-self.positions[0][0])
        ymin = int(-self.positions[0][1])
        starts = [(int(-x - xmin), int(-y - ymin)) for x, y in self.positions]
        lo_x = min(sx for sx, _ in starts)
        lo_y = min(sy for _, sy in starts)
        span_x = max(sx for sx, _ in starts) - lo_x + n
        span_y = max(sy for _, sy in starts) - lo_y + n
        g = rng(seed)
        amp = gaussian_filter(g.uniform(0.75, 1.0, (span_x, span_y)), 1.5)
        ph = gaussian_filter(g.uniform(-np.pi / 3, np.pi / 3, (span_x, span_y)), 2.0)
        self.object = amp * np.exp(1j * ph)
        i = np.arange(n)[:, None] - n / 2.0
        j = np.arange(n)[None, :] - n / 2.0
        r2 = i * i + j * j
        rf = 0.42 * n
        wamp = gaussian_filter((r2 <= rf * rf).astype(float), 2.0)
        alpha = (math.pi / 8) / (2 * rf)
        self.white_fields, self.intensities, self.windows = [], [], []
        for k, (sx, sy) in enumerate(starts):
            wf = wamp * np.exp(1j * alpha * r2 * (1 + 0.1 * k)) * 100.0
            coef = fresnel_factor(n, n, self.wavelength, self.zfds[k], self.zfs[k], pixel)
            illum = fresnel_from_detector(wf, coef)
            T = self.object[sx - lo_x:sx - lo_x + n, sy - lo_y:sy - lo_y + n]
            esw = (T - 1) * illum
            I = np.abs(fresnel_to_detector(esw, coef) + wf) ** 2
            self.white_fields.append(wf)
            self.intensities.append(poisson_scale(I, photons, seed + k) if photons else I)
            self.windows.append(T)
        self.support = disk_mask(n, n, 0.36 * n).astype(float)


def constraint_regions(n, ny=None):
    """Three complex-constraint regions inside the central support: two
    disjoint blocks and a third that overlaps the first (the earlier region
    keeps the shared pixels); their (alpha1, alpha2) and fixed c (NaN = free)."""
    ny = ny or n
    c0, c1 = n // 2, ny // 2
    q = max(2, n // 10)
    a = np.zeros((n, ny))
    b = np.zeros((n, ny))
    c = np.zeros((n, ny))
    a[c0 - q:c0, c1 - q:c1] = 1
    b[c0:c0 + q, c1:c1 + q] = 1
    c[c0 - q // 2:c0 + q // 2, c1 - q:c1] = 1
    return [a, b, c], [(0.5, 0.4), (0.3, 0.6), (0.8, 0.1)], np.array([np.nan, 0.7, np.nan])

# --------------------------------------------------------------------- Poly

def gaussian_spectrum(nlines, fwhm_frac, lambda_ref, padding, n):
    """Lines listed longest wavelength first with Gaussian weights (FWHM as a
    fraction of the reference wavelength), spaced so that PolyCDI's padding
    (int)((lambda_0/lambda_c - 1)*n/2) (PolyCDI.c++:86-87) equals `padding`."""
    sigma = fwhm_frac / (2 * math.sqrt(2 * math.log(2)))
    k = np.arange(nlines)
    best = None
    for span in np.linspace(0.01 * sigma, 0.5, 200000):
        d = span * (1 - 2 * k / (nlines - 1))
        w = np.exp(-d * d / (2 * sigma * sigma))
        wl = lambda_ref * (1 + d)
        lc = wl[int(np.argmax(w))]
        p = int((wl[0] / lc - 1.0) * n / 2)
        if p == padding:
            best = (wl, w)
            break
    if best is None:
        raise ValueError("no spacing gives padding %d" % padding)
    wl, w = best
    return np.stack([wl, w], axis=1)


def poly_forward(obj, spectrum, n_pad):
    """Polychromatic intensity of PolyCDI::expand_wl for an nx x ny object
    padded by n_pad on every side (the padding PolyCDI derives from the
    spectrum), returned on the central nx x ny window."""
    nx, ny = obj.shape
    mx, my = nx + 2 * n_pad, ny + 2 * n_pad
    p = np.zeros((mx, my), dtype=np.complex128)
    p[n_pad:n_pad + nx, n_pad:n_pad + ny] = obj
    psi = np.fft.fftshift(np.fft.fft2(p)) / math.sqrt(mx * my)
    mag2 = np.abs(psi) ** 2
    w = spectrum[:, 1] / spectrum[:, 1].sum()
    lc = spectrum[int(np.argmax(spectrum[:, 1])), 0]
    I = np.zeros((mx, my))
    ii = np.arange(mx)[:, None]
    jj = np.arange(my)[None, :]
    for (wl, _), wt in zip(spectrum, w):
        lf = wl / lc
        xv = lf * (ii - nx / 2.0) + nx / 2.0
        yv = lf * (jj - ny / 2.0) + ny / 2.0
        ok = (xv >= 0) & (xv < mx) & (yv >= 0) & (yv < my)
        xi = np.clip(xv.astype(int), 0, mx - 1)
        yi = np.clip(yv.astype(int), 0, my - 1)
        I += np.where(ok, wt * mag2[xi, yi], 0.0)
    return I[n_pad:n_pad + nx, n_pad:n_pad + ny]


class PolyCase:
    """A PolyCDI problem: disk object, 10-line Gaussian spectrum (5% FWHM)."""

    def __init__(self, n, seed, nlines=10, fwhm_frac=0.05, padding=28, radius_frac=0.15,
                 sigma=2, photons=1e9, lambda_ref=1.0e-10):
        self.nx = self.ny = n
        self.obj = disk_object(n, n, radius_frac * n, sigma, seed)
        self.spectrum = gaussian_spectrum(nlines, fwhm_frac, lambda_ref, padding, n)
        I = poly_forward(self.obj, self.spectrum, padding)
        self.intensity = poisson_scale(I, photons, seed) if photons else I
        self.support = square_support(n, n, int(2.5 * radius_frac * n))
        self.padding = padding


# ------------------------------------------------------------- FresnelCDI_WF

def fresnel_wf_factor(nx, ny, wavelength, z12, z23, pixel):
    """The zone-plate-to-detector factor of FresnelCDI_WF.c++:31-79 on the full
    grid, at the folded indices of multiply_factors (FresnelCDI_WF.c++:98-124)."""
    x_mid, y_mid = (nx - 1) / 2.0, (ny - 1) / 2.0
    sx = wavelength * z23 / (pixel * nx)
    sy = wavelength * z23 / (pixel * ny)
    i_ = np.trunc(x_mid - np.abs(x_mid - np.arange(nx))).astype(int)
    j_ = np.trunc(y_mid - np.abs(y_mid - np.arange(ny))).astype(int)
    rho2 = (sx * (x_mid - i_))[:, None] ** 2 + (sy * (y_mid - j_))[None, :] ** 2
    phi = (rho2 / z12 + rho2 / z23) * math.pi / wavelength
    return (np.sin(phi) - 1j * np.cos(phi)) / math.sqrt(nx * ny)


def fresnel_wf_to_detector(x, coef):
    """FresnelCDI_WF::propagate_to_detector: FFT, x conj(coef), swap+scale, FFT."""
    nx, ny = x.shape
    y = np.fft.fft2(x) * np.conj(coef)
    y = np.fft.fftshift(y) / math.sqrt(nx * ny)
    return np.fft.fft2(y)


class FresnelWFCase:
    """A FresnelCDI_WF problem with the reference example's geometry
    (wavelength 4.892e-10 m, zone plate 16.353 mm before focus, detector
    0.909513 m after the zone plate, 13.5 um pixels); the zone-plate diameter
    is scaled so that its projected disk has radius `radius_frac` of the grid."""

    def __init__(self, n, seed, radius_frac=0.3, wavelength=4.892e-10, z12=16.353e-3,
                 z23=0.909513 - 16.353e-3, pixel=13.5e-6, photons=None):
        self.nx = self.ny = n
        self.wavelength, self.z12, self.z23, self.pixel = wavelength, z12, z23, pixel
        delta_z = (z12 / z23) * pixel
        self.z_diameter = 2.0 * radius_frac * n * delta_z / 1.01
        r = radius_frac * n
        g = rng(seed)
        ph = gaussian_filter(g.uniform(-np.pi, np.pi, (n, n)), 3.0, mode="wrap")
        i = np.arange(n)[:, None] - (n - 1) // 2
        j = np.arange(n)[None, :] - (n - 1) // 2
        aberration = 0.5 * ((i * i + j * j) / (r * r)) ** 2
        self.zone_field = disk_mask(n, n, 0.95 * r) * np.exp(1j * (ph + aberration))
        coef = fresnel_wf_factor(n, n, wavelength, z12, z23, pixel)
        self.white_field = fresnel_wf_to_detector(self.zone_field, coef)
        I = np.abs(self.white_field) ** 2
        self.intensity = poisson_scale(I, photons, seed) if photons else I

