"""Inputs, configuration files and expected outputs for the reconstruction
tool (CDI_reconstruction, NADIA/tools/CDI_reconstruction.c).

A case writes its input files (.dbin data and support, .cplx white field,
.txt spectrum) and a configuration file into a directory; ``expected`` runs
the tool's sequence of calls on a CPU solver (the oracle, or the reference
library) -- initialise_estimate(seed) unless a starting point is given, each
algorithm for its iterations, the magnitude image after iteration i when
i % output_iterations == 0, shrink-wrap after iteration i when
i % shrinkwrap_iterations == shrinkwrap_iterations - 1 -- and returns the
final estimate, the images and (fresnel) the transmission function."""
import os

import numpy as np

import pyoracle as po
from pynadia import synth

ALG = {"ER": 0, "BIO": 1, "BOO": 2, "HIO": 3, "DM": 4, "SF": 5, "ASR": 6, "HPR": 7, "RAAR": 8}


def write_dbin(path, a):
    np.ascontiguousarray(np.asarray(a, dtype=np.float64).T).tofile(path)


def write_cplx(path, c):
    c = np.asarray(c, dtype=np.complex128)
    np.ascontiguousarray(np.stack([c.real.T, c.imag.T], -1)).tofile(path)


def read_cplx(path, nx, ny):
    raw = np.fromfile(path, dtype=np.float64).reshape(ny, nx, 2)
    return (raw[..., 0] + 1j * raw[..., 1]).T.copy()


def magnitude(c):
    return np.sqrt(c.real * c.real + c.imag * c.imag)


class CliCase:
    """kind: planar, fresnel_wf, fresnel or poly; n: grid side."""

    def __init__(self, kind, n, directory, stages=None, output_iterations=10,
                 shrinkwrap_iterations=12, info_level=0, prefix=None, starting_point=None,
                 diffraction=False):
        self.kind, self.n, self.dir = kind, n, str(directory)
        self.output_iterations = output_iterations
        self.shrinkwrap = shrinkwrap_iterations
        self.gauss_width, self.threshold = 1.5, 0.1
        self.prefix = prefix or (kind + "_out")
        self.starting_point = starting_point
        self.diffraction = diffraction
        self.stages = stages or [("ER", 4), ("HIO", 20), ("RAAR", 8), ("ER", 3)]
        self.kw = {}
        os.makedirs(self.dir, exist_ok=True)
        keys = {}
        if kind == "planar":
            c = synth.PlanarCase(n, max(3, n // 6), 2, 1e6, seed=5, support_side=int(n * 0.42))
            self.data, self.support = c.intensity, c.support
        elif kind == "fresnel":
            f = synth.FresnelCase(n, seed=4)
            self.data, self.support = f.intensity, f.support
            write_cplx(self.path("white_field.cplx"), f.white_field)
            self.kw = dict(white_field=f.white_field, wavelength=f.wavelength,
                           focal_detector_length=f.zfd, focal_sample_length=f.zfs,
                           pixel_size=f.pixel, normalisation=0.97)
            keys.update(white_field_reco_file_name="white_field.cplx",
                        beam_wavelength=f.wavelength, focal_detector_length=f.zfd,
                        focal_sample_length=f.zfs, pixel_size=f.pixel, normalisation=0.97)
        elif kind == "fresnel_wf":
            f = synth.FresnelWFCase(n, seed=6)
            self.kw = dict(wavelength=f.wavelength, zone_focal_length=f.z12,
                           focal_detector_length=f.z23, pixel_size=f.pixel)
            s = po.Oracle("fresnel_wf", n, n, **self.kw)
            s.set_wf_support(f.z_diameter)
            self.data, self.support = f.intensity, s.get_support()
            self.stages = [("ER", 12)]  # the tool runs wf_iterations of the fixed algorithm
            self.shrinkwrap = 0
            keys.update(beam_wavelength=f.wavelength, zone_focal_length=f.z12,
                        focal_detector_length=f.z23, pixel_size=f.pixel,
                        white_field_data_file_name="data.dbin",
                        white_field_support_file_name="support.dbin",
                        white_field_reco_file_name="wf_reco.cplx", wf_iterations=12)
        elif kind == "poly":
            p = synth.PolyCase(n, seed=9, padding=4, photons=1e7)
            self.data, self.support = p.intensity, p.support
            with open(self.path("spectrum.txt"), "w") as fh:
                fh.write("Energy\tF.Density\n")
                for wl, w in p.spectrum:
                    fh.write("%.9g\t%.9g\n" % (1.0 / wl, w))
            self.spectrum = po.read_spec(self.path("spectrum.txt"))
            self.kw = dict(n_best=1)
            keys.update(spectrum_file_name="spectrum.txt")
        else:
            raise ValueError(kind)
        write_dbin(self.path("data.dbin"), self.data)
        write_dbin(self.path("support.dbin"), self.support)
        keys.update(pixels_x=n, pixels_y=n, data_file_name="data.dbin",
                    support_file_name="support.dbin", output_file_name_prefix=self.prefix,
                    output_file_type="ppm", output_iterations=output_iterations,
                    algorithm=" ".join(a for a, _ in self.stages),
                    iterations=" ".join(str(k) for _, k in self.stages),
                    shrinkwrap_iterations=self.shrinkwrap, shrinkwrap_gauss_width=self.gauss_width,
                    shrinkwrap_threshold=self.threshold, info_level=info_level)
        if starting_point:
            keys["starting_point_file_name"] = starting_point
        if diffraction:
            keys["output_diffraction_estimate"] = 1
            keys["use_log_scale_for_diffraction"] = 1
        self.config = self.path(self.prefix + ".config")
        with open(self.config, "w") as fh:
            fh.write("# %s reconstruction\n" % kind)
            for k, v in keys.items():
                fh.write("%s = %s\n" % (k, ("%.17g" % v) if isinstance(v, float) else v))

    def path(self, name):
        return os.path.join(self.dir, name)

    @property
    def output_file(self):
        return "wf_reco.cplx" if self.kind == "fresnel_wf" else self.prefix + ".cplx"

    def image_names(self):
        total = sum(k for _, k in self.stages)
        oi = self.output_iterations
        return {i: "%s_%d.ppm" % (self.prefix, i) for i in range(total) if oi and i % oi == 0}

    def diffraction_names(self):
        """The tool's names for the diffraction images (the reference's tool
        appends them to the magnitude image's name instead)."""
        return {i: "%s_diffraction_%d.ppm" % (self.prefix, i) for i in self.image_names()}

    def expected(self, seed, make=po.Oracle):
        n = self.n
        s = make(self.kind, n, n, **self.kw)
        if self.kind == "poly":
            s.set_spectrum(self.spectrum)
        s.set_support(self.support)
        s.set_intensity(self.data)
        if self.starting_point:
            s.set_exit_surface_wave(read_cplx(self.path(self.starting_point), n, n))
        else:
            s.initialise_estimate(seed)
        images, diffraction, i = {}, {}, 0
        oi, k = self.output_iterations, self.shrinkwrap
        for alg, count in self.stages:
            if self.kind != "fresnel_wf":
                s.set_algorithm(ALG[alg])
            for _ in range(count):
                s.iterate()
                if oi and i % oi == 0:
                    images[i] = magnitude(s.get_exit_surface_wave())
                    if self.diffraction:
                        m = magnitude(s.propagate_to_detector(s.get_exit_surface_wave()))
                        diffraction[i] = m * m
                if k and i % k == k - 1:
                    s.apply_shrinkwrap(self.gauss_width, self.threshold)
                i += 1
        out = {"final": s.get_exit_surface_wave(), "images": images, "diffraction": diffraction}
        if self.kind == "fresnel":
            out["transmission"] = s.get_transmission()
        return out
