"""Generate the golden fixtures in tests/golden/ from the reference itself.

The reference's own sources (NADIA/src/{Complex_2D,BaseCDI,PlanarCDI,
FresnelCDI,FresnelCDI_WF,PolyCDI,TransmissionConstraint,PhaseDiverseCDI}.c++,
utils.c), compiled unmodified in their double build against
the FFTW shim by oracle/build_oracle.py, run the scenarios of tests/scenarios.py
on the synthetic inputs of pynadia.synth.  Each fixture stores the outputs
and a digest of the inputs it was made from.

Run (needs the reference sources, i.e. in the build container):
    python tests/golden/make_golden.py [case ...]
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "nadia-coecxs_b200"),
                os.path.dirname(HERE)]

import pyoracle as po  # noqa: E402
import scenarios as sc  # noqa: E402

CASES = {
    "planar_mixed_32": (sc.planar_mixed, dict(n=32)),
    "planar_mixed_32x48": (sc.planar_mixed, dict(n=32, ny=48)),
    "planar_custom_32": (sc.planar_custom, dict(n=32)),
    "fresnel_mixed_32": (sc.fresnel_mixed, dict(n=32)),
    "poly_mixed_32": (sc.poly_mixed, dict(n=32, padding=2)),
    "fresnel_wf_mixed_32": (sc.fresnel_wf_mixed, dict(n=32)),
    "phase_diverse_series_32": (sc.phase_diverse_mixed, dict(n=32)),
    "phase_diverse_parallel_g2_32": (sc.phase_diverse_mixed,
                                     dict(n=32, parallel=True, granularity=2, beta=0.8,
                                          gamma=1.5, alphas=[1.0, 0.6, 1.4])),
    "phase_diverse_align_32": (sc.phase_diverse_mixed, dict(n=32, adjust="cc")),
    "phase_diverse_minerr_32": (sc.phase_diverse_mixed, dict(n=32, adjust="me", forward=False)),
}


def input_digest(name):
    kw = CASES[name][1]
    n = kw.get("n", 32)
    h = hashlib.sha256()
    if name.startswith("phase_diverse"):
        c = sc.phase_diverse_inputs(n)
        arrs = c.intensities + c.white_fields + [c.support, np.array(c.positions)]
    elif name.startswith("planar"):
        c = sc.planar_inputs(n, ny=kw.get("ny"), beam_stop=0 if "custom" in name else 4)
        arrs = [c.intensity, c.support]
    elif name.startswith("fresnel_wf"):
        f = sc.fresnel_wf_inputs(n)
        arrs = [f.intensity, np.array([f.z_diameter, f.wavelength, f.z12, f.z23, f.pixel])]
    elif name.startswith("fresnel"):
        f = sc.fresnel_inputs(n)
        arrs = [f.intensity, f.support, f.white_field]
    else:
        p = sc.poly_inputs(n, kw["padding"])
        arrs = [p.intensity, p.support, p.spectrum]
    for a in arrs:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def reference_factory(kind, nx, ny, **kw):
    return po.Reference(kind, nx, ny, variant="64", **kw)


def main(names=None):
    if not po.reference_available("64"):
        sys.exit("oracle/_ref not built (python oracle/build_oracle.py with the reference present)")
    for name, (fn, kw) in CASES.items():
        if names and name not in names:
            continue
        res = fn(reference_factory, **kw)
        out = {k: v for k, v in res.items() if v is not None}
        out["input_digest"] = np.array(input_digest(name))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, {k: getattr(v, "shape", v) for k, v in out.items()})


if __name__ == "__main__":
    main(sys.argv[1:])
