"""Run tests/scenarios.py's planar_mixed on an FP32 handle through the C ABI
with float-rounded array inputs (as a float build's Double_2D holds them) and
save the results: the comparison point of the drop-in program's float build.
Run in its own process so that its tile choice (NADIA_TUNE=0) matches the
program's.

    python fp32_handle_run.py <n> <out.npz>"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.dirname(HERE), os.path.join(os.path.dirname(os.path.dirname(HERE)),
                                                    "nadia-coecxs_b200")]
import pynadia  # noqa: E402
import scenarios as sc  # noqa: E402


def f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


class RoundedInputs:
    def __init__(self, h):
        self.h = h

    def __getattr__(self, name):
        fn = getattr(self.h, name)
        if name in ("set_support", "set_intensity", "set_beam_stop"):
            return lambda a, *r: fn(f32(a), *r)
        return fn


def main():
    n, out = int(sys.argv[1]), sys.argv[2]
    res = sc.planar_mixed(lambda kind, nx, ny, **kw: RoundedInputs(
        pynadia.Solver(kind, nx, ny, precision=pynadia.FP32, **kw)), n=n)
    np.savez(out, errors=res["errors"], esw=res["esw"], support=res["support"])


if __name__ == "__main__":
    main()
