"""CPU checks of the copy geometry of the persistent FP32 passes
(nadia-coecxs_b200/csrc/fused32_persist.cuh, encode_one in fused32.cu), for
every persistent tile plan and every grid it can serve:

* row pass: the 3-D tensor map (4, nx, ny/4) with box (4, L rows, boxp panels)
  tiles a row tile exactly (boxp divides the panel count and is at most 256);
  the innermost box extent is a multiple of 16 bytes and the innermost
  coordinate of every copy is 0 (16-byte aligned); global strides are
  multiples of 16 bytes; no store starts at a negative coordinate; every
  shared-memory destination is 128-byte aligned; the bytes the mbarriers
  expect equal the bytes the boxes bring;
* column pass: the two bulk copies per tile are multiples of 16 bytes at
  16-byte aligned global and shared addresses;
* both: the stages and mbarriers fit the dynamic shared memory the launch
  asks for, and that stays within 227 KB.
"""
import pytest

from test_tile_plans import VARIANTS, vid

K = 4
SIZES = [256, 512, 768, 1024, 1536, 2048, 4096]
PERSISTENT = [v for v in VARIANTS if v["kind"] == "persistent"]


def box_panels(npan):
    # fused32_impl.h: the largest divisor of the panel count that is at most 256
    for d in range(min(npan, 256), 1, -1):
        if npan % d == 0:
            return d
    return 1


def test_persistent_plans_exist():
    assert {v["N"] for v in PERSISTENT} >= {256, 512, 1024, 2048}


@pytest.mark.parametrize("v", PERSISTENT, ids=vid)
def test_row_pass_tensor_copies(v):
    N, L = v["N"], v["L"]
    ny = N
    TW = N * L
    npan = ny // K
    boxp = box_panels(npan)
    assert npan % boxp == 0 and 1 <= boxp <= 256 and L <= 256
    # stages: P0, P1 (float2), x (float2), support (float), then 3 mbarriers
    P0, P1, X, S = 0, TW * 8, 2 * TW * 8, 3 * TW * 8
    bar = S + TW * 4
    smem = N * L * 28 + 24  # persist_row_smem
    assert bar % 8 == 0 and bar + 3 * 8 <= smem <= 227 * 1024
    for esz, base in ((8, P0), (8, P1), (8, X), (4, S)):
        assert (K * esz) % 16 == 0, "innermost box extent"
        boxes = 0
        for c in range(0, npan, boxp):
            dst = base + c * L * K * esz
            assert dst % 128 == 0, "shared destination of a tensor copy"
            boxes += K * L * boxp * esz
        assert boxes == TW * esz, "bytes expected on the mbarrier"
    for nx in SIZES:
        if nx % L:
            continue
        for esz in (8, 4):
            strides = (K * esz, nx * K * esz)
            assert all(s % 16 == 0 for s in strides), "global strides"
        # tiles start at row i0 = t*L >= 0 and panel c >= 0, x = 0
        tps = nx // L
        assert (tps - 1) * L + L <= nx


@pytest.mark.parametrize("v", PERSISTENT, ids=vid)
def test_column_pass_bulk_copies(v):
    N, L = v["N"], v["L"]
    TW = N * L
    P0, P1, M0, M1 = 0, TW * 8, 2 * TW * 8, 2 * TW * 8 + TW * 4
    bar = 2 * TW * 8 + 2 * TW * 4
    smem = N * L * 24 + 16  # persist_col_smem
    assert bar % 8 == 0 and bar + 2 * 8 <= smem <= 227 * 1024
    for dst in (P0, P1, M0, M1):
        assert dst % 16 == 0
    assert (TW * 8) % 16 == 0 and (TW * 4) % 16 == 0
    for ny in SIZES:
        if ny % L:
            continue
        tps = ny // L
        for t in range(tps):
            # the tile's global offset, (t % tps) * L * nx elements, for any nx
            for nx in SIZES:
                assert (t * L * nx * 8) % 16 == 0 and (t * L * nx * 4) % 16 == 0


def test_box_panels_model_matches_the_library(tmp_path):
    """The Python model of box_panels above against the library's own
    (fused32_impl.h), compiled for the host, for every panel count to 2048."""
    import os
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "bp.cpp"
    src.write_text('#include "fused32_impl.h"\n#include <cstdio>\n'
                   'int main() { for (int n = 1; n <= 2048; ++n) '
                   'printf("%d %d\\n", n, nadia::f32::box_panels(n)); }\n')
    exe = tmp_path / "bp"
    r = subprocess.run(["g++", "-std=c++17", "-I", "/usr/local/cuda/include",
                        "-I", os.path.join(root, "include"),
                        "-I", os.path.join(root, "nadia-coecxs_b200", "csrc"), str(src), "-o",
                        str(exe)], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip("host compile of fused32_impl.h failed: " + r.stderr[-300:])
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    got = {int(out[i]): int(out[i + 1]) for i in range(0, len(out), 2)}
    assert all(got[n] == box_panels(n) for n in range(1, 2049))
