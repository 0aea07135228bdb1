"""CPU checks of every FP32 tile plan compiled into the library.

The fused FP32 passes transform L signals of length N per CTA with the
Stockham schedule of nadia-coecxs_b200/csrc/fft32.cuh: each of NT threads
holds E = N*L/NT values, butterflies are dealt to threads by a column or a
row map (panel-coalesced global access), and the values move between passes
through a swizzled shared-memory tile.  The GPU tests run only the variant the
autotuner picks on the machine at hand; this file replays the index algebra
of every registered variant (fused32_v*.cu, fused32_poly.cu) in numpy:

* the thread map, twiddle exponents (t1 = (j mod Ns) * N/(Ns*R), W^(t1*r)),
  exchange addresses (including the strided form used when the swizzle
  commutes with the stride) and output positions of each pass, in both
  directions and for both maps, give the DFT of numpy's definition;
* every exchange writes each shared-memory word once, inside the tile, and
  every read finds a written word;
* the twiddle table (N entries) is never indexed past its end;
* a forward transform ends on the positions where the inverse starts, so the
  projections between them run on registers;
* the swizzle keeps each exchange within 1.25x of the ideal shared-memory
  wavefront count (swizzle_search.py's model).
"""
import os
import re
import sys
from functools import reduce
from math import gcd

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "nadia-coecxs_b200", "csrc")
K = 4  # panel width

PAT = re.compile(r"make_(variant|ping|staged_ping|staged|persistent_single|persistent_direct|persistent_ping|persistent_mstage|"
                 r"persistent_row|grouped_row_tw|grouped_row|grouped_col|persistent_tw|persistent|poly)<\s*(\d+),\s*(\d+),\s*(\d+),\s*(\d+),\s*"
                 r"Swizzle<\s*(\d+),\s*(\d+),\s*(\d+),\s*(\d+)>\s*,\s*([\d,\s]+)>")


# the classes of the mixed-length passes (fused32_mixed.cu): mix_class<N, L,
# Swizzle<...>, radices...> at kMixNT threads
MIX_PAT = re.compile(r"mix_class<\s*(\d+),\s*(\d+),\s*Swizzle<\s*(\d+),\s*(\d+),\s*(\d+),"
                     r"\s*(\d+)>\s*,\s*([\d,\s]+)>")


def registry():
    files = sorted(f for f in os.listdir(CSRC) if re.match(r"fused32_v\d+\.cu$", f))
    files.append("fused32_poly.cu")
    out = []
    for f in files:
        for m in PAT.finditer(open(os.path.join(CSRC, f)).read()):
            n, nt, L, minb, s1, s2, msk, sh = (int(m.group(i)) for i in range(2, 10))
            rad = tuple(int(r) for r in m.group(10).split(","))
            out.append(dict(kind=m.group(1), N=n, NT=nt, L=L, minb=minb, sw=(s1, s2, msk, sh),
                            rad=rad, file=f))
    src = open(os.path.join(CSRC, "fused32_mixed.cu")).read()
    nt = int(re.search(r"constexpr int kMixNT = (\d+);", src).group(1))
    for m in MIX_PAT.finditer(src):
        n, L, s1, s2, msk, sh = (int(m.group(i)) for i in range(1, 7))
        rad = tuple(int(r) for r in m.group(7).split(","))
        out.append(dict(kind="mixed", N=n, NT=nt, L=L, minb=1, sw=(s1, s2, msk, sh), rad=rad,
                        file="fused32_mixed.cu"))
    return out


VARIANTS = registry()


def vid(v):
    return "%s-%d-%dthr-L%d-%s" % (v["kind"], v["N"], v["NT"], v["L"], ".".join(map(str, v["rad"])))


def swizzle(sw):
    s1, s2, m, sh = sw

    def f(a):
        t = (a >> s1) ^ ((a >> s2) if s2 else 0)
        return a ^ ((t & m) << sh)
    return f


def stride_commutes(sw, c):
    s1, s2, _, sh = sw
    hi = max(s1, s2) + 3
    return c > 0 and c % (1 << hi) == 0 and sh + 3 <= hi


def pow2(x):
    return x > 0 and (x & (x - 1)) == 0


def colmap(beta, NR, L):
    lo = beta % K
    rest = beta // K
    return (rest // NR) * K + lo, rest % NR


def rowmap(beta, NR, L):
    kk = beta % K
    return (beta // K) % L, (beta // (K * L)) * K + kk


def emulate(v, mapf, fwd, x):
    """One tile transform as fft32.cuh performs it; x has shape (L, N)."""
    N, NT, L, rad = v["N"], v["NT"], v["L"], v["rad"]
    E, P = N * L // NT, len(rad)
    sw = swizzle(v["sw"])
    sign = -1.0 if fwd else 1.0

    def radix(p):
        return rad[p] if fwd else rad[P - 1 - p]

    def span(p):
        return reduce(lambda a, b: a * b, [radix(i) for i in range(p)], 1)

    t = np.arange(NT)
    vals = np.empty((NT, E), complex)
    R = radix(0)
    NR = N // R
    for q in range(E // R):
        s, j = mapf(t + q * NT, NR, L)
        assert (j < NR).all() and (s < L).all()
        for r in range(R):
            vals[:, q * R + r] = x[s, j + r * NR]
    for p in range(P):
        R, Ns = radix(p), span(p)
        NR, B, TSTEP = N // R, E // R, N // (Ns * R)
        F = np.exp(sign * 2j * np.pi * np.outer(np.arange(R), np.arange(R)) / R)
        for q in range(B):
            s, j = mapf(t + q * NT, NR, L)
            if Ns > 1:
                t1 = (j % Ns) * TSTEP
                assert (t1 * (R - 1)).max() < N, "twiddle index past the table"
                for r in range(1, R):
                    vals[:, q * R + r] *= np.exp(sign * 2j * np.pi * (t1 * r) / N)
            vals[:, q * R:(q + 1) * R] = vals[:, q * R:(q + 1) * R] @ F.T
        if p + 1 == P:
            break
        sm = np.full(N * L, np.nan + 0j)
        used = np.zeros(N * L, bool)
        wstride = Ns * L
        for q in range(B):
            s, j = mapf(t + q * NT, NR, L)
            base = (j // Ns) * Ns * R + j % Ns
            a0 = np.array([sw(int(b) * L + int(ss)) for b, ss in zip(base, s)])
            for r in range(R):
                a = np.array([sw(int(b + r * Ns) * L + int(ss)) for b, ss in zip(base, s)])
                if stride_commutes(v["sw"], wstride):
                    assert (a == a0 + r * wstride).all(), "swizzle does not commute"
                elif pow2(R) and pow2(wstride):   # fft32.cuh's xor_split form
                    assert (a == (a0 ^ sw(r * wstride))).all(), "xor split of a write"
                assert (a >= 0).all() and (a < N * L).all()
                assert not used[a].any() and len(set(a.tolist())) == NT, "exchange overwrites"
                used[a] = True
                sm[a] = vals[:, q * R + r]
        assert used.all()
        R2 = radix(p + 1)
        NR2 = N // R2
        rstride = NR2 * L
        for q in range(E // R2):
            s, j = mapf(t + q * NT, NR2, L)
            a0 = np.array([sw(int(jj) * L + int(ss)) for jj, ss in zip(j, s)])
            for r in range(R2):
                a = np.array([sw(int(jj + r * NR2) * L + int(ss)) for jj, ss in zip(j, s)])
                if not stride_commutes(v["sw"], rstride) and pow2(R2) and pow2(rstride):
                    assert (a == (a0 ^ sw(r * rstride))).all(), "xor split of a read"
                vals[:, q * R2 + r] = sm[a]
    R = radix(P - 1)
    NR = N // R
    X = np.full((L, N), np.nan + 0j)
    for q in range(E // R):
        s, j = mapf(t + q * NT, NR, L)
        for r in range(R):
            X[s, j + r * NR] = vals[:, q * R + r]
    assert not np.isnan(X).any(), "an output position is never written"
    return X


def out_positions(v, mapf, first_radix):
    N, NT, L = v["N"], v["NT"], v["L"]
    E = N * L // NT
    R = first_radix
    t = np.arange(NT)
    pos = []
    for q in range(E // R):
        s, j = mapf(t + q * NT, N // R, L)
        for r in range(R):
            pos.append(s * N + j + r * (N // R))
    return np.array(pos)


COLUMN_ONLY = ("persistent_single", "persistent_direct", "persistent_ping", "persistent_mstage",
               "staged", "staged_ping")


def maps_of(v):
    """The thread maps a variant runs: row-only variants have no column pass,
    column-only (one-stage persistent) variants no row pass."""
    ms = [] if v["kind"] in COLUMN_ONLY else [("row", rowmap)]
    if v["L"] % K == 0 and v["kind"] not in ("persistent_row", "grouped_row", "grouped_row_tw",
                                              "grouped_col"):
        ms.insert(0, ("col", colmap))
    return ms


def test_registry_found():
    assert len(VARIANTS) >= 40
    assert {v["N"] for v in VARIANTS} >= {256, 512, 768, 1024, 1080, 1536, 2048, 4096}


@pytest.mark.parametrize("v", VARIANTS, ids=vid)
def test_tile_shape_constraints(v):
    N, NT, L, rad = v["N"], v["NT"], v["L"], v["rad"]
    assert np.prod(rad) == N
    # whole warps, or (PolyCDI's two-CTA 1080-point tiles) a last half warp,
    # which the block reductions sum over on its own
    assert N * L % NT == 0 and (NT % 32 == 0 or (v["kind"] == "poly" and NT % 32 == 16))
    E = N * L // NT
    assert E % reduce(lambda a, b: a * b // gcd(a, b), rad) == 0
    assert all((N // r) % K == 0 for r in rad), "row tiles need N/R divisible by the panel"
    if v["kind"] not in ("persistent_row", "grouped_row", "grouped_row_tw", "grouped_col"):
        assert L % K == 0, "column tiles cover whole panels"
    if v["kind"] in ("grouped_row", "grouped_row_tw"):   # minb holds the group count
        assert v["minb"] * (N * L * 28 + 24) <= 227 * 1024
    if v["kind"] == "grouped_col":   # half panels: two P stages, one sqrt(I) panel
        assert L == 2 and v["minb"] * (N * L * 16 + N * 16 + 24) <= 227 * 1024
    if v["kind"] in ("persistent", "persistent_tw", "mixed"):
        assert N * L * 28 + 24 <= 227 * 1024
    # several CTAs per SM share its 228 KB (1 KB reserved per CTA)
    if v["kind"] == "persistent_row":
        assert v["minb"] * (N * L * 28 + 24 + 1024) <= 228 * 1024
    if v["kind"] == "persistent_single":
        assert v["minb"] * (N * L * 12 + 16 + 1024) <= 228 * 1024
    if v["kind"] == "persistent_direct":
        assert v["minb"] * (N * L * 8 + 16 + 1024) <= 228 * 1024
    if v["kind"] == "persistent_ping":
        assert v["minb"] * (N * L * 24 + 24 + 1024) <= 228 * 1024
    if v["kind"] == "persistent_mstage":
        assert N * L * 28 + 24 <= 227 * 1024
    if v["kind"] in ("staged", "staged_ping"):   # exchange tile(s) + sqrt(I) + white field
        assert N * L * (8 * (2 if v["kind"] == "staged_ping" else 1) + 12) <= 227 * 1024


@pytest.mark.parametrize("v", VARIANTS, ids=vid)
def test_tile_transform_is_the_dft(v):
    g = np.random.default_rng(v["N"] * 7 + v["NT"])
    x = g.standard_normal((v["L"], v["N"])) + 1j * g.standard_normal((v["L"], v["N"]))
    for name, mapf in maps_of(v):
        Xf = emulate(v, mapf, True, x)
        assert np.allclose(Xf, np.fft.fft(x, axis=1), rtol=0, atol=1e-9 * v["N"]), name
        Xi = emulate(v, mapf, False, x)
        assert np.allclose(Xi, v["N"] * np.fft.ifft(x, axis=1), rtol=0, atol=1e-9 * v["N"]), name
        # the forward transform's last pass leaves each thread the inputs of
        # the inverse transform's first pass: both visit positions with the
        # same radix (the inverse runs the radices reversed), and that visit
        # covers the tile once
        P = len(v["rad"])
        last_fwd_radix, first_inv_radix = v["rad"][P - 1], v["rad"][::-1][0]
        assert last_fwd_radix == first_inv_radix
        pos = out_positions(v, mapf, last_fwd_radix).ravel()
        assert len(np.unique(pos)) == pos.size == v["N"] * v["L"]


@pytest.mark.parametrize("v", VARIANTS, ids=vid)
def test_swizzle_wavefronts(v):
    here = os.path.dirname(os.path.abspath(__file__))
    if here not in sys.path:
        sys.path.insert(0, here)
    import swizzle_search as ss
    sw = swizzle(v["sw"])
    worst = 0.0
    for _, mapf in maps_of(v):
        t, i = ss.count(v["N"], v["NT"], v["L"], v["rad"], mapf, sw)
        t2, i2 = ss.count(v["N"], v["NT"], v["L"], tuple(reversed(v["rad"])), mapf, sw)
        worst = max(worst, (t + t2) / (i + i2))
    assert worst <= 1.25, "shared-memory wavefronts %.3f x ideal" % worst
