"""Choose the shared-memory swizzle of each FP32 tile variant.

For a tile (N, NT threads, L signals, radix list, thread map) this replays the
exchange pattern of fft32.cuh -- for every pass, every warp's 64-bit shared
stores of the butterfly outputs and loads of the next pass's inputs -- and
counts shared-memory wavefronts (16 lanes per wavefront for 8-byte words,
one wavefront per distinct address per bank).  It searches the family
a -> a ^ ((((a >> S1) ^ (a >> S2)) & M) << SH) for the smallest count and
prints the swizzle of each variant registered in nadia-coecxs_b200/csrc/fused32_v*.cu.

Usage: python tests/swizzle_search.py
"""
K = 4

# (N, NT, L, radices, minBlocksPerSM)
VARIANTS = {
    256: [(256, 256, 16, (16, 16), 2), (256, 128, 8, (16, 16), 4), (256, 256, 8, (8, 8, 4), 3)],
    512: [(512, 256, 8, (16, 8, 4), 2), (512, 128, 4, (16, 8, 4), 4), (512, 256, 4, (8, 8, 8), 3)],
    768: [(768, 256, 8, (8, 8, 4, 3), 2), (768, 128, 4, (8, 8, 4, 3), 4),
          (768, 256, 4, (4, 4, 4, 4, 3), 2)],
    1024: [(1024, 256, 4, (16, 16, 4), 2), (1024, 128, 4, (16, 16, 4), 4),
           (1024, 512, 4, (8, 8, 4, 4), 2), (1024, 512, 8, (16, 16, 4), 1)],
    1536: [(1536, 256, 4, (8, 8, 8, 3), 2), (1536, 512, 4, (4, 4, 4, 4, 2, 3), 1)],
    2048: [(2048, 512, 4, (16, 16, 8), 1), (2048, 256, 4, (16, 16, 8), 2),
           (2048, 1024, 4, (8, 8, 8, 4), 1), (2048, 512, 4, (8, 16, 16), 1),
           (2048, 1024, 8, (16, 16, 8), 1)],
    4096: [(4096, 1024, 4, (16, 16, 16), 1), (4096, 512, 4, (16, 16, 16), 1)],
}


def colmap(beta, NR, L):
    lo = beta % K
    rest = beta // K
    return (rest // NR) * K + lo, rest % NR


def rowmap(beta, NR, L):
    kk = beta % K
    return (beta // K) % L, (beta // (K * L)) * K + kk


def wavefronts(addrs):
    total = 0
    for half in (addrs[:16], addrs[16:]):
        if not half:   # the last warp of a tile whose thread count is not a multiple of 32
            continue
        banks = {}
        for a in half:
            banks.setdefault((2 * a) % 32, set()).add(a)
        total += max(len(v) for v in banks.values())
    return total


def count(N, NT, L, radices, mapf, sw):
    E = N * L // NT
    tot = ideal = 0
    Ns = 1
    order = list(radices)
    for p, R in enumerate(order[:-1]):
        NR, B = N // R, E // R
        for q in range(B):
            for r in range(R):
                for w in range((NT + 31) // 32):
                    addrs = []
                    for lane in range(min(32, NT - 32 * w)):
                        s, j = mapf(w * 32 + lane + q * NT, NR, L)
                        base = (j // Ns) * Ns * R + j % Ns
                        addrs.append(sw((base + r * Ns) * L + s))
                    tot += wavefronts(addrs)
                    ideal += (len(addrs) + 15) // 16
        R2 = order[p + 1]
        NR2, B2 = N // R2, E // R2
        for q in range(B2):
            for r in range(R2):
                for w in range((NT + 31) // 32):
                    addrs = []
                    for lane in range(min(32, NT - 32 * w)):
                        s, j = mapf(w * 32 + lane + q * NT, NR2, L)
                        addrs.append(sw((j + r * NR2) * L + s))
                    tot += wavefronts(addrs)
                    ideal += (len(addrs) + 15) // 16
        Ns *= R
    return tot, max(ideal, 1)


def family():
    for s1 in range(4, 9):
        for s2 in [0] + list(range(s1 + 1, 12)):
            for m in (1, 3, 7):
                for sh in (1, 2):
                    def f(a, s1=s1, s2=s2, m=m, sh=sh):
                        t = (a >> s1) ^ ((a >> s2) if s2 else 0)
                        return a ^ ((t & m) << sh)
                    yield (s1, s2, m, sh), f


def best(N, NT, L, radices):
    """Swizzle minimising the worst of the column- and row-map wavefront ratios.
    The inverse transform runs the radices reversed; its exchanges are the
    same patterns mirrored, so the forward order is scored."""
    scored = []
    for key, f in family():
        rs = []
        for m in ((colmap,) if L % K == 0 else ()) + (rowmap,):
            t, i = count(N, NT, L, radices, m, f)
            t2, i2 = count(N, NT, L, tuple(reversed(radices)), m, f)
            rs.append((t + t2) / (i + i2))
        scored.append((max(rs), sum(rs), key))
    scored.sort()
    return scored[0]


if __name__ == "__main__":
    for N, vs in VARIANTS.items():
        for (n, NT, L, rad, minb) in vs:
            worst, _, key = best(n, NT, L, rad)
            print("%d NT=%d L=%d radices=%s minb=%d swizzle=%s worst_ratio=%.3f"
                  % (n, NT, L, ".".join(map(str, rad)), minb, key, worst))
