"""The staged Sobol integers of the GPU loops, restated on the CPU.

sobol_stage_block / SobolLane (dbgenzpaper_b200/csrc/genz_step.cuh) give
the point of tile row r (first index T = B + o, B a multiple of 32) as
x(B + 32 q) ^ x(gray(k) & 3) ^ x(gray(k) & 28) with q = (o + r) >> 5 and
k = (o + r) & 31, the five bases from x(B) by the recurrence
x(32 (c + 1)) = x(32 c) ^ V[4] ^ V[5 + ctz(c + 1)].  This test follows
those steps with integers and compares every row of tiles at many first
indices (all offsets mod 32, bases near 2^32) with the direct Gray-code
integer that the checker computes (src/qmc_generators.jl:331-352 on the
32-bit grid)."""
import numpy as np


def x_direct(V, n):
    g = (n ^ (n >> 1)) & 0xFFFFFFFF
    x = 0
    for b in range(32):
        if (g >> b) & 1:
            x ^= int(V[b])
    return x


def ctz(v):
    return (v & -v).bit_length() - 1


def staged_row(V, T):
    """The 17 staged words of one dimension for a tile whose first index is T
    (shift 0), following sobol_stage_block."""
    B = T & ~31
    c = B >> 5
    xB = x_direct(V, B)
    bases = [xB]
    for s in range(1, 5):
        z = 5 + ctz(c + s)
        bases.append(bases[-1] ^ int(V[4]) ^ (int(V[z]) if z < 32 else 0))
    a = [(int(V[0]) if i & 1 else 0) ^ (int(V[1]) if i & 2 else 0) for i in range(4)]
    b = [(int(V[2]) if i & 1 else 0) ^ (int(V[3]) if i & 2 else 0) ^ (int(V[4]) if i & 4 else 0)
         for i in range(8)]
    return bases + a + b


def lane_value(tab, T, r):
    s = (T & 31) + r
    k = s & 31
    g = k ^ (k >> 1)
    return tab[s >> 5] ^ tab[5 + (g & 3)] ^ tab[9 + (g >> 2)]


def test_staged_sobol_integers_match_gray_code():
    rng = np.random.default_rng(5)
    V = [int(v) for v in rng.integers(0, 2**32, size=32, dtype=np.uint64)]
    firsts = list(range(0, 70)) + [2 * 65536 + 1, 16385, 2**31 - 77, 2**32 - 130, 2**32 - 3, 2**32 + 5,
                                   3 * 2**33 + 17]
    firsts += [int(t) for t in rng.integers(0, 2**40, size=40)]
    for T0 in firsts:
        for tile in range(3):
            T = T0 + 128 * tile
            tab = staged_row(V, T)
            for r in range(128):
                assert lane_value(tab, T, r) == x_direct(V, T + r), (T0, tile, r)


def test_sobol_first_index_follows_sobol_jl_skip(dbgz):
    """SobolQMC's skip(SobolSeq(d), 2m - 1) (src/qmc_generators.jl:57-58):
    Sobol.jl's skip makes 2^floor(log2(n + 1)) next! calls (exact = false),
    the k-th returning Gray-code point k; the first point read is the next."""
    f = dbgz.sobol_first_index
    assert f(2**16) == 2**17 + 1 and f(2**14) == 2**15 + 1
    assert f(10**4) == 2**14 + 1          # the reference's default m: not 2m
    assert f(1000) == 1025 and f(1500) == 2049 and f(1) == 3
    assert f(1000, exact=True) == 2000    # skip(s, n, exact=true)
    assert f(5, skip0=0) == 1
