"""The kernels split their linear cell, face and edge indices into (i, j, k) by a 32-bit
multiply-high and shift per divisor instead of a 64-bit division (dg_common.cuh: FastDiv,
make_fastdiv, fdiv, split3): Granlund and Montgomery's division by invariant integers (PLDI
1994, theorem 4.2, N = 32) with l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1 and
n / d = (mulhi(m, n) + n) >> l, valid for every n < 2^31 (the context refuses grids whose
index spaces reach 2^31).  This checks that arithmetic, as the header writes it, against exact
division: every divisor up to 1200, divisors near powers of two and random ones up to 2^31, each
with its edge dividends and random ones; and the three-index split of whole small index spaces."""
import random


def make_fastdiv(d: int) -> tuple[int, int]:
    l = 0
    while (1 << l) < d:
        l += 1
    m = ((1 << 32) * ((1 << l) - d)) // d + 1
    assert 0 < m < (1 << 32) or d == 1
    return m & 0xFFFFFFFF, l


def fdiv(n: int, m: int, l: int) -> int:
    t = (m * n) >> 32                       # __umulhi(m, n)
    s = (t + n) & 0xFFFFFFFF                # 32-bit sum: no wrap while n < 2^31
    assert t + n < (1 << 32)
    return s >> l


def split3(t: int, X: int, Y: int) -> tuple[int, int, int]:
    mx, lx = make_fastdiv(X)
    my, ly = make_fastdiv(Y)
    r = fdiv(t, mx, lx)
    q = fdiv(r, my, ly)
    return t - r * X, r - q * Y, q


def test_fastdiv_equals_integer_division():
    rng = random.Random(1)
    divisors = list(range(1, 1200)) + [2 ** k + o for k in range(1, 31) for o in (-1, 0, 1)] + \
        [rng.randrange(1, 2 ** 31) for _ in range(400)]
    for d in divisors:
        m, l = make_fastdiv(d)
        for n in [0, 1, d - 1, d, d + 1, 2 * d - 1, 2 ** 31 - 1, 2 ** 31 - 2] + [rng.randrange(0, 2 ** 31) for _ in range(24)]:
            if 0 <= n < 2 ** 31:
                assert fdiv(n, m, l) == n // d, (d, n)


def test_split3_inverts_the_linear_index():
    for X, Y, Z in ((257, 257, 257), (259, 3, 5), (1, 1, 7), (514, 1, 1), (33, 65, 17)):
        for t in range(0, X * Y * Z, max(1, (X * Y * Z) // 1500)):
            a, b, c = split3(t, X, Y)
            assert (a, b, c) == (t % X, (t // X) % Y, t // (X * Y)), (X, Y, t)
