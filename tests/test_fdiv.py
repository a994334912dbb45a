"""The kernels' run-time division (FDiv in openmolcas_b200/csrc/kern_common.cuh):
q = umulhi(o, m) + (o & k) with m = (2^32 - 1) / n + 1 (k = all ones for n = 1,
else 0).  The host planners only launch work whose loop extents satisfy
o * n < 2^32 (grad_div_bound in grad.cu, the bound in eri.cu); this checks that
below that bound the quotient is exact, and that the bound is where it can
first fail."""
import numpy as np

MASK = (1 << 32) - 1


def fq(o, n):
    m = 0 if n == 1 else (MASK // n + 1) & MASK
    k = MASK if n == 1 else 0
    return ((o * m) >> 32) + (o & k)


def test_exact_below_bound_small_divisors():
    for n in range(1, 1025):
        lim = ((1 << 32) - 1) // n  # largest o with o * n < 2^32
        for o in list(range(0, 3 * n)) + list(range(max(0, lim - 3 * n), lim + 1)):
            assert fq(o, n) == o // n, (n, o)


def test_exact_below_bound_random_divisors():
    rng = np.random.default_rng(3)
    for n in rng.integers(2, 1 << 20, 2000).tolist():
        lim = ((1 << 32) - 1) // n
        for o in [lim, lim - 1, lim - n, int(rng.integers(0, lim + 1)), n - 1, n, 2 * n - 1]:
            if 0 <= o <= lim:
                assert fq(o, n) == o // n, (n, o)


def test_bound_is_needed():
    # n = 3: m exceeds 2^32 / 3 by 2/3, so o/3 is overestimated by 2 o / (3 2^32);
    # with o = 2 (mod 3) that first reaches the next integer at o >= 2^31,
    # above the planners' bound 2^32 / 3
    n = 3
    o = (1 << 31) + ((2 - (1 << 31)) % 3)
    assert o % 3 == 2 and fq(o, n) != o // n and fq(o - 3, n) == (o - 3) // n
    assert o * n >= 1 << 32
