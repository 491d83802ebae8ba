"""CPU checks of the int8 path's arithmetic (BEAM_PREC_INT8): the slicing of
beam_run.cu (k_ring_scale, slice5, k_build_slices) and the level combination
of beam_tri_i8.cu, restated here in exact integer/float arithmetic.

- A value v with |v| < 2^e is a0 + a1 2^-8 + ... + a4 2^-32 (+ a remainder in
  [0, 2^-32)) in units of 2^(e-7), with a0 in [-128, 127] and a1..a4 in
  [0, 255]; each step of the cut is exact in FP64.
- The sum over a run of x z, formed from 19 slice pairs (i + j <= 5) as exact
  integer sums per level and combined in FP64, is within 2^-36 of the run's
  scale (sum |x| |z| at the legs' scales) of the exact product sum.
- The 32-bit accumulators cannot overflow for runs of up to I8_RUN_MAX = 2048
  triangles."""
from fractions import Fraction

import numpy as np

LEVELS, SLICES, RUN_MAX = 6, 5, 2048


def slice5(v: float, e: int):
    """slice5 of beam_run.cu: the five slices of v against 2^e (|v| < 2^e)."""
    u = np.ldexp(v, 7 - e)
    a = np.floor(u)
    rem = u - a
    out = [int(a)]
    for _ in range(1, SLICES):
        rem *= 256.0
        a = np.floor(rem)
        rem -= a
        out.append(int(a))
    return out


def scale_exp(values) -> int:
    """k_ring_scale: the smallest e with max |v| < 2^e (0 for all zeros)."""
    m = float(np.max(np.abs(values)))
    return 0 if m == 0.0 else int(np.frexp(m)[1])


def test_slices_reconstruct_the_value_within_one_last_digit():
    rng = np.random.default_rng(7)
    for _ in range(2000):
        vals = rng.standard_normal(16) * 10.0 ** rng.integers(-6, 6)
        e = scale_exp(vals)
        for v in vals:
            s = slice5(float(v), e)
            assert -128 <= s[0] <= 127 and all(0 <= d <= 255 for d in s[1:])
            approx = sum(Fraction(d) / Fraction(256) ** k for k, d in enumerate(s)) * Fraction(2) ** (e - 7)
            rem = Fraction(float(v)) - approx
            assert 0 <= rem < Fraction(2) ** (e - 7 - 32)


def test_slices_of_the_negated_value_are_not_negated_slices():
    # -Im is sliced on its own: for v = 1/3 against 2^0 the slices of -v differ
    # from the negated slices of v (digits 1-4 are unsigned)
    a, b = slice5(1.0 / 3.0, 0), slice5(-1.0 / 3.0, 0)
    assert a[0] == 42 and b[0] == -43 and all(0 <= d <= 255 for d in b[1:])
    assert b[1:] != [-d for d in a[1:]]


def run_sum_from_slices(x, z, ex, ez):
    """W = sum x z over a run from the slice pairs i + j < LEVELS, as the
    kernel forms it: exact integer level sums, then 2^(ex+ez-14) sum_L 2^-8L acc_L."""
    sx = [slice5(float(v), ex) for v in x]
    sz = [slice5(float(v), ez) for v in z]
    acc = [0] * LEVELS
    for a, b in zip(sz, sx):
        for i in range(SLICES):
            for j in range(SLICES):
                if i + j < LEVELS:
                    acc[i + j] += a[i] * b[j]
    w = float(acc[LEVELS - 1])
    for lvl in range(LEVELS - 2, -1, -1):
        w = w * 0.00390625 + float(acc[lvl])
    return np.ldexp(w, ex + ez - 14), acc


def test_run_sums_from_19_slice_pairs_are_within_2_pow_minus_36_of_the_run_scale():
    rng = np.random.default_rng(11)
    worst = 0.0
    for _ in range(300):
        n = int(rng.integers(1, 80))
        x = rng.standard_normal(n)
        z = rng.standard_normal(n) * 3.0
        ex, ez = scale_exp(x), scale_exp(z)
        w, _ = run_sum_from_slices(x, z, ex, ez)
        exact = sum(Fraction(float(a)) * Fraction(float(b)) for a, b in zip(x, z))
        scale = float(np.sum(np.abs(x))) * 2.0 ** ez  # |x| at its value, z at its scale
        err = abs(Fraction(w) - exact) / Fraction(scale)
        worst = max(worst, float(err))
    assert worst <= 2.0 ** -36, worst


def test_int32_accumulators_hold_the_longest_run():
    # per triangle and level: 2 parts x at most 5 slice pairs, each at most 255 x 255 in size
    bound = RUN_MAX * 2 * 5 * 255 * 255
    assert bound < 2 ** 31
