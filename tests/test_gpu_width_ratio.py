"""The FP64 kernels form the ratio of two mesh widths with a precomputed
reciprocal and two correction steps (width_ratio); the quotient must be the
division operator's, bit for bit, or the parity with the reference breaks.
This drives the library's self-test over 2^26 pseudo-random pairs of
positive operands: random significands and exponents, and the widths 10 / n
of every mesh side up to 65536."""
import ctypes

import pytest

from cloverleaf_b200 import library

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [1, 0xC10E, 2 ** 40 + 7])
def test_width_ratio_matches_division(seed):
    bad = ctypes.c_longlong(-1)
    assert library().cb_selftest_width_ratio(1 << 26, seed, ctypes.byref(bad)) == 0
    assert bad.value == 0
