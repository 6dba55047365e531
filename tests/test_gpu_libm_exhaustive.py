"""Exhaustive check of the device logf / exp2f against glibc.

Every AQ step of every P-frame (compute_aq_quant_steps, res/residual.rs:116-167) goes
through f32::ln of an MB variance and f32::exp2 of a scaled log difference; on linux-gnu
those are glibc's logf and exp2f.  The device evaluates them in double precision, rounds to
float and applies a table of the inputs whose glibc result differs.  These tests run every
f32 of the reachable ranges (and beyond them) through the device functions, the single and
the four-wide batched logf, and compare bit for bit with the host's glibc.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bits(x):
    return int(np.float32(x).view(np.uint32))


def _run(which, lo, hi):
    from riv2_b200 import encoder as E
    bad, first = C.c_uint64(0), C.c_uint32(0)
    st = E.lib().riv_test_libm_range(which, lo, hi, C.byref(bad), C.byref(first))
    assert st == 0
    return bad.value, first.value


@pytest.mark.parametrize("which", [0, 2], ids=["logf", "logf_batched"])
def test_logf_every_f32_of_the_variance_range(which):
    # the AQ variance is floored at 4 and at most 255^2/4 + ... = 16256.25; the fix-up
    # table covers [4, 16384]: check all of it (about 1.0e8 inputs)
    bad, first = _run(which, _bits(4.0), _bits(16384.0))
    assert bad == 0, f"{bad} mismatches, first at {np.uint32(first).view(np.float32)!r}"


def test_exp2f_every_f32_with_magnitude_at_most_two():
    # the AQ exponent 0.8 * (ln var - mean) / 6 stays within |x| <= 1.11; check every f32
    # with |x| <= 2, both signs (about 2.1e9 inputs)
    for lo, hi in ((0, _bits(2.0)), (0x80000000, _bits(-2.0))):
        bad, first = _run(1, lo, hi)
        assert bad == 0, f"{bad} mismatches, first at {np.uint32(first).view(np.float32)!r}"
