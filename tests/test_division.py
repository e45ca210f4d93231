"""The occlusion rows' quotient against the IEEE division.

The pair test forms each light row's quotient -D / B from a reciprocal
RN(1/B) hoisted out of its row loop and two Markstein correction steps, in
place of a division per row, wherever the pair's coefficients lie in the
ranges that keep the method free of underflow and overflow; the reciprocal
comes from the hardware approximation and one Newton-Raphson step.  The masks
then stay those of the reference only if the reciprocal is the correctly
rounded one and the quotient equals the division's in every bit: the
library's device self-check enumerates every reciprocal of the admitted range
and compares the quotient over random operands of the admitted ranges,
quotients next to rounding midpoints and quotients at small integers (where
the rows' round-up conversion turns).
"""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_row_quotient_equals_ieee_division(cuda_ok, fdzb, seed):
    trials = 1 << 26
    mismatches, checked = fdzb.check_division(trials, seed)
    assert checked > (140 << 24) + 2 * trials   # every reciprocal; three cases a trial, a few out of range
    assert mismatches == 0, f"{mismatches} of {checked} quotients differ from __fdiv_rn"
