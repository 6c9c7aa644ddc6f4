"""The solver's constraint direction d / |d| (physxcoopa_b200/csrc/pxb_quotient.cuh) against
IEEE division on the device.

The cloth and hair projections divide each component of d by its length; the library computes
the three quotients from one reciprocal (Markstein's method) instead of three IEEE divisions.
Equality with the reference needs every quotient rounded exactly as IEEE division rounds it:
the refined reciprocal must be the correctly rounded one for every divisor significand, and the
quotients must equal IEEE division on seeded random constraints (directions, random bit patterns
down to subnormals, quotients next to 1, signed zeros and +-|d|, lengths far outside a cloth's).
"""
import pytest

from physxcoopa_b200 import runtime as R

pytestmark = pytest.mark.gpu


def test_reciprocal_and_quotients_equal_ieee_division():
    ctx = R.Context(0)
    try:
        for seed in (0, 1):
            rcp_bad, q_bad = ctx.check_quotients(1 << 30, seed)
            assert rcp_bad == 0, f"{rcp_bad} divisor significands whose refined reciprocal is not correctly rounded"
            assert q_bad == 0, f"{q_bad} quotients differ from IEEE division (seed {seed})"
    finally:
        ctx.close()


def test_projection_equals_the_scalar_ieee_form():
    """The solver's projection (packed two-lane arithmetic, shared reciprocal) against the
    reference's scalar operations, every output bit, on random endpoint pairs."""
    ctx = R.Context(0)
    try:
        for seed in (0, 1):
            bad, first = ctx.check_projections(1 << 28, seed)
            assert bad == 0, f"{bad} projections differ (seed {seed}); first input {first}"
    finally:
        ctx.close()


def test_every_numerator_significand_over_a_slice_of_divisors():
    """2^11 divisor significands (evenly spread, plus both ends of the range) against all 2^23
    numerator significands. The full sweep (every one of the 2^23 divisors) runs with
    python -m physxcoopa_b200.check_division."""
    ctx = R.Context(0)
    try:
        bad = 0
        for first in (0, (1 << 22) - 512, (1 << 23) - 512):
            bad += ctx.check_quotient_significands(first, 512)
        bad += ctx.check_quotient_significands(1234567, 512)
        assert bad == 0
    finally:
        ctx.close()
