"""The certified straight-line FP64 division and square root of the FP64 RK45 attempts
(csrc/dms_fastmath.cuh) against IEEE `/` and sqrt on the B200 (B200 required).

Whenever a certificate holds, the result must have the same bits as the IEEE operation; a
failed certificate only sends the attempt back to IEEE arithmetic.  The operands cover the
trajectory ranges, arbitrary bit patterns (NaN, infinities, subnormals, zeros), quotients a
few ulp from representable values and exact quotients.  Failed certificates must stay rare
(they cost a repeated attempt) outside the arbitrary-bit-pattern class."""
import pytest

from engine_fixtures import dms_b200

pytestmark = pytest.mark.gpu


def test_certified_division_and_root_equal_ieee():
    with dms_b200.Engine(0) as e:
        n = 1 << 26
        div_bad, div_fallback, sqrt_bad, sqrt_fallback = e.check_certified_math(n, seed=12345)
    print({"n": n, "div_mismatch": div_bad, "div_fallback": div_fallback, "sqrt_mismatch": sqrt_bad,
           "sqrt_fallback": sqrt_fallback})
    assert div_bad == 0 and sqrt_bad == 0
    # a quarter of the operands are arbitrary bit patterns (many NaN, infinite or subnormal)
    assert div_fallback < 0.3 * n and sqrt_fallback < 0.3 * n
