"""The EXACT mode's divisions (step_core.cuh: div3_rn for the moments, div_rn
for the collision) give the correctly rounded quotient: checked against IEEE
division on random doubles across exponents and random divisors, each with a
planted wrong variant to show the check can fail."""
from oracle.bindings import oracle_lib


def test_div3_matches_ieee_division():
    assert oracle_lib().oracle_check_div3(5_000_000, 20261203, 0) == 0


def test_div3_check_detects_a_planted_error():
    assert oracle_lib().oracle_check_div3(1_000_000, 7, 1) > 1000


def test_checked_division_matches_ieee_division():
    import ctypes

    fb = ctypes.c_long()
    assert oracle_lib().oracle_check_div(5_000_000, 424242, 0, ctypes.byref(fb)) == 0
    # zeros (both signs) are returned as they are; the tiny samples (about 1
    # in 1000) take the IEEE fallback; other rejections would be rare near-ties
    assert 0 < fb.value < 5_000_000 // 100


def test_checked_division_detects_a_planted_error():
    import ctypes

    fb = ctypes.c_long()
    assert oracle_lib().oracle_check_div(2_000_000, 99, 1, ctypes.byref(fb)) > 1000
