"""The EXACT mode's three-operation x/3 (kernels.cu, div3_rn) is the correctly
rounded quotient: checked against IEEE division on random doubles across
exponents, with a planted wrong variant to show the check can fail."""
from oracle.bindings import oracle_lib


def test_div3_matches_ieee_division():
    assert oracle_lib().oracle_check_div3(5_000_000, 20261203, 0) == 0


def test_div3_check_detects_a_planted_error():
    assert oracle_lib().oracle_check_div3(1_000_000, 7, 1) > 1000
