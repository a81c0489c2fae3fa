"""Arithmetic claims the decode kernel rests on, checked on the CPU."""
import os


def test_division_by_three_is_correctly_rounded(oracle):
    """RN(x * RN(1/3)) corrected once by the exact fma remainder equals IEEE x / 3 for every
    float with |x| <= 1.5, the only inputs hardgelu divides (2 x 1,069,547,521 values)."""
    assert oracle.L.orc_check_div3(os.cpu_count() or 1) == 0
