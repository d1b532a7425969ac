"""The render decode's interpolation weight (t - f0) / (f1 - f0) (src/render_temporal_decode.cpp:
129-130) is formed without a division: RN(1/b) once per key interval, then a Markstein-corrected
product per frame.  It must equal IEEE single-precision division bit for bit on every pair the
decode can meet: integer frames 0 < a < b <= 65535 (the widest span a 16-bit key frame allows)."""
import pytest

pytestmark = pytest.mark.gpu


def test_interval_quotient_equals_ieee_division_exhaustively(vbt, cuda):
    bad, first = vbt.selftest_key_division(65535)
    assert bad == 0, f"{bad} mismatches, first b={first >> 16} a={first & 0xFFFF}"


def test_selftest_rejects_out_of_range_spans(vbt, cuda):
    for b_max in (0, 1, 65536):
        with pytest.raises(vbt.VbtError):
            vbt.selftest_key_division(b_max)
