"""The per-stage algorithmic bytes and FLOPs behind bench.py's roofline fractions."""

from galaxy_b200 import roofline


def test_stage_bytes_scale_and_key_width():
    n = 1 << 20
    b30 = roofline.stage_bytes(n)
    b63 = roofline.stage_bytes(n, key64=True)
    assert b30["sort"] == 4 * 16 * n and b63["sort"] == 8 * 24 * n
    assert b30["morton"] == 28 * n and b63["morton"] == 32 * n
    assert roofline.stage_bytes(2 * n)["build"] == 2 * b30["build"]
    assert roofline.stage_bytes(n, quad=True)["build"] - b30["build"] == 80 * n
    assert b30["walk"] == 140 * n


def test_walk_flops_and_fractions():
    assert roofline.walk_flops(10, 5, 3) == 200 + 120 + 54
    assert roofline.walk_flops(0, 1, 0, quad=True) == 54
    gbs, frac = roofline.hbm_fraction(6.5e9, 1.0, 6500.0)
    assert abs(gbs - 6500.0) < 1e-9 and abs(frac - 1.0) < 1e-12
    rate, f = roofline.issue_fraction(1163.28e6, 1.0, 148, 1965.0)
    assert abs(rate - 1163.28) < 1e-6 and abs(f - 1.0) < 1e-9
