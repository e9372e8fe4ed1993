"""The per-stage algorithmic bytes and FLOPs behind bench.py's roofline fractions."""

import numpy as np

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
    assert roofline.sort_passes() == 4 and roofline.sort_passes(radix_bits=10) == 3
    assert roofline.sort_passes(key64=True) == 8 and roofline.sort_passes(key64=True, radix_bits=10) == 8
    assert roofline.stage_bytes(n, radix_bits=10)["sort"] == 3 * 16 * n


def test_walk_flops_and_fractions():
    assert roofline.walk_flops(10, 5, 3) == 200 + 120 + 54
    assert roofline.walk_flops(0, 1, 0, quad=True) == 54
    gbs, frac = roofline.hbm_fraction(6.5e9, 1.0, 6500.0)
    assert abs(gbs - 6500.0) < 1e-9 and abs(frac - 1.0) < 1e-12
    rate, f = roofline.issue_fraction(1163.28e6, 1.0, 148, 1965.0)
    assert abs(rate - 1163.28) < 1e-6 and abs(f - 1.0) < 1e-9


def test_sph_roofline_reads_the_committed_profile():
    # bench.py's gas-mode roofline: instructions per gas particle from the profile in
    # profiles/, over the SPH stage time, against one warp instruction per scheduler-clock.
    import importlib.util
    import os

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    r = bench.sph_roofline(1 << 20, {"ms_sph": 28.0, "ms_sph_density": 13.0}, {"sm_max_mhz": 1965.0})
    per = r["instructions_per_gas"]
    assert per["density_instructions_per_gas"] > 1000 and per["hydro_instructions_per_gas"] > 1000
    want = (per["density_instructions_per_gas"] + per["hydro_instructions_per_gas"]) * (1 << 20) / 28e-3 / 1e9
    assert abs(r["achieved"] - want) < 1e-6 and 0.0 < r["frac"] < 1.0
    assert bench.SPH_LAUNCHES_PER_STEP == 34


def test_gas_star_mix_workload():
    from galaxy_b200 import workloads

    st = workloads.gas_star_mix(1000, 3000, seed=1)
    gas = st.kind == 1
    assert gas.sum() == 1000 and abs(st.mass.sum() - 1.0) < 1e-12
    assert np.abs(st.pos[gas]).max() <= 1.0 and np.abs(st.pos[~gas]).max() <= 3.0
    assert np.array_equal(st.pos, workloads.gas_star_mix(1000, 3000, seed=1).pos)
