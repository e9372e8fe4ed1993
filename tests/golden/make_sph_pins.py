"""Extract the reference's frozen SPH output bits into sph_pins.json (run where a checkout
of the reference project exists; the JSON is what the tests read).

    python tests/golden/make_sph_pins.py <reference checkout>
    GALAXY_REFERENCE=<reference checkout> python tests/golden/make_sph_pins.py

Sources (the reference project's own regression pins):
  solvers/tests/sph_forces.rs `isothermal_regression_pins_pre_e1b_bits`: 8 accelerations
  of hydro_accelerations on random_points(42, 8, 3.0) / random_points(43, 8, 1.0),
  masses 1 + 0.1 i, rho 0.8 + 0.05 i, h 0.9 + 0.03 i, isothermal c_s = 1.3.
  solvers/tests/sph_cfl.rs `isothermal_cfl_pins_pre_e4a_bits`: max_stable_dt of
  random_points(21, 600, 2.5) / random_points(22, 600, 1.5), unit masses, all gas,
  default params, C_CFL = 0.25.
"""

import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GALAXY_REFERENCE")
if not REF:
    sys.exit("usage: make_sph_pins.py <reference checkout> (or set GALAXY_REFERENCE)")
HERE = os.path.dirname(os.path.abspath(__file__))


def bits_in(text: str, fn: str) -> list[str]:
    start = text.index(f"fn {fn}")
    end = text.index("\n}\n", start)
    return re.findall(r"from_bits\((0x[0-9a-f]+)\)", text[start:end])


forces = open(os.path.join(REF, "solvers/tests/sph_forces.rs")).read()
cfl = open(os.path.join(REF, "solvers/tests/sph_cfl.rs")).read()
hyd = bits_in(forces, "isothermal_regression_pins_pre_e1b_bits")
cb = bits_in(cfl, "isothermal_cfl_pins_pre_e4a_bits")
assert len(hyd) == 24 and len(cb) == 1
out = {
    "hydro_isothermal_8": {
        "source": "solvers/tests/sph_forces.rs isothermal_regression_pins_pre_e1b_bits",
        "pos_seed": 42, "vel_seed": 43, "n": 8, "pos_scale": 3.0, "vel_scale": 1.0, "c_s": 1.3,
        "acc_bits": [hyd[3 * i:3 * i + 3] for i in range(8)],
    },
    "cfl_isothermal_600": {
        "source": "solvers/tests/sph_cfl.rs isothermal_cfl_pins_pre_e4a_bits",
        "pos_seed": 21, "vel_seed": 22, "n": 600, "pos_scale": 2.5, "vel_scale": 1.5, "c_cfl": 0.25,
        "min_dt_bits": cb[0],
    },
}
with open(os.path.join(HERE, "sph_pins.json"), "w") as f:
    json.dump(out, f, indent=1)
print("wrote sph_pins.json")
