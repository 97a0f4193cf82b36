"""The oracle's forward-mode (Dual) tangent against the reference's own
published Dual calibration record: twelve Newton iterations of
solver-2d/examples/m1_inverse_manning_demo.rs, whose output the reference
commits as papers/01_review/figures/data/m1_inverse_manning.csv (extracted to
tests/golden/reference_m1_inverse_manning.npz by tests/golden/make_golden.py).
Each iteration runs the f64 step for the dt sequence and the Dual step along
dn = 1 (the uniform Manning value is the variable)."""
import os

import numpy as np

from hydroflux_b200 import abi
from tests import cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                      "reference_m1_inverse_manning.npz")


def m1_config():
    w, t = (abi.HF_BC_WALL, 0.0), (abi.HF_BC_TRANSMISSIVE, 0.0)
    return abi.make_config(cfl=0.4, boundaries=abi.make_boundaries(w, w, t, t), max_dt=1e9,
                           max_steps=5000)


def test_oracle_tangent_matches_reference_newton_record(oracle):
    oracle.set_pow_mode("libm")
    z, h, hu, hv = cases.m1_state()
    cfg = m1_config()

    def centroid(n_value):
        n = np.full_like(z, n_value)
        run = oracle.sim_run(z, n, 1.0, 1.0, h, hu, hv, cfg, cases.M1_T_END, dt_log_cap=5000)
        assert run["status"] == 0 and run["t"] == cases.M1_T_END
        tan = oracle.tangent_run(z, n, np.ones_like(z), 1.0, 1.0, h, hu, hv, cfg, run["dts"])
        assert np.array_equal(tan["h"], run["h"])  # the Dual values are the f64 run
        return cases.m1_centroid(tan["h"][1], tan["dh"][1])

    rows, _ = cases.m1_newton(centroid)
    cases.assert_matches_m1_record(rows, np.load(GOLDEN)["table"])
