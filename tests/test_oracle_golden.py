"""Pins the CPU oracle to the reference's own solver outputs.

tests/golden/reference_verif.npz holds the simulated depth profiles that the
reference wrote with its own solver (papers/01_review/figures/data/verif_*.csv,
made by solver-2d/examples/gen_verification_data.rs). The oracle, run on the
same setups with the reference's loop, must reproduce every printed digit.
"""
import os

import numpy as np
import pytest

from tests import cases

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_verif.npz"))


def run_free_loop(O, case):
    from hydroflux_b200 import abi
    bcs = abi.make_boundaries(*case["bcs"])
    z, n, dx, dy = case["z"], case["n"], case["dx"], case["dy"]
    h, hu, hv = case["h"], case["hu"], case["hv"]
    t = 0.0
    while t < case["t_end"]:
        dt = min(O.cfl_time_step(z, dx, dy, h, hu, hv, case["cfl"]), case["t_end"] - t)
        h, hu, hv = O.ssprk2_step(z, dx, dy, h, hu, hv, bcs, dt, n)
        if case["friction"] is not None:
            h, hu, hv = O.manning_friction_step(n, h, hu, hv, dt, case["friction"])
        t += dt
    return h, hu, hv


@pytest.mark.parametrize("builder", cases.VERIF_CASES, ids=lambda b: b.__name__)
def test_oracle_reproduces_reference_outputs(oracle, builder):
    case = builder()
    h, _, _ = run_free_loop(oracle, case)
    sim = cases.golden_profile(case, h)
    ref = GOLDEN[case["golden"]]
    assert sim.shape == ref.shape
    tol = 0.51 * 10.0 ** (-case["decimals"])  # one unit of the printed rounding
    np.testing.assert_allclose(sim, ref, rtol=0, atol=tol)
    # The match is in fact exact to the printed digits.
    assert np.array_equal(sim, ref)
