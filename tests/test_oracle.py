"""The numpy oracle (oracle/dg_oracle.py) pinned against the reference's own outputs.

Every golden fixture under tests/golden/ was produced by the reference's CPU build
(tests/golden/make_golden.py drives oracle/ref_harness.cc).  Here the oracle, given the same
reference setup arrays, must reproduce each operator: the residual f, DU = dt Minv f, the limiter,
the CFL step, RK4 steps and SSP-RK3 steps (fixed and CFL step).  The oracle computes in float64 with
the same formulas but different summation order (numpy matmul), so agreement is to 1e-12 relative
per operator and 1e-11 after the multi-step runs.
"""
import numpy as np
import pytest

from conftest import GOLDEN, golden_cases, load_golden, rel_err
from oracle import dg_oracle as O

CASES = golden_cases()


def setup_for(name):
    meta, d = load_golden(name)
    return meta, d, O.Setup.from_golden(meta, d)


@pytest.mark.parametrize("name", CASES)
def test_oracle_residual_and_solve(name):
    meta, d, S = setup_for(name)
    f = O.residual(S, d["U0"])
    assert rel_err(f, d["f"]) < 1e-12
    DU = O.solve(S, meta["dt"], d["f"])
    assert rel_err(DU, d["DU"]) < 1e-13


@pytest.mark.parametrize("name", CASES)
def test_oracle_limiter(name):
    meta, d, S = setup_for(name)
    assert rel_err(O.limit(S, d["Uraw"]), d["Ulim"]) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_oracle_cfl_dt(name):
    meta, d, S = setup_for(name)
    # the fixtures' decks hold CFL = -1 (fixed step), so ref_meta's scaled value is -Dx/(2p+1);
    # the golden CFL step was taken with deck CFL `cfl`, i.e. scaled CFL = cfl*Dx/(2p+1)
    dt = O.dt_from_cfl(S, d["U0"], meta["cfl"] * abs(S.cfl_scaled))
    assert abs(dt - float(d["dt_cfl"][0])) <= 1e-14 * abs(float(d["dt_cfl"][0]))


@pytest.mark.parametrize("name", CASES)
def test_oracle_time_steps(name):
    meta, d, S = setup_for(name)
    n = meta["nsteps"]
    assert rel_err(O.rk4_steps(S, d["U0"], meta["dt"], n), d["rk4"]) < 1e-11
    assert rel_err(O.ssprk3_steps(S, d["U0"], meta["dt"], n), d["rk3"]) < 1e-11


@pytest.mark.parametrize("name", CASES)
def test_oracle_cfl_time_steps(name):
    import dataclasses
    meta, d, S = setup_for(name)
    S = dataclasses.replace(S, cfl_scaled=meta["cfl"] * abs(S.cfl_scaled))
    assert rel_err(O.ssprk3_steps(S, d["U0"], 0.0, meta["nsteps"]), d["rk3c"]) < 1e-11


@pytest.mark.parametrize("name", ["d1_p3_hll_m2l_periodic", "d2_p2_roe_m2l_walls", "d2_p2_rus_hrl_box"])
def test_oracle_on_package_setup_arrays(name):
    """The oracle driven by the package's host setup (what the GPU parity tests at other sizes use)
    gives the reference's answers too."""
    from conftest import problem_for
    meta, d = load_golden(name)
    S = O.Setup.from_problem(problem_for(meta))
    assert rel_err(O.residual(S, d["U0"]), d["f"]) < 1e-12
    assert rel_err(O.limit(S, d["Uraw"]), d["Ulim"]) < 1e-12


@pytest.mark.parametrize("name", [c for c in CASES if "thresholds" in load_golden(c)[0]])
def test_oracle_sensors(name):
    """SENSOR::sensing flags (sequential CPU semantics) on the raw state, exactly."""
    meta, d, S = setup_for(name)
    assert np.array_equal(O.sensors(S, d["Uraw"]), d["sens"])


def test_tube_fixture_starts_from_the_limited_initial_state():
    """The 2000-step tube fixture's U0 is the reference limiter applied to the seeded initial state
    (the oracle's m2 limiter reproduces it)."""
    import json
    import dg_b200 as dgb
    d = np.load(GOLDEN / "run_d1_tube_p2_roe_m2l_1000.npz")
    c = json.loads(str(d["meta"]))
    prob = dgb.Problem.structured(1, c["order"], c["nx"], 1, 0.0, 1.0, bc=("transmissive",) * 2, flux=c["flux"],
                                  limiter=c["limiter"], cfl=c["cfl"])
    S = O.Setup.from_problem(prob)
    U = O.limit(S, prob.init_state(c["ic"], seed=c["seed"]))
    assert rel_err(U, d["U0"]) < 1e-12
    assert all(np.isfinite(d[k]).all() for k in ("U100", "U2000"))
