"""Sensor-gated limiters (hri, m2i, pri, p0i), the primitive HR limiter (prl) and the sensors on the
GPU against the numpy oracle, at sizes and seeds the golden fixtures do not cover.

Flags must be identical (integer output, including the reference's index-order semantics);
limited states within 1e-12 relative; three SSP-RK3 steps within 1e-10.
"""
import numpy as np
import pytest

from conftest import perturbed_state, rel_err
from oracle import dg_oracle as O

pytestmark = pytest.mark.gpu

WALLS = ("reflective", "transmissive", "reflective", "transmissive")
CASES = [
    # id, dim, order, nx, ny, bc, flux, limiter, ic, thresholds
    ("2d_p2_hri_walls", 2, 2, 96, 40, WALLS, "rusanov", "hri", "shock_bubble", (0.01, 0.05, 0.01)),
    ("2d_p2_m2i_periodic", 2, 2, 64, 64, ("periodic",) * 4, "roe", "m2i", "quadrants", (0.02, 0.02, 0.02)),
    ("2d_p3_m2i_box", 2, 3, 30, 22, ("reflective",) * 4, "roe", "m2i", "quadrants", (0.02, 0.05)),
    ("2d_p1_pri", 2, 1, 70, 33, ("transmissive",) * 4, "roe", "pri", "quadrants", (0.02, 0.02)),
    ("2d_p2_p0i", 2, 2, 80, 40, ("transmissive",) * 4, "rusanov", "p0i", "shock_bubble", (0.05,)),
    ("2d_p2_prl_walls", 2, 2, 64, 32, WALLS, "rusanov", "prl", "shock_bubble", ()),
    ("2d_p2_shock_sensor_only", 2, 2, 96, 48, WALLS, "rusanov", "hri", "shock_bubble", (1e9, 0.01)),
    ("1d_p2_m2i", 1, 2, 500, 1, ("transmissive",) * 2, "roe", "m2i", "tube_noise", (0.01, 0.01, 0.01)),
    ("1d_p3_hri_wall", 1, 3, 200, 1, ("reflective",) * 2, "hll", "hri", "tube_noise", (0.01, 0.05)),
    ("1d_p1_pri_periodic", 1, 1, 300, 1, ("periodic",) * 2, "rusanov", "pri", "tube_noise", (0.001,)),
    ("1d_p2_p0i", 1, 2, 300, 1, ("transmissive",) * 2, "rusanov", "p0i", "tube_noise", (0.01,)),
    ("1d_p2_prl", 1, 2, 300, 1, ("transmissive",) * 2, "rusanov", "prl", "tube_noise", ()),
]


def make(case, seed):
    import dg_b200 as dgb
    _, dim, order, nx, ny, bc, flux, limiter, ic, th = case
    x1 = 2.0 if ic == "shock_bubble" else 1.0
    cfl = 0.15 if order == 3 else 0.3
    prob = dgb.Problem.structured(dim, order, nx, ny, 0.0, x1, 0.0, 1.0, bc, flux=flux, limiter=limiter, cfl=cfl,
                                  thresholds=th)
    return prob, O.Setup.from_problem(prob, th), perturbed_state(prob, ic, seed)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_gated_limiter_and_sensors(case):
    import dg_b200 as dgb
    prob, S, Uraw = make(case, seed=41)
    s = dgb.DGSolver(prob)
    try:
        if case[-1]:
            flags = s.sensors(Uraw)
            assert np.array_equal(flags, O.sensors(S, Uraw))
            assert 0 < np.count_nonzero(flags) < flags.size or case[4] == 1
        assert rel_err(s.limit(Uraw), O.limit(S, Uraw)) < 1e-12
    finally:
        s.close()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_gated_time_steps(case):
    import dg_b200 as dgb
    prob, S, Uraw = make(case, seed=43)
    U0 = O.limit(S, Uraw)
    s = dgb.DGSolver(prob)
    try:
        s.set_state(U0)
        s.advance(3, 0.0, scheme=dgb.SSPRK3)
        assert rel_err(s.get_state(), O.ssprk3_steps(S, U0, 0.0, 3)) < 1e-10
    finally:
        s.close()
