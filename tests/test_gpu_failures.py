"""Failure detection on the device path, in forms that fault and hang no GPU.

The reference stops its time loop when the CFL step is NaN or below 1e-14
(code/src/time_integration/rk.cc:147-148).  Here those conditions are found on the device and come
back as status codes (DGB_ERR_NONFINITE, DGB_ERR_DT_SMALL) after the step; the context stays
usable.  The tiled residual kernels wait on their TMA tile copies with a bounded poll loop; a wait
that runs out sets a flag, drains the copy with the default budget, skips the tile and the step
returns DGB_ERR_TIMEOUT.  The tests make each condition happen on purpose: a NaN written into the
state on the host, a state whose wave speed gives a step far below 1e-14, and a zero poll budget
for the first wait (dgb_set_wait_limit), so that the wait gives up before the copy lands.
"""
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
NONFINITE, DT_SMALL, TIMEOUT = 6, 7, 8


def tile_case():
    """The 32 x 8 p = 2 Rusanov m2l shock-bubble fixture (full tiles: the TMA tiled kernel)."""
    import dg_b200 as dgb
    d = dict(np.load(GOLD / "t2_p2_rus_m2l_walls.npz"))
    meta = json.loads(str(d.pop("meta")))
    x0, x1, y0, y1 = meta["dom"]
    prob = dgb.Problem.structured(2, meta["order"], meta["nx"], meta["ny"], x0, x1, y0, y1, tuple(meta["bc"]),
                                  flux=meta["flux"], limiter=meta["limiter"], cfl=meta["cfl"])
    return prob, d, meta


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def recovers(s, d, meta):
    """The context still advances the fixture's state to the reference's result."""
    import dg_b200 as dgb
    s.set_state(d["U0"])
    s.advance(meta["nsteps"], meta["dt"], scheme=dgb.SSPRK3)
    assert rel(s.get_state(), d["rk3"]) < 1e-10


def test_nan_in_state_stops_the_step_with_nonfinite():
    import dg_b200 as dgb
    prob, d, meta = tile_case()
    i = prob.info
    V = d["U0"].copy().reshape(i.n_elem, i.n_fields, i.n_s)
    V[100, 0, 4] = np.nan  # one nodal density of one element, written on the host
    V = V.reshape(-1)
    s = dgb.DGSolver(prob)
    try:
        with pytest.raises(dgb.DGBError) as e:
            s.dt_from_cfl(V)
        assert e.value.code == NONFINITE
        s.set_state(V)
        with pytest.raises(dgb.DGBError) as e:
            s.advance(1, 0.0, scheme=dgb.SSPRK3)
        assert e.value.code == NONFINITE
        recovers(s, d, meta)
    finally:
        s.close()


def test_tiny_cfl_step_stops_the_step_with_dt_small():
    import dg_b200 as dgb
    prob, d, meta = tile_case()
    i = prob.info
    # a uniform finite state moving at 1e16: CFL step ~1e-19, far below the reference's 1e-14
    rho, u, p, gam = 1.0, 1e16, 1.0, 1.4
    V = np.empty((i.n_elem, i.n_fields, i.n_s))
    V[:, 0], V[:, 1], V[:, 2] = rho, rho * u, 0.0
    V[:, 3] = p / (gam - 1.0) + 0.5 * rho * u * u
    V[:, 4] = 1.0 / (gam - 1.0)
    V = V.reshape(-1)
    s = dgb.DGSolver(prob)
    try:
        with pytest.raises(dgb.DGBError) as e:
            s.dt_from_cfl(V)
        assert e.value.code == DT_SMALL
        s.set_state(V)
        with pytest.raises(dgb.DGBError) as e:
            s.advance(1, 0.0, scheme=dgb.SSPRK3)
        assert e.value.code == DT_SMALL
        recovers(s, d, meta)
    finally:
        s.close()


@pytest.mark.parametrize("form", ["fp64", "mixed"])
def test_expired_tile_wait_returns_timeout_and_the_context_recovers(form):
    import dg_b200 as dgb
    prob, d, meta = tile_case()
    s = dgb.DGSolver(prob)
    try:
        s.set_form(form)
        s.set_wait_limit(0)  # every first wait on a tile copy gives up at once
        s.set_state(d["U0"])
        with pytest.raises(dgb.DGBError) as e:
            s.advance(1, meta["dt"], scheme=dgb.SSPRK3)
        assert e.value.code == TIMEOUT
        with pytest.raises(dgb.DGBError) as e:
            s.dg_solver(d["U0"])
        assert e.value.code == TIMEOUT
        s.set_wait_limit()  # default budget: the same context runs the fixture again
        if form == "fp64":
            recovers(s, d, meta)
            assert rel(s.dg_solver(d["U0"]), d["f"]) < 1e-12
        else:
            s.set_state(d["U0"])
            s.advance(meta["nsteps"], meta["dt"], scheme=dgb.SSPRK3)
            assert rel(s.get_state(), d["rk3"]) < 1e-5
    finally:
        s.close()
