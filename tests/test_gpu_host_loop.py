"""dgb_advance_host: the time loop with the state of record in host memory.  Every step uploads
the state, advances it one step and downloads the result, the copies in element chunks on two copy
streams.  It must give bit for bit the states, times and statuses of the same steps taken one at a
time through dgb_set_state / dgb_advance / dgb_get_state: 2D tiled and generic grids, 1D, SSP-RK3
and RK4, CFL and fixed steps, fewer elements than copy chunks, pinned and pageable host arrays, the
mixed form with the learned indicator scoring every few steps, and a host-injected NaN."""
import numpy as np
import pytest
import torch

import dg_b200 as dgb
from dg_b200 import _ffi as F
from dg_b200 import learned as L

pytestmark = pytest.mark.gpu

WALLS = ("reflective", "transmissive", "reflective", "transmissive")

CASES = [
    # id, dim, order, nx, ny, x1, bc, flux, limiter, ic, scheme, dt, steps
    ("2d_p2_rus_m2l_tiled", 2, 2, 64, 32, 2.0, WALLS, "rusanov", "m2l", "shock_bubble", dgb.SSPRK3, 0.0, 6),
    ("2d_p2_roe_hrl_generic", 2, 2, 10, 6, 1.0, ("transmissive",) * 4, "roe", "hrl", "quadrants", dgb.RK4, 0.0, 5),
    ("2d_p3_roe_m2l", 2, 3, 32, 16, 2.0, WALLS, "roe", "m2l", "shock_bubble", dgb.SSPRK3, 0.0, 4),
    ("1d_p2_roe_m2l_rk4", 1, 2, 300, 1, 1.0, ("transmissive",) * 2, "roe", "m2l", "tube_noise", dgb.RK4, 0.0, 8),
    ("1d_p1_rus_none_tiny_fixed", 1, 1, 7, 1, 1.0, ("transmissive",) * 2, "rusanov", "none", "tube_noise",
     dgb.SSPRK3, 1e-3, 5),
]


def make(case):
    """The problem and its initial state, limited as the reference limits it before its loop."""
    _, dim, order, nx, ny, x1, bc, flux, lim, ic, _scheme, _dt, _steps = case
    prob = dgb.Problem.structured(dim, order, nx, ny, 0.0, x1, 0.0, 1.0, bc, flux=flux, limiter=lim, cfl=0.3)
    U0 = prob.init_state(ic, seed=3)
    if lim != "none":
        s = dgb.DGSolver(prob)
        try:
            U0 = s.limit(U0)
        finally:
            s.close()
    return prob, U0


def one_step_at_a_time(s, U0, scheme, dt, steps):
    U = U0.copy()
    t = 0.0
    for _ in range(steps):
        s.set_state(U)
        t += s.advance(1, dt, scheme=scheme)
        s.get_state(out=U)
    return U, t


@pytest.mark.parametrize("pinned", [True, False], ids=["pinned", "pageable"])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_host_loop_matches_single_steps(case, pinned):
    prob, U0 = make(case)
    scheme, dt, steps = case[10], case[11], case[12]
    s = dgb.DGSolver(prob)
    try:
        ref, t_ref = one_step_at_a_time(s, U0, scheme, dt, steps)
        if pinned:
            buf = torch.empty(U0.size, dtype=torch.float64, pin_memory=True)
            U = buf.numpy()
        else:
            U = np.empty(U0.size)
        U[:] = U0
        t = s.advance_host(U, steps, dt, scheme=scheme)
        # the resident state is the last step's result too
        resident = s.get_state()
    finally:
        s.close()
    assert np.isfinite(ref).all() and t_ref > 0
    assert np.array_equal(U, ref)
    assert np.array_equal(resident, ref)
    assert t == t_ref


def test_host_loop_learned_indicator_interval():
    """Mixed form + learned indicator scoring every 4th step: one dgb_advance_host call of 8 steps
    equals a dgb_set_state followed by one dgb_advance of 8 steps (the call scores its first step and
    keeps the interval), downloaded once."""
    prob = dgb.Problem.structured(2, 2, 64, 32, 0.0, 2.0, 0.0, 1.0, WALLS, flux="rusanov", limiter="m2l", cfl=0.3)
    U0 = prob.init_state("shock_bubble", seed=5)
    params, _ = L.load()
    s = dgb.DGSolver(prob)
    try:
        s.set_form("mixed")
        L.set_indicator(s, params, 0.2, every=4)
        s.set_state(U0)
        t_ref = s.advance(8)
        ref = s.get_state()
        U = U0.copy()
        t = s.advance_host(U, 8)
    finally:
        s.close()
    assert np.isfinite(ref).all()
    assert np.array_equal(U, ref)
    assert t == t_ref


def test_host_loop_nonfinite_state_is_reported():
    """A NaN put into the host state stops the loop with DGB_ERR_NONFINITE, and the context still
    advances a clean state afterwards."""
    prob, U0 = make(CASES[0])
    s = dgb.DGSolver(prob)
    try:
        U = U0.copy()
        U[17] = np.nan
        with pytest.raises(dgb.DGBError) as e:
            s.advance_host(U, 3)
        assert e.value.code == F.ERR_NONFINITE
        U = U0.copy()
        t = s.advance_host(U, 2)
        assert t > 0 and np.isfinite(U).all()
    finally:
        s.close()


def test_host_loop_rejects_bad_arrays():
    prob, U0 = make(CASES[4])
    s = dgb.DGSolver(prob)
    try:
        with pytest.raises(ValueError):
            s.advance_host(U0[:-1].copy(), 1)
        with pytest.raises(ValueError):
            s.advance_host(U0.astype(np.float32), 1)
    finally:
        s.close()
