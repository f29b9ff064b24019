"""Slab mode on one GPU: the grid split into 2 to 4 y-slabs with ghost rows, every slab in this
process on its own device context, ghost rows refreshed before every stage by device-to-device
copies and the CFL wave speed max-reduced over the slabs (dg_b200.slab.LocalTransport), against the
whole grid advanced by dgb_advance.  Walls, periodic and transmissive y boundaries; p = 1..3;
SSP-RK3 and RK4; CFL and fixed steps; hrl, m2l, none; a mass fraction; GAMCONS.  The owned rows must match
the whole-grid run within 1e-13 of the state's scale (the slabs' meshes and the whole grid's differ
in the last bit of their coordinates on non-dyadic extents), and the time advanced must agree.
Without the exchange the slabs drift apart from the whole-grid run (negative control)."""
import numpy as np
import pytest

import dg_b200 as dgb
from dg_b200 import slab as S

pytestmark = pytest.mark.gpu

WALLS = ("reflective", "transmissive", "reflective", "transmissive")
PERIODIC_Y = ("periodic", "transmissive", "periodic", "transmissive")

CASES = [
    # id, order, nx, ny, nslabs, bc, flux, limiter, ic, scheme, dt, steps, extra options
    ("p2_rus_m2l_walls_2", 2, 64, 32, 2, WALLS, "rusanov", "m2l", "shock_bubble", dgb.SSPRK3, 0.0, 12, {}),
    ("p2_roe_hrl_periodic_3", 2, 64, 48, 3, PERIODIC_Y, "roe", "hrl", "quadrants", dgb.RK4, 0.0, 6, {}),
    ("p3_roe_m2l_open_2", 3, 32, 20, 2, ("transmissive",) * 4, "roe", "m2l", "shock_bubble", dgb.SSPRK3, 0.0, 6, {}),
    ("p1_rus_none_walls_4", 1, 64, 32, 4, WALLS, "rusanov", "none", "quadrants", dgb.SSPRK3, 2e-4, 10, {}),
    ("p2_rus_m2l_periodic_2", 2, 32, 24, 2, PERIODIC_Y, "rusanov", "m2l", "quadrants", dgb.SSPRK3, 0.0, 8, {}),
    ("p2_roe_m2l_walls_3_y1", 2, 64, 40, 3, WALLS, "roe", "m2l", "shock_bubble", dgb.SSPRK3, 0.0, 8, {"n_mass": 1}),
    ("p2_roe_hrl_walls_2_gamcons", 2, 64, 32, 2, WALLS, "roe", "hrl", "shock_bubble", dgb.RK4, 0.0, 6,
     {"gamma_model": "gamcons"}),
]


def setup(case):
    _, order, nx, ny, ns, bc, flux, lim, ic, scheme, dt, steps, extra = case
    x1 = 2.0 if ic == "shock_bubble" else 1.0
    dec = S.Decomposition(order, nx, ny, ns, 0.0, x1, 0.0, 1.0, bc, flux=flux, limiter=lim, cfl=0.3, **extra)
    prob = dec.global_problem()
    U0 = prob.init_state(ic, seed=11)
    whole = dgb.DGSolver(prob)
    if lim != "none":
        U0 = whole.limit(U0)
    return dec, prob, U0, whole


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_slabs_reproduce_the_whole_grid(case):
    dec, prob, U0, whole = setup(case)
    scheme, dt, steps = case[9], case[10], case[11]
    try:
        whole.set_state(U0)
        t_whole = whole.advance(steps, dt, scheme=scheme)
        ref = whole.get_state()
    finally:
        whole.close()
    run = S.SlabRun(dec, range(dec.nslabs), S.LocalTransport())
    try:
        run.set_global_state(U0)
        t = run.advance(steps, dt, scheme=scheme)
        got = run.global_state()
    finally:
        run.close()
    assert np.isfinite(ref).all()
    assert abs(t - t_whole) <= 1e-13 * t_whole
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max(), np.abs(got - ref).max()


class NoExchange(S.LocalTransport):
    def __init__(self):
        super().__init__(captured=False)  # the phase-level step driven from here, without exchanges

    def exchange(self, run):
        pass


@pytest.mark.parametrize("case", CASES[:2], ids=[c[0] for c in CASES[:2]])
def test_captured_local_step_equals_the_eager_phase_level_step(case):
    """dgb_slabs_advance_local (one graph per step of every slab) against the same slabs driven
    phase by phase from Python: the same arithmetic, bit for bit, and the same time."""
    dec, prob, U0, whole = setup(case)
    whole.close()
    scheme, dt, steps = case[9], case[10], case[11]
    out = {}
    for captured in (False, True):
        run = S.SlabRun(dec, range(dec.nslabs), S.LocalTransport(captured=captured))
        try:
            run.set_global_state(U0)
            t = run.advance(steps, dt, scheme=scheme)
            t += run.advance(1, dt, scheme=scheme)  # a second call replays the captured step
            out[captured] = (t, run.global_state())
        finally:
            run.close()
    assert out[True][0] == out[False][0]
    assert np.array_equal(out[True][1], out[False][1])


def test_without_the_exchange_the_slabs_drift():
    case = CASES[0]
    dec, prob, U0, whole = setup(case)
    try:
        whole.set_state(U0)
        whole.advance(case[11], 0.0, scheme=case[9])
        ref = whole.get_state()
    finally:
        whole.close()
    run = S.SlabRun(dec, range(dec.nslabs), NoExchange())
    try:
        run.set_global_state(U0)
        run.advance(case[11], 0.0, scheme=case[9])
        got = run.global_state()
    finally:
        run.close()
    assert np.abs(got - ref).max() > 1e-6 * np.abs(ref).max()


def test_slab_mode_rejections_and_phase_order():
    prob = dgb.Problem.structured(2, 2, 32, 16, flux="rusanov", limiter="m2i", cfl=0.3, thresholds=(0.05,))
    s = dgb.DGSolver(prob)
    try:
        with pytest.raises(dgb.DGBError):
            s.set_ghost_rows(2, 2)  # sensor flags follow the reference's element order across rows
    finally:
        s.close()
    prob = dgb.Problem.structured(2, 2, 32, 16, flux="rusanov", limiter="m2l", cfl=0.3)
    s = dgb.DGSolver(prob)
    try:
        with pytest.raises(dgb.DGBError):
            s.set_ghost_rows(8, 8)  # no owned rows left
        s.set_ghost_rows(2, 2)
        s.set_state(prob.init_state("quadrants", seed=1))
        with pytest.raises(dgb.DGBError):
            s.step_stage(0)          # no step open
        s.step_begin(dgb.SSPRK3, 0.0)
        with pytest.raises(dgb.DGBError):
            s.step_stage(1)          # stages run in order
        for k in range(3):
            s.step_stage(k)
        rc, dt = s.step_end()
        assert rc == 0 and dt > 0
        rc, _ = s.step_end()          # no step open: the status, not an exception (slabs agree first)
        assert rc == 1
    finally:
        s.close()
