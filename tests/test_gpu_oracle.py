"""CUDA path (through the C ABI) against the numpy oracle at sizes and seeds the golden fixtures
do not cover: ragged grids (extents not multiples of the 32 x 4 element tile), tile-aligned grids
(tiled kernels), p = 1..3, all fluxes, both limiters, walls / periodic / transmissive
boundaries, one to ten passive mass fractions, the GAMCONS gamma model, the 1D shock-tube workload (1000 elements, p=2, Roe, m2l,
RK4) and the 2D shock-bubble workload at its full size (512 x 256 elements, p=2, Rusanov, m2l,
SSP-RK3).

Tolerances: 1e-12 relative per operator (residual, limiter, Minv solve, CFL step), 1e-10
relative after a few RK steps, and 1e-10 in relative L1 density after 100 steps.
"""
import numpy as np
import pytest

from conftest import l1_density_error, perturbed_state, rel_err
from oracle import dg_oracle as O

pytestmark = pytest.mark.gpu

WALLS = ("reflective", "transmissive", "reflective", "transmissive")

CASES = [
    # id, dim, order, nx, ny, bc, flux, limiter, ic
    ("2d_p2_rus_m2l_ragged_walls", 2, 2, 40, 18, WALLS, "rusanov", "m2l", "shock_bubble"),
    ("2d_p1_roe_hrl_ragged_periodic", 2, 1, 26, 14, ("periodic",) * 4, "roe", "hrl", "quadrants"),
    ("2d_p3_roe_m2l_ragged", 2, 3, 18, 10, ("transmissive",) * 4, "roe", "m2l", "shock_bubble"),
    ("2d_p2_roe_hrl_tiled_box", 2, 2, 64, 32, ("reflective",) * 4, "roe", "hrl", "quadrants"),
    ("2d_p2_rus_m2l_tiled_walls", 2, 2, 96, 20, WALLS, "rusanov", "m2l", "shock_bubble"),
    ("2d_p1_rus_m2l_tiled", 2, 1, 64, 8, ("transmissive",) * 4, "rusanov", "m2l", "quadrants"),
    # extents that are not tile multiples: full tiles by the tiled kernel (TMA tile loads for an even
    # nx, plain loads for an odd one), the right and top strips by the generic kernel
    ("2d_p2_rus_m2l_strips_walls", 2, 2, 100, 46, WALLS, "rusanov", "m2l", "shock_bubble"),
    ("2d_p3_roe_hrl_strips", 2, 3, 70, 21, ("transmissive",) * 4, "roe", "hrl", "quadrants"),
    ("2d_p2_roe_m2l_odd_nx_periodic", 2, 2, 65, 20, ("periodic",) * 4, "roe", "m2l", "quadrants"),
    ("2d_p3_rus_hrl_odd_nx_walls", 2, 3, 67, 9, WALLS, "rusanov", "hrl", "shock_bubble"),
    # p=3 with hrl between walls goes unstable at CFL 0.3 in the oracle as well; run it at 0.15
    ("1d_p3_hll_hrl_walls", 1, 3, 301, 1, ("reflective",) * 2, "hll", "hrl", "tube_noise", 0.15),
    ("1d_p1_rus_m2l_periodic", 1, 1, 257, 1, ("periodic",) * 2, "rusanov", "m2l", "tube_noise"),
    ("1d_p2_roe_none", 1, 2, 123, 1, ("transmissive",) * 2, "roe", "none", "tube_noise"),
    # one passive mass fraction (last entry: n_mass)
    ("2d_p2_roe_m2l_tiled_walls_y1", 2, 2, 64, 16, WALLS, "roe", "m2l", "shock_bubble", 0.3, 1),
    ("2d_p3_rus_hrl_tiled_periodic_y1", 2, 3, 32, 8, ("periodic",) * 4, "rusanov", "hrl", "quadrants", 0.3, 1),
    ("2d_p1_rus_m2l_tiled_box_y1", 2, 1, 64, 12, ("reflective",) * 4, "rusanov", "m2l", "quadrants", 0.3, 1),
    ("1d_p2_rus_m2l_y1", 1, 2, 201, 1, ("transmissive",) * 2, "rusanov", "m2l", "tube_noise", 0.3, 1),
    ("1d_p3_hll_hrl_walls_y1", 1, 3, 97, 1, ("reflective",) * 2, "hll", "hrl", "riemann", 0.15, 1),
    # two and three mass fractions
    ("2d_p2_roe_m2l_tiled_walls_y3", 2, 2, 64, 16, WALLS, "roe", "m2l", "shock_bubble", 0.3, 3),
    ("2d_p3_rus_hrl_tiled_periodic_y2", 2, 3, 32, 8, ("periodic",) * 4, "rusanov", "hrl", "quadrants", 0.3, 2),
    ("1d_p2_rus_m2l_y2", 1, 2, 201, 1, ("transmissive",) * 2, "rusanov", "m2l", "tube_noise", 0.3, 2),
    ("1d_p1_roe_hrl_periodic_y3", 1, 1, 150, 1, ("periodic",) * 2, "roe", "hrl", "riemann", 0.3, 3),
    # four to ten (2D on 32 x 2 tiles, the faces through one buffer, the limiter passes' arrays in
    # dynamic shared memory)
    ("2d_p2_rus_m2l_tiled_walls_y10", 2, 2, 64, 10, WALLS, "rusanov", "m2l", "shock_bubble", 0.3, 10),
    ("2d_p1_roe_hrl_tiled_periodic_y7", 2, 1, 64, 6, ("periodic",) * 4, "roe", "hrl", "quadrants", 0.3, 7),
    ("2d_p3_roe_m2l_tiled_box_y4", 2, 3, 32, 6, ("reflective",) * 4, "roe", "m2l", "quadrants", 0.3, 4),
    ("1d_p2_hll_m2l_y8", 1, 2, 180, 1, ("transmissive",) * 2, "hll", "m2l", "tube_noise", 0.3, 8),
    ("1d_p3_roe_hrl_walls_y6", 1, 3, 90, 1, ("reflective",) * 2, "roe", "hrl", "riemann", 0.15, 6),
    # extents that are not tile multiples: full tiles, then the strips with the generic kernel
    ("2d_p2_rus_m2l_strips_walls_y2", 2, 2, 100, 46, WALLS, "rusanov", "m2l", "shock_bubble", 0.3, 2),
    ("2d_p3_roe_hrl_strips_y5", 2, 3, 70, 21, ("transmissive",) * 4, "roe", "hrl", "quadrants", 0.3, 5),
    ("2d_p1_rus_m2l_strips_periodic_y1", 2, 1, 50, 10, ("periodic",) * 4, "rusanov", "m2l", "quadrants", 0.3, 1),
    # the GAMCONS gamma model (last entry); limiters hrl and none (the reference's M2limiting stops
    # for this model)
    ("2d_p2_rus_hrl_tiled_walls_gc", 2, 2, 64, 16, WALLS, "rusanov", "hrl", "shock_bubble", 0.3, 0, "gamcons"),
    ("2d_p1_roe_hrl_tiled_periodic_gc", 2, 1, 64, 8, ("periodic",) * 4, "roe", "hrl", "quadrants", 0.3, 0, "gamcons"),
    ("2d_p3_roe_none_tiled_box_gc", 2, 3, 32, 6, ("reflective",) * 4, "roe", "none", "quadrants", 0.1, 0, "gamcons"),
    ("2d_p2_roe_hrl_strips_walls_gc", 2, 2, 100, 46, WALLS, "roe", "hrl", "shock_bubble", 0.3, 0, "gamcons"),
    ("1d_p2_roe_hrl_gc", 1, 2, 211, 1, ("transmissive",) * 2, "roe", "hrl", "tube_noise", 0.3, 0, "gamcons"),
    ("1d_p1_hll_hrl_periodic_gc", 1, 1, 150, 1, ("periodic",) * 2, "hll", "hrl", "riemann", 0.3, 0, "gamcons"),
    ("1d_p3_rus_none_walls_gc", 1, 3, 77, 1, ("reflective",) * 2, "rusanov", "none", "tube_noise", 0.05, 0, "gamcons"),
]


def make(case, seed):
    import dg_b200 as dgb
    _, dim, order, nx, ny, bc, flux, limiter, ic = case[:9]
    cfl = case[9] if len(case) > 9 else 0.3
    n_mass = case[10] if len(case) > 10 else 0
    gamma_model = case[11] if len(case) > 11 else "gamncon"
    x1 = 2.0 if dim == 2 and ic == "shock_bubble" else 1.0
    prob = dgb.Problem.structured(dim, order, nx, ny, 0.0, x1, 0.0, 1.0, bc, flux=flux, limiter=limiter, cfl=cfl,
                                  n_mass=n_mass, gamma_model=gamma_model)
    S = O.Setup.from_problem(prob)
    U0 = O.limit(S, perturbed_state(prob, ic, seed))
    return prob, S, U0


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_operators_match_oracle(case):
    import dg_b200 as dgb
    prob, S, U0 = make(case, seed=17)
    s = dgb.DGSolver(prob)
    try:
        assert rel_err(s.dg_solver(U0), O.residual(S, U0)) < 1e-12
        assert rel_err(s.solve(1e-3, U0), O.solve(S, 1e-3, O.residual(S, U0))) < 1e-12
        Uraw = perturbed_state(prob, case[8], 23)
        assert rel_err(s.limit(Uraw), O.limit(S, Uraw)) < 1e-12
        dt = s.dt_from_cfl(U0)
        assert abs(dt - O.dt_from_cfl(S, U0)) <= 1e-13 * dt
    finally:
        s.close()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_time_steps_match_oracle(case):
    import dg_b200 as dgb
    prob, S, U0 = make(case, seed=29)
    s = dgb.DGSolver(prob)
    try:
        s.set_state(U0)
        s.advance(3, 0.0, scheme=dgb.SSPRK3)
        assert rel_err(s.get_state(), O.ssprk3_steps(S, U0, 0.0, 3)) < 1e-10
        dt = 0.5 * O.dt_from_cfl(S, U0)  # a fixed step inside the case's CFL limit
        s.set_state(U0)
        s.advance(2, dt, scheme=dgb.RK4)
        assert rel_err(s.get_state(), O.rk4_steps(S, U0, dt, 2)) < 1e-10
    finally:
        s.close()


def test_shock_tube_workload_100_steps_l1_density():
    """1D two-fluid shock tube: [0,1], 1000 elements, p=2, Roe, m2l, RK4, transmissive ends,
    seeded +-1e-3 density noise; 100 fixed steps of the CFL-0.4 size."""
    import dg_b200 as dgb
    prob = dgb.Problem.structured(1, 2, 1000, 1, 0.0, 1.0, 0.0, 1.0, ("transmissive",) * 2, flux="roe",
                                  limiter="m2l", cfl=0.4)
    S = O.Setup.from_problem(prob)
    U0 = prob.init_state("tube_noise", seed=5)
    dt = O.dt_from_cfl(S, U0)
    s = dgb.DGSolver(prob)
    try:
        s.set_state(U0)
        s.advance(100, dt, scheme=dgb.RK4)
        Ug = s.get_state()
    finally:
        s.close()
    Uo = O.rk4_steps(S, U0, dt, 100)
    i = prob.info
    assert l1_density_error(Ug, Uo, i.n_elem, i.n_fields, i.n_s) < 1e-10


def test_shock_bubble_small_100_steps_l1_density():
    """2D shock-bubble on a 32 x 16 grid (p=2, Rusanov, m2l, SSP-RK3, CFL step), 100 steps."""
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, 2, 32, 16, 0.0, 2.0, 0.0, 1.0, WALLS, flux="rusanov", limiter="m2l", cfl=0.3)
    S = O.Setup.from_problem(prob)
    U0 = O.limit(S, prob.init_state("shock_bubble", seed=7))
    s = dgb.DGSolver(prob)
    try:
        s.set_state(U0)
        s.advance(100, 0.0, scheme=dgb.SSPRK3)
        Ug = s.get_state()
    finally:
        s.close()
    Uo = O.ssprk3_steps(S, U0, 0.0, 100)
    i = prob.info
    assert l1_density_error(Ug, Uo, i.n_elem, i.n_fields, i.n_s) < 1e-10


def test_shock_bubble_mass_fraction_100_steps_l1():
    """The 2D shock-bubble with the bubble marked by a mass fraction (rho Y = rho inside), 64 x 32
    grid, p=2, Roe, m2l, SSP-RK3, CFL step, 100 steps: relative L1 of density and of rho Y."""
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, 2, 64, 32, 0.0, 2.0, 0.0, 1.0, WALLS, flux="roe", limiter="m2l", cfl=0.3,
                                  n_mass=1)
    S = O.Setup.from_problem(prob)
    U0 = O.limit(S, prob.init_state("shock_bubble", seed=7))
    s = dgb.DGSolver(prob)
    try:
        s.set_state(U0)
        s.advance(100, 0.0, scheme=dgb.SSPRK3)
        Ug = s.get_state()
    finally:
        s.close()
    Uo = O.ssprk3_steps(S, U0, 0.0, 100)
    i = prob.info
    assert i.n_fields == 6
    assert l1_density_error(Ug, Uo, i.n_elem, i.n_fields, i.n_s) < 1e-10
    A = Ug.reshape(i.n_elem, i.n_fields, i.n_s)[:, 5]
    B = Uo.reshape(i.n_elem, i.n_fields, i.n_s)[:, 5]
    assert np.abs(A - B).sum() / np.abs(B).sum() < 1e-10
    # the marker is carried, not created: its total changes only through the open x boundaries
    assert B.sum() > 0


def test_mass_fraction_configurations_outside_the_device_path_are_rejected():
    import dg_b200 as dgb
    bad = [dict(dim=2, order=2, nx=41, ny=8, limiter="m2l"),       # odd nx: no TMA tiles
           dict(dim=1, order=2, nx=50, ny=1, limiter="m2i", thresholds=(0.05,)),  # sensor-gated limiter
           dict(dim=1, order=2, nx=50, ny=1, limiter="prl")]
    for kw in bad:
        th = kw.pop("thresholds", ())
        prob = dgb.Problem.structured(kw["dim"], kw["order"], kw["nx"], kw["ny"], flux="rusanov", limiter=kw["limiter"],
                                      cfl=0.3, thresholds=th, n_mass=1)
        with pytest.raises(dgb.DGBError) as e:
            dgb.DGSolver(prob)
        assert e.value.code == 4
    # four or more mass fractions run on 32 x 2 tiles: a grid of one element row has none
    prob = dgb.Problem.structured(2, 2, 32, 1, flux="rusanov", limiter="m2l", cfl=0.3, n_mass=4)
    with pytest.raises(dgb.DGBError) as e:
        dgb.DGSolver(prob)
    assert e.value.code == 4
    prob = dgb.Problem.structured(2, 2, 32, 8, flux="rusanov", limiter="m2l", cfl=0.3, n_mass=1)
    s = dgb.DGSolver(prob)
    try:
        with pytest.raises(dgb.DGBError):
            s.set_form("mixed")
        with pytest.raises(dgb.DGBError):
            dgb.DGBatch([s])
    finally:
        s.close()


def test_gamcons_shock_bubble_100_steps_l1():
    """The 2D shock-bubble in the GAMCONS model (64 x 32, p=2, Roe, hrl, SSP-RK3, CFL step), 100
    steps: relative L1 of density and of rho/(gamma-1)."""
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, 2, 64, 32, 0.0, 2.0, 0.0, 1.0, WALLS, flux="roe", limiter="hrl", cfl=0.3,
                                  gamma_model="gamcons")
    assert prob.info.gamma_model == 1
    S = O.Setup.from_problem(prob)
    assert S.gamcons
    U0 = O.limit(S, prob.init_state("shock_bubble", seed=7))
    s = dgb.DGSolver(prob)
    try:
        s.set_state(U0)
        s.advance(100, 0.0, scheme=dgb.SSPRK3)
        Ug = s.get_state()
    finally:
        s.close()
    Uo = O.ssprk3_steps(S, U0, 0.0, 100)
    i = prob.info
    assert l1_density_error(Ug, Uo, i.n_elem, i.n_fields, i.n_s) < 1e-10
    A = Ug.reshape(i.n_elem, i.n_fields, i.n_s)[:, 4]
    B = Uo.reshape(i.n_elem, i.n_fields, i.n_s)[:, 4]
    assert np.abs(A - B).sum() / np.abs(B).sum() < 1e-10


def test_gamcons_rusanov_2d_breaks_down_like_the_reference():
    """The reference's 2D GAMCONS Rusanov flux takes the right alpha as the left one divided twice
    by rhoL (twod_multifluid_fluxes.h:50-53); on the shock-bubble its own arithmetic (the oracle)
    turns NaN at step 16.  The device path follows it step for step and then stops with the NaN
    time-step error instead of returning a NaN state."""
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, 2, 64, 32, 0.0, 2.0, 0.0, 1.0, WALLS, flux="rusanov", limiter="hrl", cfl=0.3,
                                  gamma_model="gamcons")
    S = O.Setup.from_problem(prob)
    U0 = O.limit(S, prob.init_state("shock_bubble", seed=7))
    s = dgb.DGSolver(prob)
    try:
        s.set_state(U0)
        s.advance(8, 0.0, scheme=dgb.SSPRK3)
        assert rel_err(s.get_state(), O.ssprk3_steps(S, U0, 0.0, 8)) < 1e-9
        with pytest.raises(dgb.DGBError) as e:
            s.advance(40, 0.0, scheme=dgb.SSPRK3)
        assert e.value.code == 6
    finally:
        s.close()


def test_gamcons_configurations_outside_the_device_path_are_rejected():
    """M2L stops with GAMCONS (as in the reference), and the device path has no GAMCONS variant of
    the sensors, of mass fractions, of the mixed form or of 2D grids without TMA tiles."""
    import dg_b200 as dgb
    bad = [dict(dim=2, order=2, nx=32, ny=8, limiter="m2l"),
           dict(dim=1, order=2, nx=50, ny=1, limiter="m2l"),
           dict(dim=2, order=2, nx=41, ny=8, limiter="hrl"),               # odd nx: no TMA tiles
           dict(dim=1, order=2, nx=50, ny=1, limiter="hri", thresholds=(0.05,)),
           dict(dim=1, order=2, nx=50, ny=1, limiter="prl"),
           dict(dim=1, order=2, nx=50, ny=1, limiter="hrl", n_mass=1)]
    for kw in bad:
        th = kw.pop("thresholds", ())
        nm = kw.pop("n_mass", 0)
        prob = dgb.Problem.structured(kw["dim"], kw["order"], kw["nx"], kw["ny"], flux="rusanov", limiter=kw["limiter"],
                                      cfl=0.3, thresholds=th, n_mass=nm, gamma_model="gamcons")
        with pytest.raises(dgb.DGBError) as e:
            dgb.DGSolver(prob)
        assert e.value.code == 4, kw
    prob = dgb.Problem.structured(2, 2, 32, 8, flux="rusanov", limiter="hrl", cfl=0.3, gamma_model="gamcons")
    s = dgb.DGSolver(prob)
    try:
        with pytest.raises(dgb.DGBError):
            s.set_form("mixed")
        with pytest.raises(dgb.DGBError):
            dgb.DGBatch([s])
    finally:
        s.close()


def test_shock_bubble_full_size_one_step():
    """The 2D workload at full size (512 x 256, p=2, Rusanov, m2l): residual, limiter and one
    SSP-RK3 step (CFL 0.3) against the oracle."""
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, 2, 512, 256, 0.0, 2.0, 0.0, 1.0, WALLS, flux="rusanov", limiter="m2l", cfl=0.3)
    S = O.Setup.from_problem(prob)
    Uraw = prob.init_state("shock_bubble", seed=7)
    s = dgb.DGSolver(prob)
    try:
        U0 = s.limit(Uraw)
        assert rel_err(U0, O.limit(S, Uraw)) < 1e-12
        assert rel_err(s.dg_solver(U0), O.residual(S, U0)) < 1e-12
        s.set_state(U0)
        s.advance(1, 0.0, scheme=dgb.SSPRK3)
        assert rel_err(s.get_state(), O.ssprk3_steps(S, U0, 0.0, 1)) < 1e-11
    finally:
        s.close()
