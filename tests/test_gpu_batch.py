"""The batched ensemble (dgb_batch_*): cases of several element classes advanced together against
each case advanced alone with dgb_advance (itself parity-tested against the reference), for every
tuning the autotuner can pick; end times, per-case statistics and the rejection of unsupported
cases.  1D cases run the same per-element code and must match bit for bit.  The 2D tile body is
compiled into two kernels that read the problem's metric from different memories (kernel
parameters alone, shared memory in the batch), and the compiler forms its fused multiply-adds
differently in the two: results agree to a few ulps, bounded here by 1e-13 of the state's scale."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL_2D = 1e-13


def same(prob, a, b):
    if prob.info.dim == 1:
        return np.array_equal(a, b)
    return np.abs(a - b).max() <= TOL_2D * np.abs(a).max()


def make_cases(dgb):
    """1D Riemann problems of every order and flux, two limiters and none, ragged sizes; 2D
    four-quadrant problems on tile-multiple grids, p = 1 and 2, Rusanov and Roe."""
    specs = []
    for k, (p, ne, flux, lim) in enumerate([(1, 200, "rusanov", "m2l"), (2, 333, "roe", "m2l"), (3, 517, "hll", "hrl"),
                                            (2, 1000, "rusanov", "m2l"), (1, 64, "roe", "none"),
                                            (3, 250, "rusanov", "m2l")]):
        specs.append(((1, p, ne, 1, 0.0, 1.0, 0.0, 1.0), flux, lim, "riemann", 100 + k))
    for k, (p, nx, ny, flux, bc) in enumerate([(2, 64, 32, "rusanov", "transmissive"), (2, 96, 64, "rusanov", "reflective"),
                                               (1, 64, 64, "roe", "transmissive"), (2, 32, 48, "roe", "periodic")]):
        specs.append(((2, p, nx, ny, 0.0, 1.0, 0.0, 1.0, bc), flux, "m2l", "quadrants", 200 + k))
    cases = []
    for geo, flux, lim, ic, seed in specs:
        if geo[0] == 1:
            prob = dgb.Problem.structured(1, geo[1], geo[2], 1, geo[4], geo[5], bc=("transmissive",) * 2, flux=flux,
                                          limiter=lim, cfl=0.3)
        else:
            prob = dgb.Problem.structured(2, geo[1], geo[2], geo[3], geo[4], geo[5], geo[6], geo[7], bc=(geo[8],) * 4,
                                          flux=flux, limiter=lim, cfl=0.3)
        cases.append((prob, prob.init_state(ic, seed=seed)))
    return cases


def alone(dgb, cases, nsteps):
    out = []
    for prob, U0 in cases:
        s = dgb.DGSolver(prob)
        s.set_state(U0)
        s.advance(nsteps, 0.0, scheme=dgb.SSPRK3)
        out.append(s.get_state())
        s.close()
    return out


def batched(dgb, cases, nsteps, tune=None, t_end=0.0):
    solvers = []
    for prob, U0 in cases:
        s = dgb.DGSolver(prob)
        s.set_state(U0)
        solvers.append(s)
    b = dgb.DGBatch(solvers)
    info = b.classes()
    if tune is not None:
        info = b.autotune(tune)
        for s, (prob, U0) in zip(solvers, cases):  # the tuner leaves the states alone
            assert np.array_equal(s.get_state(), U0)
    n = b.advance(nsteps, t_end)
    stats = b.case_stats()
    timing = b.last_timing()
    states = [s.get_state() for s in solvers]
    b.close()
    for s in solvers:
        s.close()
    return states, info, n, stats, timing


def test_batch_matches_cases_alone_bit_for_bit():
    import dg_b200 as dgb
    cases = make_cases(dgb)
    ref = alone(dgb, cases, 6)
    got, info, n, (t, steps, _), (ms, launches) = batched(dgb, cases, 6)
    assert n == 6 and np.all(steps == 6) and ms > 0 and launches > 0
    # classes: (dim, order, flux, limiter)
    keys = {(c["dim"], c["order"], c["flux"], c["limiter"]) for c in info}
    assert len(keys) == len(info) == 9
    for k, (a, b) in enumerate(zip(ref, got)):
        assert np.isfinite(a).all()
        assert same(cases[k][0], a, b), f"case {k}: max diff {np.abs(a - b).max()}"


def test_batch_autotuned_configurations_match():
    import dg_b200 as dgb
    cases = make_cases(dgb)
    ref = alone(dgb, cases, 4)
    got, info, n, _, _ = batched(dgb, cases, 4, tune=2)
    assert all(c["tuned_ns"] > 0 for c in info)
    for c in info:
        if c["dim"] == 2:
            assert (c["tile_w"], c["tile_h"]) in {(32, 4), (32, 2), (16, 8)}
        else:
            assert c["tile_w"] in (64, 128, 256)
    for k, (a, b) in enumerate(zip(ref, got)):
        assert same(cases[k][0], a, b), f"case {k}"


@pytest.mark.parametrize("shape", [(32, 2, 1), (16, 8, 1), (32, 4, 2)])
def test_batch_every_tile_shape_matches(shape):
    """Each 2D residual configuration the tuner can pick, set by hand, reproduces the plain path."""
    import dg_b200 as dgb
    cases = [c for c in make_cases(dgb) if c[0].info.dim == 2]
    ref = alone(dgb, cases, 3)
    solvers = []
    for prob, U0 in cases:
        s = dgb.DGSolver(prob)
        s.set_state(U0)
        solvers.append(s)
    b = dgb.DGBatch(solvers)
    for k, c in enumerate(b.classes()):
        b.set_tuning(k, *shape, ctas_per_sm=1)
    assert all((c["tile_w"], c["tile_h"], c["unroll"]) == shape for c in b.classes())
    b.advance(3)
    for s, r, (prob, _) in zip(solvers, ref, cases):
        assert same(prob, s.get_state(), r)
    with pytest.raises(dgb.DGBError):
        b.set_tuning(0, 24, 4)
    b.close()
    for s in solvers:
        s.close()


def test_batch_end_time_and_case_stats():
    """With an end time every case stops exactly there; its final state equals the case advanced
    alone by the same CFL steps and a last step cut to land on the end time."""
    import dg_b200 as dgb
    cases = make_cases(dgb)
    t_end = 2e-3
    states, _, n, (t, steps, wall), _ = batched(dgb, cases, 10000, t_end=t_end)
    assert n < 10000  # stopped once every case was done
    assert np.all(t == t_end)
    assert np.all(steps >= 1) and np.all(wall >= 0)
    assert len(set(steps.tolist())) > 1  # the cases' own CFL steps differ
    # (2D: ulp-level differences can shift a CFL step by an ulp, never the step count here)
    for k, ((prob, U0), m, U) in enumerate(zip(cases, steps, states)):
        s = dgb.DGSolver(prob)
        s.set_state(U0)
        tt = 0.0
        for _ in range(int(m) - 1):
            tt += s.advance(1, 0.0, scheme=dgb.SSPRK3)
        assert tt < t_end
        s.advance(1, t_end - tt, scheme=dgb.SSPRK3)
        assert same(prob, s.get_state(), U), f"case {k}"
        s.close()


def test_batch_rejects_unsupported_cases():
    import dg_b200 as dgb
    p = dgb.Problem.structured(2, 2, 40, 8, flux="rusanov", limiter="m2l", cfl=0.3)  # nx not a multiple of 32
    s = dgb.DGSolver(p)
    with pytest.raises(dgb.DGBError) as e:
        dgb.DGBatch([s])
    assert e.value.code == 4
    q = dgb.Problem.structured(1, 2, 100, flux="roe", limiter="m2i", cfl=0.3, thresholds=(0.05,))
    s2 = dgb.DGSolver(q)
    with pytest.raises(dgb.DGBError) as e:
        dgb.DGBatch([s2])
    assert e.value.code == 4
    with pytest.raises(dgb.DGBError):
        dgb.DGBatch([s2, s2])
    s.close()
    s2.close()


def test_batched_golden_cases_match_the_reference():
    """Reference golden cases advanced together in batches (1D and tiled 2D classes, p = 1-3,
    Rusanov / Roe / HLL, m2l / hrl): after the fixture's SSP-RK3 steps with each case's own CFL
    step, every case equals the reference's run (the harness's Shu-Osher steps over the reference
    operators, fixture key rk3c) within the parity tests' 1e-10."""
    import json
    from pathlib import Path
    import dg_b200 as dgb
    from conftest import problem_for, rel_err
    gold = Path(__file__).resolve().parent / "golden"
    names = ["d1_p2_roe_m2l", "d1_p1_rus_hrl_wall", "d1_p3_hll_m2l_periodic", "t2_p2_rus_m2l_walls",
             "t2_p1_roe_hrl_periodic", "t2_p2_roe_m2l_box"]
    fixtures, solvers = [], []
    for n in names:
        d = dict(np.load(gold / f"{n}.npz"))
        meta = json.loads(str(d.pop("meta")))
        s = dgb.DGSolver(problem_for(meta))
        s.set_state(d["U0"])
        fixtures.append((meta, d))
        solvers.append(s)
    try:
        for nsteps in sorted({m["nsteps"] for m, _ in fixtures}):  # one batch per step count
            group = [(f, s) for f, s in zip(fixtures, solvers) if f[0]["nsteps"] == nsteps]
            b = dgb.DGBatch([s for _, s in group])
            try:
                b.advance(nsteps, 0.0)
            finally:
                b.close()
            for (meta, d), s in group:
                assert rel_err(s.get_state(), d["rk3c"]) < 1e-10, meta["name"]
    finally:
        for s in solvers:
            s.close()
