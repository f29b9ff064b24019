"""The benchmark's shock-bubble workloads over 100 steps against the reference's own runs.

Fixtures (tests/golden/make_golden.py, FULL): the reference CPU build (oracle/_ref, compiled from
the reference sources) advanced the seeded shock-bubble -- limited first, as the reference limits
its initial condition (code/src/time_integration/rk.cc:108-114) -- by 100 SSP-RK3 steps with the
CFL step (CFL 0.3) on [0, 2] x [0, 1], reflective bottom / top, transmissive left / right:
    512 x 256, p = 2, Rusanov, m2l   (the benchmark workload)
    256 x 128, p = 3, Roe, m2l       (the p = 3 Roe form, at the largest size the reference
                                      finishes in minutes)
They hold the reference's step sizes, the final cell means of density and energy, and the nodal
density of a band of element rows through the bubble.  The device path must reach the same time
and stay within 1e-10 relative L1 in density (the plain FP64 form's bar after 100 steps).
"""
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden"
CASES = ["run_d2_bubble_p2_rus_m2l_512x256", "run_d2_bubble_p3_roe_m2l_256x128"]


def l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


def run(name, form="fp64"):
    import dg_b200 as dgb
    d = dict(np.load(GOLD / f"{name}.npz"))
    m = json.loads(str(d.pop("meta")))
    x0, x1, y0, y1 = m["dom"]
    prob = dgb.Problem.structured(2, m["order"], m["nx"], m["ny"], x0, x1, y0, y1, tuple(m["bc"]), flux=m["flux"],
                                  limiter=m["limiter"], cfl=m["cfl"])
    s = dgb.DGSolver(prob)
    try:
        U0 = s.limit(prob.init_state("shock_bubble", seed=m["seed"]))
        s.set_form(form)
        s.set_state(U0)
        t = s.advance(m["steps"], 0.0, scheme=dgb.SSPRK3)
        U = s.get_state()
    finally:
        s.close()
    i = prob.info
    V = U.reshape(i.n_elem, i.n_fields, i.n_s)
    w = prob.array("phi_w").reshape(i.n_s, i.n_g).sum(axis=1) / 4.0
    r0, r1 = m["band"]
    return d, m, t, V, w, r0, r1


@pytest.mark.parametrize("name", CASES)
def test_plain_form_matches_the_reference_run_after_100_steps(name):
    d, m, t, V, w, r0, r1 = run(name)
    assert abs(t - m["t_final"]) <= 1e-10 * m["t_final"]
    assert l1(V[:, 0, :] @ w, d["rho_mean"]) < 1e-10
    assert l1(V[:, 3, :] @ w, d["E_mean"]) < 1e-10
    assert l1(V[r0 * m["nx"]:r1 * m["nx"], 0, :], d["rho_band"]) < 1e-10


@pytest.mark.parametrize("name", CASES)
def test_mixed_form_stays_near_the_reference_run(name):
    """The mixed form (FP32 contractions on FP64 anchors) over the same 100 steps: within 1e-5
    relative L1 of the reference in density and energy (per-field error of the approximate form)."""
    d, m, t, V, w, r0, r1 = run(name, "mixed")
    assert abs(t - m["t_final"]) <= 1e-6 * m["t_final"]
    assert l1(V[:, 0, :] @ w, d["rho_mean"]) < 1e-5
    assert l1(V[:, 3, :] @ w, d["E_mean"]) < 1e-5
    assert l1(V[r0 * m["nx"]:r1 * m["nx"], 0, :], d["rho_band"]) < 1e-5
