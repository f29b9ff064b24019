"""The 1D two-fluid shock tube of the benchmark configurations (1000 elements, p = 2, Roe, m2l, RK4
with the CFL step at CFL 0.4, transmissive ends, seeded density noise) against the reference's own
run of it (tests/golden/run_d1_tube_p2_roe_m2l_1000.npz): the plain FP64 form must stay within
1e-10 relative L1 density of the reference after 100 steps, and is reported (and bounded at 1e-8)
after the configuration's 2000 steps."""
import json

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def l1_rel(a, b, info, field=0):
    A = a.reshape(info.n_elem, info.n_fields, info.n_s)[:, field]
    B = b.reshape(info.n_elem, info.n_fields, info.n_s)[:, field]
    return float(np.abs(A - B).sum() / np.abs(B).sum())


def test_tube_rk4_cfl_run_matches_reference():
    import dg_b200 as dgb
    d = np.load(GOLDEN / "run_d1_tube_p2_roe_m2l_1000.npz")
    c = json.loads(str(d["meta"]))
    prob = dgb.Problem.structured(1, c["order"], c["nx"], 1, 0.0, 1.0, bc=("transmissive",) * 2, flux=c["flux"],
                                  limiter=c["limiter"], cfl=c["cfl"])
    s = dgb.DGSolver(prob)
    try:
        s.set_state(d["U0"])
        t100 = s.advance(100, 0.0, scheme=dgb.RK4)
        U100 = s.get_state()
        t2000 = t100 + s.advance(1900, 0.0, scheme=dgb.RK4)
        U2000 = s.get_state()
    finally:
        s.close()
    i = prob.info
    e100, e2000 = l1_rel(U100, d["U100"], i), l1_rel(U2000, d["U2000"], i)
    full = float(np.abs(U2000 - d["U2000"]).max() / np.abs(d["U2000"]).max())
    print(f"tube: relative L1 density after 100 steps {e100:.3e}, after 2000 {e2000:.3e} (t = {t2000:.6f}); "
          f"max |dU| / max |U| after 2000: {full:.3e}")
    assert e100 <= 1e-10
    assert e2000 <= 1e-8
