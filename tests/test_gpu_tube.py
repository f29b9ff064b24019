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


CASES_1D = [
    # order, flux, limiter, scheme, dt (0: CFL step), nsteps, elements, boundaries
    (2, "roe", "m2l", "rk4", 0.0, 40, 1000, ("transmissive",) * 2),
    (2, "roe", "m2l", "ssprk3", 0.0, 40, 1000, ("transmissive",) * 2),
    (1, "rusanov", "hrl", "rk4", 1e-4, 30, 777, ("reflective",) * 2),
    (3, "hll", "m2l", "ssprk3", 0.0, 25, 5000, ("reflective", "transmissive")),
    (3, "roe", "hrl", "rk4", 0.0, 25, 130, ("periodic",) * 2),
]


@pytest.mark.parametrize("case", CASES_1D, ids=[f"p{c[0]}_{c[1]}_{c[2]}_{c[3]}_{c[6]}" for c in CASES_1D])
def test_fused_1d_stages_equal_the_separate_kernels(case, monkeypatch):
    """1D elements in chain order: residual, stage update and limiter of a stage in one launch
    (each block of elements recomputes its two outside neighbours and limits from shared memory)
    against the separate residual and limiter kernels (DGB_1D_FUSED=0), over two calls in a row:
    the same states to rounding (the compiler may contract products into multiply-adds
    differently in the two kernels) and the same time."""
    import dg_b200 as dgb
    order, flux, lim, scheme, dt, n, ne, bc = case
    sch = dgb.RK4 if scheme == "rk4" else dgb.SSPRK3
    prob = dgb.Problem.structured(1, order, ne, 1, 0.0, 1.0, bc=bc, flux=flux, limiter=lim, cfl=0.4)
    d = np.load(GOLDEN / "run_d1_tube_p2_roe_m2l_1000.npz")
    base = d["U0"].reshape(1000, 4, 3)
    idx = (np.arange(ne) * 1000) // ne  # the shock tube's cell means resampled onto this grid
    U0 = np.repeat(base[idx].mean(axis=2)[:, :, None], order + 1, axis=2).reshape(-1)
    out = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("DGB_1D_FUSED", mode)  # read when the context is created
        s = dgb.DGSolver(prob)
        try:
            s.set_state(s.limit(U0))
            t = s.advance(n, dt, scheme=sch)
            t += s.advance(n // 2, dt, scheme=sch)
            out[mode] = (t, s.get_state(), s.last_timing())
        finally:
            s.close()
    (ts, Us, (ms_s, l_s)), (tf, Uf, (ms_f, l_f)) = out["0"], out["1"]
    print(f"1D {case}: {n // 2} steps separate {ms_s:.3f} ms ({l_s} launches), fused {ms_f:.3f} ms ({l_f})")
    assert np.isfinite(Uf).all()
    assert abs(tf - ts) <= 1e-13 * ts
    assert np.abs(Uf - Us).max() <= 1e-13 * np.abs(Us).max(), np.abs(Uf - Us).max()
