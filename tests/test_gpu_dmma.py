"""The p = 2 FP64 stage with its basis contractions on the FP64 tensor cores (DMMA,
dg_b200/csrc/device/tile2d_dmma.cuh, selected by DGB_TILE_KERNEL=dmma) against the default
one-thread-per-element tiled kernel.  Both are FP64 with the same point arithmetic and differ in the order of
their sums (and M^-1 folded into the DMMA lift tables), so one step agrees to 1e-13 relative and 20
steps to 1e-11; the results are not bit-identical, which shows that the DMMA kernel ran.  Cases:
Rusanov and Roe, SSP-RK3 and RK4, walls, periodic and transmissive boundaries, and a grid with
leftover strips (full tiles by the DMMA kernel, the strips by the generic kernel)."""
import os

import numpy as np
import pytest

import dg_b200 as dgb
from conftest import rel_err

pytestmark = pytest.mark.gpu

WALLS = ("reflective", "transmissive", "reflective", "transmissive")


def run(kind, prob, U0, dt, scheme, steps):
    os.environ["DGB_TILE_KERNEL"] = kind
    try:
        s = dgb.DGSolver(prob)
    finally:
        del os.environ["DGB_TILE_KERNEL"]
    try:
        s.set_state(U0)
        s.advance(1, dt, scheme=scheme)
        U1 = s.get_state()
        s.advance(steps - 1, dt, scheme=scheme)
        return U1, s.get_state()
    finally:
        s.close()


@pytest.mark.parametrize("flux,bc,nx,ny,ic,scheme", [
    ("rusanov", WALLS, 96, 32, "shock_bubble", dgb.SSPRK3),
    ("roe", WALLS, 64, 16, "shock_bubble", dgb.RK4),
    ("roe", ("periodic",) * 4, 64, 32, "quadrants", dgb.SSPRK3),
    ("rusanov", ("transmissive",) * 4, 100, 46, "quadrants", dgb.RK4),
])
def test_dmma_stage_matches_scalar_kernel(flux, bc, nx, ny, ic, scheme):
    x1 = 2.0 if ic == "shock_bubble" else 1.0
    prob = dgb.Problem.structured(2, 2, nx, ny, 0.0, x1, 0.0, 1.0, bc, flux=flux, limiter="m2l", cfl=0.3)
    probe = dgb.DGSolver(prob)
    try:
        U0 = probe.limit(prob.init_state(ic, seed=11))
        dt = 0.8 * probe.dt_from_cfl(U0)
    finally:
        probe.close()
    a1, a20 = run("scalar", prob, U0, dt, scheme, 20)
    b1, b20 = run("dmma", prob, U0, dt, scheme, 20)
    assert rel_err(b1, a1) < 1e-13
    assert rel_err(b20, a20) < 1e-11
    assert np.any(b1 != a1)
