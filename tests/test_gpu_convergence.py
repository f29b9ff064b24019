"""Order of accuracy of the CUDA DG path on the reference's smooth advection test (sinegam: density
and gamma perturbations carried by a uniform flow, periodic; the exact solution after one period is
the initial state).  The reference driver's ERROR diagnostic (dgb_problem_error_norms) measures
cell averages, which DG carries to higher order than the nodal solution on smooth linear problems
(toward dx^(2p+1)); the test requires at least order p + 0.6 between the last two meshes.  Measured
on a B200: 1D orders 3.0 (p=1), 4.3 (p=2), 6.2 (p=3); 2D p=2 (tiled kernels) 5.1.  RK4 with dt ~ dx
keeps the time error below the spatial one."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def density_error(dim, order, n, flux="rusanov"):
    import dg_b200 as dgb
    prob = dgb.Problem.structured(dim, order, n, n if dim == 2 else 1, 0.0, 1.0, 0.0, 1.0, ("periodic",) * 4,
                                  flux=flux, limiter="none", cfl=0.2)
    U0 = prob.init_state("sinegam")
    s = dgb.DGSolver(prob)
    try:
        nsteps = math.ceil(1.0 / s.dt_from_cfl(U0))
        s.set_state(U0)
        s.advance(nsteps, 1.0 / nsteps, scheme=dgb.RK4)
        U = s.get_state()
    finally:
        s.close()
    return prob.error_norms(U, U0)["l1"][0]


@pytest.mark.parametrize("order", [1, 2, 3])
def test_1d_sinegam_converges_at_order_p_plus_one(order):
    e = [density_error(1, order, n) for n in (16, 32, 64)]
    rates = [math.log2(e[k] / e[k + 1]) for k in range(2)]
    print(f"1D p={order}: L1 density errors {e}, observed orders {rates}")
    assert rates[-1] >= order + 0.6


def test_2d_sinegam_converges_at_order_p_plus_one():
    e = [density_error(2, 2, n, flux="roe") for n in (32, 64)]
    rate = math.log2(e[0] / e[1])
    print(f"2D p=2 (tiled): L1 density errors {e}, observed order {rate}")
    assert rate >= 2.6
