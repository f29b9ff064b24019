"""The allocation-free limiter entry point (dgb_limit_noalloc) against the regular one.

dgb_limit_noalloc serves callers that own their device buffers and cannot allocate device memory
themselves, so they cannot create a context with dgb_create.  It keeps its temporaries in a fixed
library-owned device array instead.  Here it must reproduce dgb_limit (the context path) on two
calls in a row -- the second call reuses the array the first one left behind -- within the parity
tolerance of the other GPU tests (1e-12 relative), and reject a problem larger than its array.
This file is collected last so a failure here comes after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _noalloc(prob, U_in, U_out, stream=0):
    from dg_b200 import _ffi
    return _ffi.lib().dgb_limit_noalloc(prob._h, C.c_void_p(U_in.data_ptr()), C.c_void_p(U_out.data_ptr()),
                                        C.c_void_p(stream))


@pytest.mark.parametrize("dim,order,nx,ny,limiter,bc", [
    (2, 2, 64, 32, "m2l", ("reflective", "transmissive", "reflective", "transmissive")),
    (2, 1, 48, 20, "hrl", ("periodic",) * 4),
    (1, 2, 300, 1, "m2l", ("transmissive",) * 2),
])
def test_noalloc_limiter_matches_context_limiter(dim, order, nx, ny, limiter, bc):
    import torch
    import dg_b200 as dgb
    from dg_b200 import _ffi
    prob = dgb.Problem.structured(dim, order, nx, ny, 0.0, 2.0 if dim == 2 else 1.0, 0.0, 1.0, bc,
                                  flux="rusanov", limiter=limiter, cfl=0.3)
    ic = "shock_bubble" if dim == 2 else "tube_noise"
    solver = dgb.DGSolver(prob)
    for call in range(2):
        U = prob.init_state(ic if dim == 1 else ("quadrants" if call else ic), seed=11 + call)
        expect = solver.limit(U)
        U_dev = torch.from_numpy(U).cuda()
        out = torch.empty_like(U_dev)
        rc = _noalloc(prob, U_dev, out)
        assert rc == _ffi.OK, _ffi.lib().dgb_last_error().decode()
        torch.cuda.synchronize()
        assert rel_err(out.cpu().numpy(), expect) < 1e-12
    # in place (input and output alias)
    U = prob.init_state(ic, seed=5)
    expect = solver.limit(U)
    U_dev = torch.from_numpy(U).cuda()
    assert _noalloc(prob, U_dev, U_dev) == _ffi.OK
    torch.cuda.synchronize()
    assert rel_err(U_dev.cpu().numpy(), expect) < 1e-12
    solver.close()


def test_noalloc_limiter_rejects_problems_larger_than_its_scratch():
    import torch
    import dg_b200 as dgb
    from dg_b200 import _ffi
    prob = dgb.Problem.structured(2, 3, 512, 256, flux="rusanov", limiter="m2l")
    U_dev = torch.zeros(prob.state_size, dtype=torch.float64, device="cuda")
    rc = _noalloc(prob, U_dev, U_dev)
    assert rc == _ffi.ERR_ARG
    assert "scratch" in _ffi.lib().dgb_last_error().decode()
