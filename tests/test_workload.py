"""oracle/workload.py (the reference arm's inputs, written without this package's library) against
the library's own mesh writer and initial state: the same bytes and the same state, bit for bit."""
import numpy as np
import pytest

from oracle import workload as W

WALLS = ("reflective", "transmissive", "reflective", "transmissive")


@pytest.mark.parametrize("args", [
    (2, 2, 8, 4, 0.0, 2.0, 0.0, 1.0, WALLS),
    (2, 3, 6, 4, 0.0, 2.0, 0.0, 1.0, ("transmissive",) * 4),
    (2, 1, 6, 6, 0.0, 1.0, 0.0, 1.0, ("periodic",) * 4),
    (1, 2, 24, 1, 0.0, 1.0, 0.0, 1.0, ("transmissive",) * 2),
    (1, 3, 10, 1, -0.5, 0.5, 0.0, 1.0, ("reflective",) * 2),
])
def test_mesh_file_equals_the_library_writer(tmp_path, args):
    from dg_b200.solver import write_msh
    W.structured_msh(tmp_path / "a.msh", *args)
    write_msh(tmp_path / "b.msh", *args)
    assert (tmp_path / "a.msh").read_bytes() == (tmp_path / "b.msh").read_bytes()


@pytest.mark.parametrize("order,nx,ny,seed", [(2, 8, 4, 7), (2, 32, 8, 110), (3, 6, 4, 3), (1, 16, 8, 5),
                                              (2, 512, 256, 7)])
def test_shock_bubble_equals_the_library_state(order, nx, ny, seed):
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, order, nx, ny, 0.0, 2.0, 0.0, 1.0, WALLS, flux="rusanov", limiter="m2l",
                                  cfl=0.3)
    assert np.array_equal(W.shock_bubble(order, nx, ny, seed=seed), prob.init_state("shock_bubble", seed=seed))


def test_mersenne_twister_64_known_answer():
    """The 10000th output of MT19937-64 seeded with 5489 (the C++ standard's check value)."""
    g = W.MT19937_64(5489)
    for _ in range(9999):
        g.next_u64()
    assert g.next_u64() == 9981545732273789042
