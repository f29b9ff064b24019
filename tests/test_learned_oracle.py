"""The numpy restatement of the indicator MLP (oracle/mlp_oracle.py) checks itself: its gradient
against central finite differences, and basic properties of its features."""
import numpy as np

from oracle import mlp_oracle as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(18689) * 0.1
    X = rng.standard_normal((37, 225))
    y = (rng.uniform(size=37) > 0.7).astype(float)
    _, g = M.loss_and_grad(p, X, y, 3.0)
    for k in (0, 5000, 14400, 14470, 18600, 18688):
        e = np.zeros_like(p)
        e[k] = 1e-6
        fd = (M.loss_and_grad(p + e, X, y, 3.0)[0] - M.loss_and_grad(p - e, X, y, 3.0)[0]) / 2e-6
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k]))


def test_taylor_transform_reproduces_monomials():
    T = M.taylor_transform(2)
    x = np.linspace(-1, 1, 3)
    assert np.allclose(T @ (x ** 2 / 2.0), [0, 0, 1])
    assert np.allclose(T @ np.ones(3), [1, 0, 0])


def test_features_of_uniform_state_are_trivial():
    import dg_b200 as dgb
    from oracle import dg_oracle as O
    prob = dgb.Problem.structured(2, 2, 6, 4, flux="rusanov", limiter="m2l", cfl=0.3)
    U = prob.init_state("quadrants", params=(10.0, 10.0), seed=1)  # split outside: one state
    S = O.Setup.from_problem(prob)
    X = M.features(S, U, prob.array("tensor_perm")).reshape(-1, 5, 5, 9)
    assert np.allclose(X[:, :, :, 1:], 0.0, atol=1e-12)      # no slopes anywhere
    assert np.allclose(X[:, :, :, 0], 0.0, atol=1e-12)       # neighbours' means equal the element's
    assert np.all(M.labels(S, U, prob.array("tensor_perm")) == 0)


def test_band_adds_face_neighbours():
    """The gated limiter's working set: flagged cells and their face neighbours (not diagonal
    cells), clipped at walls and wrapped by periodic boundaries."""
    import dg_b200 as dgb
    from oracle import dg_oracle as O
    from oracle import mlp_oracle as M
    prob = dgb.Problem.structured(2, 2, 8, 6, bc=("reflective", "periodic", "reflective", "periodic"), flux="rusanov",
                                  limiter="m2l")
    S = O.Setup.from_problem(prob)
    f = np.zeros(S.N_E, bool)
    f[3 * 8 + 4] = True   # interior cell (x 4, y 3)
    f[0 * 8 + 0] = True   # corner cell
    b = M.band(S, f)
    exp = {3 * 8 + 4, 3 * 8 + 3, 3 * 8 + 5, 2 * 8 + 4, 4 * 8 + 4, 0, 1, 8, 7}  # corner: right, up, periodic left
    assert set(np.nonzero(b)[0].tolist()) == exp


def test_rounding_floor_hides_fp32_level_noise():
    """Inputs below the rounding floor (5e-5 of the field scale) are zero and carry no label: a
    uniform state with 5e-7 relative noise on every node (the mixed form's FP32 flux arithmetic
    leaves up to ~7e-7 on the nodes, up to ~2e-5 on the modes) looks like the clean state, while a
    1e-3 perturbation stays visible."""
    import dg_b200 as dgb
    from oracle import dg_oracle as O
    prob = dgb.Problem.structured(2, 2, 6, 4, flux="rusanov", limiter="m2l", cfl=0.3)
    U = prob.init_state("quadrants", params=(10.0, 10.0), seed=1)
    S = O.Setup.from_problem(prob)
    perm = prob.array("tensor_perm")
    rng = np.random.default_rng(5)
    noisy = U * (1.0 + 5e-7 * rng.uniform(-1.0, 1.0, U.shape))
    assert np.all(M.features(S, noisy, perm) == 0.0)
    assert np.all(M.labels(S, noisy, perm) == 0)
    bumped = U * (1.0 + 1e-3 * rng.uniform(-1.0, 1.0, U.shape))
    assert np.abs(M.features(S, bumped, perm)).max() > 0.3
    x = np.array([-1.0, -1e-3, -5e-5, 0.0, 2e-5, 5e-5, 6e-5, 1e-3, 1.0])
    c = M.compress(x)
    assert np.all(np.diff(c) > -1e-300) and np.all(c[2:6] == 0.0) and c[6] > 0 and abs(c[-1] - 1.0) < 1e-4
