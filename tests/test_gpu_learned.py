"""Learned troubled-cell indicator on the GPU against the numpy oracle (oracle/mlp_oracle.py):
features and labels of a solver state, the FP32 training kernels (forward, backward, Adam), the
BF16 tensor-core scoring inside the limiter, and the sparse gated m2 limiter it drives.

Tolerances: features 1e-5 relative (FP32 storage); labels agree on >= 99.5% of elements (a label
is a 1e-8-relative threshold test on limiter changes, so FP64 rounding can flip a borderline one);
forward 1e-5, gradients 1e-4 relative (FP32 vs FP64); BF16 scores within 0.03 of the FP64 network;
gated limiter 1e-12 relative.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_err
from oracle import dg_oracle as O
from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def quadrant_state(nx=32, ny=32, seed=3, steps=5):
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, 2, nx, ny, flux="rusanov", limiter="m2l", cfl=0.3)
    s = dgb.DGSolver(prob)
    s.set_state(s.limit(prob.init_state("quadrants", seed=seed)))
    if steps:
        s.advance(steps, 0.0)
    return prob, s


def test_features_and_labels_match_oracle():
    import torch
    from dg_b200 import learned as L
    prob, s = quadrant_state()
    try:
        X, y = L.snapshot_samples(s)
        U = s.get_state()
    finally:
        s.close()
    S = O.Setup.from_problem(prob)
    perm = prob.array("tensor_perm")
    Xo = M.features(S, U, perm)
    yo = M.labels(S, U, perm)
    assert rel_err(X.cpu().numpy(), Xo) < 1e-5
    agree = float(np.mean(y.cpu().numpy() == yo))
    assert agree >= 0.995, agree
    assert 0 < yo.sum() < yo.size


def test_training_kernels_match_oracle():
    import torch
    from dg_b200 import _ffi as F
    from dg_b200 import learned as L
    rng = np.random.default_rng(1)
    n = 300
    p = L.init_params(4)
    X = rng.standard_normal((n, 225)).astype(np.float32)
    y = (rng.uniform(size=n) > 0.8).astype(np.float32)
    tr = L.Trainer(p, batch=n)
    Xd, yd = torch.from_numpy(X).cuda(), torch.from_numpy(y).cuda()
    prob = tr.predict(Xd).cpu().numpy()
    po, _ = M.forward(p, X.astype(np.float64))
    assert rel_err(prob, po) < 1e-5
    tr.step(Xd, yd, lr=1e-3, pos_weight=4.0)
    lo, go = M.loss_and_grad(p, X.astype(np.float64), y.astype(np.float64), 4.0)
    assert abs(tr.loss.item() - lo) < 1e-5 * max(1.0, lo)
    assert rel_err(tr.g.cpu().numpy(), go) < 1e-4
    # Adam, first step: p - lr * g / (|g| + eps)
    expect = p - 1e-3 * go / (np.abs(go) + 1e-8)
    assert rel_err(tr.params(), expect) < 1e-5


def test_bf16_scores_match_fp64_network():
    from dg_b200 import learned as L
    prob, s = quadrant_state(seed=7)
    try:
        params = L.init_params(2) * 3.0
        L.set_indicator(s, params, 0.5)
        U = s.get_state()
        sc, cnt = L.scores(s, U)
    finally:
        s.close()
    S = O.Setup.from_problem(prob)
    po, _ = M.forward(params, M.features(S, U, prob.array("tensor_perm")))
    assert np.abs(sc - po).max() < 0.03
    assert cnt == int(np.sum(sc > 0.5))


@pytest.mark.parametrize("threshold", [-1.0, 0.5])
def test_gated_limiter_matches_oracle(threshold):
    from dg_b200 import learned as L
    prob, s = quadrant_state(seed=11, steps=3)
    try:
        params = L.init_params(5) * 3.0
        U = s.get_state()
        L.set_indicator(s, params, threshold)
        sc, _ = L.scores(s, U)
        out = s.limit(U)
    finally:
        s.close()
    S = O.Setup.from_problem(prob)
    flags = sc > threshold  # the limiter works on the flagged cells and their face neighbours
    assert rel_err(out, M.gated_m2(S, U, M.band(S, flags))) < 1e-12


def test_trained_indicator_gain():
    """What the trained network (dg_b200/data/indicator_p2.npz) buys: on held-out four-quadrant
    problems it finds >= 95% of the cells the full limiter changes while flagging at most 1.3x as
    many cells as there are troubled ones; on the shock-bubble it limits a minority of cells and
    stays within 1e-4 (relative L1 density) of the full-limiter solution after 100 steps, while
    dropping the limiter altogether departs from it by far more (or fails)."""
    import dg_b200 as dgb
    from dg_b200 import learned as L
    params, meta = L.load()
    X, y = L.generate_dataset([20001, 20002], 64, 64)
    ev = L.evaluate(params, X, y, 0.2)
    assert ev["recall"] >= 0.95
    assert ev["flagged_fraction"] <= 1.3 * ev["label_fraction"]

    walls = ("reflective", "transmissive", "reflective", "transmissive")
    prob = dgb.Problem.structured(2, 2, 128, 64, 0.0, 2.0, 0.0, 1.0, walls, flux="rusanov", limiter="m2l", cfl=0.3)
    none = dgb.Problem.structured(2, 2, 128, 64, 0.0, 2.0, 0.0, 1.0, walls, flux="rusanov", limiter="none", cfl=0.3)
    full, learned, plain = dgb.DGSolver(prob), dgb.DGSolver(prob), dgb.DGSolver(none)
    try:
        U0 = full.limit(prob.init_state("shock_bubble", seed=7))
        dt = 0.8 * full.dt_from_cfl(U0)
        L.set_indicator(learned, params, 0.2)
        out = {}
        for name, s in (("full", full), ("learned", learned), ("none", plain)):
            s.set_state(U0)
            try:
                s.advance(100, dt)
                out[name] = s.get_state()
            except dgb.DGBError:
                out[name] = None
        i = prob.info
        rho = {k: (v.reshape(i.n_elem, i.n_fields, i.n_s)[:, 0] if v is not None else None) for k, v in out.items()}
        dev = lambda k: float(np.abs(rho[k] - rho["full"]).sum() / np.abs(rho["full"]).sum())
        assert rho["learned"] is not None and dev("learned") < 1e-4
        _, cnt = L.scores(learned, out["learned"])
        assert cnt < 0.5 * i.n_elem
        assert rho["none"] is None or not np.all(np.isfinite(rho["none"])) or dev("none") > 10 * dev("learned")
    finally:
        for s in (full, learned, plain):
            s.close()


def test_scoring_interval_keeps_the_full_limiter_result():
    """Scoring every 8th step (the band of the last scoring covers the discontinuities for up to
    (2p+1)/CFL = 16 steps): still within 1e-4 relative L1 density of the full limiter after 100
    steps on the shock-bubble, and the steps in between launch the four scoring kernels less
    (modes, scores, band, and the lists of the gated passes' tiles with band elements)."""
    import dg_b200 as dgb
    from dg_b200 import learned as L
    params, _ = L.load()
    walls = ("reflective", "transmissive", "reflective", "transmissive")
    prob = dgb.Problem.structured(2, 2, 128, 64, 0.0, 2.0, 0.0, 1.0, walls, flux="rusanov", limiter="m2l", cfl=0.3)
    full, learned = dgb.DGSolver(prob), dgb.DGSolver(prob)
    try:
        U0 = full.limit(prob.init_state("shock_bubble", seed=7))
        dt = 0.8 * full.dt_from_cfl(U0)
        L.set_indicator(learned, params, 0.2, every=8)
        learned.set_state(U0)
        learned.advance(1, dt)
        n_score = learned.last_timing()[1]
        learned.advance(1, dt)
        n_reuse = learned.last_timing()[1]
        assert n_reuse == n_score - 4
        out = {}
        for name, s in (("full", full), ("learned", learned)):
            s.set_state(U0)
            s.advance(100, dt)
            out[name] = s.get_state()
        i = prob.info
        rho = {k: v.reshape(i.n_elem, i.n_fields, i.n_s)[:, 0] for k, v in out.items()}
        assert float(np.abs(rho["learned"] - rho["full"]).sum() / np.abs(rho["full"]).sum()) < 1e-4
    finally:
        full.close()
        learned.close()


def test_tcgen05_scores_match_the_mma_sync_kernel():
    """The scoring GEMMs on the 5th-generation tensor cores (tcgen05.mma, accumulators in tensor
    memory) against the warp-level mma.sync kernel: the same BF16 inputs and weights with FP32
    accumulation in another order, so the scores agree to rounding and the flags almost
    everywhere."""
    import os
    from dg_b200 import learned as L
    params, _ = L.load()
    out = {}
    for kind in ("mma", "tc"):
        os.environ["DGB_INDICATOR_KERNEL"] = kind
        try:
            prob, s = quadrant_state(nx=60, ny=50, seed=13, steps=4)  # 3000 elements: a ragged last tile
        finally:
            del os.environ["DGB_INDICATOR_KERNEL"]
        try:
            L.set_indicator(s, params, 0.2)
            out[kind] = L.scores(s, s.get_state())
        finally:
            s.close()
    (sa, ca), (sb, cb) = out["mma"], out["tc"]
    assert np.abs(sa - sb).max() < 2e-3
    assert np.mean((sa > 0.2) == (sb > 0.2)) > 0.999
    assert abs(ca - cb) <= max(2, 0.001 * sa.size)


@pytest.mark.parametrize("case", ["shock_bubble", "quadrants"])
def test_mixed_form_rounding_stays_below_the_inputs_floor(case):
    """The mixed form leaves FP32 rounding in the non-constant modes of every element that the gated
    limiter does not touch (up to ~2e-5 of the field scale, mostly in the (2,2) mode); the inputs'
    floor hides it, so after 200 gated steps the network flags about as many elements of the mixed
    state as of the FP64 state (without the floor the mixed runs ended with most of the grid flagged)
    and the two runs stay within 1e-4 relative L1 density of each other."""
    import dg_b200 as dgb
    from dg_b200 import learned as L
    params, _ = L.load()
    if case == "shock_bubble":
        walls = ("reflective", "transmissive", "reflective", "transmissive")
        prob = dgb.Problem.structured(2, 2, 128, 64, 0.0, 2.0, 0.0, 1.0, walls, flux="rusanov", limiter="m2l", cfl=0.3)
        U0 = prob.init_state("shock_bubble", seed=7)
    else:
        prob = dgb.Problem.structured(2, 2, 128, 128, 0.0, 1.0, 0.0, 1.0, ("transmissive",) * 4, flux="rusanov",
                                      limiter="m2l", cfl=0.3)
        U0 = prob.init_state("quadrants", seed=4097)
    out, cnt = {}, {}
    solvers = {form: dgb.DGSolver(prob) for form in ("fp64", "mixed")}
    try:
        U0 = solvers["fp64"].limit(U0)
        dt = 0.8 * solvers["fp64"].dt_from_cfl(U0)
        for form, s in solvers.items():
            s.set_form(form)
            L.set_indicator(s, params, 0.2, every=8)
            s.set_state(U0)
            s.advance(200, dt)
            out[form] = s.get_state()
            cnt[form] = L.scores(s, out[form])[1]
    finally:
        for s in solvers.values():
            s.close()
    n = prob.info.n_elem
    assert 0 < cnt["fp64"] < 0.5 * n
    assert cnt["mixed"] <= 1.25 * cnt["fp64"] + 0.005 * n, (cnt, n)
    i = prob.info
    rho = {k: v.reshape(i.n_elem, i.n_fields, i.n_s)[:, 0] for k, v in out.items()}
    assert float(np.abs(rho["mixed"] - rho["fp64"]).sum() / np.abs(rho["fp64"]).sum()) < 1e-4
