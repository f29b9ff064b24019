"""Learned troubled-cell indicator: dataset, training on the GPU with the library's own kernels,
and the trained parameters.

The network (225 -> 64 -> 64 -> 1, GELU, sigmoid) predicts, from an element's and its four face
neighbours' normalised modes, whether the problem's m2 limiter would change that element.  Labels
come from the full limiter run on seeded four-quadrant Riemann problems (per quadrant rho, p in
U[0.1, 2], u, v in U[-1, 1], gamma in {1.4, 1.67}), p = 2, Rusanov flux, snapshots taken along
SSP-RK3 runs so that the discontinuities are the ones the solver produces: an element is labelled
when the limiter changes one of its non-constant modes by more than 1e-8 of the field scale and
its own modes rise above the inputs' rounding floor (5e-5 of the field scale; below it the mixed
form's FP32 rounding and real structure look alike, so inputs are soft-thresholded there).  Features, labels,
forward pass, backward pass and Adam updates are the CUDA kernels behind include/dgb.h
(dgb_indicator_features / _labels, dgb_mlp_forward / _backward / _adam); torch only provides device
buffers.  The solver uses the trained network through dgb_set_indicator (BF16 tensor-core scoring).

    python -m dg_b200.learned train --out dg_b200/data/indicator_p2.npz   # 4096 problems at 256^2
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time
from pathlib import Path

import numpy as np

from . import _ffi as F
from .solver import DGSolver, Problem

DATA = Path(__file__).resolve().parent / "data"
DEFAULT_WEIGHTS = DATA / "indicator_p2.npz"
N_IN, N_H = 225, 64


def n_params() -> int:
    return int(F.lib().dgb_mlp_param_count())


def init_params(seed: int = 0) -> np.ndarray:
    """Glorot-uniform weights, zero biases (flat layout W1, b1, W2, b2, w3, b3)."""
    rng = np.random.default_rng(seed)

    def glorot(fan_out, fan_in):
        lim = np.sqrt(6.0 / (fan_in + fan_out))
        return rng.uniform(-lim, lim, (fan_out, fan_in))

    p = np.concatenate([glorot(N_H, N_IN).ravel(), np.zeros(N_H), glorot(N_H, N_H).ravel(), np.zeros(N_H),
                        glorot(1, N_H).ravel(), np.zeros(1)]).astype(np.float32)
    assert p.size == n_params()
    return p


def _ptr(t) -> C.c_void_p:
    return C.c_void_p(t.data_ptr())


def snapshot_samples(solver: DGSolver):
    """Features and labels of the solver's current state (torch CUDA tensors)."""
    import torch
    n = solver.problem.info.n_elem
    X = torch.empty((n, N_IN), dtype=torch.float32, device="cuda")
    y = torch.empty(n, dtype=torch.float32, device="cuda")
    F.check(F.lib().dgb_indicator_features(solver._h, _ptr(X)))
    F.check(F.lib().dgb_indicator_labels(solver._h, _ptr(y)))
    return X, y


def quadrant_problem(nx: int, ny: int, seed: int):
    prob = Problem.structured(2, 2, nx, ny, 0.0, 1.0, 0.0, 1.0, ("transmissive",) * 4, flux="rusanov",
                              limiter="m2l", cfl=0.3)
    return prob, prob.init_state("quadrants", seed=seed)


def generate_dataset(seeds, nx: int = 64, ny: int = 64, snapshots=(1, 8, 24), keep_quiet: float = 1.0,
                     store_dtype=None, seed: int = 0):
    """Samples of every element at the given step counts of each seeded problem (the state is
    limited first, as the reference limits its initial condition).  Elements whose inputs are all
    zero -- the whole stencil below the rounding floor, so never labelled -- are kept with
    probability `keep_quiet`; `store_dtype` (torch.bfloat16, the scoring kernels' input type) halves
    the inputs' footprint."""
    import torch
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    prob, _ = quadrant_problem(nx, ny, 0)  # one mesh for every seed
    s = DGSolver(prob)
    Xs, ys = [], []
    try:
        for sd in seeds:
            s.set_state(s.limit(prob.init_state("quadrants", seed=sd)))
            done = 0
            for k in snapshots:
                if k > done:
                    s.advance(k - done, 0.0)
                    done = k
                X, y = snapshot_samples(s)
                if keep_quiet < 1.0:
                    keep = X.ne(0).any(dim=1) | (torch.rand(X.shape[0], device="cuda", generator=gen) < keep_quiet)
                    X, y = X[keep], y[keep]
                Xs.append(X.to(store_dtype) if store_dtype is not None else X)
                ys.append(y)
    finally:
        s.close()
    return torch.cat(Xs), torch.cat(ys)


class Trainer:
    """Adam on the weighted binary cross-entropy, minibatches drawn on the GPU."""

    def __init__(self, params: np.ndarray, batch: int = 8192):
        import torch
        self.torch = torch
        self.p = torch.from_numpy(params.copy()).cuda()
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.batch = batch
        self.cache = torch.empty((batch, 4 * N_H), dtype=torch.float32, device="cuda")
        self.prob = torch.empty(batch, dtype=torch.float32, device="cuda")
        self.work = torch.empty(batch * (1 + 2 * N_H), dtype=torch.float32, device="cuda")
        self.loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        self.t = 0

    def step(self, Xb, yb, lr: float, pos_weight: float) -> None:
        n = Xb.shape[0]
        L = F.lib()
        F.check(L.dgb_mlp_forward(_ptr(self.p), _ptr(Xb), n, _ptr(self.cache), _ptr(self.prob), None))
        F.check(L.dgb_mlp_backward(_ptr(self.p), _ptr(Xb), _ptr(yb), C.c_float(pos_weight), n, _ptr(self.cache),
                                   _ptr(self.prob), _ptr(self.g), _ptr(self.loss), _ptr(self.work), None))
        self.t += 1
        F.check(L.dgb_mlp_adam(_ptr(self.p), _ptr(self.g), _ptr(self.m), _ptr(self.v), self.t, C.c_float(lr), None))

    def predict(self, X):
        torch = self.torch
        out = torch.empty(X.shape[0], dtype=torch.float32, device="cuda")
        F.check(F.lib().dgb_mlp_forward(_ptr(self.p), _ptr(X), X.shape[0], None, _ptr(out), None))
        return out

    def params(self) -> np.ndarray:
        return self.p.cpu().numpy()


def train(X, y, steps: int = 3000, batch: int = 8192, lr: float = 2e-3, seed: int = 0, log_every: int = 500):
    """Trains from scratch; returns (params, history)."""
    import torch
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    npos = float(y.sum().item())
    pos_weight = float(min(max((y.numel() - npos) / max(npos, 1.0), 1.0), 20.0))
    tr = Trainer(init_params(seed), batch)
    hist = []
    for it in range(steps):
        idx = torch.randint(0, X.shape[0], (batch,), device="cuda", generator=gen)
        lr_t = lr * (0.5 * (1 + np.cos(np.pi * it / steps)))  # cosine decay
        tr.step(X.index_select(0, idx).float().contiguous(), y.index_select(0, idx).contiguous(), lr_t, pos_weight)
        if (it + 1) % log_every == 0 or it == 0:
            hist.append((it + 1, float(tr.loss.item())))
    return tr.params(), {"pos_weight": pos_weight, "loss": hist}


def evaluate(params: np.ndarray, X, y, threshold: float = 0.2) -> dict:
    """Recall / precision / flagged fraction of the FP32 network at `threshold`."""
    tr = Trainer(params, batch=1)
    p = tr.predict(X.float().contiguous())
    f = p > threshold
    yy = y > 0.5
    tp = float((f & yy).sum().item())
    return {"recall": tp / max(float(yy.sum().item()), 1.0), "precision": tp / max(float(f.sum().item()), 1.0),
            "flagged_fraction": float(f.float().mean().item()), "label_fraction": float(yy.float().mean().item()),
            "threshold": threshold}


def save(path, params: np.ndarray, meta: dict) -> None:
    Path(path).parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(path, params=params.astype(np.float32), meta=np.array(json.dumps(meta)))


def load(path=DEFAULT_WEIGHTS) -> tuple[np.ndarray, dict]:
    d = np.load(path)
    return d["params"].astype(np.float32), json.loads(str(d["meta"]))


def set_indicator(solver: DGSolver, params: np.ndarray, threshold: float = 0.2, every: int = 1) -> None:
    """Gate the solver's m2l limiter with the network `params`: elements scoring above `threshold`
    and their face neighbours are limited; the time stepper scores every `every`-th step."""
    p = np.ascontiguousarray(params, np.float32)
    F.check(F.lib().dgb_set_indicator(solver._h, p.ctypes.data_as(C.c_void_p), C.c_float(threshold)))
    F.check(F.lib().dgb_set_indicator_interval(solver._h, int(every)))


def clear_indicator(solver: DGSolver) -> None:
    F.check(F.lib().dgb_set_indicator(solver._h, None, C.c_float(0.0)))


def scores(solver: DGSolver, U) -> tuple[np.ndarray, int]:
    U = np.ascontiguousarray(U, np.float64)
    out = np.zeros(solver.problem.info.n_elem, np.float32)
    cnt = C.c_int()
    F.check(F.lib().dgb_indicator_scores(solver._h, F.dptr(U), out.ctypes.data_as(C.POINTER(C.c_float)),
                                         C.byref(cnt)))
    return out, cnt.value


def main(argv=None) -> int:
    import torch
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", default=str(DEFAULT_WEIGHTS))
    t.add_argument("--problems", type=int, default=4096)
    t.add_argument("--held-out", type=int, default=64)
    t.add_argument("--n", type=int, default=256, help="elements per direction of each training problem")
    t.add_argument("--snapshots", default="1,8,32,100", help="SSP-RK3 step counts at which samples are taken")
    t.add_argument("--keep-quiet", type=float, default=1.0 / 32,
                   help="fraction of the all-zero-input (never labelled) training samples kept")
    t.add_argument("--steps", type=int, default=12000)
    t.add_argument("--batch", type=int, default=16384)
    t.add_argument("--lr", type=float, default=2e-3)
    a = ap.parse_args(argv)
    snaps = tuple(int(v) for v in a.snapshots.split(","))
    t0 = time.time()
    X, y = generate_dataset(range(a.problems), a.n, a.n, snaps, a.keep_quiet, torch.bfloat16)
    Xv, yv = generate_dataset(range(10000, 10000 + a.held_out), a.n, a.n, snaps, 1.0, torch.bfloat16)
    t1 = time.time()
    params, hist = train(X, y, a.steps, a.batch, a.lr)
    t2 = time.time()
    ev = {f"{th}": evaluate(params, Xv, yv, th) for th in (0.2, 0.5)}
    meta = {"problems": a.problems, "n": a.n, "snapshots": list(snaps), "keep_quiet": a.keep_quiet,
            "samples": int(X.shape[0]), "label_fraction": float(y.mean().item()),
            "steps": a.steps, "batch": a.batch, "lr": a.lr, "history": hist, "held_out": ev,
            "dataset_s": round(t1 - t0, 2), "train_s": round(t2 - t1, 2),
            "recipe": f"four-quadrant problems 0..{a.problems - 1} on {a.n} x {a.n} p=2 meshes, samples after "
                      f"{a.snapshots} SSP-RK3 steps (all-zero-input samples kept at {a.keep_quiet:g}, inputs "
                      f"stored as BF16); held-out seeds 10000..{10000 + a.held_out - 1}, every element"}
    save(a.out, params, meta)
    print(json.dumps({k: v for k, v in meta.items() if k != "history"}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
