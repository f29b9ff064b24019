import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def golden_cases():
    """Operator fixtures (the driver_* fixtures hold whole reference runs instead)."""
    return sorted(p.stem for p in GOLDEN.glob("*.npz") if not p.stem.startswith(("driver_", "run_")))


def load_golden(name: str):
    d = dict(np.load(GOLDEN / f"{name}.npz"))
    meta = json.loads(str(d.pop("meta")))
    return meta, d


def problem_for(meta, **over):
    import dg_b200 as dgb
    x0, x1, y0, y1 = meta["dom"]
    kw = dict(flux=meta["flux"], limiter=meta["limiter"], cfl=meta["cfl"], thresholds=tuple(meta.get("thresholds", ())),
              n_mass=meta.get("n_mass", 0), gamma_model=meta.get("gamma_model", "gamncon"))
    kw.update(over)
    return dgb.Problem.structured(meta["dim"], meta["order"], meta["nx"], meta["ny"], x0, x1, y0, y1,
                                  tuple(meta["bc"]), **kw)


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="session")
def have_gpu():
    import torch
    return torch.cuda.is_available()


def perturbed_state(prob, ic: str, seed: int) -> np.ndarray:
    """Seeded initial condition with a 1% seeded nodal perturbation of density, momentum and
    energy (same recipe as the golden fixtures)."""
    U = prob.init_state(ic, seed=seed)
    i = prob.info
    V = U.reshape(i.n_elem, i.n_fields, i.n_s)
    rng = np.random.default_rng(seed + 1000)
    nmom = i.dim
    rho = V[:, 0, :] * (1 + 0.01 * rng.uniform(-1, 1, V[:, 0, :].shape))
    V[:, 1:1 + nmom, :] += 0.01 * rng.uniform(-1, 1, V[:, 1:1 + nmom, :].shape) * rho[:, None, :]
    V[:, 0, :] = rho
    V[:, 1 + nmom, :] *= 1 + 0.01 * rng.uniform(-1, 1, V[:, 1 + nmom, :].shape)
    return V.reshape(-1).copy()


def l1_density_error(U, Uref, n_elem, n_fields, n_s) -> float:
    """sum |rho - rho_ref| / sum |rho_ref| over all density nodes."""
    a = np.asarray(U).reshape(n_elem, n_fields, n_s)[:, 0]
    b = np.asarray(Uref).reshape(n_elem, n_fields, n_s)[:, 0]
    return float(np.abs(a - b).sum() / np.abs(b).sum())
