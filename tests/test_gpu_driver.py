"""dgbexec (the deck-driven executable) against the reference executable on the same deck: the
reference's own time loop wrote .pos files for output steps 0..3 of a 1D two-fluid shock tube
(tests/golden/driver_*.npz, from tests/golden/make_golden.py); dgbexec must write the same files --
same fields, steps and times -- with values within 1e-10 relative per file."""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(GOLDEN))
from make_golden import read_pos  # noqa: E402


def test_dgbexec_reproduces_reference_run(tmp_path):
    import dg_b200 as dgb
    d = np.load(GOLDEN / "driver_d1_sodtube_roe_m2l.npz")
    c = json.loads(str(d["meta"]))
    dgb.write_msh(tmp_path / "mesh.msh", c["dim"], c["order"], c["nx"], 1, c["dom"][0], c["dom"][1], 0.0, 1.0,
                  ("transmissive",) * 4)
    (tmp_path / "deck.inp").write_text(str(d["deck"]))
    exe = ROOT / "dg_b200" / "lib" / "dgbexec"
    r = subprocess.run([str(exe), "-d", "deck.inp", "--out", "."], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    ref = sorted(k[4:] for k in d.files if k.startswith("pos_"))
    mine = sorted(p.stem for p in tmp_path.glob("*.pos"))
    assert mine == ref
    for stem in ref:
        name, time, step, vals = read_pos(tmp_path / f"{stem}.pos")
        assert abs(time - float(d[f"time_{stem}"][0])) <= 1e-14
        rv = d[f"pos_{stem}"]
        assert vals.shape == rv.shape
        assert np.abs(vals - rv).max() <= 1e-10 * np.abs(rv).max(), stem


def test_dgbexec_error_diagnostic_matches_reference(tmp_path):
    """The reference's ERROR build on its smooth advection deck (sinegam, periodic, 40 elements,
    p=2, Rusanov, no limiter, RK4 to one period): dgbexec's error.dat against the reference's.
    The density and 1/(gamma-1) errors (3e-6, 1.5e-5) agree to 1e-4 relative; the velocity and
    pressure columns are rounding noise (~1e-14) in both runs."""
    import dg_b200 as dgb
    d = np.load(GOLDEN / "driver_d1_sinegam_rus_err.npz")
    c = json.loads(str(d["meta"]))
    dgb.write_msh(tmp_path / "mesh.msh", 1, c["order"], c["nx"], 1, 0.0, 1.0, 0.0, 1.0, ("periodic",) * 4)
    (tmp_path / "deck.inp").write_text(str(d["deck"]))
    exe = ROOT / "dg_b200" / "lib" / "dgbexec"
    r = subprocess.run([str(exe), "-d", "deck.inp", "--out", "."], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    mine = np.loadtxt(tmp_path / "error.dat")
    ref = d["error_dat"]
    assert mine.shape == ref.shape == (3, 5)
    assert np.all(mine[:, 0] == ref[:, 0])  # dx
    for col in (1, 4):                      # rho, 1/(gamma-1)
        assert np.allclose(mine[:, col], ref[:, col], rtol=1e-4, atol=0), (col, mine[:, col], ref[:, col])
    assert np.all(np.abs(mine[:, 2:4]) < 1e-12) and np.all(np.abs(ref[:, 2:4]) < 1e-12)


def test_dgbexec_conservation_output_matches_reference(tmp_path):
    """The reference's CONS build on the driver deck: conservation.dat (time and the domain
    integral of each field after the initial limiting and at every output time) written by
    dgbexec against the reference's, within 1e-10 relative per field."""
    import dg_b200 as dgb
    d = np.load(GOLDEN / "driver_d1_sodtube_roe_cons.npz")
    c = json.loads(str(d["meta"]))
    dgb.write_msh(tmp_path / "mesh.msh", c["dim"], c["order"], c["nx"], 1, c["dom"][0], c["dom"][1], 0.0, 1.0,
                  ("transmissive",) * 4)
    (tmp_path / "deck.inp").write_text(str(d["deck"]))
    assert dgb.Problem.from_deck(tmp_path / "deck.inp").info.cons_output == 1
    exe = ROOT / "dg_b200" / "lib" / "dgbexec"
    r = subprocess.run([str(exe), "-d", "deck.inp", "--out", "."], cwd=tmp_path, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    mine = np.loadtxt(tmp_path / "conservation.dat")
    ref = d["conservation_dat"]
    assert mine.shape == ref.shape == (len(c["output_times"]), 5)
    assert np.abs(mine[:, 0] - ref[:, 0]).max() <= 1e-15
    for col in range(1, 5):
        scale = np.abs(ref[:, col]).max()
        if scale == 0:
            assert np.abs(mine[:, col]).max() <= 1e-14
        else:
            assert np.abs(mine[:, col] - ref[:, col]).max() <= 1e-10 * scale, (col, mine[:, col], ref[:, col])
