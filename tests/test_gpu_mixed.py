"""The mixed-precision form (FP32 contractions / Rusanov flux on FP64 anchors, FP64 pressure
recovery, Roe solver and stage update) against the plain FP64 form.

Per operator, the mixed residual must stay within 1e-5 of the FP64 residual per field (relative to
that field's max |f|, momentum components scaled together); after 50 SSP-RK3 steps of the shock-bubble the per-field relative L1 error
of the state must stay below 1e-6.  Both are printed per field.
"""
import numpy as np
import pytest

from conftest import perturbed_state

pytestmark = pytest.mark.gpu
WALLS = ("reflective", "transmissive", "reflective", "transmissive")


def per_field(a, b, info, norm="max"):
    """Per-field error of a against b; the two momentum components are scaled together (by the
    momentum magnitude), since one of them is nearly zero in these flows."""
    A = np.asarray(a).reshape(info.n_elem, info.n_fields, info.n_s)
    B = np.asarray(b).reshape(info.n_elem, info.n_fields, info.n_s)
    red = (lambda x: np.abs(x).max()) if norm == "max" else (lambda x: np.abs(x).sum())
    out = []
    for f in range(info.n_fields):
        scale = red(B[:, f]) if f not in (1, 2) else max(red(B[:, 1]), red(B[:, 2]))
        out.append(float(red(A[:, f] - B[:, f]) / scale))
    return out


@pytest.mark.parametrize("flux,order", [("rusanov", 2), ("roe", 2), ("rusanov", 1), ("roe", 3), ("rusanov", 3)])
def test_mixed_residual_close_to_fp64(flux, order):
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, order, 64, 32, 0.0, 2.0, 0.0, 1.0, WALLS, flux=flux, limiter="m2l", cfl=0.3)
    s = dgb.DGSolver(prob)
    try:
        U0 = s.limit(perturbed_state(prob, "shock_bubble", 5))
        f64 = s.dg_solver(U0)
        s.set_form("mixed")
        fmx = s.dg_solver(U0)
        err = per_field(fmx, f64, prob.info)
        print(f"mixed residual, per-field max error / max |f| ({flux}, p={order}):", err)
        assert max(err) < 1e-5
    finally:
        s.close()


def test_mixed_steps_close_to_fp64():
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, 2, 128, 64, 0.0, 2.0, 0.0, 1.0, WALLS, flux="rusanov", limiter="m2l", cfl=0.3)
    ref = dgb.DGSolver(prob)
    mix = dgb.DGSolver(prob)
    try:
        U0 = ref.limit(prob.init_state("shock_bubble", seed=7))
        mix.set_form("mixed")
        for s in (ref, mix):
            s.set_state(U0)
            s.advance(50, 0.0, scheme=dgb.SSPRK3)
        err = per_field(mix.get_state(), ref.get_state(), prob.info, norm="l1")
        print("mixed vs FP64 after 50 SSP-RK3 steps, per-field relative L1:", err)
        assert max(err) < 1e-6
    finally:
        ref.close()
        mix.close()


def test_mixed_steps_close_to_fp64_p3_roe():
    """The 2048 x 1024 p=3 Roe configuration's form at a smaller size: 30 steps, per-field L1 and
    Linf against the FP64 form, and the drift of the conserved totals."""
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, 3, 128, 64, 0.0, 2.0, 0.0, 1.0, WALLS, flux="roe", limiter="m2l", cfl=0.3)
    ref = dgb.DGSolver(prob)
    mix = dgb.DGSolver(prob)
    try:
        U0 = ref.limit(prob.init_state("shock_bubble", seed=7))
        mix.set_form("mixed")
        tot = {}
        for name, s in (("fp64", ref), ("mixed", mix)):
            s.set_state(U0)
            c0 = s.conservation()
            s.advance(30, 0.0, scheme=dgb.SSPRK3)
            tot[name] = (c0, s.conservation())
        l1 = per_field(mix.get_state(), ref.get_state(), prob.info, norm="l1")
        li = per_field(mix.get_state(), ref.get_state(), prob.info, norm="max")
        print("p=3 Roe mixed vs FP64 after 30 steps, per-field relative L1:", l1, "Linf:", li)
        assert max(l1) < 1e-6 and max(li) < 1e-4
        # the conserved totals (which change through the open boundaries) of the two forms agree
        for name, (c0, c1) in tot.items():
            print(name, "conserved totals before/after:", c0, c1)
        c0, r1, m1 = tot["fp64"][0], tot["fp64"][1], tot["mixed"][1]
        scale = np.abs(c0).copy()
        scale[1:3] = np.abs(c0[:3]).max()  # momentum totals start near zero: mass scale
        assert np.all(np.abs(m1 - r1) <= 1e-7 * scale)
    finally:
        ref.close()
        mix.close()


def test_mixed_form_rejected_where_not_built():
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, 3, 41, 32, flux="roe", limiter="m2l")  # odd nx: no tiled kernel
    s = dgb.DGSolver(prob)
    try:
        with pytest.raises(dgb.DGBError):
            s.set_form("mixed")
    finally:
        s.close()


def test_mixed_form_on_a_grid_with_strips():
    """Extents that are not tile multiples: the full tiles in the mixed form, the leftover strips in
    FP64; 20 steps stay as close to the FP64 form as on a tile-aligned grid."""
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, 2, 100, 46, 0.0, 2.0, 0.0, 1.0, WALLS, flux="rusanov", limiter="m2l", cfl=0.3)
    ref = dgb.DGSolver(prob)
    mix = dgb.DGSolver(prob)
    try:
        U0 = ref.limit(prob.init_state("shock_bubble", seed=7))
        mix.set_form("mixed")
        for s in (ref, mix):
            s.set_state(U0)
            s.advance(20, 0.0, scheme=dgb.SSPRK3)
        l1 = per_field(mix.get_state(), ref.get_state(), prob.info, norm="l1")
        assert max(l1) < 1e-6, l1
        assert np.isfinite(mix.get_state()).all()
    finally:
        ref.close()
        mix.close()


@pytest.mark.parametrize("flux,order", [("rusanov", 2), ("roe", 2), ("roe", 3)])
def test_compressed_tile_kernel_close_to_tma_tile_kernel(flux, order, monkeypatch):
    """The mixed kernel whose shared tile holds FP64 anchors and FP32 deviations
    (DGB_MIXED_TILE=ct) against the mixed kernel that keeps the TMA-loaded FP64 tile
    (DGB_MIXED_TILE=tma): the volume terms read the same FP32 deviations; only the FP64 base of a
    face trace differs, by the FP32 rounding of one deviation.  Residual and 10 SSP-RK3 steps, per
    field."""
    import dg_b200 as dgb
    prob = dgb.Problem.structured(2, order, 64, 32, 0.0, 2.0, 0.0, 1.0, WALLS, flux=flux, limiter="m2l", cfl=0.3)
    U0, out = None, {}
    for mode in ("tma", "ct"):
        monkeypatch.setenv("DGB_MIXED_TILE", mode)  # read when the context is created
        s = dgb.DGSolver(prob)
        try:
            if U0 is None:
                U0 = s.limit(perturbed_state(prob, "shock_bubble", 5))
            s.set_form("mixed")
            f = s.dg_solver(U0)
            s.set_state(U0)
            s.advance(10, 0.0, scheme=dgb.SSPRK3)
            out[mode] = (f, s.get_state())
        finally:
            s.close()
    err_f = per_field(out["ct"][0], out["tma"][0], prob.info)
    err_u = per_field(out["ct"][1], out["tma"][1], prob.info, norm="l1")
    print(f"compressed vs TMA tile ({flux}, p={order}): residual {err_f}, 10 steps L1 {err_u}")
    assert max(err_f) < 1e-6 and max(err_u) < 1e-7
