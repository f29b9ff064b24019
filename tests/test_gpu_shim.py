"""The link-compatible shim (dg_b200/lib/libdgb_shim_<dim>d_<flux>.so: the reference's L* kernel
launchers) driven exactly as the reference's host classes drive them -- DG_SOLVER::dg_solver
(code/src/dg/dg_solver.h:292-364), Lsolver, DtFromCFL, Limiting::M2limiting / HRlimiting /
HRIlimiting / M2Ilimiting / PRIlimiting / P0Ilimiting (code/src/limiting/limiting.cc),
SENSOR::sensing -- with the BLAS products of those classes done by device matrix products, on
the reference's own setup arrays; results against the reference's golden outputs (1e-12,
sensor flags exact)."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from conftest import load_golden, rel_err

pytestmark = pytest.mark.gpu
LIB = Path(__file__).resolve().parents[1] / "dg_b200" / "lib"
FLUX = {"rusanov": "rus", "roe": "roe", "hll": "hll"}


class Shim:
    """ctypes view of one shim build; integer arguments as int, pointers as void*, doubles and
    bools by value."""

    def __init__(self, dim, flux):
        self.L = C.CDLL(str(LIB / f"libdgb_shim_{dim}d_{FLUX[flux]}.so"))

    def __getattr__(self, name):
        fn = getattr(self.L, name)

        def call(*args):
            conv = []
            for a in args:
                if isinstance(a, bool):
                    conv.append(C.c_bool(a))
                elif isinstance(a, (int, np.integer)):
                    conv.append(C.c_int(int(a)))
                elif isinstance(a, float):
                    conv.append(C.c_double(a))
                else:
                    conv.append(C.c_void_p(a.data_ptr()))
            fn.restype = None
            fn(*conv)
        return call


def dev(a):
    import torch
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a).cuda()


def zeros(n, ints=False):
    import torch
    return torch.zeros(int(n), dtype=torch.int32 if ints else torch.float64, device="cuda")


def apply(T, X, ns):
    """blasGemm('N','N', N_s, cols, N_s, 1, T, N_s, X, N_s): each column of X by the column-major T."""
    return (X.view(-1, ns) @ T.view(ns, ns)).contiguous().view(-1)


def setup(name):
    meta, d = load_golden(name)
    rm = meta["ref_meta"]
    return meta, d, rm, Shim(meta["dim"], meta["flux"])


def dg_solver(L, d, rm, U):
    """DG_SOLVER::dg_solver through the shim (dg_solver.h:292-364)."""
    D, NF, NE, Ns, NG, MT, Ms, MG, NN = (rm[k] for k in ("D", "N_F", "N_E", "N_s", "N_G", "M_T", "M_s", "M_G", "N_N"))
    UF = zeros(MT * NF * 2 * Ms)
    L.LmapToFace(Ms, MT, Ns, dev(d["ref_map"]), U, UF)
    if rm.get("rflctive", 0):
        L.LrflctiveBoundary(Ms, rm["rflctive"], dev(d["ref_boundaryMap"]), dev(d["ref_normals"]), 0, UF)
    Ug = (U.view(-1, Ns) @ dev(d["ref_phi"]).view(Ns, NG)).contiguous()
    dUg = (U.view(-1, Ns) @ dev(d["ref_dphi"]).view(Ns, NG * D)).contiguous()
    UgF = (UF.view(-1, Ms) @ dev(d["ref_psi"]).view(Ms, MG)).contiguous()
    s, f = zeros(NE * NF * NG), zeros(NE * NF * NG * D)
    L.Levaluate_sf(NG, NE, s, f, Ug, dUg, dev(d["ref_invJac"]))
    q = zeros(MT * NF * 2 * MG)
    L.Levaluate_q(MG, MT, q, UgF, dev(d["ref_normals"]))
    sJ, fJ = zeros(NE * NF * NG), zeros(NE * NF * NG * D)
    L.Lredistribute_sf(NG, NE, sJ, fJ, s, f, dev(d["ref_J"]), dev(d["ref_invJac"]))
    S = (sJ.view(-1, NG) @ dev(d["ref_phi_w"]).view(Ns, NG).T).contiguous()
    F = (fJ.view(-1, NG * D) @ dev(d["ref_dphi_w"]).view(Ns, NG * D).T).contiguous()
    qJ = zeros(MT * NF * 2 * MG)
    L.Lredistribute_q(MG, MT, qJ, q, dev(d["ref_JF"]))
    Qtcj = (qJ.view(-1, MG) @ dev(d["ref_psi_w"]).view(Ms, MG).T).contiguous()
    Q = zeros(NE * NF * Ns)
    L.LmapToElement(Ns, NE, Ms, NN, dev(d["ref_invmap"]), Q, Qtcj)
    out = zeros(NE * NF * Ns)
    L.LaddSFQ(Ns, NE, out, S, F, Q)
    return out


@pytest.mark.parametrize("name", ["d2_p2_rus_m2l", "d2_p2_roe_m2l_walls", "d1_p3_hll_m2l_periodic",
                                  "d1_p1_rus_hrl_wall", "t2_p2_roe_m2l_box"])
def test_shim_dg_solver_solve_and_dt(name):
    meta, d, rm, L = setup(name)
    U = dev(d["U0"])
    f = dg_solver(L, d, rm, U)
    assert rel_err(f.cpu().numpy(), d["f"]) < 1e-12
    DU = zeros(U.numel())
    L.Lsolver(rm["N_s"], rm["N_E"], float(meta["dt"]), dev(d["ref_Minv"]), dev(d["f"]), DU)
    assert rel_err(DU.cpu().numpy(), d["DU"]) < 1e-12
    P0 = DU.clone()
    L.Laverage_cell_p0(rm["N_s"], rm["N_E"], P0)
    m = d["DU"].reshape(-1, rm["N_s"]).mean(1, keepdims=True)
    assert np.abs(P0.cpu().numpy().reshape(-1, rm["N_s"]) - m).max() <= 1e-13 * np.abs(d["DU"]).max()
    UPA = zeros(rm["N_E"] * rm["N_s"])
    L.LfindUPA(rm["N_s"], rm["N_E"], U, UPA)
    dt = meta["cfl"] * abs(rm["cfl_scaled"]) / float(UPA.abs().max().item())
    assert abs(dt - float(d["dt_cfl"][0])) <= 1e-14 * dt


def hrl_pass(L, d, rm, x, T_in, offxy):
    """Monomials of one scalar field, limited along one direction (Lhrl1D on one field)."""
    NE, Ns, NN, D = rm["N_E"], rm["N_s"], rm["N_N"], rm["D"]
    n1 = round(Ns ** (1 / D))
    lim = zeros(NE * Ns)
    if D == 1:
        L.Lhrl1D(Ns, NE, 1, NN, 1, dev(d["ref_neighbors"]), offxy, apply(T_in, x, Ns), lim)
    else:
        L.Lhrl1D(n1, NE, 1, NN, n1, dev(d["ref_neighbors"]), offxy, apply(T_in, x, Ns), lim)
    return lim


def m2limiting(L, d, rm, U):
    """Limiting::M2limiting for the gamma model (limiting.cc:124-196 in 1D, 271-395 in 2D)."""
    NE, NF, Ns, D = rm["N_E"], rm["N_F"], rm["N_s"], rm["D"]
    iE, iG = D + 1, D + 2
    n1 = round(Ns ** (1 / D))
    sl = n1 if D == 2 else 1
    N1 = n1 if D == 2 else Ns

    def field(k):
        out = zeros(NE * Ns)
        L.Lstridedcopy(NE, Ns, Ns * NF, Ns, k * Ns, 0, U, out)
        return out
    if D == 1:
        passes = [(d["ref_Lag2Mono"], d["ref_Mono2Lag"], 0)]
    else:
        passes = [(d["ref_Lag2MonoX"], d["ref_MonoX2Lag"], 0), (d["ref_Lag2MonoY"], d["ref_MonoY2Lag"], 2)]
    nodal = {k: field(k) for k in list(range(D + 1)) + [iG]}
    p = zeros(NE * Ns)
    L.Lpressure(Ns, NE, U, p)
    E = field(iE)
    for T_in, T_out, off in passes:
        T_in, T_out = dev(T_in), dev(T_out)
        lims = {k: hrl_pass(L, d, rm, x, T_in, off) for k, x in nodal.items()}
        plim = hrl_pass(L, d, rm, p, T_in, off)
        for k in nodal:
            nodal[k] = apply(T_out, lims[k], Ns)
        if D == 2:  # the x-limited pressure, back in Lagrange form, feeds the y pass
            p = apply(T_out, plim, Ns)
        K = zeros(NE * Ns)
        if D == 1:
            L.Lkinetic_energy1D(Ns, NE, nodal[0], nodal[1], K)
        else:
            L.Lkinetic_energy2D(Ns, NE, nodal[0], nodal[1], nodal[2], K)
        rhoe = zeros(NE * Ns)
        L.Linternal_energy_multifluid(N1, NE, sl, plim, lims[iG], rhoe)
        El = zeros(NE * Ns)
        L.Lreconstruct_energy(N1, NE, sl, rhoe, apply(T_in, K, Ns), apply(T_in, E, Ns), El)
        E = apply(T_out, El, Ns)
    out = U.clone()
    for k, x in list(nodal.items()) + [(iE, E)]:
        L.Lstridedcopy(NE, Ns, Ns, Ns * NF, 0, k * Ns, x, out)
    return out


def hrlimiting(L, d, rm, U):
    """Limiting::HRlimiting 2D Cartesian (limiting.cc:28-45)."""
    NE, NF, Ns, NN = rm["N_E"], rm["N_F"], rm["N_s"], rm["N_N"]
    n1 = round(Ns ** 0.5)
    nb = dev(d["ref_neighbors"])
    A = apply(dev(d["ref_Lag2MonoX"]), U, Ns)
    Al = zeros(A.numel())  # one buffer for both passes, as the reference's _Alim
    L.Lhrl1D(n1, NE, NF, NN, n1, nb, 0, A, Al)
    A = apply(dev(d["ref_MonoX2MonoY"]), Al, Ns)
    L.Lhrl1D(n1, NE, NF, NN, n1, nb, 2, A, Al)
    return apply(dev(d["ref_MonoY2Lag"]), Al, Ns)


@pytest.mark.parametrize("name", ["d2_p2_rus_m2l", "d1_p2_roe_m2l", "t2_p2_roe_m2l_box", "d2_p2_rus_hrl_box"])
def test_shim_global_limiters(name):
    meta, d, rm, L = setup(name)
    U = dev(d["Uraw"])
    out = hrlimiting(L, d, rm, U) if meta["limiter"] == "hrl" else m2limiting(L, d, rm, U)
    assert rel_err(out.cpu().numpy(), d["Ulim"]) < 1e-12


def sensing(L, d, rm, meta, U):
    """SENSOR::sensing (sensor.cc:11-35): nodal means, then Lcalc_sensors."""
    NE, NF, Ns, NN = rm["N_E"], rm["N_F"], rm["N_s"], rm["N_N"]
    V = U.view(NE * NF, Ns)
    acc = V[:, 0].clone()
    for i in range(1, Ns):  # node order, then the 1/N_s scale (the library's cell-mean order)
        acc = acc + V[:, i]
    Uavg = (acc * (1.0 / Ns)).contiguous()
    th = list(meta.get("thresholds", ())) + [0.0] * 3
    n = len(meta.get("thresholds", ()))
    sens = zeros(NE, ints=True)
    L.Lcalc_sensors(NE, NN, n > 0, float(th[0]), n > 1, float(th[1]), n > 2, float(th[2]), dev(d["ref_neighbors"]),
                    Uavg, sens)
    return sens


@pytest.mark.parametrize("name", ["s2_p2_rus_hri_walls", "s2_p2_rus_m2i_box", "s2_p2_rus_p0i", "s2_p1_roe_pri"])
def test_shim_sensor_gated_limiters(name):
    meta, d, rm, L = setup(name)
    NE, NF, Ns, NN, NG = rm["N_E"], rm["N_F"], rm["N_s"], rm["N_N"], rm["N_G"]
    U = dev(d["Uraw"])
    sens = sensing(L, d, rm, meta, U)
    assert np.array_equal(sens.cpu().numpy(), d["sens"])
    n1 = round(Ns ** 0.5)
    tmp = zeros(U.numel())
    nb = dev(d["ref_neighbors"])
    if meta["limiter"] == "p0i":
        L.Lp0i(Ns, NE, NG, 4.0, sens, dev(d["ref_phi_w"]), U, tmp)
        L.Lcopy_detected(Ns, NE, sens, tmp, U)
    else:
        if meta["limiter"] == "pri":
            L.LCons2Prim(Ns, NE, U)
        fn = L.Lm2i1D if meta["limiter"] == "m2i" else L.Lhri1D
        for T_in, T_out, off in ((d["ref_Lag2MonoX"], d["ref_MonoX2Lag"], 0), (d["ref_Lag2MonoY"], d["ref_MonoY2Lag"], 2)):
            fn(Ns, NE, NN, nb, n1, n1, off, dev(T_in), dev(T_out), sens, U, tmp)
            L.Lcopy_detected(Ns, NE, sens, tmp, U)
        if meta["limiter"] == "pri":
            L.LPrim2Cons(Ns, NE, U)
    assert rel_err(U.cpu().numpy(), d["Ulim"]) < 1e-12


def test_shim_formater_and_sensor_output():
    """Lformater on the reference deck's initial condition against the reference's step-0 .pos values
    (written with six significant digits), its inverse round trip, and Lformat_sensor."""
    import json
    import dg_b200 as dgb
    from conftest import GOLDEN
    g = np.load(GOLDEN / "driver_d1_sodtube_roe_m2l.npz")
    c = json.loads(str(g["meta"]))
    prob = dgb.Problem.structured(1, c["order"], c["nx"], 1, c["dom"][0], c["dom"][1], bc=("transmissive",) * 2,
                                  flux="roe", limiter="m2l", cfl=c["cfl"])
    U0 = dev(prob.init_state("sodtube"))
    i = prob.info
    L = Shim(1, "roe")
    out = zeros(U0.numel())
    L.Lformater(i.n_s, i.n_elem, U0, out, False)
    o = out.cpu().numpy().reshape(i.n_elem, i.n_fields, i.n_s)
    for f, nm in enumerate(("rho", "ux", "g", "p")):
        six = np.vectorize(lambda v: float("%g" % v))(o[:, f, :])
        assert np.array_equal(six, g[f"pos_{nm}0000000000"]), nm
    back = zeros(U0.numel())
    L.Lformater(i.n_s, i.n_elem, back, out, True)
    assert rel_err(back.cpu().numpy(), U0.cpu().numpy()) < 1e-14
    sens = dev(np.arange(i.n_elem, dtype=np.int32) % 3)
    so = zeros(i.n_elem * i.n_s)
    L.Lformat_sensor(i.n_s, i.n_elem, sens, so)
    assert np.array_equal(so.cpu().numpy(), np.repeat(np.arange(i.n_elem) % 3, i.n_s).astype(float))
