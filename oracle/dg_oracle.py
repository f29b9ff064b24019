"""CPU restatement of the reference's DG residual / limiter / time-step path (numpy).

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` leg of ``bench.py`` import it.  The product (``dg_b200``) never calls it
and has no CPU fallback.

It restates, for the gamma-model multifluid Euler equations in 1D and 2D (GAMNCON, where the
last gamma-model field is 1/(gamma-1) with a non-conservative source, and GAMCONS, where it is
rho/(gamma-1) transported conservatively; with passive mass fractions rho*Y_k appended),
the arithmetic of the reference's CPU build, operating on the reference's own setup arrays
(phi, dphi, psi, J, invJac, JF, normals, map, invmap, boundaryMap, neighbors, Minv and the
Lagrange<->monomial transforms) in the reference's own layouts:

  * ``residual``   DG_SOLVER::dg_solver, code/src/dg/dg_solver.h:292-364
  * ``solve``      solve / Lsolver, code/src/time_integration/rk_kernels.cu:22-57
  * ``dt_from_cfl`` RK::DtFromCFL, code/src/time_integration/rk.cc:250-272 (findUPA
                   rk_kernels.cu:94-174, twod/oned_multifluid_upa code/src/physics/upa.h:61-85)
  * ``limit``      Limiting::HRlimiting (code/src/limiting/limiting.cc:11-100) and
                   Limiting::M2limiting (limiting.cc:123-409, gamma model) on Cartesian meshes
  * ``rk4_steps``  the RK4 step body of RK::RK_integration, rk.cc:155-209 (coefficients rk.h:44-57)
  * ``ssprk3_steps`` Shu-Osher SSP-RK3 with the reference's limiter placement (the reference has
                   no RK3; the golden vectors come from the same scheme driven over the
                   reference's own operators by oracle/ref_harness.cc)

Parity of this restatement is pinned by tests/test_oracle.py against the golden vectors in
tests/golden/*.npz, which the reference's own CPU build produced (tests/golden/make_golden.py).
All arrays are float64; the state layout is U[(e*N_F + f)*N_s + i] (code/src/main.cc:814-820).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from math import factorial

import numpy as np

# ---------------------------------------------------------------------------------------------
# setup
# ---------------------------------------------------------------------------------------------

ARRAY_NAMES = ("phi", "dphi", "phi_w", "dphi_w", "psi", "psi_w", "weight", "J", "invJac", "JF", "normals", "Minv",
               "map", "invmap", "boundaryMap", "neighbors", "Lag2Mono", "Mono2Lag", "Lag2MonoX",
               "MonoX2MonoY", "MonoY2Lag", "MonoX2Lag", "Lag2MonoY")


@dataclass
class Setup:
    """Sizes, options and reference setup arrays of one problem (names as in the reference)."""
    D: int
    N_F: int
    N_E: int
    N_s: int
    N_G: int
    M_T: int
    M_s: int
    M_G: int
    N_N: int
    flux: str                # "rusanov" | "roe" | "hll"
    limiter: str             # "none" | "hrl" | "m2l"
    cfl_scaled: float        # CFL*Dx/(2p+1) (main.cc:896-897)
    n_reflective: int        # _rflctiveIdx (dg_solver.h:112)
    a: dict = field(default_factory=dict)
    gx: float = 0.0          # constants::GLOBAL_GX / GLOBAL_GY (zero unless an IC sets gravity)
    gy: float = 0.0
    thresholds: tuple = ()   # "#sensor thresholds" of the deck (sensor.h:35-45)
    gamcons: bool = False    # GAMCONS gamma model (Makefile GAMM=GAMCONS)

    @property
    def order(self) -> int:
        return round(self.N_s ** (1.0 / self.D)) - 1

    @classmethod
    def from_golden(cls, meta: dict, d: dict) -> "Setup":
        """From a golden fixture: its metadata and its ``ref_*`` arrays (the reference's own)."""
        rm = meta["ref_meta"]
        arrays = {k[4:]: v for k, v in d.items() if k.startswith("ref_")}
        return cls(D=rm["D"], N_F=rm["N_F"], N_E=rm["N_E"], N_s=rm["N_s"], N_G=rm["N_G"], M_T=rm["M_T"],
                   M_s=rm["M_s"], M_G=rm["M_G"], N_N=rm["N_N"], flux=meta["flux"], limiter=meta["limiter"],
                   cfl_scaled=rm["cfl_scaled"], n_reflective=rm.get("rflctive", 0), a=arrays,
                   thresholds=tuple(meta.get("thresholds", ())), gamcons=meta.get("gamma_model") == "gamcons")

    @classmethod
    def from_problem(cls, prob, thresholds=()) -> "Setup":
        """From a dg_b200.Problem (host setup pinned to the reference arrays by tests)."""
        i = prob.info
        names = {0: "rusanov", 1: "hll", 2: "roe"}
        lims = {0: "none", 1: "hrl", 2: "m2l", 3: "hri", 4: "m2i", 5: "prl", 6: "pri", 7: "p0i"}
        arrays = {}
        for k in ARRAY_NAMES:
            try:
                arrays[k] = prob.array(k)
            except Exception:
                pass
        return cls(D=i.dim, N_F=i.n_fields, N_E=i.n_elem, N_s=i.n_s, N_G=i.n_g, M_T=i.n_ifaces, M_s=i.m_s,
                   M_G=i.m_g, N_N=i.n_n, flux=names[i.flux], limiter=lims[i.limiter], cfl_scaled=i.cfl_scaled,
                   n_reflective=i.n_reflective, a=arrays, thresholds=tuple(thresholds),
                   gamcons=getattr(i, "gamma_model", 0) == 1)


# ---------------------------------------------------------------------------------------------
# interface Riemann solvers (vectorised over face points); each returns (F, nc) with shape (N_F, n)
# ---------------------------------------------------------------------------------------------

def _twod_rusanov(rhoL, rhoR, vxL, vxR, vyL, vyR, EtL, EtR, alL, alR, nx, ny, YL=(), YR=(), gc=False):
    """twod_multifluid_rusanov, code/src/face_fluxes/twod_multifluid_fluxes.h:30-97; the mass
    fractions rho*Y_k (YL, YR) by the MACRO block at :89-94, whose dissipation term sits outside
    the 1/2.  gc (GAMCONS): alL, alR are the stored rho/(gamma-1) divided by the density by the
    caller (:50-53, where the right alpha is set to the already divided left one divided by rhoL
    again, which the caller reproduces), and the fifth flux is the conservative rho*alpha*vn with its dissipation
    (:82-84), with no non-conservative term."""
    vnL = vxL * nx + vyL * ny
    vnR = vxR * nx + vyR * ny
    gL = 1.0 + 1.0 / alL
    gR = 1.0 + 1.0 / alR
    pL = (gL - 1) * (EtL - 0.5 * rhoL * (vxL * vxL + vyL * vyL))
    pR = (gR - 1) * (EtR - 0.5 * rhoR * (vxR * vxR + vyR * vyR))
    aL = np.sqrt((gL * pL) / rhoL)
    aR = np.sqrt((gR * pR) / rhoR)
    HL = (EtL + pL) / rhoL
    HR = (EtR + pR) / rhoR
    lam = np.maximum(np.abs(vnL) + aL, np.abs(vnR) + aR)
    F = np.zeros((5 + len(YL),) + np.shape(rhoL))
    nc = np.zeros_like(F)
    for k in range(len(YL)):
        F[5 + k] = 0.5 * (YL[k] * vnL + YR[k] * vnR) - lam * (YR[k] - YL[k])
    F[0] = 0.5 * (rhoL * vnL + rhoR * vnR - lam * (rhoR - rhoL))
    F[1] = 0.5 * ((rhoL * vnL * vxL + pL * nx) + (rhoR * vnR * vxR + pR * nx) - lam * (rhoR * vxR - rhoL * vxL))
    F[2] = 0.5 * ((rhoL * vnL * vyL + pL * ny) + (rhoR * vnR * vyR + pR * ny) - lam * (rhoR * vyR - rhoL * vyL))
    F[3] = 0.5 * (rhoL * vnL * HL + rhoR * vnR * HR - lam * (EtR - EtL))
    if gc:
        F[4] = 0.5 * (rhoL * vnL * alL + rhoR * vnR * alR - lam * (rhoR * alR - rhoL * alL))
    else:
        F[4] = 0.5 * (-lam * (alR - alL))
        nc[4] = -0.5 * 0.5 * (vnL + vnR) * (alR - alL)
    return F, nc


def _twod_roe(rhoL, rhoR, vxL, vxR, vyL, vyR, EtL, EtR, alL, alR, nx, ny, YL=(), YR=(), gc=False):
    """twod_multifluid_roe, twod_multifluid_fluxes.h:151-342: Roe averages, wave strengths
    dV0..dV4 and right eigenvectors R of the gamma-model system; mass fractions by the
    Roe-averaged Y and its wave strength (:307-319).  gc (GAMCONS): divided alphas (:175-178) and
    the central part 0.5 (rho alpha vn)_L + (rho alpha vn)_R in the fifth flux (:294-299)."""
    tx, ty = -ny, nx
    vnL = vxL * nx + vyL * ny
    vnR = vxR * nx + vyR * ny
    vtL = vxL * tx + vyL * ty
    vtR = vxR * tx + vyR * ty
    gL = 1.0 + 1.0 / alL
    gR = 1.0 + 1.0 / alR
    pL = (gL - 1) * (EtL - 0.5 * rhoL * (vxL * vxL + vyL * vyL))
    pR = (gR - 1) * (EtR - 0.5 * rhoR * (vxR * vxR + vyR * vyR))
    HL = (EtL + pL) / rhoL
    HR = (EtR + pR) / rhoR
    iL = pL * alL
    iR = pR * alR
    RT = np.sqrt(rhoR / rhoL)
    rho = RT * rhoL
    vx = (vxL + RT * vxR) / (1 + RT)
    vy = (vyL + RT * vyR) / (1 + RT)
    vn = vx * nx + vy * ny
    vt = vx * tx + vy * ty
    H = (HL + RT * HR) / (1 + RT)
    al = (alL + RT * alR) / (1 + RT)
    g = 1 + 1.0 / al
    a = np.sqrt((g - 1) * (H - 0.5 * (vx * vx + vy * vy)))
    i = (iL + RT * iR) / (1 + RT)
    p = (g - 1) * i
    drho = rhoR - rhoL
    dp = (g - 1) * (g - 1) * (al * (iR - iL) - i * (alR - alL))
    dvn = vnR - vnL
    dvt = vtR - vtL
    dV = [(dp - rho * a * dvn) / (2 * a * a), rho * dvt / a, drho - dp / (a * a),
          (dp + rho * a * dvn) / (2 * a * a), alR - alL]
    ws = [np.abs(vn - a), np.abs(vn), np.abs(vn), np.abs(vn + a), np.abs(vn)]
    z = np.zeros_like(vx)
    one = np.ones_like(vx)
    R = [[one, vx - a * nx, vy - a * ny, H - vn * a, z],
         [z, a * tx, a * ty, vt * a, z],
         [one, vx, vy, 0.5 * (vx * vx + vy * vy), z],
         [one, vx + a * nx, vy + a * ny, H + vn * a, z],
         [z, z, z, p, one]]

    def diss(c):
        return ws[0] * dV[0] * R[0][c] + ws[1] * dV[1] * R[1][c] + ws[2] * dV[2] * R[2][c] + \
            ws[3] * dV[3] * R[3][c] + ws[4] * dV[4] * R[4][c]

    F = np.zeros((5 + len(YL),) + np.shape(rhoL))
    nc = np.zeros_like(F)
    for k in range(len(YL)):
        Y = (YL[k] / rhoL + RT * YR[k] / rhoR) / (1 + RT)
        dVY = YR[k] - YL[k] - (dV[0] + dV[2] + dV[3]) * Y
        F[5 + k] = 0.5 * (YL[k] * vnL + YR[k] * vnR) - 0.5 * (ws[0] * dV[0] * Y + ws[2] * dV[2] * Y + ws[1] * dVY * 1 +
                                                                ws[3] * dV[3] * Y)
    F[0] = 0.5 * (rhoL * vnL + rhoR * vnR) - 0.5 * diss(0)
    F[1] = 0.5 * ((rhoL * vnL * vxL + pL * nx) + (rhoR * vnR * vxR + pR * nx)) - 0.5 * diss(1)
    F[2] = 0.5 * ((rhoL * vnL * vyL + pL * ny) + (rhoR * vnR * vyR + pR * ny)) - 0.5 * diss(2)
    F[3] = 0.5 * (rhoL * vnL * HL + rhoR * vnR * HR) - 0.5 * diss(3)
    if gc:
        F[4] = 0.5 * (rhoL * vnL * alL + rhoR * vnR * alR) - 0.5 * diss(4)
    else:
        F[4] = -0.5 * diss(4)
        nc[4] = -0.5 * vn * (alR - alL)
    return F, nc


def _oned_rusanov(rhoL, rhoR, vxL, vxR, EtL, EtR, alL, alR, nx, YL=(), YR=(), gc=False):
    """oned_multifluid_rusanov, code/src/face_fluxes/oned_multifluid_fluxes.h:30-94; mass fractions
    by the MACRO block at :88-92 (dissipation outside the 1/2).  gc (GAMCONS; alphas divided by
    the caller, :46-49): conservative rho*alpha*u flux with its dissipation (:78-81)."""
    gL = 1.0 + 1.0 / alL
    gR = 1.0 + 1.0 / alR
    pL = (gL - 1) * (EtL - 0.5 * rhoL * vxL * vxL)
    pR = (gR - 1) * (EtR - 0.5 * rhoR * vxR * vxR)
    aL = np.sqrt((gL * pL) / rhoL)
    aR = np.sqrt((gR * pR) / rhoR)
    lam = np.maximum(np.abs(vxL) + aL, np.abs(vxR) + aR)
    F = np.zeros((4 + len(YL),) + np.shape(rhoL))
    nc = np.zeros_like(F)
    for k in range(len(YL)):
        F[4 + k] = 0.5 * (YL[k] * vxL + YR[k] * vxR) * nx - lam * (YR[k] - YL[k])
    F[0] = 0.5 * ((rhoL * vxL + rhoR * vxR) * nx - lam * (rhoR - rhoL))
    F[1] = 0.5 * ((rhoL * vxL * vxL + pL + rhoR * vxR * vxR + pR) * nx - lam * (rhoR * vxR - rhoL * vxL))
    F[2] = 0.5 * (((EtL + pL) * vxL + (EtR + pR) * vxR) * nx - lam * (EtR - EtL))
    if gc:
        F[3] = 0.5 * ((rhoL * vxL * alL + rhoR * vxR * alR) * nx - lam * (rhoR * alR - rhoL * alL))
    else:
        F[3] = 0.5 * (-lam * (alR - alL))
        nc[3] = -0.5 * 0.5 * (vxL + vxR) * (alR - alL) * nx
    return F, nc


def _fhll(UL, SL, FL, UR, SR, FR):
    """fhll, code/src/face_fluxes/basic_fluxes.h:24-27."""
    return (SR * FL - SL * FR + SL * SR * (UR - UL)) / np.abs(SR - SL)


def _oned_hll(rhoL, rhoR, vxL, vxR, EtL, EtR, alL, alR, nx, YL=(), YR=(), gc=False):
    """oned_multifluid_hll, oned_multifluid_fluxes.h:117-226 (wave-speed estimate Toro 10.48).  As
    in the reference, the momentum row's HLL jump uses the velocities vxL, vxR
    (oned_multifluid_fluxes.h:196), and a face with SL == 0 or SR == 0 keeps a zero flux.  gc
    (GAMCONS; alphas divided by the caller, :131-134): the alpha row is the HLL flux of
    rho*alpha*u whose state jump is the divided alpha (:180-182, 195-197, 210-212)."""
    gL = 1.0 + 1.0 / alL
    gR = 1.0 + 1.0 / alR
    pL = (gL - 1) * (EtL - 0.5 * rhoL * vxL * vxL)
    pR = (gR - 1) * (EtR - 0.5 * rhoR * vxR * vxR)
    aL = np.sqrt((gL * pL) / rhoL)
    aR = np.sqrt((gR * pR) / rhoR)
    SL = np.minimum(vxL * nx - aL, vxR * nx - aR)
    SR = np.maximum(vxL * nx + aL, vxR * nx + aR)
    vnc = -0.5 * (vxL * nx + vxR * nx) * (alL - alR)
    vncabs = -0.5 * np.abs(vxL * nx + vxR * nx) * (alL - alR)
    fL = [rhoL * vxL * nx, (rhoL * vxL * vxL + pL) * nx, (EtL + pL) * vxL * nx]
    fR = [rhoR * vxR * nx, (rhoR * vxR * vxR + pR) * nx, (EtR + pR) * vxR * nx]
    with np.errstate(divide="ignore", invalid="ignore"):
        mid = [_fhll(rhoL, SL, fL[0], rhoR, SR, fR[0]), _fhll(vxL, SL, fL[1], vxR, SR, fR[1]),
               _fhll(EtL, SL, fL[2], EtR, SR, fR[2])]
        if gc:
            mid.append(_fhll(alL, SL, rhoL * vxL * alL * nx, alR, SR, rhoR * vxR * alR * nx))
        else:
            mid.append(_fhll(alL, SL, 0.0, alR, SR, 0.0) - 0.5 * np.abs(SR + SL) / np.abs(SR - SL) * vncabs)
    if gc:
        left = [fL[0], fL[1], fL[2], rhoL * vxL * alL * nx]
        right = [fR[0], fR[1], fR[2], rhoR * vxR * alR * nx]
    else:
        left = [fL[0], fL[1], fL[2], -0.5 * vncabs]
        right = [fR[0], fR[1], fR[2], 0.5 * vncabs]
    for k in range(len(YL)):  # mass fractions (oned_multifluid_fluxes.h:186-219)
        fYL, fYR = YL[k] * vxL * nx, YR[k] * vxR * nx
        with np.errstate(divide="ignore", invalid="ignore"):
            mid.append(_fhll(YL[k], SL, fYL, YR[k], SR, fYR))
        left.append(fYL)
        right.append(fYR)
    cL = SL > 0
    cM = (SL < 0) & (SR > 0)
    cR = (SR < 0) & ~cL & ~cM
    F = np.zeros((4 + len(YL),) + np.shape(rhoL))
    nc = np.zeros_like(F)
    for k in range(4 + len(YL)):
        F[k] = np.where(cL, left[k], np.where(cM, mid[k], np.where(cR, right[k], 0.0)))
    if not gc:
        nc[3] = -0.5 * vnc
    return F, nc


def _oned_roe(rhoL, rhoR, vxL, vxR, EtL, EtR, alL, alR, nx, YL=(), YR=(), gc=False):
    """oned_multifluid_roe, oned_multifluid_fluxes.h:237-382; mass fractions :358-370.  gc
    (GAMCONS; alphas divided by the caller, :252-255): central rho*alpha*u part in the alpha row
    (:348-350), no non-conservative term."""
    gL = 1.0 + 1.0 / alL
    gR = 1.0 + 1.0 / alR
    pL = (gL - 1) * (EtL - 0.5 * rhoL * vxL * vxL)
    pR = (gR - 1) * (EtR - 0.5 * rhoR * vxR * vxR)
    RT = np.sqrt(rhoR / rhoL)
    rho = RT * rhoL
    v = (vxL + RT * vxR) / (1 + RT)
    HL = (EtL + pL) / rhoL
    HR = (EtR + pR) / rhoR
    H = (HL + RT * HR) / (1 + RT)
    al = (alL + RT * alR) / (1 + RT)
    g = 1 + 1.0 / al
    a = np.sqrt((g - 1) * (H - 0.5 * v * v))
    iL = pL * alL
    iR = pR * alR
    i = (np.sqrt(rhoL) * iL + np.sqrt(rhoR) * iR) / (np.sqrt(rhoL) + np.sqrt(rhoR))
    Dp = (g - 1) * (g - 1) * (al * (iR - iL) - i * (alR - alL))
    p = (g - 1) * i
    dV = [(Dp - rho * a * (vxR - vxL)) / (2 * a * a), (rhoR - rhoL) - Dp / (a * a),
          (Dp + rho * a * (vxR - vxL)) / (2 * a * a), alR - alL]
    ws = [np.abs(v - a), np.abs(v), np.abs(v + a), np.abs(v)]
    z = np.zeros_like(v)
    one = np.ones_like(v)
    R = [[one, v - a, H - v * a, z], [one, v, 0.5 * v * v, z], [one, v + a, H + v * a, z], [z, z, p, one]]

    def diss(c):
        return ws[0] * dV[0] * R[0][c] + ws[1] * dV[1] * R[1][c] + ws[2] * dV[2] * R[2][c] + ws[3] * dV[3] * R[3][c]

    F = np.zeros((4 + len(YL),) + np.shape(rhoL))
    nc = np.zeros_like(F)
    for k in range(len(YL)):
        Y = (YL[k] / rhoL + RT * YR[k] / rhoR) / (1 + RT)
        dVY = YR[k] - YL[k] - (dV[0] + dV[1] + dV[2]) * Y
        F[4 + k] = 0.5 * (YL[k] * vxL + YR[k] * vxR) * nx - 0.5 * (ws[0] * dV[0] * Y + ws[1] * dV[1] * Y +
                                                                     ws[1] * dVY * 1 + ws[2] * dV[2] * Y)
    F[0] = 0.5 * (rhoL * vxL + rhoR * vxR) * nx - 0.5 * diss(0)
    F[1] = 0.5 * (rhoL * vxL * vxL + pL + rhoR * vxR * vxR + pR) * nx - 0.5 * diss(1)
    F[2] = 0.5 * ((EtL + pL) * vxL + (EtR + pR) * vxR) * nx - 0.5 * diss(2)
    if gc:
        F[3] = 0.5 * (rhoL * vxL * alL + rhoR * vxR * alR) * nx - 0.5 * diss(3)
    else:
        F[3] = -0.5 * diss(3)
        nc[3] = -0.5 * v * (alR - alL) * nx
    return F, nc


# ---------------------------------------------------------------------------------------------
# residual
# ---------------------------------------------------------------------------------------------

def _reflect(S: Setup, UF: np.ndarray) -> None:
    """LrflctiveBoundary / rflctive, code/src/bc/boundaries.cu:20-67: the outside trace (side 1)
    of each reflective face gets the mirrored velocity (1D: sign flip)."""
    if S.n_reflective <= 0:
        return
    faces = S.a["boundaryMap"][:S.n_reflective]
    if S.D == 1:
        UF[faces, 1, 1, :] = -UF[faces, 1, 1, :]
        return
    n = S.a["normals"].reshape(S.M_T, S.D)
    nx = n[faces, 0][:, None]
    ny = n[faces, 1][:, None]
    nx2, ny2 = nx * nx, ny * ny
    m2nxny = -2 * nx * ny
    inv = 1.0 / (nx2 + ny2)
    vxL = UF[faces, 1, 0, :].copy()
    vyL = UF[faces, 2, 0, :].copy()
    UF[faces, 1, 1, :] = inv * ((-nx2 + ny2) * vxL + m2nxny * vyL)
    UF[faces, 2, 1, :] = inv * (m2nxny * vxL + (nx2 - ny2) * vyL)


def _evaluate_sf(S: Setup, Ug, dUg, invJac):
    """evaluate_sf, code/src/physics/physics.cu:27-363 (1D multifluid :96-143, 2D :248-301).  GAMCONS:
    gamma = 1 + rho/(stored field) and the conservative flux rho*u/(gamma-1) with no source
    (:100-104, :122-124; 2D :253-257, :278-281)."""
    NE, NF, NG, D = S.N_E, S.N_F, S.N_G, S.D
    s = np.zeros((NE, NF, NG))
    f = np.zeros((NE, NF, NG, D))
    rho = Ug[:, 0]
    if D == 1:
        u = Ug[:, 1] / rho
        Et = Ug[:, 2]
        gam = 1 + (rho if S.gamcons else 1.0) / Ug[:, 3]
        p = (gam - 1) * (Et - 0.5 * rho * u * u)
        s[:, 1] = rho * S.gx
        s[:, 2] = rho * u * S.gx
        f[:, 0, :, 0] = rho * u
        f[:, 1, :, 0] = rho * u * u + p
        f[:, 2, :, 0] = (Et + p) * u
        if S.gamcons:
            f[:, 3, :, 0] = rho * u * (1 / (gam - 1))
        else:
            s[:, 3] = -u * dUg[:, 3, :, 0] * invJac.reshape(NE, NG)
        for k in range(4, NF):  # mass fractions: flux rho*Y_k u (physics.cu:130-134)
            f[:, k, :, 0] = Ug[:, k] * u
        return s, f
    u = Ug[:, 1] / rho
    v = Ug[:, 2] / rho
    Et = Ug[:, 3]
    gam = 1 + (rho if S.gamcons else 1.0) / Ug[:, 4]
    p = (gam - 1) * (Et - 0.5 * rho * (u * u + v * v))
    s[:, 1] = rho * S.gx
    s[:, 2] = rho * S.gy
    s[:, 3] = rho * (u * S.gx + v * S.gy)
    f[:, 0, :, 0] = rho * u
    f[:, 1, :, 0] = rho * u * u + p
    f[:, 2, :, 0] = rho * u * v
    f[:, 3, :, 0] = (Et + p) * u
    f[:, 0, :, 1] = rho * v
    f[:, 1, :, 1] = rho * u * v
    f[:, 2, :, 1] = rho * v * v + p
    f[:, 3, :, 1] = (Et + p) * v
    if S.gamcons:
        f[:, 4, :, 0] = rho * u * (1 / (gam - 1))
        f[:, 4, :, 1] = rho * v * (1 / (gam - 1))
    else:
        iJ = invJac.reshape(NE, NG, D, D)  # [e, g, alpha, a]: d xi_a / d x_alpha
        vg = np.zeros((NE, NG))
        for al in range(D):
            vg += -u * dUg[:, 4, :, al] * iJ[:, :, 0, al] - v * dUg[:, 4, :, al] * iJ[:, :, 1, al]
        s[:, 4] = vg
    for k in range(5, NF):  # mass fractions: flux rho*Y_k (u, v) (physics.cu:293-298)
        f[:, k, :, 0] = Ug[:, k] * u
        f[:, k, :, 1] = Ug[:, k] * v
    return s, f


def _evaluate_q(S: Setup, UgF):
    """evaluate_q, physics.cu:367-811: Riemann flux F and non-conservative term nc per face point,
    q[t,f,0] = -F + nc, q[t,f,1] = F + nc (physics.cu:800-804)."""
    n = S.a["normals"].reshape(S.M_T, S.D)
    L, R = UgF[:, :, 0, :], UgF[:, :, 1, :]  # (M_T, N_F, M_G)
    nx = n[:, 0][:, None]
    ka = S.D + 2                              # the gamma-model field
    alL, alR = L[:, ka], R[:, ka]
    if S.gamcons:                             # divided by the density inside each flux function
        alL, alR = alL / L[:, 0], alR / R[:, 0]
        if S.D == 2 and S.flux == "rusanov":  # twod_multifluid_fluxes.h:51-52: alphaL = alphaL/rhoL;
            alR = alL / L[:, 0]                 # alphaR = alphaL/rhoL (the divided left alpha, again)
    if S.D == 1:
        fn = {"rusanov": _oned_rusanov, "hll": _oned_hll, "roe": _oned_roe}[S.flux]
        F, nc = fn(L[:, 0], R[:, 0], L[:, 1] / L[:, 0], R[:, 1] / R[:, 0], L[:, 2], R[:, 2], alL, alR, nx,
                   [L[:, k] for k in range(4, S.N_F)], [R[:, k] for k in range(4, S.N_F)], gc=S.gamcons)
    else:
        ny = n[:, 1][:, None]
        fn = {"rusanov": _twod_rusanov, "roe": _twod_roe}[S.flux]
        F, nc = fn(L[:, 0], R[:, 0], L[:, 1] / L[:, 0], R[:, 1] / R[:, 0], L[:, 2] / L[:, 0], R[:, 2] / R[:, 0],
                   L[:, 3], R[:, 3], alL, alR, nx, ny, [L[:, k] for k in range(5, S.N_F)],
                   [R[:, k] for k in range(5, S.N_F)], gc=S.gamcons)
    F = np.moveaxis(F, 0, 1)    # (M_T, N_F, M_G)
    nc = np.moveaxis(nc, 0, 1)
    q = np.empty_like(UgF)
    q[:, :, 0, :] = -F + nc
    q[:, :, 1, :] = F + nc
    return q


def residual(S: Setup, U: np.ndarray) -> np.ndarray:
    """f_rk = S + F + Q of DG_SOLVER::dg_solver (dg_solver.h:292-364), before the inverse mass
    matrix: collocation by the basis matrices (the blasGemm calls, column-major N_s x (N_E N_F)),
    physics, Riemann fluxes, Jacobian scaling (kernels.cu redistribute_sf/_q) and lifting,
    interface contributions gathered through invmap (kernels.cu mapToElement)."""
    a = S.a
    NE, NF, Ns, NG, D, MT, Ms, MG, NN = S.N_E, S.N_F, S.N_s, S.N_G, S.D, S.M_T, S.M_s, S.M_G, S.N_N
    U = np.asarray(U, np.float64)
    cols = U.reshape(NE * NF, Ns)
    UF = U[a["map"]].reshape(MT, NF, 2, Ms)                     # mapToFace, kernels.cu:41-75
    _reflect(S, UF)
    phi = a["phi"].reshape(Ns, NG)                              # phi[g + i*N_G]
    dphi = a["dphi"].reshape(Ns, NG * D)                        # dphi[(g*D+a) + i*N_G*D]
    psi = a["psi"].reshape(Ms, MG)
    Ug = (cols @ phi).reshape(NE, NF, NG)
    dUg = (cols @ dphi).reshape(NE, NF, NG, D)
    UgF = (UF.reshape(-1, Ms) @ psi).reshape(MT, NF, 2, MG)
    s, f = _evaluate_sf(S, Ug, dUg, a["invJac"])
    q = _evaluate_q(S, UgF)
    J = a["J"].reshape(NE)
    iJ = a["invJac"].reshape(NE, NG, D, D)
    sJ = s * J[:, None, None]                                    # redistribute_sf, kernels.cu:171-206
    fJ = np.zeros_like(f)
    for al in range(D):
        acc = np.zeros((NE, NF, NG))
        for k in range(D):
            acc += iJ[:, None, :, al, k] * f[:, :, :, k] * J[:, None, None]
        fJ[:, :, :, al] = acc
    phi_w = a["phi_w"].reshape(Ns, NG)
    dphi_w = a["dphi_w"].reshape(Ns, NG * D)
    Sv = sJ.reshape(-1, NG) @ phi_w.T
    Fv = fJ.reshape(-1, NG * D) @ dphi_w.T
    qJ = q * a["JF"].reshape(MT, 1, 2, 1)                        # redistribute_q, kernels.cu:208-236
    Qtcj = (qJ.reshape(-1, MG) @ a["psi_w"].reshape(Ms, MG).T).reshape(-1)
    inv = a["invmap"].reshape(NE, NF, Ms * NN, 2)                # mapToElement, kernels.cu:78-134
    # sums in the reference's order: per (e, f), over the M_s*N_N face nodes in invmap order
    dest = (np.arange(NE * NF).reshape(NE, NF, 1) * Ns + inv[..., 0]).reshape(-1)
    Q = np.bincount(dest, weights=Qtcj[inv[..., 1]].reshape(-1), minlength=NE * NF * Ns).reshape(NE, NF, Ns)
    return (Sv.reshape(NE, NF, Ns) + Fv.reshape(NE, NF, Ns) + Q).reshape(-1)


def solve(S: Setup, dt: float, f: np.ndarray) -> np.ndarray:
    """DU = dt * Minv_e f_e, solve() in rk_kernels.cu:22-57 (Minv[(e*N_s+ii)*N_s+i])."""
    M = S.a["Minv"].reshape(S.N_E, S.N_s, S.N_s)
    fe = np.asarray(f).reshape(S.N_E, S.N_F, S.N_s)
    return (dt * np.einsum("eji,efj->efi", M, fe)).reshape(-1)


def dt_from_cfl(S: Setup, U: np.ndarray, cfl_scaled: float | None = None) -> float:
    """RK::DtFromCFL (rk.cc:250-272): CFL / max over nodes of |u|+a (2D: max(|u|+a, |v|+a))."""
    V = np.asarray(U).reshape(S.N_E, S.N_F, S.N_s)
    rho = V[:, 0]
    if S.D == 1:
        u = V[:, 1] / rho
        g = 1.0 + (rho if S.gamcons else 1.0) / V[:, 3]     # upa.h:61-70
        p = (g - 1) * (V[:, 2] - 0.5 * rho * u * u)
        upa = np.abs(u) + np.sqrt(g * p / rho)
    else:
        u = V[:, 1] / rho
        v = V[:, 2] / rho
        g = 1.0 + (rho if S.gamcons else 1.0) / V[:, 4]     # upa.h:72-85
        p = (g - 1) * (V[:, 3] - 0.5 * rho * (u * u + v * v))
        a = np.sqrt(g * p / rho)
        upa = np.maximum(np.abs(u) + a, np.abs(v) + a)
    c = S.cfl_scaled if cfl_scaled is None else cfl_scaled
    return float(c / upa.reshape(-1)[np.argmax(np.abs(upa.reshape(-1)))])


# ---------------------------------------------------------------------------------------------
# limiter (hierarchical reconstruction on scaled monomials)
# ---------------------------------------------------------------------------------------------

def _int_deriv(k: int, n: int) -> float:
    """integrate_monomial_derivative, limiting_kernels.cu:1748-1760."""
    num = n - k + 1
    return 2.0 / factorial(num) if num % 2 else 0.0


def _int_deriv_bounds(k: int, n: int, a: float, b: float) -> float:
    """integrate_monomial_derivative_bounds, limiting_kernels.cu:1762-1775."""
    num = n - k + 1
    return (b ** num - a ** num) / factorial(num)


def _minmod(a, b):
    """2-argument minmod, limiting_kernels.cu:1470-1485."""
    sa = np.sign(a)
    out = sa * np.minimum(np.abs(a), np.abs(b))
    return np.where(sa != np.sign(b), 0.0, out)


def limit_monomial(AL, AC, AR):
    """limit_monomial, limiting_kernels.cu:1534-1585: for m = N..1, MUSCL minmod of the averaged
    (m-1)-th derivatives after removing the already-limited higher terms; coefficient 0 is the
    recovered cell average.  Vectorised over leading axes; last axis = monomial coefficient."""
    N = AC.shape[-1] - 1
    Alim = np.zeros_like(AC)
    avgLC = np.zeros(AC.shape[:-1])
    for m in range(N, 0, -1):
        dUL = np.zeros(AC.shape[:-1])
        dUC = np.zeros_like(dUL)
        dUR = np.zeros_like(dUL)
        RL = np.zeros_like(dUL)
        RC = np.zeros_like(dUL)
        RR = np.zeros_like(dUL)
        for n in range(m - 1, N + 1):
            w = _int_deriv(m - 1, n)
            dUL = dUL + AL[..., n] * w
            dUC = dUC + AC[..., n] * w
            dUR = dUR + AR[..., n] * w
            if n >= m + 1:
                al = Alim[..., n]
                RL = RL + al * _int_deriv_bounds(m - 1, n, -3, -1)
                RC = RC + al * w
                RR = RR + al * _int_deriv_bounds(m - 1, n, 1, 3)
        avgLL = 0.5 * (dUL - RL)
        avgLC = 0.5 * (dUC - RC)
        avgLR = 0.5 * (dUR - RR)
        Alim[..., m] = _minmod(0.5 * (avgLC - avgLL), 0.5 * (avgLR - avgLC))
    Alim[..., 0] = avgLC
    return Alim


def average_monomial(A):
    """average_monomial, limiting_kernels.cu:1777-1790: slopes to zero, keep the cell average."""
    N = A.shape[-1] - 1
    avg = sum(A[..., n] * _int_deriv(0, n) for n in range(N + 1))
    out = np.zeros_like(A)
    out[..., 0] = 0.5 * avg
    return out


def hrl1d(S: Setup, A: np.ndarray, offxy: int, all_fields: bool) -> np.ndarray:
    """hrl1D, limiting_kernels.cu:245-320, on A shaped (N_E, Nfields, slices, N+1).
    Boundary code = -neighbour (right wins); 2: average; 3: average except the wall-normal
    momentum (field 1 for x, 2 for y) when the array holds all fields, which is copied;
    4 ("leave data unchanged"): copied here (the reference leaves its output buffer as it was);
    otherwise full limiting with the two neighbours."""
    nb = S.a["neighbors"].reshape(S.N_E, S.N_N)
    left, right = nb[:, offxy], nb[:, offxy + 1]
    phys = np.zeros(S.N_E, dtype=np.int64)
    phys = np.where(left < 0, -left, phys)
    phys = np.where(right < 0, -right, phys)
    full = ~np.isin(phys, (2, 3, 4))
    Alim = np.array(A, copy=True)
    lidx = np.where(left >= 0, left, 0)
    ridx = np.where(right >= 0, right, 0)
    lim = limit_monomial(A[lidx], A, A[ridx])
    avg = average_monomial(A)
    Alim[full] = lim[full]
    Alim[phys == 2] = avg[phys == 2]
    w = phys == 3
    if np.any(w):
        Alim[w] = avg[w]
        if all_fields:
            un = 1 if offxy == 0 else 2
            Alim[w, un] = A[w, un]
    return Alim


def _apply(T: np.ndarray, X: np.ndarray, Ns: int) -> np.ndarray:
    """blasGemm('N','N', N_s, cols, N_s, 1, T, N_s, X, N_s): per column X_c -> T X_c, T column-major."""
    return X.reshape(-1, Ns) @ T.reshape(Ns, Ns)


def _binom(n: int, k: int) -> int:
    from math import comb
    return comb(n, k)


def _internal_energy(p, g):
    """internal_energy_multifluid, limiting_kernels.cu:160-200: monomial coefficients of p/(gamma-1)
    as the Leibniz product of those of p and 1/(gamma-1): I_m = sum_k C(m,k) p_{m-k} g_k."""
    out = np.zeros_like(p)
    N1 = p.shape[-1]
    for m in range(N1):
        acc = np.zeros(p.shape[:-1])
        for k in range(m + 1):
            acc = acc + float(_binom(m, k)) * p[..., m - k] * g[..., k]
        out[..., m] = acc
    return out


def _reconstruct_energy(rhoe, K, EMono):
    """reconstruct_energy, limiting_kernels.cu:111-158: E_m = rhoe_m + K_m for m >= 1, and the
    average-preserving correction of E_0."""
    N1 = rhoe.shape[-1]
    E = rhoe + K
    E0 = EMono[..., 0].copy()
    for k in range(2, N1, 2):
        E0 = E0 - 1.0 / factorial(k + 1) * (E[..., k] - EMono[..., k])
    E[..., 0] = E0
    return E


def limit(S: Setup, U: np.ndarray) -> np.ndarray:
    """The deck's limiter on U (reference Limiting::HRlimiting / M2limiting, limiting.cc)."""
    U = np.asarray(U, np.float64)
    if S.limiter == "none":
        return U.copy()
    if S.limiter == "hrl":
        return _hr(S, U)
    if S.limiter == "m2l":
        if S.gamcons:  # limiting.cc:193-194 / 410-411 stop the run
            raise NotImplementedError("M2L is only implemented for gamncon")
        return _m2(S, U)
    if S.limiter == "prl":
        return prim2cons(S, _hr(S, cons2prim(S, U)))
    if S.limiter in ("hri", "m2i", "pri", "p0i"):
        return _sensor_gated(S, U)
    raise NotImplementedError(f"limiter {S.limiter}")


def _hr(S: Setup, U: np.ndarray) -> np.ndarray:
    """Limiting::HRlimiting, limiting.cc:11-52 (1D; 2D Cartesian x then y slices)."""
    a, Ns, NE, NF = S.a, S.N_s, S.N_E, S.N_F
    if S.D == 1:
        A = _apply(a["Lag2Mono"], U, Ns).reshape(NE, NF, 1, Ns)
        Al = hrl1d(S, A, 0, True)
        return _apply(a["Mono2Lag"], Al, Ns).reshape(-1)
    n1 = S.order + 1
    A = _apply(a["Lag2MonoX"], U, Ns).reshape(NE, NF, n1, n1)
    Al = hrl1d(S, A, 0, True)
    A = _apply(a["MonoX2MonoY"], Al, Ns).reshape(NE, NF, n1, n1)
    Al = hrl1d(S, A, 2, True)
    return _apply(a["MonoY2Lag"], Al, Ns).reshape(-1)


def _m2(S: Setup, U: np.ndarray) -> np.ndarray:
    """Limiting::M2limiting, gamma model: limit rho, momenta, 1/(gamma-1) and pressure, rebuild the
    energy from the limited pressure and kinetic energy (limiting.cc:132-196 in 1D, :271-409 for
    2D Cartesian meshes: x slices, then y slices of the x-limited fields)."""
    a, Ns, NE, NF = S.a, S.N_s, S.N_E, S.N_F
    V = U.reshape(NE, NF, Ns)
    if S.D == 1:
        L2M, M2L = a["Lag2Mono"], a["Mono2Lag"]

        def lim(x):
            return hrl1d(S, _apply(L2M, x, Ns).reshape(NE, 1, 1, Ns), 0, False)

        rhoL = lim(V[:, 0])
        rhouL = lim(V[:, 1])
        gL = lim(V[:, 3])
        rho = _apply(M2L, rhoL, Ns)
        rhou = _apply(M2L, rhouL, Ns)
        gam = _apply(M2L, gL, Ns)
        p = (1.0 + 1.0 / V[:, 3] - 1) * (V[:, 2] - 0.5 * V[:, 1] * V[:, 1] / V[:, 0])  # pressure, physics.cu:891-958
        pL = lim(p)
        K = _apply(L2M, 0.5 * rhou * rhou / rho, Ns).reshape(NE, 1, 1, Ns)      # kinetic_energy1D
        rhoe = _internal_energy(pL, gL)
        EM = _apply(L2M, V[:, 2], Ns).reshape(NE, 1, 1, Ns)
        E = _apply(M2L, _reconstruct_energy(rhoe, K, EM), Ns)
        out = np.empty_like(V)
        out[:, 0], out[:, 1], out[:, 2], out[:, 3] = rho, rhou, E, gam
        for k in range(4, NF):  # mass fractions like the density (limiting.cc:184-193)
            out[:, k] = _apply(M2L, lim(V[:, k]), Ns)
        return out.reshape(-1)
    n1 = S.order + 1
    L2MX, MX2L, L2MY, MY2L = a["Lag2MonoX"], a["MonoX2Lag"], a["Lag2MonoY"], a["MonoY2Lag"]

    def mono(T, x):
        return _apply(T, x, Ns).reshape(NE, 1, n1, n1)

    # x slices
    lims = {}
    nodal = {}
    ynames = [f"y{k}" for k in range(5, NF)]  # mass fractions like the density (limiting.cc:323-331, 396-404)
    for name, x in (("rho", V[:, 0]), ("rhou", V[:, 1]), ("rhov", V[:, 2]), ("g", V[:, 4])) + tuple(
            (f"y{k}", V[:, k]) for k in range(5, NF)):
        lims[name] = hrl1d(S, mono(L2MX, x), 0, False)
        nodal[name] = _apply(MX2L, lims[name], Ns)
    rho, ru, rv = V[:, 0], V[:, 1], V[:, 2]
    p = (1.0 + 1.0 / V[:, 4] - 1) * (V[:, 3] - 0.5 * (ru * ru + rv * rv) / rho)
    pL = hrl1d(S, mono(L2MX, p), 0, False)
    pres = _apply(MX2L, pL, Ns)
    K = mono(L2MX, 0.5 * (nodal["rhou"] ** 2 + nodal["rhov"] ** 2) / nodal["rho"])
    rhoe = _internal_energy(pL, lims["g"])
    E = _apply(MX2L, _reconstruct_energy(rhoe, K, mono(L2MX, V[:, 3])), Ns)
    # y slices of the x-limited fields
    for name in ("rho", "rhou", "rhov", "g", *ynames):
        lims[name] = hrl1d(S, mono(L2MY, nodal[name]), 2, False)
        nodal[name] = _apply(MY2L, lims[name], Ns)
    pL = hrl1d(S, mono(L2MY, pres), 2, False)
    K = mono(L2MY, 0.5 * (nodal["rhou"] ** 2 + nodal["rhov"] ** 2) / nodal["rho"])
    rhoe = _internal_energy(pL, lims["g"])
    E = _apply(MY2L, _reconstruct_energy(rhoe, K, mono(L2MY, E)), Ns)
    out = np.empty_like(V)
    out[:, 0], out[:, 1], out[:, 2], out[:, 3], out[:, 4] = nodal["rho"], nodal["rhou"], nodal["rhov"], E, nodal["g"]
    for k in range(5, NF):
        out[:, k] = nodal[f"y{k}"]
    return out.reshape(-1)


# ---------------------------------------------------------------------------------------------
# time stepping
# ---------------------------------------------------------------------------------------------

RK4_BETA = (0.0, 0.5, 0.5, 1.0)               # rk.h:46-49
RK4_GAMMA = (1.0 / 6.0, 2.0 / 6.0, 2.0 / 6.0, 1.0 / 6.0)


def rk4_steps(S: Setup, U: np.ndarray, dt: float, nsteps: int) -> np.ndarray:
    """nsteps of the RK4 step body of RK::RK_integration (rk.cc:155-209): Ustar = Us + beta_k DU,
    limited for k > 0, DU = dt Minv f(Ustar), U += gamma_k DU; the limiter on the end-of-step
    state.  dt <= 0 takes the CFL step (rk.cc:141) each step."""
    U = np.array(U, np.float64, copy=True)
    DU = np.zeros_like(U)
    for _ in range(nsteps):
        Dt = dt if dt > 0 else dt_from_cfl(S, U)
        Us = U.copy()
        for k in range(4):
            Ustar = Us.copy()
            if k > 0:
                Ustar = limit(S, Ustar + RK4_BETA[k] * DU)
            DU = solve(S, Dt, residual(S, Ustar))
            U = U + RK4_GAMMA[k] * DU
        U = limit(S, U)
    return U


def ssprk3_steps(S: Setup, U: np.ndarray, dt: float, nsteps: int) -> np.ndarray:
    """nsteps of Shu-Osher SSP-RK3, each stage output limited as the reference limits RK stage
    inputs and the end-of-step state (rk.cc:176-209):
        U1 = L(Un + DU(Un)),  U2 = L(3/4 Un + 1/4 (U1 + DU(U1))),  U = L(1/3 Un + 2/3 (U2 + DU(U2)))
    with DU(X) = dt Minv f(X) and L the limiter.  dt <= 0 takes the CFL step of Un."""
    U = np.array(U, np.float64, copy=True)
    for _ in range(nsteps):
        Dt = dt if dt > 0 else dt_from_cfl(S, U)
        Un = U
        U1 = limit(S, Un + solve(S, Dt, residual(S, Un)))
        U2 = limit(S, 0.75 * Un + 0.25 * (U1 + solve(S, Dt, residual(S, U1))))
        U = limit(S, (1.0 / 3.0) * Un + (2.0 / 3.0) * (U2 + solve(S, Dt, residual(S, U2))))
    return U


# ---------------------------------------------------------------------------------------------
# sensors and the sensor-gated (per-element) limiters
# ---------------------------------------------------------------------------------------------

def cons2prim(S: Setup, U: np.ndarray) -> np.ndarray:
    """Cons2Prim, limiting_kernels.cu:1009-1059 (gamma model): (rho, u, [v,] p, alpha)."""
    V = np.array(U, np.float64, copy=True).reshape(S.N_E, S.N_F, S.N_s)
    rho, ru = V[:, 0].copy(), V[:, 1].copy()
    rv = V[:, 2].copy() if S.D == 2 else np.zeros_like(rho)
    E, al = V[:, S.D + 1].copy(), V[:, S.D + 2].copy()
    V[:, 1] = ru / rho
    if S.D == 2:
        V[:, 2] = rv / rho
    V[:, S.D + 1] = (E - 0.0 - 0.5 * (ru * ru + rv * rv) / rho) / al
    return V.reshape(-1)


def prim2cons(S: Setup, W: np.ndarray) -> np.ndarray:
    """Prim2Cons, limiting_kernels.cu:957-1007: rho u -> momentum, p alpha + kinetic -> E."""
    V = np.array(W, np.float64, copy=True).reshape(S.N_E, S.N_F, S.N_s)
    rho, u = V[:, 0].copy(), V[:, 1].copy()
    v = V[:, 2].copy() if S.D == 2 else np.zeros_like(rho)
    p, al = V[:, S.D + 1].copy(), V[:, S.D + 2].copy()
    V[:, 1] = rho * u
    if S.D == 2:
        V[:, 2] = rho * v
    V[:, S.D + 1] = p * al + 0.0 + 0.5 * rho * (u * u + v * v)
    return V.reshape(-1)


def _cell_means(S: Setup, U: np.ndarray) -> np.ndarray:
    """SENSOR::sensing's "average solution" (sensor.cc:26): nodal mean per element and field."""
    V = np.asarray(U).reshape(S.N_E, S.N_F, S.N_s)
    acc = V[:, :, 0].copy()
    for i in range(1, S.N_s):
        acc = acc + V[:, :, i]
    return acc * (1.0 / S.N_s)


def sensors(S: Setup, U: np.ndarray) -> np.ndarray:
    """SENSOR::sensing (sensor.cc:11-35) with calc_sensors (sensor_kernels.cu:19-165), CPU order.

    Each element not yet flagged tests its neighbours in order (left, right[, bottom, top]) with
    Roe-averaged cell means: sensor 1 (contact, density wave strength), sensor 2 (shock: converging
    acoustic characteristics and a pressure jump), sensor 3 (contact, gamma jump), each against its
    deck threshold; the first hit flags the element and that neighbour with the sensor number and
    stops its loop; a boundary neighbour (negative index) flags the element with 1 and stops.
    Elements are visited in index order and an element flagged by an earlier one skips its own
    tests -- this sequential order is part of the result."""
    th = list(S.thresholds)
    on1, on2, on3 = len(th) > 0, len(th) > 1, len(th) > 2
    t1 = th[0] if on1 else 0.0
    t2 = th[1] if on2 else 0.0
    t3 = th[2] if on3 else 0.0
    A = _cell_means(S, U)
    rho = A[:, 0]
    vx = A[:, 1] / rho
    vy = A[:, 2] / rho if S.D == 2 else np.zeros_like(rho)
    Et = A[:, S.D + 1]
    al = A[:, S.D + 2]
    gam = 1.0 + 1.0 / al
    pinf = (1 - 1.0 / gam) * 0.0
    p = (gam - 1) * (Et - 0.0 - 0.5 * rho * (vx * vx + vy * vy))
    ie = p * al
    with np.errstate(invalid="ignore", divide="ignore"):
        a = np.sqrt((gam * (p + pinf)) / rho)
    H = (Et + p) / rho
    nb = S.a["neighbors"].reshape(S.N_E, S.N_N)
    hit = np.zeros((S.N_E, S.N_N), dtype=np.int64)  # 0 none, 1..3 sensor, -1 boundary
    with np.errstate(invalid="ignore", divide="ignore"):
        for nn in range(S.N_N):
            r = nb[:, nn]
            ok = r >= 0
            R = np.where(ok, r, 0)
            RT = np.sqrt(rho[R] / rho)
            ux = (vx + RT * vx[R]) / (1 + RT)
            uy = (vy + RT * vy[R]) / (1 + RT)
            alr = (al + RT * al[R]) / (1 + RT)
            gr = 1 + 1.0 / alr
            Hr = (H + RT * H[R]) / (1 + RT)
            ar = np.sqrt((gr - 1) * (Hr - 0.5 * (ux * ux + uy * uy)))
            ir = (ie + RT * ie[R]) / (1 + RT)
            drho = rho[R] - rho
            dp = (gr - 1) * (gr - 1) * (alr * (ie[R] - ie) - ir * (al[R] - al))
            dV2 = drho - dp / (ar * ar)
            G = np.abs(dV2) / (rho + rho[R])
            d1 = on1 & (2 * G / ((1 + G) * (1 + G)) > t1)
            shock = ((vx - a > ux - ar) & (ux - ar > vx[R] - a[R])) | ((vy - a > uy - ar) & (uy - ar > vy[R] - a[R]))
            psi = np.abs(p[R] - p) / (p + p[R])
            d2 = on2 & shock & (2 * psi / ((1 + psi) * (1 + psi)) > t2)
            G3 = np.abs(gam[R] - gam) / (gam + gam[R])
            d3 = on3 & (2 * G3 / ((1 + G3) * (1 + G3)) > t3)
            typ = np.where(d1, 1, np.where(d2, 2, np.where(d3, 3, 0)))
            hit[:, nn] = np.where(ok, typ, -1)
    sens = np.zeros(S.N_E, dtype=np.int64)
    for e in range(S.N_E):
        if sens[e] != 0:
            continue
        for nn in range(S.N_N):
            h = hit[e, nn]
            if h == -1:
                sens[e] = 1
                break
            if h > 0:
                sens[e] = h
                sens[nb[e, nn]] = h
                break
    return sens


def _set2average(L2M, M2L, X, n1, Ns):
    """set2average, limiting_kernels.cu:1792-1827: every slice to its average; returns the nodal
    result and the limited monomial coefficients."""
    A = _apply(L2M, X, Ns).reshape(X.shape[:-1] + (Ns // n1, n1))
    Al = average_monomial(A).reshape(X.shape)
    return _apply(M2L, Al, Ns).reshape(X.shape), Al


def _HR(L2M, M2L, XL, XC, XR, n1, Ns):
    """HR, limiting_kernels.cu:1829-1868: per slice limit_monomial of the three cells."""
    sh = XC.shape[:-1] + (Ns // n1, n1)
    Al = limit_monomial(_apply(L2M, XL, Ns).reshape(sh), _apply(L2M, XC, Ns).reshape(sh),
                        _apply(L2M, XR, Ns).reshape(sh)).reshape(XC.shape)
    return _apply(M2L, Al, Ns).reshape(XC.shape), Al


def _phys_codes(S: Setup, offxy: int):
    nb = S.a["neighbors"].reshape(S.N_E, S.N_N)
    left, right = nb[:, offxy], nb[:, offxy + 1]
    phys = np.zeros(S.N_E, dtype=np.int64)
    phys = np.where(left < 0, -left, phys)
    phys = np.where(right < 0, -right, phys)
    return phys, np.where(left >= 0, left, 0), np.where(right >= 0, right, 0)


def _hri_pass(S: Setup, U: np.ndarray, offxy: int, L2M, M2L, n1: int) -> np.ndarray:
    """hri1D, limiting_kernels.cu:322-429, evaluated for every element (callers keep the flagged
    ones): per field, HR with the neighbours' nodal values, averages at transmissive boundaries,
    averages except the wall-normal momentum at walls, unchanged for code 4."""
    Ns = S.N_s
    V = np.asarray(U).reshape(S.N_E, S.N_F, Ns)
    phys, L, R = _phys_codes(S, offxy)
    full, _ = _HR(L2M, M2L, V[L], V, V[R], n1, Ns)
    avg, _ = _set2average(L2M, M2L, V, n1, Ns)
    out = V.copy()
    m = ~np.isin(phys, (2, 3, 4))
    out[m] = full[m]
    out[phys == 2] = avg[phys == 2]
    w = phys == 3
    un = 1 if offxy == 0 else 2
    for fc in range(S.N_F):
        if fc != un:
            out[w, fc] = avg[w, fc]
    return out.reshape(-1)


def _m2i_pass(S: Setup, U: np.ndarray, offxy: int, L2M, M2L, n1: int) -> np.ndarray:
    """m2i1D, limiting_kernels.cu:431-722 (gamma model), for every element: HR (or averaging at
    boundaries) of rho, momenta, 1/(gamma-1) and the nodal pressure, then the total energy rebuilt
    from the limited pressure, 1/(gamma-1) and kinetic energy (limiting_kernels.cu:1870-1990)."""
    Ns, D = S.N_s, S.D
    V = np.asarray(U).reshape(S.N_E, S.N_F, Ns)
    phys, L, R = _phys_codes(S, offxy)
    iE, iG = D + 1, D + 2
    mom = [1, 2] if D == 2 else [1]

    def press(X):
        kin = X[:, 1] * X[:, 1] + (X[:, 2] * X[:, 2] if D == 2 else 0.0)
        return (X[:, iE] - 0.5 * kin / X[:, 0]) / X[:, iG]

    pC, pL, pR = press(V), press(V[L]), press(V[R])
    out = V.copy()
    # limited / averaged primitive-like quantities, per element case
    hr = {k: _HR(L2M, M2L, V[L][:, k], V[:, k], V[R][:, k], n1, Ns) for k in [0] + mom + [iG]}
    av = {k: _set2average(L2M, M2L, V[:, k], n1, Ns) for k in [0] + mom + [iG]}
    hrp = _HR(L2M, M2L, pL, pC, pR, n1, Ns)
    avp = _set2average(L2M, M2L, pC, n1, Ns)
    full = ~np.isin(phys, (2, 3, 4))
    walls = phys == 3
    trans = phys == 2
    glim = np.where(full[:, None], hr[iG][1], av[iG][1])
    plim = np.where(full[:, None], hrp[1], avp[1])
    for k in [0] + mom + [iG]:
        out[full, k] = hr[k][0][full]
        out[trans, k] = av[k][0][trans]
    out[walls, 0] = av[0][0][walls]
    out[walls, iG] = av[iG][0][walls]
    if D == 2:
        tang = 2 if offxy == 0 else 1   # the momentum along the wall is averaged, the normal one kept
        out[walls, tang] = av[tang][0][walls]
    kin = out[:, 1] * out[:, 1] + (out[:, 2] * out[:, 2] if D == 2 else 0.0)
    K = _apply(L2M, 0.5 * kin / out[:, 0], Ns)
    sl = (S.N_E, Ns // n1, n1)
    rhoe = _internal_energy(plim.reshape(sl), glim.reshape(sl))
    EM = _apply(L2M, V[:, iE], Ns).reshape(sl)
    E = _apply(M2L, _reconstruct_energy(rhoe, K.reshape(sl), EM).reshape(S.N_E, Ns), Ns)
    act = full | walls | trans
    out[act, iE] = E[act]
    return out.reshape(-1)


def p0i_average(S: Setup, U: np.ndarray) -> np.ndarray:
    """p0i, limiting_kernels.cu:723-770: every node set to the cell average
    sum_g sum_i phi_w[i*N_G+g] U_i / |reference element| (4 for quads; 2 for lines, where the
    reference leaves the area unset, main.cc:284)."""
    ref_area = 4.0 if S.D == 2 else 2.0
    V = np.asarray(U).reshape(S.N_E, S.N_F, S.N_s)
    pw = S.a["phi_w"].reshape(S.N_s, S.N_G)
    avg = np.einsum("efi,ig->ef", V, pw) / ref_area
    return np.broadcast_to(avg[:, :, None], V.shape).reshape(-1).copy()


def _sensor_gated(S: Setup, U: np.ndarray) -> np.ndarray:
    """Limiting::HRIlimiting / PRIlimiting / M2Ilimiting / P0Ilimiting (limiting.cc:596-742): the
    sensor on the conserved state, then the per-element limiter on the flagged elements only, x
    slices then y slices (each pass reading the previous pass's state); pri works on primitive
    variables (all elements converted there and back)."""
    U = np.asarray(U, np.float64)
    flag = (sensors(S, U) != 0)
    NE, NF, Ns = S.N_E, S.N_F, S.N_s
    fl = np.repeat(flag, NF * Ns)
    if S.limiter == "p0i":
        return np.where(fl, p0i_average(S, U), U)
    W = cons2prim(S, U) if S.limiter == "pri" else U.copy()
    a = S.a
    if S.D == 1:
        passes = [(0, a["Lag2Mono"], a["Mono2Lag"], Ns)]
    else:
        n1 = S.order + 1
        passes = [(0, a["Lag2MonoX"], a["MonoX2Lag"], n1), (2, a["Lag2MonoY"], a["MonoY2Lag"], n1)]
    fn = _m2i_pass if S.limiter == "m2i" else _hri_pass
    for off, L2M, M2L, n1 in passes:
        W = np.where(fl, fn(S, W, off, L2M, M2L, n1), W)
    return prim2cons(S, W) if S.limiter == "pri" else W


# ---------------------------------------------------------------------------------------------
# ERROR diagnostic of the reference driver (code/src/main.cc:909-1038)
# ---------------------------------------------------------------------------------------------

def error_norms(S: Setup, U: np.ndarray, Uex: np.ndarray, xyz0: tuple[float, float]) -> np.ndarray:
    """[dx, L1, L2, Linf per field] of the quadrature cell integrals / dx of U against Uex after
    both go to (rho, u, (E - rho u^2/2)/alpha, alpha) on fields 0..3, alpha = 1/(gamma-1) (the
    stored field divided by rho for GAMCONS, main.cc:963-966); xyz0 = x of nodes 0 and 1 of
    element 0 (dx = their difference, main.cc:992)."""
    NE, NF, Ns, NG = S.N_E, S.N_F, S.N_s, S.N_G

    def prim(X):
        V = np.array(X, np.float64, copy=True).reshape(NE, NF, Ns)
        V[:, 1] = V[:, 1] / V[:, 0]
        if S.gamcons:
            V[:, 3] = V[:, 3] / V[:, 0]
        V[:, 2] = 1.0 / V[:, 3] * (V[:, 2] - 0.5 * V[:, 0] * V[:, 1] * V[:, 1])
        return V

    phi = S.a["phi"].reshape(Ns, NG)  # phi[i*N_G + g] (column-major N_G x N_s)
    w = S.a["weight"].reshape(-1)[:NG]
    J = S.a["J"].reshape(NE)

    def avg(V):
        Ug = np.einsum("efi,ig->efg", V, phi)
        return np.einsum("efg,g->ef", Ug, w) * J[:, None]

    dx = xyz0[1] - xyz0[0]
    E = avg(prim(Uex)) / dx - avg(prim(U)) / dx
    return np.concatenate([[dx], np.abs(E).sum(0) / NE, np.sqrt((E * E).sum(0) / NE), np.abs(E).max(0)])
