// Gamma-model (GAMNCON) multifluid physics at one point, FP64.
//
// State per point: 1D (rho, rho u, E, alpha), 2D (rho, rho u, rho v, E, alpha) with
// alpha = 1/(gamma-1) carried non-conservatively (no flux; volume source -u.grad(alpha);
// interface term ncterm), then NY passive mass fractions rho*Y_k (conservative: flux rho*Y_k u,
// interface fluxes of the MACRO blocks that follow each flux function in the reference's
// face_fluxes headers).  GC selects the reference's GAMCONS model: the fifth field is
// rho/(gamma-1), carried conservatively (flux rho u/(gamma-1), no source, ncterm 0); the flux
// functions divide it by rho on entry as the reference does.  Formulas restate the reference's:
//   volume flux/source   evaluate_sf   code/src/physics/physics.cu:96-143 (1D), 248-301 (2D)
//   Rusanov              oned_multifluid_rusanov  code/src/face_fluxes/oned_multifluid_fluxes.h:30-94
//                        twod_multifluid_rusanov  code/src/face_fluxes/twod_multifluid_fluxes.h:30-97
//   HLL (1D)             oned_multifluid_hll      oned_multifluid_fluxes.h:117-226
//   Roe                  oned_multifluid_roe      oned_multifluid_fluxes.h:237-382
//                        twod_multifluid_roe      twod_multifluid_fluxes.h:151-342
//   wave speed           oned/twod_multifluid_upa code/src/physics/upa.h:61-85
// The operation order is kept where it is natural so the FP64 results agree with the
// reference CPU build to rounding (the GPU contracts a*b+c into FMA).
#pragma once

namespace dgb {
namespace phys {

enum { FLUX_RUS = 0, FLUX_HLL = 1, FLUX_ROE = 2 };

// ---------------------------------------------------------------- 1D -------------------------
// Interface flux F[4] and ncterm for the alpha equation (F[3] holds the alpha dissipation).
// Caller forms q_L = -F + nc (element on side L) and q_R = F + nc (physics.cu:800-804).
template <int FLUX, int NY = 0, bool GC = false>
__device__ __forceinline__ void riemann1d(double rhoL, double rhoR, double vxL, double vxR, double EtL, double EtR,
                                          double alphaL, double alphaR, double nx, double* F, double& nc,
                                          const double* YL = nullptr, const double* YR = nullptr) {
  // the reference's divisions as correctly rounded reciprocals (shorter dependency chains; within
  // an ulp or two of the quotients)
  const double irL = __drcp_rn(rhoL), irR = __drcp_rn(rhoR);
  if (GC) {
    alphaL = alphaL * irL;
    alphaR = alphaR * irR;
  }
  const double gm1L = __drcp_rn(alphaL), gm1R = __drcp_rn(alphaR);  // gamma - 1 = 1/alpha
  const double gammaL = 1.0 + gm1L;
  const double gammaR = 1.0 + gm1R;
  const double pL = gm1L * (EtL - 0.5 * rhoL * vxL * vxL);
  const double pR = gm1R * (EtR - 0.5 * rhoR * vxR * vxR);
  const double aL = sqrt(gammaL * pL * irL);
  const double aR = sqrt(gammaR * pR * irR);
  if (FLUX == FLUX_RUS) {
    const double maxvap = fmax(fabs(vxL) + aL, fabs(vxR) + aR);
    F[0] = 0.5 * ((rhoL * vxL + rhoR * vxR) * nx - maxvap * (rhoR - rhoL));
    F[1] = 0.5 * ((rhoL * vxL * vxL + pL + rhoR * vxR * vxR + pR) * nx - maxvap * (rhoR * vxR - rhoL * vxL));
    F[2] = 0.5 * (((EtL + pL) * vxL + (EtR + pR) * vxR) * nx - maxvap * (EtR - EtL));
    if (GC) {  // oned_multifluid_fluxes.h:79-81
      F[3] = 0.5 * ((rhoL * vxL * alphaL + rhoR * vxR * alphaR) * nx - maxvap * (rhoR * alphaR - rhoL * alphaL));
      nc = 0.0;
    } else {
      F[3] = 0.5 * (-maxvap * (alphaR - alphaL));
      nc = -0.5 * 0.5 * (vxL + vxR) * (alphaR - alphaL) * nx;
    }
    // the reference's mass-fraction line has its dissipation outside the 1/2 (fluxes.h:90-91)
#pragma unroll
    for (int k = 0; k < NY; ++k) F[4 + k] = 0.5 * (YL[k] * vxL + YR[k] * vxR) * nx - maxvap * (YR[k] - YL[k]);
  } else if (FLUX == FLUX_HLL) {
    // Davis wave-speed estimates (Toro 10.48); fhll of basic_fluxes.h:22-27.  The momentum
    // component passes the velocities as its state jump, and no branch is taken when SL == 0,
    // both exactly as oned_multifluid_hll does.
    const double SL = fmin(vxL * nx - aL, vxR * nx - aR);
    const double SR = fmax(vxL * nx + aL, vxR * nx + aR);
    const double vnc = -0.5 * (vxL * nx + vxR * nx) * (alphaL - alphaR);
    const double vncabs = -0.5 * fabs(vxL * nx + vxR * nx) * (alphaL - alphaR);
    const double iw = __drcp_rn(fabs(SR - SL));
    auto fhll = [iw](double UL, double SLv, double FL, double UR, double SRv, double FR) {
      return (SRv * FL - SLv * FR + SLv * SRv * (UR - UL)) * iw;
    };
    F[0] = F[1] = F[2] = F[3] = 0.0;
#pragma unroll
    for (int k = 0; k < NY; ++k) F[4 + k] = 0.0;
    if (SL > 0) {
      F[0] = rhoL * vxL * nx;
      F[1] = (rhoL * vxL * vxL + pL) * nx;
      F[2] = (EtL + pL) * vxL * nx;
      F[3] = GC ? rhoL * vxL * alphaL * nx : -0.5 * vncabs;
#pragma unroll
      for (int k = 0; k < NY; ++k) F[4 + k] = YL[k] * vxL * nx;
    } else if ((SL < 0) && (SR > 0)) {
      F[0] = fhll(rhoL, SL, rhoL * vxL * nx, rhoR, SR, rhoR * vxR * nx);
      F[1] = fhll(vxL, SL, (rhoL * vxL * vxL + pL) * nx, vxR, SR, (rhoR * vxR * vxR + pR) * nx);
      F[2] = fhll(EtL, SL, (EtL + pL) * vxL * nx, EtR, SR, (EtR + pR) * vxR * nx);
      // GAMCONS: the jump term takes the divided alpha, as oned_multifluid_fluxes.h:196 does
      F[3] = GC ? fhll(alphaL, SL, rhoL * vxL * alphaL * nx, alphaR, SR, rhoR * vxR * alphaR * nx)
                : fhll(alphaL, SL, 0, alphaR, SR, 0) - 0.5 * fabs(SR + SL) * iw * vncabs;
#pragma unroll
      for (int k = 0; k < NY; ++k) F[4 + k] = fhll(YL[k], SL, YL[k] * vxL * nx, YR[k], SR, YR[k] * vxR * nx);
    } else if (SR < 0) {
      F[0] = rhoR * vxR * nx;
      F[1] = (rhoR * vxR * vxR + pR) * nx;
      F[2] = (EtR + pR) * vxR * nx;
      F[3] = GC ? rhoR * vxR * alphaR * nx : 0.5 * vncabs;
#pragma unroll
      for (int k = 0; k < NY; ++k) F[4 + k] = YR[k] * vxR * nx;
    }
    nc = GC ? 0.0 : -0.5 * vnc;
  } else {
    const double RT = sqrt(rhoR * irL);
    const double rho = RT * rhoL;
    const double i1 = __drcp_rn(1 + RT);
    const double v = (vxL + RT * vxR) * i1;
    const double HL = (EtL + pL) * irL;
    const double HR = (EtR + pR) * irR;
    const double H = (HL + RT * HR) * i1;
    const double alpha = (alphaL + RT * alphaR) * i1;
    const double gm1 = __drcp_rn(alpha);  // gamma - 1
    const double a = sqrt(gm1 * (H - 0.5 * v * v));
    const double iL = pL * alphaL;
    const double iR = pR * alphaR;
    const double sL = sqrt(rhoL), sR = sqrt(rhoR);
    const double i = (sL * iL + sR * iR) * __drcp_rn(sL + sR);
    const double Dp = gm1 * gm1 * (alpha * (iR - iL) - i * (alphaR - alphaL));
    const double p = gm1 * i;
    const double ia2 = __drcp_rn(a * a);
    const double dV0 = (Dp - rho * a * (vxR - vxL)) * (0.5 * ia2);
    const double dV1 = (rhoR - rhoL) - Dp * ia2;
    const double dV2 = (Dp + rho * a * (vxR - vxL)) * (0.5 * ia2);
    const double dV3 = alphaR - alphaL;
    const double ws0 = fabs(v - a), ws1 = fabs(v), ws2 = fabs(v + a), ws3 = fabs(v);
    // right eigenvectors R0=(1, v-a, H-va, 0), R1=(1, v, v^2/2, 0), R2=(1, v+a, H+va, 0), R3=(0,0,p,1)
    F[0] = 0.5 * (rhoL * vxL + rhoR * vxR) * nx - 0.5 * (ws0 * dV0 * 1 + ws1 * dV1 * 1 + ws2 * dV2 * 1 + ws3 * dV3 * 0);
    F[1] = 0.5 * (rhoL * vxL * vxL + pL + rhoR * vxR * vxR + pR) * nx -
           0.5 * (ws0 * dV0 * (v - a) + ws1 * dV1 * v + ws2 * dV2 * (v + a) + ws3 * dV3 * 0);
    F[2] = 0.5 * ((EtL + pL) * vxL + (EtR + pR) * vxR) * nx -
           0.5 * (ws0 * dV0 * (H - v * a) + ws1 * dV1 * (0.5 * v * v) + ws2 * dV2 * (H + v * a) + ws3 * dV3 * p);
    F[3] = (GC ? 0.5 * (rhoL * vxL * alphaL + rhoR * vxR * alphaR) * nx : 0) +
           -0.5 * (ws0 * dV0 * 0 + ws1 * dV1 * 0 + ws2 * dV2 * 0 + ws3 * dV3 * 1);
    nc = GC ? 0.0 : -0.5 * v * (alphaR - alphaL) * nx;
    // mass fractions: Roe-averaged Y and its wave strength (oned_multifluid_fluxes.h:358-370)
#pragma unroll
    for (int k = 0; k < NY; ++k) {
      const double Y = (YL[k] * irL + RT * YR[k] * irR) * i1;
      const double dVY = YR[k] - YL[k] - (dV0 + dV1 + dV2) * Y;
      F[4 + k] = 0.5 * (YL[k] * vxL + YR[k] * vxR) * nx - 0.5 * (ws0 * dV0 * Y + ws1 * dV1 * Y + ws1 * dVY * 1 + ws2 * dV2 * Y);
    }
  }
}

// ---------------------------------------------------------------- 2D -------------------------
template <int FLUX, int NY = 0, bool GC = false>
__device__ __forceinline__ void riemann2d(double rhoL, double rhoR, double vxL, double vxR, double vyL, double vyR,
                                          double EtL, double EtR, double alphaL, double alphaR, double nx, double ny,
                                          double* F, double& nc, const double* YL = nullptr,
                                          const double* YR = nullptr) {
  if (GC) {
    // twod_multifluid_rusanov runs alphaL = alphaL/rhoL; alphaR = alphaL/rhoL (fluxes.h:50-53),
    // so its right alpha is the left one divided twice by rhoL; the Roe solver divides each by
    // its own density (:175-178)
    const double aLd = alphaL / rhoL;
    alphaR = FLUX == FLUX_ROE ? alphaR / rhoR : aLd / rhoL;
    alphaL = aLd;
  }
  const double vnL = vxL * nx + vyL * ny;
  const double vnR = vxR * nx + vyR * ny;
  const double gammaL = 1.0 + 1.0 / alphaL;
  const double gammaR = 1.0 + 1.0 / alphaR;
  const double pL = (gammaL - 1) * (EtL - 0.5 * rhoL * (vxL * vxL + vyL * vyL));
  const double pR = (gammaR - 1) * (EtR - 0.5 * rhoR * (vxR * vxR + vyR * vyR));
  const double aL = sqrt((gammaL * pL) / rhoL);
  const double aR = sqrt((gammaR * pR) / rhoR);
  const double HL = (EtL + pL) / rhoL;
  const double HR = (EtR + pR) / rhoR;
  if (FLUX == FLUX_ROE) {
    const double tx = -ny, ty = nx;
    const double vtL = vxL * tx + vyL * ty;
    const double vtR = vxR * tx + vyR * ty;
    const double iL = pL * alphaL;
    const double iR = pR * alphaR;
    const double RT = sqrt(rhoR / rhoL);
    const double rho = RT * rhoL;
    const double vx = (vxL + RT * vxR) / (1 + RT);
    const double vy = (vyL + RT * vyR) / (1 + RT);
    const double vn = vx * nx + vy * ny;
    const double vt = vx * tx + vy * ty;
    const double H = (HL + RT * HR) / (1 + RT);
    const double alpha = (alphaL + RT * alphaR) / (1 + RT);
    const double gamma = 1 + 1.0 / alpha;
    const double a = sqrt((gamma - 1) * (H - 0.5 * (vx * vx + vy * vy)));
    const double i = (iL + RT * iR) / (1 + RT);
    const double p = (gamma - 1) * i;
    const double drho = rhoR - rhoL;
    const double dp = (gamma - 1) * (gamma - 1) * (alpha * (iR - iL) - i * (alphaR - alphaL));
    const double dvn = vnR - vnL;
    const double dvt = vtR - vtL;
    const double dV0 = (dp - rho * a * dvn) / (2 * a * a);
    const double dV1 = rho * dvt / a;
    const double dV2 = drho - dp / (a * a);
    const double dV3 = (dp + rho * a * dvn) / (2 * a * a);
    const double dV4 = alphaR - alphaL;
    const double ws0 = fabs(vn - a), ws1 = fabs(vn), ws2 = fabs(vn), ws3 = fabs(vn + a), ws4 = fabs(vn);
    F[0] = 0.5 * (rhoL * vnL + rhoR * vnR) - 0.5 * (ws0 * dV0 * 1 + ws1 * dV1 * 0 + ws2 * dV2 * 1 + ws3 * dV3 * 1 + ws4 * dV4 * 0);
    F[1] = 0.5 * ((rhoL * vnL * vxL + pL * nx) + (rhoR * vnR * vxR + pR * nx)) -
           0.5 * (ws0 * dV0 * (vx - a * nx) + ws1 * dV1 * (a * tx) + ws2 * dV2 * vx + ws3 * dV3 * (vx + a * nx) + ws4 * dV4 * 0);
    F[2] = 0.5 * ((rhoL * vnL * vyL + pL * ny) + (rhoR * vnR * vyR + pR * ny)) -
           0.5 * (ws0 * dV0 * (vy - a * ny) + ws1 * dV1 * (a * ty) + ws2 * dV2 * vy + ws3 * dV3 * (vy + a * ny) + ws4 * dV4 * 0);
    F[3] = 0.5 * (rhoL * vnL * HL + rhoR * vnR * HR) -
           0.5 * (ws0 * dV0 * (H - vn * a) + ws1 * dV1 * (vt * a) + ws2 * dV2 * (0.5 * (vx * vx + vy * vy)) +
                  ws3 * dV3 * (H + vn * a) + ws4 * dV4 * p);
    F[4] = (GC ? 0.5 * (rhoL * vnL * alphaL + rhoR * vnR * alphaR) : 0) +
           -0.5 * (ws0 * dV0 * 0 + ws1 * dV1 * 0 + ws2 * dV2 * 0 + ws3 * dV3 * 0 + ws4 * dV4 * 1);
    nc = GC ? 0.0 : -0.5 * vn * (alphaR - alphaL);
    // mass fractions (twod_multifluid_fluxes.h:307-319)
#pragma unroll
    for (int k = 0; k < NY; ++k) {
      const double Y = (YL[k] / rhoL + RT * YR[k] / rhoR) / (1 + RT);
      const double dVY = YR[k] - YL[k] - (dV0 + dV2 + dV3) * Y;
      F[5 + k] = 0.5 * (YL[k] * vnL + YR[k] * vnR) - 0.5 * (ws0 * dV0 * Y + ws2 * dV2 * Y + ws1 * dVY * 1 + ws3 * dV3 * Y);
    }
  } else {
    // Rusanov (2D HLL is a stub in the reference, twod_multifluid_fluxes.h:119-141; the host
    // rejects it before any launch)
    const double maxvap = fmax(fabs(vnL) + aL, fabs(vnR) + aR);
    F[0] = 0.5 * (rhoL * vnL + rhoR * vnR - maxvap * (rhoR - rhoL));
    F[1] = 0.5 * ((rhoL * vnL * vxL + pL * nx) + (rhoR * vnR * vxR + pR * nx) - maxvap * (rhoR * vxR - rhoL * vxL));
    F[2] = 0.5 * ((rhoL * vnL * vyL + pL * ny) + (rhoR * vnR * vyR + pR * ny) - maxvap * (rhoR * vyR - rhoL * vyL));
    F[3] = 0.5 * (rhoL * vnL * HL + rhoR * vnR * HR - maxvap * (EtR - EtL));
    if (GC) {  // twod_multifluid_fluxes.h:82-84
      F[4] = 0.5 * (rhoL * vnL * alphaL + rhoR * vnR * alphaR - maxvap * (rhoR * alphaR - rhoL * alphaL));
      nc = 0.0;
    } else {
      F[4] = 0.5 * (-maxvap * (alphaR - alphaL));
      nc = -0.5 * 0.5 * (vnL + vnR) * (alphaR - alphaL);
    }
    // the reference's mass-fraction line has its dissipation outside the 1/2 (fluxes.h:91-94)
#pragma unroll
    for (int k = 0; k < NY; ++k) F[5 + k] = 0.5 * (YL[k] * vnL + YR[k] * vnR) - maxvap * (YR[k] - YL[k]);
  }
}

// max(|u|+a, |v|+a) at a node (upa.h:61-85)
template <bool GC = false>
__device__ __forceinline__ double wave_speed1d(double rho, double rhou, double E, double alpha) {
  // upa.h:61-70 with correctly rounded reciprocals in place of its divisions
  const double ir = __drcp_rn(rho);
  if (GC) alpha = alpha * ir;  // upa.h:65-67
  const double u = rhou * ir;
  const double gm1 = __drcp_rn(alpha);
  const double p = gm1 * (E - 0.5 * rho * u * u);
  return fabs(u) + sqrt((1.0 + gm1) * p * ir);
}
// oned_multifluid_upa (upa.h:61-70) as the reference writes it (the launcher shim's LfindUPA)
__device__ __forceinline__ double wave_speed1d_quotients(double rho, double rhou, double E, double alpha) {
  const double u = rhou / rho;
  const double gamma = 1.0 + 1.0 / alpha;
  const double p = (gamma - 1) * (E - 0.5 * rho * u * u);
  return fabs(u) + sqrt(gamma * p / rho);
}
// twod_multifluid_upa (upa.h:72-85) as the reference writes it, with its divisions (the launcher
// shim's LfindUPA)
__device__ __forceinline__ double wave_speed2d_quotients(double rho, double rhou, double rhov, double E,
                                                         double alpha) {
  const double u = rhou / rho, v = rhov / rho;
  const double gamma = 1.0 + 1.0 / alpha;
  const double p = (gamma - 1) * (E - 0.5 * rho * (u * u + v * v));
  const double a = sqrt(gamma * p / rho);
  return fmax(fabs(u) + a, fabs(v) + a);
}

template <bool GC = false>
__device__ __forceinline__ double wave_speed2d(double rho, double rhou, double rhov, double E, double alpha) {
  // upa.h:72-85 with correctly rounded reciprocals in place of the four divisions (within an ulp
  // or two of the quotient form; the reduction reads every node of the state each step)
  const double ir = __drcp_rn(rho);
  if (GC) alpha = alpha * ir;  // upa.h:78-80
  const double u = rhou * ir, v = rhov * ir;
  const double gm1 = __drcp_rn(alpha);
  const double p = gm1 * (E - 0.5 * rho * (u * u + v * v));
  const double a = sqrt((1.0 + gm1) * p * ir);
  return fmax(fabs(u), fabs(v)) + a;
}

}  // namespace phys
}  // namespace dgb

namespace dgb {
namespace phys {

// The same 2D interface fluxes evaluated with one reciprocal per state instead of repeated
// divisions (x/rho -> x * (1/rho), gamma-1 = 1/alpha).  Agrees with riemann2d to a few ulp,
// far inside the 1e-12 parity bound; used by the tiled kernel.
template <int FLUX, int NY = 0, bool GC = false>
__device__ __forceinline__ void riemann2d_rcp(const double* L, const double* R, double nx, double ny, double* F,
                                              double& nc) {
  const double rhoL = L[0], rhoR = R[0];
  const double irL = __drcp_rn(rhoL), irR = __drcp_rn(rhoR);
  const double vxL = L[1] * irL, vyL = L[2] * irL, vxR = R[1] * irR, vyR = R[2] * irR;
  const double EtL = L[3], EtR = R[3];
  // GAMCONS: divided by rho on entry; the Rusanov solver's right alpha is the left one divided
  // twice by rhoL (see riemann2d)
  const double alphaL = GC ? L[4] * irL : L[4];
  const double alphaR = GC ? (FLUX == FLUX_ROE ? R[4] * irR : alphaL * irL) : R[4];
  const double gm1L = __drcp_rn(alphaL), gm1R = __drcp_rn(alphaR);
  const double vnL = vxL * nx + vyL * ny;
  const double vnR = vxR * nx + vyR * ny;
  const double pL = gm1L * (EtL - 0.5 * rhoL * (vxL * vxL + vyL * vyL));
  const double pR = gm1R * (EtR - 0.5 * rhoR * (vxR * vxR + vyR * vyR));
  const double aL = sqrt((1.0 + gm1L) * pL * irL);
  const double aR = sqrt((1.0 + gm1R) * pR * irR);
  const double HL = (EtL + pL) * irL;
  const double HR = (EtR + pR) * irR;
  if (FLUX == FLUX_ROE) {
    const double tx = -ny, ty = nx;
    const double vtL = vxL * tx + vyL * ty;
    const double vtR = vxR * tx + vyR * ty;
    const double iL = pL * alphaL, iR = pR * alphaR;
    const double RT = sqrt(rhoR * irL);
    const double rho = RT * rhoL;
    const double i1 = __drcp_rn(1 + RT);
    const double vx = (vxL + RT * vxR) * i1;
    const double vy = (vyL + RT * vyR) * i1;
    const double vn = vx * nx + vy * ny;
    const double vt = vx * tx + vy * ty;
    const double H = (HL + RT * HR) * i1;
    const double alpha = (alphaL + RT * alphaR) * i1;
    const double gm1 = __drcp_rn(alpha);
    const double a = sqrt(gm1 * (H - 0.5 * (vx * vx + vy * vy)));
    const double ia = __drcp_rn(a);
    const double i = (iL + RT * iR) * i1;
    const double p = gm1 * i;
    const double drho = rhoR - rhoL;
    const double dp = gm1 * gm1 * (alpha * (iR - iL) - i * (alphaR - alphaL));
    const double dvn = vnR - vnL, dvt = vtR - vtL;
    const double h2a = 0.5 * ia * ia;
    const double dV0 = (dp - rho * a * dvn) * h2a;
    const double dV1 = rho * dvt * ia;
    const double dV2 = drho - dp * (ia * ia);
    const double dV3 = (dp + rho * a * dvn) * h2a;
    const double dV4 = alphaR - alphaL;
    const double ws0 = fabs(vn - a), ws1 = fabs(vn), ws3 = fabs(vn + a);
    const double w0 = ws0 * dV0, w1 = ws1 * dV1, w2 = ws1 * dV2, w3 = ws3 * dV3, w4 = ws1 * dV4;
    F[0] = 0.5 * (rhoL * vnL + rhoR * vnR) - 0.5 * (w0 + w2 + w3);
    F[1] = 0.5 * ((rhoL * vnL * vxL + pL * nx) + (rhoR * vnR * vxR + pR * nx)) -
           0.5 * (w0 * (vx - a * nx) + w1 * (a * tx) + w2 * vx + w3 * (vx + a * nx));
    F[2] = 0.5 * ((rhoL * vnL * vyL + pL * ny) + (rhoR * vnR * vyR + pR * ny)) -
           0.5 * (w0 * (vy - a * ny) + w1 * (a * ty) + w2 * vy + w3 * (vy + a * ny));
    F[3] = 0.5 * (rhoL * vnL * HL + rhoR * vnR * HR) -
           0.5 * (w0 * (H - vn * a) + w1 * (vt * a) + w2 * (0.5 * (vx * vx + vy * vy)) + w3 * (H + vn * a) + w4 * p);
    F[4] = GC ? 0.5 * (rhoL * vnL * alphaL + rhoR * vnR * alphaR) + -0.5 * w4 : -0.5 * w4;
    nc = GC ? 0.0 : -0.5 * vn * (alphaR - alphaL);
#pragma unroll
    for (int k = 0; k < NY; ++k) {
      const double Y = (L[5 + k] * irL + RT * R[5 + k] * irR) * i1;
      const double dVY = R[5 + k] - L[5 + k] - (dV0 + dV2 + dV3) * Y;
      F[5 + k] = 0.5 * (L[5 + k] * vnL + R[5 + k] * vnR) - 0.5 * (w0 * Y + w2 * Y + ws1 * dVY * 1 + w3 * Y);
    }
  } else {
    const double maxvap = fmax(fabs(vnL) + aL, fabs(vnR) + aR);
    F[0] = 0.5 * (rhoL * vnL + rhoR * vnR - maxvap * (rhoR - rhoL));
    F[1] = 0.5 * ((rhoL * vnL * vxL + pL * nx) + (rhoR * vnR * vxR + pR * nx) - maxvap * (R[1] - L[1]));
    F[2] = 0.5 * ((rhoL * vnL * vyL + pL * ny) + (rhoR * vnR * vyR + pR * ny) - maxvap * (R[2] - L[2]));
    F[3] = 0.5 * (rhoL * vnL * HL + rhoR * vnR * HR - maxvap * (EtR - EtL));
    if (GC) {
      F[4] = 0.5 * (rhoL * vnL * alphaL + rhoR * vnR * alphaR - maxvap * (rhoR * alphaR - rhoL * alphaL));
      nc = 0.0;
    } else {
      F[4] = 0.5 * (-maxvap * (alphaR - alphaL));
      nc = -0.5 * 0.5 * (vnL + vnR) * (alphaR - alphaL);
    }
#pragma unroll
    for (int k = 0; k < NY; ++k) F[5 + k] = 0.5 * (L[5 + k] * vnL + R[5 + k] * vnR) - maxvap * (R[5 + k] - L[5 + k]);
  }
}

}  // namespace phys
}  // namespace dgb
