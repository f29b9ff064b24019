// Mixed-precision tiled 2D residual + stage update (the "mixed" form of residual2d_tile_kernel).
//
// Same tiling, face-once scheme and assembly as residual2d_tile_kernel; the arithmetic is split:
//   FP64  the state (HBM and the shared tile), per-element anchors, the values at quadrature and
//         face points (anchor + FP32 deviation), pressure recovery p = (gamma-1)(E - rho|u|^2/2)
//         from those values, the Roe solver (FLUX_ROE stays FP64 end to end), the stage update
//   FP32  the basis contractions (collocation, face traces, lift, tensor-factored M^-1), the
//         Rusanov flux and the volume flux products, all accumulated in FP32.
// Collocation is done on deviations from an anchor value of the element (its node 0): since the
// Lagrange basis sums to one (and its derivatives to zero), u(x_g) = u_0 + sum_t phi_t(x_g)
// (u_t - u_0) exactly, and the FP32 rounding only scales with the variation inside the element,
// not with the value itself.  Shared memory is ~75 KB for p = 2 (FP32 face buffer, no stage-base
// prefetch), so three 128-thread CTAs share an SM.
#pragma once
#include "tile2d.cuh"

namespace dgb {

template <int P>
struct Tab2f {
  static constexpr int N1 = P + 1, NG1 = (P == 1) ? 2 : P + 2, NS = N1 * N1, NG = NG1 * NG1;
  float dPx[NG][NS], dPy[NG][NS], Phi[NG][NS], W[NG];
  float Bf[N1][N1], wf[N1], M1i[N1][N1], B1[NG1][N1], D1[NG1][N1];
};

static __constant__ Tab2f<1> c_tab2f_p1;
static __constant__ Tab2f<2> c_tab2f_p2;
static __constant__ Tab2f<3> c_tab2f_p3;
#define DGB_TAB2F(P, member) ((P) == 1 ? c_tab2f_p1.member : (P) == 2 ? c_tab2f_p2.member : c_tab2f_p3.member)

template <int P, int TW, int TH>
struct TileDimsMixed {
  using B = TileDims<P, TW, TH>;
  static constexpr int NXF = B::NXF, NYF = B::NYF;
  static constexpr size_t off_tile = B::off_tile, off_halo = B::off_halo, off_face = B::off_face;
  static constexpr size_t smem_bytes = off_face + (size_t)6 * (NXF + NYF) * sizeof(float);
};

// Rusanov flux with FP64 pressure recovery and FP32 flux arithmetic (gamma model, GAMNCON);
// same formulas as twod_multifluid_rusanov (code/src/face_fluxes/twod_multifluid_fluxes.h:30-97)
__device__ __forceinline__ void rusanov2d_mixed(const double* L, const double* R, float nx, float ny, float F[5],
                                                float& nc) {
  const double irL = __drcp_rn(L[0]), irR = __drcp_rn(R[0]);
  const double gm1L = __drcp_rn(L[4]), gm1R = __drcp_rn(R[4]);
  const double pLd = gm1L * (L[3] - 0.5 * (L[1] * L[1] + L[2] * L[2]) * irL);
  const double pRd = gm1R * (R[3] - 0.5 * (R[1] * R[1] + R[2] * R[2]) * irR);
  const float rhoL = (float)L[0], rhoR = (float)R[0];
  const float vxL = (float)(L[1] * irL), vyL = (float)(L[2] * irL), vxR = (float)(R[1] * irR), vyR = (float)(R[2] * irR);
  const float EtL = (float)L[3], EtR = (float)R[3], pL = (float)pLd, pR = (float)pRd;
  const float vnL = vxL * nx + vyL * ny, vnR = vxR * nx + vyR * ny;
  const float aL = sqrtf((1.0f + (float)gm1L) * pL * (float)irL);
  const float aR = sqrtf((1.0f + (float)gm1R) * pR * (float)irR);
  const float HL = (EtL + pL) * (float)irL, HR = (EtR + pR) * (float)irR;
  const float lam = fmaxf(fabsf(vnL) + aL, fabsf(vnR) + aR);
  F[0] = 0.5f * (rhoL * vnL + rhoR * vnR - lam * (rhoR - rhoL));
  F[1] = 0.5f * ((rhoL * vnL * vxL + pL * nx) + (rhoR * vnR * vxR + pR * nx) - lam * (float)(R[1] - L[1]));
  F[2] = 0.5f * ((rhoL * vnL * vyL + pL * ny) + (rhoR * vnR * vyR + pR * ny) - lam * (float)(R[2] - L[2]));
  F[3] = 0.5f * (rhoL * vnL * HL + rhoR * vnR * HR - lam * (float)(R[3] - L[3]));
  const float dal = (float)(R[4] - L[4]);
  F[4] = -0.5f * lam * dal;
  nc = -0.25f * (vnL + vnR) * dal;
}

template <int P, int FLUX, int MODE, int TW, int TH>
__global__ void __launch_bounds__(TW * TH, 3)
    residual2d_tile_mixed_kernel(const TileArgs a, const __grid_constant__ CUtensorMap mapU) {
  using Dm = TileDims<P, TW, TH>;
  constexpr int N1 = Dm::N1, NS = Dm::NS, NF = 5, NT = Dm::NT, NXF = Dm::NXF, NYF = Dm::NYF;
  extern __shared__ __align__(128) unsigned char smraw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smraw);
  int* s_ok = reinterpret_cast<int*>(smraw + 8);
  int* codes = reinterpret_cast<int*>(smraw + Dm::head_bytes);
  double* Us = reinterpret_cast<double*>(smraw + Dm::off_tile);
  double* HL = reinterpret_cast<double*>(smraw + Dm::off_halo);
  double* HR = HL + TH * NF * N1;
  double* HD = HR + TH * NF * N1;
  double* HU = HD + TW * NF * N1;
  float* Fs = reinterpret_cast<float*>(smraw + Dm::off_face);  // [NXF + NYF][6]

  if (a.scal && a.scal->flags) return;
  const int tid = threadIdx.x;
  const int tx0 = blockIdx.x * TW, ty0 = blockIdx.y * TH;
  const int ld = a.ld, nx = a.nx;

  // ---------------- phase 0: tile by TMA, neighbour strips by plain loads ----------------
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  for (int k = tid; k < Dm::NCODE; k += NT) {
    int face, eo;
    if (k < TH) { face = 0; eo = (ty0 + k) * nx + tx0; }
    else if (k < 2 * TH) { face = 1; eo = (ty0 + k - TH) * nx + tx0 + TW - 1; }
    else if (k < 2 * TH + TW) { face = 2; eo = ty0 * nx + tx0 + (k - 2 * TH); }
    else { face = 3; eo = (ty0 + TH - 1) * nx + tx0 + (k - 2 * TH - TW); }
    codes[k] = __ldg(a.nbr + (size_t)face * ld + eo);
  }
  __syncthreads();
  const bool tma_ok = (smem_u32(Us) & 127u) == 0 && ((tx0 * 8) & 15) == 0;
  if (tid == 0) {
    if (tma_ok) {
      mbar_arrive_expect_tx(bar, Dm::tile_bytes);
      tma_load_3d(Us, &mapU, tx0, ty0, 0, bar);
    } else {
      atomicOr(a.errflag, (unsigned)FLAG_TIMEOUT);
    }
  }
  for (int k = tid; k < 2 * TH * NF * N1; k += NT) {
    const int side = k / (TH * NF * N1);
    const int r = k % (TH * NF * N1);
    const int ty = r / (NF * N1), f = (r / N1) % NF, j = r % N1;
    const int nb = codes[side * TH + ty];
    double v = 0.0;
    if (nb >= 0) v = __ldg(a.U + (size_t)(f * NS + (side == 0 ? P + N1 * j : N1 * j)) * ld + nb);
    (side == 0 ? HL : HR)[r] = v;
  }
  for (int k = tid; k < 2 * TW * NF * N1; k += NT) {
    const int side = k / (TW * NF * N1);
    const int r = k % (TW * NF * N1);
    const int tx = r / (NF * N1), f = (r / N1) % NF, j = r % N1;
    const int nb = codes[2 * TH + side * TW + tx];
    double v = 0.0;
    if (nb >= 0) v = __ldg(a.U + (size_t)(f * NS + (side == 0 ? j + N1 * P : j)) * ld + nb);
    (side == 0 ? HD : HU)[r] = v;
  }
  if (tid == 0) {
    bool ok = tma_ok && mbar_wait(bar, 0, a.polls);
    if (tma_ok && !ok) {
      atomicOr(a.errflag, (unsigned)FLAG_TIMEOUT);
      mbar_wait(bar, 0);
    }
    *s_ok = ok ? 1 : 0;
  }
  __syncthreads();
  if (!*s_ok) return;

  // ---------------- phase 1: face fluxes, each face of the tile once ----------------
  for (int k = tid; k < NXF + NYF; k += NT) {
    double vl[NF][N1], vr[NF][N1];
    float nxv, nyv, sgn = 1.0f;
    int code = 0, mom, g;
    bool first_edge;
    if (k < NXF) {
      g = k % N1;
      const int fy = (k / N1) % TH, fx = k / (N1 * TH);
      if (fx == 0) code = codes[fy];
      if (fx == TW) code = codes[TH + fy];
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int j = 0; j < N1; ++j) {
          vl[f][j] = fx > 0 ? Us[(f * NS + P + N1 * j) * NT + fy * TW + fx - 1] : HL[(fy * NF + f) * N1 + j];
          vr[f][j] = fx < TW ? Us[(f * NS + N1 * j) * NT + fy * TW + fx] : HR[(fy * NF + f) * N1 + j];
        }
      nxv = 1.0f;
      nyv = 0.0f;
      first_edge = fx == 0;
      mom = 1;
    } else {
      const int kk = k - NXF;
      g = kk % N1;
      const int fx = (kk / N1) % TW, fy = kk / (N1 * TW);
      if (fy == 0) code = codes[2 * TH + fx];
      if (fy == TH) code = codes[2 * TH + TW + fx];
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int j = 0; j < N1; ++j) {
          vl[f][j] = fy > 0 ? Us[(f * NS + j + N1 * P) * NT + (fy - 1) * TW + fx] : HD[(fx * NF + f) * N1 + j];
          vr[f][j] = fy < TH ? Us[(f * NS + j) * NT + fy * TW + fx] : HU[(fx * NF + f) * N1 + j];
        }
      nxv = 0.0f;
      nyv = 1.0f;
      first_edge = fy == 0;
      mom = 2;
    }
    if (code < 0) {
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int j = 0; j < N1; ++j) {
          const double own = first_edge ? vr[f][j] : vl[f][j];
          vl[f][j] = own;
          vr[f][j] = (code == -3 && f == mom) ? -own : own;
        }
      if (first_edge) { nxv = -nxv; nyv = -nyv; sgn = -1.0f; }
    }
    // traces: anchor (face node 0) + FP32 contraction of the deviations
    double L[NF], R[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      float sl = 0.f, sr = 0.f;
#pragma unroll
      for (int j = 1; j < N1; ++j) {
        sl += DGB_TAB2F(P, Bf[g][j]) * (float)(vl[f][j] - vl[f][0]);
        sr += DGB_TAB2F(P, Bf[g][j]) * (float)(vr[f][j] - vr[f][0]);
      }
      L[f] = vl[f][0] + (double)sl;
      R[f] = vr[f][0] + (double)sr;
    }
    float F[NF], nc;
    if (FLUX == phys::FLUX_ROE) {
      double Fd[NF], ncd;
      phys::riemann2d_rcp<FLUX>(L, R, (double)nxv, (double)nyv, Fd, ncd);
#pragma unroll
      for (int f = 0; f < NF; ++f) F[f] = (float)Fd[f];
      nc = (float)ncd;
    } else {
      rusanov2d_mixed(L, R, nxv, nyv, F, nc);
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) Fs[k * 6 + f] = sgn * F[f];
    Fs[k * 6 + 5] = nc;
  }
  __syncthreads();

  // ---------------- phase 2: volume terms and assembly, one thread per element ----------------
  const int tx = tid % TW, ty = tid / TW;
  const int e = (ty0 + ty) * nx + tx0 + tx;
  constexpr int NG1 = Tab2<P>::NG1;
  float r[NF][NS];
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int t = 0; t < NS; ++t) r[f][t] = 0.f;
#pragma unroll
  for (int kf = 0; kf < 4; ++kf) {
    int base;
    float s, jw;
    if (kf == 0) { base = (tx * TH + ty) * N1; s = 1.f; jw = (float)a.JFx; }
    else if (kf == 1) { base = ((tx + 1) * TH + ty) * N1; s = -1.f; jw = (float)a.JFx; }
    else if (kf == 2) { base = NXF + (ty * TW + tx) * N1; s = 1.f; jw = (float)a.JFy; }
    else { base = NXF + ((ty + 1) * TW + tx) * N1; s = -1.f; jw = (float)a.JFy; }
#pragma unroll
    for (int g = 0; g < N1; ++g) {
      const float* fp = Fs + (base + g) * 6;
      const float w = jw * DGB_TAB2F(P, wf[g]);
      float c[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) c[f] = (s * fp[f] + (f == 4 ? fp[5] : 0.f)) * w;
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        const int t = kf == 0 ? N1 * j : kf == 1 ? P + N1 * j : kf == 2 ? j : j + N1 * P;
        const float b = DGB_TAB2F(P, Bf[g][j]);
#pragma unroll
        for (int f = 0; f < NF; ++f) r[f][t] += b * c[f];
      }
    }
  }

  // volume terms: anchors in FP64, deviations contracted in FP32 (x then y), pressure in FP64
  const double* us = Us + tid;
  double anc[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) anc[f] = us[(f * NS) * NT];
  const float cx = (float)a.cx, cy = (float)a.cy, cJ = (float)a.J, sx = (float)a.sx, sy = (float)a.sy;
#pragma unroll 1  // rolled quadrature-column loop (instruction cache), as in the FP64 kernel
  for (int gx = 0; gx < NG1; ++gx) {
    float Tc[NF][N1], dT[N1];
#pragma unroll
    for (int iy = 0; iy < N1; ++iy) {
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        float sacc = 0.f;
#pragma unroll
        for (int ix = 0; ix < N1; ++ix)
          sacc += DGB_TAB2F(P, B1[gx][ix]) * (float)(us[(f * NS + ix + N1 * iy) * NT] - anc[f]);
        Tc[f][iy] = sacc;
      }
      float sd = 0.f;
#pragma unroll
      for (int ix = 0; ix < N1; ++ix)
        sd += DGB_TAB2F(P, D1[gx][ix]) * (float)(us[(4 * NS + ix + N1 * iy) * NT] - anc[4]);
      dT[iy] = sd;
    }
    float Ax[4][N1], Ay[4][N1], As[N1];
#pragma unroll
    for (int iy = 0; iy < N1; ++iy) {
      As[iy] = 0.f;
#pragma unroll
      for (int f = 0; f < 4; ++f) Ax[f][iy] = Ay[f][iy] = 0.f;
    }
#pragma unroll
    for (int gy = 0; gy < NG1; ++gy) {
      const int g = gx * NG1 + gy;
      double ug[NF];
      float dax = 0.f, day = 0.f;
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        float sacc = 0.f;
#pragma unroll
        for (int iy = 0; iy < N1; ++iy) sacc += DGB_TAB2F(P, B1[gy][iy]) * Tc[f][iy];
        ug[f] = anc[f] + (double)sacc;
      }
#pragma unroll
      for (int iy = 0; iy < N1; ++iy) {
        dax += DGB_TAB2F(P, B1[gy][iy]) * dT[iy];
        day += DGB_TAB2F(P, D1[gy][iy]) * Tc[4][iy];
      }
      const double irho = __drcp_rn(ug[0]);
      const double pd = __drcp_rn(ug[4]) * (ug[3] - 0.5 * (ug[1] * ug[1] + ug[2] * ug[2]) * irho);
      const float uu = (float)(ug[1] * irho), vv = (float)(ug[2] * irho), Et = (float)ug[3], p = (float)pd;
      const float wq = DGB_TAB2F(P, W[g]);
      const float wx = wq * cx, wy = wq * cy;
      const float mx = (float)ug[1] * wx, my = (float)ug[2] * wy;
      const float gxv[4] = {mx, mx * uu + wx * p, mx * vv, wx * ((Et + p) * uu)};
      const float gyv[4] = {my, my * uu, my * vv + wy * p, wy * ((Et + p) * vv)};
      const float gs = (wq * cJ) * (-uu * dax * sx - vv * day * sy);
      if constexpr (kSfLift) {
#pragma unroll
        for (int iy = 0; iy < N1; ++iy) {
          const float b = DGB_TAB2F(P, B1[gy][iy]), d = DGB_TAB2F(P, D1[gy][iy]);
#pragma unroll
          for (int f = 0; f < 4; ++f) { Ax[f][iy] += b * gxv[f]; Ay[f][iy] += d * gyv[f]; }
          As[iy] += b * gs;
        }
      } else {
#pragma unroll
        for (int t = 0; t < NS; ++t) {
#pragma unroll
          for (int f = 0; f < 4; ++f) r[f][t] += DGB_TAB2F(P, dPx[g][t]) * gxv[f] + DGB_TAB2F(P, dPy[g][t]) * gyv[f];
          r[4][t] += DGB_TAB2F(P, Phi[g][t]) * gs;
        }
      }
    }
    if constexpr (kSfLift) {
#pragma unroll
      for (int iy = 0; iy < N1; ++iy)
#pragma unroll
        for (int ix = 0; ix < N1; ++ix) {
          const float dx = DGB_TAB2F(P, D1[gx][ix]), bx = DGB_TAB2F(P, B1[gx][ix]);
          const int t = ix + N1 * iy;
#pragma unroll
          for (int f = 0; f < 4; ++f) r[f][t] += dx * Ax[f][iy] + bx * Ay[f][iy];
          r[4][t] += bx * As[iy];
        }
    }
  }
  if (MODE == MODE_RESIDUAL) {
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int t = 0; t < NS; ++t) a.out[(size_t)(f * NS + t) * ld + e] = (double)r[f][t];
    return;
  }
  const double dt = a.dt_override > 0 ? a.dt_override : a.scal->dt;
  const float sc = (float)(dt * a.invJ);
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    float tmp[NS];
#pragma unroll
    for (int iy = 0; iy < N1; ++iy)
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) {
        float s = 0.f;
#pragma unroll
        for (int q = 0; q < N1; ++q) s += DGB_TAB2F(P, M1i[ix][q]) * r[f][q + N1 * iy];
        tmp[ix + N1 * iy] = s;
      }
#pragma unroll
    for (int iy = 0; iy < N1; ++iy)
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) {
        float s = 0.f;
#pragma unroll
        for (int q = 0; q < N1; ++q) s += DGB_TAB2F(P, M1i[iy][q]) * tmp[ix + N1 * q];
        const double du = (double)(sc * s);
        const int t = ix + N1 * iy;
        const size_t gi = (size_t)(f * NS + t) * ld + e;
        if (MODE == MODE_SSP) {
          const double base = a.a != 0.0 ? a.a * __ldg(a.Ubase + gi) : 0.0;
          a.out[gi] = base + a.b * (us[(f * NS + t) * NT] + du);
        } else {
          a.out[gi] = du;
          if (a.Uacc) a.Uacc[gi] = a.Uacc[gi] + a.b * du;
        }
      }
  }
}

}  // namespace dgb
