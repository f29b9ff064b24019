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

// Paired FP32 arithmetic (sm_100 FFMA2 / FMUL2: two independent, correctly rounded FP32 operations
// per instruction).  The mixed kernel keeps fields (0, 1) and (2, 3) of its contractions in float2
// pairs (field 4 alone) and multiplies each pair by a broadcast basis coefficient.
__device__ __forceinline__ float2 bcast2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 dev2(double u0, double u1, double a0, double a1) {
  return make_float2((float)(u0 - a0), (float)(u1 - a1));
}

template <int P, int FLUX, int MODE, int TW, int TH>
__global__ void __launch_bounds__(TW * TH, 3)
    residual2d_tile_mixed_kernel(const TileArgs a, const __grid_constant__ CUtensorMap mapU,
                                 const __grid_constant__ CUtensorMap mapB) {
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

  pdl_wait();
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
      // the stage base (SSP) / accumulator (RK4) the epilogue reads, on its way to L2 meanwhile
      if ((MODE == MODE_SSP && a.a != 0.0) || (MODE == MODE_RK4 && a.Uacc))
        tma_prefetch_3d(&mapB, tx0, ty0, 0);
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
    // traces: anchor (face node 0) + FP32 contraction of the deviations, left and right paired
    double L[NF], R[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      float2 s = make_float2(0.f, 0.f);
#pragma unroll
      for (int j = 1; j < N1; ++j)
        s = fma2(bcast2(DGB_TAB2F(P, Bf[g][j])), dev2(vl[f][j], vr[f][j], vl[f][0], vr[f][0]), s);
      L[f] = vl[f][0] + (double)s.x;
      R[f] = vr[f][0] + (double)s.y;
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
  // accumulators: fields (0, 1) and (2, 3) as float2 pairs, field 4 alone
  const int tx = tid % TW, ty = tid / TW;
  const int e = (ty0 + ty) * nx + tx0 + tx;
  constexpr int NG1 = Tab2<P>::NG1;
  float2 r01[NS], r23[NS];
  float r4[NS];
#pragma unroll
  for (int t = 0; t < NS; ++t) { r01[t] = r23[t] = make_float2(0.f, 0.f); r4[t] = 0.f; }
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
      const float2 c01 = make_float2(s * fp[0] * w, s * fp[1] * w), c23 = make_float2(s * fp[2] * w, s * fp[3] * w);
      const float c4 = (s * fp[4] + fp[5]) * w;
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        const int t = kf == 0 ? N1 * j : kf == 1 ? P + N1 * j : kf == 2 ? j : j + N1 * P;
        const float b = DGB_TAB2F(P, Bf[g][j]);
        r01[t] = fma2(bcast2(b), c01, r01[t]);
        r23[t] = fma2(bcast2(b), c23, r23[t]);
        r4[t] = fmaf(b, c4, r4[t]);
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
    float2 T01[N1], T23[N1];
    float T4[N1], dT[N1];
#pragma unroll
    for (int iy = 0; iy < N1; ++iy) {
      float2 s01 = make_float2(0.f, 0.f), s23 = make_float2(0.f, 0.f);
      float s4 = 0.f, sd = 0.f;
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) {
        const int t = ix + N1 * iy;
        const float2 b = bcast2(DGB_TAB2F(P, B1[gx][ix]));
        s01 = fma2(b, dev2(us[(0 * NS + t) * NT], us[(1 * NS + t) * NT], anc[0], anc[1]), s01);
        s23 = fma2(b, dev2(us[(2 * NS + t) * NT], us[(3 * NS + t) * NT], anc[2], anc[3]), s23);
        const float d4 = (float)(us[(4 * NS + t) * NT] - anc[4]);
        s4 = fmaf(b.x, d4, s4);
        sd = fmaf(DGB_TAB2F(P, D1[gx][ix]), d4, sd);
      }
      T01[iy] = s01;
      T23[iy] = s23;
      T4[iy] = s4;
      dT[iy] = sd;
    }
    float2 Ax01[N1], Ax23[N1], Ay01[N1], Ay23[N1];
    float As[N1];
#pragma unroll
    for (int iy = 0; iy < N1; ++iy) {
      As[iy] = 0.f;
      Ax01[iy] = Ax23[iy] = Ay01[iy] = Ay23[iy] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int gy = 0; gy < NG1; ++gy) {
      const int g = gx * NG1 + gy;
      float2 u01 = make_float2(0.f, 0.f), u23 = make_float2(0.f, 0.f);
      float u4 = 0.f;
      float2 dd = make_float2(0.f, 0.f);  // (d alpha / dx, d alpha / dy) on the reference element
#pragma unroll
      for (int iy = 0; iy < N1; ++iy) {
        const float b = DGB_TAB2F(P, B1[gy][iy]);
        u01 = fma2(bcast2(b), T01[iy], u01);
        u23 = fma2(bcast2(b), T23[iy], u23);
        u4 = fmaf(b, T4[iy], u4);
        dd = fma2(make_float2(b, DGB_TAB2F(P, D1[gy][iy])), make_float2(dT[iy], T4[iy]), dd);
      }
      double ug[NF] = {anc[0] + (double)u01.x, anc[1] + (double)u01.y, anc[2] + (double)u23.x,
                       anc[3] + (double)u23.y, anc[4] + (double)u4};
      const float dax = dd.x, day = dd.y;
      const double irho = __drcp_rn(ug[0]);
      const double pd = __drcp_rn(ug[4]) * (ug[3] - 0.5 * (ug[1] * ug[1] + ug[2] * ug[2]) * irho);
      const float uu = (float)(ug[1] * irho), vv = (float)(ug[2] * irho), Et = (float)ug[3], p = (float)pd;
      const float wq = DGB_TAB2F(P, W[g]);
      const float wx = wq * cx, wy = wq * cy;
      const float mx = (float)ug[1] * wx, my = (float)ug[2] * wy;
      const float2 gx01 = make_float2(mx, mx * uu + wx * p), gx23 = make_float2(mx * vv, wx * ((Et + p) * uu));
      const float2 gy01 = make_float2(my, my * uu), gy23 = make_float2(my * vv + wy * p, wy * ((Et + p) * vv));
      const float gs = (wq * cJ) * (-uu * dax * sx - vv * day * sy);
#pragma unroll
      for (int iy = 0; iy < N1; ++iy) {
        const float2 b = bcast2(DGB_TAB2F(P, B1[gy][iy])), d = bcast2(DGB_TAB2F(P, D1[gy][iy]));
        Ax01[iy] = fma2(b, gx01, Ax01[iy]);
        Ax23[iy] = fma2(b, gx23, Ax23[iy]);
        Ay01[iy] = fma2(d, gy01, Ay01[iy]);
        Ay23[iy] = fma2(d, gy23, Ay23[iy]);
        As[iy] = fmaf(b.x, gs, As[iy]);
      }
    }
    // dPx = l'_ix(x_gx) l_iy(x_gy), dPy = l_ix(x_gx) l'_iy(x_gy), Phi = l_ix(x_gx) l_iy(x_gy)
#pragma unroll
    for (int iy = 0; iy < N1; ++iy)
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) {
        const float2 dx = bcast2(DGB_TAB2F(P, D1[gx][ix])), bx = bcast2(DGB_TAB2F(P, B1[gx][ix]));
        const int t = ix + N1 * iy;
        r01[t] = fma2(bx, Ay01[iy], fma2(dx, Ax01[iy], r01[t]));
        r23[t] = fma2(bx, Ay23[iy], fma2(dx, Ax23[iy], r23[t]));
        r4[t] = fmaf(bx.x, As[iy], r4[t]);
      }
  }
  pdl_trigger();
  if (MODE == MODE_RESIDUAL) {
#pragma unroll
    for (int t = 0; t < NS; ++t) {
      a.out[(size_t)(0 * NS + t) * ld + e] = (double)r01[t].x;
      a.out[(size_t)(1 * NS + t) * ld + e] = (double)r01[t].y;
      a.out[(size_t)(2 * NS + t) * ld + e] = (double)r23[t].x;
      a.out[(size_t)(3 * NS + t) * ld + e] = (double)r23[t].y;
      a.out[(size_t)(4 * NS + t) * ld + e] = (double)r4[t];
    }
    return;
  }
  const double dt = a.dt_override > 0 ? a.dt_override : a.scal->dt;
  const float sc = (float)(dt * a.invJ);
  // DU = dt/J (M1^-1 (x) M1^-1) R, first along x then along y, on the pairs and on field 4
  float2 m01[NS], m23[NS];
  float m4[NS];
#pragma unroll
  for (int iy = 0; iy < N1; ++iy)
#pragma unroll
    for (int ix = 0; ix < N1; ++ix) {
      float2 s01 = make_float2(0.f, 0.f), s23 = make_float2(0.f, 0.f);
      float s4 = 0.f;
#pragma unroll
      for (int q = 0; q < N1; ++q) {
        const float m = DGB_TAB2F(P, M1i[ix][q]);
        s01 = fma2(bcast2(m), r01[q + N1 * iy], s01);
        s23 = fma2(bcast2(m), r23[q + N1 * iy], s23);
        s4 = fmaf(m, r4[q + N1 * iy], s4);
      }
      m01[ix + N1 * iy] = s01;
      m23[ix + N1 * iy] = s23;
      m4[ix + N1 * iy] = s4;
    }
#pragma unroll
  for (int iy = 0; iy < N1; ++iy)
#pragma unroll
    for (int ix = 0; ix < N1; ++ix) {
      float2 s01 = make_float2(0.f, 0.f), s23 = make_float2(0.f, 0.f);
      float s4 = 0.f;
#pragma unroll
      for (int q = 0; q < N1; ++q) {
        const float m = DGB_TAB2F(P, M1i[iy][q]);
        s01 = fma2(bcast2(m), m01[ix + N1 * q], s01);
        s23 = fma2(bcast2(m), m23[ix + N1 * q], s23);
        s4 = fmaf(m, m4[ix + N1 * q], s4);
      }
      const int t = ix + N1 * iy;
      const double du[NF] = {(double)(sc * s01.x), (double)(sc * s01.y), (double)(sc * s23.x), (double)(sc * s23.y),
                             (double)(sc * s4)};
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const size_t gi = (size_t)(f * NS + t) * ld + e;
        if (MODE == MODE_SSP) {
          const double base = a.a != 0.0 ? a.a * __ldg(a.Ubase + gi) : 0.0;
          a.out[gi] = base + a.b * (us[(f * NS + t) * NT] + du[f]);
        } else {
          a.out[gi] = du[f];
          if (a.Uacc) a.Uacc[gi] = a.Uacc[gi] + a.b * du[f];
        }
      }
    }
}

}  // namespace dgb

namespace dgb {

// ---------------------------------------------------------------------------------------------
// Compressed-tile variant of the mixed kernel.  The shared tile holds, per element, the FP64
// anchors (node-0 values of the five fields) and the FP32 deviations of the other nodes from them
// -- 200 instead of 360 bytes per element at p = 2, 344 instead of 640 at p = 3 -- written by each
// thread for its own element from plain coalesced loads.  Collocation then reads its FP32 operands
// straight from shared memory (no FP64 subtraction and conversion per quadrature column), the CTA
// needs less shared memory, and the stage update re-reads the FP64 stage input through L2.
// The face traces are formed from the same anchors and deviations: the FP64 value of the face's
// first node plus an FP32 contraction of the other nodes' deviations from it, as in the TMA-tile
// kernel.
template <int P, int TW, int TH>
struct TileDimsMixedCT {
  static constexpr int N1 = P + 1, NS = N1 * N1, NF = 5, NT = TW * TH;
  static constexpr int NXF = (TW + 1) * TH * N1, NYF = TW * (TH + 1) * N1, NCODE = 2 * TH + 2 * TW;
  static constexpr size_t head_bytes = 128;
  static constexpr size_t code_bytes = (NCODE * 4 + 127) / 128 * 128;
  static constexpr size_t off_anc = head_bytes + code_bytes;              // double [NF][NT]
  static constexpr size_t off_d01 = off_anc + (size_t)NF * NT * 8;        // float2 [NS-1][NT]: fields 0, 1
  static constexpr size_t off_d23 = off_d01 + (size_t)(NS - 1) * NT * 8;  // float2 [NS-1][NT]: fields 2, 3
  static constexpr size_t off_d4 = off_d23 + (size_t)(NS - 1) * NT * 8;   // float  [NS-1][NT]: field 4
  static constexpr size_t off_halo = off_d4 + ((size_t)(NS - 1) * NT * 4 + 15) / 16 * 16;
  static constexpr size_t halo_doubles = (size_t)2 * TH * NF * N1 + (size_t)2 * TW * NF * N1;
  static constexpr size_t off_face = off_halo + halo_doubles * 8;
  static constexpr size_t smem_bytes = off_face + (size_t)6 * (NXF + NYF) * sizeof(float);
};

// FP32 deviation of node t of field f from the field's anchor, element i of the tile (t = 0: zero)
template <int NT>
__device__ __forceinline__ float ct_dev(const float2* d01, const float2* d23, const float* d4, int f, int t, int i) {
  if (t == 0) return 0.f;
  const int r = (t - 1) * NT + i;
  return f == 0 ? d01[r].x : f == 1 ? d01[r].y : f == 2 ? d23[r].x : f == 3 ? d23[r].y : d4[r];
}

// p = 3 (32 x 2 tiles, 64 threads): 48 KB of shared memory instead of 66 KB, four CTAs per SM
// instead of three, measured 11.3 -> 10.3 ms per step at 2048 x 1024.  p = 2: four 128-thread CTAs
// would cap the kernel at 128 registers (260 bytes of spills; measured slower), three run no faster
// than the TMA-tile kernel, which stays the default there.
template <int P>
constexpr int mixed_ct_min_blocks() { return P == 3 ? 4 : 3; }

template <int P, int FLUX, int MODE, int TW, int TH>
__global__ void __launch_bounds__(TW * TH, mixed_ct_min_blocks<P>())
    residual2d_tile_mixed_ct_kernel(const TileArgs a) {
  using Dm = TileDimsMixedCT<P, TW, TH>;
  constexpr int N1 = Dm::N1, NS = Dm::NS, NF = 5, NT = Dm::NT, NXF = Dm::NXF, NYF = Dm::NYF;
  extern __shared__ __align__(128) unsigned char smraw[];
  int* codes = reinterpret_cast<int*>(smraw + Dm::head_bytes);
  double* Anc = reinterpret_cast<double*>(smraw + Dm::off_anc);
  float2* D01 = reinterpret_cast<float2*>(smraw + Dm::off_d01);
  float2* D23 = reinterpret_cast<float2*>(smraw + Dm::off_d23);
  float* D4 = reinterpret_cast<float*>(smraw + Dm::off_d4);
  double* HL = reinterpret_cast<double*>(smraw + Dm::off_halo);
  double* HR = HL + TH * NF * N1;
  double* HD = HR + TH * NF * N1;
  double* HU = HD + TW * NF * N1;
  float* Fs = reinterpret_cast<float*>(smraw + Dm::off_face);  // [NXF + NYF][6]

  pdl_wait();
  if (a.scal && a.scal->flags) return;
  const int tid = threadIdx.x;
  const int tx0 = blockIdx.x * TW, ty0 = blockIdx.y * TH;
  const int ld = a.ld, nx = a.nx;
  const int tx = tid % TW, ty = tid / TW;
  const int e = (ty0 + ty) * nx + tx0 + tx;

  // ---------------- phase 0: own element compressed, neighbour strips by plain loads ----------------
  for (int k = tid; k < Dm::NCODE; k += NT) {
    int face, eo;
    if (k < TH) { face = 0; eo = (ty0 + k) * nx + tx0; }
    else if (k < 2 * TH) { face = 1; eo = (ty0 + k - TH) * nx + tx0 + TW - 1; }
    else if (k < 2 * TH + TW) { face = 2; eo = ty0 * nx + tx0 + (k - 2 * TH); }
    else { face = 3; eo = (ty0 + TH - 1) * nx + tx0 + (k - 2 * TH - TW); }
    codes[k] = __ldg(a.nbr + (size_t)face * ld + eo);
  }
  {
    const double* ue = a.U + e;
#pragma unroll
    for (int pr = 0; pr < 2; ++pr) {
      double u0[NS], u1[NS];
#pragma unroll
      for (int t = 0; t < NS; ++t) {
        u0[t] = __ldg(ue + (size_t)((2 * pr) * NS + t) * ld);
        u1[t] = __ldg(ue + (size_t)((2 * pr + 1) * NS + t) * ld);
      }
      Anc[(2 * pr) * NT + tid] = u0[0];
      Anc[(2 * pr + 1) * NT + tid] = u1[0];
      float2* Dp = pr == 0 ? D01 : D23;
#pragma unroll
      for (int t = 1; t < NS; ++t) Dp[(t - 1) * NT + tid] = dev2(u0[t], u1[t], u0[0], u1[0]);
    }
    double u4[NS];
#pragma unroll
    for (int t = 0; t < NS; ++t) u4[t] = __ldg(ue + (size_t)(4 * NS + t) * ld);
    Anc[4 * NT + tid] = u4[0];
#pragma unroll
    for (int t = 1; t < NS; ++t) D4[(t - 1) * NT + tid] = (float)(u4[t] - u4[0]);
  }
  // the stage base (SSP) / accumulator (RK4) the epilogue reads, on its way to L2 meanwhile: the
  // tile's rows of every (field, node) plane, 128-byte lines spread over the threads
  const double* pb = MODE == MODE_SSP && a.a != 0.0 ? a.Ubase : MODE == MODE_RK4 ? a.Uacc : nullptr;
  if (pb) {
    constexpr int LPR = TW * 8 / 128;  // lines per tile row of one plane
    for (int k = tid; k < NF * NS * TH * LPR; k += NT) {
      const int q = k / (TH * LPR), r = (k / LPR) % TH, l = k % LPR;
      const double* p = pb + (size_t)q * ld + (size_t)(ty0 + r) * nx + tx0 + l * 16;
      asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
    }
  }
  __syncthreads();  // codes
  for (int k = tid; k < 2 * TH * NF * N1; k += NT) {
    const int side = k / (TH * NF * N1);
    const int r = k % (TH * NF * N1);
    const int ry = r / (NF * N1), f = (r / N1) % NF, j = r % N1;
    const int nb = codes[side * TH + ry];
    double v = 0.0;
    if (nb >= 0) v = __ldg(a.U + (size_t)(f * NS + (side == 0 ? P + N1 * j : N1 * j)) * ld + nb);
    (side == 0 ? HL : HR)[r] = v;
  }
  for (int k = tid; k < 2 * TW * NF * N1; k += NT) {
    const int side = k / (TW * NF * N1);
    const int r = k % (TW * NF * N1);
    const int rx = r / (NF * N1), f = (r / N1) % NF, j = r % N1;
    const int nb = codes[2 * TH + side * TW + rx];
    double v = 0.0;
    if (nb >= 0) v = __ldg(a.U + (size_t)(f * NS + (side == 0 ? j + N1 * P : j)) * ld + nb);
    (side == 0 ? HD : HU)[r] = v;
  }
  __syncthreads();

  // ---------------- phase 1: face fluxes, each face of the tile once ----------------
  for (int k = tid; k < NXF + NYF; k += NT) {
    // each side: FP64 value of face node 0 and FP32 deviations of face nodes 1..P from it
    double bl[NF], br[NF];
    float dl[NF][N1], dr[NF][N1];
    float nxv, nyv, sgn = 1.0f;
    int code = 0, mom, g;
    bool first_edge;
    // in-tile element i, face nodes t_j = t0 + j * st
    auto side_tile = [&](int i, int t0, int st, double* b, float (*d)[N1]) {
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const float d0 = ct_dev<NT>(D01, D23, D4, f, t0, i);
        b[f] = Anc[f * NT + i] + (double)d0;
#pragma unroll
        for (int j = 1; j < N1; ++j) d[f][j] = ct_dev<NT>(D01, D23, D4, f, t0 + j * st, i) - d0;
      }
    };
    auto side_halo = [&](const double* H, double* b, float (*d)[N1]) {
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        b[f] = H[f * N1];
#pragma unroll
        for (int j = 1; j < N1; ++j) d[f][j] = (float)(H[f * N1 + j] - H[f * N1]);
      }
    };
    if (k < NXF) {
      g = k % N1;
      const int fy = (k / N1) % TH, fx = k / (N1 * TH);
      if (fx == 0) code = codes[fy];
      if (fx == TW) code = codes[TH + fy];
      if (fx > 0) side_tile(fy * TW + fx - 1, P, N1, bl, dl);
      else side_halo(HL + fy * NF * N1, bl, dl);
      if (fx < TW) side_tile(fy * TW + fx, 0, N1, br, dr);
      else side_halo(HR + fy * NF * N1, br, dr);
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
      if (fy > 0) side_tile((fy - 1) * TW + fx, N1 * P, 1, bl, dl);
      else side_halo(HD + fx * NF * N1, bl, dl);
      if (fy < TH) side_tile(fy * TW + fx, 0, 1, br, dr);
      else side_halo(HU + fx * NF * N1, br, dr);
      nxv = 0.0f;
      nyv = 1.0f;
      first_edge = fy == 0;
      mom = 2;
    }
    if (code < 0) {
      // domain boundary: the inside element's state on both sides, the wall-normal momentum
      // mirrored on reflective walls
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const double ob = first_edge ? br[f] : bl[f];
        const float sg = (code == -3 && f == mom) ? -1.f : 1.f;
        bl[f] = ob;
        br[f] = sg * ob;
#pragma unroll
        for (int j = 1; j < N1; ++j) {
          const float od = first_edge ? dr[f][j] : dl[f][j];
          dl[f][j] = od;
          dr[f][j] = sg * od;
        }
      }
      if (first_edge) { nxv = -nxv; nyv = -nyv; sgn = -1.0f; }
    }
    double L[NF], R[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      float2 s = make_float2(0.f, 0.f);
#pragma unroll
      for (int j = 1; j < N1; ++j) s = fma2(bcast2(DGB_TAB2F(P, Bf[g][j])), make_float2(dl[f][j], dr[f][j]), s);
      L[f] = bl[f] + (double)s.x;
      R[f] = br[f] + (double)s.y;
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
  constexpr int NG1 = Tab2<P>::NG1;
  float2 r01[NS], r23[NS];
  float r4[NS];
#pragma unroll
  for (int t = 0; t < NS; ++t) { r01[t] = r23[t] = make_float2(0.f, 0.f); r4[t] = 0.f; }
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
      const float2 c01 = make_float2(s * fp[0] * w, s * fp[1] * w), c23 = make_float2(s * fp[2] * w, s * fp[3] * w);
      const float c4 = (s * fp[4] + fp[5]) * w;
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        const int t = kf == 0 ? N1 * j : kf == 1 ? P + N1 * j : kf == 2 ? j : j + N1 * P;
        const float b = DGB_TAB2F(P, Bf[g][j]);
        r01[t] = fma2(bcast2(b), c01, r01[t]);
        r23[t] = fma2(bcast2(b), c23, r23[t]);
        r4[t] = fmaf(b, c4, r4[t]);
      }
    }
  }

  double anc[NF];
#pragma unroll
  for (int f = 0; f < NF; ++f) anc[f] = Anc[f * NT + tid];
  const float2* d01 = D01 + tid;
  const float2* d23 = D23 + tid;
  const float* d4 = D4 + tid;
  const float cx = (float)a.cx, cy = (float)a.cy, cJ = (float)a.J, sx = (float)a.sx, sy = (float)a.sy;
#pragma unroll 1
  for (int gx = 0; gx < NG1; ++gx) {
    float2 T01[N1], T23[N1];
    float T4[N1], dT[N1];
#pragma unroll
    for (int iy = 0; iy < N1; ++iy) {
      float2 s01 = make_float2(0.f, 0.f), s23 = make_float2(0.f, 0.f);
      float s4 = 0.f, sd = 0.f;
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) {
        const int t = ix + N1 * iy;
        if (t == 0) continue;  // the anchor's deviation is zero
        const float2 b = bcast2(DGB_TAB2F(P, B1[gx][ix]));
        s01 = fma2(b, d01[(t - 1) * NT], s01);
        s23 = fma2(b, d23[(t - 1) * NT], s23);
        const float v4 = d4[(t - 1) * NT];
        s4 = fmaf(b.x, v4, s4);
        sd = fmaf(DGB_TAB2F(P, D1[gx][ix]), v4, sd);
      }
      T01[iy] = s01;
      T23[iy] = s23;
      T4[iy] = s4;
      dT[iy] = sd;
    }
    float2 Ax01[N1], Ax23[N1], Ay01[N1], Ay23[N1];
    float As[N1];
#pragma unroll
    for (int iy = 0; iy < N1; ++iy) {
      As[iy] = 0.f;
      Ax01[iy] = Ax23[iy] = Ay01[iy] = Ay23[iy] = make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int gy = 0; gy < NG1; ++gy) {
      const int g = gx * NG1 + gy;
      float2 u01 = make_float2(0.f, 0.f), u23 = make_float2(0.f, 0.f);
      float u4 = 0.f;
      float2 dd = make_float2(0.f, 0.f);  // (d alpha / dx, d alpha / dy) on the reference element
#pragma unroll
      for (int iy = 0; iy < N1; ++iy) {
        const float b = DGB_TAB2F(P, B1[gy][iy]);
        u01 = fma2(bcast2(b), T01[iy], u01);
        u23 = fma2(bcast2(b), T23[iy], u23);
        u4 = fmaf(b, T4[iy], u4);
        dd = fma2(make_float2(b, DGB_TAB2F(P, D1[gy][iy])), make_float2(dT[iy], T4[iy]), dd);
      }
      double ug[NF] = {anc[0] + (double)u01.x, anc[1] + (double)u01.y, anc[2] + (double)u23.x,
                       anc[3] + (double)u23.y, anc[4] + (double)u4};
      const float dax = dd.x, day = dd.y;
      const double irho = __drcp_rn(ug[0]);
      const double pd = __drcp_rn(ug[4]) * (ug[3] - 0.5 * (ug[1] * ug[1] + ug[2] * ug[2]) * irho);
      const float uu = (float)(ug[1] * irho), vv = (float)(ug[2] * irho), Et = (float)ug[3], p = (float)pd;
      const float wq = DGB_TAB2F(P, W[g]);
      const float wx = wq * cx, wy = wq * cy;
      const float mx = (float)ug[1] * wx, my = (float)ug[2] * wy;
      const float2 gx01 = make_float2(mx, mx * uu + wx * p), gx23 = make_float2(mx * vv, wx * ((Et + p) * uu));
      const float2 gy01 = make_float2(my, my * uu), gy23 = make_float2(my * vv + wy * p, wy * ((Et + p) * vv));
      const float gs = (wq * cJ) * (-uu * dax * sx - vv * day * sy);
#pragma unroll
      for (int iy = 0; iy < N1; ++iy) {
        const float2 b = bcast2(DGB_TAB2F(P, B1[gy][iy])), d = bcast2(DGB_TAB2F(P, D1[gy][iy]));
        Ax01[iy] = fma2(b, gx01, Ax01[iy]);
        Ax23[iy] = fma2(b, gx23, Ax23[iy]);
        Ay01[iy] = fma2(d, gy01, Ay01[iy]);
        Ay23[iy] = fma2(d, gy23, Ay23[iy]);
        As[iy] = fmaf(b.x, gs, As[iy]);
      }
    }
#pragma unroll
    for (int iy = 0; iy < N1; ++iy)
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) {
        const float2 dx = bcast2(DGB_TAB2F(P, D1[gx][ix])), bx = bcast2(DGB_TAB2F(P, B1[gx][ix]));
        const int t = ix + N1 * iy;
        r01[t] = fma2(bx, Ay01[iy], fma2(dx, Ax01[iy], r01[t]));
        r23[t] = fma2(bx, Ay23[iy], fma2(dx, Ax23[iy], r23[t]));
        r4[t] = fmaf(bx.x, As[iy], r4[t]);
      }
  }
  pdl_trigger();
  if (MODE == MODE_RESIDUAL) {
#pragma unroll
    for (int t = 0; t < NS; ++t) {
      a.out[(size_t)(0 * NS + t) * ld + e] = (double)r01[t].x;
      a.out[(size_t)(1 * NS + t) * ld + e] = (double)r01[t].y;
      a.out[(size_t)(2 * NS + t) * ld + e] = (double)r23[t].x;
      a.out[(size_t)(3 * NS + t) * ld + e] = (double)r23[t].y;
      a.out[(size_t)(4 * NS + t) * ld + e] = (double)r4[t];
    }
    return;
  }
  const double dt = a.dt_override > 0 ? a.dt_override : a.scal->dt;
  const float sc = (float)(dt * a.invJ);
  float2 m01[NS], m23[NS];
  float m4[NS];
#pragma unroll
  for (int iy = 0; iy < N1; ++iy)
#pragma unroll
    for (int ix = 0; ix < N1; ++ix) {
      float2 s01 = make_float2(0.f, 0.f), s23 = make_float2(0.f, 0.f);
      float s4 = 0.f;
#pragma unroll
      for (int q = 0; q < N1; ++q) {
        const float m = DGB_TAB2F(P, M1i[ix][q]);
        s01 = fma2(bcast2(m), r01[q + N1 * iy], s01);
        s23 = fma2(bcast2(m), r23[q + N1 * iy], s23);
        s4 = fmaf(m, r4[q + N1 * iy], s4);
      }
      m01[ix + N1 * iy] = s01;
      m23[ix + N1 * iy] = s23;
      m4[ix + N1 * iy] = s4;
    }
#pragma unroll
  for (int iy = 0; iy < N1; ++iy)
#pragma unroll
    for (int ix = 0; ix < N1; ++ix) {
      float2 s01 = make_float2(0.f, 0.f), s23 = make_float2(0.f, 0.f);
      float s4 = 0.f;
#pragma unroll
      for (int q = 0; q < N1; ++q) {
        const float m = DGB_TAB2F(P, M1i[iy][q]);
        s01 = fma2(bcast2(m), m01[ix + N1 * q], s01);
        s23 = fma2(bcast2(m), m23[ix + N1 * q], s23);
        s4 = fmaf(m, m4[ix + N1 * q], s4);
      }
      const int t = ix + N1 * iy;
      const double du[NF] = {(double)(sc * s01.x), (double)(sc * s01.y), (double)(sc * s23.x), (double)(sc * s23.y),
                             (double)(sc * s4)};
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const size_t gi = (size_t)(f * NS + t) * ld + e;
        if (MODE == MODE_SSP) {
          const double base = a.a != 0.0 ? a.a * __ldg(a.Ubase + gi) : 0.0;
          a.out[gi] = base + a.b * (__ldg(a.U + gi) + du[f]);
        } else {
          a.out[gi] = du[f];
          if (a.Uacc) a.Uacc[gi] = a.Uacc[gi] + a.b * du[f];
        }
      }
    }
}

}  // namespace dgb
