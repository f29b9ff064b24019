// sm_100a kernels of the DG residual / time-step path (FP64 plain form).
//
//   residual2d_kernel  fused  collocation -> volume flux/source -> lift  +  face traces ->
//                      Riemann flux -> face lift  +  inverse mass  +  RK stage update.
//                      Replaces the 13 launches of DG_SOLVER::dg_solver
//                      (code/src/dg/dg_solver.h:292-364) plus Lsolver and the BLAS axpy/copy
//                      of RK::RK_integration (code/src/time_integration/rk.cc:164-198).
//   residual1d_kernel  the same for 1D, one thread per element.
//   lim*_kernel        hierarchical-reconstruction limiters HR / m2 (code/src/limiting/limiting.cc:11-594)
//   wavespeed_kernel   max |u|+a for the CFL step (code/src/time_integration/rk.cc:250-272)
//
// Work decomposition of residual2d_kernel: one CTA owns TE consecutive elements and stages their
// nodal state (and the neighbours' face traces) in shared memory; threads then sweep
// (element, quadrature point), (element, field, node) and (element, face, face point) work items.
// Every face flux is computed by both owners with the same canonical orientation (left/bottom
// element as the "L" state, +x/+y normal), so the two copies are bit-identical and the scheme
// stays exactly conservative without atomics.
#pragma once
#include "common.cuh"
#include "physics.cuh"

namespace dgb {

// Modes of the residual kernels.
enum { MODE_RESIDUAL = 0,  // out = S + F + Q                         (dg_solver)
       MODE_SSP = 1,       // out = a*Ubase + b*(U + dt*Minv*(S+F+Q))  (SSP-RK stage)
       MODE_RK4 = 2 };     // out = dt*Minv*(S+F+Q); Uacc += b*out     (Lsolver + axpy)

struct StageArgs {
  const double* __restrict__ U;      // stage input (internal layout)
  const double* __restrict__ Ubase;  // SSP: U^n
  double* __restrict__ out;
  double* __restrict__ Uacc;         // RK4 accumulator (may be null)
  double* __restrict__ Unext;        // RK4 (1D): the next stage input Us + beta_next * DU, or null
  const double* __restrict__ Us;     //   its Us
  double beta_next;
  const int* __restrict__ elist;     // 2D generic residual: the elements to do (null: all of them)
  int nlist;
  const int* __restrict__ nbr;       // [face][ld] neighbours, boundary codes < 0
  const DevScalars* __restrict__ scal;
  double a, b;
  double dt_override;                // > 0: use this step instead of scal->dt
};

__device__ __forceinline__ void copy_consts(Consts& dst, const Consts& src) {
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(&src);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(&dst);
  for (int k = threadIdx.x; k < (int)(sizeof(Consts) / 8); k += blockDim.x) d[k] = s[k];
}

template <int P>
struct Dims2 {
  static constexpr int N1 = P + 1;
  static constexpr int NG1 = (P == 1) ? 2 : P + 2;
  static constexpr int NS = N1 * N1;
  static constexpr int NG = NG1 * NG1;
  static constexpr int NF = 5;
};
// NY mass fractions / the GAMCONS model: NF fields, NFL of them with a conservative volume flux,
// NGV volume slots per quadrature point (x and y flux of each, and the alpha source under GAMNCON)
template <int P, int NY, bool GC>
struct Dims2V : Dims2<P> {
  static constexpr int NF = 5 + NY;
  static constexpr int NFL = 4 + NY + (GC ? 1 : 0);
  static constexpr int NGV = 2 * NFL + (GC ? 0 : 1);
};

template <int P, int TE, int NY = 0, bool GC = false>
constexpr size_t residual2d_smem_doubles() {
  using Dm = Dims2V<P, NY, GC>;
  constexpr size_t g1 = (size_t)Dm::NGV * Dm::NG * TE;
  constexpr size_t g2 = (size_t)Dm::NF * 4 * Dm::N1 * TE;
  return (size_t)Dm::NF * Dm::NS * TE * 2 + (size_t)4 * Dm::NF * Dm::N1 * TE + (g1 > g2 ? g1 : g2) +
         (size_t)3 * Dm::NG * Dm::NS;
}

// node of face k (0 L, 1 R, 2 D, 3 U) at face position j, and the matching node of the
// neighbour across that face
template <int P>
__device__ __forceinline__ int face_node(int k, int j) {
  constexpr int N1 = P + 1;
  return k == 0 ? N1 * j : k == 1 ? P + N1 * j : k == 2 ? j : j + N1 * P;
}
template <int P>
__device__ __forceinline__ int across_node(int k, int j) {
  constexpr int N1 = P + 1;
  return k == 0 ? P + N1 * j : k == 1 ? N1 * j : k == 2 ? j + N1 * P : j;
}

template <int P, int FLUX, int MODE, int TE, int NT, int NY = 0, bool GC = false>
__global__ void __launch_bounds__(NT) residual2d_kernel(const Consts cin, const StageArgs a) {
  static_assert(!(GC && NY > 0), "GAMCONS with mass fractions is not built");
  using Dm = Dims2V<P, NY, GC>;
  constexpr int N1 = Dm::N1, NG1 = Dm::NG1, NS = Dm::NS, NG = Dm::NG, NF = Dm::NF, NFL = Dm::NFL, NGV = Dm::NGV;
  constexpr int GSZ = (NGV * NG * TE > NF * 4 * N1 * TE) ? NGV * NG * TE : NF * 4 * N1 * TE;
  __shared__ Consts c;
  extern __shared__ double sm[];
  double* Us = sm;                        // [NF][NS][TE]
  double* Uh = Us + NF * NS * TE;         // [4][NF][N1][TE]  neighbour traces
  double* Rs = Uh + 4 * NF * N1 * TE;     // [NF][NS][TE]     residual
  double* G = Rs + NF * NS * TE;          // volume: [9][NG][TE]; faces: [NF][4][N1][TE]
  double* Phi = G + GSZ;                  // [NG][NS]
  double* dPx = Phi + NG * NS;
  double* dPy = dPx + NG * NS;

  const int tid = threadIdx.x;
  copy_consts(c, cin);
  if (a.scal && a.scal->flags) return;  // a failed CFL step stops the integration here
  __syncthreads();
  const int ld = c.ld;
  const int e0 = blockIdx.x * TE;
  // the element of slot el: the grid's e0 + el, or the listed one (the strips the tiled kernel
  // leaves on a grid whose extents are not tile multiples); -1 past the end
  const int NL = a.elist ? a.nlist : c.n_elem;
  auto elem = [&](int el) -> int {
    const int k = e0 + el;
    return k < NL ? (a.elist ? __ldg(a.elist + k) : k) : -1;
  };
  for (int i = tid; i < NG * NS; i += NT) {
    const int g = i / NS, t = i % NS, gx = g / NG1, gy = g % NG1, ix = t % N1, iy = t / N1;
    Phi[i] = c.Bq[gx][ix] * c.Bq[gy][iy];
    dPx[i] = c.Dq[gx][ix] * c.Bq[gy][iy];
    dPy[i] = c.Bq[gx][ix] * c.Dq[gy][iy];
  }
  // ---- stage the tile's state and the neighbours' face traces ----
  for (int i = tid; i < NF * NS * TE; i += NT) {
    const int el = i % TE, ft = i / TE, e = elem(el);
    Us[i] = e >= 0 ? __ldg(a.U + (size_t)ft * ld + e) : 0.0;
  }
  for (int i = tid; i < 4 * NF * N1 * TE; i += NT) {
    const int el = i % TE;
    int r = i / TE;
    const int j = r % N1;
    r /= N1;
    const int f = r % NF, k = r / NF, e = elem(el);
    double v = 0.0;
    if (e >= 0) {
      const int nb = __ldg(a.nbr + (size_t)k * ld + e);
      if (nb >= 0) v = __ldg(a.U + (size_t)(f * NS + across_node<P>(k, j)) * ld + nb);
      else {
        v = __ldg(a.U + (size_t)(f * NS + face_node<P>(k, j)) * ld + e);
        // reflective wall: mirror the wall-normal momentum (rflctive, code/src/bc/boundaries.cu:20-67)
        if (nb == -3 && ((k < 2 && f == 1) || (k >= 2 && f == 2))) v = -v;
      }
    }
    Uh[i] = v;
  }
  __syncthreads();

  // ---- volume: states, fluxes and the alpha source at the quadrature points ----
  for (int i = tid; i < NG * TE; i += NT) {
    const int el = i % TE, g = i / TE;
    if (elem(el) < 0) continue;
    double ug[NF], dax = 0, day = 0;
#pragma unroll
    for (int f = 0; f < NF; ++f) ug[f] = 0.0;
#pragma unroll
    for (int t = 0; t < NS; ++t) {
      const double ph = Phi[g * NS + t];
#pragma unroll
      for (int f = 0; f < NF; ++f) ug[f] += ph * Us[(f * NS + t) * TE + el];
      const double al = Us[(4 * NS + t) * TE + el];
      dax += dPx[g * NS + t] * al;
      day += dPy[g * NS + t] * al;
    }
    if constexpr (NY > 0 || GC) {
      // the volume terms of the tiled kernel's point_terms: the conservative fluxes of the NFL
      // fields (mass fractions rho Y_k u, physics.cu:293-298; GAMCONS alpha flux rho u/(gamma-1),
      // physics.cu:253-281) and, under GAMNCON, the alpha source
      const double rho = ug[0], irho = __drcp_rn(rho);
      const double uu = ug[1] * irho, vv = ug[2] * irho, Et = ug[3];
      const double gm1 = GC ? rho * __drcp_rn(ug[4]) : __drcp_rn(ug[4]);
      const double p = gm1 * (Et - 0.5 * rho * (uu * uu + vv * vv));
      const double W = c.wq[g / NG1] * c.wq[g % NG1];
      const double wx = W * (c.J * c.ixx), wy = W * (c.J * c.iyy);
      const double mx = ug[1] * wx, my = ug[2] * wy;
      double gxv[NFL], gyv[NFL];
      gxv[0] = mx; gxv[1] = mx * uu + wx * p; gxv[2] = mx * vv; gxv[3] = wx * ((Et + p) * uu);
      gyv[0] = my; gyv[1] = my * uu; gyv[2] = my * vv + wy * p; gyv[3] = wy * ((Et + p) * vv);
#pragma unroll
      for (int k = 0; k < NY; ++k) { gxv[4 + k] = wx * (ug[5 + k] * uu); gyv[4 + k] = wy * (ug[5 + k] * vv); }
      if constexpr (GC) { gxv[4] = wx * (ug[4] * uu); gyv[4] = wy * (ug[4] * vv); }
#pragma unroll
      for (int q = 0; q < NFL; ++q) {
        G[(q * NG + g) * TE + el] = gxv[q];
        G[((NFL + q) * NG + g) * TE + el] = gyv[q];
      }
      if constexpr (!GC) G[(2 * NFL * NG + g) * TE + el] = (W * c.J) * (-uu * dax * c.ixx - vv * day * c.iyy);
      continue;
    }
    // physics.cu:248-257 with correctly rounded reciprocals in place of its divisions
    const double rho = ug[0], ir = __drcp_rn(rho), u = ug[1] * ir, v = ug[2] * ir, Et = ug[3];
    const double p = __drcp_rn(ug[4]) * (Et - 0.5 * rho * (u * u + v * v));
    const double W = c.wq[g / NG1] * c.wq[g % NG1];
    const double cx = W * (c.ixx * c.J), cy = W * (c.iyy * c.J);
    G[(0 * NG + g) * TE + el] = cx * (rho * u);
    G[(1 * NG + g) * TE + el] = cx * (rho * u * u + p);
    G[(2 * NG + g) * TE + el] = cx * (rho * u * v);
    G[(3 * NG + g) * TE + el] = cx * ((Et + p) * u);
    G[(4 * NG + g) * TE + el] = cy * (rho * v);
    G[(5 * NG + g) * TE + el] = cy * (rho * u * v);
    G[(6 * NG + g) * TE + el] = cy * (rho * v * v + p);
    G[(7 * NG + g) * TE + el] = cy * ((Et + p) * v);
    // GAMNCON source -u.grad(alpha) (physics.cu:282-291)
    const double s = -u * dax * c.ixx - v * day * c.iyy;
    G[(8 * NG + g) * TE + el] = (W * c.J) * s;
  }
  __syncthreads();
  // ---- volume lift: F = dphi_w^T fJ, S = phi_w^T sJ ----
  for (int i = tid; i < NF * NS * TE; i += NT) {
    const int el = i % TE, ft = i / TE, f = ft / NS, t = ft % NS;
    double r = 0.0;
    if constexpr (NY > 0 || GC) {
      // flux slot of field f: rho, rho u, rho v, E; alpha (GAMCONS) or rho Y_k after them
      const int q = f < 4 ? f : GC ? 4 : f - 1;
      if (f == 4 && !GC) {
#pragma unroll 4
        for (int g = 0; g < NG; ++g) r += Phi[g * NS + t] * G[(2 * NFL * NG + g) * TE + el];
      } else {
#pragma unroll 4
        for (int g = 0; g < NG; ++g)
          r += dPx[g * NS + t] * G[(q * NG + g) * TE + el] + dPy[g * NS + t] * G[((NFL + q) * NG + g) * TE + el];
      }
      Rs[i] = r;
      continue;
    }
    if (f < 4) {
#pragma unroll 4
      for (int g = 0; g < NG; ++g)
        r += dPx[g * NS + t] * G[(f * NG + g) * TE + el] + dPy[g * NS + t] * G[((4 + f) * NG + g) * TE + el];
    } else {
#pragma unroll 4
      for (int g = 0; g < NG; ++g) r += Phi[g * NS + t] * G[(8 * NG + g) * TE + el];
    }
    Rs[i] = r;
  }
  __syncthreads();
  // ---- faces: Riemann flux at the face quadrature points ----
  for (int i = tid; i < 4 * N1 * TE; i += NT) {
    const int el = i % TE, r = i / TE, g = r % N1, k = r / N1, e = elem(el);
    if (e < 0) continue;
    double uo[NF], un[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      double so = 0, sn = 0;
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        so += c.Bf[g][j] * Us[(f * NS + face_node<P>(k, j)) * TE + el];
        sn += c.Bf[g][j] * Uh[((k * NF + f) * N1 + j) * TE + el];
      }
      uo[f] = so;
      un[f] = sn;
    }
    const int nb = __ldg(a.nbr + (size_t)k * ld + e);
    const bool xface = k < 2;
    // interior faces use the canonical orientation (left/bottom element is L, normal +x/+y);
    // boundary faces take the element as L with its outward normal
    const bool swapLR = nb >= 0 && (k == 0 || k == 2);
    const double sgn = swapLR ? 1.0 : -1.0;
    double nx = xface ? 1.0 : 0.0, ny = xface ? 0.0 : 1.0;
    if (nb < 0 && k == 0) nx = -1.0;
    if (nb < 0 && k == 2) ny = -1.0;
    double L[NF], R[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) { L[f] = swapLR ? un[f] : uo[f]; R[f] = swapLR ? uo[f] : un[f]; }
    double F[NF], nc;
    phys::riemann2d_rcp<FLUX, NY, GC>(L, R, nx, ny, F, nc);  // the tiled kernel's flux (reciprocals for divisions)
    const double jw = (xface ? c.JFx : c.JFy) * c.wf[g];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      const double q = sgn * F[f] + (f == 4 ? nc : 0.0);
      G[((f * 4 + k) * N1 + g) * TE + el] = q * jw;
    }
  }
  __syncthreads();
  // ---- face lift and total ----
  for (int i = tid; i < NF * NS * TE; i += NT) {
    const int el = i % TE, ft = i / TE, f = ft / NS, t = ft % NS, e = elem(el);
    const int ix = t % N1, iy = t / N1;
    double r = Rs[i];
#pragma unroll
    for (int g = 0; g < N1; ++g) {
      if (ix == 0) r += c.Bf[g][iy] * G[((f * 4 + 0) * N1 + g) * TE + el];
      if (ix == P) r += c.Bf[g][iy] * G[((f * 4 + 1) * N1 + g) * TE + el];
      if (iy == 0) r += c.Bf[g][ix] * G[((f * 4 + 2) * N1 + g) * TE + el];
      if (iy == P) r += c.Bf[g][ix] * G[((f * 4 + 3) * N1 + g) * TE + el];
    }
    if (MODE == MODE_RESIDUAL) {
      if (e >= 0) a.out[(size_t)ft * ld + e] = r;
    } else {
      Rs[i] = r;
    }
  }
  if (MODE == MODE_RESIDUAL) return;
  __syncthreads();
  // ---- epilogue: DU = dt Minv R and the stage update ----
  const double dt = a.dt_override > 0 ? a.dt_override : a.scal->dt;
  for (int i = tid; i < NF * NS * TE; i += NT) {
    const int el = i % TE, ft = i / TE, f = ft / NS, t = ft % NS, e = elem(el);
    if (e < 0) continue;
    double s = 0.0;
#pragma unroll
    for (int tt = 0; tt < NS; ++tt) s += c.Minv[t][tt] * Rs[(f * NS + tt) * TE + el];
    const double du = dt * s;
    const size_t gi = (size_t)ft * ld + e;
    if (MODE == MODE_SSP) {
      const double base = a.a != 0.0 ? a.a * __ldg(a.Ubase + gi) : 0.0;
      a.out[gi] = base + a.b * (Us[i] + du);
    } else {
      a.out[gi] = du;
      if (a.Uacc) a.Uacc[gi] += a.b * du;
    }
  }
}

// ------------------------------------------------------------------------------------------
// 1D: one thread per element, everything in registers
// ------------------------------------------------------------------------------------------
// element e (< c.n_elem) with the problem constants c (in shared memory) and dt; NY passive mass
// fractions follow the four gamma-model fields
// GC: the GAMCONS model (fields rho, rho u, E, rho/(gamma-1)): conservative alpha flux, no source
// The residual r = S + F + Q of element e (its nodal state in u, read from a.U)
template <int P, int FLUX, int NY = 0, bool GC = false>
__device__ __forceinline__ void res1d_residual(const Consts& c, const StageArgs& a, int e, double (&u)[4 + NY][P + 1],
                                               double (&r)[4 + NY][P + 1]) {
  constexpr int N1 = P + 1, NG = P + 1, NF = 4 + NY;
  const int ld = c.ld;
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int t = 0; t < N1; ++t) { u[f][t] = __ldg(a.U + (size_t)(f * N1 + t) * ld + e); r[f][t] = 0.0; }
  // volume
#pragma unroll
  for (int g = 0; g < NG; ++g) {
    double ug[NF], da = 0;
#pragma unroll
    for (int f = 0; f < NF; ++f) ug[f] = 0.0;
#pragma unroll
    for (int t = 0; t < N1; ++t) {
#pragma unroll
      for (int f = 0; f < NF; ++f) ug[f] += c.Bq[g][t] * u[f][t];
      da += c.Dq[g][t] * u[3][t];
    }
    // physics.cu:96-104 with correctly rounded reciprocals in place of its divisions
    const double rho = ug[0], vx = ug[1] * __drcp_rn(rho), Et = ug[2];
    const double gm1 = GC ? rho * __drcp_rn(ug[3]) : __drcp_rn(ug[3]);  // gamma - 1
    const double p = gm1 * (Et - 0.5 * rho * vx * vx);
    const double cx = c.wq[g] * (c.ixx * c.J);
    const double fx[3] = {rho * vx, rho * vx * vx + p, (Et + p) * vx};
    const double s = (c.wq[g] * c.J) * (-vx * da * c.ixx);  // physics.cu:126-127
    const double fa = rho * vx * __drcp_rn(gm1);              // GAMCONS alpha flux, physics.cu:122-124
#pragma unroll
    for (int t = 0; t < N1; ++t) {
#pragma unroll
      for (int f = 0; f < 3; ++f) r[f][t] += c.Dq[g][t] * (cx * fx[f]);
      if (GC) r[3][t] += c.Dq[g][t] * (cx * fa);
      else r[3][t] += c.Bq[g][t] * s;
#pragma unroll
      for (int k = 0; k < NY; ++k) r[4 + k][t] += c.Dq[g][t] * (cx * (ug[4 + k] * vx));  // physics.cu:130-134
    }
  }
  // faces: left (node 0, x = -1) and right (node P, x = +1)
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const int nb = __ldg(a.nbr + (size_t)side * ld + e);
    const int to = side == 0 ? 0 : P;
    double uo[NF], un[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      uo[f] = u[f][to];
      if (nb >= 0) un[f] = __ldg(a.U + (size_t)(f * N1 + (side == 0 ? P : 0)) * ld + nb);
      else un[f] = (nb == -3 && f == 1) ? -uo[f] : uo[f];
    }
    const bool swapLR = side == 0 && nb >= 0;
    const double sgn = swapLR ? 1.0 : -1.0;
    const double nx = (side == 0 && nb < 0) ? -1.0 : 1.0;
    double L[NF], R[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) { L[f] = swapLR ? un[f] : uo[f]; R[f] = swapLR ? uo[f] : un[f]; }
    double F[NF], nc;
    phys::riemann1d<FLUX, NY, GC>(L[0], R[0], L[1] * __drcp_rn(L[0]), R[1] * __drcp_rn(R[0]), L[2], R[2], L[3], R[3],
                                  nx, F, nc, L + 4, R + 4);
#pragma unroll
    for (int f = 0; f < NF; ++f) r[f][to] += sgn * F[f] + (f == 3 ? nc : 0.0);
  }
}

template <int P, int FLUX, int MODE, int NY = 0, bool GC = false>
__device__ __forceinline__ void res1d_body(const Consts& c, const StageArgs& a, int e, double dt) {
  constexpr int N1 = P + 1, NF = 4 + NY;
  const int ld = c.ld;
  double u[NF][N1], r[NF][N1];
  res1d_residual<P, FLUX, NY, GC>(c, a, e, u, r);
  if constexpr (MODE == MODE_RESIDUAL) {
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int t = 0; t < N1; ++t) a.out[(size_t)(f * N1 + t) * ld + e] = r[f][t];
  } else {
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int t = 0; t < N1; ++t) {
        double s = 0.0;
#pragma unroll
        for (int tt = 0; tt < N1; ++tt) s += c.Minv[t][tt] * r[f][tt];
        const double du = dt * s;
        const size_t gi = (size_t)(f * N1 + t) * ld + e;
        if (MODE == MODE_SSP) {
          const double base = a.a != 0.0 ? a.a * __ldg(a.Ubase + gi) : 0.0;
          a.out[gi] = base + a.b * (u[f][t] + du);
        } else {
          a.out[gi] = du;
          if (a.Uacc) a.Uacc[gi] += a.b * du;
          if (a.Unext) a.Unext[gi] = __ldg(a.Us + gi) + a.beta_next * du;  // rk.cc:164-170
        }
      }
  }
}

template <int P, int FLUX, int MODE, int NY = 0, bool GC = false>
__global__ void __launch_bounds__(128) residual1d_kernel(const Consts cin, const StageArgs a) {
  __shared__ Consts c;
  copy_consts(c, cin);
  if (a.scal && a.scal->flags) return;
  __syncthreads();
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= c.n_elem) return;
  const double dt = MODE == MODE_RESIDUAL ? 0.0 : (a.dt_override > 0 ? a.dt_override : a.scal->dt);
  res1d_body<P, FLUX, MODE, NY, GC>(c, a, e, dt);
}

// ------------------------------------------------------------------------------------------
// Limiters.  Fields are limited slice by slice in the scaled Taylor basis (T, Tinv).
// ------------------------------------------------------------------------------------------
template <int P>
__device__ __forceinline__ void to_mono(const double* v, double* a) {
#pragma unroll
  for (int m = 0; m <= P; ++m) {
    double s = 0;
#pragma unroll
    for (int i = 0; i <= P; ++i) s += lim_T<P>(m, i) * v[i];
    a[m] = s;
  }
}
template <int P>
__device__ __forceinline__ void to_lag(const double* a, double* v) {
#pragma unroll
  for (int i = 0; i <= P; ++i) {
    double s = 0;
#pragma unroll
    for (int m = 0; m <= P; ++m) s += lim_Tinv<P>(i, m) * a[m];
    v[i] = s;
  }
}

// Limit one slice given the nodal values of the centre and (when interior) both neighbours.
// phys: 0 interior, 2/3 flatten (zero-gradient / reflective), 4 leave unchanged, 5 copy
// (reflective wall-normal momentum under HR limiting, hrl1D limiting_kernels.cu:291-302).
template <int P>
__device__ __forceinline__ void limit_slice(int phys, const double* vL, const double* vC, const double* vR,
                                            double* lim) {
  constexpr int N1 = P + 1;
  double aC[N1];
  to_mono<P>(vC, aC);
  if (phys == 0) {
    double aL[N1], aR[N1];
    to_mono<P>(vL, aL);
    to_mono<P>(vR, aR);
    limit_monomial<P>(aL, aC, aR, lim);
  } else if (phys == 2 || phys == 3) {
    average_monomial<P>(aC, lim);
  } else {
#pragma unroll
    for (int m = 0; m < N1; ++m) lim[m] = aC[m];
  }
}

// rho e = Leibniz product of the monomial p and alpha (internal_energy_multifluid,
// limiting_kernels.cu:160-199), then E (reconstruct_energy, limiting_kernels.cu:111-156)
template <int P>
__device__ __forceinline__ void reconstruct_energy(const double* plim, const double* alim, const double* Kmono,
                                                   const double* Emono, double* Elim) {
  constexpr int N1 = P + 1;
  constexpr double binom[4][4] = {{1, 0, 0, 0}, {1, 1, 0, 0}, {1, 2, 1, 0}, {1, 3, 3, 1}};
  double rhoe[N1];
#pragma unroll
  for (int m = 0; m < N1; ++m) {
    double I = 0;
#pragma unroll
    for (int k = 0; k <= m; ++k) I += binom[m][k] * plim[m - k] * alim[k];
    rhoe[m] = I;
  }
#pragma unroll
  for (int m = 1; m < N1; ++m) Elim[m] = rhoe[m] + Kmono[m];
  double E0 = Emono[0];
#pragma unroll
  for (int k = 2; k < N1; k += 2) E0 -= DGB_LIM(P, ifact[k + 1]) * (Elim[k] - Emono[k]);
  Elim[0] = E0;
}

__device__ __forceinline__ int boundary_code(int left, int right) {
  int phys = 0;
  if (left < 0) phys = -left;
  if (right < 0) phys = -right;
  return phys;
}

struct LimArgs {
  int ld, n_elem;
};

// 2D x pass, one thread per (element, y-slice).  METHOD 2 (m2): rho, rho u, rho v, alpha and
// p are limited and E rebuilt; output X = [rho, rhou, rhov, alpha, p, E] (Lagrange).
// METHOD 1 (HR): all conserved fields limited; output X = the five conserved fields.
template <int P, int METHOD>
__global__ void __launch_bounds__(128) lim2d_xpass_kernel(const LimArgs la, const double* __restrict__ U,
                                                          const int* __restrict__ nbr, double* __restrict__ X,
                                                          const DevScalars* __restrict__ scal) {
  constexpr int N1 = P + 1, NS = N1 * N1;
  if (scal && scal->flags) return;
  const int ld = la.ld, e = blockIdx.x * blockDim.x + threadIdx.x, iy = blockIdx.y;
  if (e >= la.n_elem) return;
  const int nL = __ldg(nbr + e), nR = __ldg(nbr + (size_t)ld + e);
  const int phys = boundary_code(nL, nR);
  double v[3][5][N1];  // [L,C,R][field][ix]
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const int el = s == 0 ? nL : s == 1 ? e : nR;
    if (s != 1 && phys != 0) continue;
#pragma unroll
    for (int f = 0; f < 5; ++f)
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) v[s][f][ix] = __ldg(U + (size_t)(f * NS + ix + N1 * iy) * ld + el);
  }
  if constexpr (METHOD == 1) {
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      double lim[N1], out[N1];
      const int ph = (phys == 3 && f == 1) ? 5 : phys;
      limit_slice<P>(ph, v[0][f], v[1][f], v[2][f], lim);
      to_lag<P>(lim, out);
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) X[(size_t)(f * NS + ix + N1 * iy) * ld + e] = out[ix];
    }
  } else {
    // pressure from the unlimited state (pressure kernel, physics.cu:891-958)
    double pr[3][N1];
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      if (s != 1 && phys != 0) continue;
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) {
        const double ru = v[s][1][ix], rv = v[s][2][ix], E = v[s][3][ix];
        const double gm1 = __drcp_rn(v[s][4][ix]);
        pr[s][ix] = gm1 * (E - 0.5 * (ru * ru + rv * rv) * __drcp_rn(v[s][0][ix]));
      }
    }
    double lr[N1], lu[N1], lv[N1], la_[N1], lp[N1];
    limit_slice<P>(phys, v[0][0], v[1][0], v[2][0], lr);
    limit_slice<P>(phys, v[0][1], v[1][1], v[2][1], lu);
    limit_slice<P>(phys, v[0][2], v[1][2], v[2][2], lv);
    limit_slice<P>(phys, v[0][4], v[1][4], v[2][4], la_);
    limit_slice<P>(phys, pr[0], pr[1], pr[2], lp);
    double r_[N1], u_[N1], v_[N1], a_[N1], p_[N1], K[N1], Km[N1], Em[N1], El[N1], E_[N1];
    to_lag<P>(lr, r_);
    to_lag<P>(lu, u_);
    to_lag<P>(lv, v_);
    to_lag<P>(la_, a_);
    to_lag<P>(lp, p_);
#pragma unroll
    for (int ix = 0; ix < N1; ++ix) K[ix] = 0.5 * (u_[ix] * u_[ix] + v_[ix] * v_[ix]) * __drcp_rn(r_[ix]);
    to_mono<P>(K, Km);
    to_mono<P>(v[1][3], Em);
    reconstruct_energy<P>(lp, la_, Km, Em, El);
    to_lag<P>(El, E_);
#pragma unroll
    for (int ix = 0; ix < N1; ++ix) {
      const size_t o = (size_t)(ix + N1 * iy) * ld + e;
      X[o + (size_t)0 * NS * ld] = r_[ix];
      X[o + (size_t)1 * NS * ld] = u_[ix];
      X[o + (size_t)2 * NS * ld] = v_[ix];
      X[o + (size_t)3 * NS * ld] = a_[ix];
      X[o + (size_t)4 * NS * ld] = p_[ix];
      X[o + (size_t)5 * NS * ld] = E_[ix];
    }
  }
}

// 2D y pass, one thread per (element, x-column): reads the x-pass output X of the element and
// its bottom/top neighbours and writes the limited conserved state.
template <int P, int METHOD>
__global__ void __launch_bounds__(128) lim2d_ypass_kernel(const LimArgs la, const double* __restrict__ X,
                                                          const int* __restrict__ nbr, double* __restrict__ Uout,
                                                          const DevScalars* __restrict__ scal) {
  constexpr int N1 = P + 1, NS = N1 * N1;
  constexpr int NQ = METHOD == 1 ? 5 : 6;
  if (scal && scal->flags) return;
  const int ld = la.ld, e = blockIdx.x * blockDim.x + threadIdx.x, ix = blockIdx.y;
  if (e >= la.n_elem) return;
  const int nD = __ldg(nbr + (size_t)2 * ld + e), nU = __ldg(nbr + (size_t)3 * ld + e);
  const int phys = boundary_code(nD, nU);
  double v[3][NQ][N1];  // [D,C,U][field][iy]
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const int el = s == 0 ? nD : s == 1 ? e : nU;
    if (s != 1 && phys != 0) continue;
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
      for (int iy = 0; iy < N1; ++iy) v[s][q][iy] = __ldg(X + (size_t)(q * NS + ix + N1 * iy) * ld + el);
  }
  if constexpr (METHOD == 1) {
#pragma unroll
    for (int f = 0; f < 5; ++f) {
      double lim[N1], out[N1];
      const int ph = (phys == 3 && f == 2) ? 5 : phys;
      limit_slice<P>(ph, v[0][f], v[1][f], v[2][f], lim);
      to_lag<P>(lim, out);
#pragma unroll
      for (int iy = 0; iy < N1; ++iy) Uout[(size_t)(f * NS + ix + N1 * iy) * ld + e] = out[iy];
    }
  } else {
    double lr[N1], lu[N1], lv[N1], la_[N1], lp[N1];
    limit_slice<P>(phys, v[0][0], v[1][0], v[2][0], lr);
    limit_slice<P>(phys, v[0][1], v[1][1], v[2][1], lu);
    limit_slice<P>(phys, v[0][2], v[1][2], v[2][2], lv);
    limit_slice<P>(phys, v[0][3], v[1][3], v[2][3], la_);
    limit_slice<P>(phys, v[0][4], v[1][4], v[2][4], lp);
    double r_[N1], u_[N1], v_[N1], a_[N1], K[N1], Km[N1], Em[N1], El[N1], E_[N1];
    to_lag<P>(lr, r_);
    to_lag<P>(lu, u_);
    to_lag<P>(lv, v_);
    to_lag<P>(la_, a_);
#pragma unroll
    for (int iy = 0; iy < N1; ++iy) K[iy] = 0.5 * (u_[iy] * u_[iy] + v_[iy] * v_[iy]) * __drcp_rn(r_[iy]);
    to_mono<P>(K, Km);
    to_mono<P>(v[1][5], Em);
    reconstruct_energy<P>(lp, la_, Km, Em, El);
    to_lag<P>(El, E_);
#pragma unroll
    for (int iy = 0; iy < N1; ++iy) {
      const size_t o = (size_t)(ix + N1 * iy) * ld + e;
      Uout[o + (size_t)0 * NS * ld] = r_[iy];
      Uout[o + (size_t)1 * NS * ld] = u_[iy];
      Uout[o + (size_t)2 * NS * ld] = v_[iy];
      Uout[o + (size_t)3 * NS * ld] = E_[iy];
      Uout[o + (size_t)4 * NS * ld] = a_[iy];
    }
  }
}

// The limited nodal values o of one element from its slices v[0] (left neighbour), v[1] (itself),
// v[2] (right neighbour; the neighbours' slices are read only when phys == 0).
template <int P, int METHOD, int NY = 0>
__device__ __forceinline__ void lim1d_limit(int phys, const double (&v)[3][4 + NY][P + 1],
                                            double (&o)[4 + NY][P + 1]) {
  constexpr int N1 = P + 1, NF = 4 + NY;
  if constexpr (METHOD == 1) {
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      double lim[N1];
      const int ph = (phys == 3 && f == 1) ? 5 : phys;
      limit_slice<P>(ph, v[0][f], v[1][f], v[2][f], lim);
      to_lag<P>(lim, o[f]);
    }
  } else {
    double pr[3][N1];
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      if (s != 1 && phys != 0) continue;
#pragma unroll
      for (int i = 0; i < N1; ++i) {
        const double ru = v[s][1][i], E = v[s][2][i];
        const double gm1 = __drcp_rn(v[s][3][i]);
        pr[s][i] = gm1 * (E - 0.5 * ru * ru * __drcp_rn(v[s][0][i]));
      }
    }
    double lr[N1], lu[N1], la_[N1], lp[N1];
    limit_slice<P>(phys, v[0][0], v[1][0], v[2][0], lr);
    limit_slice<P>(phys, v[0][1], v[1][1], v[2][1], lu);
    limit_slice<P>(phys, v[0][3], v[1][3], v[2][3], la_);
    limit_slice<P>(phys, pr[0], pr[1], pr[2], lp);
    double K[N1], Km[N1], Em[N1], El[N1];
    to_lag<P>(lr, o[0]);
    to_lag<P>(lu, o[1]);
    to_lag<P>(la_, o[3]);
#pragma unroll
    for (int i = 0; i < N1; ++i) K[i] = 0.5 * o[1][i] * o[1][i] * __drcp_rn(o[0][i]);  // kinetic_energy1D
    to_mono<P>(K, Km);
    to_mono<P>(v[1][2], Em);
    reconstruct_energy<P>(lp, la_, Km, Em, El);
    to_lag<P>(El, o[2]);
#pragma unroll
    for (int k = 4; k < NF; ++k) {
      double ly[N1];
      limit_slice<P>(phys, v[0][k], v[1][k], v[2][k], ly);
      to_lag<P>(ly, o[k]);
    }
  }
}

// 1D HR / m2 limiter, one thread per element (reads U, writes Uout).  Mass fractions are limited
// like the density (HR: every field; m2: the MACRO block of M2limiting, limiting.cc:186-193).
template <int P, int METHOD, int NY = 0>
__device__ __forceinline__ void lim1d_body(int ld, int e, const double* __restrict__ U, const int* __restrict__ nbr,
                                           double* __restrict__ Uout) {
  constexpr int N1 = P + 1, NF = 4 + NY;
  const int nL = __ldg(nbr + e), nR = __ldg(nbr + (size_t)ld + e);
  const int phys = boundary_code(nL, nR);
  double v[3][NF][N1];
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const int el = s == 0 ? nL : s == 1 ? e : nR;
    if (s != 1 && phys != 0) continue;
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int i = 0; i < N1; ++i) v[s][f][i] = __ldg(U + (size_t)(f * N1 + i) * ld + el);
  }
  double o[NF][N1];
  lim1d_limit<P, METHOD, NY>(phys, v, o);
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int i = 0; i < N1; ++i) Uout[(size_t)(f * N1 + i) * ld + e] = o[f][i];
}

template <int P, int METHOD, int NY = 0>
__global__ void __launch_bounds__(128) lim1d_kernel(const LimArgs la, const double* __restrict__ U,
                                                    const int* __restrict__ nbr, double* __restrict__ Uout,
                                                    const DevScalars* __restrict__ scal) {
  if (scal && scal->flags) return;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= la.n_elem) return;
  lim1d_body<P, METHOD, NY>(la.ld, e, U, nbr, Uout);
}

// One stage of a 1D problem whose elements form a chain (the neighbours of element e are e - 1 and
// e + 1; at the ends a boundary code or, periodic, the other end): residual, stage update and the
// hrl / m2l limiter in one launch.  A CTA advances a block of RL1D_B elements plus the element on
// either side of it (recomputed here, not written), keeps the limiter's input in shared memory
// and limits the block from there, so the unlimited stage output never goes to global memory.
//   MODE_SSP  limiter input a Ubase + b (U + du)
//   MODE_RK4  accumulator acc_out = acc_in + b du (two buffers: a neighbouring block reads acc_in);
//             limiter input the next stage input Us + beta_next du, or (last stage) acc_out
// lim_out must be none of the buffers the stage reads (U, Ubase, Us, acc_in).
constexpr int RL1D_B = 64;
template <int P, int FLUX, int MODE, int METHOD>
__global__ void __launch_bounds__(96) res_lim1d_chain_kernel(const Consts cin, const StageArgs a,
                                                             const double* __restrict__ acc_in,
                                                             double* __restrict__ acc_out, int last,
                                                             double* __restrict__ lim_out) {
  constexpr int N1 = P + 1, NF = 4, B = RL1D_B;
  __shared__ Consts c;
  __shared__ double V[NF * N1][B + 2];  // limiter input of slot s: element e0 + s - 1
  copy_consts(c, cin);
  if (a.scal && a.scal->flags) return;
  __syncthreads();
  const int ld = c.ld;
  const int e0 = blockIdx.x * B, nb = min(B, c.n_elem - e0);
  const int s = threadIdx.x;
  if (s < nb + 2) {
    const bool own = s >= 1 && s <= nb;
    const int e = own ? e0 + s - 1 : s == 0 ? __ldg(a.nbr + e0) : __ldg(a.nbr + (size_t)ld + e0 + nb - 1);
    if (e >= 0) {
      const double dt = a.dt_override > 0 ? a.dt_override : a.scal->dt;
      double u[NF][N1], r[NF][N1];
      res1d_residual<P, FLUX>(c, a, e, u, r);
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int t = 0; t < N1; ++t) {
          double sm = 0.0;
#pragma unroll
          for (int tt = 0; tt < N1; ++tt) sm += c.Minv[t][tt] * r[f][tt];
          const double du = dt * sm;
          const size_t gi = (size_t)(f * N1 + t) * ld + e;
          double w;
          if constexpr (MODE == MODE_SSP) {
            const double base = a.a != 0.0 ? a.a * __ldg(a.Ubase + gi) : 0.0;
            w = base + a.b * (u[f][t] + du);
          } else {
            const double acc = __ldg(acc_in + gi) + a.b * du;
            if (own) acc_out[gi] = acc;
            w = last ? acc : __ldg(a.Us + gi) + a.beta_next * du;  // rk.cc:164-170
          }
          V[f * N1 + t][s] = w;
        }
    }
  }
  __syncthreads();
  if (s >= 1 && s <= nb) {
    const int e = e0 + s - 1;
    const int phys = boundary_code(__ldg(a.nbr + e), __ldg(a.nbr + (size_t)ld + e));
    double v[3][NF][N1];
#pragma unroll
    for (int sl = 0; sl < 3; ++sl) {
      if (sl != 1 && phys != 0) continue;
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int i = 0; i < N1; ++i) v[sl][f][i] = V[f * N1 + i][s - 1 + sl];
    }
    double o[NF][N1];
    lim1d_limit<P, METHOD>(phys, v, o);
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int i = 0; i < N1; ++i) lim_out[(size_t)(f * N1 + i) * ld + e] = o[f][i];
  }
}

// ------------------------------------------------------------------------------------------
// CFL step: max over nodes of the wave speed, then dt = CFL_scaled / max (on the device)
// ------------------------------------------------------------------------------------------
// The step dt from scal->umax (and the checks of rk.cc:146-149): by finish_dt_kernel, or by the
// last CTA of a wave-speed reduction.
// The scalars are read through volatile loads: in the last CTA of a reduction this SM may hold a
// line of them from before the other CTAs' atomics.
__device__ __forceinline__ void finish_dt(DevScalars* scal, double cfl_scaled) {
  volatile DevScalars* v = scal;
  if (v->flags) return;
  double dt;
  if (v->dt_fixed > 0) dt = v->dt_fixed;
  else {
    const double umax = __longlong_as_double((long long)v->umax);
    dt = cfl_scaled / umax;
    if (!(dt == dt)) atomicOr(&scal->flags, (unsigned)FLAG_NONFINITE);
    else if (dt < 1e-14) atomicOr(&scal->flags, (unsigned)FLAG_DT_SMALL);
  }
  v->umax = 0ull;
  if (v->flags) return;
  v->dt = dt;
  v->time = v->time + dt;
}

// copy_to (1D RK4, or null): the nf fields of every element read are also written there (the
// step's accumulator starts as the state).  finish > 0: the last CTA to add its maximum forms the
// step from it (that CFL scale), so no separate finish launch is needed; 0 leaves umax for a caller
// that reduces it further (slab mode).
// Grid: (element blocks, NS): a CTA reads one node of its elements -- five loads per element, few
// registers, full occupancy -- and strides over the elements two at a time, so that both
// elements' loads are in flight together.
template <int DIM, int NS, bool GC = false>
__global__ void __launch_bounds__(256) wavespeed_kernel(const double* __restrict__ U, int n_elem, int ld,
                                                        DevScalars* __restrict__ scal,
                                                        double* __restrict__ copy_to, int nf, double finish) {
  constexpr int NV = DIM == 1 ? 4 : 5;  // fields the wave speed reads
  pdl_wait();
  if (scal->flags) return;
  double m = 0.0;
  bool bad = false;
  const int t = blockIdx.y, stride = gridDim.x * blockDim.x;
  for (int e0 = blockIdx.x * blockDim.x + threadIdx.x; e0 < n_elem; e0 += 2 * stride) {
    double v[2][NV];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int e = e0 + r * stride;
      if (e < n_elem)
#pragma unroll
        for (int f = 0; f < NV; ++f) v[r][f] = __ldg(U + (size_t)(f * NS + t) * ld + e);
    }
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int e = e0 + r * stride;
      if (e >= n_elem) continue;
      double w;
      if constexpr (DIM == 1)
        w = phys::wave_speed1d<GC>(v[r][0], v[r][1], v[r][2], v[r][3]);
      else
        w = phys::wave_speed2d<GC>(v[r][0], v[r][1], v[r][2], v[r][3], v[r][4]);
      if (!(w == w)) bad = true;
      else m = fmax(m, fabs(w));
      if (copy_to)
        for (int f = 0; f < nf; ++f) copy_to[(size_t)(f * NS + t) * ld + e] = __ldg(U + (size_t)(f * NS + t) * ld + e);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double wm[8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) wm[w] = m;
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&scal->flags, (unsigned)FLAG_NONFINITE);
  __syncthreads();
  if (threadIdx.x == 0) {
    double mm = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) mm = fmax(mm, wm[k]);
    atomicMax(&scal->umax, (unsigned long long)__double_as_longlong(mm));
    if (finish > 0) {
      __threadfence();  // this CTA's maximum and flags before its count
      if (atomicAdd(&scal->blocks_done, 1u) == gridDim.x * gridDim.y - 1) {
        __threadfence();  // every other CTA's maximum is in umax
        scal->blocks_done = 0;
        finish_dt(scal, finish);
      }
    }
  }
}

static __global__ void finish_dt_kernel(DevScalars* scal, double cfl_scaled) { finish_dt(scal, cfl_scaled); }

// ------------------------------------------------------------------------------------------
// Layout conversion (API boundary only), RK4 helpers
// ------------------------------------------------------------------------------------------
static __global__ void ref_to_internal_kernel(const double* __restrict__ Uref, double* __restrict__ Uint,
                                       const int* __restrict__ perm, int n_elem, int nf, int ns, int ld) {
  const size_t n = (size_t)n_elem * nf * ns;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int t = (int)(i % ns);
    const size_t r = i / ns;
    const int f = (int)(r % nf);
    const int e = (int)(r / nf);
    Uint[(size_t)(f * ns + t) * ld + e] = Uref[((size_t)e * nf + f) * ns + perm[t]];
  }
}
static __global__ void internal_to_ref_kernel(const double* __restrict__ Uint, double* __restrict__ Uref,
                                       const int* __restrict__ perm, int n_elem, int nf, int ns, int ld) {
  const size_t n = (size_t)n_elem * nf * ns;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int t = (int)(i % ns);
    const size_t r = i / ns;
    const int f = (int)(r % nf);
    const int e = (int)(r / nf);
    Uref[((size_t)e * nf + f) * ns + perm[t]] = Uint[(size_t)(f * ns + t) * ld + e];
  }
}
// The same conversions through a shared-memory tile of CONV_EB elements, so that both layouts are
// read and written in contiguous runs: the element-major reference block (CONV_EB * nf * ns
// values in a row) on one side, CONV_EB consecutive elements of every (field, node) plane on the
// other.  Grid-stride over the element blocks; dynamic shared memory CONV_EB * (nf * ns + 1) doubles.
constexpr int CONV_EB = 16;
inline size_t convert_smem_bytes(int nf, int ns) { return sizeof(double) * CONV_EB * (nf * ns + 1); }
template <bool TO_INTERNAL>
__global__ void __launch_bounds__(256) convert_layout_kernel(const double* __restrict__ src, double* __restrict__ dst,
                                                             const int* __restrict__ perm, int n_elem, int nf, int ns,
                                                             int ld) {
  extern __shared__ double cs_tile[];  // [element][reference-layout value], pitch nv + 1
  const int nv = nf * ns, pitch = nv + 1, nblocks = (n_elem + CONV_EB - 1) / CONV_EB;
  for (int b = blockIdx.x; b < nblocks; b += gridDim.x) {
    const int e0 = b * CONV_EB, ne = min(CONV_EB, n_elem - e0);
    if (TO_INTERNAL) {
      const double* s = src + (size_t)e0 * nv;
      for (int j = threadIdx.x; j < ne * nv; j += blockDim.x) {
        const int el = j / nv;
        cs_tile[el * pitch + (j - el * nv)] = s[j];
      }
      __syncthreads();
      for (int j = threadIdx.x; j < nv * CONV_EB; j += blockDim.x) {
        const int q = j / CONV_EB, el = j - q * CONV_EB;  // q = f * ns + t (internal plane)
        if (el >= ne) continue;
        const int f = q / ns, t = q - f * ns;
        dst[(size_t)q * ld + e0 + el] = cs_tile[el * pitch + f * ns + __ldg(perm + t)];
      }
    } else {
      for (int j = threadIdx.x; j < nv * CONV_EB; j += blockDim.x) {
        const int q = j / CONV_EB, el = j - q * CONV_EB;
        if (el >= ne) continue;
        const int f = q / ns, t = q - f * ns;
        cs_tile[el * pitch + f * ns + __ldg(perm + t)] = src[(size_t)q * ld + e0 + el];
      }
      __syncthreads();
      double* d = dst + (size_t)e0 * nv;
      for (int j = threadIdx.x; j < ne * nv; j += blockDim.x) {
        const int el = j / nv;
        d[j] = cs_tile[el * pitch + (j - el * nv)];
      }
    }
    __syncthreads();  // the tile is rewritten by the next block
  }
}

// y = x + beta*d over n values (Ustar = Us + beta DU, rk.cc:167-168)
static __global__ void axpy_kernel(const double* __restrict__ x, const double* __restrict__ d, double beta,
                            double* __restrict__ y, size_t n, const DevScalars* __restrict__ scal) {
  if (scal && scal->flags) return;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = x[i] + beta * d[i];
}

}  // namespace dgb
