// Tiled 2D limiter passes for structured row-major grids (HR and m2 methods).
//
// Same arithmetic as lim2d_xpass_kernel / lim2d_ypass_kernel, but every element's monomial
// coefficients (and, for m2, its nodal pressure) are computed once per slice and shared through
// shared memory with the neighbours that need them, instead of being recomputed by the three
// threads that read them.
//   x pass: CTA = 30 consecutive elements of one element row (+ left/right neighbour slots),
//           threads (element slot, y-slice)
//   y pass: CTA = 32 x 4 elements (+ bottom/top neighbour rows), threads (x slot, row slot),
//           one x-column of nodes per CTA (grid z)
// Output of the x pass (global scratch X): m2 -> [rho, rhou, rhov, alpha, p, E],
// HR -> the five conserved fields, all x-limited and in Lagrange form (limiting.cc:271-409).
#pragma once
#include "kernels.cuh"

namespace dgb {

// Dynamic shared memory of the tiled limiter passes: 0 while their per-quantity arrays fit the
// static limit (up to three mass fractions), else the arrays' size
template <int P, int NY>
constexpr size_t lim2d_xpass_smem_bytes() {
  const size_t b = sizeof(double) * (5 + NY) * (P + 1) * (P + 1) * 32;
  return b <= 48 * 1024 ? 0 : b;
}
template <int P, int NY>
constexpr size_t lim2d_ypass_smem_bytes() {
  const size_t b = sizeof(double) * (5 + NY) * (P + 1) * 6 * 32;
  return b <= 48 * 1024 ? 0 : b;
}

// x pass over one block of the row ey starting at element column x0 (a multiple of 30); the CTA
// returns from here together, after its last barrier
// NY mass fractions: limited like the density (m2: the MACRO blocks of M2limiting,
// limiting.cc:327-331 and 398-404; HR: every field); in X after E (m2) or as fields (HR).
template <int P, int METHOD, int NY = 0>
__device__ __forceinline__ void lim2d_xpass_body(const LimArgs la, int nx, const double* __restrict__ U,
                                                 const int* __restrict__ nbr, double* __restrict__ X, int x0,
                                                 int ey) {
  constexpr int N1 = P + 1, NS = N1 * N1, NQ = 5 + NY, NF = 5 + NY, TWI = 30;
  // [quantity][slice][coefficient][slot]: static shared memory, or dynamic (lim2d_xpass_smem_bytes)
  // when the quantities would not fit the static limit (many mass fractions)
  double(*A)[N1][N1][32];
  if constexpr (lim2d_xpass_smem_bytes<P, NY>() == 0) {
    __shared__ double As[NQ][N1][N1][32];
    A = As;
  } else {
    extern __shared__ __align__(16) double lsm[];
    A = reinterpret_cast<double(*)[N1][N1][32]>(lsm);
  }
  const int ld = la.ld;
  const int tx = threadIdx.x, sl = threadIdx.y;
  const int ex = x0 - 1 + tx;
  // element held by this slot: interior element, or the neighbour of the adjacent interior one
  const bool interior = tx >= 1 && tx <= TWI && ex < nx;
  int e = -1;
  if (interior) e = ey * nx + ex;
  else if (tx == 0) e = __ldg(nbr + (size_t)0 * ld + ey * nx + x0);
  else if (ex - 1 < nx && ex - 1 >= 0) e = __ldg(nbr + (size_t)1 * ld + ey * nx + ex - 1);
  double v[NF][N1];
  double Em[N1];
  if (e >= 0) {
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) v[f][ix] = __ldg(U + (size_t)(f * NS + ix + N1 * sl) * ld + e);
    double q[NQ][N1];
#pragma unroll
    for (int ix = 0; ix < N1; ++ix) {
#pragma unroll
      for (int k = 5; k < NQ; ++k) q[k][ix] = v[k][ix];
      if constexpr (METHOD == 1) {
#pragma unroll
        for (int f = 0; f < 5; ++f) q[f][ix] = v[f][ix];
      } else {
        q[0][ix] = v[0][ix];
        q[1][ix] = v[1][ix];
        q[2][ix] = v[2][ix];
        q[3][ix] = v[4][ix];
        // pressure from the unlimited state (pressure kernel, physics.cu:891-958), with correctly
        // rounded reciprocals in place of its divisions
        const double ru = v[1][ix], rv = v[2][ix];
        q[4][ix] = __drcp_rn(v[4][ix]) * (v[3][ix] - 0.5 * (ru * ru + rv * rv) * __drcp_rn(v[0][ix]));
      }
    }
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      double a[N1];
      to_mono<P>(q[k], a);
#pragma unroll
      for (int m = 0; m < N1; ++m) A[k][sl][m][tx] = a[m];
    }
    if constexpr (METHOD == 2) to_mono<P>(v[3], Em);
  }
  __syncthreads();
  if (!interior) return;
  const int phys = boundary_code(__ldg(nbr + (size_t)0 * ld + e), __ldg(nbr + (size_t)1 * ld + e));
  double lim[NQ][N1];
#pragma unroll
  for (int k = 0; k < NQ; ++k) {
    double aL[N1], aC[N1], aR[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m) aC[m] = A[k][sl][m][tx];
    const int ph = (METHOD == 1 && phys == 3 && k == 1) ? 5 : phys;
    if (ph == 0) {
#pragma unroll
      for (int m = 0; m < N1; ++m) { aL[m] = A[k][sl][m][tx - 1]; aR[m] = A[k][sl][m][tx + 1]; }
      limit_monomial<P>(aL, aC, aR, lim[k]);
    } else if (ph == 2 || ph == 3) {
      average_monomial<P>(aC, lim[k]);
    } else {
#pragma unroll
      for (int m = 0; m < N1; ++m) lim[k][m] = aC[m];
    }
  }
  if constexpr (METHOD == 1) {
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      double out[N1];
      to_lag<P>(lim[k], out);
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) X[(size_t)(k * NS + ix + N1 * sl) * ld + e] = out[ix];
    }
  } else {
    double r_[N1], u_[N1], v_[N1], a_[N1], p_[N1], K[N1], Km[N1], El[N1], E_[N1];
    to_lag<P>(lim[0], r_);
    to_lag<P>(lim[1], u_);
    to_lag<P>(lim[2], v_);
    to_lag<P>(lim[3], a_);
    to_lag<P>(lim[4], p_);
#pragma unroll
    for (int ix = 0; ix < N1; ++ix) K[ix] = 0.5 * (u_[ix] * u_[ix] + v_[ix] * v_[ix]) * __drcp_rn(r_[ix]);
    to_mono<P>(K, Km);
    reconstruct_energy<P>(lim[4], lim[3], Km, Em, El);
    to_lag<P>(El, E_);
#pragma unroll
    for (int ix = 0; ix < N1; ++ix) {
      const size_t o = (size_t)(ix + N1 * sl) * ld + e;
      X[o + (size_t)0 * NS * ld] = r_[ix];
      X[o + (size_t)1 * NS * ld] = u_[ix];
      X[o + (size_t)2 * NS * ld] = v_[ix];
      X[o + (size_t)3 * NS * ld] = a_[ix];
      X[o + (size_t)4 * NS * ld] = p_[ix];
      X[o + (size_t)5 * NS * ld] = E_[ix];
    }
#pragma unroll
    for (int k = 5; k < NQ; ++k) {
      double y_[N1];
      to_lag<P>(lim[k], y_);
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) X[(size_t)((k + 1) * NS + ix + N1 * sl) * ld + e] = y_[ix];
    }
  }
}

template <int P, int METHOD, int NY = 0>
__global__ void __launch_bounds__(32 * (P + 1)) lim2d_xpass_tile_kernel(const LimArgs la, int nx,
                                                                      const double* __restrict__ U,
                                                                      const int* __restrict__ nbr,
                                                                      double* __restrict__ X,
                                                                      const DevScalars* __restrict__ scal) {
  pdl_wait();
  if (scal && scal->flags) return;
  lim2d_xpass_body<P, METHOD, NY>(la, nx, U, nbr, X, blockIdx.x * 30, blockIdx.y);
  pdl_trigger();
}

// y pass over the 32 x 4 element block at (x0, y0) for the node column ix; the CTA returns from
// here together, after its last barrier
template <int P, int METHOD, int NY = 0>
__device__ __forceinline__ void lim2d_ypass_body(const LimArgs la, int nx, int ny, const double* __restrict__ X,
                                                 const int* __restrict__ nbr, double* __restrict__ Uout, int x0,
                                                 int y0, int ix) {
  constexpr int N1 = P + 1, NS = N1 * N1, NQ = 5 + NY, THI = 4;
  // row of quantity k in X: HR -> field k; m2 -> [rho, rhou, rhov, alpha, p, E, rho Y_k]
  auto xrow = [](int k) { return (METHOD == 2 && k >= 5) ? k + 1 : k; };
  // [quantity][coefficient][row slot][x slot]: static or (many mass fractions) dynamic
  double(*B)[N1][THI + 2][32];
  if constexpr (lim2d_ypass_smem_bytes<P, NY>() == 0) {
    __shared__ double Bs[NQ][N1][THI + 2][32];
    B = Bs;
  } else {
    extern __shared__ __align__(16) double lsm[];
    B = reinterpret_cast<double(*)[N1][THI + 2][32]>(lsm);
  }
  const int ld = la.ld;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int x = x0 + tx;
  const int yy = y0 - 1 + ty;
  const bool interior = ty >= 1 && ty <= THI && yy < ny && x < nx;
  int e = -1;
  if (x < nx) {
    if (interior) e = yy * nx + x;
    else if (ty == 0) e = __ldg(nbr + (size_t)2 * ld + y0 * nx + x);
    else if (yy - 1 < ny && yy - 1 >= 0) e = __ldg(nbr + (size_t)3 * ld + (yy - 1) * nx + x);
  }
  double Em[N1];
  if (e >= 0) {
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      double col[N1], a[N1];
#pragma unroll
      for (int iy = 0; iy < N1; ++iy) col[iy] = __ldg(X + (size_t)(xrow(k) * NS + ix + N1 * iy) * ld + e);
      to_mono<P>(col, a);
#pragma unroll
      for (int m = 0; m < N1; ++m) B[k][m][ty][tx] = a[m];
    }
    if constexpr (METHOD == 2) {
      double col[N1];
#pragma unroll
      for (int iy = 0; iy < N1; ++iy) col[iy] = __ldg(X + (size_t)(5 * NS + ix + N1 * iy) * ld + e);
      to_mono<P>(col, Em);
    }
  }
  __syncthreads();
  if (!interior) return;
  const int phys = boundary_code(__ldg(nbr + (size_t)2 * ld + e), __ldg(nbr + (size_t)3 * ld + e));
  double lim[NQ][N1];
#pragma unroll
  for (int k = 0; k < NQ; ++k) {
    double aD[N1], aC[N1], aU[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m) aC[m] = B[k][m][ty][tx];
    const int ph = (METHOD == 1 && phys == 3 && k == 2) ? 5 : phys;
    if (ph == 0) {
#pragma unroll
      for (int m = 0; m < N1; ++m) { aD[m] = B[k][m][ty - 1][tx]; aU[m] = B[k][m][ty + 1][tx]; }
      limit_monomial<P>(aD, aC, aU, lim[k]);
    } else if (ph == 2 || ph == 3) {
      average_monomial<P>(aC, lim[k]);
    } else {
#pragma unroll
      for (int m = 0; m < N1; ++m) lim[k][m] = aC[m];
    }
  }
  if constexpr (METHOD == 1) {
#pragma unroll
    for (int k = 0; k < NQ; ++k) {
      double out[N1];
      to_lag<P>(lim[k], out);
#pragma unroll
      for (int iy = 0; iy < N1; ++iy) Uout[(size_t)(k * NS + ix + N1 * iy) * ld + e] = out[iy];
    }
  } else {
    double r_[N1], u_[N1], v_[N1], a_[N1], K[N1], Km[N1], El[N1], E_[N1];
    to_lag<P>(lim[0], r_);
    to_lag<P>(lim[1], u_);
    to_lag<P>(lim[2], v_);
    to_lag<P>(lim[3], a_);
#pragma unroll
    for (int iy = 0; iy < N1; ++iy) K[iy] = 0.5 * (u_[iy] * u_[iy] + v_[iy] * v_[iy]) * __drcp_rn(r_[iy]);
    to_mono<P>(K, Km);
    reconstruct_energy<P>(lim[4], lim[3], Km, Em, El);
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
#pragma unroll
    for (int k = 5; k < NQ; ++k) {
      double y_[N1];
      to_lag<P>(lim[k], y_);
#pragma unroll
      for (int iy = 0; iy < N1; ++iy) Uout[(size_t)(k * NS + ix + N1 * iy) * ld + e] = y_[iy];
    }
  }
}

template <int P, int METHOD, int NY = 0>
__global__ void __launch_bounds__(32 * 6) lim2d_ypass_tile_kernel(const LimArgs la, int nx, int ny,
                                                                  const double* __restrict__ X,
                                                                  const int* __restrict__ nbr,
                                                                  double* __restrict__ Uout,
                                                                  const DevScalars* __restrict__ scal) {
  pdl_wait();
  if (scal && scal->flags) return;
  lim2d_ypass_body<P, METHOD, NY>(la, nx, ny, X, nbr, Uout, blockIdx.x * 32, blockIdx.y * 4, blockIdx.z);
  pdl_trigger();
}

}  // namespace dgb

namespace dgb {

template <int P, int METHOD>
constexpr size_t lim2d_fused_smem_bytes() {
  return ((size_t)5 * (P + 1) * (P + 1) * 32 + (size_t)3 * (METHOD == 2 ? 6 : 5) * (P + 1) * (P + 1) * 32) *
         sizeof(double);
}

// Both limiter passes in one kernel.  A CTA owns a strip of 30 element columns and H element rows
// and walks up the strip one row at a time: the x pass of row r (threads: element slot incl. the
// left/right neighbour slots, y-slice) writes its x-limited Lagrange values into a three-row ring
// buffer in shared memory, then the y pass of row r-1 (threads: element slot, x-column) reads
// rows r-2, r-1, r from the ring and writes the limited state.  The rows below and above the strip
// are x-limited too (2/H extra x work), so the x-limited intermediate never goes to HBM.  Rows
// beyond the domain edges come from the neighbour table (periodic wrap) or are absent (walls,
// transmissive boundaries: the y pass then needs no neighbour).  Same arithmetic as
// lim2d_xpass_tile_kernel followed by lim2d_ypass_tile_kernel.  Uout must not alias U.
template <int P, int METHOD, int H>
__global__ void __launch_bounds__(32 * (P + 1)) lim2d_fused_tile_kernel(const LimArgs la, int nx, int ny,
                                                                       const double* __restrict__ U,
                                                                       const int* __restrict__ nbr,
                                                                       double* __restrict__ Uout,
                                                                       const DevScalars* __restrict__ scal) {
  constexpr int N1 = P + 1, NS = N1 * N1, NQ = 5, NQS = METHOD == 2 ? 6 : 5, TWI = 30;
  extern __shared__ __align__(16) double lsm[];
  auto A = reinterpret_cast<double(*)[N1][N1][32]>(lsm);                 // [q][slice][m][slot]
  auto XR = reinterpret_cast<double(*)[NQS][NS][32]>(lsm + NQ * N1 * N1 * 32);  // [row % 3][q][node][slot]
  if (scal && scal->flags) return;
  const int ld = la.ld;
  const int tx = threadIdx.x, sl = threadIdx.y;
  const int x0 = blockIdx.x * TWI, y0 = blockIdx.y * H;
  const int nrow = min(H, ny - y0);
  const int ex = x0 - 1 + tx;
  const bool icol = tx >= 1 && tx <= TWI && ex < nx;
  // element of column x (0 <= x < nx) in strip row s (s = 0: the row below, s = nrow + 1: above)
  auto row_elem = [&](int s, int x) -> int {
    if (s >= 1 && s <= nrow) return (y0 + s - 1) * nx + x;
    if (s == 0) return __ldg(nbr + (size_t)2 * ld + y0 * nx + x);
    return __ldg(nbr + (size_t)3 * ld + (y0 + nrow - 1) * nx + x);
  };
  auto lane_elem = [&](int s) -> int {
    if (icol) return row_elem(s, ex);
    if (tx == 0) {
      const int e1 = row_elem(s, x0);
      return e1 >= 0 ? __ldg(nbr + e1) : -1;
    }
    if (ex - 1 < nx && ex - 1 >= 0) {
      const int el = row_elem(s, ex - 1);
      return el >= 0 ? __ldg(nbr + (size_t)ld + el) : -1;
    }
    return -1;
  };
  double v[5][N1];  // raw values of this lane's slice in the current row (prefetched)
  int e = lane_elem(0);
  if (e >= 0) {
#pragma unroll
    for (int f = 0; f < 5; ++f)
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) v[f][ix] = __ldg(U + (size_t)(f * NS + ix + N1 * sl) * ld + e);
  }
  for (int s = 0; s <= nrow + 1; ++s) {
    // ---- x pass of strip row s: monomial coefficients of every slot ----
    double Em[N1];
    if (e >= 0) {
      double q[NQ][N1];
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) {
        if constexpr (METHOD == 1) {
#pragma unroll
          for (int f = 0; f < 5; ++f) q[f][ix] = v[f][ix];
        } else {
          q[0][ix] = v[0][ix];
          q[1][ix] = v[1][ix];
          q[2][ix] = v[2][ix];
          q[3][ix] = v[4][ix];
          const double ru = v[1][ix], rv = v[2][ix];
          q[4][ix] = __drcp_rn(v[4][ix]) * (v[3][ix] - 0.5 * (ru * ru + rv * rv) * __drcp_rn(v[0][ix]));
        }
      }
#pragma unroll
      for (int k = 0; k < NQ; ++k) {
        double am[N1];
        to_mono<P>(q[k], am);
#pragma unroll
        for (int m = 0; m < N1; ++m) A[k][sl][m][tx] = am[m];
      }
      if constexpr (METHOD == 2) to_mono<P>(v[3], Em);
    }
    __syncthreads();
    // ---- x pass: limit the interior slots, x-limited Lagrange values into the ring ----
    const int slot = s % 3;
    if (icol && e >= 0) {
      const int phys = boundary_code(__ldg(nbr + e), __ldg(nbr + (size_t)ld + e));
      double lim[NQ][N1];
#pragma unroll
      for (int k = 0; k < NQ; ++k) {
        double aL[N1], aC[N1], aR[N1];
#pragma unroll
        for (int m = 0; m < N1; ++m) aC[m] = A[k][sl][m][tx];
        const int ph = (METHOD == 1 && phys == 3 && k == 1) ? 5 : phys;
        if (ph == 0) {
#pragma unroll
          for (int m = 0; m < N1; ++m) { aL[m] = A[k][sl][m][tx - 1]; aR[m] = A[k][sl][m][tx + 1]; }
          limit_monomial<P>(aL, aC, aR, lim[k]);
        } else if (ph == 2 || ph == 3) {
          average_monomial<P>(aC, lim[k]);
        } else {
#pragma unroll
          for (int m = 0; m < N1; ++m) lim[k][m] = aC[m];
        }
      }
      if constexpr (METHOD == 1) {
#pragma unroll
        for (int k = 0; k < NQ; ++k) {
          double out[N1];
          to_lag<P>(lim[k], out);
#pragma unroll
          for (int ix = 0; ix < N1; ++ix) XR[slot][k][ix + N1 * sl][tx] = out[ix];
        }
      } else {
        double r_[N1], u_[N1], v_[N1], a_[N1], p_[N1], K[N1], Km[N1], El[N1], E_[N1];
        to_lag<P>(lim[0], r_);
        to_lag<P>(lim[1], u_);
        to_lag<P>(lim[2], v_);
        to_lag<P>(lim[3], a_);
        to_lag<P>(lim[4], p_);
#pragma unroll
        for (int ix = 0; ix < N1; ++ix) K[ix] = 0.5 * (u_[ix] * u_[ix] + v_[ix] * v_[ix]) * __drcp_rn(r_[ix]);
        to_mono<P>(K, Km);
        reconstruct_energy<P>(lim[4], lim[3], Km, Em, El);
        to_lag<P>(El, E_);
#pragma unroll
        for (int ix = 0; ix < N1; ++ix) {
          const int t = ix + N1 * sl;
          XR[slot][0][t][tx] = r_[ix];
          XR[slot][1][t][tx] = u_[ix];
          XR[slot][2][t][tx] = v_[ix];
          XR[slot][3][t][tx] = a_[ix];
          XR[slot][4][t][tx] = p_[ix];
          XR[slot][5][t][tx] = E_[ix];
        }
      }
    }
    __syncthreads();
    // prefetch the next row's raw values while the y pass runs
    if (s <= nrow) {
      e = lane_elem(s + 1);
      if (e >= 0) {
#pragma unroll
        for (int f = 0; f < 5; ++f)
#pragma unroll
          for (int ix = 0; ix < N1; ++ix) v[f][ix] = __ldg(U + (size_t)(f * NS + ix + N1 * sl) * ld + e);
      }
    }
    // ---- y pass of strip row s - 1 (threads: slot, x-column ix = threadIdx.y) ----
    if (s >= 2 && icol) {
      const int ix = sl;
      const int ec = (y0 + s - 2) * nx + ex;
      const int phys = boundary_code(__ldg(nbr + (size_t)2 * ld + ec), __ldg(nbr + (size_t)3 * ld + ec));
      const int cD = (s - 2) % 3, cC = (s - 1) % 3, cU = s % 3;
      double lim[NQ][N1], Emy[N1];
#pragma unroll
      for (int k = 0; k < NQ; ++k) {
        double col[N1], aC[N1];
#pragma unroll
        for (int iy = 0; iy < N1; ++iy) col[iy] = XR[cC][k][ix + N1 * iy][tx];
        to_mono<P>(col, aC);
        const int ph = (METHOD == 1 && phys == 3 && k == 2) ? 5 : phys;
        if (ph == 0) {
          double aD[N1], aU[N1];
#pragma unroll
          for (int iy = 0; iy < N1; ++iy) col[iy] = XR[cD][k][ix + N1 * iy][tx];
          to_mono<P>(col, aD);
#pragma unroll
          for (int iy = 0; iy < N1; ++iy) col[iy] = XR[cU][k][ix + N1 * iy][tx];
          to_mono<P>(col, aU);
          limit_monomial<P>(aD, aC, aU, lim[k]);
        } else if (ph == 2 || ph == 3) {
          average_monomial<P>(aC, lim[k]);
        } else {
#pragma unroll
          for (int m = 0; m < N1; ++m) lim[k][m] = aC[m];
        }
      }
      if constexpr (METHOD == 1) {
#pragma unroll
        for (int k = 0; k < NQ; ++k) {
          double out[N1];
          to_lag<P>(lim[k], out);
#pragma unroll
          for (int iy = 0; iy < N1; ++iy) Uout[(size_t)(k * NS + ix + N1 * iy) * ld + ec] = out[iy];
        }
      } else {
        double col[N1];
#pragma unroll
        for (int iy = 0; iy < N1; ++iy) col[iy] = XR[cC][5][ix + N1 * iy][tx];
        to_mono<P>(col, Emy);
        double r_[N1], u_[N1], v_[N1], a_[N1], K[N1], Km[N1], El[N1], E_[N1];
        to_lag<P>(lim[0], r_);
        to_lag<P>(lim[1], u_);
        to_lag<P>(lim[2], v_);
        to_lag<P>(lim[3], a_);
#pragma unroll
        for (int iy = 0; iy < N1; ++iy) K[iy] = 0.5 * (u_[iy] * u_[iy] + v_[iy] * v_[iy]) * __drcp_rn(r_[iy]);
        to_mono<P>(K, Km);
        reconstruct_energy<P>(lim[4], lim[3], Km, Emy, El);
        to_lag<P>(El, E_);
#pragma unroll
        for (int iy = 0; iy < N1; ++iy) {
          const size_t o = (size_t)(ix + N1 * iy) * ld + ec;
          Uout[o + (size_t)0 * NS * ld] = r_[iy];
          Uout[o + (size_t)1 * NS * ld] = u_[iy];
          Uout[o + (size_t)2 * NS * ld] = v_[iy];
          Uout[o + (size_t)3 * NS * ld] = E_[iy];
          Uout[o + (size_t)4 * NS * ld] = a_[iy];
        }
      }
    }
  }
}

}  // namespace dgb
