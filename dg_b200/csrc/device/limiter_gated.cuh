// Sensor-gated (per-element) limiters and the primitive-variable HR limiter.
//
//   hri  HR on every field of the flagged elements, x slices then y slices, each pass reading the
//        state the previous pass left (Limiting::HRIlimiting, code/src/limiting/limiting.cc:596-625,
//        hri1D limiting_kernels.cu:322-429)
//   m2i  the m2 limiter on the flagged elements, pressure recomputed from each pass's input state
//        (Limiting::M2Ilimiting, limiting.cc:661-690, m2i1D limiting_kernels.cu:431-722)
//   pri  hri on primitive variables (rho, u, [v,] p, alpha); every element goes to primitive
//        variables and back (Limiting::PRIlimiting, limiting.cc:627-659)
//   p0i  flagged elements set to their cell average (Limiting::P0Ilimiting, limiting.cc:692-710,
//        p0i limiting_kernels.cu:723-770)
//   prl  HR limiting of the primitive variables on all elements (Limiting::PRlimiting,
//        limiting.cc:102-121)
// Flags come from the sensor kernels (dgb_sensor.cu).  Unflagged elements are copied unchanged
// (converted, for pri).  One thread per (element, slice); the slice arithmetic is the same scaled
// Taylor-monomial machinery as the global limiters.
#pragma once
#include "kernels.cuh"

namespace dgb {

// gamma-model conserved <-> primitive at one node, in place (Cons2Prim / Prim2Cons,
// limiting_kernels.cu:957-1059): (rho, rho u, [rho v,] E, alpha) <-> (rho, u, [v,] p, alpha)
template <int D>
__device__ __forceinline__ void cons_to_prim(double* q) {
  const double rho = q[0], ru = q[1], rv = D == 2 ? q[2] : 0.0, E = q[D + 1], al = q[D + 2];
  q[1] = ru / rho;
  if (D == 2) q[2] = rv / rho;
  q[D + 1] = (E - 0.5 * (ru * ru + rv * rv) / rho) / al;
}
template <int D>
__device__ __forceinline__ void prim_to_cons(double* q) {
  const double rho = q[0], u = q[1], v = D == 2 ? q[2] : 0.0, p = q[D + 1], al = q[D + 2];
  q[1] = rho * u;
  if (D == 2) q[2] = rho * v;
  q[D + 1] = p * al + 0.5 * rho * (u * u + v * v);
}

// Sparse form (learned indicator): the elements come from a list; pass 0 reads the raw state U and
// writes X for the listed elements only; pass 1 reads X for listed (flagged) elements and the raw
// state `alt` for the others, and writes the listed elements of `out` (= alt): flagged entries of
// alt are written but never read in that pass.
struct GateSparse {
  const int* list = nullptr;
  const int* count = nullptr;
  const unsigned char* flag = nullptr;
  const double* alt = nullptr;
};

// The m2 limiter of one slice of one element for the sensor-gated limiters (M2Ilimiting,
// limiting.cc:661-690, m2i1D limiting_kernels.cu:431-722): pressure recomputed from this pass's
// input state, rho, alpha, p and the momenta limited (the wall-normal momentum of this pass left
// as it is at a wall), total energy rebuilt from the limited p, alpha and kinetic energy.
// c, l, r: the element's and its neighbours' nodal values [field][node] (l, r read only when
// phys == 0).
template <int D, int P, int PASS>
__device__ __forceinline__ void m2i_slice(int phys, const double (&c)[D + 3][P + 1], const double (&l)[D + 3][P + 1],
                                          const double (&r)[D + 3][P + 1], double (&res)[D + 3][P + 1]) {
  constexpr int N1 = P + 1, IE = D + 1, IA = D + 2;
  constexpr int UN = (D == 2 && PASS == 1) ? 2 : 1;  // wall-normal momentum of this pass
  // nodal pressure of the three cells (pressure, limiting_kernels.cu:1870-1897)
  double pc[N1], pl[N1], pr[N1];
  auto press = [&](const double (*v)[N1], double* p) {
#pragma unroll
    for (int k = 0; k < N1; ++k) {
      const double kin = v[1][k] * v[1][k] + (D == 2 ? v[2][k] * v[2][k] : 0.0);
      p[k] = (v[IE][k] - 0.5 * kin * __drcp_rn(v[0][k])) * __drcp_rn(v[IA][k]);  // reciprocals for divisions
    }
  };
  press(c, pc);
  if (phys == 0) {
    press(l, pl);
    press(r, pr);
  }
  double mr[N1], ma[N1], mp[N1];
  limit_slice<P>(phys, l[0], c[0], r[0], mr);
  limit_slice<P>(phys, l[IA], c[IA], r[IA], ma);
  limit_slice<P>(phys, pl, pc, pr, mp);
  to_lag<P>(mr, res[0]);
  to_lag<P>(ma, res[IA]);
#pragma unroll
  for (int f = 1; f <= D; ++f) {
    if (phys == 3 && f == UN) {
#pragma unroll
      for (int k = 0; k < N1; ++k) res[f][k] = c[f][k];
    } else {
      double mm[N1];
      limit_slice<P>(phys, l[f], c[f], r[f], mm);
      to_lag<P>(mm, res[f]);
    }
  }
  // total energy from the limited pressure, 1/(gamma-1) and kinetic energy
  double K[N1], Km[N1], Em[N1], El[N1];
#pragma unroll
  for (int k = 0; k < N1; ++k) {
    const double kin = res[1][k] * res[1][k] + (D == 2 ? res[2][k] * res[2][k] : 0.0);
    K[k] = 0.5 * kin * __drcp_rn(res[0][k]);
  }
  to_mono<P>(K, Km);
  to_mono<P>(c[IE], Em);
  reconstruct_energy<P>(mp, ma, Km, Em, El);
  to_lag<P>(El, res[IE]);
}

// One pass of hri / pri (METHOD 1) or m2i (METHOD 2).  PASS 0: x slices (row iy = blockIdx.y,
// neighbours left/right); PASS 1: y slices (column ix = blockIdx.y, neighbours bottom/top); 1D: the
// element is the slice.  IN_PRIM converts loaded values to primitive variables, OUT_CONS converts
// stored values back.  out must not alias U.
template <int D, int P, int METHOD, int PASS, bool IN_PRIM, bool OUT_CONS, bool SPARSE = false>
__global__ void __launch_bounds__(128) lim_gated_kernel(const LimArgs la, const int* __restrict__ sens,
                                                        const double* U, const int* __restrict__ nbr,
                                                        double* out, const DevScalars* __restrict__ scal,
                                                        const GateSparse sp = GateSparse()) {
  constexpr int N1 = P + 1, NS = D == 2 ? N1 * N1 : N1, NF = D + 3, IE = D + 1, IA = D + 2;
  constexpr int UN = (D == 2 && PASS == 1) ? 2 : 1;  // wall-normal momentum of this pass
  if (scal && scal->flags) return;
  const int ld = la.ld, sl = blockIdx.y;
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (SPARSE) {
    if (e >= *sp.count) return;
    e = sp.list[e];
  } else if (e >= la.n_elem) {
    return;
  }
  auto node = [&](int k) { return D == 1 ? k : (PASS == 0 ? k + N1 * sl : sl + N1 * k); };
  auto load = [&](int el, double (*v)[N1]) {
    const double* src = (SPARSE && PASS == 1 && el != e && !sp.flag[el]) ? sp.alt : U;
#pragma unroll
    for (int k = 0; k < N1; ++k) {
      double q[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) q[f] = src[(size_t)(f * NS + node(k)) * ld + el];
      if (IN_PRIM) cons_to_prim<D>(q);
#pragma unroll
      for (int f = 0; f < NF; ++f) v[f][k] = q[f];
    }
  };
  auto store = [&](double (*v)[N1]) {
#pragma unroll
    for (int k = 0; k < N1; ++k) {
      double q[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) q[f] = v[f][k];
      if (OUT_CONS) prim_to_cons<D>(q);
#pragma unroll
      for (int f = 0; f < NF; ++f) out[(size_t)(f * NS + node(k)) * ld + e] = q[f];
    }
  };
  double c[NF][N1];
  load(e, c);
  if (!SPARSE && !__ldg(sens + e)) {
    store(c);
    return;
  }
  const int o = PASS == 0 ? 0 : 2;
  const int nA = __ldg(nbr + (size_t)o * ld + e), nB = __ldg(nbr + (size_t)(o + 1) * ld + e);
  const int phys = boundary_code(nA, nB);
  if (phys == 4) {  // "leave data unchanged"
    store(c);
    return;
  }
  double l[NF][N1], r[NF][N1];
  if (phys == 0) {
    load(nA, l);
    load(nB, r);
  }
  double res[NF][N1];
  if constexpr (METHOD == 1) {
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      if (phys == 3 && f == UN) {  // the wall-normal momentum is not limited at a wall
#pragma unroll
        for (int k = 0; k < N1; ++k) res[f][k] = c[f][k];
        continue;
      }
      double lim[N1];
      limit_slice<P>(phys, l[f], c[f], r[f], lim);
      to_lag<P>(lim, res[f]);
    }
  } else {
    m2i_slice<D, P, PASS>(phys, c, l, r, res);
  }
  store(res);
}

// Tiled form of the learned indicator's gated m2 limiter on a structured row-major grid (same
// arithmetic as the sparse lim_gated_kernel<2, P, 2, PASS, false, false, true>): a CTA covers the
// tile of the dense tiled limiter pass -- PASS 0: 30 elements of one element row (threads: element
// slot with the left / right neighbour slots, x slice), PASS 1: 32 x 4 elements (threads: x slot,
// row slot with the bottom / top neighbour rows) for one node column `sl`.  Every slot's slice is
// loaded once, coalesced, and shared through shared memory; only the band elements (flag[e] != 0)
// are limited and written, and a tile without band elements is left after one block vote.
// PASS 0 reads the raw state U and writes the band's x-limited slices to X; PASS 1 reads X for band
// elements and U for the others and writes the band's result into U.  Every thread of the CTA runs
// both of the tile's barriers (the vote and the shared-slice barrier), so a CTA can run the tiles of
// a list one after another on the same shared memory.
constexpr int GATED_TW0 = 30, GATED_TW1 = 32, GATED_TH1 = 4;  // x-pass tile width, y-pass tile

template <int P, int PASS>
__device__ __forceinline__ void lim_gated_tile(const LimArgs& la, int nx, int ny, double* __restrict__ U,
                                               double* __restrict__ X, const int* __restrict__ nbr,
                                               const unsigned char* __restrict__ flag, int bxi, int byi, int slc,
                                               double (&V)[5][P + 1][PASS == 0 ? P + 1 : 6][32]) {
  constexpr int N1 = P + 1, NS = N1 * N1, NF = 5, TWI = GATED_TW0, THI = GATED_TH1;
  const int ld = la.ld, tx = threadIdx.x, ty = threadIdx.y;
  int e = -1;
  bool interior;
  int sl;  // the slice this thread's values belong to: x slice (PASS 0) or node column (PASS 1)
  if (PASS == 0) {
    const int x0 = bxi * TWI, ey = byi, ex = x0 - 1 + tx;
    sl = ty;
    interior = tx >= 1 && tx <= TWI && ex < nx;
    if (interior) e = ey * nx + ex;
    else if (tx == 0) e = __ldg(nbr + (size_t)0 * ld + ey * nx + x0);
    else if (ex - 1 < nx && ex - 1 >= 0) e = __ldg(nbr + (size_t)1 * ld + ey * nx + ex - 1);
  } else {
    const int x0 = bxi * GATED_TW1, y0 = byi * THI, x = x0 + tx, yy = y0 - 1 + ty;
    sl = slc;
    interior = ty >= 1 && ty <= THI && yy < ny && x < nx;
    if (x < nx) {
      if (interior) e = yy * nx + x;
      else if (ty == 0) e = __ldg(nbr + (size_t)2 * ld + y0 * nx + x);
      else if (yy - 1 < ny && yy - 1 >= 0) e = __ldg(nbr + (size_t)3 * ld + (yy - 1) * nx + x);
    }
  }
  const bool mine = interior && __ldg(flag + e) != 0;
  if (!__syncthreads_or(mine)) return;  // no band element in this tile
  auto node = [&](int k) { return PASS == 0 ? k + N1 * sl : sl + N1 * k; };
  if (e >= 0) {
    const double* src = (PASS == 1 && __ldg(flag + e)) ? X : U;
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int k = 0; k < N1; ++k) V[f][k][ty][tx] = src[(size_t)(f * NS + node(k)) * ld + e];
  }
  __syncthreads();
  if (!mine) return;
  const int o = PASS == 0 ? 0 : 2;
  const int phys = boundary_code(__ldg(nbr + (size_t)o * ld + e), __ldg(nbr + (size_t)(o + 1) * ld + e));
  double c[NF][N1], l[NF][N1], r[NF][N1], res[NF][N1];
  const int lx = PASS == 0 ? tx - 1 : tx, ly = PASS == 0 ? ty : ty - 1;
  const int rx = PASS == 0 ? tx + 1 : tx, ry = PASS == 0 ? ty : ty + 1;
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int k = 0; k < N1; ++k) {
      c[f][k] = V[f][k][ty][tx];
      l[f][k] = V[f][k][ly][lx];
      r[f][k] = V[f][k][ry][rx];
    }
  double* out = PASS == 0 ? X : U;
  if (phys == 4) {  // "leave data unchanged"
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int k = 0; k < N1; ++k) out[(size_t)(f * NS + node(k)) * ld + e] = c[f][k];
    return;
  }
  m2i_slice<2, P, PASS>(phys, c, l, r, res);
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int k = 0; k < N1; ++k) out[(size_t)(f * NS + node(k)) * ld + e] = res[f][k];
}

// The gated pass over a list of its tiles that hold band elements (built with the band,
// gated_tile_list_kernel), by persistent CTAs: CTA b takes list entries b, b + gridDim.x, ... (tile
// index = tile row * tiles per row + tile column); for PASS 1 blockIdx.z is the node column.  Tiles
// without band elements are not visited at all.
template <int P, int PASS>
__global__ void __launch_bounds__(PASS == 0 ? 32 * (P + 1) : 32 * 6)
    lim_gated_tile_list_kernel(const LimArgs la, int nx, int ny, double* __restrict__ U, double* __restrict__ X,
                               const int* __restrict__ nbr, const unsigned char* __restrict__ flag,
                               const int* __restrict__ tiles, const int* __restrict__ count,
                               const DevScalars* __restrict__ scal) {
  __shared__ double V[5][P + 1][PASS == 0 ? P + 1 : 6][32];
  if (scal && scal->flags) return;
  const int ntx = PASS == 0 ? (nx + GATED_TW0 - 1) / GATED_TW0 : (nx + GATED_TW1 - 1) / GATED_TW1;
  const int n = *count;
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const int t = tiles[i];
    lim_gated_tile<P, PASS>(la, nx, ny, U, X, nbr, flag, t % ntx, t / ntx, blockIdx.z, V);
  }
}

// the tiles of both gated passes that hold band elements, as two lists (order immaterial): thread
// t < n0 checks x-pass tile t (30 elements of one row), thread n0 + t checks y-pass tile t (32 x 4)
static __global__ void __launch_bounds__(256) gated_tile_list_kernel(int nx, int ny, const unsigned char* __restrict__ band,
                                                              int* __restrict__ list0, int* __restrict__ count0,
                                                              int* __restrict__ list1, int* __restrict__ count1,
                                                              const DevScalars* __restrict__ scal) {
  if (scal && scal->flags) return;
  const int ntx0 = (nx + GATED_TW0 - 1) / GATED_TW0, n0 = ntx0 * ny;
  const int ntx1 = (nx + GATED_TW1 - 1) / GATED_TW1, n1 = ntx1 * ((ny + GATED_TH1 - 1) / GATED_TH1);
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  bool any = false;
  int* list = list0;
  int* count = count0;
  int t = k;
  if (k < n0) {
    const int x0 = (k % ntx0) * GATED_TW0, y = k / ntx0;
    for (int x = x0; x < min(x0 + GATED_TW0, nx) && !any; ++x) any = band[(size_t)y * nx + x] != 0;
  } else if (k < n0 + n1) {
    t = k - n0;
    list = list1;
    count = count1;
    const int x0 = (t % ntx1) * GATED_TW1, y0 = (t / ntx1) * GATED_TH1;
    for (int y = y0; y < min(y0 + GATED_TH1, ny) && !any; ++y)
      for (int x = x0; x < min(x0 + GATED_TW1, nx) && !any; ++x) any = band[(size_t)y * nx + x] != 0;
  }
  if (any) list[atomicAdd(count, 1)] = t;
}

// p0i: flagged elements to their cell average sum_t w_t U_t (w from phi_w / |reference element|)
struct CellAverageWeights {
  double w[16];
};
template <int NS, int NF>
__global__ void __launch_bounds__(128) p0i_kernel(const LimArgs la, const int* __restrict__ sens,
                                                  const CellAverageWeights wt, double* __restrict__ U,
                                                  const DevScalars* __restrict__ scal) {
  if (scal && scal->flags) return;
  const int ld = la.ld, e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= la.n_elem || !__ldg(sens + e)) return;
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    double s = 0.0;
#pragma unroll
    for (int t = 0; t < NS; ++t) s += wt.w[t] * U[(size_t)(f * NS + t) * ld + e];
#pragma unroll
    for (int t = 0; t < NS; ++t) U[(size_t)(f * NS + t) * ld + e] = s;
  }
}

// prl: all elements to primitive variables (TO_PRIM) or back, in place
template <int D, int NS, bool TO_PRIM>
__global__ void __launch_bounds__(256) convert_state_kernel(const LimArgs la, double* __restrict__ U,
                                                            const DevScalars* __restrict__ scal) {
  constexpr int NF = D + 3;
  if (scal && scal->flags) return;
  const int ld = la.ld, e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= la.n_elem) return;
#pragma unroll
  for (int t = 0; t < NS; ++t) {
    double q[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) q[f] = U[(size_t)(f * NS + t) * ld + e];
    if (TO_PRIM) cons_to_prim<D>(q);
    else prim_to_cons<D>(q);
#pragma unroll
    for (int f = 0; f < NF; ++f) U[(size_t)(f * NS + t) * ld + e] = q[f];
  }
}

}  // namespace dgb
