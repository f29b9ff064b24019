// Device context and the device half of the C ABI (include/dgb.h).
//
// One context = one problem on one GPU: uploaded basis constants and neighbour table, the
// resident state and the stage buffers of the chosen integrator, and one CUDA stream on which
// every kernel of the context runs.  Steps of dgb_advance are captured once into a CUDA graph
// per (scheme, step mode) and replayed.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/dgb.h"
#include "device/kernels.cuh"
#include "device/tile2d.cuh"
#include "device/tile2d_dmma.cuh"
#include "device/limiter2d_tile.cuh"
#include "device/limiter_gated.cuh"
#include "device/tile2d_mixed.cuh"
#include "device/learned.cuh"
#include "device/learned_tc.cuh"
#include "device/tables.cuh"
#include "device/sensor.h"
#include "launch.h"

namespace dgb {
// 4 to 10 mass fractions (dgb_device_ny.cu)
int residual1d_many_y(dgb_ctx* c, const StageArgs& a, int mode);
int limit1d_many_y(dgb_ctx* c, const double* in, double* out);
int residual2d_many_y(dgb_ctx* c, const StageArgs& a, int mode);
int limit2d_many_y(dgb_ctx* c, double* U);
int upload_many_y_tables(const Consts& cs, int D, int p);
}  // namespace dgb
#include "host/host.h"
#include "ctx.h"

namespace dgb {
int set_error(int code, const std::string& msg);
}
const dgb::Problem& dgb_problem_ref(const dgb_problem* p);

using namespace dgb;

#define DGB_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t err_ = (call);                                                                  \
    if (err_ != cudaSuccess)                                                                    \
      return set_error(DGB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(err_));     \
  } while (0)

namespace {


double fact(int n) { double f = 1; for (int i = 2; i <= n; ++i) f *= i; return f; }

Consts make_consts(const Problem& P, int ld) {
  Consts c;
  std::memset(&c, 0, sizeof(c));
  c.p = P.p;
  c.n1 = P.p + 1;
  c.dim = P.D;
  c.ng1 = P.D == 1 ? P.p + 1 : (P.p == 1 ? 2 : P.p + 2);
  c.ns = P.N_s;
  c.ng = P.N_G;
  c.nf = P.N_F;
  c.ld = ld;
  c.n_elem = P.N_E;
  const int n1 = c.n1;
  // ascending 1D nodes (tensor order)
  std::vector<double> xs(n1);
  for (int i = 0; i < n1; ++i) xs[i] = -1.0 + 2.0 * i / P.p;
  std::vector<double> xq, wq, xf, wf;
  gauss_legendre(c.ng1, xq, wq);
  gauss_legendre(n1, xf, wf);
  for (int g = 0; g < c.ng1; ++g) {
    c.wq[g] = wq[g];
    for (int i = 0; i < n1; ++i) { c.Bq[g][i] = lagrange1d(xs, i, xq[g]); c.Dq[g][i] = dlagrange1d(xs, i, xq[g]); }
  }
  for (int g = 0; g < n1; ++g) {
    c.wf[g] = wf[g];
    for (int i = 0; i < n1; ++i) c.Bf[g][i] = lagrange1d(xs, i, xf[g]);
  }
  // element inverse mass matrix (element 0; uniform mesh) permuted to tensor order
  for (int t = 0; t < P.N_s; ++t)
    for (int u = 0; u < P.N_s; ++u) c.Minv[t][u] = P.Minv[(size_t)P.tensor_perm[u] * P.N_s + P.tensor_perm[t]];
  // Lagrange -> scaled Taylor monomials: T = V^-1 phi on the (p+1) Gauss points
  // (monovandermonde1d and Lag2Mono of main.cc:558-567, 1146-1157)
  std::vector<double> V((size_t)n1 * n1), phi1((size_t)n1 * n1);
  for (int g = 0; g < n1; ++g)
    for (int j = 0; j < n1; ++j) {
      V[g + (size_t)j * n1] = std::pow(xf[g], j) / fact(j);
      phi1[g + (size_t)j * n1] = lagrange1d(xs, j, xf[g]);
    }
  invert(V, n1);
  std::vector<double> T((size_t)n1 * n1, 0.0);
  for (int m = 0; m < n1; ++m)
    for (int i = 0; i < n1; ++i) {
      double s = 0;
      for (int g = 0; g < n1; ++g) s += V[m + (size_t)g * n1] * phi1[g + (size_t)i * n1];
      T[m + (size_t)i * n1] = s;
    }
  std::vector<double> Ti = T;
  invert(Ti, n1);
  for (int m = 0; m < n1; ++m)
    for (int i = 0; i < n1; ++i) { c.T[m][i] = T[m + (size_t)i * n1]; c.Tinv[i][m] = Ti[i + (size_t)m * n1]; }
  // limiter integrals (integrate_monomial_derivative(_bounds), limiting_kernels.cu:1748-1775)
  for (int k = 0; k < MAXN; ++k)
    for (int n = 0; n < MAXN; ++n) {
      const int num = n - k + 1;
      if (num < 1) continue;
      c.imd[k][n] = (num % 2) ? 2.0 / fact(num) : 0.0;
      c.imdL[k][n] = (std::pow(-1.0, num) - std::pow(-3.0, num)) / fact(num);
      c.imdR[k][n] = (std::pow(3.0, num) - std::pow(1.0, num)) / fact(num);
    }
  for (int k = 0; k < 8; ++k) c.ifact[k] = 1.0 / fact(k);
  const int D = P.D, NG = P.N_G;
  c.J = P.J[0];
  c.ixx = P.invJac[((size_t)0 * NG + 0) * D * D + 0];
  c.iyy = D == 2 ? P.invJac[((size_t)0 * NG + 0) * D * D + 3] : 0.0;
  c.JFx = D == 2 ? 0.5 * P.hy : 1.0;
  c.JFy = D == 2 ? 0.5 * P.hx : 1.0;
  c.cfl_scaled = P.cfl_scaled;
  return c;
}

// structured row-major grid test: interior neighbours are e-1, e+1, e-nx, e+nx
// the neighbours of element e are e - 1 and e + 1 (at the ends: a boundary code, or the other end)
bool is_chain_1d(const Problem& P) {
  if (P.D != 1 || P.N_E < 2) return false;
  const int ne = P.N_E;
  for (int e = 0; e < ne; ++e) {
    const int L = P.nbr[e], R = P.nbr[(size_t)ne + e];
    if (e > 0 ? L != e - 1 : !(L < 0 || L == ne - 1)) return false;
    if (e < ne - 1 ? R != e + 1 : !(R < 0 || R == 0)) return false;
  }
  return true;
}

bool is_row_major_grid(const Problem& P) {
  if (P.D != 2 || P.nx <= 0 || P.ny <= 0 || (long)P.nx * P.ny != P.N_E) return false;
  const int nx = P.nx, ne = P.N_E;
  for (int e = 0; e < ne; ++e) {
    const int ix = e % nx, iy = e / nx;
    const int L = P.nbr[(size_t)0 * ne + e], R = P.nbr[(size_t)1 * ne + e];
    const int Dn = P.nbr[(size_t)2 * ne + e], Up = P.nbr[(size_t)3 * ne + e];
    if (ix > 0 && L != e - 1) return false;
    if (ix < nx - 1 && R != e + 1) return false;
    if (iy > 0 && Dn != e - nx) return false;
    if (iy < P.ny - 1 && Up != e + nx) return false;
  }
  return true;
}

}  // namespace


namespace {



template <int P, int FLUX, int MODE, int NY = 0, bool GC = false>
void launch_res1d(dgb_ctx* c, const StageArgs& a) {
  const int grid = (c->ne + 127) / 128;
  ProfScope ps(c, KC_RESIDUAL);
  residual1d_kernel<P, FLUX, MODE, NY, GC><<<grid, 128, 0, c->st>>>(c->cs, a);
}

template <int P, int FLUX, int MODE>
void launch_tile2d_mixed(dgb_ctx* c, const StageArgs& s) {
  constexpr int TH = tile_h_for(P);
  if (c->mixed_ct) {
    constexpr size_t smem = TileDimsMixedCT<P, TILE_W, TH>::smem_bytes;
    auto k = residual2d_tile_mixed_ct_kernel<P, FLUX, MODE, TILE_W, TH>;
    allow_dynamic_smem(k, smem);
    const TileArgs a = tile_args(c, s);
    dim3 grid(c->nx / TILE_W, c->ny / TH);
    ProfScope ps(c, KC_RESIDUAL);
    launch_pdl(c, k, grid, dim3(TILE_W * TH), smem, a);
    return;
  }
  constexpr size_t smem = TileDimsMixed<P, TILE_W, TH>::smem_bytes;
  auto k = residual2d_tile_mixed_kernel<P, FLUX, MODE, TILE_W, TH>;
  allow_dynamic_smem(k, smem);
  const TileArgs a = tile_args(c, s);
  const CUtensorMap& mb = MODE == MODE_SSP ? map_of(c, s.Ubase)
                          : MODE == MODE_RK4 && s.Uacc ? map_of(c, s.Uacc) : map_of(c, s.U);
  dim3 grid(c->nx / TILE_W, c->ny / TH);
  ProfScope ps(c, KC_RESIDUAL);
  launch_pdl(c, k, grid, dim3(TILE_W * TH), smem, a, map_of(c, s.U), mb);
}

// p = 2 FP64 stage on the FP64 tensor cores (tile2d_dmma.cuh): same tiles and tensor map
template <int FLUX, int MODE>
void launch_tile2d_dmma(dgb_ctx* c, const StageArgs& s) {
  constexpr size_t smem = DmmaDims::smem_bytes;
  auto k = residual2d_tile_dmma_kernel<FLUX, MODE>;
  allow_dynamic_smem(k, smem);
  const TileArgs a = tile_args(c, s);
  dim3 grid(c->nx / DMMA_TW, c->ny / DMMA_TH);
  ProfScope ps(c, KC_RESIDUAL);
  k<<<grid, DMMA_THREADS, smem, c->st>>>(a, map_of(c, s.U));
}

}  // namespace

// TMA descriptor of a state buffer viewed as (x: nx, y: ny, z: N_F*N_s rows of stride ld), box
// tw x th x N_F*N_s
bool dgb::encode_state_map(dgb_ctx* c, double* ptr, CUtensorMap* map, int tw, int th) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return false;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t dims[3] = {(cuuint64_t)c->nx, (cuuint64_t)c->ny, (cuuint64_t)(c->nf * c->ns)};
  const cuuint64_t strides[2] = {(cuuint64_t)c->nx * sizeof(double), (cuuint64_t)c->ld * sizeof(double)};
  const cuuint32_t box[3] = {(cuuint32_t)tw, (cuuint32_t)th, (cuuint32_t)(c->nf * c->ns)};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, ptr, dims, strides, box, estr,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

namespace {

// NY passive mass fractions (1D or tiled 2D, FP64 form; checked at create)
template <int MODE, int NY>
int residual_ny(dgb_ctx* c, const StageArgs& a) {
  if (c->tile_tma) {  // full tiles, then the strips outside them (if any) with the generic kernel
#define T2Y(P, F)                                                               \
  case P * 10 + F:                                                              \
    launch_tile2d<P, F, MODE, NY>(c, a);                                        \
    if (c->nleft) launch_res2d<P, F, MODE, NY>(c, a, c->left, c->nleft);        \
    return 0;
    switch (c->p * 10 + c->flux) {
      T2Y(1, 0) T2Y(1, 2) T2Y(2, 0) T2Y(2, 2) T2Y(3, 0) T2Y(3, 2)
      default: return set_error(DGB_ERR_UNSUPPORTED, "no residual kernel for this (p, flux) with mass fractions");
    }
#undef T2Y
  }
  if (c->D == 1) {
#define R1Y(P, F) case P * 10 + F: launch_res1d<P, F, MODE, NY>(c, a); return 0;
    switch (c->p * 10 + c->flux) {
      R1Y(1, 0) R1Y(1, 1) R1Y(1, 2) R1Y(2, 0) R1Y(2, 1) R1Y(2, 2) R1Y(3, 0) R1Y(3, 1) R1Y(3, 2)
      default: break;
    }
#undef R1Y
  }
  return set_error(DGB_ERR_UNSUPPORTED, "no residual kernel for this (p, flux) with mass fractions");
}

// the full tiles with the tiled kernel, then the elements outside them (right and top strips of a
// grid whose extents are not tile multiples) with the generic kernel; disjoint outputs, both read
// the stage input's neighbours from global memory
template <int P, int FLUX, int MODE>
int tiles_then_strips(dgb_ctx* c, const StageArgs& a) {
  if constexpr (P == 2 && MODE != MODE_RESIDUAL) {
    if (c->tile_tma && c->tile_dmma) {
      launch_tile2d_dmma<FLUX, MODE>(c, a);
      if (c->nleft) launch_res2d<P, FLUX, MODE>(c, a, c->left, c->nleft);
      return 0;
    }
  }
  if (c->tile_tma) launch_tile2d<P, FLUX, MODE>(c, a);
  else launch_tile2d<P, FLUX, MODE, 0, false, false>(c, a);
  if (c->nleft) launch_res2d<P, FLUX, MODE>(c, a, c->left, c->nleft);
  return 0;
}

template <int MODE>
int residual_dispatch(dgb_ctx* c, const StageArgs& a) {
  if (c->tile_tma && c->form == DGB_FORM_MIXED) {
    // mixed full tiles; the strips outside them (if any) in the plain FP64 form
    const int key = c->p * 10 + c->flux;
    switch (key) {
      case 10: launch_tile2d_mixed<1, 0, MODE>(c, a); if (c->nleft) launch_res2d<1, 0, MODE>(c, a, c->left, c->nleft); return 0;
      case 12: launch_tile2d_mixed<1, 2, MODE>(c, a); if (c->nleft) launch_res2d<1, 2, MODE>(c, a, c->left, c->nleft); return 0;
      case 20: launch_tile2d_mixed<2, 0, MODE>(c, a); if (c->nleft) launch_res2d<2, 0, MODE>(c, a, c->left, c->nleft); return 0;
      case 22: launch_tile2d_mixed<2, 2, MODE>(c, a); if (c->nleft) launch_res2d<2, 2, MODE>(c, a, c->left, c->nleft); return 0;
      case 30: launch_tile2d_mixed<3, 0, MODE>(c, a); if (c->nleft) launch_res2d<3, 0, MODE>(c, a, c->left, c->nleft); return 0;
      case 32: launch_tile2d_mixed<3, 2, MODE>(c, a); if (c->nleft) launch_res2d<3, 2, MODE>(c, a, c->left, c->nleft); return 0;
      default: return set_error(DGB_ERR_UNSUPPORTED, "mixed form: p = 1..3 with Rusanov or Roe");
    }
  }
  if (c->gamcons) {  // GAMCONS: tiled 2D or 1D, FP64 form, no mass fractions (checked at create)
    if (c->D == 2) {  // full tiles, then the strips outside them (if any) with the generic kernel
#define T2G(P, F)                                                               \
  case P * 10 + F:                                                              \
    launch_tile2d<P, F, MODE, 0, true>(c, a);                                   \
    if (c->nleft) launch_res2d<P, F, MODE, 0, true>(c, a, c->left, c->nleft);   \
    return 0;
      switch (c->p * 10 + c->flux) {
        T2G(1, 0) T2G(1, 2) T2G(2, 0) T2G(2, 2) T2G(3, 0) T2G(3, 2)
        default: return set_error(DGB_ERR_UNSUPPORTED, "no GAMCONS residual kernel for this (p, flux)");
      }
#undef T2G
    }
#define R1G(P, F) case P * 10 + F: launch_res1d<P, F, MODE, 0, true>(c, a); return 0;
    switch (c->p * 10 + c->flux) {
      R1G(1, 0) R1G(1, 1) R1G(1, 2) R1G(2, 0) R1G(2, 1) R1G(2, 2) R1G(3, 0) R1G(3, 1) R1G(3, 2)
      default: return set_error(DGB_ERR_UNSUPPORTED, "no GAMCONS residual kernel for this (p, flux)");
    }
#undef R1G
  }
  if (c->nmass > 0) {
    switch (c->nmass) {
      case 1: return residual_ny<MODE, 1>(c, a);
      case 2: return residual_ny<MODE, 2>(c, a);
      case 3: return residual_ny<MODE, 3>(c, a);
      default: return c->D == 1 ? residual1d_many_y(c, a, MODE) : residual2d_many_y(c, a, MODE);
    }
  }
  if (c->tiled) {
    const int key = c->p * 10 + c->flux;
    switch (key) {
      case 10: return tiles_then_strips<1, 0, MODE>(c, a);
      case 12: return tiles_then_strips<1, 2, MODE>(c, a);
      case 20: return tiles_then_strips<2, 0, MODE>(c, a);
      case 22: return tiles_then_strips<2, 2, MODE>(c, a);
      case 30: return tiles_then_strips<3, 0, MODE>(c, a);
      case 32: return tiles_then_strips<3, 2, MODE>(c, a);
      default: break;
    }
  }
#define R2(P, F) case P * 10 + F: launch_res2d<P, F, MODE>(c, a); return 0;
#define R1(P, F) case P * 10 + F: launch_res1d<P, F, MODE>(c, a); return 0;
  const int key = c->p * 10 + c->flux;
  if (c->D == 2) {
    switch (key) {
      R2(1, 0) R2(1, 2) R2(2, 0) R2(2, 2) R2(3, 0) R2(3, 2)
      default: break;
    }
  } else {
    switch (key) {
      R1(1, 0) R1(1, 1) R1(1, 2) R1(2, 0) R1(2, 1) R1(2, 2) R1(3, 0) R1(3, 1) R1(3, 2)
      default: break;
    }
  }
#undef R2
#undef R1
  return set_error(DGB_ERR_UNSUPPORTED, "no residual kernel for this (dim, p, flux)");
}

constexpr int LIM_STRIP_H = 8;

// fused x+y limiter on a row-major grid, out of place (in != out)
template <int P, int METHOD>
void launch_lim2d_fused(dgb_ctx* c, const double* in, double* out) {
  ProfScope ps(c, KC_LIMITER);
  const LimArgs la{c->ld, c->ne};
  constexpr size_t smem = lim2d_fused_smem_bytes<P, METHOD>();
  auto k = lim2d_fused_tile_kernel<P, METHOD, LIM_STRIP_H>;
  allow_dynamic_smem(k, smem);
  dim3 grid((c->nx + 29) / 30, (c->ny + LIM_STRIP_H - 1) / LIM_STRIP_H), block(32, P + 1);
  k<<<grid, block, smem, c->st>>>(la, c->nx, c->ny, in, c->nbr, out, c->scal);
}

template <int P, int METHOD, int NY = 0>
void launch_lim2d(dgb_ctx* c, double* U) {
  if (NY == 0 && c->fused_lim) {
    cudaMemcpyAsync(c->X, U, c->nstate * sizeof(double), cudaMemcpyDeviceToDevice, c->st);
    launch_lim2d_fused<P, METHOD>(c, c->X, U);
    return;
  }
  ProfScope ps(c, KC_LIMITER);
  const LimArgs la{c->ld, c->ne};
  if (c->rowmajor) {
    dim3 gx((c->nx + 29) / 30, c->ny), bx(32, P + 1);
    launch_pdl(c, lim2d_xpass_tile_kernel<P, METHOD, NY>, gx, bx, 0, la, c->nx, (const double*)U,
               (const int*)c->nbr, c->X, (const DevScalars*)c->scal);
    dim3 gy((c->nx + 31) / 32, (c->ny + 3) / 4, P + 1), by(32, 6);
    launch_pdl(c, lim2d_ypass_tile_kernel<P, METHOD, NY>, gy, by, 0, la, c->nx, c->ny, (const double*)c->X,
               (const int*)c->nbr, U, (const DevScalars*)c->scal);
  } else if (NY == 0) {
    dim3 grid((c->ne + 127) / 128, P + 1);
    lim2d_xpass_kernel<P, METHOD><<<grid, 128, 0, c->st>>>(la, U, c->nbr, c->X, c->scal);
    lim2d_ypass_kernel<P, METHOD><<<grid, 128, 0, c->st>>>(la, c->X, c->nbr, U, c->scal);
  }
  c->counter++;
}

template <int P, int METHOD, int NY = 0>
void launch_lim1d(dgb_ctx* c, double* U) {
  const int grid = (c->ne + 127) / 128;
  {
    ProfScope ps(c, KC_LIMITER);
    const LimArgs la{c->ld, c->ne};
    lim1d_kernel<P, METHOD, NY><<<grid, 128, 0, c->st>>>(la, U, c->nbr, c->X, c->scal);
  }
  cudaMemcpyAsync(U, c->X, c->nstate * sizeof(double), cudaMemcpyDeviceToDevice, c->st);
}

// sensor-gated limiters: sensors on U, then the per-element passes (U -> X -> U in 2D)
template <int D, int P>
int launch_gated(dgb_ctx* c, double* U) {
  ProfScope ps(c, KC_LIMITER);
  SensorLaunch s = c->sl;
  s.U = U;
  if (int rc = launch_sensors(s, c->st)) return set_error(DGB_ERR_CUDA, std::string("sensors: ") + cudaGetErrorString((cudaError_t)rc));
  c->counter += 5;
  const LimArgs la{c->ld, c->ne};
  const int* sens = s.sens;
  const int g = (c->ne + 127) / 128;
  if (c->limiter == DGB_LIM_P0I) {
    p0i_kernel<(D == 2 ? (P + 1) * (P + 1) : P + 1), D + 3><<<g, 128, 0, c->st>>>(la, sens, c->p0w, U, c->scal);
    return 0;
  }
  const bool pri = c->limiter == DGB_LIM_PRI;
  if (D == 2) {
    dim3 grid(g, P + 1);
    if (c->limiter == DGB_LIM_M2I) {
      lim_gated_kernel<2, P, 2, 0, false, false><<<grid, 128, 0, c->st>>>(la, sens, U, c->nbr, c->X, c->scal);
      lim_gated_kernel<2, P, 2, 1, false, false><<<grid, 128, 0, c->st>>>(la, sens, c->X, c->nbr, U, c->scal);
    } else if (pri) {
      lim_gated_kernel<2, P, 1, 0, true, false><<<grid, 128, 0, c->st>>>(la, sens, U, c->nbr, c->X, c->scal);
      lim_gated_kernel<2, P, 1, 1, false, true><<<grid, 128, 0, c->st>>>(la, sens, c->X, c->nbr, U, c->scal);
    } else {
      lim_gated_kernel<2, P, 1, 0, false, false><<<grid, 128, 0, c->st>>>(la, sens, U, c->nbr, c->X, c->scal);
      lim_gated_kernel<2, P, 1, 1, false, false><<<grid, 128, 0, c->st>>>(la, sens, c->X, c->nbr, U, c->scal);
    }
    c->counter += 1;
  } else {
    if (c->limiter == DGB_LIM_M2I)
      lim_gated_kernel<1, P, 2, 0, false, false><<<g, 128, 0, c->st>>>(la, sens, U, c->nbr, c->X, c->scal);
    else if (pri)
      lim_gated_kernel<1, P, 1, 0, true, true><<<g, 128, 0, c->st>>>(la, sens, U, c->nbr, c->X, c->scal);
    else
      lim_gated_kernel<1, P, 1, 0, false, false><<<g, 128, 0, c->st>>>(la, sens, U, c->nbr, c->X, c->scal);
    cudaMemcpyAsync(U, c->X, c->nstate * sizeof(double), cudaMemcpyDeviceToDevice, c->st);
  }
  return 0;
}

// prl: HR of the primitive variables (all elements converted there and back)
template <int D, int P>
void launch_prl(dgb_ctx* c, double* U) {
  constexpr int NS = D == 2 ? (P + 1) * (P + 1) : P + 1;
  const LimArgs la{c->ld, c->ne};
  const int g = (c->ne + 255) / 256;
  {
    ProfScope ps(c, KC_LIMITER);
    convert_state_kernel<D, NS, true><<<g, 256, 0, c->st>>>(la, U, c->scal);
  }
  if (D == 2) launch_lim2d<P, 1>(c, U);
  else launch_lim1d<P, 1>(c, U);
  {
    ProfScope ps(c, KC_LIMITER);
    convert_state_kernel<D, NS, false><<<g, 256, 0, c->st>>>(la, U, c->scal);
  }
}

// out-of-place fused limiting (row-major grids, hrl / m2l): in -> out, in != out
int limit_to(dgb_ctx* c, const double* in, double* out) {
  const int key = c->p * 10 + c->limiter;
  switch (key) {
    case 11: launch_lim2d_fused<1, 1>(c, in, out); return 0;
    case 12: launch_lim2d_fused<1, 2>(c, in, out); return 0;
    case 21: launch_lim2d_fused<2, 1>(c, in, out); return 0;
    case 22: launch_lim2d_fused<2, 2>(c, in, out); return 0;
    case 31: launch_lim2d_fused<3, 1>(c, in, out); return 0;
    case 32: launch_lim2d_fused<3, 2>(c, in, out); return 0;
    default: return set_error(DGB_ERR_UNSUPPORTED, "fused limiter: hrl / m2l, p = 1..3");
  }
}

// learned indicator: scores and flags of U (modes, then the BF16 tensor-core MLP), then the band
// (flagged elements and their face neighbours) that the sparse limiter works on
void launch_indicator(dgb_ctx* c, const double* U) {
  ProfScope ps(c, KC_INDICATOR);
  indicator_modes_kernel<2><<<(c->ne + 127) / 128, 128, 0, c->st>>>(U, c->ld, c->ne, c->ind_modes);
  cudaMemsetAsync(c->ind_list + c->ld, 0, sizeof(int), c->st);
  IndicatorArgs a;
  a.n_elem = c->ne; a.ld = c->ld; a.threshold = c->ind_threshold; a.nbr = c->nbr; a.modes = c->ind_modes;
  a.w1 = c->ind_w; a.w2 = c->ind_w + MLP_H * IND_KPAD; a.vec = c->ind_vec;
  a.score = c->ind_score; a.flag = c->ind_flag; a.list = c->ind_list; a.count = c->ind_list + c->ld; a.scal = c->scal;
  a.errflag = &c->scal->flags;
  if (c->ind_tc) {
    // tcgen05 GEMMs on 128-element tiles, persistent: one CTA per SM
    allow_dynamic_smem(indicator_infer_tc_kernel, TCI_SMEM_BYTES);
    const int ntiles = (c->ne + TCI_M - 1) / TCI_M;
    indicator_infer_tc_kernel<<<std::min(ntiles, c->sm_count), TCI_THREADS, TCI_SMEM_BYTES, c->st>>>(a);
  } else {
    const int ntiles = (c->ne + 15) / 16;
    const int grid = std::min((ntiles + IND_WARPS - 1) / IND_WARPS, c->sm_count * 2);  // persistent: 2 CTAs per SM
    allow_dynamic_smem(indicator_infer_kernel, IND_SMEM_BYTES);
    indicator_infer_kernel<<<grid, 32 * IND_WARPS, IND_SMEM_BYTES, c->st>>>(a);
  }
  cudaMemsetAsync(c->ind_blist + c->ld, 0, sizeof(int), c->st);
  indicator_band_kernel<<<(c->ne + 255) / 256, 256, 0, c->st>>>(c->ne, c->ld, 4, c->nbr, c->ind_flag, c->ind_band,
                                                                c->ind_blist, c->ind_blist + c->ld, c->scal);
  c->counter += 2;  // three kernels (the scope counted one)
  if (c->ind_tiles) {
    // the gated passes' tiles that hold band elements
    int* l0 = c->ind_tiles;
    int* l1 = l0 + c->ind_n0;
    int* cnt = l1 + c->ind_n1;
    cudaMemsetAsync(cnt, 0, 2 * sizeof(int), c->st);
    gated_tile_list_kernel<<<(c->ind_n0 + c->ind_n1 + 255) / 256, 256, 0, c->st>>>(c->nx, c->ny, c->ind_band, l0, cnt,
                                                                                   l1, cnt + 1, c->scal);
    c->counter += 1;
  }
}

// learned-indicator-gated m2 limiter (m2i arithmetic on the band only), in place; score = false
// reuses the band of the last scoring (the time steppers score every ind_every steps).  Structured
// row-major grids: the tiled passes, which skip tiles without band elements; otherwise the passes
// over the band's element list.
void launch_learned_limiter(dgb_ctx* c, double* U, bool score) {
  if (score) launch_indicator(c, U);
  ProfScope ps(c, KC_LIMITER);
  const LimArgs la{c->ld, c->ne};
  if (c->rowmajor) {
    // persistent CTAs over the lists of tiles with band elements (built with the band): the tiles
    // without any are not launched at all
    const int* l0 = c->ind_tiles;
    const int* l1 = l0 + c->ind_n0;
    const int* cnt = l1 + c->ind_n1;
    dim3 gx(std::min(c->ind_n0, c->sm_count * 16)), bx(32, 3);
    lim_gated_tile_list_kernel<2, 0><<<gx, bx, 0, c->st>>>(la, c->nx, c->ny, U, c->X, c->nbr, c->ind_band, l0, cnt,
                                                           c->scal);
    dim3 gy(std::min(c->ind_n1, c->sm_count * 4), 1, 3), by(32, 6);
    lim_gated_tile_list_kernel<2, 1><<<gy, by, 0, c->st>>>(la, c->nx, c->ny, U, c->X, c->nbr, c->ind_band, l1,
                                                           cnt + 1, c->scal);
    c->counter += 1;
    return;
  }
  GateSparse sp;
  sp.list = c->ind_blist;
  sp.count = c->ind_blist + c->ld;
  sp.flag = c->ind_band;
  sp.alt = U;
  dim3 grid((c->ne + 127) / 128, 3);
  lim_gated_kernel<2, 2, 2, 0, false, false, true><<<grid, 128, 0, c->st>>>(la, nullptr, U, c->nbr, c->X, c->scal, sp);
  lim_gated_kernel<2, 2, 2, 1, false, false, true><<<grid, 128, 0, c->st>>>(la, nullptr, c->X, c->nbr, U, c->scal, sp);
  c->counter += 1;
}

// in-place limiting of a state buffer with the context's limiter (rescore: the learned indicator
// scores U first; the time steppers score once per step and pass false)
// hrl / m2l with NY passive mass fractions; key = p * 10 + limiter
template <int NY>
int limit_ny(dgb_ctx* c, double* U, int key) {
#define L2Y(P, M) case P * 10 + M: launch_lim2d<P, M, NY>(c, U); return 0;
#define L1Y(P, M) case P * 10 + M: launch_lim1d<P, M, NY>(c, U); return 0;
  if (c->D == 2) {
    switch (key) { L2Y(1, 1) L2Y(1, 2) L2Y(2, 1) L2Y(2, 2) L2Y(3, 1) L2Y(3, 2) default: break; }
  } else {
    switch (key) { L1Y(1, 1) L1Y(1, 2) L1Y(2, 1) L1Y(2, 2) L1Y(3, 1) L1Y(3, 2) default: break; }
  }
#undef L2Y
#undef L1Y
  return set_error(DGB_ERR_UNSUPPORTED, "limiter not available with mass fractions");
}

int limit_dispatch(dgb_ctx* c, double* U, bool rescore = true) {
  if (c->limiter == 0) return 0;
  if (c->ind_on) {
    launch_learned_limiter(c, U, rescore);
    return 0;
  }
  if (c->limiter == DGB_LIM_PRL) {
    const int k = c->D * 10 + c->p;
    switch (k) {
      case 11: launch_prl<1, 1>(c, U); return 0;
      case 12: launch_prl<1, 2>(c, U); return 0;
      case 13: launch_prl<1, 3>(c, U); return 0;
      case 21: launch_prl<2, 1>(c, U); return 0;
      case 22: launch_prl<2, 2>(c, U); return 0;
      case 23: launch_prl<2, 3>(c, U); return 0;
      default: return set_error(DGB_ERR_UNSUPPORTED, "order outside 1..3");
    }
  }
  if (c->gated) {
    const int k = c->D * 10 + c->p;
    switch (k) {
      case 11: return launch_gated<1, 1>(c, U);
      case 12: return launch_gated<1, 2>(c, U);
      case 13: return launch_gated<1, 3>(c, U);
      case 21: return launch_gated<2, 1>(c, U);
      case 22: return launch_gated<2, 2>(c, U);
      case 23: return launch_gated<2, 3>(c, U);
      default: return set_error(DGB_ERR_UNSUPPORTED, "order outside 1..3");
    }
  }
  const int key = c->p * 10 + c->limiter;
  switch (c->nmass) {
    case 0: break;
    case 1: return limit_ny<1>(c, U, key);
    case 2: return limit_ny<2>(c, U, key);
    case 3: return limit_ny<3>(c, U, key);
    default:
      if (c->D == 1) {
        if (int rc = limit1d_many_y(c, U, c->X)) return rc;
        DGB_CUDA(cudaMemcpyAsync(U, c->X, c->nstate * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
        return 0;
      }
      return limit2d_many_y(c, U);
  }
#define L2(P, M) case P * 10 + M: launch_lim2d<P, M>(c, U); return 0;
#define L1(P, M) case P * 10 + M: launch_lim1d<P, M>(c, U); return 0;
  if (c->D == 2) {
    switch (key) { L2(1, 1) L2(1, 2) L2(2, 1) L2(2, 2) L2(3, 1) L2(3, 2) default: break; }
  } else {
    switch (key) { L1(1, 1) L1(1, 2) L1(2, 1) L1(2, 2) L1(3, 1) L1(3, 2) default: break; }
  }
#undef L2
#undef L1
  return set_error(DGB_ERR_UNSUPPORTED, "limiter not available on the device path");
}

template <int DIM, int NS, bool GC>
void launch_ws(dgb_ctx* c, const double* U, int n, double* copy_to, double finish) {
  // grid.y over the nodes; about eight 256-thread CTAs per SM in all, each striding over elements
  const int gx = std::max(1, std::min((n + 255) / 256, c->sm_count * 8 / NS));
  const dim3 grid(gx, NS);
  launch_pdl(c, wavespeed_kernel<DIM, NS, GC>, grid, dim3(256), 0, U, n, c->ld, c->scal, copy_to, c->nf, finish);
}

// the wave-speed reduction into scal->umax over the elements the context owns (all of them, or
// in slab mode the rows between the ghost rows)
// finish > 0: the reduction's last CTA also forms the step dt with that CFL scale
void launch_wavespeed(dgb_ctx* c, const double* Uall, double* copy_to = nullptr, double finish = 0.0) {
  const int e0 = c->halo_lo * c->nx, n = c->ne - (c->halo_lo + c->halo_hi) * c->nx;
  const double* U = Uall + e0;  // element offset inside every (field, node) plane of stride ld
#define WS(D, NS)                                                                              \
  case D * 100 + NS:                                                                           \
    if (c->gamcons) launch_ws<D, NS, true>(c, U, n, copy_to, finish);                          \
    else launch_ws<D, NS, false>(c, U, n, copy_to, finish);                                    \
    break;
  switch (c->D * 100 + c->ns) {
    WS(1, 2) WS(1, 3) WS(1, 4) WS(2, 4) WS(2, 9) WS(2, 16)
    default: break;
  }
#undef WS
}

void launch_dt(dgb_ctx* c, const double* U, bool cfl, double* copy_to = nullptr) {
  ProfScope ps(c, KC_DT);
  if (cfl && c->cs.cfl_scaled > 0) {
    launch_wavespeed(c, U, copy_to, c->cs.cfl_scaled);
  } else {
    if (cfl) {
      launch_wavespeed(c, U, copy_to);
      c->counter++;  // two launches in this scope
    }
    finish_dt_kernel<<<1, 1, 0, c->st>>>(c->scal, c->cs.cfl_scaled);
  }
}

StageArgs stage_args(dgb_ctx* c) {
  StageArgs a;
  std::memset(&a, 0, sizeof(a));
  a.nbr = c->nbr;
  a.scal = c->scal;
  return a;
}

// Stage s (0..2) of an SSP-RK3 step on c->A (Shu-Osher form), limiter included: reads
// {A, B, C}[s], writes {B, C, A}[s].
int ssp_stage(dgb_ctx* c, int s) {
  const double coef[3][2] = {{0.0, 1.0}, {0.75, 0.25}, {1.0 / 3.0, 2.0 / 3.0}};
  double* in[3] = {c->A, c->B, c->C};
  double* out[3] = {c->B, c->C, c->A};
  StageArgs a = stage_args(c);
  a.U = in[s];
  a.Ubase = c->A;
  const bool fused = c->fused_lim && !c->ind_on;
  a.out = fused ? c->X : out[s];  // the fused limiter then writes the stage output
  a.a = coef[s][0];
  a.b = coef[s][1];
  if (int rc = residual_dispatch<MODE_SSP>(c, a)) return rc;
  if (fused) return limit_to(c, c->X, out[s]);
  return limit_dispatch(c, out[s], false);
}

// 1D hrl / m2l limiter from `in` into `out` (no copy back): the 1D steps write the limited stage
// output straight into the buffer the next stage reads
template <int P, int METHOD, int NY>
void launch_lim1d_to(dgb_ctx* c, const double* in, double* out) {
  ProfScope ps(c, KC_LIMITER);
  const LimArgs la{c->ld, c->ne};
  lim1d_kernel<P, METHOD, NY><<<(c->ne + 127) / 128, 128, 0, c->st>>>(la, in, c->nbr, out, c->scal);
}

template <int NY>
int limit1d_to_ny(dgb_ctx* c, const double* in, double* out) {
  switch (c->p * 10 + c->limiter) {
    case 11: launch_lim1d_to<1, 1, NY>(c, in, out); return 0;
    case 12: launch_lim1d_to<1, 2, NY>(c, in, out); return 0;
    case 21: launch_lim1d_to<2, 1, NY>(c, in, out); return 0;
    case 22: launch_lim1d_to<2, 2, NY>(c, in, out); return 0;
    case 31: launch_lim1d_to<3, 1, NY>(c, in, out); return 0;
    case 32: launch_lim1d_to<3, 2, NY>(c, in, out); return 0;
    default: return set_error(DGB_ERR_UNSUPPORTED, "limiter not available on the device path");
  }
}

int limit1d_to(dgb_ctx* c, const double* in, double* out) {
  switch (c->nmass) {
    case 0: return limit1d_to_ny<0>(c, in, out);
    case 1: return limit1d_to_ny<1>(c, in, out);
    case 2: return limit1d_to_ny<2>(c, in, out);
    case 3: return limit1d_to_ny<3>(c, in, out);
    default: return limit1d_many_y(c, in, out);
  }
}

// 1D with the plain hrl / m2l limiter: steps without device copies (the multi-kernel step of a
// small 1D problem is launch-latency bound, so every graph node counts)
bool lim1d_direct(const dgb_ctx* c) {
  return c->D == 1 && !c->gated && !c->ind_on && (c->limiter == DGB_LIM_HRL || c->limiter == DGB_LIM_M2L);
}

// 1D chains with hrl / m2l: residual, stage update and limiter of a stage in one launch
// (res_lim1d_chain_kernel); the stage inputs and accumulators alternate between buffers so that
// no launch writes what a neighbouring block still reads
template <int P, int FLUX, int METHOD>
void launch_res_lim1d(dgb_ctx* c, const StageArgs& a, int mode, const double* acc_in, double* acc_out, int last,
                      double* lim_out) {
  const int grid = (c->ne + RL1D_B - 1) / RL1D_B;
  ProfScope ps(c, KC_RESIDUAL);
  if (mode == MODE_SSP)
    res_lim1d_chain_kernel<P, FLUX, MODE_SSP, METHOD><<<grid, 96, 0, c->st>>>(c->cs, a, acc_in, acc_out, last, lim_out);
  else
    res_lim1d_chain_kernel<P, FLUX, MODE_RK4, METHOD><<<grid, 96, 0, c->st>>>(c->cs, a, acc_in, acc_out, last, lim_out);
}

int res_lim1d(dgb_ctx* c, const StageArgs& a, int mode, const double* acc_in, double* acc_out, int last,
              double* lim_out) {
#define RL(P, F, M)                                                   \
  case P * 100 + F * 10 + M:                                          \
    launch_res_lim1d<P, F, M>(c, a, mode, acc_in, acc_out, last, lim_out); \
    return 0;
  switch (c->p * 100 + c->flux * 10 + c->limiter) {
    RL(1, 0, 1) RL(1, 0, 2) RL(1, 1, 1) RL(1, 1, 2) RL(1, 2, 1) RL(1, 2, 2)
    RL(2, 0, 1) RL(2, 0, 2) RL(2, 1, 1) RL(2, 1, 2) RL(2, 2, 1) RL(2, 2, 2)
    RL(3, 0, 1) RL(3, 0, 2) RL(3, 1, 1) RL(3, 1, 2) RL(3, 2, 1) RL(3, 2, 2)
    default: return set_error(DGB_ERR_UNSUPPORTED, "no fused 1D stage for this (p, flux, limiter)");
  }
#undef RL
}

bool fused1d(const dgb_ctx* c) { return c->chain1d && c->nmass == 0 && !c->gamcons; }

// SSP-RK3, fused 1D stages: inputs A, X, B; limited into X, B, C; C copied to A
int step1d_ssprk3_fused(dgb_ctx* c, bool cfl) {
  launch_dt(c, c->A, cfl);
  const double coef[3][2] = {{0.0, 1.0}, {0.75, 0.25}, {1.0 / 3.0, 2.0 / 3.0}};
  const double* in[3] = {c->A, c->X, c->B};
  double* lim[3] = {c->X, c->B, c->C};
  for (int s = 0; s < 3; ++s) {
    StageArgs a = stage_args(c);
    a.U = in[s];
    a.Ubase = c->A;
    a.a = coef[s][0];
    a.b = coef[s][1];
    if (int rc = res_lim1d(c, a, MODE_SSP, nullptr, nullptr, 0, lim[s])) return rc;
  }
  DGB_CUDA(cudaMemcpyAsync(c->A, c->C, c->nstate * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  return 0;
}

// RK4, fused 1D stages: Us = A; stage inputs A, B, C, B; accumulator X (from the CFL reduction) ->
// DU -> X -> DU; limited into B, C, B and, from the last accumulator, A
int step1d_rk4_fused(dgb_ctx* c, bool cfl) {
  launch_dt(c, c->A, cfl, cfl ? c->X : nullptr);
  if (!cfl) DGB_CUDA(cudaMemcpyAsync(c->X, c->A, c->nstate * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  const double beta[4] = {0.0, 0.5, 0.5, 1.0};
  const double gam[4] = {1.0 / 6.0, 2.0 / 6.0, 2.0 / 6.0, 1.0 / 6.0};
  const double* in[4] = {c->A, c->B, c->C, c->B};
  double* lim[4] = {c->B, c->C, c->B, c->A};
  const double* ain[4] = {c->X, c->DU, c->X, c->DU};
  double* aout[4] = {c->DU, c->X, c->DU, c->X};
  for (int k = 0; k < 4; ++k) {
    StageArgs a = stage_args(c);
    a.U = in[k];
    a.Us = c->A;
    a.b = gam[k];
    a.beta_next = k < 3 ? beta[k + 1] : 0.0;
    if (int rc = res_lim1d(c, a, MODE_RK4, ain[k], aout[k], k == 3, lim[k])) return rc;
  }
  return 0;
}

// SSP-RK3, 1D: stage inputs A, X, B; unlimited outputs B, C, X; limited into X, B, A
int step1d_ssprk3(dgb_ctx* c, bool cfl) {
  if (fused1d(c)) return step1d_ssprk3_fused(c, cfl);
  launch_dt(c, c->A, cfl);
  const double coef[3][2] = {{0.0, 1.0}, {0.75, 0.25}, {1.0 / 3.0, 2.0 / 3.0}};
  const double* in[3] = {c->A, c->X, c->B};
  double* raw[3] = {c->B, c->C, c->X};
  double* lim[3] = {c->X, c->B, c->A};
  for (int s = 0; s < 3; ++s) {
    StageArgs a = stage_args(c);
    a.U = in[s];
    a.Ubase = c->A;
    a.out = raw[s];
    a.a = coef[s][0];
    a.b = coef[s][1];
    if (int rc = residual_dispatch<MODE_SSP>(c, a)) return rc;
    if (int rc = limit1d_to(c, raw[s], lim[s])) return rc;
  }
  return 0;
}

// RK4, 1D: Us = A unchanged through the step, accumulator X (copied from A by the CFL reduction),
// stage k's residual also forms the next input C = Us + beta DU, limited into B; the last stage's
// accumulator is limited into A
int step1d_rk4(dgb_ctx* c, bool cfl) {
  if (fused1d(c)) return step1d_rk4_fused(c, cfl);
  launch_dt(c, c->A, cfl, cfl ? c->X : nullptr);
  if (!cfl) cudaMemcpyAsync(c->X, c->A, c->nstate * sizeof(double), cudaMemcpyDeviceToDevice, c->st);
  const double beta[4] = {0.0, 0.5, 0.5, 1.0};
  const double gam[4] = {1.0 / 6.0, 2.0 / 6.0, 2.0 / 6.0, 1.0 / 6.0};
  for (int k = 0; k < 4; ++k) {
    StageArgs a = stage_args(c);
    a.U = k == 0 ? c->A : c->B;
    a.out = c->DU;
    a.Uacc = c->X;
    a.b = gam[k];
    a.Unext = k < 3 ? c->C : nullptr;
    a.Us = c->A;
    a.beta_next = k < 3 ? beta[k + 1] : 0.0;
    if (int rc = residual_dispatch<MODE_RK4>(c, a)) return rc;
    if (int rc = limit1d_to(c, k < 3 ? c->C : c->X, k < 3 ? c->B : c->A)) return rc;
  }
  return 0;
}

// One SSP-RK3 step on c->A; limiter after every stage.  score: the learned indicator (if set)
// scores the step's initial state (else the band of its last scoring is reused).
int step_ssprk3(dgb_ctx* c, bool cfl, bool score = true) {
  if (lim1d_direct(c)) return step1d_ssprk3(c, cfl);
  launch_dt(c, c->A, cfl);
  if (c->ind_on && score) launch_indicator(c, c->A);  // the learned indicator's band
  for (int s = 0; s < 3; ++s)
    if (int rc = ssp_stage(c, s)) return rc;
  return 0;
}

// Stage k (0..3) of a classical RK4 step in the reference's form (rk.cc:155-209): A = U, B = Us,
// C = Ustar.  The residual of the stage input (B for k = 0, C after) is accumulated into A; then
// the next stage's input C = Us + beta DU is formed and limited, or after the last stage A is
// limited.
int rk4_stage(dgb_ctx* c, int k) {
  const double beta[4] = {0.0, 0.5, 0.5, 1.0};
  const double gam[4] = {1.0 / 6.0, 2.0 / 6.0, 2.0 / 6.0, 1.0 / 6.0};
  StageArgs a = stage_args(c);
  a.U = k == 0 ? c->B : c->C;
  a.out = c->DU;
  a.Uacc = c->A;
  a.b = gam[k];
  if (int rc = residual_dispatch<MODE_RK4>(c, a)) return rc;
  if (k == 3) return limit_dispatch(c, c->A, false);
  const int grid = (int)std::min<size_t>((c->nstate + 255) / 256, 148 * 16);
  {
    ProfScope ps(c, KC_OTHER);
    axpy_kernel<<<grid, 256, 0, c->st>>>(c->B, c->DU, beta[k + 1], c->C, c->nstate, c->scal);
  }
  return limit_dispatch(c, c->C, false);
}

// One classical RK4 step (score: as step_ssprk3).
int step_rk4(dgb_ctx* c, bool cfl, bool score = true) {
  if (lim1d_direct(c)) return step1d_rk4(c, cfl);
  launch_dt(c, c->A, cfl);
  if (c->ind_on && score) launch_indicator(c, c->A);  // the learned indicator's band
  cudaMemcpyAsync(c->B, c->A, c->nstate * sizeof(double), cudaMemcpyDeviceToDevice, c->st);
  for (int k = 0; k < 4; ++k)
    if (int rc = rk4_stage(c, k)) return rc;
  return 0;
}

// layout conversions of elements [e0, e0 + n) (reference <-> internal) on the context's stream
int convert_range(dgb_ctx* c, bool to_int, const double* src, double* dst, int e0, int n) {
  const size_t per = (size_t)c->nf * c->ns, smem = convert_smem_bytes(c->nf, c->ns);
  const int grid = std::max(1, std::min((n + CONV_EB - 1) / CONV_EB, c->sm_count * 16));
  if (to_int)
    convert_layout_kernel<true><<<grid, 256, smem, c->st>>>(src + e0 * per, dst + e0, c->perm, n, c->nf, c->ns, c->ld);
  else
    convert_layout_kernel<false><<<grid, 256, smem, c->st>>>(src + e0, dst + e0 * per, c->perm, n, c->nf, c->ns, c->ld);
  DGB_CUDA(cudaGetLastError());
  return 0;
}
int to_internal(dgb_ctx* c, const double* Uref_dev, double* Uint) {
  return convert_range(c, true, Uref_dev, Uint, 0, c->ne);
}
int to_ref(dgb_ctx* c, const double* Uint, double* Uref_dev) {
  return convert_range(c, false, Uint, Uref_dev, 0, c->ne);
}
size_t ref_bytes(dgb_ctx* c) { return (size_t)c->ne * c->nf * c->ns * sizeof(double); }

int upload(dgb_ctx* c, const double* host, double* Uint) {
  DGB_CUDA(cudaMemcpyAsync(c->ref, host, ref_bytes(c), cudaMemcpyHostToDevice, c->st));
  return to_internal(c, c->ref, Uint);
}
int download(dgb_ctx* c, const double* Uint, double* host) {
  if (int rc = to_ref(c, Uint, c->ref)) return rc;
  DGB_CUDA(cudaMemcpyAsync(host, c->ref, ref_bytes(c), cudaMemcpyDeviceToHost, c->st));
  DGB_CUDA(cudaStreamSynchronize(c->st));
  return 0;
}

int reset_scalars(dgb_ctx* c, double dt_fixed) {
  std::memset(c->h_scal, 0, sizeof(DevScalars));
  c->h_scal->dt_fixed = dt_fixed;
  DGB_CUDA(cudaMemcpyAsync(c->scal, c->h_scal, sizeof(DevScalars), cudaMemcpyHostToDevice, c->st));
  return 0;
}
int read_scalars(dgb_ctx* c) {
  DGB_CUDA(cudaMemcpyAsync(c->h_scal, c->scal, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->st));
  DGB_CUDA(cudaStreamSynchronize(c->st));
  return 0;
}

int prof_collect(dgb_ctx* c) {
  if (!c->prof) return 0;
  DGB_CUDA(cudaStreamSynchronize(c->st));
  for (auto& pe : c->pev) {
    float ms = 0;
    cudaEventElapsedTime(&ms, pe.second.first, pe.second.second);
    c->kc_ms[pe.first] += ms;
    c->kc_n[pe.first] += 1;
  }
  c->pev.clear();
  c->ev_used = 0;
  return 0;
}

}  // namespace

extern "C" int dgb_create(const dgb_problem* prob, int device, dgb_ctx** out) {
  if (!prob || !out) return set_error(DGB_ERR_ARG, "null argument");
  *out = nullptr;
  const Problem& P = dgb_problem_ref(prob);
  if (!P.gpu_ok) return set_error(DGB_ERR_UNSUPPORTED, P.gpu_reason);
  if (P.D == 2 && P.flux == DGB_FLUX_HLL)
    return set_error(DGB_ERR_UNSUPPORTED, "2D HLL is a stub in the reference (twod_multifluid_fluxes.h:119-141)");
  if (P.limiter < 0 || P.limiter > 7) return set_error(DGB_ERR_UNSUPPORTED, "unknown limiter code");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(DGB_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return set_error(DGB_ERR_ARG, "bad device index");
  cudaDeviceProp prop;
  DGB_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) return set_error(DGB_ERR_NO_DEVICE, "kernels are built for sm_100a");
  DGB_CUDA(cudaSetDevice(device));
  auto* c = new dgb_ctx();
  c->device = device;
  c->sm_count = prop.multiProcessorCount;
  {
    // learned-indicator scoring: tcgen05 GEMMs (DGB_INDICATOR_KERNEL=mma: the mma.sync form)
    const char* ik = std::getenv("DGB_INDICATOR_KERNEL");
    c->ind_tc = !(ik && std::string(ik) == "mma");
    // p = 2 FP64 tiled stages: the one-thread-per-element kernel; DGB_TILE_KERNEL=dmma selects the
    // form with the basis contractions on the FP64 tensor cores (measured slower on B200, whose
    // FP64 tensor rate equals its FP64 vector rate)
    const char* tk = std::getenv("DGB_TILE_KERNEL");
    c->tile_dmma = tk && std::string(tk) == "dmma";
    // programmatic dependent launches of the 2D step's kernels unless DGB_PDL=0
    const char* pk = std::getenv("DGB_PDL");
    c->pdl = !(pk && std::string(pk) == "0");
    // mixed-form tiles: the compressed shared tile (FP64 anchors + FP32 deviations, plain loads)
    // at p = 3, the TMA-loaded FP64 tile at p = 1, 2 (the faster of the two at each order);
    // DGB_MIXED_TILE=ct / tma selects one for every order
    const char* mk = std::getenv("DGB_MIXED_TILE");
    c->mixed_ct = mk ? std::string(mk) == "ct" : P.p == 3;
    // element chunks of dgb_advance_host's copies (DGB_HOST_CHUNKS, 1 .. kHostChunks; 16 measured best)
    const char* hk = std::getenv("DGB_HOST_CHUNKS");
    c->host_chunks = hk ? std::max(1, std::min(kHostChunks, std::atoi(hk))) : kHostChunksDefault;
  }
  c->D = P.D; c->p = P.p; c->nf = P.N_F; c->ns = P.N_s; c->ne = P.N_E;
  c->ld = (P.N_E + 63) / 64 * 64;
  c->flux = P.flux; c->limiter = P.limiter;
  c->nstate = (size_t)c->nf * c->ns * c->ld;
  c->cs = make_consts(P, c->ld);
  c->nx = P.nx;
  c->ny = P.ny;
  c->hx = P.hx;
  c->hy = P.hy;
  c->rowmajor = P.D == 2 && is_row_major_grid(P) && std::getenv("DGB_NO_TILE") == nullptr;
  // 1D elements in chain order: fused residual + limiter stages (DGB_1D_FUSED=0: separate kernels)
  {
    const char* f1 = std::getenv("DGB_1D_FUSED");
    c->chain1d = P.D == 1 && is_chain_1d(P) && !(f1 && std::string(f1) == "0");
  }
  // tiled residual over the full tiles; the strips left over on other extents go to the generic
  // kernel.  Tile loads by TMA where the tensor map's row pitch nx * 8 bytes is a multiple of 16
  // (nx even), by plain loads otherwise
  c->tiled = c->rowmajor && P.p <= 3 && P.nx >= TILE_W && P.ny >= tile_h_for(P.p, P.N_Y);
  c->tile_tma = c->tiled && P.nx % 2 == 0;
  c->tiled_full = c->tile_tma && P.nx % TILE_W == 0 && P.ny % tile_h_for(P.p, P.N_Y) == 0;
  // opt-in: measured slower than the two tiled passes on 512 x 256, p = 2 (64 vs 55 us per stage)
  c->fused_lim = c->rowmajor && (P.limiter == DGB_LIM_HRL || P.limiter == DGB_LIM_M2L) &&
                 std::getenv("DGB_FUSED_LIMITER") != nullptr && P.N_Y == 0;
  c->nmass = P.N_Y;
  c->gamcons = P.gamcons;
  if (P.gamcons) {
    const char* why = nullptr;
    if (P.N_Y != 0) why = "GAMCONS with mass fractions is not on the device path";
    else if (P.D == 2 && !c->tile_tma)
      why = "GAMCONS in 2D needs a structured row-major grid with an even nx of at least 32 and at least one "
            "tile's height of rows (4; p = 3: 2)";
    else if (P.limiter == DGB_LIM_M2L)  // M2limiting stops there too (limiting.cc:193-194, 410-411)
      why = "M2L is only implemented for gamncon";
    else if (P.limiter != DGB_LIM_NONE && P.limiter != DGB_LIM_HRL)
      why = "with GAMCONS the limiter is none or hrl";
    else if (!P.thresholds.empty())
      why = "the troubled-cell sensors are built for GAMNCON";
    if (why) { delete c; return set_error(DGB_ERR_UNSUPPORTED, why); }
    c->fused_lim = false;
  }
  if (P.N_Y > 10) { delete c; return set_error(DGB_ERR_UNSUPPORTED, "at most ten mass fractions"); }
  if (P.N_Y > 3) {
    if (int rc = upload_many_y_tables(c->cs, P.D, P.p)) { delete c; return rc; }
  }
  if (P.N_Y > 0 && P.D == 2 && !c->tile_tma) {
    delete c;
    return set_error(DGB_ERR_UNSUPPORTED, "mass fractions in 2D need a structured row-major grid with an even nx of "
                                          "at least 32 and at least one tile's height of rows (4; p = 3 or more "
                                          "than three mass fractions: 2)");
  }
  if (P.N_Y > 0 && P.limiter != DGB_LIM_NONE && P.limiter != DGB_LIM_HRL && P.limiter != DGB_LIM_M2L) {
    delete c;
    return set_error(DGB_ERR_UNSUPPORTED, "with mass fractions the limiter is none, hrl or m2l");
  }
  if (int rc = upload_tables(c->cs, P.D, P.p)) { delete c; return rc; }
  auto fail = [&](cudaError_t e, const char* what) {
    dgb_destroy(c);
    return set_error(DGB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
  const size_t sb = c->nstate * sizeof(double);
  double** bufs[4] = {&c->A, &c->B, &c->C, &c->DU};
  for (auto b : bufs) {
    if ((e = cudaMalloc(b, sb)) != cudaSuccess) return fail(e, "state allocation");
    cudaMemset(*b, 0, sb);
  }
  const size_t xb = (size_t)(6 + c->nmass) * c->ns * c->ld * sizeof(double);  // m2 x pass: 6 quantities + Y_k
  if ((e = cudaMalloc(&c->X, std::max(xb, sb))) != cudaSuccess) return fail(e, "limiter scratch");
  cudaMemset(c->X, 0, std::max(xb, sb));
  if ((e = cudaMalloc(&c->ref, (size_t)c->ne * c->nf * c->ns * sizeof(double))) != cudaSuccess) return fail(e, "staging");
  if ((e = cudaMalloc(&c->nbr, (size_t)P.N_N * c->ld * sizeof(int))) != cudaSuccess) return fail(e, "neighbours");
  std::vector<int> nb((size_t)P.N_N * c->ld, -4);
  for (int k = 0; k < P.N_N; ++k)
    for (int el = 0; el < P.N_E; ++el) nb[(size_t)k * c->ld + el] = P.nbr[(size_t)k * P.N_E + el];
  cudaMemcpy(c->nbr, nb.data(), nb.size() * sizeof(int), cudaMemcpyHostToDevice);
  if ((e = cudaMalloc(&c->perm, c->ns * sizeof(int))) != cudaSuccess) return fail(e, "perm");
  cudaMemcpy(c->perm, P.tensor_perm.data(), c->ns * sizeof(int), cudaMemcpyHostToDevice);
  c->gated = P.limiter == DGB_LIM_HRI || P.limiter == DGB_LIM_M2I || P.limiter == DGB_LIM_PRI || P.limiter == DGB_LIM_P0I;
  c->has_sensors = c->gated || !P.thresholds.empty();
  if (c->has_sensors) {
    // sensor work arrays; the reference's node order for the cell means; p0i weights
    if ((e = cudaMalloc(&c->smean, (size_t)c->nf * c->ld * sizeof(double))) != cudaSuccess) return fail(e, "sensor means");
    if ((e = cudaMalloc(&c->sint, ((size_t)6 * c->ld + 64) * sizeof(int))) != cudaSuccess) return fail(e, "sensor arrays");
    cudaMemset(c->sint, 0, ((size_t)6 * c->ld + 64) * sizeof(int));
    std::vector<int> ip(c->ns);
    for (int t = 0; t < c->ns; ++t) ip[P.tensor_perm[t]] = t;
    if ((e = cudaMalloc(&c->iperm, c->ns * sizeof(int))) != cudaSuccess) return fail(e, "iperm");
    cudaMemcpy(c->iperm, ip.data(), c->ns * sizeof(int), cudaMemcpyHostToDevice);
    SensorLaunch& sl = c->sl;
    std::memset(&sl, 0, sizeof(sl));
    sl.D = c->D; sl.ns = c->ns; sl.nf = c->nf; sl.n_elem = c->ne; sl.ld = c->ld; sl.n_nbr = P.N_N;
    sl.iperm = c->iperm; sl.nbr = c->nbr; sl.mean = c->smean;
    sl.target = c->sint; sl.type = c->sint + c->ld; sl.processed = c->sint + 2 * (size_t)c->ld;
    sl.mask = c->sint + 3 * (size_t)c->ld; sl.list = c->sint + 4 * (size_t)c->ld; sl.sens = c->sint + 5 * (size_t)c->ld;
    sl.count = c->sint + 6 * (size_t)c->ld;
    for (int k = 0; k < 3; ++k) {
      sl.on[k] = k < (int)P.thresholds.size();
      sl.th[k] = sl.on[k] ? P.thresholds[k] : 0.0;
    }
    // cell average = sum_g sum_i phi_w[i*N_G + g] U_i / |reference element| (4 for quads; lines: 2)
    std::memset(&c->p0w, 0, sizeof(c->p0w));
    const double area = P.D == 2 ? 4.0 : 2.0;
    for (int t = 0; t < c->ns; ++t) {
      const int i = P.tensor_perm[t];
      double w = 0;
      for (int g = 0; g < P.N_G; ++g) w += P.phi_w[(size_t)i * P.N_G + g];
      c->p0w.w[t] = w / area;
    }
  }
  if ((e = cudaMalloc(&c->scal, sizeof(DevScalars))) != cudaSuccess) return fail(e, "scalars");
  cudaMemset(c->scal, 0, sizeof(DevScalars));
  if ((e = cudaMallocHost(&c->h_scal, sizeof(DevScalars))) != cudaSuccess) return fail(e, "pinned scalars");
  // the tensor maps are kernel arguments of every tiled launch, also of the plain-load variant
  // that never reads them: zeroed, not left undefined, when no map is encoded
  std::memset(&c->mapA, 0, sizeof(CUtensorMap));
  std::memset(&c->mapB, 0, sizeof(CUtensorMap));
  std::memset(&c->mapC, 0, sizeof(CUtensorMap));
  if (c->tile_tma) {
    // row starts must be 16-byte aligned for TMA: nx is even and ld a multiple of 64
    const int th = tile_h_for(P.p, P.N_Y);
    if (!(encode_state_map(c, c->A, &c->mapA, TILE_W, th) && encode_state_map(c, c->B, &c->mapB, TILE_W, th) &&
          encode_state_map(c, c->C, &c->mapC, TILE_W, th))) {
      if (P.N_Y > 0 || P.gamcons) return fail(cudaErrorInvalidValue, "tensor maps for the tiled residual");
      c->tile_tma = c->tiled_full = false;  // plain tile loads
    }
  }
  if (c->tiled && !c->tiled_full) {
    // the right strip (rows of the full tiles) and the top strip (all columns), in element order
    const int th = tile_h_for(P.p, P.N_Y), nxt = P.nx / TILE_W * TILE_W, nyt = P.ny / th * th;
    std::vector<int> left;
    for (int y = 0; y < P.ny; ++y)
      for (int x = (y < nyt ? nxt : 0); x < P.nx; ++x) left.push_back(y * P.nx + x);
    c->nleft = (int)left.size();
    if ((e = cudaMalloc(&c->left, left.size() * sizeof(int))) != cudaSuccess) return fail(e, "leftover list");
    cudaMemcpy(c->left, left.data(), left.size() * sizeof(int), cudaMemcpyHostToDevice);
  }
  cudaEventCreate(&c->e0);
  cudaEventCreate(&c->e1);
  if ((e = cudaDeviceSynchronize()) != cudaSuccess) return fail(e, "create");
  *out = c;
  return DGB_OK;
}

namespace dgb {
void drop_slab_graphs(dgb_ctx* c);
}

extern "C" void dgb_destroy(dgb_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->st) cudaStreamSynchronize(c->st);
  c->drop_graphs();
  dgb::drop_slab_graphs(c);
  for (double* b : c->halo_send) if (b) cudaFree(b);
  for (double* b : {c->A, c->B, c->C, c->DU, c->X, c->ref}) if (b) cudaFree(b);
  if (c->nbr) cudaFree(c->nbr);
  if (c->left) cudaFree(c->left);
  if (c->perm) cudaFree(c->perm);
  if (c->iperm) cudaFree(c->iperm);
  for (void* q : {(void*)c->ind_params, (void*)c->ind_w, (void*)c->ind_vec, (void*)c->ind_modes, (void*)c->ind_score,
                  (void*)c->ind_flag, (void*)c->ind_list, (void*)c->ind_band, (void*)c->ind_blist,
                  (void*)c->ind_tiles})
    if (q) cudaFree(q);
  if (c->smean) cudaFree(c->smean);
  if (c->sint) cudaFree(c->sint);
  if (c->scal) cudaFree(c->scal);
  if (c->h_scal) cudaFreeHost(c->h_scal);
  for (auto ev : c->ev_pool) cudaEventDestroy(ev);
  for (auto ev : c->hl_up) if (ev) cudaEventDestroy(ev);
  for (auto ev : c->hl_down) if (ev) cudaEventDestroy(ev);
  for (auto ev : c->hl_conv) if (ev) cudaEventDestroy(ev);
  if (c->hl_done) cudaEventDestroy(c->hl_done);
  for (auto st : c->hl_st) if (st) cudaStreamDestroy(st);
  if (c->e0) cudaEventDestroy(c->e0);
  if (c->e1) cudaEventDestroy(c->e1);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
}

extern "C" int dgb_set_state(dgb_ctx* c, const double* U) {
  if (!c || !U) return set_error(DGB_ERR_ARG, "null argument");
  DGB_CUDA(cudaSetDevice(c->device));
  if (int rc = upload(c, U, c->A)) return rc;
  DGB_CUDA(cudaStreamSynchronize(c->st));
  c->ind_step = 0;  // a new state: the learned indicator scores the next step
  return DGB_OK;
}

extern "C" int dgb_get_state(dgb_ctx* c, double* U) {
  if (!c || !U) return set_error(DGB_ERR_ARG, "null argument");
  DGB_CUDA(cudaSetDevice(c->device));
  return download(c, c->A, U);
}

extern "C" int dgb_set_state_device(dgb_ctx* c, const double* U_dev) {
  if (!c || !U_dev) return set_error(DGB_ERR_ARG, "null argument");
  DGB_CUDA(cudaSetDevice(c->device));
  if (int rc = to_internal(c, U_dev, c->A)) return rc;
  DGB_CUDA(cudaStreamSynchronize(c->st));
  c->ind_step = 0;
  return DGB_OK;
}

extern "C" int dgb_get_state_device(dgb_ctx* c, double* U_dev) {
  if (!c || !U_dev) return set_error(DGB_ERR_ARG, "null argument");
  DGB_CUDA(cudaSetDevice(c->device));
  if (int rc = to_ref(c, c->A, U_dev)) return rc;
  DGB_CUDA(cudaStreamSynchronize(c->st));
  return DGB_OK;
}

extern "C" int dgb_residual(dgb_ctx* c, const double* U, double* f) {
  if (!c || !U || !f) return set_error(DGB_ERR_ARG, "null argument");
  DGB_CUDA(cudaSetDevice(c->device));
  if (int rc = upload(c, U, c->B)) return rc;
  if (int rc = reset_scalars(c, 0.0)) return rc;
  StageArgs a = stage_args(c);
  a.U = c->B;
  a.out = c->C;
  if (int rc = residual_dispatch<MODE_RESIDUAL>(c, a)) return rc;
  DGB_CUDA(cudaGetLastError());
  if (int rc = download(c, c->C, f)) return rc;
  if (int rc = read_scalars(c)) return rc;
  if (c->h_scal->flags & FLAG_TIMEOUT) return set_error(DGB_ERR_TIMEOUT, "a bounded device wait expired");
  return DGB_OK;
}

extern "C" int dgb_solve(dgb_ctx* c, double dt, const double* U, double* DU) {
  if (!c || !U || !DU) return set_error(DGB_ERR_ARG, "null argument");
  if (!(dt > 0)) return set_error(DGB_ERR_ARG, "dt must be > 0");
  DGB_CUDA(cudaSetDevice(c->device));
  if (int rc = upload(c, U, c->B)) return rc;
  if (int rc = reset_scalars(c, 0.0)) return rc;
  StageArgs a = stage_args(c);
  a.U = c->B;
  a.out = c->C;
  a.Uacc = nullptr;
  a.dt_override = dt;
  if (int rc = residual_dispatch<MODE_RK4>(c, a)) return rc;
  DGB_CUDA(cudaGetLastError());
  if (int rc = download(c, c->C, DU)) return rc;
  if (int rc = read_scalars(c)) return rc;
  if (c->h_scal->flags & FLAG_TIMEOUT) return set_error(DGB_ERR_TIMEOUT, "a bounded device wait expired");
  return DGB_OK;
}

extern "C" int dgb_limit(dgb_ctx* c, double* U) {
  if (!c || !U) return set_error(DGB_ERR_ARG, "null argument");
  DGB_CUDA(cudaSetDevice(c->device));
  if (int rc = upload(c, U, c->B)) return rc;
  if (int rc = reset_scalars(c, 0.0)) return rc;
  if (int rc = limit_dispatch(c, c->B)) return rc;
  DGB_CUDA(cudaGetLastError());
  return download(c, c->B, U);
}

// ------------------------------------------------------------------------------------------
// learned troubled-cell indicator: dataset and training
// ------------------------------------------------------------------------------------------
extern "C" int dgb_mlp_param_count(void) { return MLP_NPARAM; }

extern "C" int dgb_indicator_features(dgb_ctx* c, float* X_dev) {
  if (!c || !X_dev) return set_error(DGB_ERR_ARG, "null argument");
  if (c->D != 2 || c->p != 2 || c->nmass != 0 || c->gamcons)
    return set_error(DGB_ERR_UNSUPPORTED, "the indicator is built for 2D, p = 2, GAMNCON, without mass fractions");
  DGB_CUDA(cudaSetDevice(c->device));
  indicator_features_kernel<2><<<(c->ne + 127) / 128, 128, 0, c->st>>>(c->A, c->ld, c->ne, c->nbr, X_dev);
  DGB_CUDA(cudaGetLastError());
  DGB_CUDA(cudaStreamSynchronize(c->st));
  return DGB_OK;
}

extern "C" int dgb_indicator_labels(dgb_ctx* c, float* y_dev) {
  if (!c || !y_dev) return set_error(DGB_ERR_ARG, "null argument");
  if (c->D != 2 || c->p != 2 || c->nmass != 0 || c->gamcons)
    return set_error(DGB_ERR_UNSUPPORTED, "the indicator is built for 2D, p = 2, GAMNCON, without mass fractions");
  if (c->limiter == 0) return set_error(DGB_ERR_ARG, "labels need a limiter");
  DGB_CUDA(cudaSetDevice(c->device));
  if (int rc = reset_scalars(c, 0.0)) return rc;
  DGB_CUDA(cudaMemcpyAsync(c->B, c->A, c->nstate * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  const bool ind = c->ind_on;
  c->ind_on = false;  // labels come from the problem's own (full) limiter
  const int rc = limit_dispatch(c, c->B);
  c->ind_on = ind;
  if (rc) return rc;
  indicator_labels_kernel<2><<<(c->ne + 127) / 128, 128, 0, c->st>>>(c->A, c->B, c->ld, c->ne, y_dev);
  DGB_CUDA(cudaGetLastError());
  DGB_CUDA(cudaStreamSynchronize(c->st));
  return DGB_OK;
}

extern "C" int dgb_mlp_forward(const float* params, const float* X, int n, float* cache, float* prob, void* stream) {
  if (!params || !X || !prob || n < 0) return set_error(DGB_ERR_ARG, "bad argument");
  if (n == 0) return DGB_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t smem = MLP_NPARAM * sizeof(float);
  allow_dynamic_smem(mlp_forward_kernel, smem);
  mlp_forward_kernel<<<(n + 127) / 128, 128, smem, st>>>(params, X, n, cache, prob);
  DGB_CUDA(cudaGetLastError());
  return DGB_OK;
}

extern "C" int dgb_mlp_backward(const float* params, const float* X, const float* y, float pos_weight, int n,
                                const float* cache, const float* prob, float* grad, float* loss, float* work,
                                void* stream) {
  if (!params || !X || !y || !cache || !prob || !grad || !loss || !work || n <= 0)
    return set_error(DGB_ERR_ARG, "bad argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float* dz = work;
  float* dA2 = work + n;
  float* dA1 = dA2 + (size_t)n * MLP_H;
  DGB_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), st));
  mlp_delta_kernel<<<(n + 127) / 128, 128, 0, st>>>(params, y, pos_weight, n, cache, prob, dz, dA2, dA1, loss);
  const dim3 b(16, 16);
  auto red = [&](const float* Pm, int ldp, int R, const float* Qm, int ldq, int C, float* G) {
    const dim3 g((C + 15) / 16, (R + 15) / 16);
    outer_reduce_kernel<<<g, b, 0, st>>>(n, Pm, ldp, R, Qm, ldq, C, G);
  };
  red(dA1, MLP_H, MLP_H, X, MLP_IN, MLP_IN, grad + MLP_W1);            // dW1 = dA1^T X
  red(dA1, MLP_H, MLP_H, nullptr, 0, 1, grad + MLP_B1);                // db1
  red(dA2, MLP_H, MLP_H, cache + MLP_H, MLP_CACHE, MLP_H, grad + MLP_W2);  // dW2 = dA2^T H1
  red(dA2, MLP_H, MLP_H, nullptr, 0, 1, grad + MLP_B2);                // db2
  red(cache + 3 * MLP_H, MLP_CACHE, MLP_H, dz, 1, 1, grad + MLP_W3);   // dw3 = H2^T dz
  red(dz, 1, 1, nullptr, 0, 1, grad + MLP_B3);                         // db3
  DGB_CUDA(cudaGetLastError());
  return DGB_OK;
}

extern "C" int dgb_mlp_adam(float* params, const float* grad, float* m, float* v, int t, float lr, void* stream) {
  if (!params || !grad || !m || !v || t < 1) return set_error(DGB_ERR_ARG, "bad argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  mlp_adam_kernel<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(params, grad, m, v, MLP_NPARAM, t, lr, 0.9f, 0.999f, 1e-8f);
  DGB_CUDA(cudaGetLastError());
  return DGB_OK;
}

extern "C" int dgb_set_indicator_interval(dgb_ctx* c, int steps) {
  if (!c) return set_error(DGB_ERR_ARG, "null argument");
  if (steps < 1) return set_error(DGB_ERR_ARG, "the scoring interval is at least one step");
  c->ind_every = steps;
  c->ind_step = 0;
  return DGB_OK;
}

extern "C" int dgb_set_indicator(dgb_ctx* c, const float* params, float threshold) {
  if (!c) return set_error(DGB_ERR_ARG, "null argument");
  DGB_CUDA(cudaSetDevice(c->device));
  DGB_CUDA(cudaStreamSynchronize(c->st));
  c->drop_graphs();
  c->ind_step = 0;
  if (!params) {
    c->ind_on = false;
    return DGB_OK;
  }
  if (c->D != 2 || c->p != 2 || c->limiter != DGB_LIM_M2L || c->nmass != 0 || c->gamcons)
    return set_error(DGB_ERR_UNSUPPORTED,
                     "the learned indicator gates the m2l limiter of 2D p = 2 problems without mass fractions");
  if (!c->ind_params) {
    cudaError_t e;
    if ((e = cudaMalloc(&c->ind_params, MLP_NPARAM * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc(&c->ind_w, (size_t)(MLP_H * IND_KPAD + MLP_H * MLP_H) * sizeof(__nv_bfloat16))) != cudaSuccess ||
        (e = cudaMalloc(&c->ind_vec, (3 * MLP_H + 1) * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc(&c->ind_modes, (size_t)c->ld * IND_MODES * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc(&c->ind_score, (size_t)c->ld * sizeof(float))) != cudaSuccess ||
        (e = cudaMalloc(&c->ind_flag, (size_t)c->ld)) != cudaSuccess ||
        (e = cudaMalloc(&c->ind_list, ((size_t)c->ld + 1) * sizeof(int))) != cudaSuccess ||
        (e = cudaMalloc(&c->ind_band, (size_t)c->ld)) != cudaSuccess ||
        (e = cudaMalloc(&c->ind_blist, ((size_t)c->ld + 1) * sizeof(int))) != cudaSuccess)
      return set_error(DGB_ERR_CUDA, std::string("indicator buffers: ") + cudaGetErrorString(e));
    if (c->rowmajor) {
      c->ind_n0 = (c->nx + GATED_TW0 - 1) / GATED_TW0 * c->ny;
      c->ind_n1 = (c->nx + GATED_TW1 - 1) / GATED_TW1 * ((c->ny + GATED_TH1 - 1) / GATED_TH1);
      if ((e = cudaMalloc(&c->ind_tiles, ((size_t)c->ind_n0 + c->ind_n1 + 2) * sizeof(int))) != cudaSuccess)
        return set_error(DGB_ERR_CUDA, std::string("indicator buffers: ") + cudaGetErrorString(e));
    }
  }
  std::vector<__nv_bfloat16> w((size_t)MLP_H * IND_KPAD + MLP_H * MLP_H, __float2bfloat16(0.f));
  for (int j = 0; j < MLP_H; ++j)
    for (int k = 0; k < MLP_IN; ++k)  // input k = 45 n + r sits at column 48 n + r
      w[(size_t)j * IND_KPAD + IND_NSEG * (k / 45) + k % 45] = __float2bfloat16(params[MLP_W1 + j * MLP_IN + k]);
  for (int j = 0; j < MLP_H; ++j)
    for (int i = 0; i < MLP_H; ++i) w[(size_t)MLP_H * IND_KPAD + j * MLP_H + i] = __float2bfloat16(params[MLP_W2 + j * MLP_H + i]);
  std::vector<float> vec(3 * MLP_H + 1);
  for (int j = 0; j < MLP_H; ++j) {
    vec[j] = params[MLP_B1 + j];
    vec[MLP_H + j] = params[MLP_B2 + j];
    vec[2 * MLP_H + j] = params[MLP_W3 + j];
  }
  vec[3 * MLP_H] = params[MLP_B3];
  DGB_CUDA(cudaMemcpy(c->ind_params, params, MLP_NPARAM * sizeof(float), cudaMemcpyHostToDevice));
  DGB_CUDA(cudaMemcpy(c->ind_w, w.data(), w.size() * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
  DGB_CUDA(cudaMemcpy(c->ind_vec, vec.data(), vec.size() * sizeof(float), cudaMemcpyHostToDevice));
  c->ind_threshold = threshold;
  c->ind_on = true;
  return DGB_OK;
}

extern "C" int dgb_indicator_scores(dgb_ctx* c, const double* U, float* score, int* n_flagged) {
  if (!c || !U || !score) return set_error(DGB_ERR_ARG, "null argument");
  if (!c->ind_on) return set_error(DGB_ERR_ARG, "no indicator set (dgb_set_indicator)");
  DGB_CUDA(cudaSetDevice(c->device));
  if (int rc = upload(c, U, c->B)) return rc;
  if (int rc = reset_scalars(c, 0.0)) return rc;
  launch_indicator(c, c->B);
  DGB_CUDA(cudaGetLastError());
  DGB_CUDA(cudaMemcpyAsync(score, c->ind_score, (size_t)c->ne * sizeof(float), cudaMemcpyDeviceToHost, c->st));
  int cnt = 0;
  DGB_CUDA(cudaMemcpyAsync(&cnt, c->ind_list + c->ld, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  DGB_CUDA(cudaStreamSynchronize(c->st));
  if (n_flagged) *n_flagged = cnt;
  return DGB_OK;
}

extern "C" int dgb_set_form(dgb_ctx* c, int form) {
  if (!c) return set_error(DGB_ERR_ARG, "null argument");
  if (form != DGB_FORM_FP64 && form != DGB_FORM_MIXED) return set_error(DGB_ERR_ARG, "unknown form");
  if (form == DGB_FORM_MIXED && !(c->tile_tma && c->flux != DGB_FLUX_HLL && c->nmass == 0 && !c->gamcons))
    return set_error(DGB_ERR_UNSUPPORTED,
                     "the mixed form needs a structured row-major 2D grid with even nx >= 32 and ny >= 4 "
                     "(p = 3: 2), Rusanov or Roe, no mass fractions, GAMNCON");
  if (form != c->form) {
    DGB_CUDA(cudaSetDevice(c->device));
    DGB_CUDA(cudaStreamSynchronize(c->st));
    c->drop_graphs();
    c->form = form;
  }
  return DGB_OK;
}

extern "C" int dgb_set_wait_limit(dgb_ctx* c, long long polls) {
  if (!c) return set_error(DGB_ERR_ARG, "null argument");
  if (polls < 0) return set_error(DGB_ERR_ARG, "negative poll budget");
  if (polls != c->wait_polls) {
    DGB_CUDA(cudaSetDevice(c->device));
    DGB_CUDA(cudaStreamSynchronize(c->st));
    c->drop_graphs();  // the budget is a kernel argument of the captured launches
    c->wait_polls = polls;
  }
  return DGB_OK;
}

extern "C" int dgb_sensors(dgb_ctx* c, const double* U, int* flags) {
  if (!c || !U || !flags) return set_error(DGB_ERR_ARG, "null argument");
  if (!c->has_sensors) return set_error(DGB_ERR_ARG, "the problem has no sensor thresholds");
  DGB_CUDA(cudaSetDevice(c->device));
  if (int rc = upload(c, U, c->B)) return rc;
  SensorLaunch s = c->sl;
  s.U = c->B;
  if (int rc = launch_sensors(s, c->st)) return set_error(DGB_ERR_CUDA, std::string("sensors: ") + cudaGetErrorString((cudaError_t)rc));
  DGB_CUDA(cudaMemcpyAsync(flags, s.sens, (size_t)c->ne * sizeof(int), cudaMemcpyDeviceToHost, c->st));
  DGB_CUDA(cudaStreamSynchronize(c->st));
  return DGB_OK;
}

extern "C" int dgb_cfl_dt(dgb_ctx* c, double* dt) {
  if (!c || !dt) return set_error(DGB_ERR_ARG, "null argument");
  DGB_CUDA(cudaSetDevice(c->device));
  if (int rc = reset_scalars(c, 0.0)) return rc;
  launch_dt(c, c->A, true);
  DGB_CUDA(cudaGetLastError());
  if (int rc = read_scalars(c)) return rc;
  if (c->h_scal->flags & FLAG_NONFINITE) return set_error(DGB_ERR_NONFINITE, "time step is NaN");
  if (c->h_scal->flags & FLAG_DT_SMALL) return set_error(DGB_ERR_DT_SMALL, "next time step is too small (< 1e-14)");
  *dt = c->h_scal->dt;
  return DGB_OK;
}

extern "C" int dgb_dt_from_cfl(dgb_ctx* c, const double* U, double* dt) {
  if (!c || !U || !dt) return set_error(DGB_ERR_ARG, "null argument");
  DGB_CUDA(cudaSetDevice(c->device));
  if (int rc = upload(c, U, c->B)) return rc;
  if (int rc = reset_scalars(c, 0.0)) return rc;
  launch_dt(c, c->B, true);
  DGB_CUDA(cudaGetLastError());
  if (int rc = read_scalars(c)) return rc;
  if (c->h_scal->flags & FLAG_NONFINITE) return set_error(DGB_ERR_NONFINITE, "time step is NaN");
  if (c->h_scal->flags & FLAG_DT_SMALL) return set_error(DGB_ERR_DT_SMALL, "next time step is too small (< 1e-14)");
  *dt = c->h_scal->dt;
  return DGB_OK;
}

namespace {
// captures the steps dgb_advance replays for (scheme, CFL or fixed step): the step that scores the
// learned indicator and, when scoring is every few steps, the one that does not
int ensure_step_graphs(dgb_ctx* c, int scheme, bool cfl) {
  const int si = scheme == DGB_RK4 ? 1 : 0, mi = cfl ? 1 : 0;
  for (int k = 0; k < 2; ++k) {
    const bool sc = k == 0;
    if (c->graphs[si][mi][k] || (!sc && (!c->ind_on || c->ind_every <= 1))) continue;
    cudaGraph_t g;
    DGB_CUDA(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    c->counter = 0;
    int rc = scheme == DGB_RK4 ? step_rk4(c, cfl, sc) : step_ssprk3(c, cfl, sc);
    cudaError_t ec = cudaStreamEndCapture(c->st, &g);
    if (rc) { if (ec == cudaSuccess) cudaGraphDestroy(g); return rc; }
    DGB_CUDA(ec);
    DGB_CUDA(cudaGraphInstantiate(&c->graphs[si][mi][k], g, 0));
    cudaGraphDestroy(g);
    c->graph_launches[si][mi][k] = c->counter;
  }
  return DGB_OK;
}

// the step's status from the device scalars (read after the step's last kernel)
int step_status(dgb_ctx* c, double* time) {
  if (int rc = read_scalars(c)) return rc;
  float ms = 0;
  cudaEventElapsedTime(&ms, c->e0, c->e1);
  c->last_ms = ms;
  if (time) *time += c->h_scal->time;
  if (c->h_scal->flags & FLAG_TIMEOUT) return set_error(DGB_ERR_TIMEOUT, "a bounded device wait expired");
  if (c->h_scal->flags & FLAG_NONFINITE) return set_error(DGB_ERR_NONFINITE, "time step is NaN");
  if (c->h_scal->flags & FLAG_DT_SMALL) return set_error(DGB_ERR_DT_SMALL, "next time step is too small (< 1e-14)");
  return DGB_OK;
}
}  // namespace

extern "C" int dgb_advance(dgb_ctx* c, int scheme, int nsteps, double dt, double* time) {
  if (!c) return set_error(DGB_ERR_ARG, "null context");
  if (scheme != DGB_SSPRK3 && scheme != DGB_RK4) return set_error(DGB_ERR_ARG, "scheme must be 3 or 4");
  if (nsteps < 0) return set_error(DGB_ERR_ARG, "nsteps < 0");
  if (!(dt > 0) && !(c->cs.cfl_scaled > 0)) return set_error(DGB_ERR_ARG, "no fixed dt and no positive CFL");
  DGB_CUDA(cudaSetDevice(c->device));
  const bool cfl = !(dt > 0);
  if (int rc = reset_scalars(c, cfl ? 0.0 : dt)) return rc;
  const int si = scheme == DGB_RK4 ? 1 : 0, mi = cfl ? 1 : 0;
  c->counter = 0;
  // the learned indicator scores every ind_every-th step (counted from the last state set)
  auto scores = [c]() { return !c->ind_on || c->ind_every <= 1 || c->ind_step % c->ind_every == 0; };
  if (c->prof) {
    // eager launches with per-kernel-class events
    DGB_CUDA(cudaEventRecord(c->e0, c->st));
    for (int s = 0; s < nsteps; ++s) {
      const bool sc = scores();
      int rc = scheme == DGB_RK4 ? step_rk4(c, cfl, sc) : step_ssprk3(c, cfl, sc);
      if (rc) return rc;
      ++c->ind_step;
    }
    DGB_CUDA(cudaEventRecord(c->e1, c->st));
    DGB_CUDA(cudaGetLastError());
    c->last_launches = c->counter;
    if (int rc = prof_collect(c)) return rc;
  } else {
    if (nsteps > 0)
      if (int rc = ensure_step_graphs(c, scheme, cfl)) return rc;
    DGB_CUDA(cudaEventRecord(c->e0, c->st));
    long long launches = 0;
    for (int s = 0; s < nsteps; ++s) {
      const int k = scores() ? 0 : 1;
      DGB_CUDA(cudaGraphLaunch(c->graphs[si][mi][k], c->st));
      launches += c->graph_launches[si][mi][k];
      ++c->ind_step;
    }
    DGB_CUDA(cudaEventRecord(c->e1, c->st));
    c->last_launches = launches;
  }
  return step_status(c, time);
}

// The time loop with the state of record in host memory.  Every step uploads the state from U
// (reference layout), advances it one step with the captured step and downloads the result into
// U.  The copies go in element chunks on two copy streams: the upload of chunk j for step k+1
// waits only for the download of chunk j from step k, so the two directions of the host link
// overlap; the conversion of each uploaded chunk to the internal layout runs as it lands.
extern "C" int dgb_advance_host(dgb_ctx* c, double* U, int scheme, int nsteps, double dt, double* time) {
  if (!c || !U) return set_error(DGB_ERR_ARG, "null argument");
  if (scheme != DGB_SSPRK3 && scheme != DGB_RK4) return set_error(DGB_ERR_ARG, "scheme must be 3 or 4");
  if (nsteps < 0) return set_error(DGB_ERR_ARG, "nsteps < 0");
  if (!(dt > 0) && !(c->cs.cfl_scaled > 0)) return set_error(DGB_ERR_ARG, "no fixed dt and no positive CFL");
  if (c->prof) return set_error(DGB_ERR_UNSUPPORTED, "profiling times eager launches: use dgb_advance");
  DGB_CUDA(cudaSetDevice(c->device));
  const bool cfl = !(dt > 0);
  const int si = scheme == DGB_RK4 ? 1 : 0, mi = cfl ? 1 : 0;
  if (!c->hl_st[0]) {
    for (auto& st : c->hl_st) DGB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    for (auto& e : c->hl_up) DGB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto& e : c->hl_down) DGB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto& e : c->hl_conv) DGB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    DGB_CUDA(cudaEventCreateWithFlags(&c->hl_done, cudaEventDisableTiming));
  }
  if (nsteps > 0)
    if (int rc = ensure_step_graphs(c, scheme, cfl)) return rc;
  if (int rc = reset_scalars(c, cfl ? 0.0 : dt)) return rc;
  c->ind_step = 0;  // the state comes from the host: the learned indicator scores the first step
  const size_t per = (size_t)c->nf * c->ns;  // values per element in the reference layout
  const int nch = std::min(c->host_chunks, c->ne);
  auto first = [&](int j) { return (int)((long long)c->ne * j / nch); };
  cudaStream_t up = c->hl_st[0], down = c->hl_st[1];
  DGB_CUDA(cudaEventRecord(c->e0, c->st));
  DGB_CUDA(cudaStreamWaitEvent(up, c->e0, 0));  // the copies follow the work queued before the call
  DGB_CUDA(cudaStreamWaitEvent(down, c->e0, 0));
  long long launches = 0;
  for (int s = 0; s < nsteps; ++s) {
    for (int j = 0; j < nch; ++j) {
      const int e0 = first(j), n = first(j + 1) - e0;
      if (s > 0) DGB_CUDA(cudaStreamWaitEvent(up, c->hl_down[j], 0));  // the last step's result is in U
      DGB_CUDA(cudaMemcpyAsync(c->ref + e0 * per, U + e0 * per, n * per * sizeof(double), cudaMemcpyHostToDevice, up));
      DGB_CUDA(cudaEventRecord(c->hl_up[j], up));
      DGB_CUDA(cudaStreamWaitEvent(c->st, c->hl_up[j], 0));
      if (int rc = convert_range(c, true, c->ref, c->A, e0, n)) return rc;
    }
    const int k = !c->ind_on || c->ind_every <= 1 || c->ind_step % c->ind_every == 0 ? 0 : 1;
    DGB_CUDA(cudaGraphLaunch(c->graphs[si][mi][k], c->st));
    launches += c->graph_launches[si][mi][k] + 2 * nch;
    ++c->ind_step;
    for (int j = 0; j < nch; ++j) {  // each chunk's download starts once it is converted
      const int e0 = first(j), n = first(j + 1) - e0;
      if (int rc = convert_range(c, false, c->A, c->ref, e0, n)) return rc;
      DGB_CUDA(cudaEventRecord(c->hl_conv[j], c->st));
      DGB_CUDA(cudaStreamWaitEvent(down, c->hl_conv[j], 0));
      DGB_CUDA(cudaMemcpyAsync(U + e0 * per, c->ref + e0 * per, n * per * sizeof(double), cudaMemcpyDeviceToHost, down));
      DGB_CUDA(cudaEventRecord(c->hl_down[j], down));
    }
  }
  DGB_CUDA(cudaEventRecord(c->hl_done, down));  // the context's stream waits for the last download
  DGB_CUDA(cudaStreamWaitEvent(c->st, c->hl_done, 0));
  DGB_CUDA(cudaEventRecord(c->e1, c->st));
  c->last_launches = launches;
  return step_status(c, time);
}

// ------------------------------------------------------------------------------------------
// Slab mode: a y-slab of a larger structured grid with ghost rows, stepped phase by phase so that
// the caller can exchange the ghost rows between the stages (the reference's ghost exchange,
// COMMUNICATOR::CommunicateGhosts before every residual and limiter pass, rk.cc:108-114, 173,
// 203-209, done here per slab boundary instead of per ghost element)
// ------------------------------------------------------------------------------------------
extern "C" int dgb_slab_ghost_rows(dgb_ctx* c, int lo, int hi) {
  if (!c) return set_error(DGB_ERR_ARG, "null context");
  if (!c->rowmajor) return set_error(DGB_ERR_UNSUPPORTED, "slab mode needs a structured row-major 2D grid");
  const int owned = c->ny - lo - hi;
  if (lo < 0 || hi < 0 || owned < 1 || owned < lo || owned < hi)
    return set_error(DGB_ERR_ARG, "ghost rows: 0 <= lo, hi and at least max(lo, hi, 1) owned rows");
  if (c->ind_on) return set_error(DGB_ERR_UNSUPPORTED, "slab mode does not take the learned indicator");
  if (c->limiter != DGB_LIM_NONE && c->limiter != DGB_LIM_HRL && c->limiter != DGB_LIM_M2L &&
      c->limiter != DGB_LIM_PRL)
    return set_error(DGB_ERR_UNSUPPORTED, "slab mode: the sensors follow the reference's sequential element order, "
                                          "which no ghost depth reproduces; use none, hrl, m2l or prl");
  c->halo_lo = lo;
  c->halo_hi = hi;
  c->drop_graphs();  // captured steps (own and multi-slab) hold the old rows
  return DGB_OK;
}

namespace {
int nstages(int scheme) { return scheme == DGB_RK4 ? 4 : 3; }
double* slab_state(dgb_ctx* c) { return c->slab_cur ? c->slab_cur : c->A; }
}  // namespace

extern "C" int dgb_set_cfl_scale(dgb_ctx* c, double cfl_scaled) {
  if (!c) return set_error(DGB_ERR_ARG, "null context");
  if (!std::isfinite(cfl_scaled)) return set_error(DGB_ERR_ARG, "CFL scale must be finite");
  c->cs.cfl_scaled = cfl_scaled;
  c->drop_graphs();  // captured steps hold the old value
  return DGB_OK;
}

extern "C" int dgb_step_begin(dgb_ctx* c, int scheme, double dt) {
  if (!c) return set_error(DGB_ERR_ARG, "null context");
  if (scheme != DGB_SSPRK3 && scheme != DGB_RK4) return set_error(DGB_ERR_ARG, "scheme must be 3 or 4");
  if (!(dt > 0) && !(c->cs.cfl_scaled > 0)) return set_error(DGB_ERR_ARG, "no fixed dt and no positive CFL");
  if (c->ind_on) return set_error(DGB_ERR_UNSUPPORTED, "the phase-level step does not take the learned indicator");
  if (c->slab_next >= 0) return set_error(DGB_ERR_ARG, "a step is already open (dgb_step_end first)");
  DGB_CUDA(cudaSetDevice(c->device));
  c->slab_cfl = !(dt > 0);
  if (int rc = reset_scalars(c, c->slab_cfl ? 0.0 : dt)) return rc;
  c->slab_scheme = scheme;
  c->slab_next = 0;
  c->slab_cur = c->A;
  c->counter = 0;
  DGB_CUDA(cudaEventRecord(c->e0, c->st));
  if (c->slab_cfl) {
    ProfScope ps(c, KC_DT);
    launch_wavespeed(c, c->A);  // owned rows only
  }
  DGB_CUDA(cudaGetLastError());
  return DGB_OK;
}

extern "C" int dgb_step_wavespeed_word(dgb_ctx* c, void** umax_dev) {
  if (!c || !umax_dev) return set_error(DGB_ERR_ARG, "null argument");
  *umax_dev = &c->scal->umax;
  return DGB_OK;
}

extern "C" int dgb_step_stage(dgb_ctx* c, int k) {
  if (!c) return set_error(DGB_ERR_ARG, "null context");
  if (c->slab_next < 0 || k != c->slab_next || k >= nstages(c->slab_scheme))
    return set_error(DGB_ERR_ARG, "stages run in order 0.. after dgb_step_begin");
  if (k == 0) {
    {
      ProfScope ps(c, KC_DT);
      finish_dt_kernel<<<1, 1, 0, c->st>>>(c->scal, c->cs.cfl_scaled);
    }
    if (c->slab_scheme == DGB_RK4)
      DGB_CUDA(cudaMemcpyAsync(c->B, c->A, c->nstate * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  }
  int rc;
  if (c->slab_scheme == DGB_RK4) {
    rc = rk4_stage(c, k);
    c->slab_cur = k < 3 ? c->C : c->A;
  } else {
    rc = ssp_stage(c, k);
    c->slab_cur = k == 0 ? c->B : (k == 1 ? c->C : c->A);
  }
  if (rc) return rc;
  c->slab_next = k + 1;
  DGB_CUDA(cudaGetLastError());
  return DGB_OK;
}

extern "C" int dgb_step_end(dgb_ctx* c, double* time) {
  if (!c) return set_error(DGB_ERR_ARG, "null context");
  if (c->slab_next != nstages(c->slab_scheme)) return set_error(DGB_ERR_ARG, "the step's stages have not all run");
  c->slab_next = -1;
  c->slab_cur = nullptr;
  DGB_CUDA(cudaEventRecord(c->e1, c->st));
  if (int rc = read_scalars(c)) return rc;
  float ms = 0;
  cudaEventElapsedTime(&ms, c->e0, c->e1);
  c->last_ms = ms;
  c->last_launches = c->counter;
  if (time) *time += c->h_scal->time;
  if (c->h_scal->flags & FLAG_TIMEOUT) return set_error(DGB_ERR_TIMEOUT, "a bounded device wait expired");
  if (c->h_scal->flags & FLAG_NONFINITE) return set_error(DGB_ERR_NONFINITE, "time step is NaN");
  if (c->h_scal->flags & FLAG_DT_SMALL) return set_error(DGB_ERR_DT_SMALL, "next time step is too small (< 1e-14)");
  return DGB_OK;
}

extern "C" int dgb_halo_count(dgb_ctx* c, int side, size_t* n) {
  if (!c || !n) return set_error(DGB_ERR_ARG, "null argument");
  if (side != 0 && side != 1) return set_error(DGB_ERR_ARG, "side is 0 (bottom) or 1 (top)");
  *n = (size_t)(side == 0 ? c->halo_lo : c->halo_hi) * c->nx * c->nf * c->ns;
  return DGB_OK;
}

// rows r0 .. r0 + g - 1 of every (field, node) plane <-> buf[(plane * g + row) * nx + col]
static int halo_copy(dgb_ctx* c, int r0, int g, double* buf, bool pack) {
  double* U = slab_state(c);
  const size_t w = (size_t)g * c->nx * sizeof(double), planes = (size_t)c->nf * c->ns;
  if (g == 0) return DGB_OK;
  DGB_CUDA(cudaSetDevice(c->device));
  if (pack)
    DGB_CUDA(cudaMemcpy2DAsync(buf, w, U + (size_t)r0 * c->nx, (size_t)c->ld * sizeof(double), w, planes,
                               cudaMemcpyDeviceToDevice, c->st));
  else
    DGB_CUDA(cudaMemcpy2DAsync(U + (size_t)r0 * c->nx, (size_t)c->ld * sizeof(double), buf, w, w, planes,
                               cudaMemcpyDeviceToDevice, c->st));
  return DGB_OK;
}

extern "C" int dgb_halo_pack(dgb_ctx* c, int side, double* dst_dev) {
  if (!c || !dst_dev) return set_error(DGB_ERR_ARG, "null argument");
  if (side != 0 && side != 1) return set_error(DGB_ERR_ARG, "side is 0 (bottom) or 1 (top)");
  // the owned rows next to the side, as many as that side has ghost rows
  return side == 0 ? halo_copy(c, c->halo_lo, c->halo_lo, dst_dev, true)
                   : halo_copy(c, c->ny - 2 * c->halo_hi, c->halo_hi, dst_dev, true);
}

extern "C" int dgb_halo_unpack(dgb_ctx* c, int side, const double* src_dev) {
  if (!c || !src_dev) return set_error(DGB_ERR_ARG, "null argument");
  if (side != 0 && side != 1) return set_error(DGB_ERR_ARG, "side is 0 (bottom) or 1 (top)");
  double* src = const_cast<double*>(src_dev);
  return side == 0 ? halo_copy(c, 0, c->halo_lo, src, false) : halo_copy(c, c->ny - c->halo_hi, c->halo_hi, src, false);
}

// ------------------------------------------------------------------------------------------
// Slab mode in one process: every slab context of the grid on this device, advanced together by one
// CUDA graph per step.  The graph holds every slab's CFL reduction, the MAX of their wave speeds,
// and per stage the halo exchange (each slab packs the owned rows next to its ghost sides into its
// own send buffer, each slab then copies its neighbours' send buffers into its ghost rows) and the
// stage itself.  Ordering is by graph edges only: a slab unpacks after its neighbours packed, and
// packs again after its neighbours unpacked.  Captured once per (slabs, scheme, CFL / fixed step),
// dropped when any slab's own captured steps are.
namespace {
constexpr int kMaxLocalSlabs = 16;
struct SlabGraph {
  std::vector<dgb_ctx*> ctx;
  std::vector<unsigned> gen;
  int scheme = 0;
  bool cfl = false, periodic = false;
  cudaGraphExec_t exec = nullptr;
  long long launches = 0;
};
std::vector<SlabGraph> g_slab_graphs;
std::mutex g_slab_mutex;  // guards g_slab_graphs (calls on different slab sets may come from several threads)

struct UmaxWords {
  unsigned long long* w[kMaxLocalSlabs];
  int n;
};
// MAX of the slabs' wave-speed words (bits of non-negative doubles order as integers), written back
// to every word
__global__ void umax_all_kernel(UmaxWords p) {
  unsigned long long m = 0;
  for (int i = 0; i < p.n; ++i) m = max(m, *p.w[i]);
  for (int i = 0; i < p.n; ++i) *p.w[i] = m;
}

int slab_below(int i, int n, bool periodic) { return i > 0 ? i - 1 : (periodic && n > 1 ? n - 1 : -1); }
int slab_above(int i, int n, bool periodic) { return i < n - 1 ? i + 1 : (periodic && n > 1 ? 0 : -1); }

// one step of all slabs into a graph, captured from the first slab's stream
int capture_slab_step(dgb_ctx* const* s, int n, bool periodic, int scheme, bool cfl, cudaGraphExec_t* exec,
                      long long* launches) {
  cudaStream_t s0 = s[0]->st;
  std::vector<cudaEvent_t> ev(3 * n + 1, nullptr);
  for (auto& e : ev) DGB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaEvent_t fork = ev[3 * n];
  auto destroy_events = [&]() { for (auto e : ev) cudaEventDestroy(e); };
  DGB_CUDA(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
  const int rc = [&]() -> int {
    auto fork_all = [&]() -> int {
      DGB_CUDA(cudaEventRecord(fork, s0));
      for (int i = 1; i < n; ++i) DGB_CUDA(cudaStreamWaitEvent(s[i]->st, fork, 0));
      return DGB_OK;
    };
    auto join_all = [&]() -> int {
      for (int i = 1; i < n; ++i) {
        DGB_CUDA(cudaEventRecord(ev[i], s[i]->st));
        DGB_CUDA(cudaStreamWaitEvent(s0, ev[i], 0));
      }
      return DGB_OK;
    };
    auto after = [&](int i, cudaEvent_t* set, int nb) -> int {  // stream of slab i waits for set[nb]
      if (nb >= 0 && nb != i) DGB_CUDA(cudaStreamWaitEvent(s[i]->st, set[nb], 0));
      return DGB_OK;
    };
    if (int r = fork_all()) return r;
    for (int i = 0; i < n; ++i) {
      dgb_ctx* c = s[i];
      c->counter = 0;
      c->slab_scheme = scheme;
      c->slab_next = 0;
      c->slab_cur = c->A;
      c->slab_cfl = cfl;
      if (cfl) launch_wavespeed(c, c->A);  // owned rows only
    }
    if (cfl && n > 1) {
      if (int r = join_all()) return r;
      UmaxWords w{};
      w.n = n;
      for (int i = 0; i < n; ++i) w.w[i] = &s[i]->scal->umax;
      umax_all_kernel<<<1, 1, 0, s0>>>(w);
      ++s[0]->counter;
      DGB_CUDA(cudaGetLastError());
      if (int r = fork_all()) return r;
    }
    cudaEvent_t* packed = ev.data();
    cudaEvent_t* unpacked = ev.data() + n;
    for (int k = 0; k < nstages(scheme); ++k) {
      for (int i = 0; i < n; ++i) {
        dgb_ctx* c = s[i];
        if (int r = halo_copy(c, c->halo_lo, c->halo_lo, c->halo_send[0], true)) return r;
        if (int r = halo_copy(c, c->ny - 2 * c->halo_hi, c->halo_hi, c->halo_send[1], true)) return r;
        DGB_CUDA(cudaEventRecord(packed[i], c->st));
      }
      for (int i = 0; i < n; ++i) {
        dgb_ctx* c = s[i];
        const int b = slab_below(i, n, periodic), a = slab_above(i, n, periodic);
        if (int r = after(i, packed, b)) return r;
        if (int r = after(i, packed, a)) return r;
        if (b >= 0)
          if (int r = halo_copy(c, 0, c->halo_lo, s[b]->halo_send[1], false)) return r;
        if (a >= 0)
          if (int r = halo_copy(c, c->ny - c->halo_hi, c->halo_hi, s[a]->halo_send[0], false)) return r;
        DGB_CUDA(cudaEventRecord(unpacked[i], c->st));
      }
      for (int i = 0; i < n; ++i) {  // the neighbours have read this slab's send buffers
        if (int r = after(i, unpacked, slab_below(i, n, periodic))) return r;
        if (int r = after(i, unpacked, slab_above(i, n, periodic))) return r;
      }
      for (int i = 0; i < n; ++i)
        if (int r = dgb_step_stage(s[i], k)) return r;
    }
    return join_all();
  }();
  cudaGraph_t g = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(s0, &g);
  long long nl = 0;
  for (int i = 0; i < n; ++i) {
    nl += s[i]->counter;
    s[i]->slab_next = -1;
    s[i]->slab_cur = nullptr;
  }
  destroy_events();
  if (rc || ec != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    if (rc) return rc;
    return set_error(DGB_ERR_CUDA, std::string("slab step capture: ") + cudaGetErrorString(ec));
  }
  const cudaError_t ei = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) return set_error(DGB_ERR_CUDA, std::string("slab step graph: ") + cudaGetErrorString(ei));
  *launches = nl;
  return DGB_OK;
}
}  // namespace

namespace {
// (g_slab_mutex held) every captured slab step that involves c
void drop_slab_graphs_locked(dgb_ctx* c) {
  for (size_t i = 0; i < g_slab_graphs.size();) {
    SlabGraph& g = g_slab_graphs[i];
    if (std::find(g.ctx.begin(), g.ctx.end(), c) != g.ctx.end()) {
      // replays run on the first slab's stream and use every slab's buffers: let them finish
      cudaStreamSynchronize(g.ctx[0]->st);
      if (g.exec) cudaGraphExecDestroy(g.exec);
      g_slab_graphs.erase(g_slab_graphs.begin() + i);
    } else {
      ++i;
    }
  }
}
}  // namespace

void dgb::drop_slab_graphs(dgb_ctx* c) {
  std::lock_guard<std::mutex> lock(g_slab_mutex);
  drop_slab_graphs_locked(c);
}

extern "C" int dgb_slabs_advance_local(dgb_ctx* const* slabs, int n, int periodic, int scheme, int nsteps, double dt,
                                       double* time) {
  if (!slabs || n < 1 || n > kMaxLocalSlabs) return set_error(DGB_ERR_ARG, "1 to 16 slab contexts");
  if (scheme != DGB_SSPRK3 && scheme != DGB_RK4) return set_error(DGB_ERR_ARG, "scheme must be 3 or 4");
  if (nsteps < 0) return set_error(DGB_ERR_ARG, "nsteps < 0");
  const bool cfl = !(dt > 0), per = periodic != 0;
  for (int i = 0; i < n; ++i) {
    dgb_ctx* c = slabs[i];
    if (!c) return set_error(DGB_ERR_ARG, "null slab context");
    if (c->device != slabs[0]->device) return set_error(DGB_ERR_ARG, "the slabs of a local run share one device");
    if (c->nx != slabs[0]->nx || c->nf != slabs[0]->nf || c->ns != slabs[0]->ns)
      return set_error(DGB_ERR_ARG, "the slabs of one grid have the same nx, fields and nodes");
    for (int j = 0; j < i; ++j)
      if (slabs[j] == c) return set_error(DGB_ERR_ARG, "a slab context appears twice");
    if (c->ind_on) return set_error(DGB_ERR_UNSUPPORTED, "slab mode does not take the learned indicator");
    if (c->slab_next >= 0) return set_error(DGB_ERR_ARG, "a phase-level step is open on a slab");
    if (c->prof) return set_error(DGB_ERR_UNSUPPORTED, "profiling times eager launches: use the phase-level step");
    if (cfl && !(c->cs.cfl_scaled > 0)) return set_error(DGB_ERR_ARG, "no fixed dt and no positive CFL");
    const int b = slab_below(i, n, per), a = slab_above(i, n, per);
    if ((b < 0) != (c->halo_lo == 0) || (a < 0) != (c->halo_hi == 0) || (b >= 0 && slabs[b]->halo_hi != c->halo_lo) ||
        (a >= 0 && slabs[a]->halo_lo != c->halo_hi))
      return set_error(DGB_ERR_ARG, "ghost rows do not match the slab order (dgb_slab_ghost_rows)");
  }
  DGB_CUDA(cudaSetDevice(slabs[0]->device));
  for (int i = 0; i < n; ++i)
    for (int side = 0; side < 2; ++side) {
      dgb_ctx* c = slabs[i];
      const int g = side == 0 ? c->halo_lo : c->halo_hi;
      if (g && !c->halo_send[side])
        DGB_CUDA(cudaMalloc(&c->halo_send[side], (size_t)g * c->nx * c->nf * c->ns * sizeof(double)));
    }
  std::lock_guard<std::mutex> lock(g_slab_mutex);
  for (int i = 0; i < n; ++i) {  // captures that hold a slab whose own captured steps were dropped since
    bool stale = false;
    for (const auto& g : g_slab_graphs)
      for (size_t j = 0; j < g.ctx.size(); ++j)
        if (g.ctx[j] == slabs[i] && g.gen[j] != slabs[i]->graph_gen) stale = true;
    if (stale) drop_slab_graphs_locked(slabs[i]);
  }
  SlabGraph* sg = nullptr;
  for (auto& g : g_slab_graphs) {
    if (g.scheme != scheme || g.cfl != cfl || g.periodic != per || (int)g.ctx.size() != n) continue;
    bool same = true;
    for (int i = 0; i < n && same; ++i) same = g.ctx[i] == slabs[i] && g.gen[i] == slabs[i]->graph_gen;
    if (same) { sg = &g; break; }
  }
  if (!sg && nsteps > 0) {
    SlabGraph g;
    g.ctx.assign(slabs, slabs + n);
    for (int i = 0; i < n; ++i) g.gen.push_back(slabs[i]->graph_gen);
    g.scheme = scheme;
    g.cfl = cfl;
    g.periodic = per;
    if (int rc = capture_slab_step(slabs, n, per, scheme, cfl, &g.exec, &g.launches)) return rc;
    g_slab_graphs.push_back(g);
    sg = &g_slab_graphs.back();
  }
  dgb_ctx* c0 = slabs[0];
  // every slab's scalars reset once (flags clear, time 0, the fixed step), then the steps replayed
  // on the first slab's stream; the other streams wait for it before their next work
  for (int i = 0; i < n; ++i) {
    if (int rc = reset_scalars(slabs[i], cfl ? 0.0 : dt)) return rc;
    if (i) {
      DGB_CUDA(cudaEventRecord(slabs[i]->e0, slabs[i]->st));
      DGB_CUDA(cudaStreamWaitEvent(c0->st, slabs[i]->e0, 0));
    }
  }
  DGB_CUDA(cudaEventRecord(c0->e0, c0->st));
  for (int s = 0; s < nsteps; ++s) DGB_CUDA(cudaGraphLaunch(sg->exec, c0->st));
  DGB_CUDA(cudaEventRecord(c0->e1, c0->st));
  for (int i = 1; i < n; ++i) DGB_CUDA(cudaStreamWaitEvent(slabs[i]->st, c0->e1, 0));
  unsigned flags = 0;
  for (int i = 0; i < n; ++i) {
    if (int rc = read_scalars(slabs[i])) return rc;
    flags |= slabs[i]->h_scal->flags;
  }
  float ms = 0;
  cudaEventElapsedTime(&ms, c0->e0, c0->e1);
  c0->last_ms = ms;
  c0->last_launches = sg ? sg->launches * nsteps : 0;
  if (time) *time += c0->h_scal->time;
  if (flags & FLAG_TIMEOUT) return set_error(DGB_ERR_TIMEOUT, "a bounded device wait expired");
  if (flags & FLAG_NONFINITE) return set_error(DGB_ERR_NONFINITE, "time step is NaN");
  if (flags & FLAG_DT_SMALL) return set_error(DGB_ERR_DT_SMALL, "next time step is too small (< 1e-14)");
  return DGB_OK;
}

extern "C" int dgb_stream(dgb_ctx* c, void** stream) {
  if (!c || !stream) return set_error(DGB_ERR_ARG, "null argument");
  *stream = (void*)c->st;
  return DGB_OK;
}

extern "C" int dgb_last_dt(dgb_ctx* c, double* dt) {
  if (!c || !dt) return set_error(DGB_ERR_ARG, "null argument");
  *dt = c->h_scal->dt;
  return DGB_OK;
}

extern "C" int dgb_last_timing(dgb_ctx* c, double* ms, long long* launches) {
  if (!c) return set_error(DGB_ERR_ARG, "null context");
  if (ms) *ms = c->last_ms;
  if (launches) *launches = c->last_launches;
  return DGB_OK;
}

extern "C" int dgb_set_profiling(dgb_ctx* c, int on) {
  if (!c) return set_error(DGB_ERR_ARG, "null context");
  c->prof = on != 0;
  for (int k = 0; k < KC_N; ++k) { c->kc_ms[k] = 0; c->kc_n[k] = 0; }
  return DGB_OK;
}

extern "C" int dgb_kernel_timing(dgb_ctx* c, const char* name, double* ms, long long* launches) {
  if (!c || !name) return set_error(DGB_ERR_ARG, "null argument");
  const std::string n = name;
  int k = n == "residual" ? KC_RESIDUAL : n == "limiter" ? KC_LIMITER : n == "dt" ? KC_DT
          : n == "indicator" ? KC_INDICATOR : n == "other" ? KC_OTHER : -1;
  if (k < 0) return set_error(DGB_ERR_ARG, "unknown kernel class " + n);
  if (ms) *ms = c->kc_ms[k];
  if (launches) *launches = c->kc_n[k];
  return DGB_OK;
}

extern "C" int dgb_conservation(dgb_ctx* c, double* totals) {
  if (!c || !totals) return set_error(DGB_ERR_ARG, "null argument");
  // integral of each field: sum_e sum_i U_i * (J * int phi_i) ; computed on the host from a
  // state download (diagnostic only, as DG_SOLVER::conservation is)
  std::vector<double> U((size_t)c->ne * c->nf * c->ns);
  if (int rc = dgb_get_state(c, U.data())) return rc;
  // int phi_i over the reference element, tensor factors from the volume quadrature
  const Consts& cs = c->cs;
  std::vector<double> w1(cs.n1, 0.0);
  for (int i = 0; i < cs.n1; ++i)
    for (int g = 0; g < cs.ng1; ++g) w1[i] += cs.wq[g] * cs.Bq[g][i];
  std::vector<int> perm(c->ns);
  cudaMemcpy(perm.data(), c->perm, c->ns * sizeof(int), cudaMemcpyDeviceToHost);
  for (int f = 0; f < c->nf; ++f) totals[f] = 0.0;
  for (int e = 0; e < c->ne; ++e)
    for (int f = 0; f < c->nf; ++f)
      for (int t = 0; t < c->ns; ++t) {
        const int ix = t % cs.n1, iy = t / cs.n1;
        const double w = c->D == 2 ? w1[ix] * w1[iy] : w1[ix];
        totals[f] += U[((size_t)e * c->nf + f) * c->ns + perm[t]] * w * cs.J;
      }
  return DGB_OK;
}
