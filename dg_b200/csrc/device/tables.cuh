// Reference-element tables in __constant__ memory: the limiter's monomial transforms and
// integrals (c_lim_p*) and the tensor-product tables of the 2D tiled residual kernels (c_tab2_p*,
// FP32 copies c_tab2f_p*), and in global memory the lane tables of the p = 2 DMMA residual
// (g_dmma_tab2).  Those symbols are static, one copy per translation unit (each .cu file
// is its own device module), so every .cu file that launches kernels reading them calls
// upload_tables from its own code; the function is static for the same reason.
#pragma once
#include <cuda_runtime.h>

#include <cstring>
#include <string>
#include <vector>

#include "../host/host.h"
#include "common.cuh"
#include "tile2d.cuh"
#include "tile2d_dmma.cuh"
#include "tile2d_mixed.cuh"

namespace dgb {

int set_error(int code, const std::string& msg);

template <int P>
static Tab2<P> make_tab2(const Consts& c) {
  Tab2<P> T;
  std::memset(&T, 0, sizeof(T));
  constexpr int N1 = Tab2<P>::N1, NG1 = Tab2<P>::NG1;
  for (int gx = 0; gx < NG1; ++gx)
    for (int gy = 0; gy < NG1; ++gy) {
      const int g = gx * NG1 + gy;
      T.W[g] = c.wq[gx] * c.wq[gy];
      for (int iy = 0; iy < N1; ++iy)
        for (int ix = 0; ix < N1; ++ix) {
          const int t = ix + N1 * iy;
          T.Phi[g][t] = c.Bq[gx][ix] * c.Bq[gy][iy];
          T.dPx[g][t] = c.Dq[gx][ix] * c.Bq[gy][iy];
          T.dPy[g][t] = c.Bq[gx][ix] * c.Dq[gy][iy];
        }
    }
  for (int g = 0; g < N1; ++g) {
    T.wf[g] = c.wf[g];
    for (int j = 0; j < N1; ++j) T.Bf[g][j] = c.Bf[g][j];
  }
  for (int g = 0; g < NG1; ++g) {
    T.W1[g] = c.wq[g];
    for (int i = 0; i < N1; ++i) { T.B1[g][i] = c.Bq[g][i]; T.D1[g][i] = c.Dq[g][i]; }
  }
  std::vector<double> M((size_t)N1 * N1, 0.0);
  for (int i = 0; i < N1; ++i)
    for (int j = 0; j < N1; ++j)
      for (int g = 0; g < NG1; ++g) M[i + (size_t)j * N1] += c.wq[g] * c.Bq[g][i] * c.Bq[g][j];
  invert(M, N1);
  for (int i = 0; i < N1; ++i)
    for (int j = 0; j < N1; ++j) T.M1i[i][j] = M[i + (size_t)j * N1];
  return T;
}

template <int P>
static Tab2f<P> make_tab2f(const Tab2<P>& d) {
  Tab2f<P> T;
  std::memset(&T, 0, sizeof(T));
  constexpr int N1 = Tab2<P>::N1, NG1 = Tab2<P>::NG1, NS = Tab2<P>::NS, NG = Tab2<P>::NG;
  for (int g = 0; g < NG; ++g) {
    T.W[g] = (float)d.W[g];
    for (int t = 0; t < NS; ++t) {
      T.dPx[g][t] = (float)d.dPx[g][t];
      T.dPy[g][t] = (float)d.dPy[g][t];
      T.Phi[g][t] = (float)d.Phi[g][t];
    }
  }
  for (int i = 0; i < N1; ++i) {
    T.wf[i] = (float)d.wf[i];
    for (int j = 0; j < N1; ++j) { T.Bf[i][j] = (float)d.Bf[i][j]; T.M1i[i][j] = (float)d.M1i[i][j]; }
  }
  for (int g = 0; g < NG1; ++g)
    for (int i = 0; i < N1; ++i) { T.B1[g][i] = (float)d.B1[g][i]; T.D1[g][i] = (float)d.D1[g][i]; }
  return T;
}

// Lane tables of the p = 2 DMMA residual (tile2d_dmma.cuh) from the tensor-product tables: the
// lift tables K_x = M^-1 dPx, K_y = M^-1 dPy, K_a = M^-1 Phi and the face table E = M^-1 (Bf wf on
// the face nodes), M^-1 = M1^-1 (x) M1^-1 acting on the node index, laid out per lane.
static DmmaTab2 make_dmma_tab2(const Tab2<2>& d) {
  constexpr int N1 = 3, NS = 9, NG = 16;
  DmmaTab2 T;
  std::memset(&T, 0, sizeof(T));
  double Mi[NS][NS];
  for (int t = 0; t < NS; ++t)
    for (int u = 0; u < NS; ++u) Mi[t][u] = d.M1i[t % N1][u % N1] * d.M1i[t / N1][u / N1];
  double K[3][NG][NS], E[12][NS];
  for (int g = 0; g < NG; ++g)
    for (int t = 0; t < NS; ++t) {
      double sx = 0, sy = 0, sa = 0;
      for (int u = 0; u < NS; ++u) {
        sx += Mi[t][u] * d.dPx[g][u];
        sy += Mi[t][u] * d.dPy[g][u];
        sa += Mi[t][u] * d.Phi[g][u];
      }
      K[0][g][t] = sx;
      K[1][g][t] = sy;
      K[2][g][t] = sa;
    }
  for (int k = 0; k < 12; ++k) {
    const int kf = k / 3, g = k % 3;
    double e0[NS] = {0};
    for (int j = 0; j < N1; ++j) {
      const int t = kf == 0 ? N1 * j : kf == 1 ? 2 + N1 * j : kf == 2 ? j : j + N1 * 2;
      e0[t] = d.Bf[g][j] * d.wf[g];
    }
    for (int t = 0; t < NS; ++t) {
      double s = 0;
      for (int u = 0; u < NS; ++u) s += Mi[t][u] * e0[u];
      E[k][t] = s;
    }
  }
  auto pi = [](int q, int c) { return q < 2 ? 2 * c + q : 8 + 2 * c + (q - 2); };
  const double (*tabs[3])[NS] = {d.Phi, d.dPx, d.dPy};
  for (int l = 0; l < 32; ++l) {
    const int r = l >> 2, c = l & 3;
    for (int tb = 0; tb < 3; ++tb)
      for (int s = 0; s < 2; ++s)
        for (int nb = 0; nb < 2; ++nb) T.col[(tb * 2 + s) * 2 + nb][l] = tabs[tb][8 * nb + r][1 + 4 * s + c];
    for (int dd = 0; dd < 3; ++dd)
      for (int q = 0; q < 4; ++q) T.lift[dd * 4 + q][l] = K[dd][pi(q, c)][r];
    for (int s = 0; s < 3; ++s) T.face[s][l] = E[4 * s + c][r];
  }
  for (int c = 0; c < 4; ++c) {
    for (int dd = 0; dd < 3; ++dd)
      for (int q = 0; q < 4; ++q) T.lift8[dd * 4 + q][c] = K[dd][pi(q, c)][8];
    for (int s = 0; s < 3; ++s) T.face8[s][c] = E[4 * s + c][8];
    for (int q = 0; q < 4; ++q) T.wq[q][c] = d.W[pi(q, c)];
  }
  return T;
}

// Tables of order p (and, in 2D, the tiled kernels' tables) from the problem constants.
static int upload_tables(const Consts& cs, int D, int p) {
  cudaError_t el = cudaSuccess;
  auto fill = [&](auto& t, int n1) {
    std::memset(&t, 0, sizeof(t));
    for (int m = 0; m < n1; ++m)
      for (int i = 0; i < n1; ++i) {
        t.T[m][i] = cs.T[m][i];
        t.Tinv[m][i] = cs.Tinv[m][i];
        t.imd[m][i] = cs.imd[m][i];
        t.imdL[m][i] = cs.imdL[m][i];
        t.imdR[m][i] = cs.imdR[m][i];
      }
    for (int k = 0; k < n1 + 2; ++k) t.ifact[k] = cs.ifact[k];
  };
  if (p == 1) { LimTab<1> t; fill(t, 2); el = cudaMemcpyToSymbol(c_lim_p1, &t, sizeof(t)); }
  if (p == 2) { LimTab<2> t; fill(t, 3); el = cudaMemcpyToSymbol(c_lim_p2, &t, sizeof(t)); }
  if (p == 3) { LimTab<3> t; fill(t, 4); el = cudaMemcpyToSymbol(c_lim_p3, &t, sizeof(t)); }
  if (el != cudaSuccess) return set_error(5, std::string("limiter tables: ") + cudaGetErrorString(el));
  if (D == 2) {
    cudaError_t et = cudaSuccess;
    if (p == 1) {
      auto t = make_tab2<1>(cs);
      auto tf = make_tab2f<1>(t);
      et = cudaMemcpyToSymbol(c_tab2_p1, &t, sizeof(t));
      if (et == cudaSuccess) et = cudaMemcpyToSymbol(c_tab2f_p1, &tf, sizeof(tf));
    }
    if (p == 2) {
      auto t = make_tab2<2>(cs);
      auto tf = make_tab2f<2>(t);
      et = cudaMemcpyToSymbol(c_tab2_p2, &t, sizeof(t));
      if (et == cudaSuccess) et = cudaMemcpyToSymbol(c_tab2f_p2, &tf, sizeof(tf));
      if (et == cudaSuccess) {
        const DmmaTab2 td = make_dmma_tab2(t);
        et = cudaMemcpyToSymbol(g_dmma_tab2, &td, sizeof(td));
      }
    }
    if (p == 3) {
      auto t = make_tab2<3>(cs);
      auto tf = make_tab2f<3>(t);
      et = cudaMemcpyToSymbol(c_tab2_p3, &t, sizeof(t));
      if (et == cudaSuccess) et = cudaMemcpyToSymbol(c_tab2f_p3, &tf, sizeof(tf));
    }
    if (et != cudaSuccess) return set_error(5, std::string("constant tables: ") + cudaGetErrorString(et));
  }
  return 0;
}

}  // namespace dgb
