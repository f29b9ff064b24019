// Tiled 2D residual + stage update for p = 2 in FP64 with the basis contractions on the FP64 tensor
// cores (mma.sync.aligned.m8n8k4.row.col.f64, "DMMA").
//
// Same tiles, phase 0 (tile_stage_in) and phase 1 (tile_face_fluxes) as residual2d_tile_kernel.  The
// CTA has two warps per element row of the 32 x 4 tile (256 threads), and phase 2 spreads every
// element over four lanes in the m8n8k4 fragment layout: lane l holds A[l>>2][l&3], B[l&3][l>>2] and
// C/D[l>>2][2(l&3) + i].  A warp takes 16 elements of one row as two m-blocks of 8; in every product
// the 8 rows are those elements, and lane l serves element r = l>>2 in column c = l&3:
//   collocation  u(x_g) = u_0 + sum_{t=1..8} (u_t - u_0) T[g][t] (the Lagrange basis sums to one and
//                its derivatives to zero), T = Phi for the five fields and dPx, dPy for alpha;
//                K = the 8 non-anchor nodes in two steps of 4, N = two blocks of 8 points.  Lane
//                (r, c) receives points 2c, 2c+1 (block 0) and 8+2c, 9+2c (block 1) of element r.
//   point terms  weighted fluxes and the alpha source at those four points, by the lane itself
//                (point_terms, the scalar kernel's arithmetic).
//   lift         D[e][t] = sum_k A[e][k] K[k][t] with K the x, y and alpha-source lift tables with
//                M^-1 = M1^-1 (x) M1^-1 folded in.  K step q takes from lane c its own q-th point
//                pi(q, c), so no value moves between lanes; nodes 0..7 by DMMA, node 8 by every lane
//                over its own points and a sum over the four lanes of the element.
//   face lift    the same over the element's 12 face points (3 steps of 4) with the face fluxes of
//                phase 1.
// The accumulators then hold M^-1 R; the stage update reads the stage base from global memory.
// FP64 throughout: the sums run in another order than the scalar kernel's (differences of order
// 1e-16 relative).  No mass fractions, GAMNCON, SSP and RK4 stages.
// Measured on B200 (1024 x 512 stage launch): 15.4 warps per SM against the scalar kernel's 7.8,
// but 298.5 us against 292 us.  The FP64 tensor rate equals the FP64 vector rate (36.9 TFLOP/s for
// both at 8+ warps per SM), so DMMA saves issue slots, not FP64 pipe time; without the scalar
// kernel's sum factorisation the contractions need ~30 % more FMAs, and preparing the fragments
// (tile loads, deviations, table loads, node 8, face gathers) costs what the DMMAs save in DFMA
// instructions.  Kept as an alternative (DGB_TILE_KERNEL=dmma); the scalar kernel is the default.
#pragma once
#include "tile2d.cuh"

namespace dgb {

// Lane tables (lane-minor, so that a warp's 8-byte loads are conflict-free).  pi(q, c) is the q-th
// quadrature point of column c: 2c, 2c+1, 8+2c, 9+2c.
struct DmmaTab2 {
  double col[12][32];   // [(T*2 + s)*2 + nb][l] = T[8 nb + (l>>2)][1 + 4 s + (l&3)], T = Phi, dPx, dPy
  double lift[12][32];  // [d*4 + q][l] = K_d[pi(q, l&3)][l>>2], d = x, y, alpha source
  double face[3][32];   // [s][l] = E[4 s + (l&3)][l>>2]
  double lift8[12][4];  // [d*4 + q][c] = K_d[pi(q, c)][8]
  double face8[3][4];   // [s][c] = E[4 s + c][8]
  double wq[4][4];      // [q][c] = W[pi(q, c)]
};
static __device__ DmmaTab2 g_dmma_tab2;

constexpr int DMMA_THREADS = 256, DMMA_TW = 32, DMMA_TH = 4;
struct DmmaDims {
  using B = TileDims<2, DMMA_TW, DMMA_TH, 0>;
  static constexpr size_t off_tab = (B::smem_bytes + 127) / 128 * 128;
  static constexpr size_t smem_bytes = off_tab + sizeof(DmmaTab2);
};

__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

template <int FLUX, int MODE>
__global__ void __launch_bounds__(DMMA_THREADS, 2)
    residual2d_tile_dmma_kernel(const TileArgs a, const __grid_constant__ CUtensorMap mapU) {
  static_assert(MODE == MODE_SSP || MODE == MODE_RK4, "stage kernels only");
  constexpr int P = 2, TW = DMMA_TW, TH = DMMA_TH;
  using Dm = TileDims<P, TW, TH, 0>;
  constexpr int N1 = Dm::N1, NS = Dm::NS, NF = Dm::NF, NT = Dm::NT, NXF = Dm::NXF, FS = NF + 1;
  extern __shared__ __align__(128) unsigned char smraw[];
  if (a.scal && a.scal->flags) return;
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(reinterpret_cast<uint64_t*>(smraw), 1);
    fence_mbar_init();
  }
  DmmaTab2* T = reinterpret_cast<DmmaTab2*>(smraw + DmmaDims::off_tab);
  {
    const double* src = reinterpret_cast<const double*>(&g_dmma_tab2);
    double* dst = reinterpret_cast<double*>(T);
    for (int k = tid; k < (int)(sizeof(DmmaTab2) / 8); k += DMMA_THREADS) dst[k] = src[k];
  }
  // (the first barrier inside tile_stage_in orders the table stores before their use)
  uint32_t phase = 0;
  const int tx0 = blockIdx.x * TW, ty0 = blockIdx.y * TH;
  if (!tile_stage_in<P, TW, TH, 0, true>(a, &mapU, tx0, ty0, smraw, phase, tid, DMMA_THREADS)) return;

  const double* Us = reinterpret_cast<const double*>(smraw + Dm::off_tile);  // [NF*NS][NT]
  double* HL = reinterpret_cast<double*>(smraw + Dm::off_halo);
  double* HR = HL + TH * NF * N1;
  double* HD = HR + TH * NF * N1;
  double* HU = HD + TW * NF * N1;
  double* Fs = reinterpret_cast<double*>(smraw + Dm::off_face);
  const int* codes = reinterpret_cast<const int*>(smraw + Dm::head_bytes);
  tile_face_fluxes<P, FLUX, TW, TH, 0, false>(Us, HL, HR, HD, HU, codes, Fs, tid, DMMA_THREADS, 0, Dm::NXF + Dm::NYF, 0);
  __syncthreads();

  const int lane = tid & 31, warp = tid >> 5;
  const int r = lane >> 2, c = lane & 3;
  const int ty = warp >> 1, xb = (warp & 1) * 16;
  const double dt = a.dt_override > 0 ? a.dt_override : a.scal->dt;
  const double sc = dt * a.invJ;
#pragma unroll 1
  for (int mb = 0; mb < 2; ++mb) {
    const int tx = xb + 8 * mb + r;
    const int el = ty * TW + tx;
    double acc[NF][2], p8[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) acc[f][0] = acc[f][1] = p8[f] = 0.0;

    // face lift: face point k = 4 s + c of the element (face kf = k / 3: L, R, D, U; point k % 3)
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const int k = 4 * s + c, kf = k / 3, g = k - 3 * kf;
      const int base = kf == 0 ? (tx * TH + ty) * N1
                       : kf == 1 ? ((tx + 1) * TH + ty) * N1
                       : kf == 2 ? NXF + (ty * TW + tx) * N1
                                 : NXF + ((ty + 1) * TW + tx) * N1;
      const double sgn = (kf & 1) ? -1.0 : 1.0, jw = kf < 2 ? a.JFx : a.JFy;
      const double* fp = Fs + (base + g) * FS;
      const double bf = T->face[s][lane], b8 = T->face8[s][c];
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        const double av = (sgn * fp[f] + (f == 4 ? fp[NF] : 0.0)) * jw;
        dmma884(acc[f][0], acc[f][1], av, bf);
        p8[f] = fma(av, b8, p8[f]);
      }
    }

    // volume terms, one block of 8 quadrature points at a time
    double u0[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) u0[f] = Us[(f * NS) * NT + el];
#pragma unroll
    for (int nb = 0; nb < 2; ++nb) {
      double ug[2][NF], dax[2] = {0.0, 0.0}, day[2] = {0.0, 0.0};
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        double d0 = u0[f], d1 = u0[f];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          const double av = Us[(f * NS + 1 + 4 * s + c) * NT + el] - u0[f];
          dmma884(d0, d1, av, T->col[(0 * 2 + s) * 2 + nb][lane]);
          if (f == 4) {
            dmma884(dax[0], dax[1], av, T->col[(1 * 2 + s) * 2 + nb][lane]);
            dmma884(day[0], day[1], av, T->col[(2 * 2 + s) * 2 + nb][lane]);
          }
        }
        ug[0][f] = d0;
        ug[1][f] = d1;
      }
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int q = 2 * nb + i;
        double gxv[4], gyv[4], gs;
        point_terms<NF, 4, 0, false>(ug[i], dax[i], day[i], T->wq[q][c], a, gxv, gyv, gs);
        const double kx = T->lift[0 * 4 + q][lane], ky = T->lift[1 * 4 + q][lane], ka = T->lift[2 * 4 + q][lane];
        const double kx8 = T->lift8[0 * 4 + q][c], ky8 = T->lift8[1 * 4 + q][c], ka8 = T->lift8[2 * 4 + q][c];
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          dmma884(acc[f][0], acc[f][1], gxv[f], kx);
          dmma884(acc[f][0], acc[f][1], gyv[f], ky);
          p8[f] = fma(gxv[f], kx8, fma(gyv[f], ky8, p8[f]));
        }
        dmma884(acc[4][0], acc[4][1], gs, ka);
        p8[4] = fma(gs, ka8, p8[4]);
      }
    }
    // node 8: sum over the element's four lanes
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      p8[f] += __shfl_xor_sync(0xffffffffu, p8[f], 1);
      p8[f] += __shfl_xor_sync(0xffffffffu, p8[f], 2);
    }

    // stage update of nodes 2c, 2c+1 of every field, and of node 8 of field f by lane c = f mod 4
    const size_t e = (size_t)(ty0 + ty) * a.nx + tx0 + tx;
    auto put = [&](int f, int t, double du) {
      const size_t gi = (size_t)(f * NS + t) * a.ld + e;
      if (MODE == MODE_SSP) {
        const double base = a.a != 0.0 ? a.a * __ldg(a.Ubase + gi) : 0.0;
        a.out[gi] = base + a.b * (Us[(f * NS + t) * NT + el] + du);
      } else {
        a.out[gi] = du;
        if (a.Uacc) a.Uacc[gi] = a.Uacc[gi] + a.b * du;
      }
    };
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      put(f, 2 * c, sc * acc[f][0]);
      put(f, 2 * c + 1, sc * acc[f][1]);
      if ((f & 3) == c) put(f, 8, sc * p8[f]);
    }
  }
}

}  // namespace dgb
