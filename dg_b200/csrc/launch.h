// Launch helpers shared by the translation units that launch the tiled 2D kernels (dgb_device.cu,
// dgb_device_ny.cu): programmatic launches, the tile shapes, the stage's kernel arguments.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <utility>

#include "ctx.h"
#include "device/kernels.cuh"
#include "device/tile2d.cuh"

namespace dgb {

// A launch on the context's stream, programmatic (the kernel may be scheduled while its predecessor
// finishes; it waits in pdl_wait) when the context allows it.  Only kernels that call pdl_wait
// before touching global data are launched this way.
template <typename... KArgs, typename... Args>
void launch_pdl(dgb_ctx* c, void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c->st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = c->pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
}

constexpr int TILE_W = 32, TILE_H = 4;
// p = 3 tiles are two element rows high: the per-element register state (80 nodal values per
// field set) and the shared tile then leave room for two (FP64) or three (mixed) CTAs per SM
// (and with more than three mass fractions, whose fields would not leave room for a 32 x 4 tile)
constexpr int tile_h_for(int p, int ny = 0) { return p == 3 || ny > 3 ? 2 : TILE_H; }

inline const CUtensorMap& map_of(dgb_ctx* c, const double* p) {
  if (p == c->B) return c->mapB;
  if (p == c->C) return c->mapC;
  return c->mapA;
}

// kernel arguments of the tiled residuals for one stage
inline TileArgs tile_args(dgb_ctx* c, const StageArgs& s) {
  TileArgs a;
  a.U = s.U; a.Ubase = s.Ubase; a.out = s.out; a.Uacc = s.Uacc; a.nbr = s.nbr; a.scal = s.scal;
  a.errflag = &c->scal->flags;
  a.polls = c->wait_polls;
  a.a = s.a; a.b = s.b; a.dt_override = s.dt_override;
  a.J = c->cs.J;
  a.invJ = 1.0 / c->cs.J;
  a.cx = c->cs.J * c->cs.ixx;
  a.cy = c->cs.J * c->cs.iyy;
  a.sx = c->cs.ixx;
  a.sy = c->cs.iyy;
  a.JFx = c->cs.JFx;
  a.JFy = c->cs.JFy;
  a.nx = c->nx; a.ny = c->ny; a.ld = c->ld;
  return a;
}

template <int P, int FLUX, int MODE, int NY = 0, bool GC = false, bool TMA = true>
void launch_tile2d(dgb_ctx* c, const StageArgs& s) {
  constexpr int TH = tile_h_for(P, NY);
  using Dm = TileDims<P, TILE_W, TH, NY>;
  constexpr size_t smem = Dm::smem_bytes;
  auto k = residual2d_tile_kernel<P, FLUX, MODE, TILE_W, TH, NY, GC, TMA>;
  allow_dynamic_smem(k, smem);
  const TileArgs a = tile_args(c, s);
  // (without TMA the maps are not read: the tile loads are plain)
  const CUtensorMap& mu = TMA ? map_of(c, s.U) : c->mapA;
  const CUtensorMap& mb = !TMA ? c->mapA
                          : MODE == MODE_SSP ? map_of(c, s.Ubase) : MODE == MODE_RK4 && s.Uacc ? map_of(c, s.Uacc) : mu;
  dim3 grid(c->nx / TILE_W, c->ny / TH);
  ProfScope ps(c, KC_RESIDUAL);
  launch_pdl(c, k, grid, dim3(TILE_W * TH), smem, a, mu, mb);
}

constexpr int RES2D_TE = 16;
constexpr int RES2D_NT = 256;

// generic 2D residual over every element, or over the listed ones (elist, n)
template <int P, int FLUX, int MODE, int NY = 0, bool GC = false>
void launch_res2d(dgb_ctx* c, const StageArgs& a, const int* elist = nullptr, int n = 0) {
  constexpr size_t smem = residual2d_smem_doubles<P, RES2D_TE, NY, GC>() * sizeof(double);
  auto k = residual2d_kernel<P, FLUX, MODE, RES2D_TE, RES2D_NT, NY, GC>;
  allow_dynamic_smem(k, smem);
  StageArgs s = a;
  s.elist = elist;
  s.nlist = n;
  const int grid = ((elist ? n : c->ne) + RES2D_TE - 1) / RES2D_TE;
  ProfScope ps(c, KC_RESIDUAL);
  k<<<grid, RES2D_NT, smem, c->st>>>(c->cs, s);
}

}  // namespace dgb
