// Problems with 4 to 10 passive mass fractions (the reference's MASS = 4 .. 10,
// code/Makefile:32): the residual and the hrl / m2l limiter kernels instantiated for N_Y = 4 .. 10,
// in a translation unit of their own so that they compile beside dgb_device.cu.  Same kernels as
// N_Y <= 3 -- 1D: residual1d_kernel, lim1d_kernel; 2D: the tiled residual on 32 x 2 tiles with the
// faces through one buffer, the tiled limiter passes with their arrays in dynamic shared memory --
// a mass fraction is advected like the density and limited like it (HR: every field; m2: the
// MACRO block of M2limiting).
#include <cuda_runtime.h>

#include <string>

#include "ctx.h"
#include "device/kernels.cuh"
#include "device/limiter2d_tile.cuh"
#include "device/tables.cuh"
#include "launch.h"

namespace dgb {

namespace {

template <int P, int FLUX, int MODE, int NY>
void launch_res1d_ny(dgb_ctx* c, const StageArgs& a) {
  ProfScope ps(c, KC_RESIDUAL);
  residual1d_kernel<P, FLUX, MODE, NY><<<(c->ne + 127) / 128, 128, 0, c->st>>>(c->cs, a);
}

template <int MODE, int NY>
int residual_ny(dgb_ctx* c, const StageArgs& a) {
#define R1(P, F) case P * 10 + F: launch_res1d_ny<P, F, MODE, NY>(c, a); return 0;
  switch (c->p * 10 + c->flux) {
    R1(1, 0) R1(1, 1) R1(1, 2) R1(2, 0) R1(2, 1) R1(2, 2) R1(3, 0) R1(3, 1) R1(3, 2)
    default: return set_error(DGB_ERR_UNSUPPORTED, "no residual kernel for this (p, flux)");
  }
#undef R1
}

template <int P, int METHOD, int NY>
void launch_lim1d_ny(dgb_ctx* c, const double* in, double* out) {
  ProfScope ps(c, KC_LIMITER);
  const LimArgs la{c->ld, c->ne};
  lim1d_kernel<P, METHOD, NY><<<(c->ne + 127) / 128, 128, 0, c->st>>>(la, in, c->nbr, out, c->scal);
}

template <int NY>
int limit_ny(dgb_ctx* c, const double* in, double* out) {
#define L1(P, M) case P * 10 + M: launch_lim1d_ny<P, M, NY>(c, in, out); return 0;
  switch (c->p * 10 + c->limiter) {
    L1(1, 1) L1(1, 2) L1(2, 1) L1(2, 2) L1(3, 1) L1(3, 2)
    default: return set_error(DGB_ERR_UNSUPPORTED, "with mass fractions the limiter is none, hrl or m2l");
  }
#undef L1
}

// 2D: full tiles of a structured grid (TMA tile loads: checked when the context is created), then the
// strips outside them (if any) with the generic kernel
template <int MODE, int NY>
int residual2d_ny(dgb_ctx* c, const StageArgs& a) {
#define R2(P, F)                                                               \
  case P * 10 + F:                                                             \
    launch_tile2d<P, F, MODE, NY>(c, a);                                       \
    if (c->nleft) launch_res2d<P, F, MODE, NY>(c, a, c->left, c->nleft);       \
    return 0;
  switch (c->p * 10 + c->flux) {
    R2(1, 0) R2(1, 2) R2(2, 0) R2(2, 2) R2(3, 0) R2(3, 2)
    default: return set_error(DGB_ERR_UNSUPPORTED, "no residual kernel for this (p, flux) with mass fractions");
  }
#undef R2
}

template <int P, int METHOD, int NY>
void launch_lim2d_ny(dgb_ctx* c, double* U) {
  ProfScope ps(c, KC_LIMITER);
  const LimArgs la{c->ld, c->ne};
  auto kx = lim2d_xpass_tile_kernel<P, METHOD, NY>;
  auto ky = lim2d_ypass_tile_kernel<P, METHOD, NY>;
  constexpr size_t sx = lim2d_xpass_smem_bytes<P, NY>(), sy = lim2d_ypass_smem_bytes<P, NY>();
  if (sx) allow_dynamic_smem(kx, sx);
  if (sy) allow_dynamic_smem(ky, sy);
  const dim3 gx((c->nx + 29) / 30, c->ny), bx(32, P + 1);
  launch_pdl(c, kx, gx, bx, sx, la, c->nx, (const double*)U, (const int*)c->nbr, c->X, (const DevScalars*)c->scal);
  const dim3 gy((c->nx + 31) / 32, (c->ny + 3) / 4, P + 1), by(32, 6);
  launch_pdl(c, ky, gy, by, sy, la, c->nx, c->ny, (const double*)c->X, (const int*)c->nbr, U,
             (const DevScalars*)c->scal);
}

template <int NY>
int limit2d_ny(dgb_ctx* c, double* U) {
#define L2(P, M) case P * 10 + M: launch_lim2d_ny<P, M, NY>(c, U); return 0;
  switch (c->p * 10 + c->limiter) {
    L2(1, 1) L2(1, 2) L2(2, 1) L2(2, 2) L2(3, 1) L2(3, 2)
    default: return set_error(DGB_ERR_UNSUPPORTED, "with mass fractions the limiter is none, hrl or m2l");
  }
#undef L2
}

}  // namespace

int residual2d_many_y(dgb_ctx* c, const StageArgs& a, int mode) {
#define NYC(N)                                                                   \
  case N:                                                                        \
    return mode == MODE_SSP ? residual2d_ny<MODE_SSP, N>(c, a)                   \
           : mode == MODE_RK4 ? residual2d_ny<MODE_RK4, N>(c, a) : residual2d_ny<MODE_RESIDUAL, N>(c, a);
  switch (c->nmass) {
    NYC(4) NYC(5) NYC(6) NYC(7) NYC(8) NYC(9) NYC(10)
    default: return set_error(DGB_ERR_UNSUPPORTED, "mass fractions: 4 to 10 here");
  }
#undef NYC
}

int limit2d_many_y(dgb_ctx* c, double* U) {
  switch (c->nmass) {
    case 4: return limit2d_ny<4>(c, U);
    case 5: return limit2d_ny<5>(c, U);
    case 6: return limit2d_ny<6>(c, U);
    case 7: return limit2d_ny<7>(c, U);
    case 8: return limit2d_ny<8>(c, U);
    case 9: return limit2d_ny<9>(c, U);
    case 10: return limit2d_ny<10>(c, U);
    default: return set_error(DGB_ERR_UNSUPPORTED, "mass fractions: 4 to 10 here");
  }
}

int residual1d_many_y(dgb_ctx* c, const StageArgs& a, int mode) {
#define NYC(N)                                                                   \
  case N:                                                                        \
    return mode == MODE_SSP ? residual_ny<MODE_SSP, N>(c, a)                     \
           : mode == MODE_RK4 ? residual_ny<MODE_RK4, N>(c, a) : residual_ny<MODE_RESIDUAL, N>(c, a);
  switch (c->nmass) {
    NYC(4) NYC(5) NYC(6) NYC(7) NYC(8) NYC(9) NYC(10)
    default: return set_error(DGB_ERR_UNSUPPORTED, "mass fractions: 4 to 10 here");
  }
#undef NYC
}

int limit1d_many_y(dgb_ctx* c, const double* in, double* out) {
  switch (c->nmass) {
    case 4: return limit_ny<4>(c, in, out);
    case 5: return limit_ny<5>(c, in, out);
    case 6: return limit_ny<6>(c, in, out);
    case 7: return limit_ny<7>(c, in, out);
    case 8: return limit_ny<8>(c, in, out);
    case 9: return limit_ny<9>(c, in, out);
    case 10: return limit_ny<10>(c, in, out);
    default: return set_error(DGB_ERR_UNSUPPORTED, "mass fractions: 4 to 10 here");
  }
}

}  // namespace dgb

namespace dgb {
// this module's copy of the __constant__ tables (each .cu file is its own device module)
int upload_many_y_tables(const Consts& cs, int D, int p) { return upload_tables(cs, D, p); }
}  // namespace dgb
