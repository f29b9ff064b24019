// 1D problems with 4 to 10 passive mass fractions (the reference's MASS = 4 .. 10,
// code/Makefile:32): the residual and the hrl / m2l limiter kernels instantiated for N_Y = 4 .. 10,
// in a translation unit of their own so that they compile beside dgb_device.cu.  Same kernels as
// N_Y <= 3 (residual1d_kernel, lim1d_kernel); a mass fraction is advected like the density and
// limited like it (HR: every field; m2: the MACRO block of M2limiting).
#include <cuda_runtime.h>

#include <string>

#include "ctx.h"
#include "device/kernels.cuh"
#include "device/tables.cuh"

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

}  // namespace

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
// this module's copy of the __constant__ limiter tables (each .cu file is its own device module)
int upload_many_y_tables(const Consts& cs, int p) { return upload_tables(cs, 1, p); }
}  // namespace dgb
