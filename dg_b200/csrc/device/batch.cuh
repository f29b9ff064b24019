// Batched ensemble: many independent problems advanced together, one persistent launch per
// element class (dimension, order, flux, limiter) and operator.
//
// Every case keeps its own device context (state buffers A, B, C, scratch X, neighbour table,
// scalars with its own CFL step).  A class's work is a list of items -- (case, tile origin) -- and
// a persistent grid of CTAs walks that list with a fixed stride; all items of a launch cost the
// same, so the static stride balances.  The arithmetic of an item is that of the single-problem
// kernels (the same body functions): a 1D case advanced in a batch matches the same case advanced
// alone bit for bit; in 2D the tile body reads the metric from shared memory instead of kernel
// parameters and the compiler forms some fused multiply-adds differently (a few ulps).
//
// A case whose scalars carry a flag (an error, or FLAG_DONE once it has reached its end time) is
// skipped by every item; the test is taken once per item by one thread and shared, so the CTA
// stays on the same barriers.
#pragma once
#include "kernels.cuh"
#include "limiter2d_tile.cuh"
#include "tile2d.cuh"

namespace dgb {

enum { FLAG_DONE = 8u };  // the case reached its end time; cleared when the batch run ends

struct BatchCase {
  double* A;
  double* B;
  double* C;
  double* X;
  const int* nbr;
  DevScalars* scal;
  int nx, ny, ld, ne;
  double J, invJ, cx, cy, sx, sy, JFx, JFy;  // metric of the uniform element (2D tile kernel)
  double cfl_scaled;
};

// TMA descriptors of a 2D case's A, B, C for the class's tile shape (64-byte aligned in global
// memory, written by the host before any launch that reads them)
struct alignas(64) BatchMaps {
  CUtensorMap m[3];
};

// per-case progress of a batch run (device)
struct BatchProgress {
  int steps;                        // steps taken in this run
  int pad_;
  unsigned long long t_done_ns;     // global timer when the case reached its end time
};

// SSP-RK3 (Shu-Osher) stage s: input, output and coefficients out = a*A + b*(in + dt L(in))
__device__ __forceinline__ double* stage_in(const BatchCase& c, int s) { return s == 0 ? c.A : s == 1 ? c.B : c.C; }
__device__ __forceinline__ double* stage_out(const BatchCase& c, int s) { return s == 0 ? c.B : s == 1 ? c.C : c.A; }
__device__ __forceinline__ double stage_a(int s) { return s == 0 ? 0.0 : s == 1 ? 0.75 : 1.0 / 3.0; }
__device__ __forceinline__ double stage_b(int s) { return s == 0 ? 1.0 : s == 1 ? 0.25 : 2.0 / 3.0; }

// case flags of item `it`, read once by thread 0 and shared through `slot`
__device__ __forceinline__ unsigned item_flags(const BatchCase* cases, int ci, unsigned* slot) {
  __syncthreads();  // the previous item's shared-memory users are done
  if (threadIdx.x == 0 && threadIdx.y == 0) *slot = *(volatile unsigned*)&cases[ci].scal->flags;
  __syncthreads();
  return *slot;
}

// ---------------------------------------------------------------------------------------------
// 2D residual + SSP stage update, tiles of TW x TH elements (items: case, tx0, ty0)
// ---------------------------------------------------------------------------------------------
template <int P, int TW, int TH>
constexpr size_t batch_tile2d_smem_bytes() {
  return (TileDims<P, TW, TH>::smem_bytes + 127) / 128 * 128 + (sizeof(TileArgs) + 127) / 128 * 128;
}

template <int P, int FLUX, int TW, int TH, int UNROLL>
__global__ void __launch_bounds__(TW * TH, 2)
    batch_tile2d_kernel(const BatchCase* __restrict__ cases, const BatchMaps* __restrict__ maps,
                        const int4* __restrict__ items, int n_items, int stage) {
  extern __shared__ __align__(128) unsigned char smraw[];
  using Dm = TileDims<P, TW, TH>;
  TileArgs* sa = reinterpret_cast<TileArgs*>(smraw + (Dm::smem_bytes + 127) / 128 * 128);
  unsigned* s_flags = reinterpret_cast<unsigned*>(smraw + 16);  // head: mbarrier, ok flag, this
  if (threadIdx.x == 0) {
    mbar_init(reinterpret_cast<uint64_t*>(smraw), 1);
    fence_mbar_init();
  }
  uint32_t phase = 0;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const int4 item = __ldg(items + it);
    fence_proxy_async_smem();  // this CTA's generic accesses to the tile buffers precede the next copies
    if (item_flags(cases, item.x, s_flags)) continue;
    if (threadIdx.x == 0) {
      const BatchCase& c = cases[item.x];
      TileArgs a;
      a.U = stage_in(c, stage);
      a.Ubase = c.A;
      a.out = stage_out(c, stage);
      a.Uacc = nullptr;
      a.nbr = c.nbr;
      a.scal = c.scal;
      a.errflag = &c.scal->flags;
      a.a = stage_a(stage);
      a.b = stage_b(stage);
      a.dt_override = 0.0;
      a.invJ = c.invJ; a.cx = c.cx; a.cy = c.cy; a.sx = c.sx; a.sy = c.sy;
      a.J = c.J; a.JFx = c.JFx; a.JFy = c.JFy;
      a.nx = c.nx; a.ny = c.ny; a.ld = c.ld;
      *sa = a;
    }
    __syncthreads();
    const CUtensorMap* mu = &maps[item.x].m[stage];
    const CUtensorMap* mb = &maps[item.x].m[0];
    tile2d_body<P, FLUX, MODE_SSP, TW, TH, UNROLL>(*sa, mu, mb, item.y, item.z, smraw, phase);
  }
}

// ---------------------------------------------------------------------------------------------
// 2D limiter passes (hrl: METHOD 1, m2l: METHOD 2) on the stage output, via the case's scratch X
// x items: (case, x0 multiple of 30, row);  y items: (case, x0 multiple of 32, y0 multiple of 4, node column)
// ---------------------------------------------------------------------------------------------
template <int P, int METHOD>
__global__ void __launch_bounds__(32 * (P + 1)) batch_lim2d_x_kernel(const BatchCase* __restrict__ cases,
                                                                   const int4* __restrict__ items, int n_items,
                                                                   int stage) {
  __shared__ unsigned s_flags;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const int4 item = __ldg(items + it);
    if (item_flags(cases, item.x, &s_flags)) continue;
    const BatchCase& c = cases[item.x];
    const LimArgs la{c.ld, c.ne};
    lim2d_xpass_body<P, METHOD>(la, c.nx, stage_out(c, stage), c.nbr, c.X, item.y, item.z);
  }
}

template <int P, int METHOD>
__global__ void __launch_bounds__(32 * 6) batch_lim2d_y_kernel(const BatchCase* __restrict__ cases,
                                                             const int4* __restrict__ items, int n_items, int stage) {
  __shared__ unsigned s_flags;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const int4 item = __ldg(items + it);
    if (item_flags(cases, item.x, &s_flags)) continue;
    const BatchCase& c = cases[item.x];
    const LimArgs la{c.ld, c.ne};
    lim2d_ypass_body<P, METHOD>(la, c.nx, c.ny, c.X, c.nbr, stage_out(c, stage), item.y, item.z, item.w);
  }
}

// ---------------------------------------------------------------------------------------------
// 1D residual + SSP stage update, one thread per element (items: case, first element).  With a
// limiter the stage result goes to X and the limiter writes the stage output.
// ---------------------------------------------------------------------------------------------
template <int P, int FLUX, bool LIMITED>
__global__ void __launch_bounds__(256) batch_res1d_kernel(const BatchCase* __restrict__ cases,
                                                          const Consts* __restrict__ consts,
                                                          const int4* __restrict__ items, int n_items, int stage) {
  __shared__ Consts c;
  __shared__ unsigned s_flags;
  int loaded = -1;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const int4 item = __ldg(items + it);
    if (item_flags(cases, item.x, &s_flags)) continue;
    if (item.x != loaded) {  // per-case constants (metric, inverse mass matrix, ld)
      copy_consts(c, consts[item.x]);
      loaded = item.x;
      __syncthreads();
    }
    const BatchCase& bc = cases[item.x];
    const int e = item.y + threadIdx.x;
    if (e >= c.n_elem) continue;
    StageArgs a;
    a.U = stage_in(bc, stage);
    a.Ubase = bc.A;
    a.out = LIMITED ? bc.X : stage_out(bc, stage);
    a.Uacc = nullptr;
    a.nbr = bc.nbr;
    a.scal = bc.scal;
    a.a = stage_a(stage);
    a.b = stage_b(stage);
    a.dt_override = 0.0;
    res1d_body<P, FLUX, MODE_SSP>(c, a, e, bc.scal->dt);
  }
}

template <int P, int METHOD>
__global__ void __launch_bounds__(256) batch_lim1d_kernel(const BatchCase* __restrict__ cases,
                                                          const int4* __restrict__ items, int n_items, int stage) {
  __shared__ unsigned s_flags;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const int4 item = __ldg(items + it);
    if (item_flags(cases, item.x, &s_flags)) continue;
    const BatchCase& bc = cases[item.x];
    const int e = item.y + threadIdx.x;
    if (e >= bc.ne) continue;
    lim1d_body<P, METHOD>(bc.ld, e, bc.X, bc.nbr, stage_out(bc, stage));
  }
}

// ---------------------------------------------------------------------------------------------
// CFL step of every case: max |u|+a over its nodes (items: case, first element of 256), then
// dt = CFL_scaled / max, cut to the case's end time
// ---------------------------------------------------------------------------------------------
template <int DIM, int NS>
__global__ void __launch_bounds__(256) batch_wavespeed_kernel(const BatchCase* __restrict__ cases,
                                                              const int4* __restrict__ items, int n_items) {
  __shared__ unsigned s_flags;
  __shared__ double wm[8];
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const int4 item = __ldg(items + it);
    if (item_flags(cases, item.x, &s_flags)) continue;
    const BatchCase& c = cases[item.x];
    const int e = item.y + threadIdx.x, ld = c.ld;
    const double* U = c.A;
    double m = 0.0;
    bool bad = false;
    if (e < c.ne) {
#pragma unroll
      for (int t = 0; t < NS; ++t) {
        double w;
        if (DIM == 1)
          w = phys::wave_speed1d(__ldg(U + (size_t)(0 * NS + t) * ld + e), __ldg(U + (size_t)(1 * NS + t) * ld + e),
                                 __ldg(U + (size_t)(2 * NS + t) * ld + e), __ldg(U + (size_t)(3 * NS + t) * ld + e));
        else
          w = phys::wave_speed2d(__ldg(U + (size_t)(0 * NS + t) * ld + e), __ldg(U + (size_t)(1 * NS + t) * ld + e),
                                 __ldg(U + (size_t)(2 * NS + t) * ld + e), __ldg(U + (size_t)(3 * NS + t) * ld + e),
                                 __ldg(U + (size_t)(4 * NS + t) * ld + e));
        if (!(w == w)) bad = true;
        else m = fmax(m, fabs(w));
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) wm[w] = m;
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&c.scal->flags, (unsigned)FLAG_NONFINITE);
    __syncthreads();
    if (threadIdx.x == 0) {
      double mm = 0.0;
      for (int k = 0; k < (int)(blockDim.x >> 5); ++k) mm = fmax(mm, wm[k]);
      atomicMax(&c.scal->umax, (unsigned long long)__double_as_longlong(mm));
    }
  }
}

__device__ __forceinline__ unsigned long long global_timer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// one thread per case of the class: the finish of the CFL step (as finish_dt_kernel), with the end
// time: a case at or past t_end (> 0) stops (FLAG_DONE, completion time recorded)
__global__ void batch_finish_dt_kernel(const BatchCase* __restrict__ cases, BatchProgress* __restrict__ prog,
                                       const int* __restrict__ case_ids, int n, const double* __restrict__ t_end_p) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double t_end = *t_end_p;
  const int ci = case_ids[k];
  DevScalars* s = cases[ci].scal;
  if (s->flags) return;
  if (t_end > 0 && s->time >= t_end) {
    s->flags |= FLAG_DONE;
    prog[ci].t_done_ns = global_timer_ns();
    s->umax = 0ull;
    return;
  }
  const double umax = __longlong_as_double((long long)s->umax);
  double dt = cases[ci].cfl_scaled / umax;
  s->umax = 0ull;
  if (!(dt == dt)) { s->flags |= FLAG_NONFINITE; return; }
  if (dt < 1e-14) { s->flags |= FLAG_DT_SMALL; return; }
  prog[ci].steps += 1;
  if (t_end > 0 && s->time + dt >= t_end) {  // last step: lands on t_end exactly
    s->dt = t_end - s->time;
    s->time = t_end;
    return;
  }
  s->dt = dt;
  s->time += dt;
}

__global__ void batch_start_kernel(unsigned long long* t0) { *t0 = global_timer_ns(); }

}  // namespace dgb
