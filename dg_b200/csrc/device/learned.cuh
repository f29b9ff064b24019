// Learned troubled-cell indicator: features, labels and the MLP's training kernels.
//
// Network: 225 -> 64 -> 64 -> 1, GELU hidden activations, sigmoid output.  Input of element e
// (2D, p = 2): the 9 scaled-Taylor modes of each of the 5 fields of e and of its left, right,
// bottom and top neighbours (the element itself where a neighbour is a boundary), minus e's own
// cell value on the constant mode and divided by e's field scale (|mode 0| for rho, E, alpha;
// sqrt(|rho_0 E_0|) for both momenta): x[(n*5 + f)*9 + k], n = self, L, R, D, U.
// Each input is then soft-thresholded by the rounding floor 5e-5 and compressed by the fixed signed
// logarithm: x -> sign(x) log(1 + max(|x| - 5e-5, 0) / 1e-5) / log(1 + 1e5).  The values span many
// decades and the decision lives in their magnitude; below the floor sits rounding, not structure:
// the mixed form's FP32 flux arithmetic leaves normalised non-constant modes of 1e-6 to 2e-5 in
// smooth elements that no limiter touches (measured over 500 steps of the 512 x 256 shock-bubble
// and 400 of the 1024^2 four-quadrant problem; mostly the (2,2) mode), where plain FP64 has ~1e-15.
// Label: 1 when the full limiter of the problem changes any non-constant mode of any field of
// the element by more than 1e-8 of that field's scale, in an element whose own normalised
// non-constant modes rise above the floor (the limiter only shrinks modes, so elsewhere its change
// is below the floor too, and no input could tell it from rounding).
// Parameters (FP32, one flat array): W1[64][225], b1[64], W2[64][64], b2[64], w3[64], b3.
// The training kernels are plain FP32: the network is tiny, the batches are ~10^4 samples.
#pragma once
#include <cuda_bf16.h>

#include "kernels.cuh"

namespace dgb {

constexpr int MLP_IN = 225, MLP_H = 64;
constexpr int MLP_W1 = 0, MLP_B1 = MLP_W1 + MLP_H * MLP_IN, MLP_W2 = MLP_B1 + MLP_H, MLP_B2 = MLP_W2 + MLP_H * MLP_H,
              MLP_W3 = MLP_B2 + MLP_H, MLP_B3 = MLP_W3 + MLP_H, MLP_NPARAM = MLP_B3 + 1;
constexpr int MLP_CACHE = 4 * MLP_H;  // per sample: A1, H1, A2, H2
constexpr double IND_LABEL_TOL = 1e-8;
constexpr double IND_FEAT_FLOOR = 5e-5;                     // rounding floor of the normalised inputs
constexpr double IND_FEAT_S0 = 1e-5;                        // compression scale above the floor
constexpr double IND_FEAT_NORM = 11.512935464920228;       // log(1 + 1 / IND_FEAT_S0)

__device__ __forceinline__ double feature_compress(double x) {
  return copysign(log1p(fmax(fabs(x) - IND_FEAT_FLOOR, 0.0) / IND_FEAT_S0) / IND_FEAT_NORM, x);
}

__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad_f(float x) {
  return 0.5f * (1.f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// 2D scaled-Taylor modes of one element: a[f][mx + N1*my] = sum T[mx][ix] T[my][iy] u_f(ix, iy)
template <int P>
__device__ __forceinline__ void element_modes(const double* __restrict__ U, int ld, int e,
                                              double a[5][(P + 1) * (P + 1)]) {
  constexpr int N1 = P + 1, NS = N1 * N1;
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    double tx[NS];  // x transform of every row
#pragma unroll
    for (int iy = 0; iy < N1; ++iy) {
      double row[N1], m[N1];
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) row[ix] = __ldg(U + (size_t)(f * NS + ix + N1 * iy) * ld + e);
      to_mono<P>(row, m);
#pragma unroll
      for (int mx = 0; mx < N1; ++mx) tx[mx + N1 * iy] = m[mx];
    }
#pragma unroll
    for (int mx = 0; mx < N1; ++mx) {
      double col[N1], m[N1];
#pragma unroll
      for (int iy = 0; iy < N1; ++iy) col[iy] = tx[mx + N1 * iy];
      to_mono<P>(col, m);
#pragma unroll
      for (int my = 0; my < N1; ++my) a[f][mx + N1 * my] = m[my];
    }
  }
}

template <int P>
__device__ __forceinline__ void field_scales(const double a[5][(P + 1) * (P + 1)], double s[5]) {
  s[0] = fabs(a[0][0]) + 1e-300;
  s[3] = fabs(a[3][0]) + 1e-300;
  s[4] = fabs(a[4][0]) + 1e-300;
  s[1] = s[2] = sqrt(fabs(a[0][0] * a[3][0])) + 1e-300;
}

// features of every element of the state (one thread per element), X row-major [n][225]
template <int P>
__global__ void __launch_bounds__(128) indicator_features_kernel(const double* __restrict__ U, int ld, int n_elem,
                                                                 const int* __restrict__ nbr,
                                                                 float* __restrict__ X) {
  constexpr int NS = (P + 1) * (P + 1);
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_elem) return;
  double a[5][NS], s[5], a0[5];
  element_modes<P>(U, ld, e, a);
  field_scales<P>(a, s);
#pragma unroll
  for (int f = 0; f < 5; ++f) a0[f] = a[f][0];
  float* x = X + (size_t)e * MLP_IN;
  for (int n = 0; n < 5; ++n) {
    int el = e;
    if (n > 0) {
      const int nb = __ldg(nbr + (size_t)(n - 1) * ld + e);
      el = nb >= 0 ? nb : e;
    }
    if (n > 0) element_modes<P>(U, ld, el, a);
#pragma unroll
    for (int f = 0; f < 5; ++f)
#pragma unroll
      for (int k = 0; k < NS; ++k)
        x[(n * 5 + f) * NS + k] = (float)feature_compress((a[f][k] - (k == 0 ? a0[f] : 0.0)) / s[f]);
  }
}

// labels: does the full limiter (Ulim) change a non-constant mode of an element with modes above
// the rounding floor?
template <int P>
__global__ void __launch_bounds__(128) indicator_labels_kernel(const double* __restrict__ U,
                                                               const double* __restrict__ Ulim, int ld, int n_elem,
                                                               float* __restrict__ y) {
  constexpr int NS = (P + 1) * (P + 1);
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_elem) return;
  double a[5][NS], b[5][NS], s[5];
  element_modes<P>(U, ld, e, a);
  element_modes<P>(Ulim, ld, e, b);
  field_scales<P>(a, s);
  bool changed = false, above = false;
#pragma unroll
  for (int f = 0; f < 5; ++f)
#pragma unroll
    for (int k = 1; k < NS; ++k) {
      changed |= fabs(b[f][k] - a[f][k]) > IND_LABEL_TOL * s[f];
      above |= fabs(a[f][k]) > IND_FEAT_FLOOR * s[f];
    }
  y[e] = (changed && above) ? 1.f : 0.f;
}

// ---------------------------------------------------------------------------------------------
// training (FP32)
// ---------------------------------------------------------------------------------------------

// forward, one thread per sample; weights staged in shared memory
__global__ void __launch_bounds__(128) mlp_forward_kernel(const float* __restrict__ prm, const float* __restrict__ X,
                                                          int n, float* __restrict__ cache, float* __restrict__ prob) {
  extern __shared__ float wsm[];  // W1, b1, W2, b2, w3, b3
  for (int k = threadIdx.x; k < MLP_NPARAM; k += blockDim.x) wsm[k] = prm[k];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float* x = X + (size_t)s * MLP_IN;
  float h1[MLP_H], h2[MLP_H];
  float* c = cache ? cache + (size_t)s * MLP_CACHE : nullptr;
  for (int j = 0; j < MLP_H; ++j) {
    float acc = wsm[MLP_B1 + j];
    const float* w = wsm + MLP_W1 + j * MLP_IN;
    for (int k = 0; k < MLP_IN; ++k) acc += w[k] * __ldg(x + k);
    h1[j] = gelu_f(acc);
    if (c) { c[j] = acc; c[MLP_H + j] = h1[j]; }
  }
  float z = wsm[MLP_B3];
  for (int j = 0; j < MLP_H; ++j) {
    float acc = wsm[MLP_B2 + j];
    const float* w = wsm + MLP_W2 + j * MLP_H;
#pragma unroll 8
    for (int i = 0; i < MLP_H; ++i) acc += w[i] * h1[i];
    h2[j] = gelu_f(acc);
    if (c) { c[2 * MLP_H + j] = acc; c[3 * MLP_H + j] = h2[j]; }
    z += wsm[MLP_W3 + j] * h2[j];
  }
  prob[s] = 1.f / (1.f + expf(-z));
}

// per-sample error signals of the weighted binary cross-entropy (mean over the batch):
// dz, dA2 [n][64], dA1 [n][64]; the loss is accumulated into *loss
__global__ void __launch_bounds__(128) mlp_delta_kernel(const float* __restrict__ prm, const float* __restrict__ y,
                                                        float pos_weight, int n, const float* __restrict__ cache,
                                                        const float* __restrict__ prob, float* __restrict__ dz,
                                                        float* __restrict__ dA2, float* __restrict__ dA1,
                                                        float* __restrict__ loss) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (s < n) {
    const float p = prob[s], t = y[s];
    const float w = t > 0.5f ? pos_weight : 1.f;
    const float inv_n = 1.f / (float)n;
    const float pc = fminf(fmaxf(p, 1e-7f), 1.f - 1e-7f);
    l = -w * (t * logf(pc) + (1.f - t) * logf(1.f - pc)) * inv_n;
    const float d = w * (p - t) * inv_n;
    dz[s] = d;
    const float* c = cache + (size_t)s * MLP_CACHE;
    float g2[MLP_H];
    for (int j = 0; j < MLP_H; ++j) {
      g2[j] = d * prm[MLP_W3 + j] * gelu_grad_f(c[2 * MLP_H + j]);
      dA2[(size_t)s * MLP_H + j] = g2[j];
    }
    for (int i = 0; i < MLP_H; ++i) {
      float acc = 0.f;
      for (int j = 0; j < MLP_H; ++j) acc += prm[MLP_W2 + j * MLP_H + i] * g2[j];
      dA1[(size_t)s * MLP_H + i] = acc * gelu_grad_f(c[i]);
    }
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// G[r][c] = sum_s P[s*ldp + r] * Q[s*ldq + c] (r < R, c < C); Q == nullptr: Q = 1 (column sums)
__global__ void __launch_bounds__(256) outer_reduce_kernel(int n, const float* __restrict__ Pm, int ldp, int R,
                                                           const float* __restrict__ Qm, int ldq, int C,
                                                           float* __restrict__ G) {
  __shared__ float sp[16][17], sq[16][17];
  const int tr = threadIdx.y, tc = threadIdx.x;
  const int r = blockIdx.y * 16 + tr, c = blockIdx.x * 16 + tc;
  float acc = 0.f;
  for (int s0 = 0; s0 < n; s0 += 16) {
    const int sp_s = s0 + tc, rr = blockIdx.y * 16 + tr;  // load P[s0 + tc][rr] into sp[tr][tc]
    sp[tr][tc] = (sp_s < n && rr < R) ? Pm[(size_t)sp_s * ldp + rr] : 0.f;
    const int sq_s = s0 + tr, cc = blockIdx.x * 16 + tc;  // load Q[s0 + tr][cc] into sq[tr][tc]
    sq[tr][tc] = (sq_s < n && cc < C) ? (Qm ? Qm[(size_t)sq_s * ldq + cc] : 1.f) : 0.f;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 16; ++k) acc += sp[tr][k] * sq[k][tc];
    __syncthreads();
  }
  if (r < R && c < C) G[(size_t)r * C + c] = acc;
}

// Adam (bias-corrected), t >= 1
__global__ void __launch_bounds__(256) mlp_adam_kernel(float* __restrict__ prm, const float* __restrict__ g,
                                                       float* __restrict__ m, float* __restrict__ v, int np, int t,
                                                       float lr, float b1, float b2, float eps) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= np) return;
  const float gk = g[k];
  const float mk = b1 * m[k] + (1.f - b1) * gk;
  const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
  m[k] = mk;
  v[k] = vk;
  const float mh = mk / (1.f - powf(b1, (float)t)), vh = vk / (1.f - powf(b2, (float)t));
  prm[k] -= lr * mh / (sqrtf(vh) + eps);
}

}  // namespace dgb

namespace dgb {

// ---------------------------------------------------------------------------------------------
// inference inside the limiter
// ---------------------------------------------------------------------------------------------
// The scoring kernel lays the inputs out with each neighbour's 45 values padded to 48 (k' = 48 n +
// 9 f + m; 240 = 15 k-tiles of 16), so that a lane writes one neighbour's values with 16-byte
// stores; W1 is stored with the same padded column order.
constexpr int IND_KPAD = 240, IND_NSEG = 48;
constexpr int IND_W1S = IND_KPAD + 8;    // shared row strides (bf16) that keep the fragment loads
constexpr int IND_FTS = 264;             // free of bank conflicts (and 16-byte aligned rows)
constexpr int IND_W2S = MLP_H + 8;
// per element, 64 floats = 256 bytes, 16-byte aligned parts: [0, 10) the 5 constant modes as
// FP64 (neighbour differences of nearly equal means must not cancel in FP32), [16, 56) the other
// 40 modes (field f at 16 + 8 f), [56, 61) the 5 inverse field scales
constexpr int IND_MODES = 64, IND_M_SLOPE = 16, IND_M_ISCALE = 56;

// modes and scales of every element (FP64 transform)
template <int P>
__global__ void __launch_bounds__(128) indicator_modes_kernel(const double* __restrict__ U, int ld, int n_elem,
                                                              float* __restrict__ M) {
  constexpr int NS = (P + 1) * (P + 1);
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_elem) return;
  double a[5][NS], s[5];
  element_modes<P>(U, ld, e, a);
  field_scales<P>(a, s);
  float* m = M + (size_t)e * IND_MODES;
  double* m0 = reinterpret_cast<double*>(m);
#pragma unroll
  for (int f = 0; f < 5; ++f) {
    m0[f] = a[f][0];
#pragma unroll
    for (int k = 1; k < NS; ++k) m[IND_M_SLOPE + f * (NS - 1) + k - 1] = (float)a[f][k];
    m[IND_M_ISCALE + f] = (float)(1.0 / s[f]);
  }
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

struct IndicatorArgs {
  int n_elem, ld;
  float threshold;
  const int* nbr;
  const float* modes;            // [n_elem][50]
  const __nv_bfloat16* w1;       // [64][IND_KPAD] bf16 (zero padded)
  const __nv_bfloat16* w2;       // [64][64] bf16
  const float* vec;              // b1[64], b2[64], w3[64], b3 (FP32)
  float* score;                  // [n_elem]
  unsigned char* flag;           // [n_elem]
  int* list;                     // flagged elements
  int* count;
  const DevScalars* scal;
  unsigned int* errflag;         // receives FLAG_TIMEOUT when a bounded wait runs out
};

// the input compression in FP32 with the hardware base-2 logarithm
__device__ __forceinline__ float feature_compress_fast(float x) {
  const float m = fmaxf(fabsf(x) - (float)IND_FEAT_FLOOR, 0.f);
  const float l = __log2f(fmaf(m, (float)(1.0 / IND_FEAT_S0), 1.f));
  return copysignf(l * (float)(0.69314718055994531 / IND_FEAT_NORM), x);
}

// GELU in its tanh form with the hardware tanh (scoring only; inputs are BF16 anyway)
__device__ __forceinline__ float gelu_fast(float x) {
  const float u = 0.7978845608028654f * fmaf(0.044715f * x, x * x, x);
  float th;
  asm("tanh.approx.f32 %0, %1;" : "=f"(th) : "f"(u));
  return 0.5f * x * (1.f + th);
}

// MLP scores on BF16 tensor cores (mma.sync m16n8k16, FP32 accumulation): a warp scores 16
// elements; layer-1 accumulators become layer-2 A fragments without leaving registers.
// Persistent CTAs of IND_WARPS warps sharing one copy of the weights (2 CTAs, 16 warps per SM: the
// feature gathers are latency-bound and need the warps).  Elements scoring above the threshold
// are flagged and appended to the list.
constexpr int IND_WARPS = 8;
constexpr size_t IND_SMEM_BYTES =
    ((size_t)MLP_H * IND_W1S + (size_t)MLP_H * IND_W2S + (size_t)IND_WARPS * 16 * IND_FTS) * sizeof(__nv_bfloat16) +
    (3 * MLP_H + 4) * sizeof(float) + IND_WARPS * 80 * sizeof(int);

__global__ void __launch_bounds__(32 * IND_WARPS, 2) indicator_infer_kernel(const IndicatorArgs a) {
  extern __shared__ __align__(16) unsigned char ism[];
  __nv_bfloat16* w1s = reinterpret_cast<__nv_bfloat16*>(ism);          // [64][IND_W1S]
  __nv_bfloat16* w2s = w1s + MLP_H * IND_W1S;                           // [64][IND_W2S]
  __nv_bfloat16* fts0 = w2s + MLP_H * IND_W2S;                          // per warp: [16][IND_W1S]
  float* vs = reinterpret_cast<float*>(fts0 + IND_WARPS * 16 * IND_FTS);  // b1, b2, w3, b3
  int* eidx0 = reinterpret_cast<int*>(vs + 3 * MLP_H + 4);              // per warp: [16][5]
  if (a.scal && a.scal->flags) return;
  for (int i = threadIdx.x; i < IND_WARPS * 16 * IND_FTS; i += blockDim.x) fts0[i] = __float2bfloat16(0.f);
  for (int i = threadIdx.x; i < MLP_H * IND_KPAD; i += blockDim.x)
    w1s[(i / IND_KPAD) * IND_W1S + i % IND_KPAD] = a.w1[i];
  for (int i = threadIdx.x; i < MLP_H * MLP_H; i += blockDim.x) w2s[(i / MLP_H) * IND_W2S + i % MLP_H] = a.w2[i];
  for (int i = threadIdx.x; i < 3 * MLP_H + 1; i += blockDim.x) vs[i] = a.vec[i];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const uint32_t* w1w = reinterpret_cast<const uint32_t*>(w1s);
  const uint32_t* w2w = reinterpret_cast<const uint32_t*>(w2s);
  const int ntiles = (a.n_elem + 15) / 16;
  __syncthreads();
  __nv_bfloat16* ft = fts0 + warp * 16 * IND_FTS;
  const uint32_t* ftw = reinterpret_cast<const uint32_t*>(ft);
  for (int tile = blockIdx.x * IND_WARPS + warp; tile < ntiles; tile += gridDim.x * IND_WARPS) {
    const int r0 = tile * 16 + g, r1 = r0 + 8;
    const bool ok0 = r0 < a.n_elem, ok1 = r1 < a.n_elem;
    // element indices of the 16 rows (self, L, R, D, U), then the features into shared memory:
    // 25 (neighbour, field) groups of 9 modes per row, several groups in flight per lane
    int* eidx = eidx0 + warp * 80;
    for (int q = lane; q < 80; q += 32) {
      const int row = q / 5, n = q - 5 * row, es = tile * 16 + row;
      int v = es < a.n_elem ? es : -1;
      if (v >= 0 && n > 0) {
        const int nb = __ldg(a.nbr + (size_t)(n - 1) * a.ld + es);
        v = nb >= 0 ? nb : es;
      }
      eidx[q] = v;
    }
    __syncwarp();
    // one lane per (row, neighbour): the neighbour's whole record by 16-byte loads, 45 features out
    for (int q = lane; q < 80; q += 32) {
      const int row = q / 5, n = q - 5 * row;
      const int es = eidx[row * 5], en = eidx[row * 5 + n];
      uint4* dst = reinterpret_cast<uint4*>(ft + row * IND_FTS + n * IND_NSEG);
      if (es < 0) {
#pragma unroll
        for (int j = 0; j < IND_NSEG / 8; ++j) dst[j] = make_uint4(0u, 0u, 0u, 0u);
        continue;
      }
      const float4* rs = reinterpret_cast<const float4*>(a.modes + (size_t)es * IND_MODES);
      const float4* rn = reinterpret_cast<const float4*>(a.modes + (size_t)en * IND_MODES);
      float4 sv[3], nv[3], sl[10], isc[2];
#pragma unroll
      for (int k = 0; k < 3; ++k) { sv[k] = __ldg(rs + k); nv[k] = __ldg(rn + k); }
#pragma unroll
      for (int k = 0; k < 10; ++k) sl[k] = __ldg(rn + IND_M_SLOPE / 4 + k);
#pragma unroll
      for (int k = 0; k < 2; ++k) isc[k] = __ldg(rs + IND_M_ISCALE / 4 + k);
      const double* s0 = reinterpret_cast<const double*>(sv);
      const double* n0 = reinterpret_cast<const double*>(nv);
      const float* slp = reinterpret_cast<const float*>(sl);
      const float* is = reinterpret_cast<const float*>(isc);
      float v[IND_NSEG];
#pragma unroll
      for (int f = 0; f < 5; ++f) {
        v[f * 9] = feature_compress_fast((float)(n0[f] - s0[f]) * is[f]);
#pragma unroll
        for (int m = 1; m < 9; ++m) v[f * 9 + m] = feature_compress_fast(slp[f * 8 + m - 1] * is[f]);
      }
      v[45] = v[46] = v[47] = 0.f;
#pragma unroll
      for (int j = 0; j < IND_NSEG / 8; ++j)
        dst[j] = make_uint4(pack_bf16(v[8 * j], v[8 * j + 1]), pack_bf16(v[8 * j + 2], v[8 * j + 3]),
                            pack_bf16(v[8 * j + 4], v[8 * j + 5]), pack_bf16(v[8 * j + 6], v[8 * j + 7]));
    }
    __syncwarp();
    // layer 1: [16 x 240] x [240 x 64]
    float h[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) h[j][0] = h[j][1] = h[j][2] = h[j][3] = 0.f;
#pragma unroll 5
    for (int kk = 0; kk < IND_KPAD / 16; ++kk) {
      const int k0 = kk * 16 + 2 * t, k1 = k0 + 8;
      uint32_t af[4];
      af[0] = ftw[(g * IND_FTS + k0) >> 1];
      af[1] = ftw[((g + 8) * IND_FTS + k0) >> 1];
      af[2] = ftw[(g * IND_FTS + k1) >> 1];
      af[3] = ftw[((g + 8) * IND_FTS + k1) >> 1];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int n = 8 * j + g;
        mma_bf16_16816(h[j], af, w1w[(n * IND_W1S + k0) >> 1], w1w[(n * IND_W1S + k1) >> 1]);
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = 8 * j + 2 * t;
      h[j][0] = gelu_fast(h[j][0] + vs[c]);
      h[j][1] = gelu_fast(h[j][1] + vs[c + 1]);
      h[j][2] = gelu_fast(h[j][2] + vs[c]);
      h[j][3] = gelu_fast(h[j][3] + vs[c + 1]);
    }
    // layer 2: [16 x 64] x [64 x 64], A fragments from the layer-1 accumulators
    float h2[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j) h2[j][0] = h2[j][1] = h2[j][2] = h2[j][3] = 0.f;
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      uint32_t af[4];
      af[0] = pack_bf16(h[2 * kk][0], h[2 * kk][1]);
      af[1] = pack_bf16(h[2 * kk][2], h[2 * kk][3]);
      af[2] = pack_bf16(h[2 * kk + 1][0], h[2 * kk + 1][1]);
      af[3] = pack_bf16(h[2 * kk + 1][2], h[2 * kk + 1][3]);
      const int k0 = kk * 16 + 2 * t, k1 = k0 + 8;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int n = 8 * j + g;
        mma_bf16_16816(h2[j], af, w2w[(n * IND_W2S + k0) >> 1], w2w[(n * IND_W2S + k1) >> 1]);
      }
    }
    // layer 3 and the decision (FP32): row sums over the quad of lanes sharing a row
    float z0 = 0.f, z1 = 0.f;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = 8 * j + 2 * t;
      z0 += gelu_fast(h2[j][0] + vs[MLP_H + c]) * vs[2 * MLP_H + c] + gelu_fast(h2[j][1] + vs[MLP_H + c + 1]) * vs[2 * MLP_H + c + 1];
      z1 += gelu_fast(h2[j][2] + vs[MLP_H + c]) * vs[2 * MLP_H + c] + gelu_fast(h2[j][3] + vs[MLP_H + c + 1]) * vs[2 * MLP_H + c + 1];
    }
    z0 += __shfl_xor_sync(0xffffffffu, z0, 1);
    z0 += __shfl_xor_sync(0xffffffffu, z0, 2);
    z1 += __shfl_xor_sync(0xffffffffu, z1, 1);
    z1 += __shfl_xor_sync(0xffffffffu, z1, 2);
    // decisions; flagged rows appended to the list with one atomic per warp
    const float b3 = vs[3 * MLP_H];
    bool f0 = false, f1 = false;
    if (t == 0) {
      if (ok0) {
        const float sc = 1.f / (1.f + expf(-(z0 + b3)));
        a.score[r0] = sc;
        f0 = sc > a.threshold;
        a.flag[r0] = f0;
      }
      if (ok1) {
        const float sc = 1.f / (1.f + expf(-(z1 + b3)));
        a.score[r1] = sc;
        f1 = sc > a.threshold;
        a.flag[r1] = f1;
      }
    }
    const unsigned m0 = __ballot_sync(0xffffffffu, f0), m1 = __ballot_sync(0xffffffffu, f1);
    const int n0 = __popc(m0), ntot = n0 + __popc(m1);
    int base = 0;
    if (lane == 0 && ntot) base = atomicAdd(a.count, ntot);
    base = __shfl_sync(0xffffffffu, base, 0);
    const unsigned below = (1u << lane) - 1u;
    if (f0) a.list[base + __popc(m0 & below)] = r0;
    if (f1) a.list[base + n0 + __popc(m1 & below)] = r1;
    __syncwarp();
  }
}

// The band: flagged elements and their face neighbours (the flags are taken once per step on the
// step's initial state; a discontinuity moves well under one element per step at CFL < 1).
__global__ void __launch_bounds__(256) indicator_band_kernel(int n_elem, int ld, int n_nbr, const int* __restrict__ nbr,
                                                             const unsigned char* __restrict__ flag,
                                                             unsigned char* __restrict__ band, int* __restrict__ list,
                                                             int* __restrict__ count, const DevScalars* __restrict__ scal) {
  if (scal && scal->flags) return;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  bool b = false;
  if (e < n_elem) {
    b = flag[e] != 0;
    for (int k = 0; k < n_nbr && !b; ++k) {
      const int n = __ldg(nbr + (size_t)k * ld + e);
      b = n >= 0 && flag[n] != 0;
    }
    band[e] = b;
  }
  const unsigned m = __ballot_sync(0xffffffffu, b);
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == 0 && m) base = atomicAdd(count, __popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (b) list[base + __popc(m & ((1u << lane) - 1u))] = e;
}

}  // namespace dgb
