// Learned-indicator scoring on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Same network, inputs and decisions as indicator_infer_kernel (learned.cuh), with the two hidden
// layers as UMMA GEMMs: a CTA scores tiles of 128 elements (the M dimension of one MMA).
//   features   512 threads assemble the tile's 128 x 240 BF16 inputs (five neighbours of 48 padded
//              values per element) straight into shared memory in the canonical K-major layout of
//              the tensor cores: 8-row x 16-byte core matrices, chunk kc of row group rg at
//              (kc * 16 + rg) * 128 bytes (no swizzle)
//   layer 1    one thread issues 15 tcgen05.mma (M 128, N 64, K 16, BF16 x BF16 -> FP32) against W1
//              (64 x 240, same layout, loaded once per CTA); the accumulators live in tensor memory
//              (TMEM columns 0..63); tcgen05.commit arrives on an mbarrier when they are done
//   epilogue   every warp reads a 32-lane x 16-column block of the accumulators (tcgen05.ld),
//              adds b1, GELU, and writes the BF16 hidden values as the next GEMM's A operand
//   layer 2    4 tcgen05.mma against W2 (64 x 64) into TMEM columns 64..127
//   layer 3    GELU(+ b2) . w3 per element from the second accumulators, sigmoid, threshold, flag
//              list (one atomic per warp)
// Every wait on the MMA completion is bounded: when it runs out the kernel records FLAG_TIMEOUT,
// waits once more with the default budget, frees its tensor memory and returns.
#pragma once
#include "learned.cuh"
#include "tile2d.cuh"  // FLAG_TIMEOUT
#include "tma.cuh"

namespace dgb {

// ---- tcgen05 / TMEM primitives (PTX ISA, sm_100a) ----
__device__ __forceinline__ void tmem_alloc_warp(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish_warp() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc_warp(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, both K-major; accumulate != 0 adds to D
__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  const uint32_t no_mask = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(no_mask), "r"(no_mask), "r"(no_mask), "r"(no_mask)
      : "memory");
}
// arrive on `bar` once every MMA this thread issued before has completed
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane, waited for before return
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n\ttcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// shared-memory matrix descriptor, K-major, no swizzle: start address, LBO = byte distance between
// the core matrices of one MMA's two K halves, SBO = between 8-row groups (sm100 descriptor
// version 1; base offset 0)
__device__ __forceinline__ uint64_t umma_desc_kmajor(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// instruction descriptor: D FP32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12 = 1), both K-major,
// N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t umma_idesc_bf16_f32(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

constexpr int TCI_M = 128, TCI_THREADS = 512, TCI_TMEM_COLS = 128;
// accumulator columns per warp: the 4 warps of a lane quarter split the 64 columns of each layer
constexpr int TCI_CW = MLP_H * TCI_M / TCI_THREADS;
static_assert(TCI_CW == 16, "one 32x32b.x16 TMEM load per warp and layer");
constexpr int TCI_K1 = IND_KPAD / 8, TCI_K2 = MLP_H / 8;  // 16-byte chunks along K: 30, 8
// shared memory (bytes); every operand region 128-byte aligned
constexpr size_t TCI_OFF_EIDX = 128;                                   // int [128][5]
constexpr size_t TCI_OFF_VEC = TCI_OFF_EIDX + TCI_M * 5 * 4;           // float b1, b2, w3, b3
constexpr size_t TCI_OFF_ZP = TCI_OFF_VEC + 1024;                      // float [column group][128]
constexpr size_t TCI_OFF_W1 = TCI_OFF_ZP + (TCI_THREADS / TCI_M) * TCI_M * 4;  // 64 x 240 bf16
constexpr size_t TCI_OFF_W2 = TCI_OFF_W1 + (size_t)MLP_H * IND_KPAD * 2;
constexpr size_t TCI_OFF_A1 = TCI_OFF_W2 + (size_t)MLP_H * MLP_H * 2;  // 128 x 240 bf16
constexpr size_t TCI_OFF_A2 = TCI_OFF_A1 + (size_t)TCI_M * IND_KPAD * 2;
constexpr size_t TCI_SMEM_BYTES = TCI_OFF_A2 + (size_t)TCI_M * MLP_H * 2;
static_assert(TCI_OFF_W1 % 128 == 0 && TCI_OFF_W2 % 128 == 0 && TCI_OFF_A1 % 128 == 0 && TCI_OFF_A2 % 128 == 0,
              "UMMA operands must be 128-byte aligned");
static_assert(TCI_SMEM_BYTES <= 227 * 1024, "shared memory");

// byte offset of the 16-byte chunk kc of row r in a K-major operand of `rows` rows
__device__ __forceinline__ uint32_t kmajor_chunk(int r, int kc, int rows) {
  return (uint32_t)(((kc * (rows / 8) + (r >> 3)) << 7) + ((r & 7) << 4));
}

__global__ void __launch_bounds__(TCI_THREADS, 1) indicator_infer_tc_kernel(const IndicatorArgs a) {
  extern __shared__ __align__(128) unsigned char tsm[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(tsm);
  uint32_t* s_taddr = reinterpret_cast<uint32_t*>(tsm + 8);
  int* s_ok = reinterpret_cast<int*>(tsm + 12);
  int* eidx = reinterpret_cast<int*>(tsm + TCI_OFF_EIDX);
  float* vs = reinterpret_cast<float*>(tsm + TCI_OFF_VEC);
  float* zp = reinterpret_cast<float*>(tsm + TCI_OFF_ZP);
  unsigned char* w1s = tsm + TCI_OFF_W1;
  unsigned char* w2s = tsm + TCI_OFF_W2;
  unsigned char* a1s = tsm + TCI_OFF_A1;
  unsigned char* a2s = tsm + TCI_OFF_A2;
  if (a.scal && a.scal->flags) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // ---- set-up: tensor memory, barrier, weights in the UMMA layout ----
  if (warp == 0) {
    tmem_alloc_warp(s_taddr, TCI_TMEM_COLS);
    tmem_relinquish_warp();
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  for (int i = tid; i < MLP_H * TCI_K1; i += TCI_THREADS) {  // W1 [n][k], 16-byte chunks
    const int n = i / TCI_K1, kc = i % TCI_K1;
    *reinterpret_cast<uint4*>(w1s + kmajor_chunk(n, kc, MLP_H)) =
        *reinterpret_cast<const uint4*>(a.w1 + (size_t)n * IND_KPAD + kc * 8);
  }
  for (int i = tid; i < MLP_H * TCI_K2; i += TCI_THREADS) {
    const int n = i / TCI_K2, kc = i % TCI_K2;
    *reinterpret_cast<uint4*>(w2s + kmajor_chunk(n, kc, MLP_H)) =
        *reinterpret_cast<const uint4*>(a.w2 + (size_t)n * MLP_H + kc * 8);
  }
  for (int i = tid; i < 3 * MLP_H + 1; i += TCI_THREADS) vs[i] = a.vec[i];
  fence_proxy_async_smem();
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
  const uint32_t taddr = *s_taddr;
  constexpr uint32_t idesc = umma_idesc_bf16_f32(TCI_M, MLP_H);
  const uint32_t a1 = smem_u32(a1s), a2 = smem_u32(a2s), w1 = smem_u32(w1s), w2 = smem_u32(w2s);
  // this warp's accumulator block: TMEM lanes 32 (warp % 4) .., columns TCI_CW (warp / 4) ..
  const int q = warp & 3, h = warp >> 2, row = 32 * q + lane;
  const uint32_t tq = taddr + ((uint32_t)(32 * q) << 16) + (uint32_t)(TCI_CW * h);
  uint32_t phase = 0;
  bool ok = true;
  auto wait_mma = [&]() -> bool {  // uniform across the CTA
    if (tid == 0) {
      bool done = mbar_wait(bar, phase & 1u);
      if (!done) {
        atomicOr(a.errflag, (unsigned)FLAG_TIMEOUT);
        mbar_wait(bar, phase & 1u);
      }
      *s_ok = done ? 1 : 0;
    }
    ++phase;
    __syncthreads();
    tc_fence_after_sync();
    return *s_ok != 0;
  };

  const int ntiles = (a.n_elem + TCI_M - 1) / TCI_M;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    // ---- features: element indices of (row, neighbour), then one work item per (row, neighbour)
    for (int qq = tid; qq < TCI_M * 5; qq += TCI_THREADS) {
      const int r = qq / 5, n = qq - 5 * r, es = tile * TCI_M + r;
      int v = es < a.n_elem ? es : -1;
      if (v >= 0 && n > 0) {
        const int nb = __ldg(a.nbr + (size_t)(n - 1) * a.ld + es);
        v = nb >= 0 ? nb : es;
      }
      eidx[qq] = v;
    }
    __syncthreads();
    for (int qq = tid; qq < TCI_M * 5; qq += TCI_THREADS) {
      const int r = qq / 5, n = qq - 5 * r;
      const int es = eidx[r * 5], en = eidx[qq];
      if (es < 0) {
#pragma unroll
        for (int j = 0; j < IND_NSEG / 8; ++j)
          *reinterpret_cast<uint4*>(a1s + kmajor_chunk(r, 6 * n + j, TCI_M)) = make_uint4(0u, 0u, 0u, 0u);
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
        *reinterpret_cast<uint4*>(a1s + kmajor_chunk(r, 6 * n + j, TCI_M)) =
            make_uint4(pack_bf16(v[8 * j], v[8 * j + 1]), pack_bf16(v[8 * j + 2], v[8 * j + 3]),
                       pack_bf16(v[8 * j + 4], v[8 * j + 5]), pack_bf16(v[8 * j + 6], v[8 * j + 7]));
    }
    fence_proxy_async_smem();
    tc_fence_before_sync();
    __syncthreads();
    // ---- layer 1: [128 x 240] x [240 x 64] into TMEM columns 0..63 ----
    if (tid == 0) {
      tc_fence_after_sync();
#pragma unroll 1
      for (int s = 0; s < TCI_K1 / 2; ++s)
        umma_f16(taddr, umma_desc_kmajor(a1 + 4096u * s, 2048u, 128u), umma_desc_kmajor(w1 + 2048u * s, 1024u, 128u),
                 idesc, s > 0);
      umma_commit(bar);
    }
    if (!(ok = wait_mma())) break;
    {
      float acc[TCI_CW];
      tmem_ld16(tq, acc);
#pragma unroll
      for (int c = 0; c < TCI_CW / 8; ++c) {  // this warp's hidden units = A2 chunks (TCI_CW / 8) h + c
        uint32_t p[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int u = 8 * c + 2 * j;
          p[j] = pack_bf16(gelu_fast(acc[u] + vs[TCI_CW * h + u]), gelu_fast(acc[u + 1] + vs[TCI_CW * h + u + 1]));
        }
        *reinterpret_cast<uint4*>(a2s + kmajor_chunk(row, (TCI_CW / 8) * h + c, TCI_M)) =
            make_uint4(p[0], p[1], p[2], p[3]);
      }
    }
    fence_proxy_async_smem();
    tc_fence_before_sync();
    __syncthreads();
    // ---- layer 2: [128 x 64] x [64 x 64] into TMEM columns 64..127 ----
    if (tid == 0) {
      tc_fence_after_sync();
#pragma unroll 1
      for (int s = 0; s < TCI_K2 / 2; ++s)
        umma_f16(taddr + MLP_H, umma_desc_kmajor(a2 + 4096u * s, 2048u, 128u),
                 umma_desc_kmajor(w2 + 2048u * s, 1024u, 128u), idesc, s > 0);
      umma_commit(bar);
    }
    if (!(ok = wait_mma())) break;
    {
      float acc[TCI_CW];
      tmem_ld16(tq + MLP_H, acc);
      float z = 0.f;
#pragma unroll
      for (int u = 0; u < TCI_CW; ++u)
        z += gelu_fast(acc[u] + vs[MLP_H + TCI_CW * h + u]) * vs[2 * MLP_H + TCI_CW * h + u];
      zp[h * TCI_M + row] = z;
    }
    tc_fence_before_sync();
    __syncthreads();
    // ---- decisions (warps 0..3: one row each), flagged rows appended with one atomic per warp
    if (h == 0) {
      const int e = tile * TCI_M + row;
      bool f = false;
      if (e < a.n_elem) {
        float z = vs[3 * MLP_H];
#pragma unroll
        for (int g = 0; g < TCI_THREADS / TCI_M; ++g) z += zp[g * TCI_M + row];
        const float sc = 1.f / (1.f + expf(-z));
        a.score[e] = sc;
        f = sc > a.threshold;
        a.flag[e] = f;
      }
      const unsigned m = __ballot_sync(0xffffffffu, f);
      int base = 0;
      if (lane == 0 && m) base = atomicAdd(a.count, __popc(m));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (f) a.list[base + __popc(m & ((1u << lane) - 1u))] = e;
    }
  }
  // ---- release the tensor memory (every tcgen05.ld of this CTA has completed) ----
  tc_fence_before_sync();
  __syncthreads();
  tc_fence_after_sync();
  if (warp == 0) tmem_dealloc_warp(taddr, TCI_TMEM_COLS);
}

}  // namespace dgb
