// The device context of one problem (the opaque dgb_ctx of include/dgb.h), shared by the
// single-problem entry points (dgb_device.cu) and the batched ensemble (dgb_batch.cu).
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "../../include/dgb.h"
#include "device/common.cuh"
#include "device/limiter_gated.cuh"
#include "device/sensor.h"

namespace dgb {
// Dynamic shared memory above 48 KB is opted into per kernel, and cudaFuncSetAttribute acts on the
// current device only: done once per (kernel, device), under a lock
inline cudaError_t allow_dynamic_smem(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({kernel, dev})) return cudaSuccess;
  err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (err == cudaSuccess) done.insert({kernel, dev});
  return err;
}
template <typename K>
inline cudaError_t allow_dynamic_smem(K* kernel, size_t bytes) {
  return allow_dynamic_smem(reinterpret_cast<const void*>(kernel), bytes);
}

// element chunks of the host-resident time loop's copies (dgb_advance_host): at most, by default
constexpr int kHostChunks = 16, kHostChunksDefault = 16;

enum { KC_RESIDUAL = 0, KC_LIMITER = 1, KC_DT = 2, KC_INDICATOR = 3, KC_OTHER = 4, KC_N = 5 };
}

struct dgb_ctx {
  int device = 0;
  cudaStream_t st = nullptr;
  int D = 1, p = 1, nf = 4, ns = 2, ne = 0, ld = 0, flux = 2, limiter = 0;
  int nx = 0, ny = 0;
  int nmass = 0;          // passive mass fractions (fields D+3 .. nf-1)
  bool gamcons = false;   // GAMCONS gamma model (fifth field rho/(gamma-1), conservative)
  // slab mode (dgb_slab_ghost_rows): ghost rows at the bottom / top of a structured grid, filled by
  // the caller's halo exchange; the phase-level step (dgb_step_*) and its position
  int halo_lo = 0, halo_hi = 0;
  double* slab_cur = nullptr;   // the buffer the next stage reads (packed / unpacked by dgb_halo_*)
  int slab_scheme = 0, slab_next = -1;
  bool slab_cfl = false;
  bool tiled = false;     // structured row-major grid with at least one full tile: tiled residual kernel
  bool tile_tma = false;  // ... with tensor maps for its tile loads (row pitch nx * 8 a multiple of 16)
  bool tiled_full = false;  // ... with TMA and extents that are tile multiples (no leftover strips)
  int* left = nullptr;    // the elements outside the full tiles (generic residual kernel), nleft of them
  int nleft = 0;
  int form = DGB_FORM_FP64;  // arithmetic of the residual: plain FP64 or mixed FP32/FP64
  long long wait_polls = 1ll << 22;  // poll budget of the residual kernels' first wait per tile copy
  bool rowmajor = false;  // structured row-major grid: tiled limiter passes
  bool chain1d = false;   // 1D elements in chain order: fused residual + limiter stages
  bool fused_lim = false; // row-major grid, hrl / m2l: both limiter passes in one kernel (opt-in)
  CUtensorMap mapA, mapB, mapC;  // TMA descriptors of the state buffers (tiled kernel)
  double hx = 0, hy = 0;
  size_t nstate = 0;
  dgb::Consts cs;
  double *A = nullptr, *B = nullptr, *C = nullptr, *DU = nullptr, *X = nullptr, *ref = nullptr;
  int *nbr = nullptr, *perm = nullptr;
  // sensor-gated limiters (hri, m2i, pri, p0i): sensor work arrays and flags
  bool gated = false, has_sensors = false;
  int sm_count = 148;           // multiprocessors of the device
  bool ind_on = false;          // learned indicator gates the limiter (dgb_set_indicator)
  bool mixed_ct = false;        // mixed form: the compressed-tile kernel (else the TMA-tile kernel)
  bool pdl = true;              // programmatic dependent launches (kernels that wait in pdl_wait)
  bool tile_dmma = false;       // p = 2 FP64 stages: the DMMA residual (else the scalar tiled kernel)
  bool ind_tc = true;           // scoring GEMMs on tcgen05 (else the mma.sync kernel)
  float ind_threshold = 0.2f;
  float* ind_params = nullptr;  // FP32 parameters (MLP_NPARAM)
  __nv_bfloat16* ind_w = nullptr;  // W1 [64][IND_KPAD] then W2 [64][64], BF16
  float* ind_vec = nullptr;     // b1, b2, w3, b3
  float* ind_modes = nullptr;   // [N_E][IND_MODES]
  float* ind_score = nullptr;   // [N_E]
  unsigned char* ind_flag = nullptr;
  int* ind_list = nullptr;      // [N_E] + count
  unsigned char* ind_band = nullptr;  // flagged elements and their neighbours
  int* ind_blist = nullptr;     // [N_E] + count: the band as a list
  int* ind_tiles = nullptr;     // row-major grids: the gated passes' tiles with band elements,
  int ind_n0 = 0, ind_n1 = 0;   //   [n0] x-pass tiles, [n1] y-pass tiles, then the two counts
  dgb::SensorLaunch sl;
  int* iperm = nullptr;
  double* smean = nullptr;
  int* sint = nullptr;          // target, type, processed, mask, list (ld each), count, flags (ld)
  dgb::CellAverageWeights p0w;       // p0i: cell-average weights in internal node order
  dgb::DevScalars* scal = nullptr;
  dgb::DevScalars* h_scal = nullptr;  // pinned
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double last_ms = 0.0;
  long long last_launches = 0;
  long long launches_per_step = 0;
  // captured steps per [scheme: SSP-RK3, RK4][CFL step][the step scores the learned indicator]
  cudaGraphExec_t graphs[2][2][2] = {};
  long long graph_launches[2][2][2] = {};
  int ind_every = 1;       // steps between scorings of the learned indicator (1: every step)
  long long ind_step = 0;  // steps taken since the last dgb_set_state / dgb_set_indicator
  // destroys the captured steps (their kernel arguments or launch sequence changed)
  unsigned graph_gen = 0;   // counts drop_graphs calls (captured slab steps compare it)
  double* halo_send[2] = {nullptr, nullptr};  // slab mode, local exchange: packed owned rows per side
  // dgb_advance_host: upload / download streams, per-chunk events (uploaded, downloaded, converted
  // for the download), the end of the last download
  int host_chunks = dgb::kHostChunksDefault;
  cudaStream_t hl_st[2] = {nullptr, nullptr};
  cudaEvent_t hl_up[dgb::kHostChunks] = {}, hl_down[dgb::kHostChunks] = {}, hl_conv[dgb::kHostChunks] = {};
  cudaEvent_t hl_done = nullptr;
  void drop_graphs() {
    ++graph_gen;
    for (auto& a : graphs)
      for (auto& b : a)
        for (auto& g : b)
          if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  }
  // profiling (per kernel class)
  bool prof = false;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pev;
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  double kc_ms[dgb::KC_N] = {0, 0, 0, 0, 0};
  long long kc_n[dgb::KC_N] = {0, 0, 0, 0, 0};
  long long counter = 0;  // launches issued since the last reset
};


namespace dgb {
int set_error(int code, const std::string& msg);

// an event of the context's profiling pool (reused from one profiled call to the next)
inline cudaEvent_t pool_event(dgb_ctx* c) {
  if (c->ev_used == c->ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    c->ev_pool.push_back(e);
  }
  return c->ev_pool[c->ev_used++];
}

// one kernel launch of kernel class kc: counted, and bracketed by events when profiling is on
struct ProfScope {
  dgb_ctx* c;
  int kc;
  cudaEvent_t a = nullptr, b = nullptr;
  ProfScope(dgb_ctx* ctx, int k) : c(ctx), kc(k) {
    c->counter++;
    if (c->prof) { a = pool_event(c); b = pool_event(c); cudaEventRecord(a, c->st); }
  }
  ~ProfScope() {
    if (c->prof) { cudaEventRecord(b, c->st); c->pev.push_back({kc, {a, b}}); }
  }
};
// TMA descriptor of one of the context's state buffers with a tw x th element box
bool encode_state_map(dgb_ctx* c, double* ptr, CUtensorMap* map, int tw, int th);
}
