// Batched ensemble (include/dgb.h, "Batched ensemble"): many independent problems, each with its
// own device context and CFL step, advanced together with SSP-RK3.
//
// The cases are grouped into element classes (dimension, order, flux, limiter).  Per class and
// operator there is one persistent launch over a list of work items (device/batch.cuh); one step of
// the whole ensemble -- per class: wave speeds, the step's finish, three stages of residual and
// limiter -- is captured once into a CUDA graph whose class branches run concurrently on their own
// streams, and replayed.  Tile shape, quadrature-loop unrolling and persistent grid size of the
// residual launches are chosen per class by the autotuner below, which times the candidates on
// the cases' current states.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/dgb.h"
#include "ctx.h"
#include "device/batch.cuh"
#include "device/tables.cuh"

using namespace dgb;

#define DGB_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t err_ = (call);                                                                  \
    if (err_ != cudaSuccess)                                                                    \
      return set_error(DGB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(err_));     \
  } while (0)

namespace {

// residual tile shapes of the 2D classes: width, height (elements), unrolling of the quadrature
// column loop
struct Shape2 {
  int tw, th, unroll;
};
constexpr Shape2 kShapes2[] = {{32, 4, 1}, {32, 2, 1}, {16, 8, 1}, {32, 4, 2}};
constexpr int kNShapes2 = sizeof(kShapes2) / sizeof(kShapes2[0]);
constexpr int kChunks1[] = {64, 128, 256};  // elements per CTA item of the 1D classes

struct Class {
  int D = 1, p = 1, flux = 0, limiter = 0;
  std::vector<int> cases;  // batch indices
  cudaStream_t st = nullptr;
  int* d_ids = nullptr;
  // work items
  int4* d_res = nullptr;  // 2D: tiles of the chosen shape; 1D: element chunks (also the 1D limiter's)
  int n_res = 0;
  int4* d_x = nullptr;  // 2D limiter x pass
  int n_x = 0;
  int4* d_y = nullptr;  // 2D limiter y pass
  int n_y = 0;
  int4* d_ws = nullptr;  // wave speed: chunks of 256 elements
  int n_ws = 0;
  // tuning
  int shape = 0;         // 2D: index into kShapes2
  int chunk = 128;       // 1D: elements per item
  int ctas_per_sm = 0;   // persistent grid of the residual (0: the occupancy limit)
  std::vector<int> valid_shapes;
  double tuned_us = 0.0;  // measured stage-0 residual time of the chosen configuration
};

}  // namespace

struct dgb_batch {
  int device = 0, n = 0, sm_count = 148;
  std::vector<dgb_ctx*> ctx;
  std::vector<Class> cls;
  BatchCase* d_cases = nullptr;
  BatchMaps* d_maps = nullptr;
  Consts* d_consts = nullptr;
  BatchProgress* d_prog = nullptr;
  unsigned long long* d_t0 = nullptr;
  double* d_tend = nullptr;
  int* d_active = nullptr;
  int* h_active = nullptr;  // pinned
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr, fork = nullptr;
  std::vector<cudaEvent_t> joins;
  cudaGraphExec_t graph = nullptr;
  long long launches_per_step = 0, last_launches = 0;
  double last_ms = 0.0;
  int last_steps = 0;
};

namespace {

int4 item(int c, int x, int y, int z) { return make_int4(c, x, y, z); }

template <typename T>
int upload_vec(const std::vector<T>& v, T** d) {
  if (*d) cudaFree(*d);
  *d = nullptr;
  if (v.empty()) return 0;
  DGB_CUDA(cudaMalloc(d, v.size() * sizeof(T)));
  DGB_CUDA(cudaMemcpy(*d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return 0;
}

// residual items of a class for its current tuning; 2D: TMA maps of its cases for the shape
int build_res_items(dgb_batch* b, Class& k) {
  std::vector<int4> it;
  if (k.D == 2) {
    const Shape2 s = kShapes2[k.shape];
    std::vector<BatchMaps> maps(k.cases.size());
    for (size_t j = 0; j < k.cases.size(); ++j) {
      dgb_ctx* c = b->ctx[k.cases[j]];
      for (int ty = 0; ty < c->ny; ty += s.th)
        for (int tx = 0; tx < c->nx; tx += s.tw) it.push_back(item(k.cases[j], tx, ty, 0));
      double* bufs[3] = {c->A, c->B, c->C};
      for (int q = 0; q < 3; ++q)
        if (!encode_state_map(c, bufs[q], &maps[j].m[q], s.tw, s.th))
          return set_error(DGB_ERR_CUDA, "batch: TMA descriptor of a case could not be encoded");
    }
    for (size_t j = 0; j < k.cases.size(); ++j)
      DGB_CUDA(cudaMemcpy(b->d_maps + k.cases[j], &maps[j], sizeof(BatchMaps), cudaMemcpyHostToDevice));
  } else {
    for (int ci : k.cases)
      for (int e = 0; e < b->ctx[ci]->ne; e += k.chunk) it.push_back(item(ci, e, 0, 0));
  }
  k.n_res = (int)it.size();
  return upload_vec(it, &k.d_res);
}

int build_items(dgb_batch* b, Class& k) {
  std::vector<int4> ws, xs, ys;
  for (int ci : k.cases) {
    dgb_ctx* c = b->ctx[ci];
    for (int e = 0; e < c->ne; e += 256) ws.push_back(item(ci, e, 0, 0));
    if (k.D == 2 && k.limiter) {
      for (int y = 0; y < c->ny; ++y)
        for (int x = 0; x < c->nx; x += 30) xs.push_back(item(ci, x, y, 0));
      for (int ix = 0; ix <= k.p; ++ix)
        for (int y = 0; y < c->ny; y += 4)
          for (int x = 0; x < c->nx; x += 32) ys.push_back(item(ci, x, y, ix));
    }
  }
  k.n_ws = (int)ws.size();
  k.n_x = (int)xs.size();
  k.n_y = (int)ys.size();
  if (int rc = upload_vec(ws, &k.d_ws)) return rc;
  if (int rc = upload_vec(xs, &k.d_x)) return rc;
  if (int rc = upload_vec(ys, &k.d_y)) return rc;
  std::vector<int> ids(k.cases.begin(), k.cases.end());
  if (int rc = upload_vec(ids, &k.d_ids)) return rc;
  return build_res_items(b, k);
}

template <typename K>
int persistent_grid(dgb_batch* b, K kernel, int threads, size_t smem, int n_items, int per_sm) {
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem);
  occ = std::max(occ, 1);
  if (per_sm > 0) occ = std::min(occ, per_sm);
  return std::max(1, std::min(n_items, b->sm_count * occ));
}

// ---- launchers (templated on the class's compile-time parameters) ----

template <int P, int FLUX, int TW, int TH, int UNROLL>
int launch_tile2d_batch(dgb_batch* b, const Class& k, int stage, cudaStream_t st) {
  auto kern = batch_tile2d_kernel<P, FLUX, TW, TH, UNROLL>;
  constexpr size_t smem = batch_tile2d_smem_bytes<P, TW, TH>();
  DGB_CUDA(allow_dynamic_smem(kern, smem));
  const int grid = persistent_grid(b, kern, TW * TH, smem, k.n_res, k.ctas_per_sm);
  kern<<<grid, TW * TH, smem, st>>>(b->d_cases, b->d_maps, k.d_res, k.n_res, stage);
  return 0;
}

template <int P, int FLUX>
int tile2d_shape(dgb_batch* b, const Class& k, int stage, cudaStream_t st) {
  switch (k.shape) {
    case 0: return launch_tile2d_batch<P, FLUX, 32, 4, 1>(b, k, stage, st);
    case 1: return launch_tile2d_batch<P, FLUX, 32, 2, 1>(b, k, stage, st);
    case 2: return launch_tile2d_batch<P, FLUX, 16, 8, 1>(b, k, stage, st);
    case 3: return launch_tile2d_batch<P, FLUX, 32, 4, 2>(b, k, stage, st);
    default: return set_error(DGB_ERR_ARG, "batch: tile shape");
  }
}

template <int P, int FLUX, bool LIM>
int launch_res1d_batch(dgb_batch* b, const Class& k, int stage, cudaStream_t st) {
  auto kern = batch_res1d_kernel<P, FLUX, LIM>;
  const int grid = persistent_grid(b, kern, k.chunk, 0, k.n_res, k.ctas_per_sm);
  kern<<<grid, k.chunk, 0, st>>>(b->d_cases, b->d_consts, k.d_res, k.n_res, stage);
  return 0;
}

template <int P, int FLUX>
int res1d_lim(dgb_batch* b, const Class& k, int stage, cudaStream_t st) {
  return k.limiter ? launch_res1d_batch<P, FLUX, true>(b, k, stage, st)
                   : launch_res1d_batch<P, FLUX, false>(b, k, stage, st);
}

int launch_residual(dgb_batch* b, const Class& k, int stage, cudaStream_t st) {
  const int key = k.D * 100 + k.p * 10 + k.flux;
  switch (key) {
    case 210: return tile2d_shape<1, 0>(b, k, stage, st);
    case 212: return tile2d_shape<1, 2>(b, k, stage, st);
    case 220: return tile2d_shape<2, 0>(b, k, stage, st);
    case 222: return tile2d_shape<2, 2>(b, k, stage, st);
    case 110: return res1d_lim<1, 0>(b, k, stage, st);
    case 111: return res1d_lim<1, 1>(b, k, stage, st);
    case 112: return res1d_lim<1, 2>(b, k, stage, st);
    case 120: return res1d_lim<2, 0>(b, k, stage, st);
    case 121: return res1d_lim<2, 1>(b, k, stage, st);
    case 122: return res1d_lim<2, 2>(b, k, stage, st);
    case 130: return res1d_lim<3, 0>(b, k, stage, st);
    case 131: return res1d_lim<3, 1>(b, k, stage, st);
    case 132: return res1d_lim<3, 2>(b, k, stage, st);
    default: return set_error(DGB_ERR_UNSUPPORTED, "batch: no residual for this class");
  }
}

template <int P, int M>
int launch_lim2d_batch(dgb_batch* b, const Class& k, int stage, cudaStream_t st) {
  auto kx = batch_lim2d_x_kernel<P, M>;
  auto ky = batch_lim2d_y_kernel<P, M>;
  const int gx = persistent_grid(b, kx, 32 * (P + 1), 0, k.n_x, 0);
  const int gy = persistent_grid(b, ky, 32 * 6, 0, k.n_y, 0);
  kx<<<gx, dim3(32, P + 1), 0, st>>>(b->d_cases, k.d_x, k.n_x, stage);
  ky<<<gy, dim3(32, 6), 0, st>>>(b->d_cases, k.d_y, k.n_y, stage);
  return 0;
}

template <int P, int M>
int launch_lim1d_batch(dgb_batch* b, const Class& k, int stage, cudaStream_t st) {
  auto kern = batch_lim1d_kernel<P, M>;
  const int grid = persistent_grid(b, kern, k.chunk, 0, k.n_res, 0);
  kern<<<grid, k.chunk, 0, st>>>(b->d_cases, k.d_res, k.n_res, stage);
  return 0;
}

// returns the number of launches enqueued (>= 0) or -(status)
int launch_limiter(dgb_batch* b, const Class& k, int stage, cudaStream_t st) {
  if (!k.limiter) return 0;
  const int key = k.D * 100 + k.p * 10 + k.limiter;
  int rc;
  switch (key) {
    case 211: rc = launch_lim2d_batch<1, 1>(b, k, stage, st); break;
    case 212: rc = launch_lim2d_batch<1, 2>(b, k, stage, st); break;
    case 221: rc = launch_lim2d_batch<2, 1>(b, k, stage, st); break;
    case 222: rc = launch_lim2d_batch<2, 2>(b, k, stage, st); break;
    case 111: rc = launch_lim1d_batch<1, 1>(b, k, stage, st); break;
    case 112: rc = launch_lim1d_batch<1, 2>(b, k, stage, st); break;
    case 121: rc = launch_lim1d_batch<2, 1>(b, k, stage, st); break;
    case 122: rc = launch_lim1d_batch<2, 2>(b, k, stage, st); break;
    case 131: rc = launch_lim1d_batch<3, 1>(b, k, stage, st); break;
    case 132: rc = launch_lim1d_batch<3, 2>(b, k, stage, st); break;
    default: return -set_error(DGB_ERR_UNSUPPORTED, "batch: no limiter for this class");
  }
  if (rc) return -rc;
  return k.D == 2 ? 2 : 1;
}

int launch_dt(dgb_batch* b, const Class& k, cudaStream_t st) {
  const int ns = k.D == 2 ? (k.p + 1) * (k.p + 1) : k.p + 1;
  const int key = k.D * 100 + ns;
  auto go = [&](auto kern) {
    const int grid = persistent_grid(b, kern, 256, 0, k.n_ws, 0);
    kern<<<grid, 256, 0, st>>>(b->d_cases, k.d_ws, k.n_ws);
  };
  switch (key) {
    case 102: go(batch_wavespeed_kernel<1, 2>); break;
    case 103: go(batch_wavespeed_kernel<1, 3>); break;
    case 104: go(batch_wavespeed_kernel<1, 4>); break;
    case 204: go(batch_wavespeed_kernel<2, 4>); break;
    case 209: go(batch_wavespeed_kernel<2, 9>); break;
    default: return set_error(DGB_ERR_UNSUPPORTED, "batch: no wave-speed kernel for this class");
  }
  const int nc = (int)k.cases.size();
  batch_finish_dt_kernel<<<(nc + 127) / 128, 128, 0, st>>>(b->d_cases, b->d_prog, k.d_ids, nc, b->d_tend);
  return 0;
}

// one step of one class on stream st; returns launches (>= 0) or -(status)
int enqueue_class_step(dgb_batch* b, const Class& k, cudaStream_t st) {
  int n = 0;
  if (int rc = launch_dt(b, k, st)) return -rc;
  n += 2;
  for (int s = 0; s < 3; ++s) {
    if (int rc = launch_residual(b, k, s, st)) return -rc;
    n += 1;
    const int nl = launch_limiter(b, k, s, st);
    if (nl < 0) return nl;
    n += nl;
  }
  return n;
}

// the whole ensemble's step: class branches forked from and joined into b->st
int enqueue_step(dgb_batch* b) {
  DGB_CUDA(cudaEventRecord(b->fork, b->st));
  long long n = 0;
  for (size_t j = 0; j < b->cls.size(); ++j) {
    Class& k = b->cls[j];
    DGB_CUDA(cudaStreamWaitEvent(k.st, b->fork, 0));
    const int r = enqueue_class_step(b, k, k.st);
    if (r < 0) return -r;
    n += r;
    DGB_CUDA(cudaEventRecord(b->joins[j], k.st));
    DGB_CUDA(cudaStreamWaitEvent(b->st, b->joins[j], 0));
  }
  DGB_CUDA(cudaGetLastError());
  b->launches_per_step = n;
  return 0;
}

void drop_graph(dgb_batch* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
}

__global__ void count_active_kernel(const BatchCase* __restrict__ cases, int n, int* active) {
  int a = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) a += cases[i].scal->flags == 0;
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  __shared__ int s[32];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
    *active = t;
  }
}

__global__ void clear_done_kernel(const BatchCase* __restrict__ cases, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) cases[i].scal->flags &= ~(unsigned)FLAG_DONE;
}

int reset_cases(dgb_batch* b) {
  for (dgb_ctx* c : b->ctx) {
    std::memset(c->h_scal, 0, sizeof(DevScalars));
    DGB_CUDA(cudaMemcpyAsync(c->scal, c->h_scal, sizeof(DevScalars), cudaMemcpyHostToDevice, b->st));
  }
  DGB_CUDA(cudaMemsetAsync(b->d_prog, 0, b->n * sizeof(BatchProgress), b->st));
  return 0;
}

}  // namespace

extern "C" int dgb_batch_create(dgb_ctx* const* cases, int n, dgb_batch** out) {
  if (!cases || !out || n <= 0) return set_error(DGB_ERR_ARG, "batch: null argument or no cases");
  *out = nullptr;
  const int dev = cases[0] ? cases[0]->device : 0;
  std::map<std::tuple<int, int, int, int>, int> key2cls;
  auto* b = new dgb_batch();
  b->device = dev;
  b->n = n;
  auto fail = [&](int rc) {
    dgb_batch_destroy(b);
    return rc;
  };
  for (int i = 0; i < n; ++i) {
    dgb_ctx* c = cases[i];
    if (!c) return fail(set_error(DGB_ERR_ARG, "batch: null case"));
    if (c->device != dev) return fail(set_error(DGB_ERR_ARG, "batch: cases on different devices"));
    for (int j = 0; j < i; ++j)
      if (cases[j] == c) return fail(set_error(DGB_ERR_ARG, "batch: a context appears twice"));
    if (c->nmass != 0 || c->gamcons)
      return fail(set_error(DGB_ERR_UNSUPPORTED, "batch: GAMNCON cases without mass fractions"));
    if (c->form != DGB_FORM_FP64 || c->ind_on || c->fused_lim)
      return fail(set_error(DGB_ERR_UNSUPPORTED, "batch: plain FP64 form with the two-pass limiter only"));
    if (c->limiter != DGB_LIM_NONE && c->limiter != DGB_LIM_HRL && c->limiter != DGB_LIM_M2L)
      return fail(set_error(DGB_ERR_UNSUPPORTED, "batch: limiter none, hrl or m2l"));
    if (c->D == 2 && (!c->tiled_full || c->p > 2))
      return fail(set_error(DGB_ERR_UNSUPPORTED,
                            "batch: 2D cases must be structured row-major grids, p <= 2, nx % 32 == 0, ny % 4 == 0"));
    if (!(c->cs.cfl_scaled > 0)) return fail(set_error(DGB_ERR_ARG, "batch: every case needs a positive CFL"));
    b->ctx.push_back(c);
    const auto key = std::make_tuple(c->D, c->p, c->flux, c->limiter);
    auto f = key2cls.find(key);
    if (f == key2cls.end()) {
      Class k;
      k.D = c->D; k.p = c->p; k.flux = c->flux; k.limiter = c->limiter;
      key2cls[key] = (int)b->cls.size();
      b->cls.push_back(k);
      f = key2cls.find(key);
    }
    b->cls[f->second].cases.push_back(i);
  }
  if (cudaSetDevice(dev) != cudaSuccess) return fail(set_error(DGB_ERR_CUDA, "batch: device"));
  cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, dev);
  std::vector<BatchCase> hc(n);
  std::vector<Consts> hk(n);
  for (int i = 0; i < n; ++i) {
    dgb_ctx* c = b->ctx[i];
    BatchCase& q = hc[i];
    std::memset(&q, 0, sizeof(q));
    q.A = c->A; q.B = c->B; q.C = c->C; q.X = c->X; q.nbr = c->nbr; q.scal = c->scal;
    q.nx = c->nx; q.ny = c->ny; q.ld = c->ld; q.ne = c->ne;
    q.J = c->cs.J;
    q.invJ = 1.0 / c->cs.J;
    q.cx = c->cs.J * c->cs.ixx;
    q.cy = c->cs.J * c->cs.iyy;
    q.sx = c->cs.ixx;
    q.sy = c->cs.iyy;
    q.JFx = c->cs.JFx;
    q.JFy = c->cs.JFy;
    q.cfl_scaled = c->cs.cfl_scaled;
    hk[i] = c->cs;
  }
  if (int rc = upload_vec(hc, &b->d_cases)) return fail(rc);
  if (int rc = upload_vec(hk, &b->d_consts)) return fail(rc);
  if (cudaMalloc(&b->d_maps, n * sizeof(BatchMaps)) != cudaSuccess ||
      cudaMalloc(&b->d_prog, n * sizeof(BatchProgress)) != cudaSuccess ||
      cudaMalloc(&b->d_t0, sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&b->d_tend, sizeof(double)) != cudaSuccess || cudaMalloc(&b->d_active, sizeof(int)) != cudaSuccess ||
      cudaMallocHost(&b->h_active, sizeof(int)) != cudaSuccess)
    return fail(set_error(DGB_ERR_CUDA, "batch: allocation"));
  cudaMemset(b->d_maps, 0, n * sizeof(BatchMaps));
  cudaMemset(b->d_prog, 0, n * sizeof(BatchProgress));
  cudaMemset(b->d_tend, 0, sizeof(double));
  if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&b->e0) != cudaSuccess || cudaEventCreate(&b->e1) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
    return fail(set_error(DGB_ERR_CUDA, "batch: stream / events"));
  for (Class& k : b->cls) {
    if (cudaStreamCreateWithFlags(&k.st, cudaStreamNonBlocking) != cudaSuccess)
      return fail(set_error(DGB_ERR_CUDA, "batch: class stream"));
    cudaEvent_t j;
    if (cudaEventCreateWithFlags(&j, cudaEventDisableTiming) != cudaSuccess)
      return fail(set_error(DGB_ERR_CUDA, "batch: class event"));
    b->joins.push_back(j);
    if (k.D == 2) {
      for (int s = 0; s < kNShapes2; ++s) {
        bool ok = true;
        for (int ci : k.cases) ok = ok && b->ctx[ci]->nx % kShapes2[s].tw == 0 && b->ctx[ci]->ny % kShapes2[s].th == 0;
        if (ok) k.valid_shapes.push_back(s);
      }
      k.shape = k.valid_shapes.front();  // 32 x 4 is always valid for a tiled case
    }
    // this file's copies of the constant tables (every case of a group has the same order)
    if (int rc = upload_tables(b->ctx[k.cases.front()]->cs, k.D, k.p)) return fail(rc);
    if (int rc = build_items(b, k)) return fail(rc);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(set_error(DGB_ERR_CUDA, "batch: create"));
  *out = b;
  return DGB_OK;
}

extern "C" void dgb_batch_destroy(dgb_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->st) cudaStreamSynchronize(b->st);
  drop_graph(b);
  for (Class& k : b->cls) {
    if (k.st) { cudaStreamSynchronize(k.st); cudaStreamDestroy(k.st); }
    for (void* q : {(void*)k.d_ids, (void*)k.d_res, (void*)k.d_x, (void*)k.d_y, (void*)k.d_ws})
      if (q) cudaFree(q);
  }
  for (void* q : {(void*)b->d_cases, (void*)b->d_maps, (void*)b->d_consts, (void*)b->d_prog, (void*)b->d_t0,
                  (void*)b->d_tend, (void*)b->d_active})
    if (q) cudaFree(q);
  if (b->h_active) cudaFreeHost(b->h_active);
  for (cudaEvent_t e : b->joins) cudaEventDestroy(e);
  for (cudaEvent_t e : {b->e0, b->e1, b->fork})
    if (e) cudaEventDestroy(e);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
}

extern "C" int dgb_batch_n_classes(dgb_batch* b) { return b ? (int)b->cls.size() : 0; }

extern "C" int dgb_batch_class_info(dgb_batch* b, int k, int* info) {
  if (!b || !info || k < 0 || k >= (int)b->cls.size()) return set_error(DGB_ERR_ARG, "batch: bad class index");
  const Class& c = b->cls[k];
  info[0] = c.D;
  info[1] = c.p;
  info[2] = c.flux;
  info[3] = c.limiter;
  info[4] = (int)c.cases.size();
  info[5] = c.D == 2 ? kShapes2[c.shape].tw : c.chunk;
  info[6] = c.D == 2 ? kShapes2[c.shape].th : 1;
  info[7] = c.D == 2 ? kShapes2[c.shape].unroll : 0;
  info[8] = c.ctas_per_sm;
  info[9] = (int)(c.tuned_us * 1000.0 + 0.5);  // ns
  return DGB_OK;
}

extern "C" int dgb_batch_autotune(dgb_batch* b, int reps) {
  if (!b) return set_error(DGB_ERR_ARG, "batch: null");
  if (reps < 1) reps = 5;
  DGB_CUDA(cudaSetDevice(b->device));
  // the stage-0 residual reads A and writes B (or X): the states are untouched; the scalars (dt,
  // time) of one CFL step are saved and put back
  if (int rc = reset_cases(b)) return rc;
  double zero = 0.0;
  DGB_CUDA(cudaMemcpyAsync(b->d_tend, &zero, sizeof(double), cudaMemcpyHostToDevice, b->st));
  for (Class& k : b->cls)
    if (int rc = launch_dt(b, k, b->st)) return rc;
  DGB_CUDA(cudaStreamSynchronize(b->st));
  for (Class& k : b->cls) {
    struct Cand {
      int shape, chunk, per_sm;
    };
    std::vector<Cand> cand;
    if (k.D == 2) {
      for (int s : k.valid_shapes)
        for (int ps : {0, 1}) cand.push_back({s, 0, ps});
    } else {
      for (int ch : kChunks1)
        for (int ps : {0, 4}) cand.push_back({0, ch, ps});
    }
    double best = 1e30;
    Cand pick = cand.front();
    for (const Cand& cd : cand) {
      k.shape = cd.shape;
      if (k.D == 1) k.chunk = cd.chunk;
      k.ctas_per_sm = cd.per_sm;
      if (int rc = build_res_items(b, k)) return rc;
      for (int w = 0; w < 2; ++w)
        if (int rc = launch_residual(b, k, 0, b->st)) return rc;
      DGB_CUDA(cudaEventRecord(b->e0, b->st));
      for (int r = 0; r < reps; ++r)
        if (int rc = launch_residual(b, k, 0, b->st)) return rc;
      DGB_CUDA(cudaEventRecord(b->e1, b->st));
      DGB_CUDA(cudaEventSynchronize(b->e1));
      float ms = 0;
      DGB_CUDA(cudaEventElapsedTime(&ms, b->e0, b->e1));
      const double us = 1e3 * ms / reps;
      if (us < best) { best = us; pick = cd; }
    }
    k.shape = pick.shape;
    if (k.D == 1) k.chunk = pick.chunk;
    k.ctas_per_sm = pick.per_sm;
    k.tuned_us = best;
    if (int rc = build_res_items(b, k)) return rc;
  }
  DGB_CUDA(cudaGetLastError());
  if (int rc = reset_cases(b)) return rc;
  DGB_CUDA(cudaStreamSynchronize(b->st));
  drop_graph(b);
  return DGB_OK;
}

extern "C" int dgb_batch_set_tuning(dgb_batch* b, int k, int tile_w, int tile_h, int unroll, int ctas_per_sm) {
  if (!b || k < 0 || k >= (int)b->cls.size()) return set_error(DGB_ERR_ARG, "batch: bad class index");
  if (ctas_per_sm < 0) return set_error(DGB_ERR_ARG, "batch: ctas_per_sm < 0");
  DGB_CUDA(cudaSetDevice(b->device));
  Class& c = b->cls[k];
  if (c.D == 2) {
    int found = -1;
    for (int s : c.valid_shapes)
      if (kShapes2[s].tw == tile_w && kShapes2[s].th == tile_h && kShapes2[s].unroll == unroll) found = s;
    if (found < 0) return set_error(DGB_ERR_ARG, "batch: tile shape not among this group's candidates");
    c.shape = found;
  } else {
    if (std::find(std::begin(kChunks1), std::end(kChunks1), tile_w) == std::end(kChunks1))
      return set_error(DGB_ERR_ARG, "batch: elements per CTA must be 64, 128 or 256");
    c.chunk = tile_w;
  }
  c.ctas_per_sm = ctas_per_sm;
  c.tuned_us = 0.0;
  if (int rc = build_res_items(b, c)) return rc;
  drop_graph(b);
  return DGB_OK;
}

extern "C" int dgb_batch_advance(dgb_batch* b, int nsteps, double t_end, int* steps_run) {
  if (!b) return set_error(DGB_ERR_ARG, "batch: null");
  if (nsteps < 0) return set_error(DGB_ERR_ARG, "batch: nsteps < 0");
  DGB_CUDA(cudaSetDevice(b->device));
  if (!b->graph) {
    cudaGraph_t g;
    DGB_CUDA(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_step(b);
    const cudaError_t ec = cudaStreamEndCapture(b->st, &g);
    if (rc) {
      if (ec == cudaSuccess) cudaGraphDestroy(g);
      return rc;
    }
    DGB_CUDA(ec);
    DGB_CUDA(cudaGraphInstantiate(&b->graph, g, 0));
    cudaGraphDestroy(g);
  }
  if (int rc = reset_cases(b)) return rc;
  const double te = t_end > 0 ? t_end : 0.0;
  DGB_CUDA(cudaMemcpyAsync(b->d_tend, &te, sizeof(double), cudaMemcpyHostToDevice, b->st));
  DGB_CUDA(cudaStreamSynchronize(b->st));
  batch_start_kernel<<<1, 1, 0, b->st>>>(b->d_t0);
  DGB_CUDA(cudaEventRecord(b->e0, b->st));
  int s = 0;
  for (; s < nsteps; ++s) {
    DGB_CUDA(cudaGraphLaunch(b->graph, b->st));
    if (te > 0 && (s + 1) % 16 == 0) {  // every case at its end time (or failed): stop early
      count_active_kernel<<<1, 256, 0, b->st>>>(b->d_cases, b->n, b->d_active);
      DGB_CUDA(cudaMemcpyAsync(b->h_active, b->d_active, sizeof(int), cudaMemcpyDeviceToHost, b->st));
      DGB_CUDA(cudaStreamSynchronize(b->st));
      if (*b->h_active == 0) { ++s; break; }
    }
  }
  DGB_CUDA(cudaEventRecord(b->e1, b->st));
  DGB_CUDA(cudaEventSynchronize(b->e1));
  float ms = 0;
  DGB_CUDA(cudaEventElapsedTime(&ms, b->e0, b->e1));
  b->last_ms = ms;
  b->last_steps = s;
  b->last_launches = b->launches_per_step * s;
  if (steps_run) *steps_run = s;
  // errors of any case; then the stop marks are cleared so that the contexts are usable alone
  int first_bad = -1;
  unsigned bad_flags = 0;
  for (int i = 0; i < b->n; ++i) {
    dgb_ctx* c = b->ctx[i];
    DGB_CUDA(cudaMemcpy(c->h_scal, c->scal, sizeof(DevScalars), cudaMemcpyDeviceToHost));
    const unsigned f = c->h_scal->flags & ~(unsigned)FLAG_DONE;
    if (f && first_bad < 0) { first_bad = i; bad_flags = f; }
  }
  clear_done_kernel<<<(b->n + 127) / 128, 128, 0, b->st>>>(b->d_cases, b->n);
  DGB_CUDA(cudaStreamSynchronize(b->st));
  DGB_CUDA(cudaGetLastError());
  if (first_bad >= 0) {
    const std::string w = "batch case " + std::to_string(first_bad) + ": ";
    if (bad_flags & FLAG_TIMEOUT) return set_error(DGB_ERR_TIMEOUT, w + "a bounded device wait expired");
    if (bad_flags & FLAG_NONFINITE) return set_error(DGB_ERR_NONFINITE, w + "time step is NaN");
    return set_error(DGB_ERR_DT_SMALL, w + "next time step is too small (< 1e-14)");
  }
  return DGB_OK;
}

extern "C" int dgb_batch_case_stats(dgb_batch* b, double* time, int* steps, double* wall_ms) {
  if (!b) return set_error(DGB_ERR_ARG, "batch: null");
  DGB_CUDA(cudaSetDevice(b->device));
  std::vector<BatchProgress> pr(b->n);
  unsigned long long t0 = 0;
  DGB_CUDA(cudaMemcpy(pr.data(), b->d_prog, b->n * sizeof(BatchProgress), cudaMemcpyDeviceToHost));
  DGB_CUDA(cudaMemcpy(&t0, b->d_t0, sizeof(t0), cudaMemcpyDeviceToHost));
  for (int i = 0; i < b->n; ++i) {
    dgb_ctx* c = b->ctx[i];
    DGB_CUDA(cudaMemcpy(c->h_scal, c->scal, sizeof(DevScalars), cudaMemcpyDeviceToHost));
    if (time) time[i] = c->h_scal->time;
    if (steps) steps[i] = pr[i].steps;
    if (wall_ms) wall_ms[i] = pr[i].t_done_ns ? 1e-6 * (double)(pr[i].t_done_ns - t0) : -1.0;
  }
  return DGB_OK;
}

extern "C" int dgb_batch_last_timing(dgb_batch* b, double* ms, long long* launches) {
  if (!b) return set_error(DGB_ERR_ARG, "batch: null");
  if (ms) *ms = b->last_ms;
  if (launches) *launches = b->last_launches;
  return DGB_OK;
}
