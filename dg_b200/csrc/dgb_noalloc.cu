// dgb_limit_noalloc: the slope limiter without any device allocation.
//
// Who needs it: code that owns its device buffers and may not allocate device memory itself --
// for example a host application that runs under a fixed device-memory budget it has already
// claimed (a memory pool sized at start-up), or a caller that must not trigger an allocation
// (and its implicit device synchronisation) in the middle of its time loop.  Such a caller cannot
// use dgb_create, which allocates the state buffers and the limiter scratch of a context.
//
// This entry point takes the state in the caller's device memory and keeps its temporaries in
// one file-scope __device__ array of fixed size (kNoAllocScratchBytes below), which every GPU
// that loads this library holds until the process exits.  Nothing here calls cudaMalloc,
// cudaFree or an allocating library routine.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dgb.h"
#include "device/limiter2d_tile.cuh"
#include "host/host.h"

namespace dgb {
int set_error(int code, const std::string& msg);
}
const dgb::Problem& dgb_problem_ref(const dgb_problem* p);

using namespace dgb;

namespace {

// Maximum scratch: 128 MiB.  Layout per call: neighbour table (4 x ld int32), tensor node
// permutation (16 int32, padded to 256 bytes), the state in the library's internal layout
// (N_F x N_s x ld doubles) and the limiter's x-pass output (6 x N_s x ld doubles).
constexpr size_t kNoAllocScratchBytes = size_t(128) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_dev[kMaxDevices] = {nullptr};

double fact(int n) { double f = 1; for (int i = 2; i <= n; ++i) f *= i; return f; }

// limiter tables of order P from the reference element alone (same construction as the context's)
template <int P>
LimTab<P> make_limtab() {
  constexpr int n1 = P + 1;
  LimTab<P> t;
  std::memset(&t, 0, sizeof(t));
  std::vector<double> xs(n1), xf, wf;
  for (int i = 0; i < n1; ++i) xs[i] = -1.0 + 2.0 * i / P;
  gauss_legendre(n1, xf, wf);
  std::vector<double> V((size_t)n1 * n1), phi1((size_t)n1 * n1);
  for (int g = 0; g < n1; ++g)
    for (int j = 0; j < n1; ++j) {
      V[g + (size_t)j * n1] = std::pow(xf[g], j) / fact(j);
      phi1[g + (size_t)j * n1] = lagrange1d(xs, j, xf[g]);
    }
  invert(V, n1);
  std::vector<double> T((size_t)n1 * n1, 0.0);
  for (int m = 0; m < n1; ++m)
    for (int i = 0; i < n1; ++i) {
      double s = 0;
      for (int g = 0; g < n1; ++g) s += V[m + (size_t)g * n1] * phi1[g + (size_t)i * n1];
      T[m + (size_t)i * n1] = s;
    }
  std::vector<double> Ti = T;
  invert(Ti, n1);
  for (int m = 0; m < n1; ++m)
    for (int i = 0; i < n1; ++i) { t.T[m][i] = T[m + (size_t)i * n1]; t.Tinv[i][m] = Ti[i + (size_t)m * n1]; }
  for (int k = 0; k < n1; ++k)
    for (int n = 0; n < n1; ++n) {
      const int num = n - k + 1;
      if (num < 1) continue;
      t.imd[k][n] = (num % 2) ? 2.0 / fact(num) : 0.0;
      t.imdL[k][n] = (std::pow(-1.0, num) - std::pow(-3.0, num)) / fact(num);
      t.imdR[k][n] = (std::pow(3.0, num) - std::pow(1.0, num)) / fact(num);
    }
  for (int k = 0; k < P + 3; ++k) t.ifact[k] = 1.0 / fact(k);
  return t;
}

// Once per device, with that device current: the device address of the scratch array and the
// limiter tables of this translation unit's kernels.
int setup_device(int dev, void** scratch) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (dev < 0 || dev >= kMaxDevices) return set_error(DGB_ERR_ARG, "device index out of range");
  if (g_scratch_dev[dev]) {
    *scratch = g_scratch_dev[dev];
    return DGB_OK;
  }
  void* ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if (e != cudaSuccess || !ptr)
    return set_error(DGB_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
  const LimTab<1> t1 = make_limtab<1>();
  const LimTab<2> t2 = make_limtab<2>();
  const LimTab<3> t3 = make_limtab<3>();
  if ((e = cudaMemcpyToSymbol(c_lim_p1, &t1, sizeof(t1))) != cudaSuccess ||
      (e = cudaMemcpyToSymbol(c_lim_p2, &t2, sizeof(t2))) != cudaSuccess ||
      (e = cudaMemcpyToSymbol(c_lim_p3, &t3, sizeof(t3))) != cudaSuccess)
    return set_error(DGB_ERR_CUDA, std::string("limiter tables: ") + cudaGetErrorString(e));
  g_scratch_dev[dev] = ptr;
  *scratch = ptr;
  return DGB_OK;
}

struct View {
  int D, p, nf, ns, ne, ld, nx, ny;
  bool rowmajor;
  const int* nbr;
  const int* perm;
  double* Uint;
  double* X;
};

template <int P, int METHOD>
void launch(const View& v, cudaStream_t st) {
  const LimArgs la{v.ld, v.ne};
  if (v.D == 1) {
    lim1d_kernel<P, METHOD><<<(v.ne + 127) / 128, 128, 0, st>>>(la, v.Uint, v.nbr, v.X, nullptr);
    return;
  }
  if (v.rowmajor) {
    dim3 gx((v.nx + 29) / 30, v.ny), bx(32, P + 1);
    lim2d_xpass_tile_kernel<P, METHOD><<<gx, bx, 0, st>>>(la, v.nx, v.Uint, v.nbr, v.X, nullptr);
    dim3 gy((v.nx + 31) / 32, (v.ny + 3) / 4, P + 1), by(32, 6);
    lim2d_ypass_tile_kernel<P, METHOD><<<gy, by, 0, st>>>(la, v.nx, v.ny, v.X, v.nbr, v.Uint, nullptr);
  } else {
    dim3 grid((v.ne + 127) / 128, P + 1);
    lim2d_xpass_kernel<P, METHOD><<<grid, 128, 0, st>>>(la, v.Uint, v.nbr, v.X, nullptr);
    lim2d_ypass_kernel<P, METHOD><<<grid, 128, 0, st>>>(la, v.X, v.nbr, v.Uint, nullptr);
  }
}

// The neighbour table nbr[k*ld + e] of a structured grid (a 1D chain or a row-major nx x ny grid)
// from the rule of each side (a boundary code < 0, or kSideWrap: the element on the opposite
// side); columns beyond N_E hold the "frozen" code -4.  Filled on the device, so a call on a
// structured problem copies nothing from the host.
struct SideRules {
  int rule[4];
};

__global__ void structured_nbr_kernel(int* nbr, int ld, int ne, int nx, int ny, int nsides, SideRules r) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ld) return;
  const int ix = e % nx, iy = e / nx;
  for (int k = 0; k < nsides; ++k) {
    int v = -4;
    if (e < ne) {
      const bool edge = k == 0 ? ix == 0 : k == 1 ? ix == nx - 1 : k == 2 ? iy == 0 : iy == ny - 1;
      const int inner = k == 0 ? e - 1 : k == 1 ? e + 1 : k == 2 ? e - nx : e + nx;
      const int wrap = k == 0 ? e + nx - 1 : k == 1 ? e - (nx - 1) : k == 2 ? e + (ny - 1) * nx : e - (ny - 1) * nx;
      v = !edge ? inner : r.rule[k] == Problem::kSideWrap ? wrap : r.rule[k];
    }
    nbr[(size_t)k * ld + e] = v;
  }
}

struct NodePerm {
  int t[MAXNS];
};

__global__ void store_perm_kernel(int* dst, int n, NodePerm p) {
  if ((int)threadIdx.x < n) dst[threadIdx.x] = p.t[threadIdx.x];
}

}  // namespace

extern "C" int dgb_limit_noalloc(const dgb_problem* prob, const double* U_in_dev, double* U_out_dev, void* stream) {
  if (!prob || !U_in_dev || !U_out_dev) return set_error(DGB_ERR_ARG, "null argument");
  const Problem& P = dgb_problem_ref(prob);
  if (!P.gpu_ok) return set_error(DGB_ERR_UNSUPPORTED, P.gpu_reason);
  if (P.N_Y != 0 || P.gamcons)
    return set_error(DGB_ERR_UNSUPPORTED, "dgb_limit_noalloc: GAMNCON problems without mass fractions");
  if (P.limiter != DGB_LIM_HRL && P.limiter != DGB_LIM_M2L)
    return set_error(DGB_ERR_UNSUPPORTED, "dgb_limit_noalloc supports the hrl and m2l limiters");
  const int ld = (P.N_E + 63) / 64 * 64;
  const size_t nbr_bytes = (size_t)P.N_N * ld * sizeof(int);
  const size_t perm_off = (nbr_bytes + 255) / 256 * 256;
  const size_t uint_off = perm_off + 256;
  const size_t uint_bytes = (size_t)P.N_F * P.N_s * ld * sizeof(double);
  const size_t x_off = uint_off + (uint_bytes + 255) / 256 * 256;
  const size_t x_bytes = (size_t)std::max(6, P.N_F) * P.N_s * ld * sizeof(double);
  const size_t need = x_off + x_bytes;
  if (need > kNoAllocScratchBytes)
    return set_error(DGB_ERR_ARG, "dgb_limit_noalloc: this problem needs " + std::to_string(need) +
                                      " bytes of scratch but the library holds " +
                                      std::to_string(kNoAllocScratchBytes) + " (" + std::to_string(P.N_E) +
                                      " elements of order " + std::to_string(P.p) + " is too large)");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(DGB_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  void* scratch = nullptr;
  if (int rc = setup_device(dev, &scratch)) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char* base = static_cast<unsigned char*>(scratch);
  View v;
  v.D = P.D; v.p = P.p; v.nf = P.N_F; v.ns = P.N_s; v.ne = P.N_E; v.ld = ld; v.nx = P.nx; v.ny = P.ny;
  v.rowmajor = P.D == 2 && P.structured;
  v.nbr = reinterpret_cast<const int*>(base);
  v.perm = reinterpret_cast<const int*>(base + perm_off);
  v.Uint = reinterpret_cast<double*>(base + uint_off);
  v.X = reinterpret_cast<double*>(base + x_off);
  // the neighbour table: built on the device for a structured grid whose sides each follow one
  // rule (found when the problem was set up); otherwise copied from the host (a pageable copy:
  // CUDA stages it before returning, after synchronising the stream)
  const int nsides = P.D == 1 ? 2 : 4;
  bool uniform = P.structured;
  for (int k = 0; k < nsides; ++k) uniform = uniform && P.side_rule[k] != Problem::kSideMixed;
  if (uniform) {
    SideRules r;
    for (int k = 0; k < 4; ++k) r.rule[k] = P.side_rule[k];
    structured_nbr_kernel<<<(ld + 255) / 256, 256, 0, st>>>(reinterpret_cast<int*>(base), ld, P.N_E, P.nx, P.ny,
                                                             nsides, r);
  } else {
    std::vector<int> nb((size_t)P.N_N * ld, -4);
    for (int k = 0; k < P.N_N; ++k)
      for (int el = 0; el < P.N_E; ++el) nb[(size_t)k * ld + el] = P.nbr[(size_t)k * P.N_E + el];
    if ((e = cudaMemcpyAsync(base, nb.data(), nbr_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
      return set_error(DGB_ERR_CUDA, std::string("neighbour upload: ") + cudaGetErrorString(e));
  }
  NodePerm np;
  for (int t = 0; t < MAXNS; ++t) np.t[t] = t < P.N_s ? P.tensor_perm[t] : 0;
  store_perm_kernel<<<1, 32, 0, st>>>(reinterpret_cast<int*>(base + perm_off), P.N_s, np);
  const int grid = (int)std::min<size_t>(((size_t)P.N_E * P.N_F * P.N_s + 255) / 256, 148 * 32);
  ref_to_internal_kernel<<<grid, 256, 0, st>>>(U_in_dev, v.Uint, v.perm, P.N_E, P.N_F, P.N_s, ld);
  const int key = P.p * 10 + P.limiter;
  switch (key) {
    case 11: launch<1, 1>(v, st); break;
    case 12: launch<1, 2>(v, st); break;
    case 21: launch<2, 1>(v, st); break;
    case 22: launch<2, 2>(v, st); break;
    case 31: launch<3, 1>(v, st); break;
    case 32: launch<3, 2>(v, st); break;
    default: return set_error(DGB_ERR_UNSUPPORTED, "order outside 1..3");
  }
  // the 1D limiter writes its result to the x-pass buffer, the 2D passes back into Uint
  internal_to_ref_kernel<<<grid, 256, 0, st>>>(P.D == 1 ? v.X : v.Uint, U_out_dev, v.perm, P.N_E, P.N_F, P.N_s, ld);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return set_error(DGB_ERR_CUDA, std::string("dgb_limit_noalloc: ") + cudaGetErrorString(e));
  return DGB_OK;
}
