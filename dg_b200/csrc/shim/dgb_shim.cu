// Link-compatible shim: the reference's extern "C" kernel launchers (code/src/dg/kernels.h,
// physics/physics.h, bc/boundaries.h, time_integration/rk_kernels.h, limiting/limiting_kernels.h,
// sensors/sensor_kernels.h, printer/printer_kernels.h) with the same names, signatures, device
// pointers and reference layouts, implemented with this library's CUDA code, so that the
// reference's own host classes (DG_SOLVER, RK, Limiting, SENSOR, PRINTER) can drive them for A/B
// runs.  Like the reference, one build per configuration: DGB_SHIM_D (1 or 2; N_F = 4 or 5, the
// GAMNCON gamma model, no mass fractions) and DGB_SHIM_FLUX (0 Rusanov, 1 HLL (1D), 2 Roe).
// Gravity (constants::GLOBAL_GX / GY) is taken as zero.  Launches go to the default stream, as
// the reference's do; errors are reported on stderr (the reference's launchers return void).
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "device/physics.cuh"
#include "device/sensor.h"

#ifndef DGB_SHIM_D
#define DGB_SHIM_D 2
#endif
#ifndef DGB_SHIM_FLUX
#define DGB_SHIM_FLUX 0
#endif

typedef double scalar;

namespace {

constexpr int D = DGB_SHIM_D, N_F = D + 3, FLUX = DGB_SHIM_FLUX;
constexpr int kBlock = 256;

inline int blocks(long n) { return (int)((n + kBlock - 1) / kBlock); }
void check(const char* who) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) std::fprintf(stderr, "dgb shim %s: %s\n", who, cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------------------------
// dg/kernels.h
// ---------------------------------------------------------------------------------------------
__global__ void map_to_face(long n, const int* map, const scalar* U, scalar* UF) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k < n) UF[k] = U[map[k]];
}

__global__ void map_to_element(int N_s, int N_E, int M_s, int N_N, const int* invmap, scalar* Q, const scalar* q) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // (e, fc)
  if (k >= (long)N_E * N_F) return;
  scalar* out = Q + k * N_s;
  for (int i = 0; i < N_s; ++i) out[i] = 0.0;
  const int* im = invmap + k * M_s * N_N * 2;
  for (int i = 0; i < M_s * N_N; ++i) out[im[2 * i]] += q[im[2 * i + 1]];
}

__global__ void redistribute_sf(int N_G, int N_E, scalar* sJ, scalar* fJ, const scalar* s, const scalar* f,
                                const scalar* J, const scalar* invJac) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // ((e*N_F + fc)*N_G + g)
  if (k >= (long)N_E * N_F * N_G) return;
  const int g = (int)(k % N_G);
  const long ef = k / N_G;
  const int e = (int)(ef / N_F);
  const scalar j = J[e];
  sJ[k] = s[k] * j;
  for (int al = 0; al < D; ++al) {
    scalar sol = 0.0;
    for (int a = 0; a < D; ++a) sol += invJac[(((long)e * N_G + g) * D + al) * D + a] * f[k * D + a] * j;
    fJ[k * D + al] = sol;
  }
}

__global__ void redistribute_q(int M_G, int M_T, scalar* qJ, const scalar* q, const scalar* JF) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // (((t*N_F + fc)*2 + d)*M_G + g)
  if (k >= (long)M_T * N_F * 2 * M_G) return;
  const int d = (int)((k / M_G) % 2);
  const long t = k / ((long)M_G * 2 * N_F);
  qJ[k] = q[k] * JF[t * 2 + d];
}

__global__ void add_sfq(long n, scalar* A, const scalar* S, const scalar* F, const scalar* Q) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k < n) A[k] = S[k] + F[k] + Q[k];
}

// ---------------------------------------------------------------------------------------------
// physics/physics.h (gamma model, GAMNCON)
// ---------------------------------------------------------------------------------------------
__global__ void evaluate_sf(int N_G, int N_E, scalar* s, scalar* f, const scalar* Ug, const scalar* dUg,
                            const scalar* invJac) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // (e, g)
  if (k >= (long)N_E * N_G) return;
  const int e = (int)(k / N_G), g = (int)(k % N_G);
  auto idx = [&](int fc) { return ((long)e * N_F + fc) * N_G + g; };
  const scalar rho = Ug[idx(0)], u = Ug[idx(1)] / rho;
  if (D == 1) {
    const scalar Et = Ug[idx(2)], gamma = 1 + 1.0 / Ug[idx(3)];
    const scalar p = (gamma - 1) * (Et - 0.5 * rho * u * u);
    s[idx(0)] = 0; s[idx(1)] = 0; s[idx(2)] = 0;
    f[idx(0)] = rho * u;
    f[idx(1)] = rho * u * u + p;
    f[idx(2)] = (Et + p) * u;
    s[idx(3)] = -u * dUg[idx(3)] * invJac[(long)e * N_G + g];
    f[idx(3)] = 0;
  } else {
    const scalar v = Ug[idx(2)] / rho, Et = Ug[idx(3)], gamma = 1 + 1.0 / Ug[idx(4)];
    const scalar p = (gamma - 1) * (Et - 0.5 * rho * (u * u + v * v));
    for (int fc = 0; fc < 4; ++fc) s[idx(fc)] = 0;
    const scalar fx[5] = {rho * u, rho * u * u + p, rho * u * v, (Et + p) * u, 0};
    const scalar fy[5] = {rho * v, rho * u * v, rho * v * v + p, (Et + p) * v, 0};
    for (int fc = 0; fc < 5; ++fc) { f[idx(fc) * 2 + 0] = fx[fc]; f[idx(fc) * 2 + 1] = fy[fc]; }
    scalar vg = 0;
    for (int al = 0; al < 2; ++al)
      vg += -u * dUg[idx(4) * 2 + al] * invJac[(((long)e * N_G + g) * 2 + 0) * 2 + al] -
            v * dUg[idx(4) * 2 + al] * invJac[(((long)e * N_G + g) * 2 + 1) * 2 + al];
    s[idx(4)] = vg;
  }
}

__global__ void evaluate_q(int M_G, int M_T, scalar* q, const scalar* UgF, const scalar* normals) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // (t, g)
  if (k >= (long)M_T * M_G) return;
  const long t = k / M_G;
  const int g = (int)(k % M_G);
  auto L = [&](int fc) { return UgF[((t * N_F + fc) * 2 + 0) * M_G + g]; };
  auto R = [&](int fc) { return UgF[((t * N_F + fc) * 2 + 1) * M_G + g]; };
  double F[5] = {0, 0, 0, 0, 0}, nc = 0;
  if (D == 1) {
    dgb::phys::riemann1d<FLUX>(L(0), R(0), L(1) / L(0), R(1) / R(0), L(2), R(2), L(3), R(3), normals[t * D], F, nc);
  } else {
    dgb::phys::riemann2d<FLUX == 1 ? 0 : FLUX>(L(0), R(0), L(1) / L(0), R(1) / R(0), L(2) / L(0), R(2) / R(0), L(3),
                                                R(3), L(4), R(4), normals[t * D], normals[t * D + 1], F, nc);
  }
  for (int fc = 0; fc < N_F; ++fc) {
    const scalar ncf = fc == N_F - 1 ? nc : 0.0;
    q[((t * N_F + fc) * 2 + 0) * M_G + g] = -F[fc] + ncf;
    q[((t * N_F + fc) * 2 + 1) * M_G + g] = F[fc] + ncf;
  }
}

__global__ void kinetic_energy(long n, const scalar* rho, const scalar* rhou, const scalar* rhov, scalar* K) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const scalar kin = rhou[k] * rhou[k] + (rhov ? rhov[k] * rhov[k] : 0.0);
  K[k] = 0.5 * kin / rho[k];
}

__global__ void pressure(int N_s, int N_E, const scalar* U, scalar* p) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // (e, i)
  if (k >= (long)N_E * N_s) return;
  const long e = k / N_s;
  const int i = (int)(k % N_s);
  auto u = [&](int fc) { return U[(e * N_F + fc) * N_s + i]; };
  const scalar gamma = 1.0 + 1.0 / u(N_F - 1);
  const scalar kin = D == 1 ? u(1) * u(1) : u(1) * u(1) + u(2) * u(2);
  p[k] = (gamma - 1) * (u(D + 1) - 0.5 * kin / u(0));
}

// ---------------------------------------------------------------------------------------------
// bc/boundaries.h, time_integration/rk_kernels.h
// ---------------------------------------------------------------------------------------------
__global__ void reflective(int M_s, int M_B, const int* boundaryMap, const scalar* normals, int start, scalar* UF) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // (b, j)
  if (k >= (long)M_B * M_s) return;
  const long t = boundaryMap[start + k / M_s];
  const int j = (int)(k % M_s);
  if (D == 1) {
    UF[((t * N_F + 1) * 2 + 1) * M_s + j] = -UF[((t * N_F + 1) * 2 + 1) * M_s + j];
  } else {
    const scalar nx = normals[t * 2], ny = normals[t * 2 + 1];
    const scalar nx2 = nx * nx, ny2 = ny * ny, m2nxny = -2 * nx * ny, inv = 1.0 / (nx2 + ny2);
    const scalar vxL = UF[((t * N_F + 1) * 2 + 0) * M_s + j], vyL = UF[((t * N_F + 2) * 2 + 0) * M_s + j];
    UF[((t * N_F + 1) * 2 + 1) * M_s + j] = inv * ((-nx2 + ny2) * vxL + m2nxny * vyL);
    UF[((t * N_F + 2) * 2 + 1) * M_s + j] = inv * (m2nxny * vxL + (nx2 - ny2) * vyL);
  }
}

__global__ void solve(int N_s, int N_E, scalar Dt, const scalar* Minv, const scalar* f, scalar* DU) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // ((e*N_F + fc)*N_s + i)
  if (k >= (long)N_E * N_F * N_s) return;
  const int i = (int)(k % N_s);
  const long ef = k / N_s, e = ef / N_F;
  scalar sol = 0.0;
  for (int ii = 0; ii < N_s; ++ii) sol += Minv[(e * N_s + ii) * N_s + i] * f[ef * N_s + ii];
  DU[k] = Dt * sol;
}

__global__ void average_cell_p0(int N_s, int N_E, scalar* DU) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // (e, fc)
  if (k >= (long)N_E * N_F) return;
  scalar avg = 0.0;
  for (int i = 0; i < N_s; ++i) avg += DU[k * N_s + i];
  avg = avg / N_s;
  for (int i = 0; i < N_s; ++i) DU[k * N_s + i] = avg;
}

__global__ void find_upa(int N_s, int N_E, const scalar* U, scalar* UPA) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // (e, i)
  if (k >= (long)N_E * N_s) return;
  const long e = k / N_s;
  const int i = (int)(k % N_s);
  auto u = [&](int fc) { return U[(e * N_F + fc) * N_s + i]; };
  UPA[k] = D == 1 ? dgb::phys::wave_speed1d_quotients(u(0), u(1), u(2), u(3))
                  : dgb::phys::wave_speed2d_quotients(u(0), u(1), u(2), u(3), u(4));
}

}  // namespace

extern "C" void LmapToFace(int M_s, int M_T, int N_s, int* map, scalar* U, scalar* UF) {
  const long n = (long)M_T * N_F * 2 * M_s;
  map_to_face<<<blocks(n), kBlock>>>(n, map, U, UF);
  check("LmapToFace");
}
extern "C" void LmapToElement(int N_s, int N_E, int M_s, int N_N, int* invmap, scalar* Q, scalar* q) {
  map_to_element<<<blocks((long)N_E * N_F), kBlock>>>(N_s, N_E, M_s, N_N, invmap, Q, q);
  check("LmapToElement");
}
extern "C" void Lredistribute_sf(int N_G, int N_E, scalar* sJ, scalar* fJ, scalar* s, scalar* f, scalar* J,
                                 scalar* invJac) {
  redistribute_sf<<<blocks((long)N_E * N_F * N_G), kBlock>>>(N_G, N_E, sJ, fJ, s, f, J, invJac);
  check("Lredistribute_sf");
}
extern "C" void Lredistribute_q(int M_G, int M_T, scalar* qJ, scalar* q, scalar* JF) {
  redistribute_q<<<blocks((long)M_T * N_F * 2 * M_G), kBlock>>>(M_G, M_T, qJ, q, JF);
  check("Lredistribute_q");
}
extern "C" void LaddSFQ(int N_s, int N_E, scalar* A, scalar* S, scalar* F, scalar* Q) {
  const long n = (long)N_E * N_F * N_s;
  add_sfq<<<blocks(n), kBlock>>>(n, A, S, F, Q);
  check("LaddSFQ");
}
extern "C" void Levaluate_sf(int N_G, int N_E, scalar* s, scalar* f, scalar* Ug, scalar* dUg, scalar* invJac) {
  evaluate_sf<<<blocks((long)N_E * N_G), kBlock>>>(N_G, N_E, s, f, Ug, dUg, invJac);
  check("Levaluate_sf");
}
extern "C" void Levaluate_q(int M_G, int M_T, scalar* q, scalar* UgF, scalar* normals) {
  evaluate_q<<<blocks((long)M_T * M_G), kBlock>>>(M_G, M_T, q, UgF, normals);
  check("Levaluate_q");
}
extern "C" void Lkinetic_energy1D(int N_s, int N_E, scalar* rho, scalar* rhou, scalar* K) {
  const long n = (long)N_E * N_s;
  kinetic_energy<<<blocks(n), kBlock>>>(n, rho, rhou, nullptr, K);
  check("Lkinetic_energy1D");
}
extern "C" void Lkinetic_energy2D(int N_s, int N_E, scalar* rho, scalar* rhou, scalar* rhov, scalar* K) {
  const long n = (long)N_E * N_s;
  kinetic_energy<<<blocks(n), kBlock>>>(n, rho, rhou, rhov, K);
  check("Lkinetic_energy2D");
}
extern "C" void Lpressure(int N_s, int N_E, scalar* U, scalar* p) {
  pressure<<<blocks((long)N_E * N_s), kBlock>>>(N_s, N_E, U, p);
  check("Lpressure");
}
extern "C" void LrflctiveBoundary(int M_s, int M_B, int* boundaryMap, scalar* normals, int start, scalar* UF) {
  if (M_B <= 0) return;
  reflective<<<blocks((long)M_B * M_s), kBlock>>>(M_s, M_B, boundaryMap, normals, start, UF);
  check("LrflctiveBoundary");
}
extern "C" void Lsolver(int N_s, int N_E, scalar Dt, scalar* Minv, scalar* f, scalar* DU) {
  solve<<<blocks((long)N_E * N_F * N_s), kBlock>>>(N_s, N_E, Dt, Minv, f, DU);
  check("Lsolver");
}
extern "C" void Laverage_cell_p0(const int N_s, const int N_E, scalar* DU) {
  average_cell_p0<<<blocks((long)N_E * N_F), kBlock>>>(N_s, N_E, DU);
  check("Laverage_cell_p0");
}
extern "C" void LfindUPA(const int N_s, const int N_E, scalar* U, scalar* UPA) {
  find_upa<<<blocks((long)N_E * N_s), kBlock>>>(N_s, N_E, U, UPA);
  check("LfindUPA");
}

// ---------------------------------------------------------------------------------------------
// limiting/limiting_kernels.h: hierarchical reconstruction on scaled monomials, runtime order
// ---------------------------------------------------------------------------------------------
namespace {

__device__ double ifactorial(int n) {
  double f = 1.0;
  for (int k = 2; k <= n; ++k) f *= k;
  return 1.0 / f;
}
// integral over [-1, 1] of the k-th derivative of x^n / n!
__device__ double imd(int k, int n) {
  const int num = n - k + 1;
  return (num % 2) ? 2.0 * ifactorial(num) : 0.0;
}
// the same integral over [a, b]
__device__ double imd_bounds(int k, int n, double a, double b) {
  const int num = n - k + 1;
  return (pow(b, num) - pow(a, num)) * ifactorial(num);
}
__device__ double minmod2v(double a, double b) {
  const int sa = a > 0 ? 1 : (a < 0 ? -1 : 0), sb = b > 0 ? 1 : (b < 0 ? -1 : 0);
  if (sa != sb) return 0.0;
  return sa * fmin(fabs(a), fabs(b));
}
// limit_monomial (limiting_kernels.cu:1534-1585) for a monomial of order N
__device__ void limit_mono(int N, const double* AL, const double* AC, const double* AR, double* Alim) {
  double avgLC = 0.0;
  for (int m = N; m > 0; --m) {
    double dUL = 0, dUC = 0, dUR = 0, RL = 0, RC = 0, RR = 0;
    for (int n = m - 1; n <= N; ++n) {
      const double w = imd(m - 1, n);
      dUL += AL[n] * w;
      dUC += AC[n] * w;
      dUR += AR[n] * w;
      if (n >= m + 1) {
        RL += Alim[n] * imd_bounds(m - 1, n, -3, -1);
        RC += Alim[n] * w;
        RR += Alim[n] * imd_bounds(m - 1, n, 1, 3);
      }
    }
    const double LL = 0.5 * (dUL - RL);
    avgLC = 0.5 * (dUC - RC);
    const double LR = 0.5 * (dUR - RR);
    Alim[m] = minmod2v(0.5 * (avgLC - LL), 0.5 * (LR - avgLC));
  }
  Alim[0] = avgLC;
}
// average_monomial (limiting_kernels.cu:1777-1790)
__device__ void average_mono(int N, const double* A, double* Alim) {
  double avg = 0.0;
  for (int n = 0; n <= N; ++n) { avg += A[n] * imd(0, n); Alim[n] = 0.0; }
  Alim[0] = 0.5 * avg;
}

__global__ void strided_copy(int count, int blocklen, int strideA, int strideB, int offsetA, int offsetB,
                             const scalar* A, scalar* B) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= (long)count * blocklen) return;
  const long b = k / blocklen;
  const int j = (int)(k % blocklen);
  B[offsetB + b * strideB + j] = A[offsetA + b * strideA + j];
}

__global__ void reconstruct_energy(int N_s, int N_E, int slicenum, const scalar* rhoeLim, const scalar* KLim,
                                   const scalar* EMono, scalar* ELim) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // (e, slice)
  if (k >= (long)N_E * slicenum) return;
  const long base = k * N_s;
  for (int i = 1; i < N_s; ++i) ELim[base + i] = rhoeLim[base + i] + KLim[base + i];
  double E0 = EMono[base];
  for (int m = 2; m < N_s; m += 2) E0 -= ifactorial(m + 1) * (ELim[base + m] - EMono[base + m]);
  ELim[base] = E0;
}

__global__ void internal_energy(int N_s, int N_E, int slicenum, const scalar* p, const scalar* g, scalar* rhoe) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // (e, slice, i)
  if (k >= (long)N_E * slicenum * N_s) return;
  const int i = (int)(k % N_s);
  const long base = k - i;
  double I = 0.0, c = 1.0;  // c = binomial(i, kk)
  for (int kk = 0; kk <= i; ++kk) {
    I += c * p[base + i - kk] * g[base + kk];
    c = c * (i - kk) / (kk + 1);
  }
  rhoe[k] = I;
}

// hrl1D (limiting_kernels.cu:245-320)
__global__ void hrl1d(int N_s, int N_E, int Nfields, int N_N, int slicenum, const int* neighbors, int offxy,
                      const scalar* A, scalar* Alim) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // ((e*Nfields + fc)*slicenum + slice)
  if (k >= (long)N_E * Nfields * slicenum) return;
  const int slice = (int)(k % slicenum);
  const long ef = k / slicenum;
  const int fc = (int)(ef % Nfields);
  const long e = ef / Nfields;
  const int N = N_s - 1;
  const int left = neighbors[e * N_N + offxy], right = neighbors[e * N_N + offxy + 1];
  int physical = 0;
  if (left < 0) physical = -left;
  if (right < 0) physical = -right;
  const long idx = ef * N_s * slicenum + slice * N_s;
  if (physical == 4) return;  // left unchanged, as the reference leaves it
  if (physical == 2) { average_mono(N, A + idx, Alim + idx); return; }
  if (physical == 3) {
    const int un = offxy == 0 ? 1 : (offxy == 2 ? 2 : 0);
    if (fc != un) average_mono(N, A + idx, Alim + idx);
    else for (int n = 0; n <= N; ++n) Alim[idx + n] = A[idx + n];
    return;
  }
  const long iL = ((long)left * Nfields + fc) * N_s * slicenum + slice * N_s;
  const long iR = ((long)right * Nfields + fc) * N_s * slicenum + slice * N_s;
  limit_mono(N, A + iL, A + idx, A + iR, Alim + idx);
}

constexpr int kMaxNs = 16;

// y = M x, M column-major n x n (gemv, limiting_kernels.cu:1699-1716)
__device__ void gemv_cm(int n, const scalar* M, const double* x, double* y) {
  for (int m = 0; m < n; ++m) {
    double s = 0.0;
    for (int q = 0; q < n; ++q) s += M[q * n + m] * x[q];
    y[m] = s;
  }
}
// set2average / HR on a nodal vector u (limiting_kernels.cu:1792-1868); monolim receives Alim
__device__ void set2average_v(int N_s, int N_s1D, int slicenum, const scalar* L2M, const scalar* M2L, double* u,
                              double* monolim) {
  double A[kMaxNs], Al[kMaxNs];
  gemv_cm(N_s, L2M, u, A);
  for (int s = 0; s < slicenum; ++s) average_mono(N_s1D - 1, A + s * N_s1D, Al + s * N_s1D);
  gemv_cm(N_s, M2L, Al, u);
  if (monolim) for (int i = 0; i < N_s; ++i) monolim[i] = Al[i];
}
__device__ void hr_v(int N_s, int N_s1D, int slicenum, const scalar* L2M, const scalar* M2L, const double* uL,
                     double* uC, const double* uR, double* monolim) {
  double AL[kMaxNs], AC[kMaxNs], AR[kMaxNs], Al[kMaxNs];
  gemv_cm(N_s, L2M, uL, AL);
  gemv_cm(N_s, L2M, uC, AC);
  gemv_cm(N_s, L2M, uR, AR);
  for (int s = 0; s < slicenum; ++s)
    limit_mono(N_s1D - 1, AL + s * N_s1D, AC + s * N_s1D, AR + s * N_s1D, Al + s * N_s1D);
  gemv_cm(N_s, M2L, Al, uC);
  if (monolim) for (int i = 0; i < N_s; ++i) monolim[i] = Al[i];
}

// hri1D (limiting_kernels.cu:322-429), one thread per (flagged element, field)
__global__ void hri1d(int N_s, int N_E, int N_N, const int* neighbors, int N_s1D, int slicenum, int offxy,
                      const scalar* L2M, const scalar* M2L, const int* sensors, const scalar* U, scalar* Unew) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= (long)N_E * N_F) return;
  const long e = k / N_F;
  const int fc = (int)(k % N_F);
  if (sensors[e] == 0) return;
  const int left = neighbors[e * N_N + offxy], right = neighbors[e * N_N + offxy + 1];
  int physical = 0;
  if (left < 0) physical = -left;
  if (right < 0) physical = -right;
  double uC[kMaxNs];
  for (int i = 0; i < N_s; ++i) uC[i] = U[(e * N_F + fc) * N_s + i];
  if (physical == 2) {
    set2average_v(N_s, N_s1D, slicenum, L2M, M2L, uC, nullptr);
  } else if (physical == 3) {
    const int un = offxy == 0 ? 1 : (offxy == 2 ? 2 : 0);
    if (fc != un) set2average_v(N_s, N_s1D, slicenum, L2M, M2L, uC, nullptr);
  } else if (physical != 4) {
    double uL[kMaxNs], uR[kMaxNs];
    for (int i = 0; i < N_s; ++i) { uL[i] = U[((long)left * N_F + fc) * N_s + i]; uR[i] = U[((long)right * N_F + fc) * N_s + i]; }
    hr_v(N_s, N_s1D, slicenum, L2M, M2L, uL, uC, uR, nullptr);
  }
  for (int i = 0; i < N_s; ++i) Unew[(e * N_F + fc) * N_s + i] = uC[i];
}

// m2i1D (limiting_kernels.cu:431-722), gamma model, one thread per flagged element
__global__ void m2i1d(int N_s, int N_E, int N_N, const int* neighbors, int N_s1D, int slicenum, int offxy,
                      const scalar* L2M, const scalar* M2L, const int* sensors, const scalar* U, scalar* Unew) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= N_E || sensors[e] == 0) return;
  constexpr int IE = D + 1, IG = D + 2;
  const int left = neighbors[e * N_N + offxy], right = neighbors[e * N_N + offxy + 1];
  int physical = 0;
  if (left < 0) physical = -left;
  if (right < 0) physical = -right;
  double c[N_F][kMaxNs];
  for (int fc = 0; fc < N_F; ++fc)
    for (int i = 0; i < N_s; ++i) c[fc][i] = U[(e * N_F + fc) * N_s + i];
  auto press = [&](double (*v)[kMaxNs], double* p) {
    for (int i = 0; i < N_s; ++i) {
      const double kin = v[1][i] * v[1][i] + (D == 2 ? v[2][i] * v[2][i] : 0.0);
      p[i] = (v[IE][i] - 0.5 * kin / v[0][i]) / v[IG][i];
    }
  };
  double pC[kMaxNs], gLim[kMaxNs], pLim[kMaxNs];
  press(c, pC);
  if (physical != 4) {
    if (physical == 2 || physical == 3) {
      set2average_v(N_s, N_s1D, slicenum, L2M, M2L, c[0], nullptr);
      if (physical == 2) {
        for (int f = 1; f <= D; ++f) set2average_v(N_s, N_s1D, slicenum, L2M, M2L, c[f], nullptr);
      } else if (D == 2) {  // the wall-normal momentum is not limited
        set2average_v(N_s, N_s1D, slicenum, L2M, M2L, c[offxy == 0 ? 2 : 1], nullptr);
      }
      set2average_v(N_s, N_s1D, slicenum, L2M, M2L, c[IG], gLim);
      set2average_v(N_s, N_s1D, slicenum, L2M, M2L, pC, pLim);
    } else {
      double l[N_F][kMaxNs], r[N_F][kMaxNs], pL[kMaxNs], pR[kMaxNs];
      for (int fc = 0; fc < N_F; ++fc)
        for (int i = 0; i < N_s; ++i) {
          l[fc][i] = U[((long)left * N_F + fc) * N_s + i];
          r[fc][i] = U[((long)right * N_F + fc) * N_s + i];
        }
      press(l, pL);
      press(r, pR);
      for (int f = 0; f <= D; ++f) hr_v(N_s, N_s1D, slicenum, L2M, M2L, l[f], c[f], r[f], nullptr);
      hr_v(N_s, N_s1D, slicenum, L2M, M2L, l[IG], c[IG], r[IG], gLim);
      hr_v(N_s, N_s1D, slicenum, L2M, M2L, pL, pC, pR, pLim);
    }
    // kinetic (limited rho, momenta), internal (limited p, alpha) and total energy
    double tmp[kMaxNs], KL[kMaxNs], rhoe[kMaxNs], EM[kMaxNs], EL[kMaxNs];
    for (int i = 0; i < N_s; ++i) tmp[i] = 0.5 * (c[1][i] * c[1][i] + (D == 2 ? c[2][i] * c[2][i] : 0.0)) / c[0][i];
    gemv_cm(N_s, L2M, tmp, KL);
    for (int s = 0; s < slicenum; ++s)
      for (int i = 0; i < N_s1D; ++i) {
        double I = 0.0, bc = 1.0;
        for (int kk = 0; kk <= i; ++kk) {
          I += bc * pLim[s * N_s1D + i - kk] * gLim[s * N_s1D + kk];
          bc = bc * (i - kk) / (kk + 1);
        }
        rhoe[s * N_s1D + i] = I;
      }
    gemv_cm(N_s, L2M, c[IE], EM);
    for (int s = 0; s < slicenum; ++s) {
      const int b = s * N_s1D;
      for (int i = 1; i < N_s1D; ++i) EL[b + i] = rhoe[b + i] + KL[b + i];
      double E0 = EM[b];
      for (int m = 2; m < N_s1D; m += 2) E0 -= ifactorial(m + 1) * (EL[b + m] - EM[b + m]);
      EL[b] = E0;
    }
    gemv_cm(N_s, M2L, EL, c[IE]);
  }
  for (int fc = 0; fc < N_F; ++fc)
    for (int i = 0; i < N_s; ++i) Unew[(e * N_F + fc) * N_s + i] = c[fc][i];
}

__global__ void p0i(int N_s, int N_E, int N_G, scalar refArea, const int* sensors, const scalar* phi_w,
                    const scalar* U, scalar* Unew) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // (e, fc)
  if (k >= (long)N_E * N_F || sensors[k / N_F] == 0) return;
  scalar avg = 0.0;
  for (int g = 0; g < N_G; ++g)
    for (int i = 0; i < N_s; ++i) avg += phi_w[i * N_G + g] * U[k * N_s + i];
  avg = avg / refArea;
  for (int i = 0; i < N_s; ++i) Unew[k * N_s + i] = avg;
}

__global__ void change_basis(int size1, int size2, int N_E, const scalar* T, const scalar* U, scalar* Unew) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // ((e*N_F + fc)*size1 + i)
  if (k >= (long)N_E * N_F * size1) return;
  const int i = (int)(k % size1);
  const long ef = k / size1, e = ef / N_F;
  scalar sol = 0.0;
  for (int ii = 0; ii < size2; ++ii) sol += T[(e * size1 + i) * size2 + ii] * U[ef * size2 + ii];
  Unew[k] = sol;
}

__global__ void prim_cons(int N_s, int N_E, scalar* U, bool to_prim) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // (e, i)
  if (k >= (long)N_E * N_s) return;
  const long e = k / N_s;
  const int i = (int)(k % N_s);
  auto at = [&](int fc) -> scalar& { return U[(e * N_F + fc) * N_s + i]; };
  const scalar rho = at(0), a1 = at(1), a2 = D == 2 ? at(2) : 0.0, a3 = at(D + 1), al = at(D + 2);
  if (to_prim) {
    at(1) = a1 / rho;
    if (D == 2) at(2) = a2 / rho;
    at(D + 1) = (a3 - 0.0 - 0.5 * (a1 * a1 + a2 * a2) / rho) / al;
  } else {
    at(1) = rho * a1;
    if (D == 2) at(2) = rho * a2;
    at(D + 1) = a3 * al + 0.0 + 0.5 * rho * (a1 * a1 + a2 * a2);
  }
}

__global__ void copy_detected(int N_s, int N_E, const int* sensors, const scalar* Uold, scalar* U) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= (long)N_E * N_F * N_s || sensors[k / ((long)N_F * N_s)] == 0) return;
  U[k] = Uold[k];
}

__global__ void transpose_to(int rows, int cols, const int* in, int* out) {  // out[c*rows + r] = in[r*cols + c]
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k < (long)rows * cols) out[(k % cols) * rows + k / cols] = in[k];
}
__global__ void transpose_to_d(int rows, int cols, const scalar* in, scalar* out) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k < (long)rows * cols) out[(k % cols) * rows + k / cols] = in[k];
}

__global__ void formater(int N_s, int N_E, scalar* U, scalar* out, bool inverse) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;  // (e, i)
  if (k >= (long)N_E * N_s) return;
  const long e = k / N_s;
  const int i = (int)(k % N_s);
  auto u = [&](int fc) -> scalar& { return U[(e * N_F + fc) * N_s + i]; };
  auto o = [&](int fc) -> scalar& { return out[(e * N_F + fc) * N_s + i]; };
  if (!inverse) {
    const scalar rho = u(0), ux = u(1) / rho, uy = D == 2 ? u(2) / rho : 0.0, et = u(D + 1);
    const scalar gamma = 1 + 1.0 / u(D + 2);
    o(0) = rho;
    o(1) = ux;
    if (D == 2) o(2) = uy;
    o(D + 1) = gamma;
    o(D + 2) = (gamma - 1) * (et - 0.5 * (ux * ux + uy * uy) * rho);
  } else {
    const scalar rho = o(0), ux = o(1), uy = D == 2 ? o(2) : 0.0, gamma = o(D + 1), p = o(D + 2);
    u(0) = rho;
    u(1) = rho * ux;
    if (D == 2) u(2) = rho * uy;
    u(D + 1) = p / (gamma - 1) + 0.5 * rho * (ux * ux + uy * uy);
    u(D + 2) = 1.0 / (gamma - 1);
  }
}

__global__ void format_sensor(int N_s, int N_E, const int* sensor, scalar* out) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k < (long)N_E * N_s) out[k] = sensor[k / N_s];
}

// sensor work arrays, grown on demand (the reference's sensor launcher allocates nothing; here the
// exact-order evaluation needs O(N_E) scratch)
struct SensorScratch {
  int cap = 0, nnbr = 0;
  int* ints = nullptr;
  double* mean = nullptr;
} g_sens;

}  // namespace

extern "C" void Lstridedcopy(int count, int blocklen, int strideA, int strideB, int offsetA, int offsetB, scalar* A,
                             scalar* B) {
  strided_copy<<<blocks((long)count * blocklen), kBlock>>>(count, blocklen, strideA, strideB, offsetA, offsetB, A, B);
  check("Lstridedcopy");
}
extern "C" void Lreconstruct_energy(int N_s, int N_E, int slicenum, scalar* rhoeLim, scalar* KLim, scalar* EMono,
                                    scalar* ELim) {
  reconstruct_energy<<<blocks((long)N_E * slicenum), kBlock>>>(N_s, N_E, slicenum, rhoeLim, KLim, EMono, ELim);
  check("Lreconstruct_energy");
}
extern "C" void Linternal_energy_multifluid(int N_s, int N_E, int slicenum, scalar* p, scalar* g, scalar* rhoe) {
  internal_energy<<<blocks((long)N_E * slicenum * N_s), kBlock>>>(N_s, N_E, slicenum, p, g, rhoe);
  check("Linternal_energy_multifluid");
}
extern "C" void Lhrl1D(int N_s, int N_E, int Nfields, int N_N, int slicenum, int* neighbors, int offxy, scalar* A,
                       scalar* Alim) {
  hrl1d<<<blocks((long)N_E * Nfields * slicenum), kBlock>>>(N_s, N_E, Nfields, N_N, slicenum, neighbors, offxy, A, Alim);
  check("Lhrl1D");
}
extern "C" void Lhri1D(int N_s, int N_E, int N_N, int* neighbors, int N_s1D, int slicenum, int offxy, scalar* Lag2Mono,
                       scalar* Mono2Lag, int* sensors, scalar* U, scalar* Unew) {
  hri1d<<<blocks((long)N_E * N_F), kBlock>>>(N_s, N_E, N_N, neighbors, N_s1D, slicenum, offxy, Lag2Mono, Mono2Lag,
                                             sensors, U, Unew);
  check("Lhri1D");
}
extern "C" void Lm2i1D(int N_s, int N_E, int N_N, int* neighbors, int N_s1D, int slicenum, int offxy, scalar* Lag2Mono,
                       scalar* Mono2Lag, int* sensors, scalar* U, scalar* Unew) {
  m2i1d<<<blocks(N_E), 128>>>(N_s, N_E, N_N, neighbors, N_s1D, slicenum, offxy, Lag2Mono, Mono2Lag, sensors, U, Unew);
  check("Lm2i1D");
}
extern "C" void Lp0i(int N_s, int N_E, int N_G, scalar refArea, int* sensors, scalar* phi_w, scalar* U, scalar* Unew) {
  p0i<<<blocks((long)N_E * N_F), kBlock>>>(N_s, N_E, N_G, refArea, sensors, phi_w, U, Unew);
  check("Lp0i");
}
extern "C" void LChangeBasis(int size1, int size2, int N_E, scalar* Transform, scalar* U, scalar* Unew) {
  change_basis<<<blocks((long)N_E * N_F * size1), kBlock>>>(size1, size2, N_E, Transform, U, Unew);
  check("LChangeBasis");
}
extern "C" void LPrim2Cons(int N_s, int N_E, scalar* U) {
  prim_cons<<<blocks((long)N_E * N_s), kBlock>>>(N_s, N_E, U, false);
  check("LPrim2Cons");
}
extern "C" void LCons2Prim(int N_s, int N_E, scalar* U) {
  prim_cons<<<blocks((long)N_E * N_s), kBlock>>>(N_s, N_E, U, true);
  check("LCons2Prim");
}
extern "C" void Lcopy_detected(int N_s, int N_E, int* sensors, scalar* Uold, scalar* U) {
  copy_detected<<<blocks((long)N_E * N_F * N_s), kBlock>>>(N_s, N_E, sensors, Uold, U);
  check("Lcopy_detected");
}
extern "C" void Lcalc_sensors(int N_E, int N_N, bool sensor1, scalar thresh1, bool sensor2, scalar thresh2,
                              bool sensor3, scalar thresh3, int* neighbors, scalar* Uavg, int* sensors) {
  if (N_E <= 0) return;
  if (g_sens.cap < N_E || g_sens.nnbr < N_N) {
    cudaFree(g_sens.ints);
    cudaFree(g_sens.mean);
    g_sens.cap = N_E;
    g_sens.nnbr = N_N;
    if (cudaMalloc(&g_sens.ints, ((size_t)(5 + N_N) * N_E + 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&g_sens.mean, (size_t)N_F * N_E * sizeof(double)) != cudaSuccess) {
      std::fprintf(stderr, "dgb shim Lcalc_sensors: out of device memory\n");
      g_sens.cap = 0;
      return;
    }
  }
  int* nbrT = g_sens.ints + (size_t)5 * N_E;  // neighbours and means in the element-fastest layout
  transpose_to<<<blocks((long)N_E * N_N), kBlock>>>(N_E, N_N, neighbors, nbrT);
  transpose_to_d<<<blocks((long)N_E * N_F), kBlock>>>(N_E, N_F, Uavg, g_sens.mean);
  dgb::SensorLaunch s{};
  s.D = D; s.ns = 1; s.nf = N_F; s.n_elem = N_E; s.ld = N_E; s.n_nbr = N_N;
  s.U = nullptr; s.iperm = nullptr; s.nbr = nbrT; s.mean = g_sens.mean;
  s.on[0] = sensor1; s.on[1] = sensor2; s.on[2] = sensor3;
  s.th[0] = thresh1; s.th[1] = thresh2; s.th[2] = thresh3;
  s.target = g_sens.ints; s.type = g_sens.ints + N_E; s.processed = g_sens.ints + 2 * (size_t)N_E;
  s.mask = g_sens.ints + 3 * (size_t)N_E; s.list = g_sens.ints + 4 * (size_t)N_E;
  s.count = g_sens.ints + (size_t)(5 + N_N) * N_E;
  s.sens = sensors;
  const int rc = dgb::launch_sensors_from_means(s, 0);
  if (rc) std::fprintf(stderr, "dgb shim Lcalc_sensors: %s\n", cudaGetErrorString((cudaError_t)rc));
}
extern "C" void Lformater(int N_s, int N_E, scalar* U, scalar* output, bool inverse) {
  formater<<<blocks((long)N_E * N_s), kBlock>>>(N_s, N_E, U, output, inverse);
  check("Lformater");
}
extern "C" void Lformat_sensor(int N_s, int N_E, int* sensor, scalar* output) {
  format_sensor<<<blocks((long)N_E * N_s), kBlock>>>(N_s, N_E, sensor, output);
  check("Lformat_sensor");
}
