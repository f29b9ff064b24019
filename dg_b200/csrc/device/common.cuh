// Device-side data description shared by all kernels.
//
// Internal state layout ("field-node-major SoA"): U[(f*N_s + t)*ld + e], with
//   f  field, t = ix + (p+1)*iy the tensor-product node index (nodes ascending in x, then y),
//   e  element (mesh order), ld = element count rounded up to a multiple of 64.
// Each (field, node) row is a contiguous run over elements, so a warp touching 32 consecutive
// elements reads 256 contiguous bytes; neighbour traces of a row-major mesh are the same runs
// shifted by +-1 or +-nx.  The reference layout U[(e*N_F+f)*N_s+i] is converted at the API
// boundary only.
#pragma once
#include <cstdint>

namespace dgb {

constexpr int MAXN = 4;    // nodes per direction (p <= 3)
constexpr int MAXG = 5;    // volume quadrature points per direction (p + 2)
constexpr int MAXNS = 16;  // nodes per element

// Small per-problem constants (copied into shared memory by the kernels that index them).
struct Consts {
  int p, n1, ng1, ns, ng, nf, dim;
  int ld, n_elem;
  int pad_;
  // volume quadrature (1D factors): Bq[g][i] = l_i(xq_g), Dq[g][i] = l_i'(xq_g), weights wq
  double Bq[MAXG][MAXN], Dq[MAXG][MAXN], wq[MAXG];
  // face quadrature (p+1 Gauss points): Bf[g][i] = l_i(xf_g), weights wf
  double Bf[MAXN][MAXN], wf[MAXN];
  // element inverse mass matrix in tensor order (Minv[t][t'])
  double Minv[MAXNS][MAXNS];
  // 1D Lagrange -> scaled Taylor monomial transform in tensor (ascending) node order and inverse
  double T[MAXN][MAXN], Tinv[MAXN][MAXN];
  // limiter integrals (limiting_kernels.cu:1748-1775): imd[k][n] = int_{-1}^{1} d^k/dx^k x^n/n!,
  // imdL[k][n] over [-3,-1], imdR[k][n] over [1,3]; ifact[k] = 1/k!
  double imd[MAXN][MAXN], imdL[MAXN][MAXN], imdR[MAXN][MAXN], ifact[8];
  // metric of the uniform Cartesian element: J = hx*hy/4 (1D: hx/2), invJac = diag(2/hx, 2/hy)
  double J, ixx, iyy;
  // face Jacobians: x-faces (constant x) and y-faces
  double JFx, JFy;
  double cfl_scaled;
};

// Device scalars of one context (time step, accumulated time, reduction slot, flags).
struct DevScalars {
  double dt;                   // current step
  double time;                 // accumulated time
  unsigned long long umax;     // max wave speed as ordered bits (non-negative doubles)
  unsigned int flags;          // bit 0: NaN wave speed / dt, bit 1: dt < 1e-14
  unsigned int blocks_done;    // CTAs of a wave-speed reduction that have added their maximum
  double dt_fixed;             // fixed step (> 0) or 0 for the CFL step
};

enum { FLAG_NONFINITE = 1u, FLAG_DT_SMALL = 2u };

// Programmatic dependent launch (a kernel launched with programmatic stream serialization may be
// scheduled before its predecessor in the stream has finished): pdl_wait blocks until the
// predecessor grid has completed and its memory is visible (at once when the launch was not
// programmatic), so it comes before a kernel's first access to global data; pdl_trigger lets the
// next kernel's CTAs be scheduled as this one's finish.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ int signum_d(double v) { return v > 0 ? 1 : (v < 0 ? -1 : 0); }

// minmod of two arguments (limiting_kernels.cu:1470-1486)
__device__ __forceinline__ double minmod2(double a, double b) {
  const int sa = signum_d(a);
  if (sa != signum_d(b)) return 0.0;
  const double fa = fabs(a), fb = fabs(b);
  return fa < fb ? sa * fa : sa * fb;
}

// 1D tables of the limiter for order P (reference element, identical for every problem):
//   T, Tinv   Lagrange (ascending nodes) <-> scaled Taylor monomial x^n/n! transforms
//   imd[k][n] = int_{-1}^{1} d^k/dx^k x^n/n! dx, imdL over [-3,-1], imdR over [1,3]
//             (integrate_monomial_derivative(_bounds), limiting_kernels.cu:1748-1775)
//   ifact[k]  = 1/k!
template <int P>
struct LimTab {
  double T[P + 1][P + 1], Tinv[P + 1][P + 1];
  double imd[P + 1][P + 1], imdL[P + 1][P + 1], imdR[P + 1][P + 1];
  double ifact[P + 3];
};
// one copy per translation unit (each .cu file is its own device module)
static __constant__ LimTab<1> c_lim_p1;
static __constant__ LimTab<2> c_lim_p2;
static __constant__ LimTab<3> c_lim_p3;
// by-name access (a reference to a __constant__ object can be materialised as a local copy)
#define DGB_LIM(P, member) ((P) == 1 ? c_lim_p1.member : (P) == 2 ? c_lim_p2.member : c_lim_p3.member)

// Hierarchical-reconstruction limiting of one 1D slice of scaled Taylor coefficients
// (limit_monomial, limiting_kernels.cu:1534-1583).  N = polynomial order.
template <int N>
__device__ __forceinline__ void limit_monomial(const double* AL, const double* AC, const double* AR, double* Alim) {
  double avgLC = 0.0;
#pragma unroll
  for (int m = N; m > 0; --m) {
    double dUL = 0, dUC = 0, dUR = 0, RL = 0, RC = 0, RR = 0;
#pragma unroll
    for (int n = m - 1; n <= N; ++n) {
      const double integral = DGB_LIM(N, imd[m - 1][n]);
      dUL += AL[n] * integral;
      dUC += AC[n] * integral;
      dUR += AR[n] * integral;
      if (n >= m + 1) {
        const double al = Alim[n];
        RL += al * DGB_LIM(N, imdL[m - 1][n]);
        RC += al * integral;
        RR += al * DGB_LIM(N, imdR[m - 1][n]);
      }
    }
    const double avgLL = 0.5 * (dUL - RL);
    avgLC = 0.5 * (dUC - RC);
    const double avgLR = 0.5 * (dUR - RR);
    const double c1 = 0.5 * (avgLC - avgLL);
    const double c2 = 0.5 * (avgLR - avgLC);
    Alim[m] = minmod2(c1, c2);
  }
  Alim[0] = avgLC;
}

// average_monomial (limiting_kernels.cu:1777-1790): keep the cell average, zero the slopes
template <int N>
__device__ __forceinline__ void average_monomial(const double* A, double* Alim) {
  double avg = 0;
#pragma unroll
  for (int n = 0; n <= N; ++n) { avg += A[n] * DGB_LIM(N, imd[0][n]); Alim[n] = 0; }
  Alim[0] = 0.5 * avg;
}

template <int P>
__device__ __forceinline__ double lim_T(int m, int i) { return DGB_LIM(P, T[m][i]); }
template <int P>
__device__ __forceinline__ double lim_Tinv(int i, int m) { return DGB_LIM(P, Tinv[i][m]); }

}  // namespace dgb
