// Tiled 2D residual + stage update for structured (row-major nx x ny) Cartesian meshes.
//
// One CTA owns a TW x TH tile of elements, one thread per element.
//   phase 0  the tile's nodal state and the four neighbour face-trace strips -> shared memory
//            (coalesced: a warp reads 32 consecutive elements of one (field, node) row)
//   phase 1  every face of the tile exactly once: (TW+1)*TH x-faces and TW*(TH+1) y-faces,
//            spread evenly over the threads (work item = face quadrature point); Riemann flux in
//            the canonical orientation (left/bottom state first, +x/+y normal)
//   phase 2  per element (thread): state from shared memory into registers, volume terms at the
//            (p+2)^2 quadrature points with the reference-element tables read as warp-uniform
//            __constant__ operands, face contributions from phase 1, tensor-factored inverse mass
//            M^-1 = (1/J) M1^-1 (x) M1^-1, stage update, coalesced stores.
// Equivalent to DG_SOLVER::dg_solver (code/src/dg/dg_solver.h:292-364) + Lsolver + the RK
// register update, up to FP64 rounding.
#pragma once
#include "common.cuh"
#include "physics.cuh"
#include "tma.cuh"

namespace dgb {

// Reference-element tables of the tiled kernel (tensor node order t = ix + (p+1)*iy,
// quadrature point g = gx*(p+2) + gy).
template <int P>
struct Tab2 {
  static constexpr int N1 = P + 1, NG1 = (P == 1) ? 2 : P + 2, NS = N1 * N1, NG = NG1 * NG1;
  double Phi[NG][NS];   // l_ix(x_gx) l_iy(x_gy)
  double dPx[NG][NS];   // l_ix'(x_gx) l_iy(x_gy)
  double dPy[NG][NS];   // l_ix(x_gx) l_iy'(x_gy)
  double W[NG];         // w_gx w_gy
  double Bf[N1][N1];    // l_j(xf_g) on the p+1 face Gauss points
  double wf[N1];
  double M1i[N1][N1];   // inverse of the 1D reference mass matrix (exact with p+2 Gauss points)
  double B1[NG1][N1];   // l_i(x_g) on the p+2 volume Gauss points (1D factor)
  double D1[NG1][N1];   // l_i'(x_g)
  double W1[NG1];       // 1D volume weights
};

static __constant__ Tab2<1> c_tab2_p1;
static __constant__ Tab2<2> c_tab2_p2;
static __constant__ Tab2<3> c_tab2_p3;

// by-name access to the table of order P (a reference to a __constant__ object could be
// materialised as a local-memory copy)
#define DGB_TAB2(P, member) ((P) == 1 ? c_tab2_p1.member : (P) == 2 ? c_tab2_p2.member : c_tab2_p3.member)

struct TileArgs {
  const double* __restrict__ U;
  const double* __restrict__ Ubase;
  double* __restrict__ out;
  double* __restrict__ Uacc;
  const int* __restrict__ nbr;
  const DevScalars* __restrict__ scal;
  unsigned int* errflag;  // receives FLAG_TIMEOUT when a bounded wait runs out
  long long polls = kDefaultPolls;  // budget of the first wait on each tile copy (then drained)
  double a, b, dt_override;
  double invJ;           // 1 / J
  double cx, cy;         // J * 2/hx, J * 2/hy  (volume flux metric)
  double sx, sy;         // 2/hx, 2/hy          (gradient metric of the alpha source)
  double J;
  double JFx, JFy;       // face Jacobians of x-faces and y-faces
  int nx, ny, ld;
};

template <int P, int TW, int TH, int NY = 0>
struct TileDims {
  static constexpr int N1 = P + 1, NS = N1 * N1, NF = 5 + NY, NT = TW * TH;
  static constexpr int NXF = (TW + 1) * TH * N1;  // x-face points
  static constexpr int NYF = TW * (TH + 1) * N1;  // y-face points
  static constexpr int NCODE = 2 * TH + 2 * TW;   // boundary codes / neighbours of the tile edges
  static constexpr size_t head_bytes = 128;        // mbarrier + ok flag
  static constexpr size_t code_bytes = (NCODE * 4 + 127) / 128 * 128;
  static constexpr size_t tile_doubles = (size_t)NF * NS * NT;
  static constexpr uint32_t tile_bytes = (uint32_t)(tile_doubles * 8);
  static constexpr size_t halo_doubles = (size_t)2 * TH * NF * N1 + (size_t)2 * TW * NF * N1;
  // p = 3, or more than three mass fractions: the x-faces and then the y-faces pass through one
  // face buffer, and the stage base is read from global memory in the epilogue instead of being
  // prefetched into it (p = 3: 70 instead of 93 KB per 64-thread CTA, three CTAs per SM instead of
  // two; ten mass fractions at p = 2: 131 KB, within one CTA's limit)
  static constexpr bool split_faces = P == 3 || NY > 3;
  static constexpr int NFREC = split_faces ? (NXF > NYF ? NXF : NYF) : NXF + NYF;  // face records held
  static constexpr size_t face_doubles = (size_t)(NF + 1) * NFREC;  // NF fluxes + ncterm per point
  // otherwise the face buffer is reused for the prefetched stage base, so it is at least one tile
  static constexpr size_t fbuf_doubles =
      split_faces || face_doubles > tile_doubles ? face_doubles : tile_doubles;
  // byte offsets; every region a TMA copy lands in starts on a 128-byte boundary
  static constexpr size_t off_tile = head_bytes + code_bytes;
  static constexpr size_t off_halo = off_tile + (tile_doubles * 8 + 127) / 128 * 128;
  static constexpr size_t off_face = off_halo + (halo_doubles * 8 + 127) / 128 * 128;
  static constexpr size_t smem_bytes = off_face + fbuf_doubles * 8;
  static_assert(off_tile % 128 == 0 && off_face % 128 == 0, "TMA destinations must be 128-byte aligned");
};

enum { FLAG_TIMEOUT = 4u };

// Unrolling of the outer quadrature-column loop of the volume terms.  Fully unrolled, the
// straight-line kernel body outgrows the instruction cache once several warps per scheduler run
// different parts of it; rolled, the column index is warp-uniform and the tables stay
// constant-bank operands.  Measured at p = 2 (512 x 256): rolled 85.4 us, unrolled by 2 84.1 us
// per launch; the other orders keep the loop rolled.
#ifndef DGB_VOL_UNROLL
#define DGB_VOL_UNROLL 0
#endif
template <int P>
constexpr int vol_unroll() { return DGB_VOL_UNROLL > 0 ? DGB_VOL_UNROLL : (P == 2 ? 2 : 1); }
// Lift of the volume terms: sum-factorised (1) -- per quadrature column, contract over the
// points of the column first, then one rank-1 update per node -- or direct (0) with the
// tensor-product tables dPx, dPy, Phi.
#ifndef DGB_SF_LIFT
#define DGB_SF_LIFT 1
#endif
constexpr bool kSfLift = DGB_SF_LIFT != 0;

// Face fluxes of a tile, each face once: (TW+1)*TH x-faces and TW*(TH+1) y-faces, one work item
// per face quadrature point spread over `nthr` threads, Riemann flux in the canonical orientation
// (left/bottom state first, +x/+y normal).  Record k of Fs holds the NF fluxes and the ncterm;
// boundary faces seen from the right/top element store -F so that every consumer forms (+F + nc)
// on its left/bottom face and (-F + nc) on its right/top face.
// Work items k0 <= k < k1 (x-faces first, then y-faces); item k goes to record k - rec0.
template <int P, int FLUX, int TW, int TH, int NY, bool GC>
__device__ __forceinline__ void tile_face_fluxes(const double* Us, const double* HL, const double* HR,
                                                 const double* HD, const double* HU, const int* codes, double* Fs,
                                                 int tid, int nthr, int k0, int k1, int rec0) {
  using Dm = TileDims<P, TW, TH, NY>;
  constexpr int N1 = Dm::N1, NS = Dm::NS, NF = Dm::NF, NT = Dm::NT, NXF = Dm::NXF;
  constexpr int FS = NF + 1;
  for (int k = k0 + tid; k < k1; k += nthr) {
    double L[NF], R[NF];
    double nxv, nyv, sgn = 1.0;
    double vl[NF][N1], vr[NF][N1];
    int code = 0;
    bool first_edge;
    int mom;
    int g;
    if (k < NXF) {
      // x-face fx (0..TW) of row fy; left element (fx-1, fy), right element (fx, fy)
      g = k % N1;
      const int fy = (k / N1) % TH, fx = k / (N1 * TH);
      if (fx == 0) code = codes[fy];
      if (fx == TW) code = codes[TH + fy];
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int j = 0; j < N1; ++j) {
          vl[f][j] = fx > 0 ? Us[(f * NS + P + N1 * j) * NT + fy * TW + fx - 1] : HL[(fy * NF + f) * N1 + j];
          vr[f][j] = fx < TW ? Us[(f * NS + N1 * j) * NT + fy * TW + fx] : HR[(fy * NF + f) * N1 + j];
        }
      nxv = 1.0;
      nyv = 0.0;
      first_edge = fx == 0;
      mom = 1;
    } else {
      const int kk = k - NXF;
      g = kk % N1;
      const int fx = (kk / N1) % TW, fy = kk / (N1 * TW);
      if (fy == 0) code = codes[2 * TH + fx];
      if (fy == TH) code = codes[2 * TH + TW + fx];
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int j = 0; j < N1; ++j) {
          vl[f][j] = fy > 0 ? Us[(f * NS + j + N1 * P) * NT + (fy - 1) * TW + fx] : HD[(fx * NF + f) * N1 + j];
          vr[f][j] = fy < TH ? Us[(f * NS + j) * NT + fy * TW + fx] : HU[(fx * NF + f) * N1 + j];
        }
      nxv = 0.0;
      nyv = 1.0;
      first_edge = fy == 0;
      mom = 2;
    }
    if (code < 0) {
      // domain boundary: the inside element is L with its outward normal, the mirror state is R
      // (reflective walls mirror the wall-normal momentum, code/src/bc/boundaries.cu:20-67)
#pragma unroll
      for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int j = 0; j < N1; ++j) {
          const double own = first_edge ? vr[f][j] : vl[f][j];
          vl[f][j] = own;
          vr[f][j] = (code == -3 && f == mom) ? -own : own;
        }
      if (first_edge) { nxv = -nxv; nyv = -nyv; sgn = -1.0; }
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      double sl = 0, sr = 0;
#pragma unroll
      for (int j = 0; j < N1; ++j) { sl += DGB_TAB2(P, Bf[g][j]) * vl[f][j]; sr += DGB_TAB2(P, Bf[g][j]) * vr[f][j]; }
      L[f] = sl;
      R[f] = sr;
    }
    double F[NF], nc;
    phys::riemann2d_rcp<FLUX, NY, GC>(L, R, nxv, nyv, F, nc);
    // boundary faces seen from the right/top element store -F so that every consumer forms
    // (+F + nc) on its left/bottom face and (-F + nc) on its right/top face
#pragma unroll
    for (int f = 0; f < NF; ++f) Fs[(k - rec0) * FS + f] = sgn * F[f];
    Fs[(k - rec0) * FS + NF] = nc;
  }
}

// Phase 0 of a tile (origin tx0, ty0): boundary codes of the tile edges, the tile's nodal state
// (TMA copy, or plain coalesced loads when TMA = false) and the four neighbour face-node strips into
// shared memory, by `nthr` threads.  Returns whether the tile copy arrived (CTA-uniform); a copy that
// could not start or whose bounded wait ran out sets FLAG_TIMEOUT.  `phase` counts the mbarrier's
// completed phases.
template <int P, int TW, int TH, int NY, bool TMA>
__device__ __forceinline__ bool tile_stage_in(const TileArgs& a, const CUtensorMap* mapU, int tx0, int ty0,
                                              unsigned char* smraw, uint32_t& phase, int tid, int nthr) {
  using Dm = TileDims<P, TW, TH, NY>;
  constexpr int N1 = Dm::N1, NS = Dm::NS, NF = Dm::NF, NT = Dm::NT;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smraw);
  int* s_ok = reinterpret_cast<int*>(smraw + 8);
  int* codes = reinterpret_cast<int*>(smraw + Dm::head_bytes);  // [L: TH][R: TH][D: TW][U: TW]
  double* Us = reinterpret_cast<double*>(smraw + Dm::off_tile);  // [NF*NS][NT]
  double* HL = reinterpret_cast<double*>(smraw + Dm::off_halo);  // [TH][NF][N1] left neighbours' right-face nodes
  double* HR = HL + TH * NF * N1;          // [TH][NF][N1]
  double* HD = HR + TH * NF * N1;          // [TW][NF][N1]  bottom neighbours' top-face nodes
  double* HU = HD + TW * NF * N1;          // [TW][NF][N1]
  double* Fs = reinterpret_cast<double*>(smraw + Dm::off_face);
  const int ld = a.ld, nx = a.nx;
  for (int k = tid; k < Dm::NCODE; k += nthr) {
    int face, eo;
    if (k < TH) { face = 0; eo = (ty0 + k) * nx + tx0; }
    else if (k < 2 * TH) { face = 1; eo = (ty0 + k - TH) * nx + tx0 + TW - 1; }
    else if (k < 2 * TH + TW) { face = 2; eo = ty0 * nx + tx0 + (k - 2 * TH); }
    else { face = 3; eo = (ty0 + TH - 1) * nx + tx0 + (k - 2 * TH - TW); }
    codes[k] = __ldg(a.nbr + (size_t)face * ld + eo);
  }
  __syncthreads();
  // a TMA copy must land on a 128-byte shared boundary and start on a 16-byte global column;
  // otherwise record the fault and skip the copy (the wait below then reports it)
  const bool tma_ok = TMA && (smem_u32(Us) & 127u) == 0 && (smem_u32(Fs) & 127u) == 0 && ((tx0 * 8) & 15) == 0;
  if constexpr (!TMA) {
    for (int k = tid; k < NF * NS * NT; k += nthr) {  // [plane][row][column], as the tensor map lands it
      const int q = k / NT, el = k % NT;
      Us[k] = __ldg(a.U + (size_t)q * ld + (size_t)(ty0 + el / TW) * nx + tx0 + el % TW);
    }
  }
  if (TMA && tid == 0) {
    if (tma_ok) {
      mbar_arrive_expect_tx(bar, Dm::tile_bytes);
      tma_load_3d(Us, mapU, tx0, ty0, 0, bar);
    } else {
      atomicOr(a.errflag, (unsigned)FLAG_TIMEOUT);
    }
  }
  for (int k = tid; k < 2 * TH * NF * N1; k += nthr) {
    const int side = k / (TH * NF * N1);
    const int r = k % (TH * NF * N1);
    const int ty = r / (NF * N1), f = (r / N1) % NF, j = r % N1;
    const int nb = codes[side * TH + ty];
    double v = 0.0;
    if (nb >= 0) v = __ldg(a.U + (size_t)(f * NS + (side == 0 ? P + N1 * j : N1 * j)) * ld + nb);
    (side == 0 ? HL : HR)[r] = v;
  }
  for (int k = tid; k < 2 * TW * NF * N1; k += nthr) {
    const int side = k / (TW * NF * N1);
    const int r = k % (TW * NF * N1);
    const int tx = r / (NF * N1), f = (r / N1) % NF, j = r % N1;
    const int nb = codes[2 * TH + side * TW + tx];
    double v = 0.0;
    if (nb >= 0) v = __ldg(a.U + (size_t)(f * NS + (side == 0 ? j + N1 * P : j)) * ld + nb);
    (side == 0 ? HD : HU)[r] = v;
  }
  if (tid == 0) {
    bool ok = !TMA || (tma_ok && mbar_wait(bar, phase & 1, a.polls));
    if (TMA && tma_ok && !ok) {
      atomicOr(a.errflag, (unsigned)FLAG_TIMEOUT);
      mbar_wait(bar, phase & 1);
    }
    *s_ok = ok ? 1 : 0;
  }
  if (tma_ok) ++phase;
  __syncthreads();
  return *s_ok != 0;
}

// Weighted volume terms at one quadrature point of quadrature weight Wg: gxv / gyv the x / y fluxes
// of the NFL fields with a conservative flux (times Wg and the metric factors cx, cy), gs the
// non-conservative source of alpha = 1/(gamma-1) (times Wg J), from the point values ug and the
// reference derivatives (dax, day) of alpha (evaluate_sf, code/src/physics/physics.cu:248-301).
template <int NF, int NFL, int NY, bool GC>
__device__ __forceinline__ void point_terms(const double (&ug)[NF], double dax, double day, double Wg,
                                            const TileArgs& a, double (&gxv)[NFL], double (&gyv)[NFL], double& gs) {
  const double rho = ug[0], irho = __drcp_rn(rho);
  const double uu = ug[1] * irho, vv = ug[2] * irho, Et = ug[3];
  const double gm1 = GC ? rho * __drcp_rn(ug[4]) : __drcp_rn(ug[4]);  // gamma - 1
  const double p = gm1 * (Et - 0.5 * rho * (uu * uu + vv * vv));
  const double wx = Wg * a.cx, wy = Wg * a.cy;
  const double mx = ug[1] * wx, my = ug[2] * wy;
  gxv[0] = mx; gxv[1] = mx * uu + wx * p; gxv[2] = mx * vv; gxv[3] = wx * ((Et + p) * uu);
  gyv[0] = my; gyv[1] = my * uu; gyv[2] = my * vv + wy * p; gyv[3] = wy * ((Et + p) * vv);
#pragma unroll
  for (int k = 0; k < NY; ++k) { gxv[4 + k] = wx * (ug[5 + k] * uu); gyv[4 + k] = wy * (ug[5 + k] * vv); }
  if constexpr (GC) { gxv[4] = wx * (ug[4] * uu); gyv[4] = wy * (ug[4] * vv); }
  gs = (Wg * a.J) * (-uu * dax * a.sx - vv * day * a.sy);
}

// The work of one tile (origin tx0, ty0).  The caller has initialised the mbarrier at the start of
// shared memory; `phase` counts its completed phases (a persistent caller runs many tiles on one
// barrier).  Every early return is taken by the whole CTA, after its last barrier.
// NY passive mass fractions rho*Y_k follow the five gamma-model fields: conservative volume flux
// rho*Y_k (u, v) (physics.cu:293-298) and the interface fluxes of phys::riemann2d_rcp.
// GC: the GAMCONS model (fifth field rho/(gamma-1), conservative flux rho u/(gamma-1), no source;
// physics.cu:253-281), with NY = 0.
// TMA = false: the tile and the stage base come in by plain coalesced loads (grids whose row pitch
// nx * 8 bytes is not a multiple of 16, which a tensor map cannot describe); same arithmetic.
template <int P, int FLUX, int MODE, int TW, int TH, int UNROLL, int NY = 0, bool GC = false, bool TMA = true>
__device__ __forceinline__ void tile2d_body(const TileArgs& a, const CUtensorMap* mapU, const CUtensorMap* mapB,
                                            int tx0, int ty0, unsigned char* smraw, uint32_t& phase) {
  static_assert(!(GC && NY > 0), "GAMCONS with mass fractions is not built");
  using Dm = TileDims<P, TW, TH, NY>;
  constexpr int N1 = Dm::N1, NS = Dm::NS, NF = Dm::NF, NT = Dm::NT, NXF = Dm::NXF;
  constexpr int FS = NF + 1;             // face record: NF fluxes, ncterm
  constexpr int NFL = 4 + NY + (GC ? 1 : 0);  // fields with a volume flux (rho, rho u, rho v, E, alpha | rho Y_k)
  auto fld = [](int k) { return (GC || k < 4) ? k : k + 1; };
  uint64_t* bar = reinterpret_cast<uint64_t*>(smraw);
  int* s_ok = reinterpret_cast<int*>(smraw + 8);
  int* codes = reinterpret_cast<int*>(smraw + Dm::head_bytes);  // [L: TH][R: TH][D: TW][U: TW]
  double* Us = reinterpret_cast<double*>(smraw + Dm::off_tile);  // [NF*NS][NT]
  double* HL = reinterpret_cast<double*>(smraw + Dm::off_halo);  // [TH][NF][N1] left neighbours' right-face nodes
  double* HR = HL + TH * NF * N1;          // [TH][NF][N1]
  double* HD = HR + TH * NF * N1;          // [TW][NF][N1]  bottom neighbours' top-face nodes
  double* HU = HD + TW * NF * N1;          // [TW][NF][N1]
  double* Fs = reinterpret_cast<double*>(smraw + Dm::off_face);  // [NXF + NYF][6] F[5], nc

  const int tid = threadIdx.x;
  const int ld = a.ld, nx = a.nx;
  constexpr bool kSplit = Dm::split_faces;
  constexpr bool kPrefetch = MODE != MODE_RESIDUAL && !kSplit;
  constexpr int NYF = Dm::NYF;

  // ---------------- phase 0: stage the tile (TMA) and the neighbour strips ----------------
  if (!tile_stage_in<P, TW, TH, NY, TMA>(a, mapU, tx0, ty0, smraw, phase, tid, NT)) return;

  // ---------------- phase 1: face fluxes, each face of the tile once ----------------
  tile_face_fluxes<P, FLUX, TW, TH, NY, GC>(Us, HL, HR, HD, HU, codes, Fs, tid, NT, 0, kSplit ? NXF : NXF + NYF, 0);
  __syncthreads();

  // ---------------- phase 2: volume terms and assembly, one thread per element ----------------
  const int tx = tid % TW, ty = tid / TW;
  const int e = (ty0 + ty) * nx + tx0 + tx;
  constexpr int NG1 = Tab2<P>::NG1;
  double r[NF][NS];
#pragma unroll
  for (int f = 0; f < NF; ++f)
#pragma unroll
    for (int t = 0; t < NS; ++t) r[f][t] = 0.0;
  // face contributions of the four faces (L: +F+nc, R: -F+nc, D: +F+nc, U: -F+nc); split faces:
  // the x-faces' records, then (after the y-faces replaced them) the y-faces'
#pragma unroll
  for (int kf = 0; kf < 4; ++kf) {
    if (kSplit && kf == 2) {
      __syncthreads();  // every thread has read its x-face records
      tile_face_fluxes<P, FLUX, TW, TH, NY, GC>(Us, HL, HR, HD, HU, codes, Fs, tid, NT, NXF, NXF + NYF, NXF);
      __syncthreads();
    }
    const int yrec = kSplit ? 0 : NXF;  // first y-face record in the buffer
    int base;
    double s, jw;
    if (kf == 0) { base = (tx * TH + ty) * N1; s = 1.0; jw = a.JFx; }
    else if (kf == 1) { base = ((tx + 1) * TH + ty) * N1; s = -1.0; jw = a.JFx; }
    else if (kf == 2) { base = yrec + (ty * TW + tx) * N1; s = 1.0; jw = a.JFy; }
    else { base = yrec + ((ty + 1) * TW + tx) * N1; s = -1.0; jw = a.JFy; }
#pragma unroll
    for (int g = 0; g < N1; ++g) {
      const double* fp = Fs + (base + g) * FS;
      const double w = jw * DGB_TAB2(P, wf[g]);
      double c[NF];
#pragma unroll
      for (int f = 0; f < NF; ++f) c[f] = (s * fp[f] + (f == 4 ? fp[NF] : 0.0)) * w;
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        const int t = kf == 0 ? N1 * j : kf == 1 ? P + N1 * j : kf == 2 ? j : j + N1 * P;
        const double b = DGB_TAB2(P, Bf[g][j]);
#pragma unroll
        for (int f = 0; f < NF; ++f) r[f][t] += b * c[f];
      }
    }
  }
  double* Ub = Fs;  // prefetched stage base (SSP) / accumulator (RK4), [NF*NS][NT]
  const bool need = kPrefetch && ((MODE == MODE_SSP && a.a != 0.0) || (MODE == MODE_RK4 && a.Uacc != nullptr));
  if (kPrefetch) {
    // the face buffer is free once every thread has read its face fluxes
    fence_proxy_async_smem();
    __syncthreads();
    if constexpr (TMA) {
      if (tid == 0 && need) {
        mbar_arrive_expect_tx(bar, Dm::tile_bytes);
        tma_load_3d(Ub, mapB, tx0, ty0, 0, bar);
      }
    } else if (need) {
      const double* base = MODE == MODE_SSP ? a.Ubase : a.Uacc;
      for (int k = tid; k < NF * NS * NT; k += NT) {
        const int q = k / NT, el = k % NT;
        Ub[k] = __ldg(base + (size_t)q * ld + (size_t)(ty0 + el / TW) * nx + tx0 + el % TW);
      }
    }
  }

  // volume terms: collocation sum-factorised (x-contraction per quadrature column gx, then y per
  // point), lift accumulated per point with the tensor-product derivative tables
  const double* us = Us + tid;  // thread-private column of the tile: us[(f*NS + t)*NT]
#pragma unroll(UNROLL)
  for (int gx = 0; gx < NG1; ++gx) {
    double Tc[NF][N1], dT[N1];  // column values: sum_ix l_ix(x_gx) u(ix, iy), and of l' for alpha
#pragma unroll
    for (int iy = 0; iy < N1; ++iy) {
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        double sacc = 0;
#pragma unroll
        for (int ix = 0; ix < N1; ++ix) sacc += DGB_TAB2(P, B1[gx][ix]) * us[(f * NS + ix + N1 * iy) * NT];
        Tc[f][iy] = sacc;
      }
      double sd = 0;
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) sd += DGB_TAB2(P, D1[gx][ix]) * us[(4 * NS + ix + N1 * iy) * NT];
      dT[iy] = sd;
    }
    double Ax[NFL][N1], Ay[NFL][N1], As[N1];  // column sums of the sum-factorised lift
#pragma unroll
    for (int iy = 0; iy < N1; ++iy) {
      As[iy] = 0.0;
#pragma unroll
      for (int f = 0; f < NFL; ++f) Ax[f][iy] = Ay[f][iy] = 0.0;
    }
#pragma unroll
    for (int gy = 0; gy < NG1; ++gy) {
      const int g = gx * NG1 + gy;
      double ug[NF], dax = 0, day = 0;
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        double sacc = 0;
#pragma unroll
        for (int iy = 0; iy < N1; ++iy) sacc += DGB_TAB2(P, B1[gy][iy]) * Tc[f][iy];
        ug[f] = sacc;
      }
#pragma unroll
      for (int iy = 0; iy < N1; ++iy) { dax += DGB_TAB2(P, B1[gy][iy]) * dT[iy]; day += DGB_TAB2(P, D1[gy][iy]) * Tc[4][iy]; }
      double gxv[NFL], gyv[NFL], gs;
      point_terms<NF, NFL, NY, GC>(ug, dax, day, DGB_TAB2(P, W[g]), a, gxv, gyv, gs);
      if constexpr (kSfLift) {
#pragma unroll
        for (int iy = 0; iy < N1; ++iy) {
          const double b = DGB_TAB2(P, B1[gy][iy]), d = DGB_TAB2(P, D1[gy][iy]);
#pragma unroll
          for (int f = 0; f < NFL; ++f) { Ax[f][iy] += b * gxv[f]; Ay[f][iy] += d * gyv[f]; }
          if (!GC) As[iy] += b * gs;
        }
      } else {
#pragma unroll
        for (int t = 0; t < NS; ++t) {
#pragma unroll
          for (int f = 0; f < NFL; ++f) r[fld(f)][t] += DGB_TAB2(P, dPx[g][t]) * gxv[f] + DGB_TAB2(P, dPy[g][t]) * gyv[f];
          if (!GC) r[4][t] += DGB_TAB2(P, Phi[g][t]) * gs;
        }
      }
    }
    if constexpr (kSfLift) {
      // dPx = l'_ix(x_gx) l_iy(x_gy), dPy = l_ix(x_gx) l'_iy(x_gy), Phi = l_ix(x_gx) l_iy(x_gy)
#pragma unroll
      for (int iy = 0; iy < N1; ++iy)
#pragma unroll
        for (int ix = 0; ix < N1; ++ix) {
          const double dx = DGB_TAB2(P, D1[gx][ix]), bx = DGB_TAB2(P, B1[gx][ix]);
          const int t = ix + N1 * iy;
#pragma unroll
          for (int f = 0; f < NFL; ++f) r[fld(f)][t] += dx * Ax[f][iy] + bx * Ay[f][iy];
          if (!GC) r[4][t] += bx * As[iy];
        }
    }
  }
  if (MODE == MODE_RESIDUAL) {
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
      for (int t = 0; t < NS; ++t) a.out[(size_t)(f * NS + t) * ld + e] = r[f][t];
    return;
  }
  if (need) {
    if (TMA && tid == 0) {
      bool ok = mbar_wait(bar, phase & 1, a.polls);
      if (!ok) {
        atomicOr(a.errflag, (unsigned)FLAG_TIMEOUT);
        mbar_wait(bar, phase & 1);
      }
      *s_ok = ok ? 1 : 0;
    }
    if (TMA) ++phase;
    __syncthreads();
    if (!*s_ok) return;
  }
  const double dt = a.dt_override > 0 ? a.dt_override : a.scal->dt;
  const double sc = dt * a.invJ;
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    // DU = dt/J (M1^-1 (x) M1^-1) R : first along x then along y
    double tmp[NS];
#pragma unroll
    for (int iy = 0; iy < N1; ++iy)
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) {
        double s = 0;
#pragma unroll
        for (int q = 0; q < N1; ++q) s += DGB_TAB2(P, M1i[ix][q]) * r[f][q + N1 * iy];
        tmp[ix + N1 * iy] = s;
      }
#pragma unroll
    for (int iy = 0; iy < N1; ++iy)
#pragma unroll
      for (int ix = 0; ix < N1; ++ix) {
        double s = 0;
#pragma unroll
        for (int q = 0; q < N1; ++q) s += DGB_TAB2(P, M1i[iy][q]) * tmp[ix + N1 * q];
        const double du = sc * s;
        const int t = ix + N1 * iy;
        const size_t gi = (size_t)(f * NS + t) * ld + e;
        if (MODE == MODE_SSP) {
          const double ub = kPrefetch ? Ub[(f * NS + t) * NT + tid] : (a.a != 0.0 ? __ldg(a.Ubase + gi) : 0.0);
          const double base = a.a != 0.0 ? a.a * ub : 0.0;
          a.out[gi] = base + a.b * (us[(f * NS + t) * NT] + du);
        } else {
          a.out[gi] = du;
          if (a.Uacc) a.Uacc[gi] = (kPrefetch ? Ub[(f * NS + t) * NT + tid] : a.Uacc[gi]) + a.b * du;
        }
      }
  }
}

template <int P, int FLUX, int MODE, int TW, int TH, int NY = 0, bool GC = false, bool TMA = true>
__global__ void __launch_bounds__(TW * TH, 2)
    residual2d_tile_kernel(const TileArgs a, const __grid_constant__ CUtensorMap mapU,
                           const __grid_constant__ CUtensorMap mapB) {
  extern __shared__ __align__(128) unsigned char smraw[];
  pdl_wait();
  if (a.scal && a.scal->flags) return;
  if (threadIdx.x == 0) {
    mbar_init(reinterpret_cast<uint64_t*>(smraw), 1);
    fence_mbar_init();
  }
  uint32_t phase = 0;
  tile2d_body<P, FLUX, MODE, TW, TH, vol_unroll<P>(), NY, GC, TMA>(a, &mapU, &mapB, blockIdx.x * TW, blockIdx.y * TH,
                                                             smraw, phase);
  pdl_trigger();
}

}  // namespace dgb
