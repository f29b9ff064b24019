// Problem setup: the host-side sequence of the reference driver (code/src/main.cc:273-860)
// rebuilt from scratch, producing the same arrays in the same layouts, plus the compact
// tensor-product description used by the device kernels.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>

#include "host.h"

namespace dgb {

namespace {

int lin_type(int p) { return p == 1 ? MSH_LIN_2 : p == 2 ? MSH_LIN_3 : p == 3 ? MSH_LIN_4 : MSH_LIN_5; }
int qua_type(int p) { return p == 1 ? MSH_QUA_4 : p == 2 ? MSH_QUA_9 : p == 3 ? MSH_QUA_16 : MSH_QUA_25; }

// Element quadrature of gaussIntegration::getLine/getQuad(2p+1)
// (code/src/quadratures/GaussQuadratureLin.cc:16-37, GaussQuadratureQuad.cc:113-149):
// lines use n = p+1 Gauss points; quads use the 2x2 rule of GQQ4 for p = 1 and the
// (p+2) x (p+2) tensor rule (x index outer, y index inner) for p >= 2.
void element_quadrature(int dim, int p, std::vector<double>& pts, std::vector<double>& w) {
  pts.clear();
  w.clear();
  if (dim == 1) {
    std::vector<double> x, ww;
    gauss_legendre(p + 1, x, ww);
    for (int i = 0; i <= p; ++i) { pts.push_back(x[i]); pts.push_back(0.0); w.push_back(ww[i]); }
    return;
  }
  if (p == 1) {
    const double a = 1.0 / std::sqrt(3.0);
    const double q[4][2] = {{a, a}, {-a, a}, {a, -a}, {-a, -a}};
    for (auto& v : q) { pts.push_back(v[0]); pts.push_back(v[1]); w.push_back(1.0); }
    return;
  }
  const int n = p + 2;
  std::vector<double> x, ww;
  gauss_legendre(n, x, ww);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) { pts.push_back(x[i]); pts.push_back(x[j]); w.push_back(ww[i] * ww[j]); }
}

struct Basis {
  int dim, p;
  std::vector<double> n1;      // 1D nodes in LIN order
  std::vector<double> ref;     // reference node coordinates (N_s x 2)
  std::vector<int> ix, iy;     // 1D node indices of each element node
  int ns() const { return (int)ix.size(); }
  double f(int i, double x, double y) const {
    double v = lagrange1d(n1, ix[i], x);
    if (dim == 2) v *= lagrange1d(n1, iy[i], y);
    return v;
  }
  double df(int i, int a, double x, double y) const {
    if (dim == 1) return dlagrange1d(n1, ix[i], x);
    if (a == 0) return dlagrange1d(n1, ix[i], x) * lagrange1d(n1, iy[i], y);
    return lagrange1d(n1, ix[i], x) * dlagrange1d(n1, iy[i], y);
  }
};

Basis make_basis(int dim, int p) {
  Basis b;
  b.dim = dim;
  b.p = p;
  b.n1 = line_nodes(p);
  auto find1 = [&](double v) {
    int best = 0;
    for (int k = 0; k <= p; ++k)
      if (std::fabs(b.n1[k] - v) < std::fabs(b.n1[best] - v)) best = k;
    return best;
  };
  if (dim == 1) {
    for (int k = 0; k <= p; ++k) { b.ref.push_back(b.n1[k]); b.ref.push_back(0.0); b.ix.push_back(k); b.iy.push_back(0); }
  } else {
    b.ref = quad_nodes(p);
    for (size_t k = 0; k < b.ref.size() / 2; ++k) { b.ix.push_back(find1(b.ref[2 * k])); b.iy.push_back(find1(b.ref[2 * k + 1])); }
  }
  return b;
}

// C (m x n) = A (m x k) * B (k x n), column-major.
std::vector<double> matmul(const std::vector<double>& A, const std::vector<double>& B, int m, int k, int n) {
  std::vector<double> C((size_t)m * n, 0.0);
  for (int j = 0; j < n; ++j)
    for (int l = 0; l < k; ++l) {
      const double b = B[l + (size_t)j * k];
      for (int i = 0; i < m; ++i) C[i + (size_t)j * m] += A[i + (size_t)l * m] * b;
    }
  return C;
}

double factorial(int n) { double f = 1; for (int i = 2; i <= n; ++i) f *= i; return f; }

// monovandermonde1d (main.cc:1146-1157): V(i,j) = r_i^j / j!
std::vector<double> mono_vandermonde(const std::vector<double>& r, int p) {
  const int n = (int)r.size();
  std::vector<double> V((size_t)n * (p + 1));
  for (int j = 0; j <= p; ++j)
    for (int i = 0; i < n; ++i) V[i + (size_t)j * n] = std::pow(r[i], j) / factorial(j);
  return V;
}

Status fail(int code, const std::string& msg) { Status s; s.code = code; s.msg = msg; return s; }

}  // namespace

Status build_problem(Mesh&& mesh, int dim, int p, const std::string& kind, int flux, int limiter, double cfl,
                     const std::vector<double>& thresholds, const std::vector<double>& out_times, double final_time,
                     Problem& P, int n_mass, bool gamcons) {
  P = Problem();
  if (dim != 1 && dim != 2) return fail(1, "dimension must be 1 or 2");
  if (n_mass < 0 || n_mass > 10) return fail(1, "mass fractions: 0..10 (MASS of the reference Makefile)");
  if (p < 1 || p > 4) return fail(4, "polynomial order must be 1..4");
  if (dim == 1 && kind != "lin") return fail(4, "1D problems use 'lin' elements");
  if (dim == 2 && kind != "qua") return fail(4, "2D problems use 'qua' elements (triangles are outside this path)");
  P.D = dim;
  P.p = p;
  P.N_Y = n_mass;
  P.gamcons = gamcons;
  P.N_F = (dim == 1 ? 4 : 5) + n_mass;
  P.flux = flux;
  P.limiter = limiter;
  P.cfl = cfl;
  P.thresholds = thresholds;
  P.output_times = out_times;
  P.final_time = final_time;
  P.mesh = std::move(mesh);
  const int nsides = dim == 1 ? 0 : 4;
  P.N_N = dim == 1 ? 2 : 4;
  P.face_type = dim == 1 ? MSH_PNT : lin_type(p);
  P.elem_type = dim == 1 ? lin_type(p) : qua_type(p);
  auto it = P.mesh.by_type.find(P.elem_type);
  if (it == P.mesh.by_type.end() || it->second.empty())
    return fail(3, "mesh has no elements of Gmsh type " + std::to_string(P.elem_type) + " for order " + std::to_string(p));
  P.elements = it->second;
  const Basis B = make_basis(dim, p);
  P.N_s = B.ns();
  P.N_E = (int)P.elements.size();
  for (auto& e : P.elements)
    if ((int)e.nodes.size() != P.N_s) return fail(3, "element node count mismatch");
  P.closures = closures_for(dim, p);
  P.ref_nodes = B.ref;

  // ---- interfaces (simpleInterface::BuildInterfaces, simpleMesh.cc:770-989) ----
  struct IF { int phys = 0; int el[2] = {-1, -1}; int cl[2] = {-1, -1}; };
  std::map<std::vector<int>, IF> imap;
  auto fit = P.mesh.by_type.find(P.face_type);
  if (fit != P.mesh.by_type.end())
    for (auto& fe : fit->second) {
      std::vector<int> key = fe.nodes;
      std::sort(key.begin(), key.end());
      IF v; v.phys = fe.ptag;
      imap[key] = v;
    }
  for (int e = 0; e < P.N_E; ++e) {
    const Element& el = P.elements[e];
    for (size_t j = 0; j < P.closures.size(); ++j) {
      std::vector<int> key;
      for (int c : P.closures[j]) key.push_back(el.nodes[c]);
      std::sort(key.begin(), key.end());
      IF& f = imap[key];
      if (f.el[0] < 0) {
        f.el[0] = e; f.cl[0] = (int)j;
        if (f.phys == 2 || f.phys == 3 || f.phys == 4) { f.el[1] = e; f.cl[1] = (int)j; }
      } else if (f.el[0] != e) {
        if (f.el[1] < 0) { f.el[1] = e; f.cl[1] = (int)j + nsides; }
        else if (f.el[1] != e) return fail(3, "interface shared by more than two elements");
      }
    }
  }
  // periodic pairing (pairPeriodic, simpleMesh.cc:21-88)
  {
    const double eps = 1e-8;
    std::vector<std::pair<const std::vector<int>*, IF*>> per;
    for (auto& kv : imap) if (kv.second.phys == 1) per.push_back({&kv.first, &kv.second});
    auto box = [&](const std::vector<int>& n, double& xs, double& xe, double& ys, double& ye) {
      xs = xe = P.mesh.x[n[0]]; ys = ye = P.mesh.y[n[0]];
      for (int k : n) { xs = std::min(xs, P.mesh.x[k]); xe = std::max(xe, P.mesh.x[k]); ys = std::min(ys, P.mesh.y[k]); ye = std::max(ye, P.mesh.y[k]); }
    };
    for (size_t a = 0; a < per.size(); ++a) {
      IF* f1 = per[a].second;
      if (f1->el[1] >= 0) continue;
      for (size_t b = 0; b < per.size(); ++b) {
        IF* f2 = per[b].second;
        if (f2->el[1] >= 0 || f1->el[1] >= 0) continue;
        bool paired = false;
        if (dim == 1) {
          double x1 = P.mesh.x[(*per[a].first)[0]], x2 = P.mesh.x[(*per[b].first)[0]];
          paired = std::fabs(x1 - x2) > eps;
        } else {
          double xs1, xe1, ys1, ye1, xs2, xe2, ys2, ye2;
          box(*per[a].first, xs1, xe1, ys1, ye1);
          box(*per[b].first, xs2, xe2, ys2, ye2);
          if (std::fabs(xs1 - xs2) < eps && std::fabs(xe1 - xe2) < eps && std::fabs(ys1 - ys2) < eps && std::fabs(ye1 - ye2) < eps) paired = false;
          else if (std::fabs(ys1 - ye1) > eps) paired = std::fabs(ys1 - ys2) < eps && std::fabs(ye1 - ye2) < eps;
          else if (std::fabs(xs1 - xe1) > eps) paired = std::fabs(xs1 - xs2) < eps && std::fabs(xe1 - xe2) < eps;
        }
        if (paired) {
          f1->el[1] = f2->el[0]; f1->cl[1] = f2->cl[0] + nsides;
          f2->el[1] = f1->el[0]; f2->cl[1] = f1->cl[0] + nsides;
        }
      }
    }
  }
  for (auto& kv : imap) {
    if (kv.second.el[0] < 0 || kv.second.el[1] < 0) return fail(3, "interface without an element on each side");
    Interface I; I.phys = kv.second.phys;
    I.el[0] = kv.second.el[0]; I.el[1] = kv.second.el[1];
    I.cl[0] = kv.second.cl[0]; I.cl[1] = kv.second.cl[1];
    P.ifaces.push_back(I);
  }
  P.M_T = (int)P.ifaces.size();

  // ---- quadrature and basis values (main.cc:312-441) ----
  element_quadrature(dim, p, P.qpts, P.qw);
  P.N_G = (int)P.qw.size();
  if (dim == 1) { P.fqpts = {0.0}; P.fqw = {1.0}; P.M_s = 1; P.M_G = 1; }
  else {
    std::vector<double> x, w;
    gauss_legendre(p + 1, x, w);
    P.fqpts = x; P.fqw = w; P.M_s = p + 1; P.M_G = p + 1;
  }
  const int NG = P.N_G, NS = P.N_s, D = dim;
  P.phi.assign((size_t)NG * NS, 0.0);
  P.dphi.assign((size_t)NG * D * NS, 0.0);
  P.phi_w.assign((size_t)NG * NS, 0.0);
  P.dphi_w.assign((size_t)NG * D * NS, 0.0);
  for (int g = 0; g < NG; ++g)
    for (int i = 0; i < NS; ++i) {
      const double xq = P.qpts[2 * g], yq = P.qpts[2 * g + 1];
      P.phi[g + (size_t)i * NG] = B.f(i, xq, yq);
      P.phi_w[g + (size_t)i * NG] = P.phi[g + (size_t)i * NG] * P.qw[g];
      for (int a = 0; a < D; ++a) {
        P.dphi[(g * D + a) + (size_t)i * NG * D] = B.df(i, a, xq, yq);
        P.dphi_w[(g * D + a) + (size_t)i * NG * D] = P.dphi[(g * D + a) + (size_t)i * NG * D] * P.qw[g];
      }
    }
  P.psi.assign((size_t)P.M_G * P.M_s, 0.0);
  P.dpsi.assign((size_t)P.M_G * P.M_s, 0.0);
  P.psi_w.assign((size_t)P.M_G * P.M_s, 0.0);
  if (dim == 1) { P.psi[0] = 1.0; P.dpsi[0] = 0.0; P.psi_w[0] = 1.0; }
  else {
    for (int g = 0; g < P.M_G; ++g)
      for (int j = 0; j < P.M_s; ++j) {
        P.psi[g + (size_t)j * P.M_G] = lagrange1d(B.n1, j, P.fqpts[g]);
        P.dpsi[g + (size_t)j * P.M_G] = dlagrange1d(B.n1, j, P.fqpts[g]);
        P.psi_w[g + (size_t)j * P.M_G] = P.psi[g + (size_t)j * P.M_G] * P.fqw[g];
      }
  }

  // ---- element node coordinates, centroids, cartesian test (main.cc:450-470) ----
  const int NE = P.N_E;
  P.xyz_nodes.assign((size_t)NS * NE * D, 0.0);
  for (int e = 0; e < NE; ++e)
    for (int i = 0; i < NS; ++i) {
      const int n = P.elements[e].nodes[i];
      P.xyz_nodes[i + (size_t)(e * D + 0) * NS] = P.mesh.x[n];
      if (D == 2) P.xyz_nodes[i + (size_t)(e * D + 1) * NS] = P.mesh.y[n];
    }
  auto X = [&](int i, int e, int a) { return P.xyz_nodes[i + (size_t)(e * D + a) * NS]; };
  if (dim == 1) P.cartesian = true;
  else {
    const double x0 = X(0, 0, 0), y0 = X(0, 0, 1), x1 = X(1, 0, 0), y1 = X(1, 0, 1);
    const double x2 = X(2, 0, 0), y2 = X(2, 0, 1), x3 = X(3, 0, 0), y3 = X(3, 0, 1);
    P.cartesian = std::fabs((x1 - x0) * (x2 - x1) + (y1 - y0) * (y2 - y1)) < 1e-9 &&
                  std::fabs((x2 - x1) * (x3 - x2) + (y2 - y1) * (y3 - y2)) < 1e-9;  // simpleMesh.cc:1102-1133
  }

  // ---- normals (simpleMesh::buildNormals, simpleMesh.cc:206-319): outward from el[0] ----
  P.normals.assign((size_t)D * P.M_T, 0.0);
  for (int t = 0; t < P.M_T; ++t) {
    const Interface& I = P.ifaces[t];
    const int e = I.el[0];
    const auto& cl = P.closures[I.cl[0]];
    double n[2] = {0, 0};
    if (dim == 1) {
      n[0] = (cl[0] == 0) ? -1.0 : 1.0;
      if (X(1, e, 0) < X(0, e, 0)) n[0] = -n[0];
    } else {
      // straight edge from closure vertex a to b, element vertices counter-clockwise
      const double ax = X(cl[0], e, 0), ay = X(cl[0], e, 1), bx = X(cl[1], e, 0), by = X(cl[1], e, 1);
      double nx = by - ay, ny = -(bx - ax);
      // orientation of the element (signed area of the corner polygon)
      double area = 0;
      for (int k = 0; k < 4; ++k) area += X(k, e, 0) * X((k + 1) % 4, e, 1) - X((k + 1) % 4, e, 0) * X(k, e, 1);
      if (area < 0) { nx = -nx; ny = -ny; }
      const double nn = std::sqrt(nx * nx + ny * ny);
      n[0] = nx / nn; n[1] = ny / nn;
    }
    for (int a = 0; a < D; ++a) P.normals[a + (size_t)t * D] = n[a];
  }

  // ---- boundary list (buildBoundary, simpleMesh.cc:462-532): reflective then "otherone" (5) ----
  for (int t = 0; t < P.M_T; ++t) if (P.ifaces[t].phys == 3) P.boundary_map.push_back(t);
  for (int t = 0; t < P.M_T; ++t) if (P.ifaces[t].phys == 5) P.boundary_map.push_back(t);
  P.M_B = (int)P.boundary_map.size();

  // ---- neighbours (buildNeighbors, simpleMesh.cc:664-754) ----
  P.neighbors.assign((size_t)P.N_N * NE, 0);
  {
    std::vector<int> nn(NE, 0);
    const double eps = 1e-6;
    for (int t = 0; t < P.M_T; ++t) {
      const Interface& I = P.ifaces[t];
      const int e1 = I.el[0];
      int e2 = I.el[1];
      if (e2 == e1 && (I.phys == 2 || I.phys == 3 || I.phys == 4)) e2 = -I.phys;
      if (!P.cartesian) {
        P.neighbors[e1 * P.N_N + nn[e1]++] = e2;
        if (e2 >= 0) P.neighbors[e2 * P.N_N + nn[e2]++] = e1;
        continue;
      }
      const double nx = P.normals[(size_t)t * D], ny = D == 2 ? P.normals[(size_t)t * D + 1] : 0.0;
      int s1, s2;
      if (std::fabs(ny) < eps && nx < 0) { s1 = 0; s2 = 1; }
      else if (std::fabs(ny) < eps && nx > 0) { s1 = 1; s2 = 0; }
      else if (std::fabs(nx) < eps && ny < 0) { s1 = 2; s2 = 3; }
      else if (std::fabs(nx) < eps && ny > 0) { s1 = 3; s2 = 2; }
      else return fail(3, "error in neighbour creation: face normal is not axis-aligned");
      P.neighbors[e1 * P.N_N + s1] = e2;
      if (e2 >= 0) P.neighbors[e2 * P.N_N + s2] = e1;
    }
  }

  // ---- Jacobians (dg_jacobians_elements, dg_functions.cc:33-72) ----
  P.J.assign(NE, 0.0);
  P.invJac.assign((size_t)NG * D * NE * D, 0.0);
  for (int e = 0; e < NE; ++e) {
    double det0 = 0.0;
    for (int g = 0; g < NG; ++g) {
      double Jm[2][2] = {{0, 0}, {0, 0}};  // Jm[alpha][a] = dx_alpha / dxi_a
      for (int al = 0; al < D; ++al)
        for (int a = 0; a < D; ++a) {
          double s = 0;
          for (int i = 0; i < NS; ++i) s += X(i, e, al) * P.dphi[(g * D + a) + (size_t)i * NG * D];
          Jm[al][a] = s;
        }
      if (g == 0) det0 = D == 1 ? std::sqrt(Jm[0][0] * Jm[0][0]) : Jm[0][0] * Jm[1][1] - Jm[1][0] * Jm[0][1];
      auto IJ = [&](int al, int a) -> double& { return P.invJac[(((size_t)e * NG + g) * D + al) * D + a]; };
      if (D == 1) IJ(0, 0) = 1.0 / Jm[0][0];
      else {
        IJ(0, 0) = 1.0 / det0 * Jm[1][1];
        IJ(1, 0) = -1.0 / det0 * Jm[1][0];
        IJ(0, 1) = -1.0 / det0 * Jm[0][1];
        IJ(1, 1) = 1.0 / det0 * Jm[0][0];
      }
    }
    P.J[e] = std::fabs(det0);
  }
  // faces (dg_jacobians_face, dg_functions.cc:74-95)
  P.JF.assign((size_t)2 * P.M_T, 0.0);
  for (int t = 0; t < P.M_T; ++t)
    for (int d = 0; d < 2; ++d) {
      if (D == 1) { P.JF[t * 2 + d] = 1.0; continue; }
      const Interface& I = P.ifaces[t];
      const auto& cl = P.closures[I.cl[d]];
      double det = 0;
      for (int al = 0; al < D; ++al) {
        double s = 0;
        for (int j = 0; j < P.M_s; ++j) s += X(cl[j], I.el[d], al) * P.dpsi[0 + (size_t)j * P.M_G];
        det += s * s;
      }
      P.JF[t * 2 + d] = std::sqrt(det);
    }

  // ---- inverse mass matrices (dg_inverse_mass_matrix, dg_functions.cc:98-174) ----
  P.Minv.assign((size_t)NS * NS * NE, 0.0);
  {
    std::vector<double> Mref((size_t)NS * NS, 0.0);  // phi^T phi_w (without J)
    for (int j = 0; j < NS; ++j)
      for (int i = 0; i < NS; ++i) {
        double s = 0;
        for (int g = 0; g < NG; ++g) s += P.phi[g + (size_t)i * NG] * P.phi_w[g + (size_t)j * NG];
        Mref[i + (size_t)j * NS] = s;
      }
    std::map<double, std::vector<double>> cache;
    for (int e = 0; e < NE; ++e) {
      auto c = cache.find(P.J[e]);
      if (c == cache.end()) {
        std::vector<double> M(Mref);
        for (double& v : M) v *= P.J[e];
        if (!invert(M, NS)) return fail(3, "singular mass matrix");
        c = cache.emplace(P.J[e], M).first;
      }
      const auto& Mi = c->second;
      for (int k = 0; k < NS; ++k)
        for (int i = 0; i < NS; ++i) P.Minv[((size_t)e * NS + k) * NS + i] = Mi[i + (size_t)k * NS];
    }
  }

  // ---- maps (dg_mappings, dg_functions.cc:177-238) ----
  const int NF = P.N_F, MS = P.M_s;
  P.map.assign((size_t)MS * P.M_T * NF * 2, 0);
  P.invmap.assign((size_t)MS * P.N_N * NE * NF * 2, 0);
  {
    std::vector<int> cnt((size_t)NF * NE, 0);
    for (int t = 0; t < P.M_T; ++t) {
      const Interface& I = P.ifaces[t];
      const int e1 = I.el[0], e2 = I.el[1];
      const auto& cl1 = P.closures[I.cl[0]];
      const auto& cl2 = P.closures[I.cl[1]];
      for (int fc = 0; fc < NF; ++fc)
        for (int j = 0; j < MS; ++j) {
          P.map[((size_t)(t * NF + fc) * 2 + 0) * MS + j] = (e1 * NF + fc) * NS + cl1[j];
          P.map[((size_t)(t * NF + fc) * 2 + 1) * MS + j] = (e2 * NF + fc) * NS + cl2[j];
          int& c1 = cnt[(size_t)e1 * NF + fc];
          P.invmap[(((size_t)e1 * NF + fc) * MS * P.N_N + c1) * 2 + 0] = cl1[j];
          P.invmap[(((size_t)e1 * NF + fc) * MS * P.N_N + c1) * 2 + 1] = ((t * NF + fc) * 2 + 0) * MS + j;
          ++c1;
          if (I.phys == 0) {
            int& c2 = cnt[(size_t)e2 * NF + fc];
            P.invmap[(((size_t)e2 * NF + fc) * MS * P.N_N + c2) * 2 + 0] = cl2[j];
            P.invmap[(((size_t)e2 * NF + fc) * MS * P.N_N + c2) * 2 + 1] = ((t * NF + fc) * 2 + 1) * MS + j;
            ++c2;
          }
        }
    }
  }

  // ---- limiter transforms (main.cc:558-583, 1348-1524) ----
  {
    std::vector<double> lq, lw;
    gauss_legendre(p + 1, lq, lw);  // getLine(2p+1)
    const int n1 = p + 1;
    std::vector<double> V = mono_vandermonde(lq, p);
    if (!invert(V, n1)) return fail(3, "singular monomial Vandermonde");
    std::vector<double> phi1((size_t)n1 * n1);
    for (int g = 0; g < n1; ++g)
      for (int i = 0; i < n1; ++i) phi1[g + (size_t)i * n1] = lagrange1d(B.n1, i, lq[g]);
    std::vector<double> T1 = matmul(V, phi1, n1, n1, n1);  // Lag -> mono in LIN node order
    if (dim == 1) {
      P.Lag2Mono = T1;
      P.Mono2Lag = T1;
      if (!invert(P.Mono2Lag, n1)) return fail(3, "singular Lag2Mono");
    } else if (P.cartesian) {
      // permutations of cartesian_permutations (main.cc:1348-1460) from element 0's nodes
      std::vector<double> xlvl(n1), ylvl(n1);
      double xmin = X(0, 0, 0), xmax = xmin, ymin = X(0, 0, 1), ymax = ymin;
      for (int i = 1; i < NS; ++i) {
        xmax = std::max(xmax, X(i, 0, 0)); xmin = std::min(xmin, X(i, 0, 0));
        ymax = std::max(ymax, X(i, 0, 1)); ymin = std::min(ymin, X(i, 0, 1));
      }
      const double dxl = (xmax - xmin) / p, dyl = (ymax - ymin) / p;
      xlvl[0] = xmin; xlvl[1] = xmax; ylvl[0] = ymin; ylvl[1] = ymax;
      for (int k = 2; k < n1; ++k) { xlvl[k] = xmin + (k - 1) * dxl; ylvl[k] = ymin + (k - 1) * dyl; }
      std::vector<double> Px((size_t)NS * NS, 0.0), Py((size_t)NS * NS, 0.0);
      int pc = 0;
      for (int yc = 0; yc < n1; ++yc) {
        std::vector<int> tmp;
        for (int i = 0; i < NS; ++i) if (std::fabs(ylvl[yc] - X(i, 0, 1)) < 1e-9) tmp.push_back(i);
        for (int xc = 0; xc < n1; ++xc)
          for (int i : tmp) if (std::fabs(xlvl[xc] - X(i, 0, 0)) < 1e-9) Px[pc++ + (size_t)i * NS] = 1.0;
      }
      pc = 0;
      for (int xc = 0; xc < n1; ++xc) {
        std::vector<int> tmp;
        for (int i = 0; i < NS; ++i) if (std::fabs(xlvl[xc] - X(i, 0, 0)) < 1e-9) tmp.push_back(i);
        for (int yc = 0; yc < n1; ++yc)
          for (int i : tmp) if (std::fabs(ylvl[yc] - X(i, 0, 1)) < 1e-9) Py[pc++ + (size_t)i * NS] = 1.0;
      }
      std::vector<double> Diag((size_t)NS * NS, 0.0);
      for (int b = 0; b < n1; ++b)
        for (int i = 0; i < n1; ++i)
          for (int j = 0; j < n1; ++j) Diag[(i + b * n1) + (size_t)(j + b * n1) * NS] = T1[i + (size_t)j * n1];
      P.Lag2MonoX = matmul(Diag, Px, NS, NS, NS);
      std::vector<double> MonoX2LagLocal = P.Lag2MonoX;
      if (!invert(MonoX2LagLocal, NS)) return fail(3, "singular Lag2MonoX");
      std::vector<double> Lag2MonoYLocal = matmul(Diag, Py, NS, NS, NS);
      P.MonoY2Lag = Lag2MonoYLocal;
      if (!invert(P.MonoY2Lag, NS)) return fail(3, "singular Lag2MonoY");
      P.MonoX2MonoY = matmul(Lag2MonoYLocal, MonoX2LagLocal, NS, NS, NS);
      // Limiting constructor (limiting.h:318-319): MonoX2Lag = MonoY2Lag*MonoX2MonoY,
      // Lag2MonoY = MonoX2MonoY*Lag2MonoX
      P.MonoX2Lag = matmul(P.MonoY2Lag, P.MonoX2MonoY, NS, NS, NS);
      P.Lag2MonoY = matmul(P.MonoX2MonoY, P.Lag2MonoX, NS, NS, NS);
    }
  }

  // ---- Dx and the CFL scale (simpleMesh::setDx, simpleMesh.cc:1140-1190; main.cc:896-897) ----
  if (dim == 1) {
    P.dx_min = X(1, 0, 0) - X(0, 0, 0);
    for (int e = 0; e < NE; ++e) P.dx_min = std::min(P.dx_min, X(1, e, 0) - X(0, e, 0));
  } else {
    auto cen = [&](int e, int a) { double c = 0; for (int k = 0; k < 4; ++k) c += X(k, e, a); return c / 4; };
    auto dist = [](double x0, double y0, double x1, double y1, double x2, double y2) {
      return std::fabs((x2 - x1) * (y1 - y0) - (x1 - x0) * (y2 - y1)) / std::sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
    };
    double d = dist(cen(0, 0), cen(0, 1), X(0, 0, 0), X(0, 0, 1), X(1, 0, 0), X(1, 0, 1));
    for (int e = 0; e < NE; ++e)
      for (int k = 0; k < 4; ++k)
        d = std::min(d, dist(cen(e, 0), cen(e, 1), X(k, e, 0), X(k, e, 1), X((k + 1) % 4, e, 0), X((k + 1) % 4, e, 1)));
    P.dx_min = 2 * d;
  }
  P.cfl_scaled = cfl * P.dx_min / (2.0 * p + 1);

  // ---- device description: Cartesian, uniformly oriented, uniform size ----
  P.gpu_ok = true;
  if (p > 3) { P.gpu_ok = false; P.gpu_reason = "device kernels are instantiated for p = 1..3"; }
  if (P.gpu_ok && !P.cartesian) { P.gpu_ok = false; P.gpu_reason = "device path needs a Cartesian mesh"; }
  if (P.gpu_ok) {
    const double hx0 = X(1, 0, 0) - X(0, 0, 0);
    const double hy0 = D == 2 ? X(3, 0, 1) - X(0, 0, 1) : 0.0;
    for (int e = 0; e < NE && P.gpu_ok; ++e) {
      const double hx = X(1, e, 0) - X(0, e, 0);
      bool good = hx > 0 && std::fabs(hx - hx0) <= 1e-9 * std::fabs(hx0);
      if (D == 2) {
        const double hy = X(3, e, 1) - X(0, e, 1);
        good = good && hy > 0 && std::fabs(hy - hy0) <= 1e-9 * std::fabs(hy0) &&
               std::fabs(X(1, e, 1) - X(0, e, 1)) <= 1e-9 * hy0 && std::fabs(X(3, e, 0) - X(0, e, 0)) <= 1e-9 * hx0;
      }
      if (!good) { P.gpu_ok = false; P.gpu_reason = "device path needs uniform, uniformly oriented axis-aligned elements"; }
    }
    P.hx = hx0;
    P.hy = hy0;
  }
  if (P.gpu_ok) {
    const int n1 = p + 1;
    P.tensor_perm.assign(NS, -1);
    for (int k = 0; k < NS; ++k) {
      const int ix = (int)std::lround((B.ref[2 * k] + 1.0) * p / 2.0);
      const int iy = D == 2 ? (int)std::lround((B.ref[2 * k + 1] + 1.0) * p / 2.0) : 0;
      P.tensor_perm[ix + n1 * iy] = k;
    }
    P.nbr.assign((size_t)P.N_N * NE, 0);
    for (int e = 0; e < NE; ++e)
      for (int k = 0; k < P.N_N; ++k) P.nbr[(size_t)k * NE + e] = P.neighbors[(size_t)e * P.N_N + k];
    // structured extents: row-major full grid
    if (D == 1) { P.nx = NE; P.ny = 1; }
    else {
      int nxg = 0;
      while (nxg < NE && P.neighbors[(size_t)nxg * P.N_N + 1] == nxg + 1) ++nxg;
      nxg += 1;
      if (nxg > 0 && NE % nxg == 0) { P.nx = nxg; P.ny = NE / nxg; }
    }
    classify_grid(P);
  }
  return Status();
}

// Structured order and per-side boundary rules of the device neighbour table P.nbr (see host.h).
void classify_grid(Problem& P) {
  const int NE = P.N_E, nx = P.nx, ny = P.ny, nsides = P.D == 1 ? 2 : 4;
  P.structured = false;
  for (int k = 0; k < 4; ++k) P.side_rule[k] = Problem::kSideMixed;
  if (nx <= 0 || ny <= 0 || (long)nx * ny != NE) return;
  auto nb = [&](int k, int e) { return P.nbr[(size_t)k * NE + e]; };
  for (int e = 0; e < NE; ++e) {
    const int ix = e % nx, iy = e / nx;
    if (ix > 0 && nb(0, e) != e - 1) return;
    if (ix < nx - 1 && nb(1, e) != e + 1) return;
    if (P.D == 2 && iy > 0 && nb(2, e) != e - nx) return;
    if (P.D == 2 && iy < ny - 1 && nb(3, e) != e + nx) return;
  }
  P.structured = true;
  for (int k = 0; k < nsides; ++k) {
    // the boundary elements of side k, the element a wrap would reach, and their rule
    const int n = k < 2 ? ny : nx;
    int rule = 0;
    for (int j = 0; j < n; ++j) {
      int e, wrap;
      if (k == 0) { e = j * nx; wrap = e + nx - 1; }
      else if (k == 1) { e = j * nx + nx - 1; wrap = j * nx; }
      else if (k == 2) { e = j; wrap = (ny - 1) * nx + j; }
      else { e = (ny - 1) * nx + j; wrap = j; }
      const int v = nb(k, e);
      const int r = v < 0 ? v : (v == wrap ? Problem::kSideWrap : Problem::kSideMixed);
      if (r == Problem::kSideMixed || (j > 0 && r != rule)) { rule = Problem::kSideMixed; break; }
      rule = r;
    }
    P.side_rule[k] = rule;
  }
}

// ---------------------------------------------------------------------------------------
// Initial states (reference layout U[(e*N_F+f)*N_s+i])
// ---------------------------------------------------------------------------------------
Status init_state(const Problem& P, const std::string& ic, const std::vector<double>& prm, uint64_t seed, double* U) {
  const int NS = P.N_s, NF = P.N_F, NE = P.N_E, D = P.D;
  auto X = [&](int i, int e, int a) { return P.xyz_nodes[i + (size_t)(e * D + a) * NS]; };
  // passive mass fractions: rho*Y_k with Y_k the region indicator `ymark` of the state set last (1
  // for the first / left / bubble region, 0 elsewhere) for even k and its complement for odd k
  double ymark = 0.0;
  auto setY = [&](int e, int i, double rho) {
    for (int k = 0; k < P.N_Y; ++k) U[(e * NF + NF - P.N_Y + k) * NS + i] = rho * (k % 2 ? 1.0 - ymark : ymark);
  };
  auto set = [&](int e, int i, const double* prim) {  // prim = rho, u, v, p, gamma (1D: rho,u,p,gamma)
    setY(e, i, prim[0]);
    double* u = U;
    if (D == 1) {
      const double rho = prim[0], vx = prim[1], pr = prim[2], g = prim[3];
      u[(e * NF + 0) * NS + i] = rho;
      u[(e * NF + 1) * NS + i] = rho * vx;
      u[(e * NF + 2) * NS + i] = 1.0 / (g - 1.0) * pr + 0.5 * rho * vx * vx;
      u[(e * NF + 3) * NS + i] = P.gamcons ? rho / (g - 1.0) : 1.0 / (g - 1.0);
    } else {
      const double rho = prim[0], vx = prim[1], vy = prim[2], pr = prim[3], g = prim[4];
      u[(e * NF + 0) * NS + i] = rho;
      u[(e * NF + 1) * NS + i] = rho * vx;
      u[(e * NF + 2) * NS + i] = rho * vy;
      u[(e * NF + 3) * NS + i] = 1.0 / (g - 1.0) * pr + 0.5 * rho * (vx * vx + vy * vy);
      u[(e * NF + 4) * NS + i] = P.gamcons ? rho / (g - 1.0) : 1.0 / (g - 1.0);
    }
  };
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> U01(0.0, 1.0);
  if (ic == "sodtube" && D == 1) {
    // init_dg_sodtube_multifluid (code/src/ic/init_cond.cc:400-424): split on the element's
    // first node at x < 1e-8 (buildLRstates_multifluid, init_cond.cc:351-398)
    const double L[4] = {1.0, 0.0, 1.0, 1.4}, R[4] = {0.125, 0.0, 0.1, 1.6};
    for (int e = 0; e < NE; ++e)
      for (int i = 0; i < NS; ++i) {
        ymark = X(0, e, 0) < 1e-8 ? 1.0 : 0.0;
        set(e, i, X(0, e, 0) < 1e-8 ? L : R);
      }
    return Status();
  }
  if (ic == "tube_noise" && D == 1) {
    // two-fluid shock tube: left (rho 1, p 1, gamma 1.4), right (rho 0.125, p 0.1, gamma 1.6),
    // split at params[0] (default 0.5), seeded uniform noise of amplitude params[1] (default 1e-3)
    // on the nodal density.
    const double xs = prm.size() > 0 ? prm[0] : 0.5, amp = prm.size() > 1 ? prm[1] : 1e-3;
    for (int e = 0; e < NE; ++e) {
      const bool left = X(0, e, 0) < xs - 1e-12;
      for (int i = 0; i < NS; ++i) {
        double s[4] = {left ? 1.0 : 0.125, 0.0, left ? 1.0 : 0.1, left ? 1.4 : 1.6};
        s[0] += amp * (2.0 * U01(rng) - 1.0);
        ymark = left ? 1.0 : 0.0;
        set(e, i, s);
      }
    }
    return Status();
  }
  if (ic == "riemann" && D == 1) {
    // two-fluid Riemann problem split at params[0] (default domain centre): left and right
    // rho, p ~ U[0.1, 2], u ~ U[-1, 1], gamma in {1.4, 1.67}, seeded; element-wise constant
    double xmin = 1e300, xmax = -1e300;
    for (size_t k = 0; k < P.mesh.x.size(); ++k) { xmin = std::min(xmin, P.mesh.x[k]); xmax = std::max(xmax, P.mesh.x[k]); }
    const double xs = prm.size() > 0 ? prm[0] : 0.5 * (xmin + xmax);
    double q[2][4];
    for (int k = 0; k < 2; ++k) {
      q[k][0] = 0.1 + 1.9 * U01(rng);
      q[k][1] = -1.0 + 2.0 * U01(rng);
      q[k][2] = 0.1 + 1.9 * U01(rng);
      q[k][3] = U01(rng) < 0.5 ? 1.4 : 1.67;
    }
    for (int e = 0; e < NE; ++e) {
      double cx = 0;
      for (int k = 0; k < NS; ++k) cx += X(k, e, 0);
      cx /= NS;
      ymark = cx >= xs ? 0.0 : 1.0;
      for (int i = 0; i < NS; ++i) set(e, i, q[cx >= xs ? 1 : 0]);
    }
    return Status();
  }
  if (ic == "sinegam") {
    // init_dg_sinegam_multifluid (code/src/ic/init_cond.cc:551-618): uniform velocity 1 (1D; (1, 1)
    // in 2D) and pressure 1, density 1 + 0.2 sin(4 pi x) and gamma 1.4 + 0.2 sin(2 pi x) (1D), or
    // both perturbations 0.2 sin(2 pi x) sin(2 pi y) (2D): pure advection, periodic on the unit
    // interval / square
    const double rho0 = 1.0, u0 = 1.0, g0 = 1.4, Ag = 0.20, Ar = 0.20, p0 = 1.0;
    for (int e = 0; e < NE; ++e)
      for (int i = 0; i < NS; ++i) {
        const double x = X(i, e, 0);
        if (D == 1) {
          const double sr = Ar * std::sin(4 * M_PI * x), sg = Ag * std::sin(2 * M_PI * x);
          const double s[4] = {rho0 + sr, u0, p0, g0 + sg};
          set(e, i, s);
        } else {
          const double y = X(i, e, 1);
          const double sr = Ar * std::sin(2.0 * M_PI * x) * std::sin(2.0 * M_PI * y);
          const double sg = Ag * std::sin(2.0 * M_PI * x) * std::sin(2.0 * M_PI * y);
          const double s[5] = {rho0 + sr, u0, 1.0, p0, g0 + sg};
          set(e, i, s);
        }
      }
    return Status();
  }
  if (ic == "shock_bubble" && D == 2) {
    // Mach-1.5 shock in air (gamma 1.4, pre-shock rho 1, p 1) at x = params[0] (default 0.2)
    // moving in +x into a circular bubble of radius 0.2 at (0.5, 0.5): gamma 1.67, rho 0.138,
    // in pressure equilibrium; the radius carries a seeded 1% perturbation sum_k a_k cos(k th + ph_k).
    const double xs = prm.size() > 0 ? prm[0] : 0.2;
    const double g = 1.4, M = 1.5, rho1 = 1.0, p1 = 1.0;
    const double a1 = std::sqrt(g * p1 / rho1);
    const double p2 = p1 * (1.0 + 2.0 * g / (g + 1.0) * (M * M - 1.0));
    const double rho2 = rho1 * (g + 1.0) * M * M / ((g - 1.0) * M * M + 2.0);
    const double us = M * a1;
    const double u2 = us * (1.0 - rho1 / rho2);
    double amp[8], ph[8];
    for (int k = 0; k < 8; ++k) { amp[k] = 0.01 * 0.2 * (2.0 * U01(rng) - 1.0) / 8.0 * 2.0; ph[k] = 2.0 * M_PI * U01(rng); }
    for (int e = 0; e < NE; ++e)
      for (int i = 0; i < NS; ++i) {
        const double x = X(i, e, 0), y = X(i, e, 1);
        const double dx = x - 0.5, dy = y - 0.5, th = std::atan2(dy, dx);
        double r = 0.2;
        for (int k = 0; k < 8; ++k) r += amp[k] * std::cos((k + 2) * th + ph[k]);
        double s[5];
        ymark = 0.0;
        if (x < xs) { s[0] = rho2; s[1] = u2; s[2] = 0; s[3] = p2; s[4] = g; }
        else if (dx * dx + dy * dy < r * r) { s[0] = 0.138; s[1] = 0; s[2] = 0; s[3] = p1; s[4] = 1.67; ymark = 1.0; }
        else { s[0] = rho1; s[1] = 0; s[2] = 0; s[3] = p1; s[4] = g; }
        set(e, i, s);
      }
    return Status();
  }
  if (ic == "quadrants" && D == 2) {
    // four-quadrant Riemann problem split at (params[0], params[1]) (default domain centre):
    // per quadrant rho, p ~ U[0.1, 2], u, v ~ U[-1, 1], gamma in {1.4, 1.67}, seeded.
    double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300;
    for (size_t k = 0; k < P.mesh.x.size(); ++k) {
      xmin = std::min(xmin, P.mesh.x[k]); xmax = std::max(xmax, P.mesh.x[k]);
      ymin = std::min(ymin, P.mesh.y[k]); ymax = std::max(ymax, P.mesh.y[k]);
    }
    const double xc = prm.size() > 0 ? prm[0] : 0.5 * (xmin + xmax), yc = prm.size() > 1 ? prm[1] : 0.5 * (ymin + ymax);
    double q[4][5];
    for (int k = 0; k < 4; ++k) {
      q[k][0] = 0.1 + 1.9 * U01(rng);
      q[k][1] = -1.0 + 2.0 * U01(rng);
      q[k][2] = -1.0 + 2.0 * U01(rng);
      q[k][3] = 0.1 + 1.9 * U01(rng);
      q[k][4] = U01(rng) < 0.5 ? 1.4 : 1.67;
    }
    for (int e = 0; e < NE; ++e) {
      // element-wise constant (quadrant of the element centre) so every jump sits on faces
      double cx = 0, cy = 0;
      for (int k = 0; k < 4; ++k) { cx += X(k, e, 0); cy += X(k, e, 1); }
      cx /= 4; cy /= 4;
      const int k = (cx >= xc ? 1 : 0) + (cy >= yc ? 2 : 0);
      ymark = (k == 0 || k == 3) ? 1.0 : 0.0;
      for (int i = 0; i < NS; ++i) set(e, i, q[k]);
    }
    return Status();
  }
  Status s;
  s.code = 1;
  s.msg = "unknown initial condition '" + ic + "' for this dimension";
  return s;
}

// ---------------------------------------------------------------------------------------
// ERROR diagnostic of the reference driver (code/src/main.cc:909-1038, built with ERRR=ERROR):
// both states go to (rho, u, (E - rho u^2/2)/alpha, alpha) on their fields 0..3 (the reference
// applies this 1D formula on the same field indices in 2D as well), the cell integrals of every
// field at the element quadrature points are divided by the width dx of element 0 (its nodes 0
// and 1), and the differences give L1 = sum|E|/N_E, L2 = sqrt(sum E^2/N_E), Linf = max|E| per field.
// ---------------------------------------------------------------------------------------
Status error_norms(const Problem& P, const double* U, const double* Uexact, double* out) {
  const int NS = P.N_s, NF = P.N_F, NE = P.N_E, NG = P.N_G, D = P.D;
  auto prim = [&](const double* src) {
    std::vector<double> V(src, src + (size_t)NE * NF * NS);
    for (int e = 0; e < NE; ++e)
      for (int i = 0; i < NS; ++i) {
        double* f = &V[(size_t)e * NF * NS + i];
        f[1 * NS] = f[1 * NS] / f[0];
        if (P.gamcons) f[3 * NS] = f[3 * NS] / f[0];
        f[2 * NS] = 1.0 / f[3 * NS] * (f[2 * NS] - 0.5 * f[0] * f[1 * NS] * f[1 * NS]);
      }
    return V;
  };
  const std::vector<double> A = prim(U), B = prim(Uexact);
  auto averages = [&](const std::vector<double>& V) {
    std::vector<double> avg((size_t)NE * NF, 0.0);
    for (int e = 0; e < NE; ++e)
      for (int fc = 0; fc < NF; ++fc)
        for (int g = 0; g < NG; ++g) {
          double ug = 0.0;
          for (int i = 0; i < NS; ++i) ug += P.phi[g + (size_t)i * NG] * V[((size_t)e * NF + fc) * NS + i];
          avg[(size_t)e * NF + fc] += ug * P.J[e] * P.qw[g];
        }
    return avg;
  };
  const std::vector<double> a = averages(A), b = averages(B);
  const double dx = P.xyz_nodes[1 + (size_t)(0 * D + 0) * NS] - P.xyz_nodes[0 + (size_t)(0 * D + 0) * NS];
  out[0] = dx;
  for (int fc = 0; fc < NF; ++fc) {
    double e1 = 0.0, e2 = 0.0, ei = 0.0;
    for (int e = 0; e < NE; ++e) {
      const double E = b[(size_t)e * NF + fc] / dx - a[(size_t)e * NF + fc] / dx;
      e1 += std::fabs(E);
      e2 += E * E;
      if (ei < std::fabs(E)) ei = std::fabs(E);
    }
    out[1 + fc] = e1 / (double)NE;
    out[1 + NF + fc] = std::sqrt(e2 / (double)NE);
    out[1 + 2 * NF + fc] = ei;
  }
  return Status();
}

// ---------------------------------------------------------------------------------------
// .pos output / restart (simpleMesh::writeSolution / readSolution, simpleMesh.cc:322-459;
// field formatting of printer_{oned,twod}_multifluid.cu, names of printer.cc:11-74)
// ---------------------------------------------------------------------------------------
static std::vector<std::pair<std::string, std::string>> pos_names(int D, int NY) {
  std::vector<std::pair<std::string, std::string>> n;
  if (D == 1) n = {{"Rho", "rho"}, {"Ux", "ux"}, {"G", "g"}, {"P", "p"}};
  else n = {{"Rho", "rho"}, {"Ux", "ux"}, {"Uy", "uy"}, {"G", "g"}, {"P", "p"}};
  for (int k = 0; k < NY; ++k) n.push_back({"Y" + std::to_string(k), "y" + std::to_string(k)});  // printer.cc:65-71
  return n;
}

Status write_pos(const Problem& P, const double* U, int step, double time, const std::string& dir) {
  const int NS = P.N_s, NF = P.N_F, NE = P.N_E;
  std::vector<double> out((size_t)NS * NE * NF);
  for (int e = 0; e < NE; ++e)
    for (int i = 0; i < NS; ++i) {
      const double rho = U[(e * NF + 0) * NS + i];
      const double ux = U[(e * NF + 1) * NS + i] / rho;
      if (P.D == 1) {
        const double et = U[(e * NF + 2) * NS + i];
        const double g = P.gamcons ? 1 + rho / U[(e * NF + 3) * NS + i] : 1 + 1.0 / U[(e * NF + 3) * NS + i];
        out[(e * NF + 0) * NS + i] = rho;
        out[(e * NF + 1) * NS + i] = ux;
        out[(e * NF + 2) * NS + i] = g;
        out[(e * NF + 3) * NS + i] = (g - 1) * (et - 0.5 * ux * ux * rho);
      } else {
        const double uy = U[(e * NF + 2) * NS + i] / rho;
        const double et = U[(e * NF + 3) * NS + i];
        const double g = P.gamcons ? 1 + rho / U[(e * NF + 4) * NS + i] : 1 + 1.0 / U[(e * NF + 4) * NS + i];
        out[(e * NF + 0) * NS + i] = rho;
        out[(e * NF + 1) * NS + i] = ux;
        out[(e * NF + 2) * NS + i] = uy;
        out[(e * NF + 3) * NS + i] = g;
        out[(e * NF + 4) * NS + i] = (g - 1) * (et - 0.5 * (ux * ux + uy * uy) * rho);
      }
      for (int k = NF - P.N_Y; k < NF; ++k) out[(e * NF + k) * NS + i] = U[(e * NF + k) * NS + i] / rho;
    }
  const auto names = pos_names(P.D, P.N_Y);
  for (int fc = 0; fc < NF; ++fc) {
    char stepstr[32];
    snprintf(stepstr, sizeof stepstr, "%010d", step);
    const std::string fn = dir + "/" + names[fc].second + stepstr + ".pos";
    FILE* f = fopen(fn.c_str(), "w");
    if (!f) { Status s; s.code = 2; s.msg = "cannot write " + fn; return s; }
    fprintf(f, "$MeshFormat\n2.1 0 8\n$EndMeshFormat\n$ElementNodeData\n1\n\"%s\"\n1\n%.20g\n4\n%d\n1\n%d\n0\n",
            names[fc].first.c_str(), time, step, NE);
    for (int e = 0; e < NE; ++e) {
      fprintf(f, "%d %d ", P.elements[e].id, NS);
      for (int i = 0; i < NS; ++i) fprintf(f, "%.20g ", out[(e * NF + fc) * NS + i]);
      fprintf(f, "\n");
    }
    fprintf(f, "$EndElementNodeData\n");
    fclose(f);
  }
  return Status();
}

Status read_pos(const Problem& P, int step, const std::string& dir, double& time, double* U) {
  const int NS = P.N_s, NF = P.N_F, NE = P.N_E;
  std::vector<double> out((size_t)NS * NE * NF);
  const auto names = pos_names(P.D, P.N_Y);
  for (int fc = 0; fc < NF; ++fc) {
    char stepstr[32];
    snprintf(stepstr, sizeof stepstr, "%010d", step);
    const std::string fn = dir + "/" + names[fc].second + stepstr + ".pos";
    std::ifstream in(fn);
    Status s;
    if (!in.is_open()) { s.code = 2; s.msg = "no file named " + fn; return s; }
    std::string line;
    for (int k = 0; k < 7; ++k) std::getline(in, line);
    in >> time; std::getline(in, line);
    std::getline(in, line); std::getline(in, line); std::getline(in, line);
    int fsize = 0, fid = -1;
    in >> fsize; std::getline(in, line);
    if (fsize != NE) { s.code = 2; s.msg = "file has a different number of elements than the mesh"; return s; }
    in >> fid; std::getline(in, line);
    if (fid != 0) { s.code = 2; s.msg = "file has a different partition number"; return s; }
    for (int e = 0; e < NE; ++e) {
      int id = 0, nb = 0;
      in >> id >> nb;
      if (id != P.elements[e].id || nb != NS) { s.code = 2; s.msg = "file has a problem (element id or node count)"; return s; }
      for (int i = 0; i < NS; ++i) in >> out[(e * NF + fc) * NS + i];
      std::getline(in, line);
    }
  }
  for (int e = 0; e < NE; ++e)
    for (int i = 0; i < NS; ++i) {
      const double rho = out[(e * NF + 0) * NS + i], ux = out[(e * NF + 1) * NS + i];
      if (P.D == 1) {
        const double g = out[(e * NF + 2) * NS + i], pr = out[(e * NF + 3) * NS + i];
        U[(e * NF + 0) * NS + i] = rho;
        U[(e * NF + 1) * NS + i] = rho * ux;
        U[(e * NF + 2) * NS + i] = pr / (g - 1) + 0.5 * rho * ux * ux;
        U[(e * NF + 3) * NS + i] = P.gamcons ? rho / (g - 1) : 1.0 / (g - 1);
      } else {
        const double uy = out[(e * NF + 2) * NS + i], g = out[(e * NF + 3) * NS + i], pr = out[(e * NF + 4) * NS + i];
        U[(e * NF + 0) * NS + i] = rho;
        U[(e * NF + 1) * NS + i] = rho * ux;
        U[(e * NF + 2) * NS + i] = rho * uy;
        U[(e * NF + 3) * NS + i] = pr / (g - 1) + 0.5 * rho * (ux * ux + uy * uy);
        U[(e * NF + 4) * NS + i] = P.gamcons ? rho / (g - 1) : 1.0 / (g - 1);
      }
      for (int k = NF - P.N_Y; k < NF; ++k) U[(e * NF + k) * NS + i] = rho * out[(e * NF + k) * NS + i];
    }
  return Status();
}

}  // namespace dgb
