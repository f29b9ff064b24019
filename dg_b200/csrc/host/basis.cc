// Nodal Lagrange bases, Gauss-Legendre quadrature, closures and a small dense inverse.
//
// Conventions follow the reference's Gmsh-derived basis code:
//   * 1D nodes ordered -1, +1, then the interior equispaced nodes
//     (generate1DPoints, code/src/polynomials/polynomialBasis.cc:20-31);
//   * quadrilateral nodes ordered corners, edge nodes edge by edge, then the interior nodes
//     recursively (gmshGeneratePointsQuad, polynomialBasis.cc:713-751); for p = 2 the single
//     interior node is the centre;
//   * edge closures {j, j+1, edge-interior nodes} and their reversals at j + 4
//     (generate2dEdgeClosure, polynomialBasis.cc:911-926); vertex closures in 1D
//     (generate1dVertexClosure, :928-934).
// The reference evaluates its Lagrange functions through an inverted monomial Vandermonde
// matrix (polynomialBasis.cc:753-778); the same functions are evaluated here in product form,
// which agrees with it to rounding.
#include <cmath>
#include <utility>

#include "host.h"

namespace dgb {

std::vector<double> line_nodes(int order) {
  std::vector<double> n(order + 1, 0.0);
  if (order > 0) {
    n[0] = -1.0;
    n[1] = 1.0;
    const double dd = 2.0 / order;
    for (int i = 2; i < order + 1; ++i) n[i] = -1.0 + dd * (i - 1);
  }
  return n;
}

static void quad_nodes_rec(int order, std::vector<double>& out) {
  if (order == 0) {
    out.push_back(0.0);
    out.push_back(0.0);
    return;
  }
  const double c[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
  std::vector<double> pts;
  for (auto& v : c) { pts.push_back(v[0]); pts.push_back(v[1]); }
  if (order > 1) {
    const int edges[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
    for (auto& e : edges) {
      for (int i = 1; i < order; ++i) {
        pts.push_back(pts[2 * e[0]] + i * (pts[2 * e[1]] - pts[2 * e[0]]) / order);
        pts.push_back(pts[2 * e[0] + 1] + i * (pts[2 * e[1] + 1] - pts[2 * e[0] + 1]) / order);
      }
    }
    std::vector<double> inner;
    quad_nodes_rec(order - 2, inner);
    const double s = 1.0 - 2.0 / order;
    for (double v : inner) pts.push_back(v * s);
  }
  out.insert(out.end(), pts.begin(), pts.end());
}

std::vector<double> quad_nodes(int order) {
  std::vector<double> out;
  quad_nodes_rec(order, out);
  return out;
}

std::vector<std::vector<int>> closures_for(int dim, int order) {
  std::vector<std::vector<int>> cl;
  if (dim == 1) {
    cl = {{0}, {1}};
  } else {
    const int nNod = 4;
    cl.assign(2 * nNod, {});
    for (int j = 0; j < nNod; ++j) {
      cl[j].push_back(j);
      cl[j].push_back((j + 1) % nNod);
      cl[nNod + j].push_back((j + 1) % nNod);
      cl[nNod + j].push_back(j);
      for (int i = 0; i < order - 1; ++i) {
        cl[j].push_back(nNod + (order - 1) * j + i);
        cl[nNod + j].push_back(nNod + (order - 1) * (j + 1) - i - 1);
      }
    }
  }
  return cl;
}

// Gauss-Legendre nodes (ascending) and weights by Newton iteration on P_n.
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
    double dp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = pk;
      }
      if (n == 1) { p1 = z; p0 = 1.0; }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-17) break;
    }
    // final derivative at the converged root
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= n; ++k) {
      double pk = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
      p0 = p1;
      p1 = pk;
    }
    if (n == 1) { p1 = z; p0 = 1.0; }
    dp = n * (z * p1 - p0) / (z * z - 1.0);
    x[n - 1 - i] = z;
    w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
  if (n % 2 == 1) x[n / 2] = 0.0;
  for (int i = 0; i < n / 2; ++i) {  // exact symmetry
    double a = 0.5 * (std::fabs(x[i]) + std::fabs(x[n - 1 - i]));
    double b = 0.5 * (w[i] + w[n - 1 - i]);
    x[i] = -a; x[n - 1 - i] = a;
    w[i] = b; w[n - 1 - i] = b;
  }
}

double lagrange1d(const std::vector<double>& nodes, int i, double x) {
  double v = 1.0;
  for (size_t m = 0; m < nodes.size(); ++m)
    if ((int)m != i) v *= (x - nodes[m]) / (nodes[i] - nodes[m]);
  return v;
}

double dlagrange1d(const std::vector<double>& nodes, int i, double x) {
  double s = 0.0;
  for (size_t m = 0; m < nodes.size(); ++m) {
    if ((int)m == i) continue;
    double t = 1.0 / (nodes[i] - nodes[m]);
    for (size_t k = 0; k < nodes.size(); ++k)
      if ((int)k != i && k != m) t *= (x - nodes[k]) / (nodes[i] - nodes[k]);
    s += t;
  }
  return s;
}

// In-place inverse of a column-major n x n matrix by LU with partial pivoting
// (same role as fullMatrix<double>::invert via dgetrf/dgetri, code/src/matrix/fullMatrix.cc:432).
bool invert(std::vector<double>& A, int n) {
  std::vector<double> LU(A);
  std::vector<int> piv(n);
  auto at = [&](int r, int c) -> double& { return LU[r + (size_t)c * n]; };
  for (int k = 0; k < n; ++k) {
    int pr = k;
    double best = std::fabs(at(k, k));
    for (int r = k + 1; r < n; ++r)
      if (std::fabs(at(r, k)) > best) { best = std::fabs(at(r, k)); pr = r; }
    if (best == 0.0) return false;
    piv[k] = pr;
    if (pr != k)
      for (int c = 0; c < n; ++c) std::swap(at(k, c), at(pr, c));
    for (int r = k + 1; r < n; ++r) {
      at(r, k) /= at(k, k);
      for (int c = k + 1; c < n; ++c) at(r, c) -= at(r, k) * at(k, c);
    }
  }
  // solve for each column of the identity (with row permutation)
  std::vector<double> inv((size_t)n * n, 0.0);
  for (int col = 0; col < n; ++col) {
    std::vector<double> b(n, 0.0);
    b[col] = 1.0;
    for (int k = 0; k < n; ++k) std::swap(b[k], b[piv[k]]);
    for (int r = 0; r < n; ++r)
      for (int c = 0; c < r; ++c) b[r] -= at(r, c) * b[c];
    for (int r = n - 1; r >= 0; --r) {
      for (int c = r + 1; c < n; ++c) b[r] -= at(r, c) * b[c];
      b[r] /= at(r, r);
    }
    for (int r = 0; r < n; ++r) inv[r + (size_t)col * n] = b[r];
  }
  A.swap(inv);
  return true;
}

}  // namespace dgb
