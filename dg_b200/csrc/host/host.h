// Host-side setup of the DG problem (C++17, no GPU).  Builds every array the reference
// driver builds before time integration (code/src/main.cc:273-860), in the reference's own
// layouts, plus the compact tensor-product description the device kernels use.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace dgb {

// Gmsh element type codes (code/src/gmsh/GmshDefines.h:65-148).
enum GmshType { MSH_LIN_2 = 1, MSH_QUA_4 = 3, MSH_LIN_3 = 8, MSH_QUA_9 = 10, MSH_PNT = 15,
                MSH_LIN_4 = 26, MSH_QUA_16 = 36, MSH_LIN_5 = 27, MSH_QUA_25 = 37 };

struct Status {
  int code = 0;
  std::string msg;
  bool ok() const { return code == 0; }
};

struct Element {
  int id = 0;         // Gmsh element id
  int type = 0;       // Gmsh element type
  int ptag = 0;       // physical tag
  int partition = 0;  // 0-based partition
  std::vector<int> nodes;  // 0-based node indices
};

struct Mesh {
  std::vector<double> x, y, z;                 // node coordinates
  std::map<int, std::vector<Element>> by_type; // elements of partition 0, file order
};

struct Interface {
  int phys = 0;          // physical tag (0 interior)
  int el[2] = {-1, -1};  // element indices (into the element list of the element type)
  int cl[2] = {-1, -1};  // closure ids
};

struct Deck {
  std::string time_integration;
  double dt_out = -1.0;
  std::vector<double> output_times;
  double final_time = 0.0;
  double cfl = 0.0;
  int order = 1;
  std::string mesh_file, elem_type;
  std::string limiter;
  std::string ic;
  std::vector<double> ic_inputs, thresholds, particles;
  int restart_step = 0;
  std::map<std::string, std::string> make_options;  // "#Make options" KEY=VALUE pairs
};

// Everything that main.cc computes before RK_integration, in reference layouts
// (fullMatrix is column-major; pointer layouts as in main.cc:766-820).
struct Problem {
  // configuration
  int D = 1, p = 1, N_F = 4;
  int N_Y = 0;                        // passive mass fractions rho*Y_k, fields D+3 .. N_F-1
  int flux = 2, limiter = 0;
  bool error_output = false;          // deck "#Make options" ERRR=ERROR: error.dat after the run
  bool cons_output = false;           // deck "#Make options" CONS=CONS: conservation.dat at outputs
  bool gamcons = false;               // GAMCONS gamma model: field D+2 holds rho/(gamma-1)
  double cfl = -1.0;
  std::vector<double> thresholds;
  std::vector<double> output_times;
  double final_time = 0.0;
  std::string deck_dir;
  std::string deck_ic;                // "#initial condition" of the deck ("" for built problems)
  std::vector<double> deck_ic_inputs; // "#ic inputs"
  // sizes
  int N_E = 0, N_s = 0, N_G = 0, M_T = 0, M_s = 0, M_G = 0, N_N = 0, M_B = 0;
  int elem_type = 0, face_type = 0;
  bool cartesian = false;
  // mesh
  Mesh mesh;
  std::vector<Element> elements;
  std::vector<Interface> ifaces;
  std::vector<std::vector<int>> closures;
  std::vector<double> ref_nodes;  // reference-element node coordinates (N_s x 2, row-major)
  // basis / quadrature (column-major fullMatrix layouts)
  std::vector<double> qpts, qw;         // element quadrature points (N_G x 2 row-major), weights
  std::vector<double> fqpts, fqw;       // face quadrature
  std::vector<double> phi, dphi, phi_w, dphi_w, psi, dpsi, psi_w;
  // geometry
  std::vector<double> xyz_nodes;  // XYZNodes(i, e*D+alpha) column-major N_s x (N_E*D)
  std::vector<double> J, invJac, JF, normals;
  std::vector<double> Minv;
  std::vector<int> map, invmap, neighbors, boundary_map;
  double dx_min = 0.0, cfl_scaled = 0.0;
  // limiter transforms (N_s x N_s column-major)
  std::vector<double> Lag2Mono, Mono2Lag, Lag2MonoX, MonoX2MonoY, MonoY2Lag, MonoX2Lag, Lag2MonoY;
  // ---- compact description for the device path (tensor-product, Cartesian, uniform) ----
  bool gpu_ok = false;
  std::string gpu_reason;
  int nx = 0, ny = 0;                 // structured extents when the mesh is a full grid
  std::vector<int> tensor_perm;       // tensor node t -> Gmsh node index
  std::vector<int> nbr;               // [face k][e], k = L,R(,D,U); boundary codes < 0
  double hx = 0.0, hy = 0.0;          // uniform element sizes
  // Structured element order: 1D elements in a chain (neighbours e -+ 1), or a row-major nx x ny
  // 2D grid (e -+ 1, e -+ nx); and, per side (L, R, D, U), the one rule its boundary elements share:
  // a boundary code (< 0), kSideWrap (periodic: the element on the opposite side) or kSideMixed.
  // Found once when the problem is set up.
  static constexpr int kSideWrap = 1, kSideMixed = 2;
  bool structured = false;
  int side_rule[4] = {kSideMixed, kSideMixed, kSideMixed, kSideMixed};
};

// deck.cc
Status read_deck(const std::string& path, Deck& d);
// mesh.cc
Status read_msh(const std::string& path, Mesh& m);
Status write_msh(const std::string& path, const Mesh& m);
void structured_mesh(int dim, int order, int nx, int ny, double x0, double x1, double y0, double y1,
                     const int bc[4], Mesh& m);
// basis.cc
std::vector<double> line_nodes(int order);              // LIN_{p+1} node order: -1, 1, interior
std::vector<double> quad_nodes(int order);              // QUA_{(p+1)^2} Gmsh node order (x,y pairs)
std::vector<std::vector<int>> closures_for(int dim, int order);
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w);
double lagrange1d(const std::vector<double>& nodes, int i, double x);
double dlagrange1d(const std::vector<double>& nodes, int i, double x);
bool invert(std::vector<double>& A, int n);  // column-major in-place inverse (partial pivoting LU)
// setup.cc
void classify_grid(Problem& P);  // fills Problem::structured and side_rule (setup.cc)
Status build_problem(Mesh&& mesh, int dim, int order, const std::string& elem_kind, int flux, int limiter,
                     double cfl, const std::vector<double>& thresholds, const std::vector<double>& out_times,
                     double final_time, Problem& P, int n_mass = 0, bool gamcons = false);
Status init_state(const Problem& P, const std::string& ic, const std::vector<double>& params, uint64_t seed,
                  double* U);
Status write_pos(const Problem& P, const double* U, int step, double time, const std::string& dir);
// the ERROR diagnostic of the reference driver: [dx, L1(N_F), L2(N_F), Linf(N_F)]
Status error_norms(const Problem& P, const double* U, const double* Uexact, double* out);
Status read_pos(const Problem& P, int step, const std::string& dir, double& time, double* U);

}  // namespace dgb
