// Gmsh 2.2 ASCII mesh I/O and an in-memory structured mesh generator.
//
// Reader semantics follow simpleMesh::load (code/src/mesh/simpleMesh.cc:141-204): node ids are
// made 0-based, element tags are (physical, elementary, ..., partition at tag index 3), and
// elements are kept per Gmsh type in file order.  Only partition 1 is accepted: the device
// path is single-GPU and has no ghost exchange (the reference exits when a partition exceeds
// the process count, simpleMesh.cc:183).
#include <cmath>
#include <cstdio>
#include <fstream>
#include <algorithm>
#include <iomanip>
#include <sstream>

#include "host.h"

namespace dgb {

static int lin_type(int p) { return p == 1 ? MSH_LIN_2 : p == 2 ? MSH_LIN_3 : p == 3 ? MSH_LIN_4 : MSH_LIN_5; }
static int qua_type(int p) { return p == 1 ? MSH_QUA_4 : p == 2 ? MSH_QUA_9 : p == 3 ? MSH_QUA_16 : MSH_QUA_25; }

Status read_msh(const std::string& path, Mesh& m) {
  Status st;
  std::ifstream in(path);
  if (!in.is_open()) { st.code = 2; st.msg = "cannot open mesh file " + path; return st; }
  std::string line;
  // skip to $Nodes (the reference skips the 3-line $MeshFormat block)
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line == "$Nodes") break;
  }
  if (line != "$Nodes") { st.code = 2; st.msg = "mesh has no $Nodes section: " + path; return st; }
  long nn = 0;
  if (!(in >> nn) || nn <= 0) { st.code = 2; st.msg = "bad node count"; return st; }
  m.x.assign(nn, 0.0); m.y.assign(nn, 0.0); m.z.assign(nn, 0.0);
  std::vector<long> ids(nn);
  std::map<long, long> remap;
  bool contiguous = true;
  for (long i = 0; i < nn; ++i) {
    long id;
    if (!(in >> id >> m.x[i] >> m.y[i] >> m.z[i])) { st.code = 2; st.msg = "bad node line"; return st; }
    ids[i] = id;
    if (id != i + 1) contiguous = false;
  }
  if (!contiguous)
    for (long i = 0; i < nn; ++i) remap[ids[i]] = i;
  std::getline(in, line);
  std::getline(in, line);
  if (!line.empty() && line.back() == '\r') line.pop_back();
  if (line != "$EndNodes") { st.code = 2; st.msg = "missing $EndNodes"; return st; }
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line == "$Elements") break;
  }
  if (line != "$Elements") { st.code = 2; st.msg = "mesh has no $Elements section"; return st; }
  long ne = 0;
  if (!(in >> ne) || ne < 0) { st.code = 2; st.msg = "bad element count"; return st; }
  std::getline(in, line);
  for (long k = 0; k < ne; ++k) {
    if (!std::getline(in, line)) { st.code = 2; st.msg = "truncated $Elements section"; return st; }
    std::istringstream sl(line);
    Element el;
    int ntags = 0;
    if (!(sl >> el.id >> el.type >> ntags)) { st.code = 2; st.msg = "bad element line: " + line; return st; }
    int partition = 1;
    for (int j = 0; j < ntags; ++j) {
      int tag = 0;
      sl >> tag;
      if (j == 0) el.ptag = tag;
      else if (j == 3) partition = tag;
    }
    long nid;
    while (sl >> nid) el.nodes.push_back(contiguous ? (int)(nid - 1) : (int)remap[nid]);
    if (partition != 1) {
      st.code = 4;
      st.msg = "mesh partition " + std::to_string(partition) + " found: the device path runs one partition";
      return st;
    }
    el.partition = 0;
    m.by_type[el.type].push_back(std::move(el));
  }
  std::getline(in, line);
  if (!line.empty() && line.back() == '\r') line.pop_back();
  if (line != "$EndElements") { st.code = 2; st.msg = "missing $EndElements"; return st; }
  return st;
}

Status write_msh(const std::string& path, const Mesh& m) {
  Status st;
  FILE* f = fopen(path.c_str(), "w");
  if (!f) { st.code = 2; st.msg = "cannot write " + path; return st; }
  fprintf(f, "$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%zu\n", m.x.size());
  for (size_t i = 0; i < m.x.size(); ++i) fprintf(f, "%zu %.17g %.17g %.17g\n", i + 1, m.x[i], m.y[i], m.z[i]);
  size_t ne = 0;
  for (auto& kv : m.by_type) ne += kv.second.size();
  fprintf(f, "$EndNodes\n$Elements\n%zu\n", ne);
  // lower-dimensional (boundary) elements first, as gmsh writes them
  std::vector<const Element*> all;
  for (auto& kv : m.by_type) for (auto& e : kv.second) all.push_back(&e);
  std::sort(all.begin(), all.end(), [](const Element* a, const Element* b) { return a->id < b->id; });
  for (const Element* e : all) {
    fprintf(f, "%d %d 2 %d %d", e->id, e->type, e->ptag, e->ptag);
    for (int n : e->nodes) fprintf(f, " %d", n + 1);
    fprintf(f, "\n");
  }
  fprintf(f, "$EndElements\n");
  fclose(f);
  return st;
}

// Structured mesh: a (p*nx+1) x (p*ny+1) lattice of nodes, elements row-major (x fastest),
// element nodes in Gmsh order; boundary elements first (bottom, right, top, left in 2D;
// left, right points in 1D) with the physical tags bc[].
void structured_mesh(int dim, int p, int nx, int ny, double x0, double x1, double y0, double y1,
                     const int bc[4], Mesh& m) {
  m = Mesh();
  int id = 1;
  if (dim == 1) {
    const long N = (long)p * nx + 1;
    m.x.resize(N); m.y.assign(N, 0.0); m.z.assign(N, 0.0);
    for (long i = 0; i < N; ++i) m.x[i] = x0 + (x1 - x0) * (double)i / (double)(N - 1);
    m.x[N - 1] = x1;
    Element l; l.id = id++; l.type = MSH_PNT; l.ptag = bc[0]; l.nodes = {0};
    Element r; r.id = id++; r.type = MSH_PNT; r.ptag = bc[1]; r.nodes = {(int)(N - 1)};
    m.by_type[MSH_PNT] = {l, r};
    auto& els = m.by_type[lin_type(p)];
    els.reserve(nx);
    for (int e = 0; e < nx; ++e) {
      Element el; el.id = id++; el.type = lin_type(p); el.ptag = 100;
      el.nodes.push_back(p * e);
      el.nodes.push_back(p * e + p);
      for (int k = 1; k < p; ++k) el.nodes.push_back(p * e + k);
      els.push_back(std::move(el));
    }
    return;
  }
  const long NX = (long)p * nx + 1, NY = (long)p * ny + 1;
  m.x.resize(NX * NY); m.y.resize(NX * NY); m.z.assign(NX * NY, 0.0);
  for (long j = 0; j < NY; ++j)
    for (long i = 0; i < NX; ++i) {
      m.x[j * NX + i] = (i == NX - 1) ? x1 : x0 + (x1 - x0) * (double)i / (double)(NX - 1);
      m.y[j * NX + i] = (j == NY - 1) ? y1 : y0 + (y1 - y0) * (double)j / (double)(NY - 1);
    }
  auto nid = [&](long i, long j) { return (int)(j * NX + i); };
  auto lin = [&](std::vector<int> idx) {  // ends first, then interior in order
    std::vector<int> o = {idx.front(), idx.back()};
    for (size_t k = 1; k + 1 < idx.size(); ++k) o.push_back(idx[k]);
    return o;
  };
  auto& bl = m.by_type[lin_type(p)];
  auto addb = [&](int tag, std::vector<int> idx) {
    Element e; e.id = id++; e.type = lin_type(p); e.ptag = tag; e.nodes = lin(idx); bl.push_back(std::move(e));
  };
  for (int i = 0; i < nx; ++i) { std::vector<int> v; for (int k = 0; k <= p; ++k) v.push_back(nid(p * i + k, 0)); addb(bc[0], v); }
  for (int j = 0; j < ny; ++j) { std::vector<int> v; for (int k = 0; k <= p; ++k) v.push_back(nid(NX - 1, p * j + k)); addb(bc[1], v); }
  for (int i = 0; i < nx; ++i) { std::vector<int> v; for (int k = 0; k <= p; ++k) v.push_back(nid(p * i + k, NY - 1)); addb(bc[2], v); }
  for (int j = 0; j < ny; ++j) { std::vector<int> v; for (int k = 0; k <= p; ++k) v.push_back(nid(0, p * j + k)); addb(bc[3], v); }
  const std::vector<double> loc = quad_nodes(p);
  const int ns = (int)loc.size() / 2;
  std::vector<int> di(ns), dj(ns);
  for (int k = 0; k < ns; ++k) {
    di[k] = (int)std::lround((loc[2 * k] + 1.0) * p / 2.0);
    dj[k] = (int)std::lround((loc[2 * k + 1] + 1.0) * p / 2.0);
  }
  auto& els = m.by_type[qua_type(p)];
  els.reserve((size_t)nx * ny);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      Element el; el.id = id++; el.type = qua_type(p); el.ptag = 100;
      el.nodes.resize(ns);
      for (int k = 0; k < ns; ++k) el.nodes[k] = nid((long)p * i + di[k], (long)p * j + dj[k]);
      els.push_back(std::move(el));
    }
}

}  // namespace dgb
