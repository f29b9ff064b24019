// C ABI of the host setup layer (declared in include/dgb.h).
#include <algorithm>
#include <cstring>
#include <string>

#include "../../../include/dgb.h"
#include "host.h"

struct dgb_problem {
  dgb::Problem P;
};

namespace dgb {
thread_local std::string g_last_error;
int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
}  // namespace dgb

using dgb::set_error;

extern "C" const char* dgb_last_error(void) { return dgb::g_last_error.c_str(); }
extern "C" int dgb_abi_version(void) { return DGB_ABI_VERSION; }

static int limiter_code(const std::string& s) {
  // main.cc:167-175
  if (s == "hrl") return 1;
  if (s == "m2l") return 2;
  if (s == "hri") return 3;
  if (s == "m2i") return 4;
  if (s == "prl") return 5;
  if (s == "pri") return 6;
  if (s == "p0i") return 7;
  return 0;
}

extern "C" int dgb_problem_from_deck(const char* deck_path, dgb_problem** out) {
  if (!deck_path || !out) return set_error(DGB_ERR_ARG, "null argument");
  *out = nullptr;
  dgb::Deck d;
  dgb::Status st = dgb::read_deck(deck_path, d);
  if (!st.ok()) return set_error(st.code, st.msg);
  std::string dir = deck_path;
  size_t slash = dir.find_last_of('/');
  dir = slash == std::string::npos ? std::string(".") : dir.substr(0, slash);
  int dim = 0;
  if (d.elem_type == "lin") dim = 1;
  else if (d.elem_type == "qua") dim = 2;
  else return set_error(DGB_ERR_UNSUPPORTED, "element type '" + d.elem_type + "' is outside the device path (lin, qua)");
  auto mo = d.make_options.find("DIMS");
  if (mo != d.make_options.end() && ((mo->second == "ONED") != (dim == 1)))
    return set_error(DGB_ERR_ARG, "#Make options DIMS does not match the element type");
  int flux = DGB_FLUX_ROE;
  mo = d.make_options.find("FLUX");
  if (mo != d.make_options.end()) {
    if (mo->second == "RUS" || mo->second == "LLF") flux = DGB_FLUX_RUSANOV;
    else if (mo->second == "HLL") flux = DGB_FLUX_HLL;
    else if (mo->second == "ROE") flux = DGB_FLUX_ROE;
    else return set_error(DGB_ERR_ARG, "unknown FLUX " + mo->second);
  }
  int n_mass = 0;
  mo = d.make_options.find("MASS");
  if (mo != d.make_options.end()) n_mass = std::atoi(mo->second.c_str());
  bool gamcons = false;
  mo = d.make_options.find("GAMM");
  if (mo != d.make_options.end()) {
    if (mo->second == "GAMCONS") gamcons = true;
    else if (mo->second != "GAMNCON") return set_error(DGB_ERR_ARG, "unknown GAMM " + mo->second);
  }
  if (d.order < 1) return set_error(DGB_ERR_UNSUPPORTED, "order 0 is outside the device path");
  // output times (RK constructor, rk.h:61-84); the intended (int)(Tf/DtOut)+1 count is used
  std::vector<double> outt = d.output_times;
  double tf = d.final_time;
  if (outt.empty() && d.dt_out > 0) {
    int n = (int)(d.final_time / d.dt_out + 1e-9) + 1;
    for (int k = 0; k < n; ++k) outt.push_back(k * d.dt_out);
    tf = outt.back();
  } else if (!outt.empty()) {
    tf = outt.back();
  }
  std::string mpath = d.mesh_file;
  if (!mpath.empty() && mpath[0] != '/') mpath = dir + "/" + mpath;
  dgb::Mesh m;
  st = dgb::read_msh(mpath, m);
  if (!st.ok()) return set_error(st.code, st.msg);
  auto* pr = new dgb_problem();
  st = dgb::build_problem(std::move(m), dim, d.order, d.elem_type, flux, limiter_code(d.limiter), d.cfl,
                          d.thresholds, outt, tf, pr->P, n_mass, gamcons);
  if (!st.ok()) { delete pr; return set_error(st.code, st.msg); }
  pr->P.deck_dir = dir;
  mo = d.make_options.find("ERRR");
  pr->P.error_output = mo != d.make_options.end() && mo->second == "ERROR";
  mo = d.make_options.find("CONS");
  pr->P.cons_output = mo != d.make_options.end() && mo->second == "CONS";
  pr->P.deck_ic = d.ic;
  pr->P.deck_ic_inputs = d.ic_inputs;
  *out = pr;
  return DGB_OK;
}

static dgb::Mesh mesh_from_spec(const dgb_mesh_spec* s) {
  dgb::Mesh m;
  dgb::structured_mesh(s->dim, s->order, s->nx, s->dim == 1 ? 1 : s->ny, s->x0, s->x1, s->y0, s->y1, s->bc, m);
  return m;
}

static int check_spec(const dgb_mesh_spec* s) {
  if (!s) return set_error(DGB_ERR_ARG, "null mesh spec");
  if (s->dim != 1 && s->dim != 2) return set_error(DGB_ERR_ARG, "dim must be 1 or 2");
  if (s->order < 1 || s->order > 4) return set_error(DGB_ERR_ARG, "order must be 1..4");
  if (s->nx < 1 || (s->dim == 2 && s->ny < 1)) return set_error(DGB_ERR_ARG, "element counts must be >= 1");
  if (!(s->x1 > s->x0) || (s->dim == 2 && !(s->y1 > s->y0))) return set_error(DGB_ERR_ARG, "empty domain");
  for (int k = 0; k < (s->dim == 1 ? 2 : 4); ++k)
    if (s->bc[k] < 1 || s->bc[k] > 4) return set_error(DGB_ERR_ARG, "boundary tags must be 1..4");
  return DGB_OK;
}

extern "C" int dgb_problem_structured(const dgb_mesh_spec* mesh, const dgb_options* opt, dgb_problem** out) {
  if (!opt || !out) return set_error(DGB_ERR_ARG, "null argument");
  *out = nullptr;
  int rc = check_spec(mesh);
  if (rc) return rc;
  if (opt->flux < 0 || opt->flux > 2) return set_error(DGB_ERR_ARG, "bad flux");
  if (opt->limiter < 0 || opt->limiter > 7) return set_error(DGB_ERR_ARG, "bad limiter");
  if (opt->n_mass < 0 || opt->n_mass > 10) return set_error(DGB_ERR_ARG, "n_mass must be 0..10");
  if (opt->gamma_model != DGB_GAMNCON && opt->gamma_model != DGB_GAMCONS) return set_error(DGB_ERR_ARG, "bad gamma model");
  std::vector<double> th(opt->thresholds, opt->thresholds + std::max(0, std::min(3, opt->n_thresholds)));
  auto* pr = new dgb_problem();
  dgb::Status st = dgb::build_problem(mesh_from_spec(mesh), mesh->dim, mesh->order, mesh->dim == 1 ? "lin" : "qua",
                                      opt->flux, opt->limiter, opt->cfl, th, {}, 0.0, pr->P, opt->n_mass,
                                      opt->gamma_model == DGB_GAMCONS);
  if (!st.ok()) { delete pr; return set_error(st.code, st.msg); }
  *out = pr;
  return DGB_OK;
}

extern "C" int dgb_mesh_write_msh(const dgb_mesh_spec* mesh, const char* path) {
  int rc = check_spec(mesh);
  if (rc) return rc;
  if (!path) return set_error(DGB_ERR_ARG, "null path");
  dgb::Status st = dgb::write_msh(path, mesh_from_spec(mesh));
  return st.ok() ? DGB_OK : set_error(st.code, st.msg);
}

extern "C" void dgb_problem_destroy(dgb_problem* p) { delete p; }

extern "C" int dgb_problem_info(const dgb_problem* p, dgb_info* o) {
  if (!p || !o) return set_error(DGB_ERR_ARG, "null argument");
  const dgb::Problem& P = p->P;
  std::memset(o, 0, sizeof(*o));
  o->dim = P.D; o->order = P.p; o->n_fields = P.N_F;
  o->n_elem = P.N_E; o->n_s = P.N_s; o->n_g = P.N_G;
  o->n_ifaces = P.M_T; o->m_s = P.M_s; o->m_g = P.M_G; o->n_n = P.N_N;
  o->n_reflective = (int)std::count_if(P.ifaces.begin(), P.ifaces.end(), [](const dgb::Interface& I) { return I.phys == 3; });
  o->cartesian = P.cartesian ? 1 : 0;
  o->gpu_supported = P.gpu_ok ? 1 : 0;
  o->flux = P.flux; o->limiter = P.limiter;
  o->nx = P.nx; o->ny = P.ny;
  o->cfl = P.cfl; o->dx_min = P.dx_min; o->cfl_scaled = P.cfl_scaled;
  o->final_time = P.final_time;
  o->n_output_times = (int)P.output_times.size();
  o->error_output = P.error_output ? 1 : 0;
  o->cons_output = P.cons_output ? 1 : 0;
  o->gamma_model = P.gamcons ? DGB_GAMCONS : DGB_GAMNCON;
  return DGB_OK;
}

template <typename T>
static int export_vec(const std::vector<T>& v, void* dst, size_t nbytes, size_t* size_out) {
  if (size_out) { *size_out = v.size() * sizeof(T); return DGB_OK; }
  if (nbytes != v.size() * sizeof(T)) return set_error(DGB_ERR_ARG, "size mismatch for array export");
  if (!v.empty()) std::memcpy(dst, v.data(), nbytes);
  return DGB_OK;
}

static int array_op(const dgb_problem* p, const char* name, void* dst, size_t nbytes, size_t* size_out) {
  if (!p || !name) return set_error(DGB_ERR_ARG, "null argument");
  const dgb::Problem& P = p->P;
  const std::string n = name;
  if (n == "phi") return export_vec(P.phi, dst, nbytes, size_out);
  if (n == "dphi") return export_vec(P.dphi, dst, nbytes, size_out);
  if (n == "phi_w") return export_vec(P.phi_w, dst, nbytes, size_out);
  if (n == "dphi_w") return export_vec(P.dphi_w, dst, nbytes, size_out);
  if (n == "psi") return export_vec(P.psi, dst, nbytes, size_out);
  if (n == "psi_w") return export_vec(P.psi_w, dst, nbytes, size_out);
  if (n == "weight") return export_vec(P.qw, dst, nbytes, size_out);
  if (n == "J") return export_vec(P.J, dst, nbytes, size_out);
  if (n == "invJac") return export_vec(P.invJac, dst, nbytes, size_out);
  if (n == "JF") return export_vec(P.JF, dst, nbytes, size_out);
  if (n == "normals") return export_vec(P.normals, dst, nbytes, size_out);
  if (n == "Minv") return export_vec(P.Minv, dst, nbytes, size_out);
  if (n == "map") return export_vec(P.map, dst, nbytes, size_out);
  if (n == "invmap") return export_vec(P.invmap, dst, nbytes, size_out);
  if (n == "neighbors") return export_vec(P.neighbors, dst, nbytes, size_out);
  if (n == "boundaryMap") return export_vec(P.boundary_map, dst, nbytes, size_out);
  if (n == "Lag2Mono") return export_vec(P.Lag2Mono, dst, nbytes, size_out);
  if (n == "Mono2Lag") return export_vec(P.Mono2Lag, dst, nbytes, size_out);
  if (n == "Lag2MonoX") return export_vec(P.Lag2MonoX, dst, nbytes, size_out);
  if (n == "MonoX2MonoY") return export_vec(P.MonoX2MonoY, dst, nbytes, size_out);
  if (n == "MonoY2Lag") return export_vec(P.MonoY2Lag, dst, nbytes, size_out);
  if (n == "MonoX2Lag") return export_vec(P.MonoX2Lag, dst, nbytes, size_out);
  if (n == "Lag2MonoY") return export_vec(P.Lag2MonoY, dst, nbytes, size_out);
  if (n == "xyz_nodes") return export_vec(P.xyz_nodes, dst, nbytes, size_out);
  if (n == "output_times") return export_vec(P.output_times, dst, nbytes, size_out);
  if (n == "tensor_perm") return export_vec(P.tensor_perm, dst, nbytes, size_out);
  return set_error(DGB_ERR_ARG, "unknown array name " + n);
}

extern "C" int dgb_problem_array_size(const dgb_problem* p, const char* name, size_t* nbytes) {
  if (!nbytes) return set_error(DGB_ERR_ARG, "null argument");
  return array_op(p, name, nullptr, 0, nbytes);
}

extern "C" int dgb_problem_get_array(const dgb_problem* p, const char* name, void* dst, size_t nbytes) {
  if (!dst && nbytes) return set_error(DGB_ERR_ARG, "null destination");
  return array_op(p, name, dst, nbytes, nullptr);
}

extern "C" int dgb_problem_init_state(const dgb_problem* p, const char* ic, const double* params, int nparams,
                                      uint64_t seed, double* U) {
  if (!p || !U || (nparams > 0 && !params)) return set_error(DGB_ERR_ARG, "null argument");
  std::vector<double> prm(params, params + std::max(0, nparams));
  if (!ic) {  // the deck's own initial condition and inputs
    if (p->P.deck_ic.empty()) return set_error(DGB_ERR_ARG, "the problem has no deck initial condition");
    if (nparams == 0) prm = p->P.deck_ic_inputs;
  }
  dgb::Status st = dgb::init_state(p->P, ic ? std::string(ic) : p->P.deck_ic, prm, seed, U);
  return st.ok() ? DGB_OK : set_error(st.code, st.msg);
}

extern "C" int dgb_write_pos(const dgb_problem* p, const double* U, int step, double time, const char* dir) {
  if (!p || !U || !dir) return set_error(DGB_ERR_ARG, "null argument");
  dgb::Status st = dgb::write_pos(p->P, U, step, time, dir);
  return st.ok() ? DGB_OK : set_error(st.code, st.msg);
}

extern "C" int dgb_read_pos(const dgb_problem* p, int step, const char* dir, double* time, double* U) {
  if (!p || !U || !dir || !time) return set_error(DGB_ERR_ARG, "null argument");
  dgb::Status st = dgb::read_pos(p->P, step, dir, *time, U);
  return st.ok() ? DGB_OK : set_error(st.code, st.msg);
}

// access for the device layer
const dgb::Problem& dgb_problem_ref(const dgb_problem* p) { return p->P; }

extern "C" int dgb_problem_error_norms(const dgb_problem* p, const double* U, const double* U_exact, double* out) {
  if (!p || !U || !U_exact || !out) return set_error(DGB_ERR_ARG, "null argument");
  dgb::Status st = dgb::error_norms(p->P, U, U_exact, out);
  if (!st.ok()) return set_error(st.code, st.msg);
  return DGB_OK;
}
