// dgbexec: runs a reference input deck on the GPU through the C ABI -- the B200 counterpart of the
// reference's executable (code/src/main.cc) and its time loop RK::RK_integration
// (code/src/time_integration/rk.cc:11-247):
//   * deck, Gmsh mesh and the deck's initial condition (dgb_problem_from_deck, init_state(NULL));
//   * CFL >= 0: the initial condition is written as output step 0 and then limited; every step
//     takes the CFL step, clipped to land on the next output time (that step is then written) and
//     on the final time (rk.cc:134-149, 207-228);
//   * CFL < 0: a fixed step of output_times[1] - output_times[0], clipped to the final time, and
//     no output (rk.cc:136-139);
//   * output in the reference's .pos format (one file per field and output step) in --out;
//   * with "#Make options" ERRR=ERROR, error.dat (main.cc:909-1038) in --out after the run;
//   * with "#Make options" CONS=CONS, one line of conservation.dat in --out (appended, as the
//     reference opens it, dg_solver.h:238-240) after the initial limiting and at every output
//     time: the time and the domain integral of each field (DG_SOLVER::conservation,
//     dg_solver.h:367-389; rk.cc:120-121, 228-229).
// A NaN or too small time step ends the run with exit status 1 and the reference's message.
//
// usage: dgbexec [-d deck.inp] [--out DIR] [--scheme rk4|ssprk3] [--form fp64|mixed] [--device N]
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "dgb.h"

namespace {

int fail(const char* what) {
  std::fprintf(stderr, "dgbexec: %s: %s\n", what, dgb_last_error());
  return 2;
}

// one line of conservation.dat: "%20.16E\t" for the time and for each field total
int write_conservation(dgb_ctx* ctx, int nf, double T, const std::string& dir) {
  std::vector<double> tot(nf);
  if (dgb_conservation(ctx, tot.data())) return fail("conservation");
  const std::string fn = dir + "/conservation.dat";
  FILE* f = std::fopen(fn.c_str(), "a");
  if (!f) { std::fprintf(stderr, "dgbexec: cannot write %s\n", fn.c_str()); return 2; }
  std::fprintf(f, "%20.16E\t", T);
  for (int k = 0; k < nf; ++k) std::fprintf(f, "%20.16E\t", tot[k]);
  std::fprintf(f, "\n");
  std::fclose(f);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  std::string deck = "deck.inp", out = ".";
  int scheme = DGB_RK4, form = DGB_FORM_FP64, device = 0;
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto next = [&]() -> std::string {
      if (i + 1 >= argc) { std::fprintf(stderr, "dgbexec: %s needs a value\n", a.c_str()); std::exit(2); }
      return argv[++i];
    };
    if (a == "-d" || a == "--deck") deck = next();
    else if (a == "--out") out = next();
    else if (a == "--scheme") scheme = next() == "ssprk3" ? DGB_SSPRK3 : DGB_RK4;
    else if (a == "--form") form = next() == "mixed" ? DGB_FORM_MIXED : DGB_FORM_FP64;
    else if (a == "--device") device = std::atoi(next().c_str());
    else {
      std::fprintf(stderr, "usage: dgbexec [-d deck.inp] [--out DIR] [--scheme rk4|ssprk3] [--form fp64|mixed] "
                           "[--device N]\n");
      return 2;
    }
  }
  dgb_problem* prob = nullptr;
  if (dgb_problem_from_deck(deck.c_str(), &prob)) return fail("deck");
  dgb_info info;
  dgb_problem_info(prob, &info);
  size_t nb = 0;
  std::vector<double> times;
  if (dgb_problem_array_size(prob, "output_times", &nb) == DGB_OK && nb) {
    times.resize(nb / sizeof(double));
    dgb_problem_get_array(prob, "output_times", times.data(), nb);
  }
  if (times.size() < 2) {
    std::fprintf(stderr, "dgbexec: the deck needs at least two output times\n");
    return 2;
  }
  const size_t n = (size_t)info.n_elem * info.n_fields * info.n_s;
  std::vector<double> U(n);
  if (dgb_problem_init_state(prob, nullptr, nullptr, 0, 0, U.data())) return fail("initial condition");
  dgb_ctx* ctx = nullptr;
  if (dgb_create(prob, device, &ctx)) return fail("device context");
  if (form != DGB_FORM_FP64 && dgb_set_form(ctx, form)) return fail("form");
  const double cfl = info.cfl, tf = info.final_time;
  int count = 0;
  double T = 0.0;
  if (cfl >= 0) {
    if (dgb_write_pos(prob, U.data(), count, T, out.c_str())) return fail("output");
    std::printf("Initial condition written to output file.\n");
    if (info.limiter != DGB_LIM_NONE && dgb_limit(ctx, U.data())) return fail("limiter");
  }
  if (dgb_set_state(ctx, U.data())) return fail("state");
  if (cfl >= 0 && info.cons_output)
    if (int rc = write_conservation(ctx, info.n_fields, T, out)) return rc;
  ++count;
  double tout = times[std::min<size_t>(count, times.size() - 1)];
  bool done = false;
  long steps = 0;
  while (!done) {
    double dt;
    bool output = false;
    if (cfl < 0) {
      dt = times[1] - times[0];
      if (dt > tf - T) { dt = tf - T; done = true; }
    } else {
      const int rc = dgb_cfl_dt(ctx, &dt);
      if (rc == DGB_ERR_DT_SMALL) {
        std::printf("Next time step is too small (<1e-14). Exiting at step %7ld and time %e.\n", steps, T);
        return 1;
      }
      if (rc == DGB_ERR_NONFINITE) {
        std::printf("Time step is NaN. Exiting at step %7ld and time %e.\n", steps, T);
        return 1;
      }
      if (rc) return fail("time step");
      if (dt > tf - T) { dt = tf - T; output = true; done = true; }
      else if (dt > tout - T) { dt = tout - T; output = true; }
    }
    double t_step = 0.0;
    const int rc = dgb_advance(ctx, scheme, 1, dt, &t_step);
    if (rc == DGB_ERR_NONFINITE || rc == DGB_ERR_DT_SMALL) {
      std::printf("Solution became non-finite at step %7ld and time %e.\n", steps, T);
      return 1;
    }
    if (rc) return fail("step");
    T += dt;
    ++steps;
    if (output) {
      if (dgb_get_state(ctx, U.data())) return fail("state");
      if (dgb_write_pos(prob, U.data(), count, T, out.c_str())) return fail("output");
      std::printf("Solution written to file at step %7ld and time %e.\n", steps, T);
      if (info.cons_output)
        if (int rc = write_conservation(ctx, info.n_fields, T, out)) return rc;
      ++count;
      if ((size_t)count < times.size()) tout = times[count];
    }
  }
  if (info.error_output) {
    // the ERROR block of the reference driver (main.cc:909-1038): final state against the deck's
    // initial condition re-evaluated, written as error.dat (dx, then L1 / L2 / Linf per field)
    std::vector<double> Uex(n), err(1 + 3 * (size_t)info.n_fields);
    if (dgb_get_state(ctx, U.data())) return fail("state");
    if (dgb_problem_init_state(prob, nullptr, nullptr, 0, 0, Uex.data())) return fail("initial condition");
    if (dgb_problem_error_norms(prob, U.data(), Uex.data(), err.data())) return fail("error norms");
    const std::string fn = out + "/error.dat";
    FILE* f = std::fopen(fn.c_str(), "w");
    if (!f) { std::fprintf(stderr, "dgbexec: cannot write %s\n", fn.c_str()); return 2; }
    for (int row = 0; row < 3; ++row) {
      std::fprintf(f, "%12.7f\t", err[0]);
      for (int fc = 0; fc < info.n_fields; ++fc) std::fprintf(f, "%20.16E\t", err[1 + row * info.n_fields + fc]);
      std::fprintf(f, "\n");
    }
    std::fclose(f);
  }
  dgb_destroy(ctx);
  dgb_problem_destroy(prob);
  return 0;
}
