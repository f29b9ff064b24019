// Input deck reader.  Same file format as deck::readDeck (code/src/deck/deck.cc:11-64):
// lines before "#Code options" are ignored by the solver (an optional "#Make options" block of
// KEY=VALUE lines there carries the compile-time flags, as tests/runtests.py:80-87 reads them),
// then "#key" lines each followed by their value line(s).  At least 8 mandatory entries must be
// present (deck.cc:58-61; "#mesh file" counts twice).
#include <fstream>
#include <sstream>

#include "host.h"

namespace dgb {

static std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  size_t b = s.find_last_not_of(" \t\r\n");
  return s.substr(a, b - a + 1);
}

static std::vector<double> numbers(const std::vector<std::string>& lines, size_t from) {
  std::vector<double> v;
  for (size_t k = from; k < lines.size(); ++k) {
    std::istringstream is(lines[k]);
    double t;
    while (is >> t) v.push_back(t);
  }
  return v;
}

Status read_deck(const std::string& path, Deck& d) {
  Status st;
  std::ifstream in(path);
  if (!in.is_open()) { st.code = 2; st.msg = "no deck file " + path; return st; }
  std::string line;
  bool in_make = false, found = false;
  while (std::getline(in, line)) {
    std::string t = trim(line);
    if (t == "#Code options") { found = true; break; }
    if (t == "#Make options") { in_make = true; continue; }
    if (in_make) {
      size_t eq = t.find('=');
      if (eq != std::string::npos) d.make_options[trim(t.substr(0, eq))] = trim(t.substr(eq + 1));
    }
  }
  if (!found) { st.code = 2; st.msg = "deck has no #Code options line"; return st; }
  // group "#key" lines with the value lines that follow them
  std::vector<std::pair<std::string, std::vector<std::string>>> entries;
  while (std::getline(in, line)) {
    std::string t = trim(line);
    if (t.empty()) continue;
    if (t[0] == '#') entries.push_back({t, {}});
    else if (!entries.empty()) entries.back().second.push_back(t);
  }
  int cnt = 0;
  for (auto& kv : entries) {
    const std::string& k = kv.first;
    const auto& v = kv.second;
    auto first = [&]() -> std::string { return v.empty() ? std::string() : v[0]; };
    if (k == "#time integration") { d.time_integration = first(); ++cnt; }
    else if (k == "#output time step size") { d.dt_out = std::atof(first().c_str()); ++cnt; }
    else if (k == "#output time array") { d.output_times = numbers(v, 0); ++cnt; }
    else if (k == "#final time") { d.final_time = std::atof(first().c_str()); ++cnt; }
    else if (k == "#Courant-Friedrichs-Lewy condition") { d.cfl = std::atof(first().c_str()); ++cnt; }
    else if (k == "#order") { d.order = std::atoi(first().c_str()); ++cnt; }
    else if (k == "#mesh file") {
      d.mesh_file = first(); ++cnt;
      d.elem_type = v.size() > 1 ? v[1] : ""; ++cnt;
    }
    else if (k == "#limiter") { d.limiter = first(); ++cnt; }
    else if (k == "#initial condition") {
      ++cnt;
      std::istringstream is(first());
      is >> d.ic;
      double t;
      while (is >> t) d.ic_inputs.push_back(t);
      auto more = numbers(v, 1);
      d.ic_inputs.insert(d.ic_inputs.end(), more.begin(), more.end());
    }
    else if (k == "#sensor thresholds") { d.thresholds = numbers(v, 0); }
    else if (k == "#lagrange particles") { d.particles = numbers(v, 0); }
    else if (k == "#restart step") { d.restart_step = std::atoi(first().c_str()); }
    // unrecognised options are ignored, as deck.cc:52-55 does
  }
  if (cnt < 8) { st.code = 2; st.msg = "input deck is incomplete"; return st; }
  return st;
}

}  // namespace dgb
