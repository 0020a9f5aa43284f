// namelist.cpp -- parser for the &hipft_input_parameters namelist group.
//
// Supports what hipft.in files use: `name = value` and
// `name = v1, v2, ...` (per-realization vectors), `name(i) = value`,
// logicals (.true./.false./T/F), quoted strings, Fortran `d` exponents and
// `!` comments.  After parsing, per-realization vectors are filled from the
// scalar defaults where they hold the reference's sentinels
// (src/hipft.f90:8542-8579) and method presets are validated (8583-8608).
#include "namelist.h"

#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <map>
#include <sstream>

namespace hipft {
namespace {

std::string lower(std::string s) {
  for (auto &c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}
std::string trim(const std::string &s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

// Splits on commas that are outside quotes.
std::vector<std::string> split_values(const std::string &v) {
  std::vector<std::string> out;
  std::string cur;
  char q = 0;
  for (char c : v) {
    if (q) {
      cur += c;
      if (c == q) q = 0;
    } else if (c == '\'' || c == '"') {
      q = c;
      cur += c;
    } else if (c == ',') {
      out.push_back(trim(cur));
      cur.clear();
    } else {
      cur += c;
    }
  }
  if (!trim(cur).empty()) out.push_back(trim(cur));
  return out;
}

bool to_double(const std::string &s, double &v) {
  std::string t = lower(trim(s));
  for (auto &c : t)
    if (c == 'd') c = 'e';
  char *end = nullptr;
  v = std::strtod(t.c_str(), &end);
  return end && *end == 0 && !t.empty();
}
bool to_long(const std::string &s, long &v) {
  double d;
  if (!to_double(s, d)) return false;
  v = (long)d;
  return (double)v == d;
}
bool to_bool(const std::string &s, bool &v) {
  std::string t = lower(trim(s));
  if (t == ".true." || t == "t" || t == ".t." || t == "true") { v = true; return true; }
  if (t == ".false." || t == "f" || t == ".f." || t == "false") { v = false; return true; }
  return false;
}
std::string to_string_value(const std::string &s) {
  std::string t = trim(s);
  if (t.size() >= 2 && (t[0] == '\'' || t[0] == '"') && t.back() == t[0]) return t.substr(1, t.size() - 2);
  return t;
}

}  // namespace

bool parse_namelist(const std::string &text, Namelist &nl, std::string &err) {
  // Collect the body of the group, dropping comments (outside quotes).
  std::istringstream in(text);
  std::string line, body;
  bool inside = false, done = false;
  while (!done && std::getline(in, line)) {
    std::string clean;
    char q = 0;
    for (char c : line) {
      if (q) {
        clean += c;
        if (c == q) q = 0;
      } else if (c == '\'' || c == '"') {
        q = c;
        clean += c;
      } else if (c == '!') {
        break;
      } else {
        clean += c;
      }
    }
    std::string t = trim(clean);
    if (t.empty()) continue;
    if (!inside) {
      if (lower(t).rfind("&hipft_input_parameters", 0) == 0) {
        inside = true;
        t = trim(t.substr(23));
        if (t.empty()) continue;
      } else {
        continue;
      }
    }
    size_t slash = std::string::npos;
    q = 0;
    for (size_t i = 0; i < t.size(); ++i) {
      if (q) { if (t[i] == q) q = 0; continue; }
      if (t[i] == '\'' || t[i] == '"') q = t[i];
      else if (t[i] == '/') { slash = i; break; }
    }
    if (slash != std::string::npos) {
      t = t.substr(0, slash);
      done = true;
    }
    body += " " + t + "\n";
  }
  if (!inside) {
    err = "no &hipft_input_parameters group";
    return false;
  }
  // Tokenise "name = values" assignments: a new assignment starts at an
  // identifier followed by '=' (optionally with an (index)).
  struct Assign { std::string name; long index; std::string value; };
  std::vector<Assign> assigns;
  {
    size_t i = 0, n = body.size();
    std::string pending_name;
    long pending_index = 0;
    std::string value;
    bool have = false;
    auto flush = [&]() {
      if (have) assigns.push_back({pending_name, pending_index, trim(value)});
      value.clear();
    };
    char q = 0;
    while (i < n) {
      char c = body[i];
      if (!q && (std::isalpha((unsigned char)c) || c == '_')) {
        size_t j = i;
        while (j < n && (std::isalnum((unsigned char)body[j]) || body[j] == '_')) ++j;
        size_t k = j;
        long idx = 0;
        if (k < n && body[k] == '(') {
          size_t e = body.find(')', k);
          if (e != std::string::npos) {
            idx = std::atol(body.substr(k + 1, e - k - 1).c_str());
            k = e + 1;
          }
        }
        size_t m = k;
        while (m < n && (body[m] == ' ' || body[m] == '\t')) ++m;
        bool prev_ok = (i == 0) || body[i - 1] == ' ' || body[i - 1] == '\n' || body[i - 1] == ',' ||
                       body[i - 1] == '\t';
        if (prev_ok && m < n && body[m] == '=' && (m + 1 >= n || body[m + 1] != '=')) {
          flush();
          pending_name = lower(body.substr(i, j - i));
          pending_index = idx;
          have = true;
          i = m + 1;
          continue;
        }
        value += body.substr(i, j - i);
        i = j;
        continue;
      }
      if (q) {
        if (c == q) q = 0;
      } else if (c == '\'' || c == '"') {
        q = c;
      }
      value += (c == '\n') ? ' ' : c;
      ++i;
    }
    flush();
  }

  std::map<std::string, std::vector<double> *> rvec = {
      {"diffusion_coef_constants", &nl.diffusion_coef_constants},
      {"flow_attenuate_values", &nl.flow_attenuate_values},
      {"flow_dr_coef_p0_values", &nl.flow_dr_coef_p0_values},
      {"flow_dr_coef_p2_values", &nl.flow_dr_coef_p2_values},
      {"flow_dr_coef_p4_values", &nl.flow_dr_coef_p4_values},
      {"flow_mf_coef_p1_values", &nl.flow_mf_coef_p1_values},
      {"flow_mf_coef_p3_values", &nl.flow_mf_coef_p3_values},
      {"flow_mf_coef_p5_values", &nl.flow_mf_coef_p5_values},
      {"assimilate_data_lat_limits", &nl.assimilate_data_lat_limits},
      {"assimilate_data_mu_powers", &nl.assimilate_data_mu_powers},
      {"assimilate_data_mu_limits", &nl.assimilate_data_mu_limits},
      {"source_rfe_total_unsigned_flux_per_hours", &nl.source_rfe_total_unsigned_flux_per_hours},
  };
  // Sentinels of the reference's DATA statements (src/hipft.f90:593-706).
  for (auto &kv : rvec) {
    double sentinel = (kv.first.find("coef_p") != std::string::npos) ? -1000000.0 : -1.0;
    kv.second->assign(kMaxRealizations, sentinel);
  }
  std::map<std::string, int *> ints = {
      {"verbose", &nl.verbose}, {"res_nt", &nl.res_nt}, {"res_np", &nl.res_np},
      {"n_realizations", &nl.n_realizations}, {"validation_run", &nl.validation_run},
      {"flow_dr_model", &nl.flow_dr_model}, {"flow_mf_model", &nl.flow_mf_model},
      {"flow_num_method", &nl.flow_num_method}, {"diffusion_num_method", &nl.diffusion_num_method},
      {"diffusion_subcycles", &nl.diffusion_subcycles}, {"source_rfe_model", &nl.source_rfe_model}};
  std::map<std::string, long *> longs = {{"output_map_idx_start", &nl.output_map_idx_start},
                                         {"output_map_idx_cadence", &nl.output_map_idx_cadence},
                                         {"source_rfe_seed", &nl.source_rfe_seed}};
  std::map<std::string, double *> dbls = {
      {"validation_run_width", &nl.validation_run_width},
      {"initial_map_mult_fac", &nl.initial_map_mult_fac},
      {"output_map_time_cadence", &nl.output_map_time_cadence},
      {"output_history_time_cadence", &nl.output_history_time_cadence},
      {"time_start", &nl.time_start}, {"time_end", &nl.time_end}, {"dt_min", &nl.dt_min},
      {"dt_max", &nl.dt_max}, {"pole_flux_lat_limit", &nl.pole_flux_lat_limit},
      {"flow_vp_rigid_omega", &nl.flow_vp_rigid_omega}, {"flow_rigid_omega", &nl.flow_rigid_omega},
      {"flow_vt_const", &nl.flow_vt_const}, {"flow_attenuate_value", &nl.flow_attenuate_value},
      {"flow_dr_coef_p0_value", &nl.flow_dr_coef_p0_value},
      {"flow_dr_coef_p2_value", &nl.flow_dr_coef_p2_value},
      {"flow_dr_coef_p4_value", &nl.flow_dr_coef_p4_value},
      {"flow_mf_coef_p1_value", &nl.flow_mf_coef_p1_value},
      {"flow_mf_coef_p3_value", &nl.flow_mf_coef_p3_value},
      {"flow_mf_coef_p5_value", &nl.flow_mf_coef_p5_value}, {"upwind", &nl.upwind},
      {"weno_eps", &nl.weno_eps}, {"diffusion_coef_constant", &nl.diffusion_coef_constant},
      {"diffusion_coef_factor", &nl.diffusion_coef_factor},
      {"assimilate_data_mult_fac", &nl.assimilate_data_mult_fac},
      {"assimilate_data_lat_limit", &nl.assimilate_data_lat_limit},
      {"assimilate_data_mu_power", &nl.assimilate_data_mu_power},
      {"assimilate_data_mu_limit", &nl.assimilate_data_mu_limit},
      {"source_rfe_total_unsigned_flux_per_hour", &nl.source_rfe_total_unsigned_flux_per_hour},
      {"source_rfe_lifetime", &nl.source_rfe_lifetime}};
  std::map<std::string, bool *> bools = {
      {"initial_map_flux_balance", &nl.initial_map_flux_balance},
      {"output_map_flux_balance", &nl.output_map_flux_balance}, {"output_map_2d", &nl.output_map_2d},
      {"output_single_precision", &nl.output_single_precision},
      {"strang_splitting", &nl.strang_splitting}, {"advance_flow", &nl.advance_flow},
      {"ragged_realizations", &nl.ragged_realizations},
      {"flow_attenuate", &nl.flow_attenuate}, {"use_flow_from_files", &nl.use_flow_from_files},
      {"advance_diffusion", &nl.advance_diffusion}, {"diffusion_coef_grid", &nl.diffusion_coef_grid},
      {"advance_source", &nl.advance_source}, {"assimilate_data", &nl.assimilate_data},
      {"assimilate_data_balance_flux", &nl.assimilate_data_balance_flux},
      {"assimilate_data_add", &nl.assimilate_data_add},
      {"assimilate_data_custom_from_mu", &nl.assimilate_data_custom_from_mu},
      {"output_flows", nullptr}, {"source_from_file", &nl.source_from_file}};
  std::map<std::string, std::string *> strs = {
      {"initial_map_filename", &nl.initial_map_filename},
      {"output_map_root_filename", &nl.output_map_root_filename},
      {"output_map_directory", &nl.output_map_directory},
      {"diffusion_coef_filename", &nl.diffusion_coef_filename},
      {"assimilate_data_map_list_filename", &nl.assimilate_data_map_list_filename},
      {"assimilate_data_map_root_dir", &nl.assimilate_data_map_root_dir},
      {"output_flows_directory", nullptr}, {"output_flows_root_filename", nullptr},
      {"flow_list_filename", &nl.flow_list_filename}, {"flow_root_dir", &nl.flow_root_dir},
      {"source_filename", &nl.source_filename}};
  std::map<std::string, int> ignored_ints = {};

  for (const auto &a : assigns) {
    std::vector<std::string> vals = split_values(a.value);
    if (vals.empty()) {
      err = "no value for " + a.name;
      return false;
    }
    if (rvec.count(a.name)) {
      auto *vec = rvec[a.name];
      long start = a.index > 0 ? a.index - 1 : 0;
      for (size_t q = 0; q < vals.size(); ++q) {
        double v;
        if (!to_double(vals[q], v) || start + (long)q >= kMaxRealizations) {
          err = "bad value for " + a.name;
          return false;
        }
        (*vec)[start + q] = v;
      }
      continue;
    }
    const std::string &v = vals[0];
    bool ok = true;
    if (ints.count(a.name)) {
      long x = 0;
      ok = to_long(v, x);
      *ints[a.name] = (int)x;
    } else if (longs.count(a.name)) {
      ok = to_long(v, *longs[a.name]);
    } else if (dbls.count(a.name)) {
      double x = 0;
      ok = to_double(v, x);
      if (dbls[a.name]) *dbls[a.name] = x;
    } else if (bools.count(a.name)) {
      bool x = false;
      ok = to_bool(v, x);
      if (bools[a.name]) *bools[a.name] = x;
    } else if (strs.count(a.name)) {
      if (strs[a.name]) *strs[a.name] = to_string_value(v);
    } else if (ignored_ints.count(a.name)) {
      long x = 0;
      ok = to_long(v, x);
    } else {
      err = "unknown namelist variable " + a.name;
      return false;
    }
    if (!ok) {
      err = "bad value for " + a.name + ": " + v;
      return false;
    }
  }

  // process_input_parameters (src/hipft.f90:8458-8614)
  if (nl.output_map_time_cadence > 0 && nl.output_map_idx_cadence > 0) {
    err = "cannot use both output_map_time_cadence and output_map_idx_cadence";
    return false;
  }
  if (nl.n_realizations < 1 || nl.n_realizations > kMaxRealizations) {
    err = "n_realizations out of range";
    return false;
  }
  if (nl.initial_map_filename.empty() && (nl.res_np < 3 || nl.res_nt < 3)) {
    err = "must specify an input map or res_nt, res_np >= 3";
    return false;
  }
  if (!nl.initial_map_filename.empty() && nl.res_np * nl.res_nt > 0) {
    nl.res_nt = 0;
    nl.res_np = 0;
  }
  if (nl.flow_num_method < 1 || nl.flow_num_method > 4) {
    err = "invalid flow_num_method (valid: 1..4)";
    return false;
  }
  auto fill = [&](std::vector<double> &vec, double scalar, std::function<bool(double)> sentinel) {
    for (auto &x : vec)
      if (sentinel(x)) x = scalar;
    vec.resize(nl.n_realizations);
  };
  auto neg = [](double x) { return x < 0.0; };
  auto big = [](double x) { return x < -100000.0; };
  fill(nl.assimilate_data_lat_limits, nl.assimilate_data_lat_limit, neg);
  fill(nl.assimilate_data_mu_limits, nl.assimilate_data_mu_limit, neg);
  fill(nl.assimilate_data_mu_powers, nl.assimilate_data_mu_power, neg);
  fill(nl.flow_dr_coef_p0_values, nl.flow_dr_coef_p0_value, big);
  fill(nl.flow_dr_coef_p2_values, nl.flow_dr_coef_p2_value, big);
  fill(nl.flow_dr_coef_p4_values, nl.flow_dr_coef_p4_value, big);
  fill(nl.flow_mf_coef_p1_values, nl.flow_mf_coef_p1_value, big);
  fill(nl.flow_mf_coef_p3_values, nl.flow_mf_coef_p3_value, big);
  fill(nl.flow_mf_coef_p5_values, nl.flow_mf_coef_p5_value, big);
  fill(nl.flow_attenuate_values, nl.flow_attenuate_value, neg);
  fill(nl.diffusion_coef_constants, nl.diffusion_coef_constant, neg);
  fill(nl.source_rfe_total_unsigned_flux_per_hours, nl.source_rfe_total_unsigned_flux_per_hour, neg);
  return true;
}

bool read_namelist(const std::string &path, Namelist &nl, std::string &err) {
  std::ifstream f(path);
  if (!f) {
    err = "could not open the input file " + path;
    return false;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  return parse_namelist(ss.str(), nl, err);
}

}  // namespace hipft
