// driver.cpp -- standalone driver over the C ABI (hipft_run).
//
// Mirrors `program HIPFT` (src/hipft.f90:869-968) for the flux-transport
// path: setup (reading hipft.in, realization parameters, the initial map or
// a validation map, flows, diffusion, data-assimilation list), then per step
// update_step -> flux_transport_step -> time += dt -> data assimilation ->
// analysis -> history output -> map output, until time_end.  History files
// use the reference's names and Fortran formats (src/hipft.f90:1616-1646,
// 2633-2634); maps are written as the reference's write_map does
// (src/hipft.f90:2801-2917): <root>_initial.h5 after setup, numbered maps in
// output_map_directory at the output cadence (listed in
// hipft_output_map_list.out, src/hipft.f90:2700-2798), <root>_final.h5 at the
// end, and for validation runs the analytic maps of src/hipft.f90:1891-2102.
#include <sys/stat.h>

#include <cfloat>
#include <ctime>
#include <cstdint>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/hipft_gpu.h"
#include "namelist.h"

namespace hipft {
namespace {

constexpr double c_pi = 3.1415926535897932;
constexpr double c_pi_two = 1.5707963267948966;
constexpr double c_pi_four = 0.7853981633974483;
constexpr double c_twopi = 6.2831853071795864;
constexpr double c_threepi_two = 4.71238898038469;
constexpr double c_km_s_to_rs_hr = 0.005172413793103448;
constexpr double c_rsun_cm2 = 4.84416e21;        // src/hipft.f90:119
constexpr double c_input_flux_fac = 1.0e21;      // src/hipft.f90:132

// Fortran 1PE23.15E3: sign column, one digit, 15 decimals, 3-digit exponent.
std::string fmt_e(double v) {
  char b[64];
  std::snprintf(b, sizeof b, "%.15E", v);
  std::string s(b);
  size_t e = s.find('E');
  std::string mant = s.substr(0, e);
  int ex = std::atoi(s.c_str() + e + 1);
  char eb[16];
  std::snprintf(eb, sizeof eb, "E%c%03d", ex < 0 ? '-' : '+', ex < 0 ? -ex : ex);
  std::string r = mant + eb;
  while (r.size() < 23) r = " " + r;
  return r;
}
std::string rjust(const std::string &s, size_t w) { return s.size() >= w ? s : std::string(w - s.size(), ' ') + s; }
std::string fmt_i(long v, int w) { return rjust(std::to_string(v), (size_t)w); }

// Y_lm by the first modified forward column recursion of Holmes &
// Featherstone (2002), as tesseral_spherical_harmonic (src/hipft.f90:2390-2533).
// Y is (np, nt) with phi fastest.
void spherical_harmonic(int m, int l, const std::vector<double> &pv, const std::vector<double> &tv,
                        std::vector<double> &Y) {
  const double lpi = 3.141592653589793;
  int am = std::abs(m), nt = (int)tv.size(), np = (int)pv.size();
  std::vector<double> ct(nt), P(nt, 1.0), Pm(nt, 0.0);
  for (int i = 0; i < nt; ++i) ct[i] = std::cos(tv[i]);
  if (am > 0) {
    for (int i = 0; i < nt; ++i) P[i] = std::sqrt(3.0);
    for (int im = 2; im <= am; ++im)
      for (int i = 0; i < nt; ++i) P[i] = std::sqrt((2.0 * im + 1.0) / (2.0 * im)) * P[i];
  }
  for (int il = am + 1; il <= l; ++il) {
    double a = std::sqrt(((2.0 * il - 1.0) * (2.0 * il + 1.0)) / (double)((il - am) * (il + am)));
    double b = std::sqrt(((2.0 * il + 1.0) * (il + am - 1.0) * (il - am - 1.0)) /
                         ((il - am) * (il + am) * (2.0 * il - 3.0)));
    for (int i = 0; i < nt; ++i) {
      double Pl = a * ct[i] * P[i] - b * Pm[i];
      Pm[i] = P[i];
      P[i] = Pl;
    }
  }
  double norm = 1.0 / std::sqrt(4.0 * lpi);
  for (int i = 0; i < nt; ++i) {
    double s = std::sin(tv[i]), sp = 1.0;
    for (int q = 0; q < am; ++q) sp *= s;
    P[i] = (((am % 2) ? -1.0 : 1.0) * sp) * norm * P[i];
  }
  int pos = (m + 1 >= 0) ? 1 : 0;
  Y.assign((size_t)np * nt, 0.0);
  for (int j = 0; j < nt; ++j)
    for (int i = 0; i < np; ++i)
      Y[(size_t)j * np + i] = P[j] * (pos * std::cos(m * pv[i]) + (1.0 - pos) * std::sin(am * pv[i]));
}

struct DAList {
  std::vector<double> times;  // hours since the first map
  std::vector<std::string> files;
};

bool read_da_list(const std::string &path, DAList &L, std::string &err) {
  std::ifstream in(path);
  if (!in) {
    err = "cannot open assimilation map list " + path;
    return false;
  }
  // rows as READ(...,'(A19,1X,A19,1X,F13.5,1X,A)') reads them
  // (src/hipft.f90:3987-4001): two 19-character date fields, the actual
  // Julian day in columns 41-53 and the map's relative path after column 54,
  // whatever single character separates the fields (blank or comma)
  std::string line;
  std::getline(in, line);  // header row
  std::vector<double> jd;
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.find_first_not_of(" \t") == std::string::npos) continue;
    if (line.size() < 55) {
      err = "malformed row in assimilation map list " + path + ": " + line;
      return false;
    }
    std::string f13 = line.substr(40, 13), digits;
    for (char c : f13)
      if (c != ' ') digits += (c == 'd' || c == 'D') ? 'E' : c;  // blanks are ignored in a numeric field
    char *end = nullptr;
    double j = std::strtod(digits.c_str(), &end);
    if (digits.empty() || *end != '\0') {
      err = "bad Julian day in assimilation map list " + path + ": " + f13;
      return false;
    }
    if (digits.find_first_of(".eEdD") == std::string::npos) j /= 1.0e5;  // F13.5 without a point
    std::string file = line.substr(54);
    while (!file.empty() && (file.back() == ' ' || file.back() == '\t')) file.pop_back();
    jd.push_back(j);
    L.files.push_back(file);
  }
  if (jd.empty()) {
    err = "empty assimilation map list " + path;
    return false;
  }
  for (double j : jd) L.times.push_back(24.0 * j - 24.0 * jd[0]);
  return true;
}

// Fortran 1PE25.15 (two-digit exponent): right-justified in 25 columns.
std::string fmt_pe25(double v) {
  char b[64];
  std::snprintf(b, sizeof b, "%.15E", v);
  return rjust(b, 25);
}

// mkdir -p of a relative or absolute directory
bool make_dirs(const std::string &d) {
  std::string cur;
  size_t i = 0;
  while (i <= d.size()) {
    size_t j = d.find('/', i);
    if (j == std::string::npos) j = d.size();
    cur = d.substr(0, j);
    if (!cur.empty()) {
      struct stat st;
      if (stat(cur.c_str(), &st) != 0) {
        if (mkdir(cur.c_str(), 0755) != 0) return false;
      } else if (!S_ISDIR(st.st_mode)) {
        return false;
      }
    }
    i = j + 1;
  }
  return true;
}

// Flow list of use_flow_from_files, read as READ(...,'(F11.5,1X,A11,1X,A11)')
// reads it (src/hipft.f90:3735-3746): the Julian day in columns 1-11, the
// theta-velocity file in 13-23 and the phi-velocity file in 25-35.
struct FlowFiles {
  std::vector<double> times;  // flow_from_files_times, hours
  std::vector<std::string> vt, vp;
  int idx = 0;  // current entry, 1-based
  double t_cur = 0.0, t_next = 0.0, dt_last = 0.0;
};

// A Fortran F edit field: blanks ignored, D exponents, implied decimals.
bool f_field(const std::string &fld, int decimals, double &v) {
  std::string digits;
  for (char c : fld)
    if (c != ' ') digits += (c == 'd' || c == 'D') ? 'E' : c;
  if (digits.empty()) return false;
  char *end = nullptr;
  v = std::strtod(digits.c_str(), &end);
  if (*end != '\0') return false;
  if (digits.find_first_of(".eE") == std::string::npos) v /= std::pow(10.0, decimals);
  return true;
}

std::string a_field(const std::string &line, size_t pos, size_t n) {
  std::string f = pos < line.size() ? line.substr(pos, n) : std::string();
  while (!f.empty() && (f.back() == ' ' || f.back() == '\t')) f.pop_back();
  return f;
}

bool read_flow_list(const std::string &path, FlowFiles &L, std::string &err) {
  std::ifstream in(path);
  if (!in) {
    err = "cannot open flow list " + path;
    return false;
  }
  std::string line;
  std::getline(in, line);  // header row
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.find_first_not_of(" \t") == std::string::npos) continue;
    double jd;
    if (!f_field(line.substr(0, 11), 5, jd)) {
      err = "bad Julian day in flow list " + path + ": " + line;
      return false;
    }
    L.times.push_back(24.0 * jd);
    L.vt.push_back(a_field(line, 12, 11));
    L.vp.push_back(a_field(line, 24, 11));
  }
  if (L.times.size() < 2) {
    err = "the flow list " + path + " needs at least two entries";
    return false;
  }
  // src/hipft.f90:3750-3753, in place and in order: entries after the first
  // subtract the already-zeroed first one (no effect when the list starts at 0)
  for (size_t i = 0; i < L.times.size(); ++i) L.times[i] = L.times[i] - L.times[0];
  return true;
}

// Normal deviates for the random flux emergence source: get_gaussian
// (src/hipft.f90:8616-8670), the Marsaglia-Bray polar method, with its second
// deviate kept for the next call.  The uniform numbers come from xoshiro256**
// (Blackman and Vigna) seeded through splitmix64 from source_rfe_seed; the
// reference draws them with gfortran's RANDOM_NUMBER, so a seeded run here
// is reproducible but does not repeat the reference's random field.
struct Gaussian {
  uint64_t s[4] = {1, 2, 3, 4};
  bool second = false;
  double v = 0.0, sln = 0.0;
  void seed(uint64_t x) {
    for (auto &w : s) {
      x += 0x9e3779b97f4a7c15ULL;
      uint64_t z = x;
      z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
      z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
      w = z ^ (z >> 31);
    }
    second = false;
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }  // [0, 1)
  double operator()() {
    if (second) {
      second = false;
      return v * sln;
    }
    second = true;
    double u, q;
    for (;;) {
      u = 2.0 * uniform() - 1.0;
      v = 2.0 * uniform() - 1.0;
      q = u * u + v * v;
      if (q < 1.0 && q > 0.0) break;
    }
    sln = std::sqrt(-(2.0 * std::log(q)) / q);
    return u * sln;
  }
};

// interp2d with flint's monotonicity check and interp (src/hipft.f90:
// 7992-8073, 8083-8176, 8178-8210): bilinear from (xi, yi, fi(nxi, nyi)) onto
// (x, y); points outside the table are 0.  Returns false when a scale is not
// strictly increasing.
bool interp2d(const std::vector<double> &xi, const std::vector<double> &yi, const std::vector<double> &fi,
              const std::vector<double> &x, const std::vector<double> &y, std::vector<double> &f) {
  const int nxi = (int)xi.size(), nyi = (int)yi.size(), nx = (int)x.size(), ny = (int)y.size();
  for (int i = 0; i + 1 < nxi; ++i)
    if (xi[i + 1] <= xi[i]) return false;
  for (int i = 0; i + 1 < nyi; ++i)
    if (yi[i + 1] <= yi[i]) return false;
  auto interp = [](const std::vector<double> &t, double xv, int &i0, int &i1, double &a) {
    const int n = (int)t.size();
    if (n == 1 && xv == t[0]) {
      i0 = i1 = 0;
      a = 0.0;
      return true;
    }
    for (int i = 0; i < n - 1; ++i)
      if (xv >= t[i] && xv <= t[i + 1]) {
        i0 = i;
        i1 = i + 1;
        a = (t[i] == t[i + 1]) ? 0.0 : (xv - t[i]) / (t[i + 1] - t[i]);
        return true;
      }
    return false;
  };
  f.assign((size_t)nx * ny, 0.0);
  for (int j = 0; j < ny; ++j) {
    const double yv = y[j];
    int jj, jp;
    double ay;
    if (yv < yi[0] || yv > yi[nyi - 1] || !interp(yi, yv, jj, jp, ay)) continue;
    for (int i = 0; i < nx; ++i) {
      const double xv = x[i];
      int ii, ip;
      double ax;
      if (xv < xi[0] || xv > xi[nxi - 1] || !interp(xi, xv, ii, ip, ax)) continue;
      auto F = [&](int a, int b) { return fi[(size_t)b * nxi + a]; };
      f[(size_t)j * nx + i] =
          (1.0 - ax) * ((1.0 - ay) * F(ii, jj) + ay * F(ii, jp)) + ax * ((1.0 - ay) * F(ip, jj) + ay * F(ip, jp));
    }
  }
  return true;
}

struct Run {
  Namelist nl;
  FlowFiles ff;
  // realizations of this rank (set_local_number_of_realizations): global
  // realization roff+i is local i; shard == NULL on a single process
  const hipft_shard *shard = nullptr;
  int rank = 0, nranks = 1, roff = 0;
  // sources (module sources, src/hipft.f90:290-304)
  Gaussian gauss;
  int rfe1 = 0, rfe2 = 1;
  double time_of_next_source_rfe = 0.0, time_of_prev_source_rfe = 0.0;
  std::vector<double> uf_rvec;
  std::string dir;
  std::string map_dir;             // output_map_directory (relative to the run directory)
  std::vector<double> pscale, tscale;  // the map scales: p(1:npm1), t(1:ntm)
  hipft_gpu *h = nullptr;
  int nr = 0;
  // time stepping state (globals / flows / diffusion modules)
  double time = 0.0, dtime_global = 0.0, dtmax_flow = 0.0, dtime_advection_used = 0.0;
  long ntime = 0, idx_hist = 0, idx_out = 0;
  bool timestep_needs_updating = true, timestep_flow_needs_updating = true, time_step_changed = false;
  bool output_current_map = false;
  double dt_euler = 0.0;
  int64_t niters = 0, subcycles = 0;
  // ragged batches: each realization's own Euler limit, stage count and subcycles
  std::vector<double> r_dt_euler, r_dtmax_flow;
  std::vector<int64_t> r_niters, r_subcycles, r_substeps;
  // DA
  DAList da;
  bool da_active = false;
  int da_idx = 0;
  double time_of_next_input_map = 0.0;
  std::vector<double> hist;
  std::string err;

  std::string path(const std::string &f) const {
    if (f.empty() || f[0] == '/') return f;
    return dir + "/" + f;
  }
  std::string rname(const char *kind, int i) const {
    char b[64];
    std::snprintf(b, sizeof b, "hipft_history_%s_r%06d.out", kind, roff + i);
    return path(b);
  }

  int red(int op, double *v) {
    if (!shard) return HIPFT_OK;
    if (shard->allreduce(shard->user, op, v) != 0) {
      err = "all-reduce callback failed";
      return HIPFT_ECOMM;
    }
    return HIPFT_OK;
  }

  bool history_due() const {
    if (nl.output_history_time_cadence > 0.0)
      return time >= nl.time_start + (double)idx_hist * nl.output_history_time_cadence;
    return true;
  }

  // analysis_step + output_histories (src/hipft.f90:3135-3145, 2637-2690)
  int analysis_and_history() {
    if (!history_due()) return HIPFT_OK;
    int rc = hipft_gpu_analysis(h, time, hist.data());
    if (rc) return rc;
    idx_hist++;
    for (int i = 1; i <= nr; ++i) {
      FILE *fn = std::fopen(rname("num", i).c_str(), "a");
      FILE *fs = std::fopen(rname("sol", i).c_str(), "a");
      if (!fn || !fs) {
        if (fn) std::fclose(fn);
        if (fs) std::fclose(fs);
        return HIPFT_EIO;
      }
      const bool rg = nl.ragged_realizations && !r_dt_euler.empty();
      const double dfl = (rg && !r_dtmax_flow.empty()) ? r_dtmax_flow[i - 1] : dtmax_flow;
      std::string ln = fmt_i(ntime, 10) + " " + fmt_e(time) + " " + fmt_e(dtime_global) + " " + fmt_e(dfl) +
                       " " + fmt_e(dtime_advection_used) + " " + fmt_e(rg ? r_dt_euler[i - 1] : dt_euler) + " " +
                       fmt_i((long)(rg ? r_niters[i - 1] : niters), 15) + " " +
                       fmt_i((long)(rg ? r_subcycles[i - 1] : subcycles), 15) + "\n";
      std::fputs(ln.c_str(), fn);
      std::string ls = fmt_i(ntime, 10) + " " + fmt_e(time) + " ";
      const double *v = &hist[(size_t)(i - 1) * 14];
      for (int q = 0; q < 14; ++q) ls += fmt_e(v[q]) + " ";
      ls += "\n";
      std::fputs(ls.c_str(), fs);
      std::fclose(fn);
      std::fclose(fs);
    }
    return HIPFT_OK;
  }

  // generate_rfe (src/hipft.f90:8809-8921): the random map, then the frame
  int generate_rfe(int slot) {
    hipft_info inf;
    hipft_gpu_info(h, &inf);
    const int ntm = inf.ntm, npm = inf.npm;
    const double normfac = c_pi / std::sqrt(c_twopi);
    std::vector<double> rnd((size_t)ntm * npm, 0.0);
    for (int k = 2; k <= npm - 1; ++k)
      for (int j = 1; j <= ntm; ++j) rnd[(size_t)(k - 1) * ntm + (j - 1)] = normfac * gauss();
    return hipft_gpu_set_rfe_frame(h, slot, nl.source_rfe_model, rnd.data(), uf_rvec.data());
  }

  // load_source (src/hipft.f90:7050-7213)
  int load_source() {
    hipft_info inf;
    hipft_gpu_info(h, &inf);
    const int ntm = inf.ntm, npm = inf.npm;
    if (nl.source_from_file) {
      int nd = 0;
      int64_t dims[3];
      std::string f = path(nl.source_filename);
      int rc = hipft_h5_read(f.c_str(), &nd, dims, nullptr, nullptr, nullptr, nullptr);
      if (rc || nd != 2) {
        err = "cannot read the source file " + f + " as a 2D map";
        return rc ? rc : HIPFT_EINVAL;
      }
      const int nfp = (int)dims[0], nft = (int)dims[1];
      std::vector<double> sf((size_t)nfp * nft), pf(nfp), tf(nft);
      rc = hipft_h5_read(f.c_str(), &nd, dims, sf.data(), pf.data(), tf.data(), nullptr);
      if (rc) return rc;
      std::vector<double> fi((size_t)nft * nfp);  // TRANSPOSE: (nft, nfp), theta fastest
      for (int jp = 0; jp < nfp; ++jp)
        for (int it = 0; it < nft; ++it) fi[(size_t)jp * nft + it] = sf[(size_t)it * nfp + jp];
      std::vector<double> p(pscale);
      p.push_back(pscale[1] + c_twopi);  // p(npm) = p(2) + 2 pi (src/hipft.f90:2131)
      std::vector<double> out;
      if (!interp2d(tf, pf, fi, tscale, p, out)) {
        err = "the source file's scales are not monotonically increasing";
        return HIPFT_EINVAL;
      }
      rc = hipft_gpu_set_source_file(h, out.data());
      if (rc) return rc;
    }
    if (nl.source_rfe_model > 0) {
      if (nl.source_rfe_seed != -9999) gauss.seed((uint64_t)nl.source_rfe_seed);
      else {  // RANDOM_SEED(); every rank takes rank 0's draws (the reference broadcasts them)
        double sd = (rank == 0) ? (double)((std::time(nullptr) ^ ((uint64_t)(uintptr_t)this >> 4)) & 0xffffffffULL)
                                : -1.0;
        int rc = red(HIPFT_RED_MAX, &sd);
        if (rc) return rc;
        gauss.seed((uint64_t)sd);
      }
      const double num_cells = (double)ntm * (npm - 2);
      uf_rvec.assign(nr, 0.0);
      for (int i = 0; i < nr; ++i)
        uf_rvec[i] = (nl.source_rfe_model == 1)
                         ? nl.source_rfe_total_unsigned_flux_per_hours[i] * c_input_flux_fac / (c_rsun_cm2 * num_cells)
                         : nl.source_rfe_total_unsigned_flux_per_hours[i] * c_input_flux_fac /
                               (c_rsun_cm2 * 4.0 * c_pi);
      rfe1 = 0;
      rfe2 = 1;
      int rc = generate_rfe(rfe1);
      if (rc) return rc;
      rc = generate_rfe(rfe2);
      if (rc) return rc;
      time_of_next_source_rfe = time + nl.source_rfe_lifetime;
      time_of_prev_source_rfe = time;
    }
    return HIPFT_OK;
  }

  // update_source (src/hipft.f90:3875-3947)
  int update_source() {
    const bool rfe = nl.source_rfe_model > 0;
    double alpha = 0.0;
    if (rfe) {
      if (time >= time_of_next_source_rfe) {
        time_of_prev_source_rfe = time_of_next_source_rfe;
        time_of_next_source_rfe = time_of_prev_source_rfe + nl.source_rfe_lifetime;
        std::swap(rfe1, rfe2);
        int rc = generate_rfe(rfe2);
        if (rc) return rc;
      }
      alpha = (time - time_of_prev_source_rfe) / nl.source_rfe_lifetime;
    }
    return hipft_gpu_update_source(h, nl.source_from_file, rfe, rfe1, rfe2, alpha);
  }

  // read_2d_file of one flow pair and hand it to the library
  // (add_flow_from_files src/hipft.f90:3578-3634, load_flow_from_files 3765-3800)
  int read_flow_pair(int idx, int at_load) {
    hipft_info inf;
    hipft_gpu_info(h, &inf);
    const int64_t ntm = inf.ntm, nt = ntm + 1, np = inf.npm, npm1 = inf.npm - 1;
    std::vector<double> vt, vp;
    const std::string *names[2] = {&ff.vt[idx - 1], &ff.vp[idx - 1]};
    std::vector<double> *dst[2] = {&vt, &vp};
    const int64_t want[2][2] = {{npm1, nt}, {np, ntm}};
    for (int q = 0; q < 2; ++q) {
      std::string f = nl.flow_root_dir + "/" + *names[q];
      if (f[0] != '/') f = path(f);
      int nd = 0;
      int64_t dims[3];
      int rc = hipft_h5_read(f.c_str(), &nd, dims, nullptr, nullptr, nullptr, nullptr);
      if (rc || nd != 2 || dims[0] != want[q][0] || dims[1] != want[q][1]) {
        err = "cannot read flow file " + f + " as a 2D map of the run's grid";
        return rc ? rc : HIPFT_EINVAL;
      }
      dst[q]->resize((size_t)(dims[0] * dims[1]));
      rc = hipft_h5_read(f.c_str(), &nd, dims, dst[q]->data(), nullptr, nullptr, nullptr);
      if (rc) return rc;
    }
    return hipft_gpu_set_flow_from_files(h, vt.data(), vp.data(), at_load);
  }

  // load_flow_from_files (src/hipft.f90:3675-3800)
  int load_flow_from_files() {
    if (!read_flow_list(path(nl.flow_list_filename), ff, err)) return HIPFT_EIO;
    const int n = (int)ff.times.size();
    const double span = ff.times[n - 1] - ff.times[0];
    const double tsf = nl.time_start - std::floor(nl.time_start / span) * span;  // MODULO
    int idx = 0;
    for (int i = 1; i < n; ++i)
      if (std::fabs(ff.times[i] - tsf) < std::fabs(ff.times[idx] - tsf)) idx = i;
    idx += 1;
    if (ff.times[idx - 1] > tsf) idx -= 1;
    ff.idx = idx;
    int rc = read_flow_pair(idx, 1);
    if (rc) return rc;
    ff.dt_last = ff.times[n - 1] - ff.times[n - 2];
    ff.t_cur = nl.time_start - tsf + ff.times[idx - 1];
    const double delta = (idx + 1 > n) ? ff.dt_last : ff.times[idx] - ff.times[idx - 1];
    ff.t_next = ff.t_cur + delta;
    return HIPFT_OK;
  }

  // the file part of add_flow_from_files (src/hipft.f90:3552-3658)
  int advance_flow_files() {
    if (!(nl.advance_flow && nl.use_flow_from_files) || time < ff.t_next) return HIPFT_OK;
    const int n = (int)ff.times.size();
    ff.idx += 1;
    if (ff.idx > n) ff.idx = 1;
    int rc = read_flow_pair(ff.idx, 0);
    if (rc) return rc;
    ff.t_cur = ff.t_next;
    const double delta = (ff.idx + 1 > n) ? ff.dt_last : ff.times[ff.idx] - ff.times[ff.idx - 1];
    ff.t_next = ff.t_cur + delta;
    return HIPFT_OK;
  }

  // write_2d_file / write_3d_file (src/hipft.f90:6353-6493): PT data
  // (n1, n2[, n3]) with scales s1, s2 and realization numbers 1..n3.
  // (n1, n2[, n3]) with scales s1, s2 and realization numbers 1..n3.  With
  // `gathered`, f holds this rank's n3 realizations and rank 0 writes all
  // ranks' (MPI_Gatherv in the reference); otherwise rank 0 writes its own.
  int write_pt(const std::string &fname, int n1, int n2, int n3, const double *f, const double *s1,
               const double *s2, bool two_d, bool gathered = true) {
    std::vector<double> all;
    if (shard && gathered) {
      const size_t plane = (size_t)n1 * n2;
      if (rank == 0) all.resize(plane * nl.n_realizations);
      if (shard->gather(shard->user, f, (int64_t)(plane * n3), rank == 0 ? all.data() : nullptr) != 0) {
        err = "gather callback failed";
        return HIPFT_ECOMM;
      }
      f = all.data();
      n3 = nl.n_realizations;
    }
    if (rank != 0) return HIPFT_OK;
    std::vector<double> s3(n3);
    for (int i = 0; i < n3; ++i) s3[i] = (double)(i + 1);
    int64_t dims[3] = {n1, n2, two_d ? 1 : n3};
    int rc = hipft_h5_write(path(fname).c_str(), two_d ? 2 : 3, dims, f, s1, s2, two_d ? nullptr : s3.data(),
                            nl.output_single_precision ? 1 : 0);
    if (rc) err = "cannot write the map file " + path(fname);
    return rc;
  }

  // write_map (src/hipft.f90:2801-2917): the current field, flux-balanced
  // on a copy when output_map_flux_balance, as PT with one-point phi overlap.
  int write_map(const std::string &fname) {
    hipft_info inf;
    hipft_gpu_info(h, &inf);
    const int ntm = inf.ntm, npm = inf.npm, npm1 = npm - 1;
    std::vector<double> f((size_t)ntm * npm * nr);
    int rc = hipft_gpu_get_field(h, f.data());
    if (rc) return rc;
    if (nl.output_map_flux_balance) {
      // balance_flux (src/hipft.f90:8752-8807) on the copy
      std::vector<double> fp(nr), fm(nr);
      rc = hipft_gpu_get_flux(h, fp.data(), fm.data());
      if (rc) return rc;
      for (int i = 0; i < nr; ++i) {
        if (fm[i] + fp[i] == 0.0) continue;
        const double ratio = std::sqrt(std::fabs(fp[i] / fm[i]));
        double *a = &f[(size_t)i * ntm * npm];
        for (size_t q = 0; q < (size_t)ntm * npm; ++q) a[q] = (a[q] > 0) ? a[q] / ratio : a[q] * ratio;
      }
    }
    std::vector<double> fout((size_t)npm1 * ntm * nr);
    for (int i = 0; i < nr; ++i)
      for (int j = 0; j < ntm; ++j)
        for (int k = 0; k < npm1; ++k)
          fout[((size_t)i * ntm + j) * npm1 + k] = f[((size_t)i * npm + k) * ntm + j];
    return write_pt(fname, npm1, ntm, nr, fout.data(), pscale.data(), tscale.data(),
                    nl.output_map_2d && nl.n_realizations == 1);
  }

  // output_map (src/hipft.f90:2700-2798)
  int output_map() {
    if (nl.output_map_idx_cadence > 0 && ntime % nl.output_map_idx_cadence == 0) output_current_map = true;
    if (nl.output_map_time_cadence > 0.0 &&
        time >= nl.time_start + (double)(idx_out - (nl.output_map_idx_start - 1)) * nl.output_map_time_cadence)
      output_current_map = true;
    if (output_current_map) {
      idx_out++;
      char idx[32];
      std::snprintf(idx, sizeof idx, "%06ld", idx_out);
      const std::string base = nl.output_map_root_filename + "_idx" + idx + ".h5";
      int rc = write_map(map_dir + "/" + base);
      if (rc) return rc;
      output_current_map = false;
      if (rank != 0) return HIPFT_OK;
      FILE *fl = std::fopen(path("hipft_output_map_list.out").c_str(), "a");
      if (!fl) return HIPFT_EIO;
      std::string ln = fmt_i(idx_out, 10) + "   " + fmt_pe25(time) + "    " + base + "\n";
      std::fputs(ln.c_str(), fl);
      std::fclose(fl);
    }
    return HIPFT_OK;
  }

  // update_timestep (src/hipft.f90:4308-4461)
  int update_timestep() {
    if (timestep_needs_updating) {
      dtime_global = nl.time_end - time;
      time_step_changed = true;
      if (nl.advance_flow) {
        dtmax_flow = DBL_MAX;
        if (nl.ragged_realizations) r_dtmax_flow.assign(nr, DBL_MAX);
        if (timestep_flow_needs_updating) {
          int rc = hipft_gpu_flow_dtmax(h, &dtmax_flow);
          if (rc) return rc;
          // each realization's own limit, for its history (the step takes the smallest)
          if (nl.ragged_realizations && (rc = hipft_gpu_flow_dtmax_each(h, r_dtmax_flow.data()))) return rc;
          timestep_flow_needs_updating = false;
        }
        if (dtmax_flow < dtime_global) dtime_global = dtmax_flow;
      }
      if (nl.dt_max < dtime_global) dtime_global = nl.dt_max;
      if (dtime_global < nl.dt_min) std::fprintf(stderr, "   UPDATE_TIMESTEP: Warning! Time step is smaller than DTMIN!\n");
      timestep_needs_updating = false;
    }
    if (nl.output_map_time_cadence > 0.0) {
      double tn = nl.time_start + (double)(idx_out - (nl.output_map_idx_start - 1)) * nl.output_map_time_cadence;
      if (time + dtime_global >= tn) {
        dtime_global = tn - time;
        timestep_needs_updating = timestep_flow_needs_updating = time_step_changed = true;
      }
    }
    if (da_active && time + dtime_global >= time_of_next_input_map) {
      dtime_global = time_of_next_input_map - time;
      timestep_needs_updating = timestep_flow_needs_updating = time_step_changed = true;
    }
    if (nl.advance_flow && nl.use_flow_from_files && time + dtime_global >= ff.t_next) {  // src/hipft.f90:4415
      dtime_global = ff.t_next - time;
      timestep_needs_updating = timestep_flow_needs_updating = time_step_changed = true;
    }
    if (nl.advance_source && nl.source_rfe_model > 0 &&
        time + dtime_global >= time_of_next_source_rfe) {  // src/hipft.f90:4431-4442
      dtime_global = std::min(time_of_next_source_rfe - time, 0.5 * nl.source_rfe_lifetime);
      timestep_needs_updating = timestep_flow_needs_updating = time_step_changed = true;
    }
    if (time + dtime_global >= nl.time_end) {
      dtime_global = nl.time_end - time;
      timestep_needs_updating = false;
      time_step_changed = true;
    }
    return HIPFT_OK;
  }

  static void cycle_cb(void *user, int, double time_stepped, double, int64_t s, int64_t sc) {
    Run *r = (Run *)user;
    if (r->nl.verbose <= 1) return;
    r->niters = s;
    r->subcycles = sc;
    double tt = r->time;
    r->time = r->time + time_stepped;
    int rc = r->analysis_and_history();
    if (rc && r->err.empty()) r->err = "history output inside the diffusion step failed";
    r->time = tt;
  }

  int apply_data_assimilation() {
    if (!(da_active && time >= time_of_next_input_map)) return HIPFT_OK;
    std::string f = nl.assimilate_data_map_root_dir + "/" + da.files[da_idx];
    if (f[0] != '/') f = path(f);
    int nd = 0;
    int64_t dims[3];
    int rc = hipft_h5_read(f.c_str(), &nd, dims, nullptr, nullptr, nullptr, nullptr);
    if (rc) {
      err = "cannot read assimilation map " + f;
      return rc;
    }
    std::vector<double> data((size_t)(dims[0] * dims[1] * dims[2]));
    rc = hipft_h5_read(f.c_str(), &nd, dims, data.data(), nullptr, nullptr, nullptr);
    if (rc) return rc;
    hipft_info inf;
    hipft_gpu_info(h, &inf);
    if (dims[0] != inf.npm - 1 || dims[1] != inf.ntm || dims[2] < 3) {
      err = "assimilation map size does not match the run's grid";
      return HIPFT_EINVAL;
    }
    hipft_da_opts o{};
    o.add = nl.assimilate_data_add;
    o.custom_from_mu = nl.assimilate_data_custom_from_mu;
    o.balance_flux = nl.assimilate_data_balance_flux;
    o.mult_fac = nl.assimilate_data_mult_fac;
    o.mu_power = nl.assimilate_data_mu_powers.data();
    o.mu_limit = nl.assimilate_data_mu_limits.data();
    o.lat_limit = nl.assimilate_data_lat_limits.data();
    rc = hipft_gpu_assimilate(h, data.data(), &o);
    if (rc) return rc;
    da_idx++;
    if (da_idx >= (int)da.files.size()) da_active = false;
    else time_of_next_input_map = da.times[da_idx];
    return HIPFT_OK;
  }

  int setup(int device) {
    nr = nl.n_realizations;
    if (shard) {  // set_local_number_of_realizations (src/hipft.f90:1025-1037)
      const int avg = nl.n_realizations / nranks, rem = nl.n_realizations - avg * nranks;
      nr = avg + (rank < rem ? 1 : 0);
      roff = rank * avg + std::min(rank, rem);
      if (nr < 1) {
        err = "more ranks than realizations";
        return HIPFT_EINVAL;
      }
      for (auto *v : {&nl.diffusion_coef_constants, &nl.flow_attenuate_values, &nl.flow_dr_coef_p0_values,
                      &nl.flow_dr_coef_p2_values, &nl.flow_dr_coef_p4_values, &nl.flow_mf_coef_p1_values,
                      &nl.flow_mf_coef_p3_values, &nl.flow_mf_coef_p5_values, &nl.assimilate_data_lat_limits,
                      &nl.assimilate_data_mu_powers, &nl.assimilate_data_mu_limits,
                      &nl.source_rfe_total_unsigned_flux_per_hours})
        *v = std::vector<double>(v->begin() + roff, v->begin() + roff + nr);
    }
    hist.assign((size_t)nr * 14, 0.0);
    if (!nl.diffusion_coef_filename.empty()) {
      err = "diffusion_coef_filename is not supported yet";
      return HIPFT_EINVAL;
    }
    // initial condition (load_initial_condition, src/hipft.f90:1741-2187)
    int n1, n2;
    std::vector<double> s1, s2, f_local;
    if (nl.initial_map_filename.empty()) {
      n1 = nl.res_np;
      n2 = nl.res_nt;
      double d1 = c_twopi / (n1 - 1), d2 = c_pi / (n2 - 1);
      for (int i = 1; i <= n1; ++i) s1.push_back((i - 1) * d1);
      for (int i = 1; i <= n2; ++i) s2.push_back((i - 1) * d2);
      f_local.assign((size_t)n1 * n2 * nr, 0.0);
    } else {
      int nd = 0;
      int64_t dims[3];
      std::string f = path(nl.initial_map_filename);
      int rc = hipft_h5_read(f.c_str(), &nd, dims, nullptr, nullptr, nullptr, nullptr);
      if (rc) {
        err = "cannot read the initial map " + f;
        return rc;
      }
      n1 = (int)dims[0];
      n2 = (int)dims[1];
      std::vector<double> all((size_t)(dims[0] * dims[1] * dims[2]));
      s1.resize(n1);
      s2.resize(n2);
      rc = hipft_h5_read(f.c_str(), &nd, dims, all.data(), s1.data(), s2.data(), nullptr);
      if (rc) return rc;
      f_local.assign((size_t)n1 * n2 * nr, 0.0);
      size_t plane = (size_t)n1 * n2;
      if (nd == 2) {
        for (int i = 0; i < nr; ++i) std::copy(all.begin(), all.begin() + plane, f_local.begin() + plane * i);
      } else {
        if (dims[2] != nl.n_realizations) {
          err = "number of realizations in the input map differs from n_realizations";
          return HIPFT_EINVAL;
        }
        std::copy(all.begin() + plane * roff, all.begin() + plane * (roff + nr), f_local.begin());
      }
    }
    double vt_const = nl.flow_vt_const, vp_omega = nl.flow_vp_rigid_omega;
    std::vector<double> fval_u0;
    size_t plane = (size_t)n1 * n2;
    const bool two_d = nl.output_map_2d && nl.n_realizations == 1;
    if (nl.validation_run == 1) {
      std::vector<double> Y0, Y5;
      spherical_harmonic(0, 6, s1, s2, Y0);
      spherical_harmonic(5, 6, s1, s2, Y5);
      fval_u0.assign(plane * nr, 0.0);
      for (int i = 0; i < nr; ++i)
        for (size_t q = 0; q < plane; ++q) fval_u0[plane * i + q] = Y0[q] + std::sqrt(14.0 / 11.0) * Y5[q];
      // initial and final analytic maps (src/hipft.f90:1921-2031)
      int rc = write_pt(nl.output_map_root_filename + "_initial_0.h5", n1, n2, nr, fval_u0.data(), s1.data(),
                        s2.data(), two_d);
      if (rc) return rc;
      std::vector<double> fa(plane * nr);
      for (int i = 0; i < nr; ++i)
        for (size_t q = 0; q < plane; ++q)
          fa[plane * i + q] = fval_u0[plane * i + q] * std::exp(-42.0 * nl.diffusion_coef_constants[i] *
                                                                nl.diffusion_coef_factor * nl.time_end);
      rc = write_pt(nl.output_map_root_filename + "_final_analytic.h5", n1, n2, nr, fa.data(), s1.data(),
                    s2.data(), two_d);
      if (rc) return rc;
      f_local = fval_u0;
    } else if (nl.validation_run == 2) {
      double vt_end_loc = c_pi_four;
      if (std::fabs(vt_const) > 0.0) {
        vt_const = (c_pi_two / (nl.time_end - nl.time_start)) / c_km_s_to_rs_hr;
        vt_end_loc = 3.0 * c_pi_four;
      }
      if (std::fabs(vp_omega) > 0.0) vp_omega = (c_twopi / (nl.time_end - nl.time_start)) / c_km_s_to_rs_hr;
      double w = nl.validation_run_width;
      std::vector<double> fa(plane);
      for (int i = 0; i < nr; ++i)
        for (int j = 1; j <= n2; ++j) {
          double sti = (j > 1 && j < n2) ? 1.0 / std::sin(s2[j - 1]) : 0.0;
          for (int k = 1; k <= n1; ++k) {
            double a = s2[j - 1] - c_pi_four, b1 = s1[k - 1] - c_pi_two, b2 = s1[k - 1] - c_threepi_two;
            f_local[plane * i + (size_t)(j - 1) * n1 + (k - 1)] =
                -sti * std::exp(-(a * a) / w - (b1 * b1) / w) + sti * std::exp(-(a * a) / w - (b2 * b2) / w);
            if (i == 0) {
              double e = s2[j - 1] - vt_end_loc;
              fa[(size_t)(j - 1) * n1 + (k - 1)] =
                  -sti * std::exp(-(e * e) / w - (b1 * b1) / w) + sti * std::exp(-(e * e) / w - (b2 * b2) / w);
            }
          }
        }
      // final analytic map of the first realization (src/hipft.f90:2062-2097)
      int rc = write_pt(nl.output_map_root_filename + "_final_analytic.h5", n1, n2, 1, fa.data(), s1.data(),
                        s2.data(), true, false);
      if (rc) return rc;
    }
    pscale = s1;
    tscale = s2;
    hipft_grid g{};
    g.ntm = n2;
    g.npm1 = n1;
    g.nr = nr;
    g.device = device;
    g.t = s2.data();
    g.p = s1.data();
    hipft_params P{};
    P.advance_flow = nl.advance_flow;
    P.flow_num_method = nl.flow_num_method;
    P.upwind = nl.upwind;
    P.weno_eps = nl.weno_eps;
    P.strang_splitting = nl.strang_splitting;
    P.advance_diffusion = nl.advance_diffusion;
    P.diffusion_num_method = nl.diffusion_num_method;
    P.diffusion_subcycles = nl.diffusion_subcycles;
    P.diffusion_coef_grid = nl.diffusion_coef_grid;
    P.diffusion_coef_factor = nl.diffusion_coef_factor;
    P.diffusion_coef_constants = nl.diffusion_coef_constants.data();
    P.pole_flux_lat_limit = nl.pole_flux_lat_limit;
    P.verbose = nl.verbose;
    P.advance_source = nl.advance_source;
    int rc = hipft_gpu_create(&g, &P, &h);
    if (rc) {
      err = "hipft_gpu_create failed";
      return rc;
    }
    if (shard) {
      rc = hipft_gpu_set_allreduce(h, shard->allreduce, shard->user);
      if (rc) return rc;
    }
    rc = hipft_gpu_load_initial_map(h, f_local.data(), nl.initial_map_flux_balance, nl.initial_map_mult_fac);
    if (rc) return rc;
    if (nl.ragged_realizations) {
      rc = hipft_gpu_set_ragged(h, 1);
      if (rc) {
        err = "ragged_realizations: the method switches do not allow a ragged batch";
        return rc;
      }
      r_dt_euler.assign(nr, 0.0);
      r_niters.assign(nr, 0);
      r_subcycles.assign(nr, nl.diffusion_subcycles);
      r_substeps.assign(nr, 1);
      rc = hipft_gpu_ragged_schedule(h, nullptr, nullptr, nullptr, r_dt_euler.data());
      if (rc) return rc;
    }
    rc = write_map(nl.output_map_root_filename + "_initial.h5");  // src/hipft.f90:2185
    if (rc) return rc;
    if (nl.validation_run == 1) rc = hipft_gpu_set_validation(h, 1, fval_u0.data(), 0, 0, 0, nl.time_start);
    else if (nl.validation_run == 2)
      rc = hipft_gpu_set_validation(h, 2, nullptr, nl.validation_run_width, vt_const, vp_omega, nl.time_start);
    if (rc) return rc;
    if (nl.advance_flow) {
      hipft_flow_def d{};
      d.flow_dr_model = nl.flow_dr_model;
      d.flow_mf_model = nl.flow_mf_model;
      d.dr_p0 = nl.flow_dr_coef_p0_values.data();
      d.dr_p2 = nl.flow_dr_coef_p2_values.data();
      d.dr_p4 = nl.flow_dr_coef_p4_values.data();
      d.mf_p1 = nl.flow_mf_coef_p1_values.data();
      d.mf_p3 = nl.flow_mf_coef_p3_values.data();
      d.mf_p5 = nl.flow_mf_coef_p5_values.data();
      d.flow_vp_rigid_omega = vp_omega;
      d.flow_vt_const = vt_const;
      d.flow_rigid_omega = nl.flow_rigid_omega;
      d.flow_attenuate = nl.flow_attenuate;
      d.flow_attenuate_values = nl.flow_attenuate_values.data();
      rc = hipft_gpu_set_flow(h, &d);
      if (rc) return rc;
      if (nl.use_flow_from_files) {
        rc = load_flow_from_files();
        if (rc) return rc;
      }
    }
    time = nl.time_start;
    if (nl.advance_source) {
      rc = load_source();
      if (rc) return rc;
    }
    hipft_info inf;
    hipft_gpu_info(h, &inf);
    dt_euler = inf.dtime_diffusion_euler;
    subcycles = nl.diffusion_subcycles;
    idx_out = nl.output_map_idx_start - 1;
    if (nl.output_map_idx_cadence > 0 || nl.output_map_time_cadence > 0.0) {
      output_current_map = true;
      // output directory and map list (src/hipft.f90:1194-1210, 1654-1664)
      map_dir = nl.output_map_directory;
      if (rank == 0) {
        if (!make_dirs(path(map_dir))) {
          std::printf(" ### Could not make map output subdirectory, using ./\n");
          map_dir = ".";
        }
        FILE *fl = std::fopen(path("hipft_output_map_list.out").c_str(), "w");
        if (!fl) {
          err = "cannot create hipft_output_map_list.out in " + dir;
          return HIPFT_EIO;
        }
        std::string hdr = rjust("IDX", 10) + " " + rjust("TIME", 25) + " FILENAME\n";
        std::fputs(hdr.c_str(), fl);
        std::fclose(fl);
      }
      if (shard) {  // the directory rank 0 settled on (an index into two choices)
        double fallback = (map_dir == ".") ? 1.0 : 0.0;
        int rc = red(HIPFT_RED_MAX, &fallback);
        if (rc) return rc;
        if (fallback > 0.0) map_dir = ".";
      }
    }
    if (nl.assimilate_data) {
      if (!read_da_list(path(nl.assimilate_data_map_list_filename), da, err)) return HIPFT_EIO;
      // load_data_assimilation time bookkeeping (src/hipft.f90:4017-4042)
      int best = 0;
      double bd = DBL_MAX;
      for (size_t q = 0; q < da.times.size(); ++q) {
        double d = std::fabs(da.times[q] - nl.time_start);
        if (d < bd) { bd = d; best = (int)q; }
      }
      da_active = true;
      if (nl.time_start <= 0.0) {
        da_idx = 0;
        time_of_next_input_map = 0.0;
      } else if (nl.time_start > da.times.back()) {
        da_active = false;
      } else if (nl.time_start <= da.times[best]) {
        da_idx = best;
        time_of_next_input_map = da.times[best];
      } else {
        da_idx = best + 1;
        time_of_next_input_map = da.times[best + 1];
      }
    }
    // history files with headers (create_and_open_output_log_files, src/hipft.f90:1601-1648)
    const char *numh[] = {"TIME", "DTIME", "DTIME_ADV_STB", "DTIME_ADV_USED", "DTIME_DIFF_STB", "N_DIFF_PER_STEP",
                          "N_DIFF_CYCLES"};
    const char *solh[] = {"TIME", "BR_MIN", "BR_MAX", "BR_ABS_MIN", "FLUX_POSITIVE", "FLUX_NEGATIVE",
                          "NPOLE_FLUX_POSITIVE", "NPOLE_FLUX_NEGATIVE", "SPOLE_FLUX_POSITIVE",
                          "SPOLE_FLUX_NEGATIVE", "NPOLE_AREA", "SPOLE_AREA", "EQ_DIPOLE", "AX_DIPOLE",
                          "VALIDATION_ERR_HHabs"};
    for (int i = 1; i <= nr; ++i) {
      FILE *fn = std::fopen(rname("num", i).c_str(), "w");
      FILE *fs = std::fopen(rname("sol", i).c_str(), "w");
      if (!fn || !fs) {
        if (fn) std::fclose(fn);
        if (fs) std::fclose(fs);
        err = "cannot create history files in " + dir;
        return HIPFT_EIO;
      }
      std::string a = rjust("STEP", 10) + " ";
      for (auto *s : numh) a += rjust(s, 22) + " ";
      std::fputs((a + "\n").c_str(), fn);
      std::string b = rjust("STEP", 10) + " ";
      for (auto *s : solh) b += rjust(s, 22) + " ";
      std::fputs((b + "\n").c_str(), fs);
      std::fclose(fn);
      std::fclose(fs);
    }
    rc = analysis_and_history();
    if (rc) return rc;
    return output_map();
  }

  int main_loop() {
    for (;;) {
      ntime++;
      if (nl.advance_flow) {
        int upd = 0;
        int rc = advance_flow_files();
        if (rc) return rc;
        rc = hipft_gpu_update_flow(h, &upd);
        if (rc) return rc;
        if (upd) timestep_flow_needs_updating = timestep_needs_updating = true;
      }
      if (nl.advance_source) {
        int rc = update_source();
        if (rc) return rc;
      }
      int rc = update_timestep();
      if (rc) return rc;
      hipft_diffusion_info di{};
      double dtl = dtime_global;
      if (nl.advance_flow) dtime_advection_used = nl.strang_splitting ? dtl * 0.5 : dtl;
      rc = hipft_gpu_flux_transport_step(h, dtl, &Run::cycle_cb, this, nl.advance_diffusion ? &di : nullptr);
      if (rc) return rc;
      if (!err.empty()) return HIPFT_EIO;
      if (nl.advance_diffusion) {
        niters = di.sts_s;
        subcycles = di.subcycles;
        if (nl.ragged_realizations) {
          rc = hipft_gpu_ragged_schedule(h, r_niters.data(), r_subcycles.data(), r_substeps.data(), r_dt_euler.data());
          if (rc) return rc;
        }
      }
      time = time + dtime_global;
      rc = apply_data_assimilation();
      if (rc) return rc;
      rc = analysis_and_history();
      if (rc) return rc;
      rc = output_map();
      if (rc) return rc;
      if (nl.verbose >= 0) {
        std::printf(" Completed step: %10ld  Time: %14.3f / %14.3f  dt: %12.6f\n", ntime, time, nl.time_end,
                    dtime_global);
      }
      if (time >= nl.time_end) break;
      FILE *stop = std::fopen(path("STOPRUN").c_str(), "r");
      double stopped = stop ? 1.0 : 0.0;
      if (stop) std::fclose(stop);
      rc = red(HIPFT_RED_MAX, &stopped);  // every rank stops at the same step
      if (rc) return rc;
      if (stopped > 0.0) {
        std::printf(" ### NOTE: The run was stopped prematurely via STOPRUN!\n");
        break;
      }
    }
    return HIPFT_OK;
  }
};

}  // namespace
}  // namespace hipft

extern "C" int hipft_run_shard(const char *namelist_path, const char *run_dir, int device,
                               const hipft_shard *shard, double *f_out, size_t f_len) {
  if (!namelist_path || !run_dir) return HIPFT_EINVAL;
  if (shard && (shard->nranks < 1 || shard->rank < 0 || shard->rank >= shard->nranks || !shard->allreduce ||
                !shard->gather))
    return HIPFT_EINVAL;
  hipft::Run r;
  r.dir = run_dir;
  if (shard) {
    r.shard = shard;
    r.rank = shard->rank;
    r.nranks = shard->nranks;
  }
  std::string err;
  if (!hipft::read_namelist(namelist_path, r.nl, err)) {
    std::fprintf(stderr, "### ERROR in READ_INPUT_FILE: %s\n", err.c_str());
    return HIPFT_EINVAL;
  }
  int rc = r.setup(device);
  if (rc == HIPFT_OK) rc = r.main_loop();
  if (rc == HIPFT_OK) rc = r.write_map(r.nl.output_map_root_filename + "_final.h5");  // wrap_it_up
  if (rc == HIPFT_OK && f_out) {
    hipft_info inf;
    hipft_gpu_info(r.h, &inf);
    if (f_len != (size_t)inf.ntm * inf.npm * inf.nr) rc = HIPFT_EINVAL;
    else rc = hipft_gpu_get_field(r.h, f_out);
  }
  if (rc != HIPFT_OK) {
    char msg[512] = "";
    if (r.h) hipft_gpu_last_error(r.h, msg, sizeof msg);
    std::fprintf(stderr, "### ERROR in HIPFT (code %d): %s %s\n", rc, r.err.c_str(), msg);
  }
  hipft_gpu_destroy(r.h);
  return rc;
}

extern "C" int hipft_run_field(const char *namelist_path, const char *run_dir, int device, double *f_out,
                               size_t f_len) {
  return hipft_run_shard(namelist_path, run_dir, device, nullptr, f_out, f_len);
}

extern "C" int hipft_run(const char *namelist_path, const char *run_dir, int device) {
  return hipft_run_shard(namelist_path, run_dir, device, nullptr, nullptr, 0);
}
