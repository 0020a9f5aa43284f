// namelist.h -- the &hipft_input_parameters group of hipft.in.
//
// Names, defaults and the per-realization fill-in follow the reference's
// input_parameters module (src/hipft.f90:493-726) and
// process_input_parameters (src/hipft.f90:8458-8614).
#pragma once
#include <string>
#include <vector>

namespace hipft {

constexpr int kMaxRealizations = 2000;  // src/hipft.f90:236

struct Namelist {
  int verbose = 0;
  int res_nt = 0, res_np = 0;
  int n_realizations = 1;
  int validation_run = 0;
  double validation_run_width = 0.03;
  std::string initial_map_filename;
  bool initial_map_flux_balance = false;
  double initial_map_mult_fac = 1.0;
  std::string output_map_root_filename = "hipft_brmap";
  std::string output_map_directory = "output_maps";
  bool output_map_flux_balance = false;
  long output_map_idx_start = 1;
  long output_map_idx_cadence = 0;
  double output_map_time_cadence = 0.0;
  bool output_map_2d = true;
  double output_history_time_cadence = 0.0;
  bool output_single_precision = true;
  double time_start = 0.0, time_end = 1.0;
  double dt_min = 1.0e-15, dt_max = 1.7976931348623157e308;
  bool strang_splitting = false;
  // not a reference key: every realization keeps its own diffusion schedule
  // (hipft_gpu_set_ragged); the histories then report each one's own
  bool ragged_realizations = false;
  double pole_flux_lat_limit = 30.0;
  bool advance_flow = false;
  double flow_vp_rigid_omega = 0.0, flow_rigid_omega = 0.0, flow_vt_const = 0.0;
  bool flow_attenuate = false;
  double flow_attenuate_value = 500.0;
  int flow_dr_model = 0, flow_mf_model = 0;
  double flow_dr_coef_p0_value = 46.0, flow_dr_coef_p2_value = -262.0,
         flow_dr_coef_p4_value = -379.0;
  double flow_mf_coef_p1_value = 22.0, flow_mf_coef_p3_value = 11.0,
         flow_mf_coef_p5_value = -28.0;
  bool use_flow_from_files = false;
  std::string flow_list_filename, flow_root_dir = ".";
  int flow_num_method = 4;
  double upwind = 1.0, weno_eps = 0.0;
  bool advance_diffusion = false;
  double diffusion_coef_constant = 0.0;
  std::string diffusion_coef_filename;
  bool diffusion_coef_grid = false;
  double diffusion_coef_factor = 7.43162901307967e-09;
  int diffusion_num_method = 3;
  int diffusion_subcycles = 0;
  bool advance_source = false;
  int source_rfe_model = 0;
  long source_rfe_seed = -9999;
  double source_rfe_total_unsigned_flux_per_hour = 0.0, source_rfe_lifetime = 0.3;
  bool source_from_file = false;
  std::string source_filename;
  std::vector<double> source_rfe_total_unsigned_flux_per_hours;
  bool assimilate_data = false, assimilate_data_balance_flux = false;
  double assimilate_data_mult_fac = 1.0;
  std::string assimilate_data_map_list_filename, assimilate_data_map_root_dir = ".";
  bool assimilate_data_add = false, assimilate_data_custom_from_mu = false;
  double assimilate_data_lat_limit = 0.0, assimilate_data_mu_power = 4.0,
         assimilate_data_mu_limit = 0.1;
  // Per-realization vectors, resized to n_realizations after processing.
  std::vector<double> diffusion_coef_constants, flow_attenuate_values, flow_dr_coef_p0_values,
      flow_dr_coef_p2_values, flow_dr_coef_p4_values, flow_mf_coef_p1_values,
      flow_mf_coef_p3_values, flow_mf_coef_p5_values, assimilate_data_lat_limits,
      assimilate_data_mu_powers, assimilate_data_mu_limits;
};

// Parses the namelist text; unknown names are reported through `err`.
// Returns false on a syntax error or an invalid setting.
bool parse_namelist(const std::string &text, Namelist &nl, std::string &err);
// Reads and parses a file.
bool read_namelist(const std::string &path, Namelist &nl, std::string &err);

}  // namespace hipft
