/*
 * hipft_oracle.c -- CPU restatement of HipFT's flux-transport time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: it restates,
 * routine by routine and in the same loop order and constants, the
 * reference's Fortran solver (src/hipft.f90, v1.19.3).  Only the tests,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py may load it;
 * nothing in the hipft_b200 product links it or falls back to it.
 *
 * Pinned against the reference testsuite's golden histories
 * (testsuite/<case>/reference/hipft_history_{sol,num}_r00000N.out, 16
 * significant digits, every step) by tests/test_oracle_golden.py.
 *
 * Indexing follows the Fortran: 1-based macros over column-major storage,
 * f(ntm,npm,nr) with theta fastest.  Compile with -ffp-contract=off so that
 * a*b+c is never fused (the GPU library is built with --fmad=false to match).
 *
 * Citations are "F:line" into src/hipft.f90.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <stdint.h>

/* ---------------------------------------------------------------- constants
 * F:83-136 */
static const double zero = 0.0, one = 1.0, two = 2.0, three = 3.0,
                    four = 4.0, six = 6.0, nine = 9.0, ten = 10.0,
                    fifteen = 15.0, sixteen = 16.0, half = 0.5,
                    quarter = 0.25, twentyfour = 24.0, twentyfive = 25.0,
                    three_quarter = 0.75;
static const double sixth = 0.16666666666666666;
static const double two_third = 0.66666666666666666;
static const double third = 0.33333333333333333;
static const double pi = 3.1415926535897932;
static const double pi_two = 1.5707963267948966;
static const double pi_four = 0.7853981633974483;
static const double pi_i = 0.3183098861837907;
static const double twopi = 6.2831853071795864;
static const double twopi_i = 0.15915494309189535;
static const double threepi_two = 4.71238898038469;
static const double threepi_four = 2.356194490192345;
static const double d2r = 0.017453292519943295;
static const double rsun_cm2 = 4.84416e21;
static const double km_s_to_rs_hr = 0.005172413793103448;
static const double m_s_to_rs_hr = 5.172413793103448e-06;
static const double safety = 0.95;
#define SMALL_VALUE DBL_MIN
#define LARGE_VALUE DBL_MAX

/* ------------------------------------------------------------------ params */
typedef struct {
  int verbose;
  int res_nt, res_np, n_realizations;
  int validation_run;
  double validation_run_width;
  int initial_map_flux_balance;
  double initial_map_mult_fac;
  double output_map_time_cadence;
  long output_map_idx_cadence, output_map_idx_start;
  double output_history_time_cadence;
  double time_start, time_end, dt_min, dt_max;
  int strang_splitting;
  double pole_flux_lat_limit;
  int advance_flow;
  double flow_vp_rigid_omega, flow_rigid_omega, flow_vt_const;
  int flow_attenuate;
  int flow_dr_model, flow_mf_model;
  int flow_num_method;
  double upwind, weno_eps;
  int advance_diffusion;
  double diffusion_coef_factor;
  int diffusion_coef_grid;
  int diffusion_num_method, diffusion_subcycles;
  int assimilate_data, assimilate_data_balance_flux, assimilate_data_add,
      assimilate_data_custom_from_mu;
  double assimilate_data_mult_fac;
  /* per-realization parameter vectors, length n_realizations (F:2252-2344) */
  const double *diffusion_coef_constants, *flow_attenuate_values,
      *flow_dr_coef_p0_values, *flow_dr_coef_p2_values,
      *flow_dr_coef_p4_values, *flow_mf_coef_p1_values,
      *flow_mf_coef_p3_values, *flow_mf_coef_p5_values,
      *assimilate_data_lat_limits, *assimilate_data_mu_powers,
      *assimilate_data_mu_limits;
  int output_map_flux_balance;
  /* flows from files (use_flow_from_files): the list's Julian days and the
   * files' contents in PT order, vt (npm1, nt) and vp (np, ntm) per entry, m/s */
  int use_flow_from_files, n_flows;
  const double *flow_jd, *flow_vt, *flow_vp;
  /* sources (advance_source): random flux emergence with a seeded generator
   * (seed -9999: seed 0), per-realization unsigned flux per hour; the source
   * file's data (nfp, nft) PT and its scales */
  int advance_source, source_rfe_model;
  long source_rfe_seed;
  double source_rfe_lifetime;
  const double *source_rfe_flux;
  int source_from_file, source_nfp, source_nft;
  const double *source_data, *source_pf, *source_tf;
} orc_params;

/* History rows, one block of nr rows per output event.
 * sol: [row][realization][16] = step,time,14 diagnostics (F:2676-2683)
 * num: [row][realization][8]  = step,time,dt,dtflow,dtadv,dteuler,s,sc */
typedef struct {
  long cap, nrows;
  double *sol, *num;
  /* maps the reference writes (write_map F:2801-2917), as f(ntm,npm,nr),
   * flux-balanced copies when output_map_flux_balance; NULL = not kept.
   * maps[map_cap]: numbered outputs with their index and time. */
  long map_cap, n_maps;
  long *map_idx;
  double *map_time, *maps, *map_initial, *map_final;
} orc_hist;

/* ------------------------------------------------------------------ state */
typedef struct {
  const orc_params *P;
  int nr, nt, ntm, np, npm, npm1, ntm1;
  double *t, *p, *th, *ph, *dt, *dth, *dp, *dph, *dt_i, *dth_i, *dp_i, *dph_i;
  double *st, *sth, *ct, *cth, *st_i, *sth_i;
  double *f, *fval_u0; /* fval_u0 is PT (npm1,ntm,nr) */
  double time, dtime_global, dtmax_flow, dtime_advection_used;
  long ntime, idx_hist, idx_out;
  int timestep_needs_updating, timestep_flow_needs_updating, flow_needs_updating;
  int time_step_changed;
  int adv_time, adv_space; /* 1 FE 2 SSPRK33 3 SSPRK43 ; 1 UW 2 WENO3 */
  int output_current_map, output_current_history;
  double flow_vp_rigid_omega, flow_vt_const;
  /* flows */
  double *vt, *vp, *alpha_t, *alpha_p;
  double bc_flow_npole_fac, bc_flow_spole_fac;
  double *D_C_CPt, *D_C_MCt, *D_M_Tt, *D_CP_Tt, *D_P_Tt, *D_MC_Tt, *weno_eps_t;
  double *D_C_CPp, *D_C_MCp, *D_M_Tp, *D_CP_Tp, *D_P_Tp, *D_MC_Tp, *weno_eps_p;
  double *atten_i;
  /* sources (module sources F:290-304) and the generator of get_gaussian */
  double *source, *source_file, *source_rfe[2], *uf;
  int rfe1, rfe2;
  double time_of_next_source_rfe, time_of_prev_source_rfe;
  uint64_t rng[4];
  int g_second;
  double g_v, g_sln;
  /* flows from files: current pair (flow_from_files_current_vt/vp) and times */
  double *fvt, *fvp, *flow_times;
  int flow_idx;
  double time_of_current_input_flow, time_of_next_input_flow, flow_dt_last;
  /* diffusion */
  double *dcoef, *coef; /* dcoef (nt,np,nr); coef (2:ntm-1,2:npm-1,5,nr) */
  double bc_diffusion_npole_fac, bc_diffusion_spole_fac;
  double dtime_diffusion_euler;
  int auto_sc;
  long diffusion_subcycles;
  long sts_s;
  int need_to_load_sts;
  double *sts_uj, *sts_vj, *sts_ubj, *sts_gj, *sts_b;
  long n_stable_diffusion_cycles;
  /* analysis */
  double *h; /* [nr][14] */
  /* assimilation */
  int n_da, da_idx;
  const double *da_times, *da_maps;
  double time_of_next_input_map;
  int da_active;
  int *tidx0, *tidx1;
  orc_hist *hist;
  double cell_updates; /* unique cells x stages advanced (for throughput) */
} orc;

#define A3(a, j, k, i, n1, n2) \
  (a)[((size_t)(i)-1) * (size_t)(n2) * (size_t)(n1) + ((size_t)(k)-1) * (size_t)(n1) + (size_t)((j)-1)]
#define F(j, k, i) A3(S->f, j, k, i, S->ntm, S->npm)
#define V1(a, j) (a)[(j)-1]

static double *dalloc(size_t n) {
  double *x = (double *)calloc(n ? n : 1, sizeof(double));
  if (!x) { fprintf(stderr, "oracle: out of memory\n"); exit(3); }
  return x;
}

static double sgn(double a, double b) { return copysign(fabs(a), b); }
static double dmax(double a, double b) { return a > b ? a : b; }
static double dmin(double a, double b) { return a < b ? a : b; }
/* Fortran MODULO for reals */
static double fmodulo(double a, double p) { return a - floor(a / p) * p; }

/* --------------------------------------------------------------- set_mesh
 * F:6495-6653.  t(ntm), p(npm) must already be filled. */
static int set_mesh(orc *S) {
  int i;
  const double eps = 1.e-5;
  int ntm = S->ntm, npm = S->npm, nt = S->nt, np = S->np, ntm1 = S->ntm1,
      npm1 = S->npm1;
  if (fabs(V1(S->t, 1)) > eps || fabs(V1(S->t, ntm) - pi) > eps ||
      fabs(V1(S->p, 1)) > eps || fabs(V1(S->p, npm - 1) - twopi) > eps)
    return -1;
  S->dt = dalloc(ntm); S->dt_i = dalloc(ntm); S->st = dalloc(ntm);
  S->st_i = dalloc(ntm); S->ct = dalloc(ntm); S->dp = dalloc(npm);
  S->dp_i = dalloc(npm); S->th = dalloc(nt); S->ph = dalloc(np);
  S->dth = dalloc(nt); S->dth_i = dalloc(nt); S->sth = dalloc(nt);
  S->sth_i = dalloc(nt); S->cth = dalloc(nt); S->dph = dalloc(np);
  S->dph_i = dalloc(np);
  for (i = 2; i <= ntm1; i++) {
    V1(S->th, i) = half * (V1(S->t, i) + V1(S->t, i - 1));
    V1(S->dth, i) = V1(S->t, i) - V1(S->t, i - 1);
  }
  V1(S->th, 1) = V1(S->th, 2) - V1(S->dth, 2);
  V1(S->th, nt) = V1(S->th, ntm1) + V1(S->dth, ntm1);
  V1(S->dth, 1) = V1(S->dth, 2);
  V1(S->dth, nt) = V1(S->dth, ntm1);
  for (i = 1; i <= nt; i++) V1(S->dth_i, i) = one / V1(S->dth, i);
  for (i = 1; i <= ntm; i++) {
    V1(S->dt, i) = V1(S->th, i + 1) - V1(S->th, i);
    V1(S->dt_i, i) = one / V1(S->dt, i);
  }
  for (i = 1; i <= ntm; i++) V1(S->st, i) = sin(V1(S->t, i));
  V1(S->st, 1) = 0.; V1(S->st, ntm) = 0.;
  for (i = 1; i <= ntm; i++) V1(S->ct, i) = cos(V1(S->t, i));
  V1(S->ct, 1) = one; V1(S->ct, ntm) = one;
  for (i = 2; i <= ntm - 1; i++) V1(S->st_i, i) = one / V1(S->st, i);
  V1(S->st_i, 1) = 0.; V1(S->st_i, ntm) = 0.;
  for (i = 1; i <= nt; i++) V1(S->sth, i) = sin(fabs(V1(S->th, i)));
  for (i = 2; i <= ntm1; i++) V1(S->sth_i, i) = one / V1(S->sth, i);
  V1(S->sth_i, 1) = 0.; V1(S->sth_i, nt) = 0.;
  for (i = 1; i <= nt; i++) V1(S->cth, i) = cos(V1(S->th, i));
  for (i = 2; i <= np; i++) {
    V1(S->ph, i) = half * (V1(S->p, i) + V1(S->p, i - 1));
    V1(S->dph, i) = V1(S->p, i) - V1(S->p, i - 1);
  }
  V1(S->ph, 1) = V1(S->ph, npm1) - twopi;
  V1(S->dph, 1) = V1(S->dph, npm1);
  for (i = 1; i <= np; i++) V1(S->dph_i, i) = one / V1(S->dph, i);
  for (i = 1; i <= npm - 1; i++) V1(S->dp, i) = V1(S->ph, i + 1) - V1(S->ph, i);
  V1(S->dp, npm) = V1(S->dp, 2);
  for (i = 1; i <= npm; i++) V1(S->dp_i, i) = one / V1(S->dp, i);
  return 0;
}

/* ------------------------------------------------------- periodic seams
 * F:4841-4925 */
static void set_periodic_bc_1d(double *a, int n1) {
  V1(a, 1) = V1(a, n1 - 1);
  V1(a, n1) = V1(a, 2);
}
static void set_periodic_bc_3d(double *a, int n1, int n2, int n3) {
  for (int j = 1; j <= n1; j++)
    for (int i = 1; i <= n3; i++) {
      A3(a, j, 1, i, n1, n2) = A3(a, j, n2 - 1, i, n1, n2);
      A3(a, j, n2, i, n1, n2) = A3(a, j, 2, i, n1, n2);
    }
}

/* ------------------------------------------ tesseral spherical harmonic
 * F:2390-2533 (Holmes & Featherstone 2002 forward column recursion).
 * Y(np,nt) with phi fastest. */
static void tesseral_spherical_harmonic(int m, int l, const double *pvec,
                                        const double *tvec, int np, int nt,
                                        double *Y) {
  const double lpi = 3.141592653589793;
  int abs_m = abs(m), i, im, il, j;
  double *cos_t = dalloc(nt), *Pold = dalloc(nt), *Poldold = dalloc(nt);
  for (i = 0; i < nt; i++) {
    cos_t[i] = cos(tvec[i]);
    Pold[i] = 1.0;
    Poldold[i] = 0.;
  }
  if (abs_m > 0) {
    for (i = 0; i < nt; i++) Pold[i] = sqrt(3.0);
    for (im = 2; im <= abs_m; im++)
      for (i = 0; i < nt; i++)
        Pold[i] = sqrt((2.0 * im + 1.0) / (2.0 * im)) * Pold[i];
  }
  for (il = abs_m + 1; il <= l; il++) {
    double anm = sqrt(((2.0 * il - 1.0) * (2.0 * il + 1.0)) /
                      (double)((il - abs_m) * (il + abs_m)));
    double bnm = sqrt(((2.0 * il + 1.0) * (il + abs_m - 1.0) * (il - abs_m - 1.0)) /
                      ((il - abs_m) * (il + abs_m) * (2.0 * il - 3.0)));
    for (i = 0; i < nt; i++) {
      double Pl = anm * cos_t[i] * Pold[i] - bnm * Poldold[i];
      Poldold[i] = Pold[i];
      Pold[i] = Pl;
    }
  }
  double one_over_sqrt_4pi = 1.0 / sqrt(4.0 * lpi);
  for (i = 0; i < nt; i++) {
    double s = sin(tvec[i]), sp = 1.0;
    for (im = 0; im < abs_m; im++) sp *= s;
    double sgnm = (abs_m % 2) ? -1.0 : 1.0;
    Pold[i] = (sgnm * sp) * one_over_sqrt_4pi * Pold[i];
  }
  int pos = (m + 1 >= 0) ? 1 : 0;
  for (j = 0; j < nt; j++)
    for (i = 0; i < np; i++)
      Y[(size_t)j * np + i] =
          Pold[j] * (pos * cos(m * pvec[i]) + (1.0 - pos) * sin(abs_m * pvec[i]));
  free(cos_t); free(Pold); free(Poldold);
}

/* --------------------------------------------------------------- get_flux
 * F:8672-8750 on one realization's (ntm,npm) slab */
static void get_flux(orc *S, const double *map, double *flux_p, double *flux_m) {
  int ntm = S->ntm, npm = S->npm;
  double fp = zero, fm = zero;
  for (int k = 1; k <= npm - 1; k++)
    for (int j = 1; j <= ntm; j++) {
      double da_t, da_p;
      if (j == 1) {
        double tav = half * (V1(S->t, 1) + V1(S->t, 2));
        da_t = quarter * sin(tav) * V1(S->dth, 2);
      } else if (j == ntm) {
        double tav = half * (V1(S->t, ntm) + V1(S->t, ntm - 1));
        da_t = quarter * sin(tav) * V1(S->dth, ntm);
      } else {
        da_t = V1(S->st, j) * V1(S->dt, j);
      }
      if (k == 1) da_p = half * V1(S->dph, 1);
      else if (k == npm - 1) da_p = half * V1(S->dph, npm - 1);
      else da_p = V1(S->dp, k);
      double fv = map[(size_t)(k - 1) * ntm + (j - 1)] * da_t * da_p;
      if (fv > zero) fp = fp + fv; else fm = fm + fv;
    }
  *flux_p = fp;
  *flux_m = fm;
}

/* F:8752-8807 */
static void balance_flux(orc *S, double *map) {
  double fp, fm;
  get_flux(S, map, &fp, &fm);
  if (fm + fp == zero) return;
  double ratio = sqrt(fabs(fp / fm));
  size_t n = (size_t)S->ntm * S->npm;
  for (size_t q = 0; q < n; q++) {
    double br = map[q];
    map[q] = (br > 0) ? br / ratio : br * ratio;
  }
}

/* ----------------------------------------------------- analysis_step
 * F:3098-3336.  Fills S->h[nr][14]. */
static void analysis_step(orc *S) {
  const orc_params *P = S->P;
  int ntm = S->ntm, npm = S->npm, nr = S->nr, npm1 = S->npm1;
  double *fval = dalloc((size_t)(npm - 1) * ntm * nr); /* fval(npm-1,ntm,nr) */
#define FVAL(i, j, k) fval[((size_t)(k)-1) * (npm - 1) * ntm + ((size_t)(j)-1) * (npm - 1) + ((i)-1)]
  if (P->validation_run == 1) {
    for (int k = 1; k <= nr; k++) {
      double e = exp(-42.0 * P->diffusion_coef_constants[k - 1] *
                     P->diffusion_coef_factor * (S->time - P->time_start));
      for (int j = 1; j <= ntm; j++)
        for (int i = 1; i <= npm - 1; i++)
          FVAL(i, j, k) = S->fval_u0[((size_t)(k - 1) * ntm + (j - 1)) * npm1 + (i - 1)] * e;
    }
  } else if (P->validation_run == 2) {
    double w = P->validation_run_width;
    for (int k = 1; k <= nr; k++)
      for (int j = 1; j <= ntm; j++)
        for (int i = 1; i <= npm - 1; i++) {
          double vtt = S->flow_vt_const * km_s_to_rs_hr * (S->time - P->time_start);
          double vpt = S->flow_vp_rigid_omega * km_s_to_rs_hr * (S->time - P->time_start);
          double p1 = fmodulo(pi_two + vpt, twopi);
          double p2 = fmodulo(threepi_two + vpt, twopi);
          double a = V1(S->t, j) - pi_four - vtt;
          double b1 = V1(S->p, i) - p1, b2 = V1(S->p, i) - p2;
          FVAL(i, j, k) = -V1(S->st_i, j) * exp(-(a * a) / w - (b1 * b1) / w) +
                          V1(S->st_i, j) * exp(-(a * a) / w - (b2 * b2) / w);
        }
  } else {
    for (int k = 1; k <= nr; k++)
      for (int j = 1; j <= ntm; j++)
        for (int i = 1; i <= npm - 1; i++) FVAL(i, j, k) = F(j, i, k);
  }
  for (int k = 1; k <= nr; k++) {
    double mn = LARGE_VALUE, mx = SMALL_VALUE, mnabs = LARGE_VALUE, verr = zero,
           sumfval2 = zero;
    for (int j = 1; j <= npm - 2; j++)
      for (int i = 1; i <= ntm; i++) {
        double fij = F(i, j, k);
        mn = dmin(fij, mn);
        mx = dmax(fij, mx);
        mnabs = dmin(fabs(fij), mnabs);
        double d = fij - FVAL(j, i, k);
        double fv = d * d;
        double fv2 = fabs(fij) * fabs(FVAL(j, i, k));
        verr = verr + fv;
        sumfval2 = sumfval2 + fv2;
      }
    double *h = S->h + (size_t)(k - 1) * 14;
    h[0] = mn; h[1] = mx; h[2] = mnabs;
    if (sumfval2 == zero) h[13] = sqrt(verr / ((double)ntm * (npm - 1)));
    else h[13] = sqrt(verr / sumfval2);
  }
  free(fval);
#undef FVAL
  for (int k = 1; k <= nr; k++) {
    double fxp = 0, fxm = 0, fxp_pn = 0, fxm_pn = 0, fxp_ps = 0, fxm_ps = 0,
           a_pn = 0, a_ps = 0, eqd1 = 0, eqd2 = 0, axd = 0;
    for (int i = 1; i <= npm - 1; i++)
      for (int j = 1; j <= ntm; j++) {
        double tav, sn_t, cs_t, d_t, da_t, da_p;
        if (j == 1) {
          tav = half * (V1(S->t, 1) + V1(S->t, 2));
          sn_t = sin(tav); cs_t = cos(tav); d_t = V1(S->dth, 2);
          da_t = quarter * sn_t * d_t;
        } else if (j == ntm) {
          tav = half * (V1(S->t, ntm) + V1(S->t, ntm - 1));
          sn_t = sin(tav); cs_t = cos(tav); d_t = V1(S->dth, ntm);
          da_t = quarter * sn_t * d_t;
        } else {
          sn_t = sin(V1(S->t, j)); cs_t = cos(V1(S->t, j)); d_t = V1(S->dt, j);
          da_t = sn_t * d_t;
        }
        if (i == 1) da_p = half * V1(S->dph, 1);
        else if (i == npm - 1) da_p = half * V1(S->dph, npm - 1);
        else da_p = V1(S->dp, i);
        double cs_p = cos(V1(S->p, i)), sn_p = sin(V1(S->p, i));
        double fji = F(j, i, k);
        double fv = fji * da_t * da_p;
        if (fv > 0.) fxp = fxp + fv; else fxm = fxm + fv;
        if (V1(S->t, j) <= P->pole_flux_lat_limit * d2r) {
          if (fv > 0.) fxp_pn = fxp_pn + fv; else fxm_pn = fxm_pn + fv;
          a_pn = a_pn + da_t * da_p;
        }
        if (V1(S->t, j) >= pi - P->pole_flux_lat_limit * d2r) {
          if (fv > 0.) fxp_ps = fxp_ps + fv; else fxm_ps = fxm_ps + fv;
          a_ps = a_ps + da_t * da_p;
        }
        eqd1 = eqd1 + fji * sn_t * cs_p * da_t * da_p;
        eqd2 = eqd2 + fji * sn_t * sn_p * da_t * da_p;
        axd = axd + fji * cs_t * da_t * da_p;
      }
    double *h = S->h + (size_t)(k - 1) * 14;
    h[3] = rsun_cm2 * fxp; h[4] = rsun_cm2 * fxm;
    h[5] = rsun_cm2 * fxp_pn; h[6] = rsun_cm2 * fxm_pn;
    h[7] = rsun_cm2 * fxp_ps; h[8] = rsun_cm2 * fxm_ps;
    h[9] = rsun_cm2 * a_pn; h[10] = rsun_cm2 * a_ps;
    h[12] = three_quarter * pi_i * axd;
    eqd1 = three_quarter * pi_i * eqd1;
    eqd2 = three_quarter * pi_i * eqd2;
    h[11] = sqrt(eqd1 * eqd1 + eqd2 * eqd2);
  }
}

static int history_due(orc *S) {
  const orc_params *P = S->P;
  if (P->output_history_time_cadence > 0.0)
    return S->time >= P->time_start + S->idx_hist * P->output_history_time_cadence;
  return 1;
}

/* analysis_step + output_histories (F:3135-3145, F:2637-2690) */
static void analysis_and_history(orc *S) {
  if (!history_due(S)) return;
  analysis_step(S);
  S->idx_hist++;
  orc_hist *H = S->hist;
  if (!H || H->nrows >= H->cap) { if (H) H->nrows++; return; }
  for (int i = 0; i < S->nr; i++) {
    double *srow = H->sol + ((size_t)H->nrows * S->nr + i) * 16;
    double *nrow = H->num + ((size_t)H->nrows * S->nr + i) * 8;
    srow[0] = (double)S->ntime; srow[1] = S->time;
    memcpy(srow + 2, S->h + (size_t)i * 14, 14 * sizeof(double));
    long niters = (S->P->diffusion_num_method == 1) ? S->n_stable_diffusion_cycles : S->sts_s;
    nrow[0] = (double)S->ntime; nrow[1] = S->time; nrow[2] = S->dtime_global;
    nrow[3] = S->dtmax_flow; nrow[4] = S->dtime_advection_used;
    nrow[5] = S->dtime_diffusion_euler; nrow[6] = (double)niters;
    nrow[7] = (double)S->diffusion_subcycles;
  }
  H->nrows++;
}

/* ------------------------------------------------------------ load_weno
 * F:6846-6938 */
static void load_weno(orc *S) {
  int nt = S->nt, np = S->np, ntm = S->ntm, npm = S->npm, nr = S->nr;
  S->alpha_t = dalloc((size_t)ntm * npm * nr);
  S->alpha_p = dalloc((size_t)ntm * npm * nr);
  S->D_C_CPt = dalloc(nt); S->D_C_MCt = dalloc(nt); S->D_M_Tt = dalloc(nt);
  S->D_CP_Tt = dalloc(nt); S->D_P_Tt = dalloc(nt); S->D_MC_Tt = dalloc(nt);
  S->weno_eps_t = dalloc(ntm);
  S->D_C_CPp = dalloc(np); S->D_C_MCp = dalloc(np); S->D_M_Tp = dalloc(np);
  S->D_CP_Tp = dalloc(np); S->D_P_Tp = dalloc(np); S->D_MC_Tp = dalloc(np);
  S->weno_eps_p = dalloc(npm);
  for (int j = 1; j <= ntm; j++)
    V1(S->weno_eps_t, j) = (S->P->weno_eps <= 0.) ? V1(S->dt, j) : S->P->weno_eps;
  for (int k = 1; k <= npm; k++)
    V1(S->weno_eps_p, k) = (S->P->weno_eps <= 0.) ? V1(S->dp, k) : S->P->weno_eps;
  for (int j = 2; j <= nt - 2; j++) {
    double *d = S->dt;
    double tot = V1(d, j - 1) + V1(d, j) + V1(d, j + 1);
    V1(S->D_C_CPt, j) = V1(d, j) / (V1(d, j) + V1(d, j + 1));
    V1(S->D_C_MCt, j) = V1(d, j) / (V1(d, j - 1) + V1(d, j));
    V1(S->D_M_Tt, j) = V1(d, j - 1) / tot;
    V1(S->D_CP_Tt, j) = (V1(d, j) + V1(d, j + 1)) / tot;
    V1(S->D_P_Tt, j) = V1(d, j + 1) / tot;
    V1(S->D_MC_Tt, j) = (V1(d, j - 1) + V1(d, j)) / tot;
  }
  for (int k = 2; k <= np - 1; k++) {
    double *d = S->dp;
    double tot = V1(d, k - 1) + V1(d, k) + V1(d, k + 1);
    V1(S->D_C_CPp, k) = V1(d, k) / (V1(d, k) + V1(d, k + 1));
    V1(S->D_C_MCp, k) = V1(d, k) / (V1(d, k - 1) + V1(d, k));
    V1(S->D_M_Tp, k) = V1(d, k - 1) / tot;
    V1(S->D_CP_Tp, k) = (V1(d, k) + V1(d, k + 1)) / tot;
    V1(S->D_P_Tp, k) = V1(d, k + 1) / tot;
    V1(S->D_MC_Tp, k) = (V1(d, k - 1) + V1(d, k)) / tot;
  }
  set_periodic_bc_1d(S->D_C_CPp, np); set_periodic_bc_1d(S->D_C_MCp, np);
  set_periodic_bc_1d(S->D_M_Tp, np); set_periodic_bc_1d(S->D_CP_Tp, np);
  set_periodic_bc_1d(S->D_P_Tp, np); set_periodic_bc_1d(S->D_MC_Tp, np);
}

/* -------------------------------------------------------- set_lf_alpha
 * F:6940-7048 */
static void set_lf_alpha(orc *S) {
  int nt = S->nt, np = S->np, ntm = S->ntm, npm = S->npm, nr = S->nr;
#define VT(j, k, i) fabs(A3(S->vt, j, k, i, nt, npm))
#define VP(j, k, i) fabs(A3(S->vp, j, k, i, ntm, np))
#define AT(j, k, i) A3(S->alpha_t, j, k, i, ntm, npm)
#define AP(j, k, i) A3(S->alpha_p, j, k, i, ntm, npm)
#pragma omp parallel for
  for (int i = 1; i <= nr; i++) {
    for (int k = 1; k <= npm; k++) {
      for (int j = 3; j <= nt - 3; j++)
        AT(j, k, i) = dmax(dmax(dmax(dmax(dmax(VT(j - 2, k, i), VT(j - 1, k, i)), VT(j, k, i)),
                                     VT(j + 1, k, i)), VT(j + 2, k, i)), VT(j + 3, k, i));
      int j = 1;
      AT(j, k, i) = dmax(dmax(dmax(VT(j, k, i), VT(j + 1, k, i)), VT(j + 2, k, i)), VT(j + 3, k, i));
      j = 2;
      AT(j, k, i) = dmax(dmax(dmax(dmax(VT(j - 1, k, i), VT(j, k, i)), VT(j + 1, k, i)),
                              VT(j + 2, k, i)), VT(j + 3, k, i));
      j = nt - 2;
      AT(j, k, i) = dmax(dmax(dmax(dmax(VT(j - 2, k, i), VT(j - 1, k, i)), VT(j, k, i)),
                              VT(j + 1, k, i)), VT(j + 2, k, i));
      j = nt - 1;
      AT(j, k, i) = dmax(dmax(dmax(VT(j - 2, k, i), VT(j - 1, k, i)), VT(j, k, i)), VT(j + 1, k, i));
    }
    for (int k = 3; k <= np - 3; k++)
      for (int j = 2; j <= ntm - 1; j++)
        AP(j, k, i) = dmax(dmax(dmax(dmax(dmax(VP(j, k - 2, i), VP(j, k - 1, i)), VP(j, k, i)),
                                     VP(j, k + 1, i)), VP(j, k + 2, i)), VP(j, k + 3, i));
    for (int j = 2; j <= ntm - 1; j++) {
      int k = 2;
      AP(j, k, i) = dmax(dmax(dmax(dmax(dmax(VP(j, np - 2, i), VP(j, k - 1, i)), VP(j, k, i)),
                                   VP(j, k + 1, i)), VP(j, k + 2, i)), VP(j, k + 3, i));
      k = np - 2;
      AP(j, k, i) = dmax(dmax(dmax(dmax(dmax(VP(j, k - 2, i), VP(j, k - 1, i)), VP(j, k, i)),
                                   VP(j, k + 1, i)), VP(j, k + 2, i)), VP(j, 3, i));
      k = np - 1;
      AP(j, k, i) = dmax(dmax(dmax(dmax(dmax(VP(j, k - 2, i), VP(j, k - 1, i)), VP(j, k, i)),
                                   VP(j, k + 1, i)), VP(j, 3, i)), VP(j, 4, i));
    }
  }
  set_periodic_bc_3d(S->alpha_p, ntm, npm, nr);
#undef VT
#undef VP
#undef AT
#undef AP
}

/* --------------------------------------------------------- update_flow
 * F:3371-3523 with add_flow_*_analytic F:7219-7285 */
/* One pair of flow files into fvt, fvp: add_flow_from_files F:3578-3634
 * (at_load = 0: set_periodic_bc_3d on both) and load_flow_from_files
 * F:3775-3800 (at_load = 1: only vt's column npm from column 2). */
static void read_flow_pair(orc *S, int idx, int at_load) {
  const orc_params *P = S->P;
  int nt = S->nt, ntm = S->ntm, npm = S->npm, np = S->np, npm1 = S->npm1, nr = S->nr;
  const double *ft = P->flow_vt + (size_t)(idx - 1) * npm1 * nt;
  const double *fp = P->flow_vp + (size_t)(idx - 1) * np * ntm;
  for (int k = 1; k <= nr; k++) {
    for (int j = 1; j <= npm1; j++)
      for (int i = 1; i <= nt; i++)
        A3(S->fvt, i, j, k, nt, npm) = m_s_to_rs_hr * ft[(size_t)(i - 1) * npm1 + (j - 1)];
    for (int j = 1; j <= np; j++)
      for (int i = 1; i <= ntm; i++)
        A3(S->fvp, i, j, k, ntm, np) = m_s_to_rs_hr * fp[(size_t)(i - 1) * np + (j - 1)];
  }
  if (at_load) {
    for (int k = 1; k <= nr; k++)
      for (int i = 1; i <= nt; i++) A3(S->fvt, i, npm, k, nt, npm) = A3(S->fvt, i, 2, k, nt, npm);
  } else {
    set_periodic_bc_3d(S->fvt, nt, npm, nr);
    set_periodic_bc_3d(S->fvp, ntm, np, nr);
  }
}

/* load_flow_from_files F:3675-3800 (times as the reference computes them). */
static void load_flow_from_files(orc *S) {
  const orc_params *P = S->P;
  int n = P->n_flows;
  S->flow_times = dalloc(n);
  for (int i = 0; i < n; i++) S->flow_times[i] = twentyfour * P->flow_jd[i];
  /* F:3750-3753: in place and in order, so entries after the first subtract
   * the already-zeroed first entry (no effect when the list starts at 0) */
  for (int i = 0; i < n; i++) S->flow_times[i] = S->flow_times[i] - S->flow_times[0];
  double span = S->flow_times[n - 1] - S->flow_times[0];
  double tsf = P->time_start - floor(P->time_start / span) * span; /* MODULO */
  int idx = 0;
  double best = fabs(S->flow_times[0] - tsf);
  for (int i = 1; i < n; i++)
    if (fabs(S->flow_times[i] - tsf) < best) { best = fabs(S->flow_times[i] - tsf); idx = i; }
  idx += 1; /* 1-based */
  if (S->flow_times[idx - 1] > tsf) idx -= 1;
  S->flow_idx = idx;
  S->fvt = dalloc((size_t)S->nt * S->npm * S->nr);
  S->fvp = dalloc((size_t)S->ntm * S->np * S->nr);
  read_flow_pair(S, idx, 1);
  S->flow_dt_last = S->flow_times[n - 1] - S->flow_times[n - 2];
  S->time_of_current_input_flow = P->time_start - tsf + S->flow_times[idx - 1];
  double delta = (idx + 1 > n) ? S->flow_dt_last : S->flow_times[idx] - S->flow_times[idx - 1];
  S->time_of_next_input_flow = S->time_of_current_input_flow + delta;
}

/* add_flow_from_files F:3525-3673 */
static void add_flow_from_files(orc *S) {
  const orc_params *P = S->P;
  int n = P->n_flows;
  if (S->time >= S->time_of_next_input_flow) {
    S->flow_idx += 1;
    if (S->flow_idx > n) S->flow_idx = 1;
    read_flow_pair(S, S->flow_idx, 0);
    S->time_of_current_input_flow = S->time_of_next_input_flow;
    double delta = (S->flow_idx + 1 > n) ? S->flow_dt_last
                                         : S->flow_times[S->flow_idx] - S->flow_times[S->flow_idx - 1];
    S->time_of_next_input_flow = S->time_of_current_input_flow + delta;
  }
  size_t nv = (size_t)S->nt * S->npm * S->nr, np_ = (size_t)S->ntm * S->np * S->nr;
  for (size_t q = 0; q < nv; q++) S->vt[q] = S->vt[q] + S->fvt[q];
  for (size_t q = 0; q < np_; q++) S->vp[q] = S->vp[q] + S->fvp[q];
}

static void update_flow(orc *S) {
  const orc_params *P = S->P;
  int nt = S->nt, np = S->np, ntm = S->ntm, npm = S->npm, nr = S->nr;
  if (!S->flow_needs_updating) return;
  S->flow_needs_updating = 0;
  S->timestep_flow_needs_updating = 1;
  S->timestep_needs_updating = 1;
  memset(S->vt, 0, sizeof(double) * (size_t)nt * npm * nr);
  memset(S->vp, 0, sizeof(double) * (size_t)ntm * np * nr);
  if (P->use_flow_from_files) { /* F:3417-3420: first, it overwrites */
    add_flow_from_files(S);
    S->flow_needs_updating = 1;
  }
  if (P->flow_mf_model == 1) {
    for (int i = 1; i <= nr; i++)
      for (int k = 1; k <= npm; k++)
        for (int j = 1; j <= nt; j++) {
          double c = V1(S->cth, j);
          double c3 = c * c * c, c5 = c * c * c * c * c;
          A3(S->vt, j, k, i, nt, npm) =
              A3(S->vt, j, k, i, nt, npm) -
              m_s_to_rs_hr * V1(S->sth, j) *
                  (P->flow_mf_coef_p1_values[i - 1] * c +
                   P->flow_mf_coef_p3_values[i - 1] * c3 +
                   P->flow_mf_coef_p5_values[i - 1] * c5);
        }
  }
  if (P->flow_dr_model == 1) {
    for (int i = 1; i <= nr; i++)
      for (int k = 1; k <= np; k++)
        for (int j = 1; j <= ntm; j++) {
          double c = V1(S->ct, j);
          double c2 = c * c, c4 = c2 * c2;
          A3(S->vp, j, k, i, ntm, np) =
              A3(S->vp, j, k, i, ntm, np) +
              m_s_to_rs_hr * V1(S->st, j) *
                  (P->flow_dr_coef_p0_values[i - 1] +
                   P->flow_dr_coef_p2_values[i - 1] * c2 +
                   P->flow_dr_coef_p4_values[i - 1] * c4);
        }
  }
  if (S->flow_vp_rigid_omega != 0.) {
    for (int i = 1; i <= nr; i++)
      for (int k = 1; k <= np; k++)
        for (int j = 1; j <= ntm; j++)
          A3(S->vp, j, k, i, ntm, np) = A3(S->vp, j, k, i, ntm, np) +
                                        S->flow_vp_rigid_omega * km_s_to_rs_hr * V1(S->st, j);
  }
  if (S->flow_vt_const != 0.) {
    for (int i = 1; i <= nr; i++)
      for (int k = 1; k <= npm; k++)
        for (int j = 1; j <= nt; j++)
          A3(S->vt, j, k, i, nt, npm) = A3(S->vt, j, k, i, nt, npm) + S->flow_vt_const * km_s_to_rs_hr;
  }
  if (P->flow_rigid_omega != 0.) {
    double vr = P->flow_rigid_omega * km_s_to_rs_hr;
    for (int i = 1; i <= nr; i++)
      for (int k = 1; k <= npm; k++)
        for (int j = 1; j <= nt; j++) {
          double cp = cos(V1(S->p, k)), c = V1(S->cth, j), s = V1(S->sth, j);
          double acp = fabs(cp);
          double p1 = -2 * c * fabs(s * cp);
          double p2 = (cp * c * c - cp) * acp * acp * acp;
          double p3 = (-3 * cp * c * c + 2 * cp) * acp;
          double p4 = sgn(one, cp) * c * c;
          double p5 = 2 * acp * acp * acp * c * fabs(s);
          double p6 = (-cp * cp * cp * cp + 3 * cp * cp - 1) * c * c;
          double p7 = (-2 * cp * cp * cp * s + 2 * s * cp) * c;
          double p8 = cp * cp * cp * cp - 2 * cp * cp + 1;
          double p9 = fabs(s * cp) * sin(V1(S->p, k)) * vr;
          double p10 = (cp * cp * cp * cp - 3 * cp * cp + 1) * c * c;
          double p11 = (2 * cp * cp * cp * s - 2 * s * cp) * c;
          double p12 = cp * cp * cp * cp + 2 * cp * cp;
          double *v = &A3(S->vt, j, k, i, nt, npm);
          *v = *v + (-((p1 + (p2 + p3 + p4) * sgn(one, s) + p5 + p6 + p7 + p8) * p9) /
                     sqrt(p10 + p11 - p12));
          if (fabs(*v) > 1.0e5 || fabs(*v) < -1.0e-5) *v = 0;
        }
    for (int i = 1; i <= nr; i++)
      for (int k = 1; k <= np; k++)
        for (int j = 1; j <= ntm; j++) {
          double cph = cos(V1(S->ph, k)), c = V1(S->ct, j), s = V1(S->st, j);
          double p1 = vr * (cph * cph * c + s * cph - c) * sgn(one, cph) * fabs(s);
          double p2 = (cph * cph * cph * cph - 3 * cph * cph + 1) * c * c;
          double p3 = (2 * cph * cph * cph * s - 2 * s * cph) * c;
          double p4 = cph * cph * cph * cph + 2 * cph * cph;
          double *v = &A3(S->vp, j, k, i, ntm, np);
          *v = *v - p1 / sqrt(p2 + p3 - p4);
          if (fabs(*v) > 1.0e5 || fabs(*v) < -1.0e-5) *v = 0;
        }
  }
  if (P->flow_attenuate) {
    for (int i = 1; i <= nr; i++)
      for (int k = 2; k <= npm - 1; k++)
        for (int j = 2; j <= nt - 1; j++) {
          double b = dmax(fabs(F(j - 1, k, i)), fabs(F(j, k, i)));
          A3(S->vt, j, k, i, nt, npm) *= (one - tanh(b * S->atten_i[i - 1]));
        }
    for (int i = 1; i <= nr; i++)
      for (int k = 2; k <= np - 1; k++)
        for (int j = 1; j <= ntm; j++) {
          double b = dmax(fabs(F(j, k - 1, i)), fabs(F(j, k, i)));
          A3(S->vp, j, k, i, ntm, np) *= (one - tanh(b * S->atten_i[i - 1]));
        }
    set_periodic_bc_3d(S->vt, nt, npm, nr);
    set_periodic_bc_3d(S->vp, ntm, np, nr);
    S->flow_needs_updating = 1;
  }
  if (S->adv_space == 2) set_lf_alpha(S);
}

/* ----------------------------------------------------- get_flow_dtmax
 * F:7287-7350 */
static double get_flow_dtmax(orc *S) {
  int nt = S->nt, np = S->np, ntm = S->ntm, npm = S->npm, nr = S->nr;
  double dtmax = LARGE_VALUE;
  for (int i = 1; i <= nr; i++)
    for (int k = 2; k <= npm - 1; k++)
      for (int j = 2; j <= ntm - 1; j++) {
        double kdotv = dmax(fabs(A3(S->vt, j, k, i, nt, npm)), fabs(A3(S->vt, j + 1, k, i, nt, npm))) *
                           V1(S->dt_i, j) +
                       dmax(fabs(A3(S->vp, j, k, i, ntm, np)), fabs(A3(S->vp, j, k + 1, i, ntm, np))) *
                           V1(S->st_i, j) * V1(S->dp_i, k);
        double deltat = half / dmax(kdotv, SMALL_VALUE);
        dtmax = dmin(dtmax, deltat);
      }
  double d = safety * dtmax;
  if (S->P->strang_splitting) d = two * d;
  if (S->adv_time == 3) d = two * d;
  return d;
}

/* ------------------------------------------------- advection operators
 * upwind F:7615-7709 */
static void advection_operator_upwind(orc *S, const double *x, double *aop) {
  int nt = S->nt, np = S->np, ntm = S->ntm, npm = S->npm, nr = S->nr, ntm1 = S->ntm1,
      npm1 = S->npm1;
  double up = S->P->upwind;
  double *flux_t = dalloc((size_t)nt * npm * nr), *flux_p = dalloc((size_t)ntm * np * nr);
#define X(j, k, i) A3(x, j, k, i, ntm, npm)
#define FT(j, k, i) A3(flux_t, j, k, i, nt, npm)
#define FP(j, k, i) A3(flux_p, j, k, i, ntm, np)
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 1; i <= nr; i++)
    for (int k = 1; k <= npm; k++) {
      for (int j = 2; j <= ntm1; j++) {
        double v = A3(S->vt, j, k, i, nt, npm);
        double cct = sgn(up, v);
        FT(j, k, i) = v * half * ((one - cct) * X(j, k, i) + (one + cct) * X(j - 1, k, i));
      }
      if (k >= 2 && k <= npm1)
        for (int j = 2; j <= ntm - 1; j++) {
          double v = A3(S->vp, j, k, i, ntm, np);
          double ccp = sgn(up, v);
          FP(j, k, i) = v * half * ((one - ccp) * X(j, k, i) + (one + ccp) * X(j, k - 1, i));
        }
    }
  set_periodic_bc_3d(flux_p, ntm, np, nr);
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 1; i <= nr; i++)
    for (int k = 2; k <= npm - 1; k++)
      for (int j = 2; j <= ntm - 1; j++)
        A3(aop, j, k, i, ntm, npm) =
            ((V1(S->sth, j + 1) * FT(j + 1, k, i) - V1(S->sth, j) * FT(j, k, i)) * V1(S->st_i, j) *
                 V1(S->dt_i, j) +
             (FP(j, k + 1, i) - FP(j, k, i)) * V1(S->st_i, j) * V1(S->dp_i, k));
  for (int i = 1; i <= nr; i++) {
    double fn = zero, fs = zero;
    for (int k = 2; k <= npm - 1; k++) {
      fn = fn + FT(2, k, i) * V1(S->dp, k);
      fs = fs + FT(ntm1, k, i) * V1(S->dp, k);
    }
    for (int k = 2; k <= npm - 1; k++) {
      A3(aop, 1, k, i, ntm, npm) = fn * S->bc_flow_npole_fac;
      A3(aop, ntm, k, i, ntm, npm) = -fs * S->bc_flow_spole_fac;
    }
  }
  set_periodic_bc_3d(aop, ntm, npm, nr);
  free(flux_t); free(flux_p);
#undef FT
#undef FP
#undef X
}

/* WENO3 F:7711-7925 */
static double weno_face(double LNm2, double LNm1, double LN0, double LPm1, double LP0,
                        double LPp1, double DCMC_m1, double DCMC_0, double DCCP_m1,
                        double DCCP_0, double DPT_m1, double DMCT_m1, double DMT_0,
                        double DCPT_0, double eps_m1, double eps_0) {
  /* face between cells (j-1) and j; LN*: LN(j-2),LN(j-1),LN(j); LP*: LP(j-1),LP(j),LP(j+1) */
  double p0m = (one + DCMC_m1) * LNm1 - DCMC_m1 * LNm2;
  double p1m = DCMC_0 * LNm1 + DCCP_m1 * LN0;
  double p0p = (one + DCCP_0) * LP0 - DCCP_0 * LPp1;
  double p1p = DCCP_m1 * LP0 + DCMC_0 * LPm1;
  double t0 = DCMC_m1 * (LNm1 - LNm2), t1 = DCCP_m1 * (LN0 - LNm1);
  double t2 = DCCP_0 * (LPp1 - LP0), t3 = DCMC_0 * (LP0 - LPm1);
  double B0m = four * (t0 * t0), B1m = four * (t1 * t1);
  double B0p = four * (t2 * t2), B1p = four * (t3 * t3);
  double e0 = eps_m1 + B0m, e1 = eps_m1 + B1m, e2 = eps_0 + B0p, e3 = eps_0 + B1p;
  double w0m = DPT_m1 / (e0 * e0);
  double w1m = DMCT_m1 / (e1 * e1);
  double w0p = DMT_0 / (e2 * e2);
  double w1p = DCPT_0 / (e3 * e3);
  double wm_sum = w0m + w1m, wp_sum = w0p + w1p;
  double OM0m = w0m / wm_sum, OM1m = w1m / wm_sum;
  double OM0p = w0p / wp_sum, OM1p = w1p / wp_sum;
  double um = OM0m * p0m + OM1m * p1m;
  double upv = OM0p * p0p + OM1p * p1p;
  return upv + um;
}

static void advection_operator_weno3(orc *S, const double *x, double *aop) {
  int nt = S->nt, np = S->np, ntm = S->ntm, npm = S->npm, nr = S->nr, npm1 = S->npm1;
  double up = S->P->upwind;
  double *flux_t = dalloc((size_t)nt * npm * nr);
  double *flux_p = dalloc((size_t)ntm * np * nr);
  size_t nLp = (size_t)ntm * (npm + 1) * nr; /* LP(ntm,0:npm,nr) */
  double *LP = dalloc(nLp), *LN = dalloc(nLp);
#define X(j, k, i) A3(x, j, k, i, ntm, npm)
#define LPT(j, k, i) A3(LP, j, k, i, ntm, npm)
#define LNT(j, k, i) A3(LN, j, k, i, ntm, npm)
#define LPP(j, k, i) A3(LP, j, (k) + 1, i, ntm, npm + 1)
#define LNP(j, k, i) A3(LN, j, (k) + 1, i, ntm, npm + 1)
#define VTv(j, k, i) A3(S->vt, j, k, i, nt, npm)
#define VPv(j, k, i) A3(S->vp, j, k, i, ntm, np)
  /* theta: LLF split (F:7766-7769), WENO faces (F:7773-7803), upwind next
   * to the poles (F:7807-7817).  Each phi column is independent. */
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 1; i <= nr; i++)
    for (int k = 1; k <= npm; k++) {
      for (int j = 1; j <= ntm; j++) {
        LPT(j, k, i) = half * X(j, k, i) * (VTv(j + 1, k, i) - A3(S->alpha_t, j, k, i, ntm, npm));
        LNT(j, k, i) = half * X(j, k, i) * (VTv(j, k, i) + A3(S->alpha_t, j, k, i, ntm, npm));
      }
      for (int j = 3; j <= nt - 2; j++)
        A3(flux_t, j, k, i, nt, npm) = weno_face(
            LNT(j - 2, k, i), LNT(j - 1, k, i), LNT(j, k, i), LPT(j - 1, k, i), LPT(j, k, i),
            LPT(j + 1, k, i), V1(S->D_C_MCt, j - 1), V1(S->D_C_MCt, j), V1(S->D_C_CPt, j - 1),
            V1(S->D_C_CPt, j), V1(S->D_P_Tt, j - 1), V1(S->D_MC_Tt, j - 1), V1(S->D_M_Tt, j),
            V1(S->D_CP_Tt, j), V1(S->weno_eps_t, j - 1), V1(S->weno_eps_t, j));
      double v = VTv(2, k, i);
      double cct = sgn(up, v);
      A3(flux_t, 2, k, i, nt, npm) = v * half * ((one - cct) * X(2, k, i) + (one + cct) * X(1, k, i));
      v = VTv(nt - 1, k, i);
      cct = sgn(up, v);
      A3(flux_t, nt - 1, k, i, nt, npm) =
          v * half * ((one - cct) * X(ntm, k, i) + (one + cct) * X(ntm - 1, k, i));
    }
  /* phi: split (F:7833-7836), periodic pad (F:7840-7845), faces (F:7850-7880) */
  memset(LP, 0, sizeof(double) * nLp);
  memset(LN, 0, sizeof(double) * nLp);
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 1; i <= nr; i++)
    for (int k = 1; k <= npm - 1; k++)
      for (int j = 2; j <= ntm - 1; j++) {
        LPP(j, k, i) = half * X(j, k, i) * (VPv(j, k + 1, i) - A3(S->alpha_p, j, k, i, ntm, npm));
        LNP(j, k, i) = half * X(j, k, i) * (VPv(j, k, i) + A3(S->alpha_p, j, k, i, ntm, npm));
      }
  for (int i = 1; i <= nr; i++)
    for (int j = 2; j <= ntm - 1; j++) {
      LPP(j, 0, i) = LPP(j, npm - 2, i);
      LNP(j, 0, i) = LNP(j, npm - 2, i);
      LPP(j, npm, i) = LPP(j, 2, i);
      LNP(j, npm, i) = LNP(j, 2, i);
    }
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 1; i <= nr; i++)
    for (int k = 2; k <= npm1; k++)
      for (int j = 2; j <= ntm - 1; j++)
        A3(flux_p, j, k, i, ntm, np) = weno_face(
            LNP(j, k - 2, i), LNP(j, k - 1, i), LNP(j, k, i), LPP(j, k - 1, i), LPP(j, k, i),
            LPP(j, k + 1, i), V1(S->D_C_MCp, k - 1), V1(S->D_C_MCp, k), V1(S->D_C_CPp, k - 1),
            V1(S->D_C_CPp, k), V1(S->D_P_Tp, k - 1), V1(S->D_MC_Tp, k - 1), V1(S->D_M_Tp, k),
            V1(S->D_CP_Tp, k), V1(S->weno_eps_p, k - 1), V1(S->weno_eps_p, k));
  set_periodic_bc_3d(flux_p, ntm, np, nr);
  /* divergence (F:7890-7898) and pole rings (F:7902-7915) */
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 1; i <= nr; i++)
    for (int k = 2; k <= npm - 1; k++)
      for (int j = 2; j <= ntm - 1; j++)
        A3(aop, j, k, i, ntm, npm) =
            ((V1(S->sth, j + 1) * A3(flux_t, j + 1, k, i, nt, npm) -
              V1(S->sth, j) * A3(flux_t, j, k, i, nt, npm)) *
                 V1(S->st_i, j) * V1(S->dt_i, j) +
             (A3(flux_p, j, k + 1, i, ntm, np) - A3(flux_p, j, k, i, ntm, np)) * V1(S->st_i, j) *
                 V1(S->dp_i, k));
  for (int i = 1; i <= nr; i++) {
    double fn = zero, fs = zero;
    for (int k = 2; k <= npm - 1; k++) {
      fn = fn + A3(flux_t, 2, k, i, nt, npm) * V1(S->dp, k);
      fs = fs + A3(flux_t, nt - 1, k, i, nt, npm) * V1(S->dp, k);
    }
    for (int k = 2; k <= npm - 1; k++) {
      A3(aop, 1, k, i, ntm, npm) = fn * S->bc_flow_npole_fac;
      A3(aop, ntm, k, i, ntm, npm) = -fs * S->bc_flow_spole_fac;
    }
  }
  set_periodic_bc_3d(aop, ntm, npm, nr);
  free(flux_t); free(flux_p); free(LP); free(LN);
#undef LPT
#undef LNT
#undef LPP
#undef LNP
#undef VTv
#undef VPv
#undef X
}

static void advection_operator(orc *S, const double *x, double *aop) {
  S->cell_updates += (double)S->ntm * (S->npm - 2) * S->nr;
  if (S->adv_space == 1) advection_operator_upwind(S, x, aop);
  else advection_operator_weno3(S, x, aop);
}

/* ------------------------------------------------ advection integrators
 * FE F:7409-7451, SSPRK33 F:7453-7513, SSPRK43 F:7515-7582 */
static void advection_step(orc *S, double dtl) {
  size_t n = (size_t)S->ntm * S->npm * S->nr;
  double *f = S->f;
  S->dtime_advection_used = dtl;
  double *aop = dalloc(n);
  if (S->adv_time == 1) {
    advection_operator(S, f, aop);
    for (size_t q = 0; q < n; q++) f[q] = f[q] - dtl * aop[q];
  } else if (S->adv_time == 2) {
    double *f1 = dalloc(n);
    advection_operator(S, f, aop);
    for (size_t q = 0; q < n; q++) f1[q] = f[q] - dtl * aop[q];
    advection_operator(S, f1, aop);
    for (size_t q = 0; q < n; q++)
      f1[q] = three_quarter * f[q] + quarter * f1[q] - quarter * dtl * aop[q];
    advection_operator(S, f1, aop);
    for (size_t q = 0; q < n; q++)
      f[q] = third * f[q] + two_third * f1[q] - two_third * dtl * aop[q];
    free(f1);
  } else {
    double *f1 = dalloc(n);
    advection_operator(S, f, aop);
#pragma omp parallel for
    for (size_t q = 0; q < n; q++) f1[q] = f[q] - half * dtl * aop[q];
    advection_operator(S, f1, aop);
    for (size_t q = 0; q < n; q++) f1[q] = f1[q] - half * dtl * aop[q];
    advection_operator(S, f1, aop);
    for (size_t q = 0; q < n; q++)
      f1[q] = two_third * f[q] + third * f1[q] - sixth * dtl * aop[q];
    advection_operator(S, f1, aop);
    for (size_t q = 0; q < n; q++) f[q] = f1[q] - half * dtl * aop[q];
    free(f1);
  }
  free(aop);
}

/* ------------------------------------------------- diffusion operator
 * diffusion_operator_cd F:7927-7990 */
#define COEF(j, k, d, i) \
  S->coef[((((size_t)(i)-1) * 5 + ((d)-1)) * (size_t)(S->npm - 2) + ((k)-2)) * (size_t)(S->ntm - 2) + ((j)-2)]
#define DC(j, k, i) A3(S->dcoef, j, k, i, S->nt, S->np)
static void diffusion_operator_cd(orc *S, const double *x, double *y) {
  int ntm = S->ntm, npm = S->npm, nr = S->nr, nt = S->nt;
#define X(j, k, i) A3(x, j, k, i, ntm, npm)
#pragma omp parallel for collapse(2) schedule(static)
  for (int i = 1; i <= nr; i++)
    for (int k = 2; k <= npm - 1; k++)
      for (int j = 2; j <= ntm - 1; j++)
        A3(y, j, k, i, ntm, npm) = COEF(j, k, 1, i) * X(j, k - 1, i) + COEF(j, k, 2, i) * X(j - 1, k, i) +
                                   COEF(j, k, 3, i) * X(j, k, i) + COEF(j, k, 4, i) * X(j + 1, k, i) +
                                   COEF(j, k, 5, i) * X(j, k + 1, i);
  for (int i = 1; i <= nr; i++) {
    double fn = zero, fs = zero;
    for (int k = 2; k <= npm - 1; k++) {
      fn = fn + (DC(1, k, i) + DC(2, k, i)) * (X(2, k, i) - X(1, k, i)) * V1(S->dp, k);
      fs = fs + (DC(nt - 1, k, i) + DC(nt, k, i)) * (X(ntm, k, i) - X(ntm - 1, k, i)) * V1(S->dp, k);
    }
    for (int k = 1; k <= npm; k++) {
      A3(y, 1, k, i, ntm, npm) = fn * S->bc_diffusion_npole_fac;
      A3(y, ntm, k, i, ntm, npm) = -fs * S->bc_diffusion_spole_fac;
    }
  }
  set_periodic_bc_3d(y, ntm, npm, nr);
#undef X
}

/* ----------------------------------------------------- load_diffusion
 * F:6655-6844, load_diffusion_matrix F:4927-4983, euler dt F:4985-5040 */
static void load_diffusion(orc *S) {
  const orc_params *P = S->P;
  int nt = S->nt, np = S->np, ntm = S->ntm, npm = S->npm, nr = S->nr;
  S->dcoef = dalloc((size_t)nt * np * nr);
  for (int i = 1; i <= nr; i++)
    for (int k = 1; k <= np; k++)
      for (int j = 1; j <= nt; j++) DC(j, k, i) = P->diffusion_coef_constants[i - 1];
  if (P->diffusion_coef_grid)
    for (int i = 1; i <= nr; i++)
      for (int k = 1; k <= np; k++)
        for (int j = 1; j <= nt; j++) {
          double a = V1(S->dth, j), b = V1(S->dph, k) * V1(S->sth, j);
          DC(j, k, i) = DC(j, k, i) + (a * a + b * b);
        }
  for (size_t q = 0; q < (size_t)nt * np * nr; q++) S->dcoef[q] = P->diffusion_coef_factor * S->dcoef[q];
  S->coef = dalloc((size_t)(ntm - 2) * (npm - 2) * 5 * nr);
  for (int i = 1; i <= nr; i++)
    for (int k = 2; k <= npm - 1; k++)
      for (int j = 2; j <= ntm - 1; j++) {
        COEF(j, k, 1, i) = half * (DC(j, k, i) + DC(j + 1, k, i)) * V1(S->dph_i, k) * V1(S->dp_i, k) *
                           V1(S->st_i, j) * V1(S->st_i, j);
        COEF(j, k, 2, i) = half * (DC(j, k, i) + DC(j, k + 1, i)) * V1(S->dth_i, j) * V1(S->dt_i, j) *
                           V1(S->st_i, j) * V1(S->sth, j);
        COEF(j, k, 4, i) = half * (DC(j + 1, k, i) + DC(j + 1, k + 1, i)) * V1(S->dth_i, j + 1) *
                           V1(S->dt_i, j) * V1(S->st_i, j) * V1(S->sth, j + 1);
        COEF(j, k, 5, i) = half * (DC(j, k + 1, i) + DC(j + 1, k + 1, i)) * V1(S->dph_i, k + 1) *
                           V1(S->dp_i, k) * V1(S->st_i, j) * V1(S->st_i, j);
        COEF(j, k, 3, i) = -(COEF(j, k, 1, i) + COEF(j, k, 2, i) + COEF(j, k, 4, i) + COEF(j, k, 5, i));
      }
  double max_eig = 0.;
  for (int i = 1; i <= nr; i++)
    for (int k = 2; k <= npm - 1; k++)
      for (int j = 2; j <= ntm - 1; j++) {
        double g = zero;
        for (int d = 1; d <= 5; d++) g = g + fabs(COEF(j, k, d, i));
        max_eig = dmax(g, max_eig);
      }
  S->dtime_diffusion_euler = safety * (two / max_eig);
  S->auto_sc = (P->diffusion_subcycles == 0);
  S->diffusion_subcycles = P->diffusion_subcycles;
  S->bc_diffusion_npole_fac = pi_i * V1(S->dth_i, 2) * V1(S->dth_i, 2);
  S->bc_diffusion_spole_fac = pi_i * V1(S->dth_i, nt - 1) * V1(S->dth_i, nt - 1);
}

/* ------------------------------------------------------------- PTL dt
 * get_dtime_diffusion_ptl F:5042-5161 */
static void get_dtime_diffusion_ptl(orc *S, double *dtime_ptl) {
  int ntm = S->ntm, npm = S->npm, nr = S->nr;
  const double safe = 0.95, fmin = 1e-14;
  double dtime_in = *dtime_ptl;
  double dptl = LARGE_VALUE;
  size_t n = (size_t)ntm * npm * nr;
  double *Af = dalloc(n);
  diffusion_operator_cd(S, S->f, Af);
  double axabsmax = -one;
  for (size_t q = 0; q < n; q++)
    if (fabs(S->f[q]) > fmin) axabsmax = dmax(fabs(Af[q]), axabsmax);
  if (axabsmax > zero) {
#define AF(j, k, i) A3(Af, j, k, i, ntm, npm)
    for (int i = 1; i <= nr; i++)
      for (int k = 2; k <= npm - 1; k++)
        for (int j = 2; j <= ntm - 1; j++) {
          if (axabsmax == fabs(AF(j, k, i)) && fabs(F(j, k, i)) > fmin) {
            double du, df;
            du = F(j, k, i) - F(j - 1, k, i); df = AF(j, k, i) - AF(j - 1, k, i);
            if (du * df < -fmin) dptl = dmin(-du / df, dptl);
            du = F(j, k, i) - F(j + 1, k, i); df = AF(j, k, i) - AF(j + 1, k, i);
            if (du * df < -fmin) dptl = dmin(-du / df, dptl);
            du = F(j, k, i) - F(j, k - 1, i); df = AF(j, k, i) - AF(j, k - 1, i);
            if (du * df < -fmin) dptl = dmin(-du / df, dptl);
            du = F(j, k, i) - F(j, k + 1, i); df = AF(j, k, i) - AF(j, k + 1, i);
            if (du * df < -fmin) dptl = dmin(-du / df, dptl);
          }
        }
#undef AF
    dptl = safe * dptl;
    if (dptl < dtime_in) dptl = dtime_in;
  }
  *dtime_ptl = dptl;
  free(Af);
}

/* ---------------------------------------------------------- load_sts
 * RKL2 F:5244-5359, RKG2 F:5361-5475 */
static void load_sts(orc *S, double dtl) {
  long s;
  double w;
  if (S->P->diffusion_num_method == 2) {
    double sr = half * (sqrt(nine + sixteen * (dtl / S->dtime_diffusion_euler)) - one);
    s = (long)ceil(sr);
  } else {
    double sr = half * (sqrt(twentyfive + twentyfour * (dtl / S->dtime_diffusion_euler)) - three);
    s = (long)ceil(sr);
  }
  if (s < 3) s = 3;
  if (s % 2 == 0) s = s + 1;
  S->sts_s = s;
  free(S->sts_uj); free(S->sts_vj); free(S->sts_ubj); free(S->sts_gj); free(S->sts_b);
  S->sts_uj = dalloc(s + 1); S->sts_vj = dalloc(s + 1); S->sts_ubj = dalloc(s + 1);
  S->sts_gj = dalloc(s + 1); S->sts_b = dalloc(s + 1);
  double *b = S->sts_b, *uj = S->sts_uj, *vj = S->sts_vj, *ubj = S->sts_ubj, *gj = S->sts_gj;
  if (S->P->diffusion_num_method == 2) {
    w = four / (double)(s * s + s - 2);
    b[1] = one / three; b[2] = one / three;
    uj[1] = -9999.; vj[1] = -9999.; ubj[1] = four / (three * (double)(s * s + s - 2)); gj[1] = -9999.;
    uj[2] = three / two; vj[2] = -half; ubj[2] = uj[2] * w; gj[2] = -w;
    for (long j = 3; j <= s; j++) {
      b[j] = ((double)(j * j + j) - two) / (two * (double)j * (double)(j + 1));
      double bj_bjm1 = b[j] / b[j - 1], bj_bjm2 = b[j] / b[j - 2];
      uj[j] = bj_bjm1 * (two - one / (double)j);
      vj[j] = bj_bjm2 * (one / (double)j - one);
      ubj[j] = uj[j] * w;
      gj[j] = (b[j - 1] - one) * ubj[j];
    }
  } else {
    w = six / (double)((s + 4) * (s - 1));
    b[1] = one / three; b[2] = one / fifteen;
    uj[1] = one; vj[1] = -9999.; ubj[1] = w; gj[1] = -9999.;
    uj[2] = one / two; vj[2] = -one / ten; ubj[2] = uj[2] * w; gj[2] = zero;
    for (long j = 3; j <= s; j++) {
      b[j] = (four * (double)(j - 1) * (double)(j + 4)) /
             (three * (double)j * (double)(j + 1) * (double)(j + 2) * (double)(j + 3));
      double bj_bjm1 = b[j] / b[j - 1], bj_bjm2 = b[j] / b[j - 2];
      uj[j] = bj_bjm1 * (two + one / (double)j);
      vj[j] = -bj_bjm2 * (one / (double)j + one);
      ubj[j] = uj[j] * w;
      gj[j] = (half * (double)j * ((double)j + one) * b[j - 1] - one) * ubj[j];
    }
  }
}

/* diffusion_step_sts_cd F:5163-5242 */
static void diffusion_step_sts_cd(orc *S, double dtl) {
  if (S->need_to_load_sts) {
    load_sts(S, dtl);
    S->need_to_load_sts = 0;
  }
  size_t n = (size_t)S->ntm * S->npm * S->nr;
  double *u0 = dalloc(n), *dty0 = dalloc(n), *ykm1 = dalloc(n), *ukm1 = dalloc(n), *ukm2 = dalloc(n);
  double *f = S->f;
  diffusion_operator_cd(S, f, dty0);
  for (size_t q = 0; q < n; q++) {
    u0[q] = f[q];
    ukm2[q] = f[q];
    dty0[q] = dtl * dty0[q];
    ukm1[q] = f[q] + S->sts_ubj[1] * dty0[q];
  }
  S->cell_updates += (double)S->ntm * (S->npm - 2) * S->nr * (double)S->sts_s;
  for (long k = 2; k <= S->sts_s; k++) {
    diffusion_operator_cd(S, ukm1, ykm1);
    double uj = S->sts_uj[k], vj = S->sts_vj[k], ubj = S->sts_ubj[k], gj = S->sts_gj[k];
#pragma omp parallel for
    for (size_t q = 0; q < n; q++) {
      f[q] = uj * ukm1[q] + vj * ukm2[q] + (one - uj - vj) * u0[q] + ubj * dtl * ykm1[q] + gj * dty0[q];
      ukm2[q] = ukm1[q];
      ukm1[q] = f[q];
    }
  }
  free(u0); free(dty0); free(ykm1); free(ukm1); free(ukm2);
}

/* diffusion_step_fe_cd F:7352-7407 */
static void diffusion_step_fe_cd(orc *S, double dtl) {
  size_t n = (size_t)S->ntm * S->npm * S->nr;
  double *fold = dalloc(n);
  double r = dtl / S->dtime_diffusion_euler;
  long nc = (long)ceil(r);
  S->n_stable_diffusion_cycles = nc;
  double dte = dtl / (double)nc;
  S->cell_updates += (double)S->ntm * (S->npm - 2) * S->nr * (double)nc;
  for (long i = 1; i <= nc; i++) {
    diffusion_operator_cd(S, S->f, fold);
    for (size_t q = 0; q < n; q++) S->f[q] = S->f[q] + dte * fold[q];
  }
  free(fold);
}

/* diffusion_step F:4551-4695 */
static void diffusion_step(orc *S, double dtl) {
  const orc_params *P = S->P;
  const int max_sc = 60;
  int i = 1, done = 0;
  double time_stepped = 0., dtl2;
  dtl2 = S->auto_sc ? zero : dtl / (double)S->diffusion_subcycles;
  for (;;) {
    if (S->auto_sc) {
      get_dtime_diffusion_ptl(S, &dtl2);
      S->need_to_load_sts = 1;
    }
    if (S->auto_sc && time_stepped + dtl2 >= dtl) {
      dtl2 = dtl - time_stepped;
      S->need_to_load_sts = 1;
      done = 1;
    }
    if (S->auto_sc && i == max_sc - 1) {
      dtl2 = dtl - time_stepped;
      S->need_to_load_sts = 1;
      done = 1;
    }
    if (S->auto_sc && P->verbose > 0) S->diffusion_subcycles = (long)ceil((dtl - time_stepped) / dtl2);
    if (P->diffusion_num_method == 1) diffusion_step_fe_cd(S, dtl2);
    else diffusion_step_sts_cd(S, dtl2);
    time_stepped = time_stepped + dtl2;
    if (P->verbose > 1) {
      double tt = S->time;
      S->time = S->time + time_stepped;
      analysis_and_history(S);
      S->time = tt;
    }
    if (!S->auto_sc && i == S->diffusion_subcycles) done = 1;
    if (done) break;
    i = i + 1;
  }
  if (S->auto_sc) S->diffusion_subcycles = i;
}

/* --------------------------------------------------- flux_transport_step
 * F:4463-4507 (sources are out of scope) */
static void source_step(orc *S, double dtl);

static void flux_transport_step(orc *S) {
  const orc_params *P = S->P;
  double dtl = S->dtime_global;
  if (P->strang_splitting) {
    double h = dtl * half;
    if (P->advance_source) source_step(S, h);
    if (P->advance_flow) advection_step(S, h);
    if (P->advance_diffusion) diffusion_step(S, dtl);
    if (P->advance_flow) advection_step(S, h);
    if (P->advance_source) source_step(S, h);
  } else {
    if (P->advance_flow) advection_step(S, dtl);
    if (P->advance_diffusion) diffusion_step(S, dtl);
    if (P->advance_source) source_step(S, dtl);
  }
}

/* ----------------------------------------------------------------- sources
 * get_gaussian F:8616-8670 (Marsaglia-Bray polar method, second deviate kept
 * for the next call) over xoshiro256** uniforms seeded through splitmix64:
 * the same generator as the library's driver (the reference uses gfortran's
 * RANDOM_NUMBER, whose stream is not restated here). */
static void rng_seed(orc *S, uint64_t x) {
  for (int q = 0; q < 4; q++) {
    x += 0x9e3779b97f4a7c15ULL;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    S->rng[q] = z ^ (z >> 31);
  }
  S->g_second = 0;
}
static uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static double rng_uniform(orc *S) {
  uint64_t *s = S->rng;
  const uint64_t r = rotl64(s[1] * 5, 7) * 9, t = s[1] << 17;
  s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3]; s[2] ^= t; s[3] = rotl64(s[3], 45);
  return (double)(r >> 11) * 0x1.0p-53;
}
static double get_gaussian(orc *S) {
  if (S->g_second) { S->g_second = 0; return S->g_v * S->g_sln; }
  S->g_second = 1;
  double u, q;
  for (;;) {
    u = 2.0 * rng_uniform(S) - one;
    S->g_v = 2.0 * rng_uniform(S) - one;
    q = u * u + S->g_v * S->g_v;
    if (q < one && q > 0.) break;
  }
  S->g_sln = sqrt(-(2.0 * log(q)) / q);
  return u * S->g_sln;
}

/* generate_rfe F:8809-8921 followed by balance_flux of each realization */
static void generate_rfe(orc *S, double *rfe) {
  const orc_params *P = S->P;
  int ntm = S->ntm, npm = S->npm, nr = S->nr;
  double *rnd = dalloc((size_t)ntm * npm);
  const double normfac = pi / sqrt(twopi);
  for (int k = 2; k <= npm - 1; k++)
    for (int j = 1; j <= ntm; j++) rnd[(size_t)(k - 1) * ntm + (j - 1)] = normfac * get_gaussian(S);
  for (int k = 2; k <= npm - 1; k++)
    for (int j = 1; j <= ntm; j++) {
      double da_ti = 0.;
      if (P->source_rfe_model == 1) {
        if (j == 1) {
          double tav = half * (V1(S->t, 1) + V1(S->t, 2));
          da_ti = one / (quarter * sin(tav) * V1(S->dth, 2));
        } else if (j == ntm) {
          double tav = half * (V1(S->t, ntm) + V1(S->t, ntm - 1));
          da_ti = one / (quarter * sin(tav) * V1(S->dth, ntm));
        } else {
          da_ti = V1(S->st_i, j) * V1(S->dt_i, j);
        }
      }
      for (int i = 1; i <= nr; i++) {
        double r = rnd[(size_t)(k - 1) * ntm + (j - 1)];
        A3(rfe, j, k, i, ntm, npm) = (P->source_rfe_model == 1) ? r * S->uf[i - 1] * da_ti * V1(S->dp_i, k)
                                                                : r * S->uf[i - 1];
      }
    }
  for (int i = 1; i <= nr; i++)
    for (int j = 1; j <= ntm; j++) {
      A3(rfe, j, 1, i, ntm, npm) = A3(rfe, j, npm - 1, i, ntm, npm);
      A3(rfe, j, npm, i, ntm, npm) = A3(rfe, j, 2, i, ntm, npm);
    }
  for (int i = 1; i <= nr; i++) {
    double fn1 = zero, fs1 = zero;
    for (int k = 1; k <= npm - 2; k++) {
      fn1 = fn1 + A3(rfe, 1, k, i, ntm, npm) * V1(S->dp, k);
      fs1 = fs1 + A3(rfe, ntm, k, i, ntm, npm) * V1(S->dp, k);
    }
    fn1 = fn1 * twopi_i;
    fs1 = fs1 * twopi_i;
    for (int k = 1; k <= npm; k++) {
      A3(rfe, 1, k, i, ntm, npm) = fn1;
      A3(rfe, ntm, k, i, ntm, npm) = fs1;
    }
  }
  for (int i = 1; i <= nr; i++) balance_flux(S, rfe + (size_t)(i - 1) * ntm * npm);
  free(rnd);
}

/* interp2d F:7992-8073 (flint's check F:8135-8150, interp F:8178-8210) */
static int interp_1(const double *x, int n, double xv, int *i0, int *i1, double *a) {
  if (n == 1 && xv == x[0]) { *i0 = *i1 = 0; *a = 0.; return 1; }
  for (int i = 0; i < n - 1; i++)
    if (xv >= x[i] && xv <= x[i + 1]) {
      *i0 = i; *i1 = i + 1;
      *a = (x[i] == x[i + 1]) ? 0. : (xv - x[i]) / (x[i + 1] - x[i]);
      return 1;
    }
  return 0;
}
static int interp2d(int nxi, int nyi, const double *xi, const double *yi, const double *fi, int nx, int ny,
                    const double *x, const double *y, double *f) {
  for (int i = 0; i + 1 < nxi; i++) if (xi[i + 1] <= xi[i]) return 1;
  for (int i = 0; i + 1 < nyi; i++) if (yi[i + 1] <= yi[i]) return 1;
  for (int j = 0; j < ny; j++) {
    int jj, jp; double ay;
    for (int i = 0; i < nx; i++) f[(size_t)j * nx + i] = 0.;
    if (y[j] < yi[0] || y[j] > yi[nyi - 1] || !interp_1(yi, nyi, y[j], &jj, &jp, &ay)) continue;
    for (int i = 0; i < nx; i++) {
      int ii, ip; double ax;
      if (x[i] < xi[0] || x[i] > xi[nxi - 1] || !interp_1(xi, nxi, x[i], &ii, &ip, &ax)) continue;
#define FI(a, b) fi[(size_t)(b) * nxi + (a)]
      f[(size_t)j * nx + i] = (one - ax) * ((one - ay) * FI(ii, jj) + ay * FI(ii, jp)) +
                              ax * ((one - ay) * FI(ip, jj) + ay * FI(ip, jp));
#undef FI
    }
  }
  return 0;
}

/* load_source F:7050-7213 */
static int load_source(orc *S) {
  const orc_params *P = S->P;
  int ntm = S->ntm, npm = S->npm, nr = S->nr;
  size_t n = (size_t)ntm * npm * nr;
  S->source = dalloc(n);
  if (P->source_from_file) {
    int nfp = P->source_nfp, nft = P->source_nft;
    double *fi = dalloc((size_t)nft * nfp), *ft = dalloc((size_t)ntm * npm);
    for (int jp = 0; jp < nfp; jp++)
      for (int it = 0; it < nft; it++) fi[(size_t)jp * nft + it] = P->source_data[(size_t)it * nfp + jp];
    if (interp2d(nft, nfp, P->source_tf, P->source_pf, fi, ntm, npm, &V1(S->t, 1), &V1(S->p, 1), ft)) return 4;
    S->source_file = dalloc(n);
    for (int i = 1; i <= nr; i++) memcpy(S->source_file + (size_t)(i - 1) * ntm * npm, ft, sizeof(double) * ntm * npm);
    free(fi); free(ft);
  }
  if (P->source_rfe_model > 0) {
    rng_seed(S, (uint64_t)(P->source_rfe_seed == -9999 ? 0 : P->source_rfe_seed));
    S->uf = dalloc(nr);
    double num_cells = (double)ntm * (npm - 2);
    for (int i = 0; i < nr; i++)
      S->uf[i] = (P->source_rfe_model == 1) ? P->source_rfe_flux[i] * 1.0e21 / (rsun_cm2 * num_cells)
                                            : P->source_rfe_flux[i] * 1.0e21 / (rsun_cm2 * four * pi);
    S->source_rfe[0] = dalloc(n);
    S->source_rfe[1] = dalloc(n);
    S->rfe1 = 0; S->rfe2 = 1;
    generate_rfe(S, S->source_rfe[S->rfe1]);
    generate_rfe(S, S->source_rfe[S->rfe2]);
    S->time_of_next_source_rfe = S->time + P->source_rfe_lifetime;
    S->time_of_prev_source_rfe = S->time;
  }
  return 0;
}

/* update_source F:3875-3947 */
static void update_source(orc *S) {
  const orc_params *P = S->P;
  size_t n = (size_t)S->ntm * S->npm * S->nr;
  for (size_t q = 0; q < n; q++) S->source[q] = 0.;
  if (P->source_from_file)
    for (size_t q = 0; q < n; q++) S->source[q] = S->source[q] + S->source_file[q];
  if (P->source_rfe_model > 0) {
    if (S->time >= S->time_of_next_source_rfe) {
      S->time_of_prev_source_rfe = S->time_of_next_source_rfe;
      S->time_of_next_source_rfe = S->time_of_prev_source_rfe + P->source_rfe_lifetime;
      int t = S->rfe1; S->rfe1 = S->rfe2; S->rfe2 = t;
      generate_rfe(S, S->source_rfe[S->rfe2]);
    }
    double alpha = (S->time - S->time_of_prev_source_rfe) / P->source_rfe_lifetime;
    const double *r1 = S->source_rfe[S->rfe1], *r2 = S->source_rfe[S->rfe2];
    for (size_t q = 0; q < n; q++) S->source[q] = S->source[q] + (one - alpha) * r1[q] + alpha * r2[q];
  }
}

/* source_step F:4697-4732 */
static void source_step(orc *S, double dtl) {
  size_t n = (size_t)S->ntm * S->npm * S->nr;
  for (size_t q = 0; q < n; q++) S->f[q] = S->f[q] + dtl * S->source[q];
}

/* ------------------------------------------------------ update_timestep
 * F:4308-4461 */
static void update_timestep(orc *S) {
  const orc_params *P = S->P;
  if (S->timestep_needs_updating) {
    S->dtime_global = P->time_end - S->time;
    S->time_step_changed = 1;
    if (P->advance_flow) {
      S->dtmax_flow = LARGE_VALUE;
      if (S->timestep_flow_needs_updating) {
        S->dtmax_flow = get_flow_dtmax(S);
        S->timestep_flow_needs_updating = 0;
      }
      if (S->dtmax_flow < S->dtime_global) S->dtime_global = S->dtmax_flow;
    }
    if (P->dt_max < S->dtime_global) S->dtime_global = P->dt_max;
    S->timestep_needs_updating = 0;
  }
  if (P->output_map_time_cadence > 0.0) {
    double tn = P->time_start + (double)(S->idx_out - (P->output_map_idx_start - 1)) * P->output_map_time_cadence;
    if (S->time + S->dtime_global >= tn) {
      S->dtime_global = tn - S->time;
      S->timestep_needs_updating = 1;
      S->timestep_flow_needs_updating = 1;
      S->time_step_changed = 1;
    }
  }
  if (S->da_active) {
    if (S->time + S->dtime_global >= S->time_of_next_input_map) {
      S->dtime_global = S->time_of_next_input_map - S->time;
      S->timestep_needs_updating = 1;
      S->timestep_flow_needs_updating = 1;
      S->time_step_changed = 1;
    }
  }
  if (P->advance_flow && P->use_flow_from_files) { /* F:4415-4426 */
    if (S->time + S->dtime_global >= S->time_of_next_input_flow) {
      S->dtime_global = S->time_of_next_input_flow - S->time;
      S->timestep_needs_updating = 1;
      S->flow_needs_updating = 1;
      S->timestep_flow_needs_updating = 1;
      S->time_step_changed = 1;
    }
  }
  if (P->advance_source && P->source_rfe_model > 0) { /* F:4431-4442 */
    if (S->time + S->dtime_global >= S->time_of_next_source_rfe) {
      S->dtime_global = fmin(S->time_of_next_source_rfe - S->time, half * P->source_rfe_lifetime);
      S->timestep_needs_updating = 1;
      S->timestep_flow_needs_updating = 1;
      S->time_step_changed = 1;
    }
  }
  if (S->time + S->dtime_global >= P->time_end) {
    S->dtime_global = P->time_end - S->time;
    S->timestep_needs_updating = 0;
    S->time_step_changed = 1;
  }
  if (P->advance_diffusion && S->time_step_changed) S->need_to_load_sts = 1;
}

/* ------------------------------------------------- data assimilation
 * load_data_assimilation time bookkeeping F:4010-4042 and lat-limit
 * indices F:4066-4079; apply_data_assimilation F:4148-4306;
 * assimilate_new_data F:4083-4146.  Map times are given in hours since the
 * first map (24*jd - 24*jd(1)). */
static void load_data_assimilation(orc *S) {
  const orc_params *P = S->P;
  int i = 0;
  double best = LARGE_VALUE;
  for (int q = 0; q < S->n_da; q++) {
    double d = fabs(S->da_times[q] - P->time_start);
    if (d < best) { best = d; i = q; }
  }
  S->da_active = 1;
  if (P->time_start <= zero) {
    S->da_idx = 0;
    S->time_of_next_input_map = zero;
  } else if (P->time_start > S->da_times[S->n_da - 1]) {
    S->da_active = 0;
    S->da_idx = -9999;
    S->time_of_next_input_map = -9999.9;
  } else {
    if (P->time_start <= S->da_times[i]) {
      S->da_idx = i;
      S->time_of_next_input_map = S->da_times[i];
    } else {
      S->da_idx = i + 1;
      S->time_of_next_input_map = S->da_times[i + 1];
    }
  }
  S->tidx0 = (int *)calloc(S->nr, sizeof(int));
  S->tidx1 = (int *)calloc(S->nr, sizeof(int));
  for (int r = 0; r < S->nr; r++) {
    S->tidx0[r] = -1; S->tidx1[r] = -1;
    for (int j = 1; j <= S->ntm; j++)
      if (V1(S->t, j) >= P->assimilate_data_lat_limits[r] * d2r && S->tidx0[r] == -1) S->tidx0[r] = j;
    for (int j = S->ntm; j >= 1; j--)
      if (V1(S->t, j) <= (pi - P->assimilate_data_lat_limits[r] * d2r) && S->tidx1[r] == -1) S->tidx1[r] = j;
  }
}

/* The blend of one map (npm1, ntm, 3) into every realization
 * (src/hipft.f90:4228-4271, 4083-4146). */
static void da_blend(orc *S, const double *map) {
  const orc_params *P = S->P;
  int ntm = S->ntm, npm = S->npm, npm1 = S->npm1, nr = S->nr;
  size_t plane = (size_t)npm1 * ntm;
  double *w = dalloc(plane), *d = dalloc(plane);
  double *deltaf = dalloc((size_t)ntm * npm * nr);
  for (int i = 1; i <= nr; i++) {
    for (size_t q = 0; q < plane; q++) {
      w[q] = map[plane + q];
      d[q] = map[q];
    }
    if (P->assimilate_data_custom_from_mu)
      for (size_t q = 0; q < plane; q++) {
        double mu = map[2 * plane + q];
        w[q] = (mu > P->assimilate_data_mu_limits[i - 1]) ? pow(mu, P->assimilate_data_mu_powers[i - 1]) : zero;
      }
    if (P->assimilate_data_lat_limits[i - 1] > 0) {
      for (int k = 1; k <= S->tidx0[i - 1]; k++)
        for (int l = 1; l <= npm1; l++) w[(size_t)(k - 1) * npm1 + (l - 1)] = zero;
      for (int k = S->tidx1[i - 1]; k <= ntm; k++)
        for (int l = 1; l <= npm1; l++) w[(size_t)(k - 1) * npm1 + (l - 1)] = zero;
    }
    for (size_t q = 0; q < plane; q++) d[q] = P->assimilate_data_mult_fac * d[q];
    for (int k = 1; k <= npm1; k++)
      for (int j = 1; j <= ntm; j++) {
        size_t q = (size_t)(j - 1) * npm1 + (k - 1);
        A3(deltaf, j, k, i, ntm, npm) = P->assimilate_data_add ? w[q] * d[q] : w[q] * (d[q] - F(j, k, i));
      }
  }
  set_periodic_bc_3d(deltaf, ntm, npm, nr);
  if (P->assimilate_data_balance_flux)
    for (int i = 1; i <= nr; i++) balance_flux(S, deltaf + (size_t)(i - 1) * ntm * npm);
  size_t n = (size_t)ntm * npm * nr;
  for (size_t q = 0; q < n; q++) S->f[q] = S->f[q] + deltaf[q];
  set_periodic_bc_3d(S->f, ntm, npm, nr);
  free(w); free(d); free(deltaf);
}

static void apply_data_assimilation(orc *S) {
  if (!(S->da_active && S->time >= S->time_of_next_input_map)) return;
  const double *map = S->da_maps + (size_t)S->da_idx * S->npm1 * S->ntm * 3; /* (npm1,ntm,3) */
  da_blend(S, map);
  S->da_idx++;
  if (S->da_idx >= S->n_da) S->da_active = 0;
  else S->time_of_next_input_map = S->da_times[S->da_idx];
}

/* write_map's copy of f (F:2829-2843): balanced per realization if asked. */
static void capture_map(orc *S, double *dst) {
  if (!dst) return;
  const size_t plane = (size_t)S->ntm * S->npm;
  memcpy(dst, S->f, sizeof(double) * plane * S->nr);
  if (S->P->output_map_flux_balance)
    for (int i = 1; i <= S->nr; i++) balance_flux(S, dst + (size_t)(i - 1) * plane);
}

/* output_map (F:2700-2798): the map index drives dt cuts; the maps
 * themselves are kept in the history struct when it asks for them. */
static void output_map_index(orc *S) {
  const orc_params *P = S->P;
  if (P->output_map_idx_cadence > 0 && S->ntime % P->output_map_idx_cadence == 0) S->output_current_map = 1;
  if (P->output_map_time_cadence > 0.0 &&
      S->time >= P->time_start + (double)(S->idx_out - (P->output_map_idx_start - 1)) * P->output_map_time_cadence)
    S->output_current_map = 1;
  if (S->output_current_map) {
    S->idx_out++;
    orc_hist *H = S->hist;
    if (H && H->maps && H->n_maps < H->map_cap) {
      capture_map(S, H->maps + (size_t)H->n_maps * S->ntm * S->npm * S->nr);
      H->map_idx[H->n_maps] = S->idx_out;
      H->map_time[H->n_maps] = S->time;
      H->n_maps++;
    }
    S->output_current_map = 0;
  }
}

/* ------------------------------------------------------------ orc_run
 * setup F:1147-1277 + main loop F:903-948.
 *   n1,n2: PT sizes of the initial map (phi, theta); s1,s2 its scales.
 *   map_pt: (n1,n2,nr) or NULL (then a zero / validation map on a uniform
 *           res_np x res_nt grid is made as the reference does, F:1793-1818).
 *   f_out:  (ntm, npm, nr) final field (may be NULL).
 * Returns 0 on success. */
int orc_run(const orc_params *P, int n1, int n2, const double *s1in, const double *s2in, const double *map_pt,
            int n_da, const double *da_times, const double *da_maps, double *f_out, orc_hist *hist,
            long max_steps, double *timing_out) {
  orc Sx;
  orc *S = &Sx;
  memset(S, 0, sizeof(*S));
  S->P = P;
  S->hist = hist;
  if (hist) hist->nrows = 0;
  int nr = P->n_realizations;
  S->nr = nr;
  double *s1, *s2, *f_local;
  if (!map_pt) {
    n1 = P->res_np; n2 = P->res_nt;
    double d1 = twopi / (n1 - 1), d2 = pi / (n2 - 1);
    s1 = dalloc(n1); s2 = dalloc(n2);
    for (int i = 1; i <= n1; i++) s1[i - 1] = (i - 1) * d1;
    for (int i = 1; i <= n2; i++) s2[i - 1] = (i - 1) * d2;
    f_local = dalloc((size_t)n1 * n2 * nr);
  } else {
    s1 = dalloc(n1); s2 = dalloc(n2);
    memcpy(s1, s1in, sizeof(double) * n1);
    memcpy(s2, s2in, sizeof(double) * n2);
    f_local = dalloc((size_t)n1 * n2 * nr);
    memcpy(f_local, map_pt, sizeof(double) * (size_t)n1 * n2 * nr);
  }
  S->flow_vp_rigid_omega = P->flow_vp_rigid_omega;
  S->flow_vt_const = P->flow_vt_const;
  size_t plane = (size_t)n1 * n2;
  if (P->validation_run == 1) {
    S->fval_u0 = dalloc(plane * nr);
    double *Y = dalloc(plane);
    for (int i = 0; i < nr; i++) {
      tesseral_spherical_harmonic(0, 6, s1, s2, n1, n2, Y);
      memcpy(f_local + plane * i, Y, sizeof(double) * plane);
      tesseral_spherical_harmonic(5, 6, s1, s2, n1, n2, Y);
      memcpy(S->fval_u0 + plane * i, Y, sizeof(double) * plane);
    }
    free(Y);
    for (size_t q = 0; q < plane * nr; q++) S->fval_u0[q] = f_local[q] + sqrt(14.0 / 11.0) * S->fval_u0[q];
    memcpy(f_local, S->fval_u0, sizeof(double) * plane * nr);
  } else if (P->validation_run == 2) {
    double vt_end_loc;
    if (fabs(S->flow_vt_const) > zero) {
      S->flow_vt_const = (pi_two / (P->time_end - P->time_start)) / km_s_to_rs_hr;
      vt_end_loc = threepi_four;
    } else {
      vt_end_loc = pi_four;
    }
    (void)vt_end_loc;
    if (fabs(S->flow_vp_rigid_omega) > zero)
      S->flow_vp_rigid_omega = (twopi / (P->time_end - P->time_start)) / km_s_to_rs_hr;
    double w = P->validation_run_width;
    for (int k = 0; k < nr; k++)
      for (int j = 1; j <= n2; j++) {
        double sti = (j > 1 && j < n2) ? one / sin(s2[j - 1]) : zero;
        for (int i = 1; i <= n1; i++) {
          double a = s2[j - 1] - pi_four, b1 = s1[i - 1] - pi_two, b2 = s1[i - 1] - threepi_two;
          f_local[plane * k + (size_t)(j - 1) * n1 + (i - 1)] =
              -sti * exp(-(a * a) / w - (b1 * b1) / w) + sti * exp(-(a * a) / w - (b2 * b2) / w);
        }
      }
  }
  /* set resolution, transpose PT->TP, periodicity, poles: F:2106-2157 */
  S->ntm1 = n2; S->npm1 = n1;
  S->ntm = n2; S->npm = n1 + 1; S->nt = n2 + 1; S->np = n1 + 1;
  int ntm = S->ntm, npm = S->npm, npm1 = S->npm1;
  S->t = dalloc(ntm); S->p = dalloc(npm);
  S->f = dalloc((size_t)ntm * npm * nr);
  for (int i = 1; i <= nr; i++)
    for (int k = 1; k <= npm1; k++)
      for (int j = 1; j <= ntm; j++) F(j, k, i) = f_local[plane * (i - 1) + (size_t)(j - 1) * n1 + (k - 1)];
  for (int i = 1; i <= nr; i++)
    for (int j = 1; j <= ntm; j++) {
      F(j, 1, i) = half * (F(j, 1, i) + F(j, npm1, i));
      F(j, npm1, i) = F(j, 1, i);
      F(j, npm1 + 1, i) = F(j, 2, i);
    }
  for (int j = 1; j <= ntm; j++) V1(S->t, j) = s2[j - 1];
  for (int k = 1; k <= npm1; k++) V1(S->p, k) = s1[k - 1];
  V1(S->p, npm1 + 1) = V1(S->p, 2) + twopi;
  if (set_mesh(S)) return -1;
  for (int i = 1; i <= nr; i++) {
    double fn1 = 0., fs1 = 0.;
    for (int k = 2; k <= npm - 1; k++) {
      fn1 = fn1 + F(1, k, i) * V1(S->dp, k);
      fs1 = fs1 + F(ntm, k, i) * V1(S->dp, k);
    }
    for (int k = 1; k <= npm; k++) {
      F(1, k, i) = fn1 * twopi_i;
      F(ntm, k, i) = fs1 * twopi_i;
    }
  }
  if (P->initial_map_flux_balance)
    for (int i = 1; i <= nr; i++) balance_flux(S, S->f + (size_t)(i - 1) * ntm * npm);
  for (size_t q = 0; q < (size_t)ntm * npm * nr; q++) S->f[q] = P->initial_map_mult_fac * S->f[q];
  if (hist) capture_map(S, hist->map_initial); /* <root>_initial.h5, F:2185 */
  free(s1); free(s2); free(f_local);

  S->time = P->time_start;
  S->timestep_needs_updating = 1;
  S->timestep_flow_needs_updating = 1;
  S->flow_needs_updating = 1;
  S->need_to_load_sts = 1;
  S->idx_out = P->output_map_idx_start - 1;
  if (P->flow_num_method == 1) { S->adv_time = 1; S->adv_space = 1; }
  else if (P->flow_num_method == 2) { S->adv_time = 2; S->adv_space = 1; }
  else if (P->flow_num_method == 3) { S->adv_time = 2; S->adv_space = 2; }
  else { S->adv_time = 3; S->adv_space = 2; }
  if (P->output_map_idx_cadence > 0 || P->output_map_time_cadence > 0.) S->output_current_map = 1;
  if (P->advance_flow) {
    S->vt = dalloc((size_t)S->nt * npm * nr);
    S->vp = dalloc((size_t)ntm * S->np * nr);
    if (S->adv_space == 2) load_weno(S);
    S->bc_flow_npole_fac = two * V1(S->dth_i, 2) * pi_i;
    S->bc_flow_spole_fac = two * V1(S->dth_i, S->nt - 1) * pi_i;
    if (P->flow_attenuate) {
      S->atten_i = dalloc(nr);
      for (int i = 0; i < nr; i++)
        S->atten_i[i] = (P->flow_attenuate_values[i] > zero) ? one / P->flow_attenuate_values[i] : DBL_MAX;
    }
    if (P->use_flow_from_files) {
      if (P->n_flows < 2 || !P->flow_jd || !P->flow_vt || !P->flow_vp) return 3;
      load_flow_from_files(S); /* F:2564 */
    }
  }
  if (P->advance_diffusion) load_diffusion(S);
  if (P->advance_source) {
    int rc = load_source(S);
    if (rc) return rc;
  }
  if (P->assimilate_data && n_da > 0) {
    S->n_da = n_da; S->da_times = da_times; S->da_maps = da_maps;
    load_data_assimilation(S);
  }
  S->h = dalloc((size_t)nr * 14);
  analysis_and_history(S);
  output_map_index(S);
  /* main loop */
  for (;;) {
    S->ntime++;
    if (P->advance_flow) update_flow(S);
    if (P->advance_source) update_source(S);
    update_timestep(S);
    flux_transport_step(S);
    S->time = S->time + S->dtime_global;
    apply_data_assimilation(S);
    analysis_and_history(S);
    output_map_index(S);
    if (S->time >= P->time_end) break;
    if (max_steps > 0 && S->ntime >= max_steps) break;
  }
  if (f_out) memcpy(f_out, S->f, sizeof(double) * (size_t)ntm * npm * nr);
  if (hist) capture_map(S, hist->map_final); /* <root>_final.h5, F:1390 */
  if (timing_out) {
    timing_out[0] = (double)S->ntime;
    timing_out[1] = S->time;
    timing_out[2] = S->cell_updates;
  }
  return 0;
}

/* Grid sizes the caller must allocate f_out with: ntm, npm. */
void orc_sizes(const orc_params *P, int n1, int n2, int *ntm, int *npm) {
  if (n1 <= 0) { n1 = P->res_np; n2 = P->res_nt; }
  *ntm = n2;
  *npm = n1 + 1;
}

/* One assimilation blend on a given field (test entry point): t[ntm], p[npm1]
 * scales, f (ntm, npm1+1, nr) theta fastest updated in place, map3
 * (npm1, ntm, 3).  Returns 0 on success. */
int orc_da_blend(const orc_params *P, int ntm, int npm1, const double *t, const double *p, double *f,
                 const double *map3) {
  orc Sx;
  orc *S = &Sx;
  memset(S, 0, sizeof(*S));
  S->P = P;
  S->nr = P->n_realizations;
  S->ntm1 = ntm; S->npm1 = npm1;
  S->ntm = ntm; S->npm = npm1 + 1; S->nt = ntm + 1; S->np = npm1 + 1;
  S->t = dalloc(ntm); S->p = dalloc(S->npm);
  for (int j = 1; j <= ntm; j++) V1(S->t, j) = t[j - 1];
  for (int k = 1; k <= npm1; k++) V1(S->p, k) = p[k - 1];
  V1(S->p, npm1 + 1) = V1(S->p, 2) + twopi;
  if (set_mesh(S)) return -1;
  S->f = f;
  S->n_da = 1;
  S->da_times = NULL;
  S->tidx0 = (int *)calloc(S->nr, sizeof(int));
  S->tidx1 = (int *)calloc(S->nr, sizeof(int));
  for (int r = 0; r < S->nr; r++) {
    S->tidx0[r] = -1; S->tidx1[r] = -1;
    for (int j = 1; j <= S->ntm; j++)
      if (V1(S->t, j) >= P->assimilate_data_lat_limits[r] * d2r && S->tidx0[r] == -1) S->tidx0[r] = j;
    for (int j = S->ntm; j >= 1; j--)
      if (V1(S->t, j) <= (pi - P->assimilate_data_lat_limits[r] * d2r) && S->tidx1[r] == -1) S->tidx1[r] = j;
  }
  da_blend(S, map3);
  return 0;
}

/* get_flux (F:8672-8750) of every realization of f (ntm, npm1+1, nr), theta
 * fastest, on the mesh of the scales t[ntm], p[npm1] (test entry point).
 * flux_p, flux_m receive nr values each.  Returns 0 on success. */
int orc_get_flux(int ntm, int npm1, int nr, const double *t, const double *p, const double *f, double *flux_p,
                 double *flux_m) {
  orc Sx;
  orc *S = &Sx;
  memset(S, 0, sizeof(*S));
  S->nr = nr;
  S->ntm1 = ntm; S->npm1 = npm1;
  S->ntm = ntm; S->npm = npm1 + 1; S->nt = ntm + 1; S->np = npm1 + 1;
  S->t = dalloc(ntm); S->p = dalloc(S->npm);
  for (int j = 1; j <= ntm; j++) V1(S->t, j) = t[j - 1];
  for (int k = 1; k <= npm1; k++) V1(S->p, k) = p[k - 1];
  V1(S->p, npm1 + 1) = V1(S->p, 2) + twopi;
  if (set_mesh(S)) return -1;
  for (int i = 0; i < nr; i++)
    get_flux(S, f + (size_t)i * ntm * S->npm, &flux_p[i], &flux_m[i]);
  return 0;
}
