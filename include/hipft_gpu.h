/*
 * hipft_gpu.h -- C ABI of the B200 (sm_100a) flux-transport library.
 *
 * Drop-in for the hot-path subroutines of HipFT (src/hipft.f90, v1.19.3).
 * HipFT keeps its solver state in Fortran module arrays; this library keeps
 * the same state on the GPU behind an opaque handle.  Every entry point takes
 * plain host pointers and sizes, copies what it needs, and returns an int
 * status (HIPFT_OK = 0).  Host buffers are only borrowed for the duration of
 * a call.  A handle is used from one host thread (the reference runs
 * MPI_THREAD_FUNNELED, src/hipft.f90:1090).
 *
 * Field layout at the ABI is the reference's: f(ntm, npm, nr) in Fortran
 * column-major order, theta fastest, with the two-point periodic overlap in
 * phi (npm = npm1 + 1; column 1 == column npm-1, column npm == column 2),
 * src/hipft.f90:2114-2126.  Data-assimilation maps are the reference's
 * (npm1, ntm, 3) phi-fastest slices [data, weight, mu], src/hipft.f90:4234.
 *
 * Each declaration cites the reference routine it replaces.
 */
#ifndef HIPFT_GPU_H
#define HIPFT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference prints and calls endrun(.true.)
 * (src/hipft.f90:970-1004); a Fortran shim maps a nonzero status to that. */
enum {
  HIPFT_OK = 0,
  HIPFT_EINVAL = 1,   /* bad argument or size                              */
  HIPFT_ECUDA = 2,    /* CUDA runtime error (message in hipft_gpu_last_error) */
  HIPFT_ETIMEOUT = 3, /* a bounded device wait gave up                     */
  HIPFT_ENAN = 4,     /* non-finite value detected                          */
  HIPFT_ESTATE = 5,   /* call out of order (e.g. step before set_field)     */
  HIPFT_EIO = 6,      /* file could not be read/written                     */
  HIPFT_ENOMEM = 7,   /* device allocation failed                           */
  HIPFT_ECOMM = 8     /* the all-reduce callback reported an error          */
};

typedef struct hipft_gpu hipft_gpu;

/* Mesh and realization count.  Replaces set_mesh's inputs
 * (src/hipft.f90:6495-6653): t(ntm1) and p(npm1) are the map scales. */
typedef struct {
  int ntm;          /* theta points including both poles                    */
  int npm1;         /* phi points including 0 and 2*pi (one-point overlap)  */
  int nr;           /* realizations held by this handle                     */
  int device;       /* CUDA device ordinal                                  */
  const double *t;  /* [ntm]  theta scale, t[0]=0, t[ntm-1]=pi              */
  const double *p;  /* [npm1] phi scale,   p[0]=0, p[npm1-1]=2*pi           */
} hipft_grid;

/* Numerical-method switches with the reference's namelist names and
 * meanings (src/hipft.f90:580-700, presets 8583-8608). */
typedef struct {
  int advance_flow;
  int flow_num_method;        /* 1 FE+UW, 2 SSPRK33+UW, 3 SSPRK33+WENO3, 4 SSPRK43+WENO3 */
  double upwind;              /* upwind coefficient (1 = full upwind)        */
  double weno_eps;            /* <=0: epsilon = cell width                    */
  int strang_splitting;       /* 1: A(dt/2) D(dt) A(dt/2), else A(dt) D(dt)   */
  int advance_diffusion;
  int diffusion_num_method;   /* 1 Euler, 2 RKL2, 3 RKG2                      */
  int diffusion_subcycles;    /* 0 = automatic (PTL) subcycling               */
  int diffusion_coef_grid;    /* add grid-based diffusion                      */
  double diffusion_coef_factor; /* km^2/s -> Rs^2/hr by default               */
  const double *diffusion_coef_constants; /* [nr], km^2/s; also validation 1   */
  double pole_flux_lat_limit; /* degrees, for the polar-flux diagnostics       */
  int verbose;
  int advance_source;         /* source steps in flux_transport_step           */
} hipft_params;

/* Analytic / prescribed flow definition (update_flow, src/hipft.f90:3371-3523;
 * add_flow_*_analytic 7219-7285).  Per-realization vectors have length nr
 * and may be NULL when their model is off. */
typedef struct {
  int flow_dr_model;          /* 1: vp += st*(p0 + p2 ct^2 + p4 ct^4) [m/s]   */
  int flow_mf_model;          /* 1: vt -= sth*(p1 c + p3 c^3 + p5 c^5) [m/s]  */
  const double *dr_p0, *dr_p2, *dr_p4;
  const double *mf_p1, *mf_p3, *mf_p5;
  double flow_vp_rigid_omega; /* km/s, vp += omega*st                          */
  double flow_vt_const;       /* km/s                                          */
  double flow_rigid_omega;    /* km/s, rotated rigid rotation (2-D)            */
  int flow_attenuate;         /* attenuate by tanh(|Br|/value) each step       */
  const double *flow_attenuate_values; /* [nr], Gauss                          */
} hipft_flow_def;

/* Data-assimilation options (apply_data_assimilation, src/hipft.f90:4148-4306;
 * assimilate_new_data 4083-4146). */
typedef struct {
  int add;                    /* assimilate_data_add: f += w*d instead of blend */
  int custom_from_mu;         /* weight = mu^power where mu > limit, else 0    */
  int balance_flux;           /* multiplicative balance of the increment       */
  double mult_fac;            /* assimilate_data_mult_fac                      */
  const double *mu_power;     /* [nr]                                          */
  const double *mu_limit;     /* [nr]                                          */
  const double *lat_limit;    /* [nr] degrees; <=0 disables the cap mask       */
} hipft_da_opts;

/* What one diffusion_step did (history columns, src/hipft.f90:2666-2670). */
typedef struct {
  double dtime_diffusion_euler; /* Gershgorin explicit-Euler limit            */
  int64_t sts_s;                /* stages in the last super-step (or Euler cycles) */
  int64_t subcycles;            /* diffusion cycles taken (or its diagnostic)  */
  int64_t total_stages;         /* stage launches summed over the call         */
} hipft_diffusion_info;

/* Called after each diffusion cycle (the reference's verbose>1 per-cycle
 * analysis + history output, src/hipft.f90:4659-4669).  time_stepped is the
 * amount of the step covered so far; subcycle_diag is the
 * CEILING((dt - time_stepped)/dt_cycle) diagnostic. */
typedef void (*hipft_cycle_cb)(void *user, int cycle, double time_stepped, double dt_cycle,
                               int64_t sts_s, int64_t subcycle_diag);

/* ---- lifecycle ------------------------------------------------------- */

/* setup's device part: set_mesh (6495), load_flows (2535) + load_weno (6846),
 * load_diffusion (6655) + load_diffusion_matrix (4927) +
 * get_dtime_diffusion_euler (4985).  Allocates all device memory. */
int hipft_gpu_create(const hipft_grid *grid, const hipft_params *params, hipft_gpu **out);
int hipft_gpu_destroy(hipft_gpu *h);
/* Copies the last error message (NUL terminated). */
int hipft_gpu_last_error(const hipft_gpu *h, char *buf, size_t len);
/* Library version string and the device it was built for ("sm_100a"). */
const char *hipft_gpu_version(void);

/* ---- field I/O ---------------------------------------------------------- */

/* f(ntm, npm, nr), theta fastest (replaces `!$omp target enter data
 * map(to:f)`, src/hipft.f90:2159). */
int hipft_gpu_set_field(hipft_gpu *h, const double *f);
/* Copies f back (replaces `!$omp target update from`, src/hipft.f90:2844). */
int hipft_gpu_get_field(hipft_gpu *h, double *f);
/* Initial map in the file's PT layout (npm1, ntm, nr): transpose, periodic
 * fix-up, m=0 poles, optional balance, multiply (src/hipft.f90:2116-2172). */
int hipft_gpu_load_initial_map(hipft_gpu *h, const double *map_pt, int flux_balance,
                               double mult_fac);

/* ---- several processes (realizations split over ranks) ------------------- */

/* The reference splits the realizations over MPI ranks
 * (set_local_number_of_realizations, src/hipft.f90:1006-1063) and keeps one
 * time step for all of them with four scalar all-reduces: the explicit
 * diffusion limit (MIN, src/hipft.f90:5036), PTL's max |A f| (MAX, 5103) and
 * time step (MIN, 5141), and the flow CFL limit (MIN, 7345).  A handle that
 * holds one rank's realizations gets those reductions through this callback:
 * it replaces *value by the MIN (op 0) or MAX (op 1) over all ranks and
 * returns 0 (anything else becomes HIPFT_ECOMM).  Every rank calls the
 * library in the same sequence, so the callbacks happen in the same order on
 * all ranks.  Setting it reduces the explicit diffusion limit at once, so
 * all ranks call this right after hipft_gpu_create. */
enum { HIPFT_RED_MIN = 0, HIPFT_RED_MAX = 1 };
typedef int (*hipft_allreduce_cb)(void *user, int op, double *value);
int hipft_gpu_set_allreduce(hipft_gpu *h, hipft_allreduce_cb cb, void *user);

/* ---- flows -------------------------------------------------------------- */

/* Stores the flow definition; marks the flow for (re)building. */
int hipft_gpu_set_flow(hipft_gpu *h, const hipft_flow_def *def);
/* update_flow (src/hipft.f90:3371): rebuilds vt, vp (and the WENO LF alpha,
 * set_lf_alpha 6940) when needed.  *updated = 1 when the flow changed, which
 * tells the caller to recompute the CFL limit. */
int hipft_gpu_update_flow(hipft_gpu *h, int *updated);
/* Flows from files (use_flow_from_files): the 2-D flow, shared by all
 * realizations, that update_flow starts from before adding the analytic
 * models (flow_from_files_current_vt/vp of add_flow_from_files,
 * src/hipft.f90:3525-3673, and load_flow_from_files, 3675-3800).
 * vt_pt: the theta-velocity file as read, (npm1, nt) phi fastest, in m/s;
 * vp_pt: the phi-velocity file, (np, ntm).  at_load != 0 applies the
 * load-time phi rule (vt column npm = column 2), else the update rule
 * (set_periodic_bc_3d on both).  The flow is then rebuilt at every
 * update_flow, as the reference does while flows come from files. */
int hipft_gpu_set_flow_from_files(hipft_gpu *h, const double *vt_pt, const double *vp_pt, int at_load);
/* get_flow_dtmax (src/hipft.f90:7287-7350): CFL limit over all cells and
 * realizations, x2 for Strang splitting, x2 for SSPRK(4,3). */
int hipft_gpu_flow_dtmax(hipft_gpu *h, double *dtmax);

/* ---- sources (advance_source) ---------------------------------------------- */

/* The source from a file, already on the main mesh (load_source interpolates
 * the file with interp2d, src/hipft.f90:7094-7146): data (ntm, npm), theta
 * fastest, the same for every realization. */
int hipft_gpu_set_source_file(hipft_gpu *h, const double *data_tp);
/* generate_rfe (src/hipft.f90:8809-8921) into frame slot 0 or 1, then
 * balance_flux of each realization (src/hipft.f90:3931-3934, 7199-7202).
 * model 1: flux per cell, 2: flux per unit area.  rnd_tp (ntm, npm), theta
 * fastest: the reference's rnd_nums, normal deviates times pi/sqrt(2 pi),
 * read on columns 2..npm-1 only.  uf [nr]: unsigned flux per hour per cell
 * (model 1) or per unit area (model 2) in code units. */
int hipft_gpu_set_rfe_frame(hipft_gpu *h, int slot, int model, const double *rnd_tp, const double *uf);
/* update_source (src/hipft.f90:3875-3947): source = [file] +
 * [(1-alpha) frame(slot1) + alpha frame(slot2)]. */
int hipft_gpu_update_source(hipft_gpu *h, int use_file, int use_rfe, int slot1, int slot2, double alpha);
/* source_step (src/hipft.f90:4697-4732): f += dt * source.
 * flux_transport_step calls it when advance_source is set. */
int hipft_gpu_source_step(hipft_gpu *h, double dt);

/* ---- the time step -------------------------------------------------------- */

/* advection_step (src/hipft.f90:4509) with FE / SSPRK(3,3) / SSPRK(4,3)
 * (7409-7582) over upwind or WENO3 operators (7615-7925). */
int hipft_gpu_advection_step(hipft_gpu *h, double dt);
/* diffusion_step (src/hipft.f90:4551): subcycling (fixed or PTL,
 * get_dtime_diffusion_ptl 5042) of Euler / RKL2 / RKG2 (5163-5475) through
 * diffusion_operator_cd (7927).  cb may be NULL. */
int hipft_gpu_diffusion_step(hipft_gpu *h, double dt, hipft_cycle_cb cb, void *user,
                             hipft_diffusion_info *info);
/* flux_transport_step (src/hipft.f90:4463): Strang A(dt/2) D(dt) A(dt/2) or
 * Lie A(dt) D(dt), as selected at create time. */
int hipft_gpu_flux_transport_step(hipft_gpu *h, double dt, hipft_cycle_cb cb, void *user,
                                  hipft_diffusion_info *info);

/* ---- data assimilation --------------------------------------------------- */

/* Blend one observed map into every realization: per-realization mu-power
 * weights and latitude caps, mult factor, f += w*(d - f) (or w*d), seam,
 * optional balance.  data3_pt: (npm1, ntm, 3) phi fastest. */
int hipft_gpu_assimilate(hipft_gpu *h, const double *data3_pt, const hipft_da_opts *opts);

/* ---- diagnostics ---------------------------------------------------------- */

/* Validation modes of analysis_step (src/hipft.f90:3148-3175):
 * mode 1: fval = fval_u0_pt * exp(-42 D factor (time - time_start));
 *         fval_u0_pt is (npm1, ntm, nr) PT.
 * mode 2: analytic Gaussian pair moved by vt_const / vp_omega (km/s). */
int hipft_gpu_set_validation(hipft_gpu *h, int mode, const double *fval_u0_pt, double width,
                             double vt_const, double vp_omega, double time_start);
/* analysis_step (src/hipft.f90:3098-3336): hist is [nr][14] =
 * BR_MIN, BR_MAX, BR_ABS_MIN, FLUX_POSITIVE, FLUX_NEGATIVE,
 * NPOLE_FLUX_POSITIVE, NPOLE_FLUX_NEGATIVE, SPOLE_FLUX_POSITIVE,
 * SPOLE_FLUX_NEGATIVE, NPOLE_AREA, SPOLE_AREA, EQ_DIPOLE, AX_DIPOLE,
 * VALIDATION_ERR_HHabs. */
int hipft_gpu_analysis(hipft_gpu *h, double time, double *hist);
/* get_flux (src/hipft.f90:8672): flux_p[nr], flux_m[nr] of the field. */
int hipft_gpu_get_flux(hipft_gpu *h, double *flux_p, double *flux_m);
/* balance_flux (src/hipft.f90:8752) on every realization of the field. */
int hipft_gpu_balance_flux(hipft_gpu *h);

/* ---- introspection --------------------------------------------------------- */

typedef struct {
  int ntm, npm, nr, ldt;        /* ldt: padded theta stride on the device     */
  double dtime_diffusion_euler;
  int64_t sts_s;
  int64_t kernel_launches;      /* launches of this library's kernels so far  */
  int64_t cell_stage_updates;   /* unique cells x stages advanced so far      */
  size_t device_bytes;          /* device memory held by the handle           */
  int64_t rkg2_stages;          /* super-step stages k >= 2 run so far         */
  int64_t rkg2_cell_stages;     /* unique cells x stages k >= 2 advanced so far */
} hipft_info;
int hipft_gpu_info(const hipft_gpu *h, hipft_info *info);
/* Per-kernel timing with CUDA events on the handle's stream.  Kinds:
 * 0 RKG2/RKL2 stages k >= 2 (the fused Laplacian + combine kernels, one
 * or two stages per launch), 1 advection stage
 * (fused WENO3/upwind operator + SSPRK combine), 2 pole-ring sums,
 * 3 everything else.  Enabling resets the counters. */
enum { HIPFT_K_STS = 0, HIPFT_K_ADV = 1, HIPFT_K_RING = 2, HIPFT_K_OTHER = 3, HIPFT_K_NKINDS = 4 };
int hipft_gpu_set_profiling(hipft_gpu *h, int on);
/* Launch count and summed device time (ms) of one kernel kind since
 * profiling was enabled (synchronizes the stream). */
int hipft_gpu_kernel_time(hipft_gpu *h, int kind, int64_t *launches, double *total_ms);
/* No counterpart in the reference: a one-line description of how the handle
 * runs (shared or ragged schedule; the two-stage RKG2 kernel the autotuner
 * picked for this grid and its timed launch, or the one HIPFT_STS_PAIR fixed). */
int hipft_gpu_describe(hipft_gpu *h, char *buf, size_t len);
/* Runs subsequent work on a caller-owned cudaStream_t (NULL: the handle's). */
int hipft_gpu_set_stream(hipft_gpu *h, void *cuda_stream);
int hipft_gpu_synchronize(hipft_gpu *h);
/* Zero-copy view of the current field for the PyTorch binding: the device
 * address of f(j, k, i) at (*ptr)[(i-1)*npm*ldt + (k-1)*ldt + (j-1)] (theta
 * padded to *ldt).  Returns after the handle's stream has finished, so the
 * field may be read on any stream.  Valid until the next call that advances,
 * assimilates or sets the field (the library rotates its buffers). */
int hipft_gpu_field_device_ptr(hipft_gpu *h, double **ptr, int *ldt);
/* No counterpart in the reference: a self-check of the error path that every
 * bounded device wait of this library takes.  A kernel waits on an mbarrier
 * that nothing completes, gives up after `limit` polls (1..2^22) and sets the
 * handle's error flag; the call then returns HIPFT_ETIMEOUT, as a stalled
 * copy would, and the handle stays usable. */
int hipft_gpu_check_bounded_wait(hipft_gpu *h, unsigned int limit);

/* ---- ragged batches (no counterpart in the reference) ---------------------- */

/* The reference advances all realizations with one schedule: one dt, one
 * explicit-Euler limit, one RKG2/RKL2 stage count and one PTL subcycle
 * sequence, from global MIN/MAX reductions (src/hipft.f90:5036, 5103, 5141,
 * 7345); that is this library's default ("plain" mode).  on = 1 switches a
 * handle to ragged batching: every realization keeps the schedule it would
 * have if it were run alone -- its own Gershgorin limit (get_dtime_diffusion_
 * euler, 4985), its own PTL subcycles (get_dtime_diffusion_ptl, 5042) and
 * stage counts (load_sts_rkg2 5361 / rkl2 5244), and, when a step is longer
 * than its own CFL limit (get_flow_dtmax, 7287), ceil(dt / limit) advection
 * substeps -- while each launch still covers every realization that has work
 * left.  A step of a ragged batch therefore equals, realization by
 * realization, the reference run with that realization alone at the same
 * dt.  Needs RKG2 or RKL2 with per-realization constant coefficients,
 * SSPRK(3,3) or SSPRK(4,3) advection, and no all-reduce callback (else
 * HIPFT_EINVAL / HIPFT_ESTATE).  The cycle callback of diffusion_step is not
 * called in ragged mode; hipft_gpu_ragged_schedule reports the schedule. */
int hipft_gpu_set_ragged(hipft_gpu *h, int on);
/* get_flow_dtmax (src/hipft.f90:7287-7350) of each realization alone:
 * dtmax[nr] (x2 for Strang, x2 for SSPRK(4,3), as the reference scales it). */
int hipft_gpu_flow_dtmax_each(hipft_gpu *h, double *dtmax);
/* Per-realization schedule of the last ragged step (arrays of nr, each may
 * be NULL): stage count of the last super-step, diffusion subcycles,
 * advection substeps per advection call, and the Euler limit. */
int hipft_gpu_ragged_schedule(hipft_gpu *h, int64_t *sts_s, int64_t *subcycles, int64_t *adv_substeps,
                              double *dt_euler);

/* on = 1: every hipft_gpu_flux_transport_step runs as ONE launch of a CUDA
 * graph captured on the first such step (and again when flows, tables or
 * modes it baked in change).  No counterpart in the reference, whose step
 * (flux_transport_step, src/hipft.f90:4463-4507) is a host loop over kernels.
 * The decisions the host-driven step takes between launches -- PTL subcycle
 * lengths (get_dtime_diffusion_ptl, 5042-5161), RKG2/RKL2 stage counts and
 * coefficients (5244-5475), advection substeps of ragged batches -- are taken
 * by device kernels with the same arithmetic, and the loops they size are
 * conditional WHILE nodes, so a graph-run step gives the same field, bit for
 * bit, as the host-driven step, in plain and in ragged mode.  The step then
 * needs no host synchronization (unless an info struct is passed).  Needs
 * RKG2 or RKL2 with per-realization constant coefficients (or no diffusion),
 * no sources and no all-reduce callback (else HIPFT_EINVAL / HIPFT_ESTATE);
 * flux_transport_step with a cycle callback returns HIPFT_ESTATE. */
int hipft_gpu_set_graph(hipft_gpu *h, int on);

/* ---- allocation-free flux integral ------------------------------------------ */

/* No counterpart in the reference: get_flux (src/hipft.f90:8672) for callers
 * that cannot allocate GPU memory -- e.g. a Fortran code whose maps live in
 * OpenMP `target enter data` mappings and are handed over as use_device_ptr
 * addresses, or an application that runs the GPU from a fixed arena.  It
 * allocates nothing: f_dev is the caller's device field f(j,k,i) at
 * f_dev[((i-1)*(npm1+1) + (k-1))*ldt + (j-1)] (ldt >= ntm), t/p are the host
 * scales, flux_p/flux_m receive nr values each.  Its scratch is one
 * file-scope device array of about 1.6 MB that every GPU loading the library
 * keeps until exit; it bounds the sizes to ntm <= 16384, npm1 <= 16384,
 * nr <= 2000 and 2*nr*ceil(npm1/16) <= 131072 (else HIPFT_EINVAL).  Calls
 * share that scratch, so calls that overlap on the GPU race.  The first call
 * on a device looks up the scratch address (do it before any stream
 * capture).  err (may be NULL) receives a message on failure. */
int hipft_get_flux_noalloc(const double *f_dev, int ntm, int npm1, int nr, int ldt, const double *t,
                           const double *p, double *flux_p, double *flux_m, void *cuda_stream, char *err,
                           size_t err_len);

/* ---- standalone driver ----------------------------------------------------- */

/* Runs `program HIPFT` (src/hipft.f90:869-968) for the hot-path subset: reads
 * the hipft.in namelist at `namelist_path`, resolves file names relative to
 * `run_dir`, writes hipft_history_{num,sol}_rNNNNNN.out (formats of
 * src/hipft.f90:1616-1646, 2633-2634) into `run_dir`. */
int hipft_run(const char *namelist_path, const char *run_dir, int device);
/* Same, and copies the final field f(ntm, npm, nr) into f_out when f_len
 * equals ntm*npm*nr (the data of the reference's hipft_brmap_final.h5,
 * wrap_it_up src/hipft.f90:1381-1412, before its PT transpose). */
int hipft_run_field(const char *namelist_path, const char *run_dir, int device, double *f_out, size_t f_len);

/* One rank of a run whose realizations are split over processes, as the
 * reference splits them over MPI ranks (src/hipft.f90:1006-1063: rank r takes
 * the next floor(n/nranks) realizations, the low ranks one more).  allreduce:
 * the scalar reductions of hipft_gpu_set_allreduce; gather: rank 0's `global`
 * receives every rank's `local` (n_local doubles) concatenated in rank order,
 * the other ranks pass global = NULL (write_map's MPI_Gatherv,
 * src/hipft.f90:2874-2896); both return 0 on success.  Every rank writes the
 * history files of its own realizations, rank 0 the maps and the map list.
 * f_out receives this rank's realizations (f_len = ntm*npm*nr_local). */
typedef struct {
  int rank, nranks;
  hipft_allreduce_cb allreduce;
  int (*gather)(void *user, const double *local, int64_t n_local, double *global);
  void *user;
} hipft_shard;
int hipft_run_shard(const char *namelist_path, const char *run_dir, int device, const hipft_shard *shard,
                    double *f_out, size_t f_len);

/* ---- discrete adjoint (PyTorch binding; no reference counterpart) ---------- */

/* Reverse pass of one flux_transport_step for gradients of a map misfit.
 * Device pointers, each a field in the handle's layout (nr x npm x ldt,
 * theta padded to ldt, see hipft_gpu_field_device_ptr):
 *   f_in  the step's input field (unchanged);
 *   fbar  in: cotangent of the step's output, out: cotangent of its input,
 *         both "folded" (phi seam columns 1 and npm carry nothing; their
 *         dependence is on columns npm-1 and 2);
 *   dacc  [nr] += sum over RKG2 stages of mu~_k dt <A^T Wbar, Y_{k-1}> (the
 *         derivative with respect to the diffusion coefficient constant c
 *         is dacc / c);
 *   gflow 5 fields += per-cell flow cotangents: theta LN (vt(j)+at(j)),
 *         theta LP (vt(j+1)-at(j)), theta upwind faces (vt(j)), phi LN
 *         (vp+ap), phi LP (vp-ap), each already multiplied by x/2.
 * The step is replayed from f_in with every stage input kept; its schedule
 * (PTL subcycle dts, RKG2 stage counts) is the forward's and is held fixed.
 * Requires WENO3+SSPRK(4,3) with analytic flows or flows from files (not
 * attenuated or rotated flows, which depend on the field or are NaN; with a
 * 2-D flow the gflow cotangents are per cell of that flow), RKG2 with
 * per-realization constant diffusion coefficients and no sources (else
 * HIPFT_ESTATE).  The current field becomes the step's output. */
int hipft_adj_step(hipft_gpu *h, double dt, const double *f_in, double *fbar, double *dacc, double *gflow);
/* hipft_adj_step in two halves, for checkpoint segments that are taped once:
 * hipft_adj_record runs one flux_transport_step of the current field (the
 * field becomes its output, as with hipft_gpu_flux_transport_step, bit for
 * bit) and pushes the step's tape onto a stack; hipft_adj_reverse runs the
 * reverse pass of the most recently recorded step (same fbar, dacc, gflow
 * arguments as hipft_adj_step) and pops its tape.  A segment of n steps is
 * recorded in order and reversed in the opposite order; hipft_adj_recorded
 * gives the number of steps on the stack and (slots_used may be NULL) the
 * tape fields they hold. */
int hipft_adj_record(hipft_gpu *h, double dt);
int hipft_adj_reverse(hipft_gpu *h, double *fbar, double *dacc, double *gflow);
int hipft_adj_recorded(hipft_gpu *h, int64_t *n, int64_t *slots_used);
/* Drops every recorded step and keeps the tape memory for the next ones. */
int hipft_adj_clear(hipft_gpu *h);
/* Replace the current field from device memory in the handle's layout
 * (nr x npm x ldt), e.g. a checkpoint taken through
 * hipft_gpu_field_device_ptr; cached pole sums are dropped. */
int hipft_gpu_set_field_device(hipft_gpu *h, const double *f_dev);
/* Most fields the adjoint's tape has held at once since the last release
 * (tape slots of the recorded steps plus the block-recompute fields; device
 * memory, fieldn doubles each). */
int hipft_adj_tape_fields(hipft_gpu *h, int64_t *n);
/* Tape budget of one recorded step.  A super-step of s RKG2 stages keeps all
 * s+1 stage fields when they fit max_fields (0: half of the free device
 * memory at the time); otherwise it keeps stage checkpoints -- the pair
 * (Y_{c-1}, Y_c) every q stages, q even near sqrt(2 s) -- and the reverse pass
 * recomputes one block of q stages at a time from its pair (about
 * 2 sqrt(2 s) fields, one more forward pass of the diffusion).
 * stage_spacing > 0 (even) forces that q.  Results do not depend on q. */
int hipft_adj_set_tape_limit(hipft_gpu *h, int64_t max_fields, int64_t stage_spacing);
/* Frees the tape and drops recorded steps (the tape grows to the largest
 * set of recorded steps seen and is otherwise kept until the handle is
 * destroyed). */
int hipft_adj_release(hipft_gpu *h);
/* Reverse of one data-assimilation blend (apply_data_assimilation,
 * src/hipft.f90:4116-4141, same map and options as the forward call):
 * fbar (device, the handle's layout, folded) becomes (1 - w) fbar on every
 * core cell for the blend f += w (d - f), and is unchanged for the additive
 * form f += w d.  The balanced increment (balance_flux, 8794-8801) needs
 * the field it was applied to: hipft_adj_assimilate_at (here HIPFT_ESTATE). */
int hipft_adj_assimilate(hipft_gpu *h, const double *data3_pt, const hipft_da_opts *o, double *fbar);
/* Reverse of one data-assimilation step given the field it was applied to,
 * the balanced increment included (apply_data_assimilation,
 * src/hipft.f90:4116-4141, with balance_flux of the increment, 8752-8807):
 * f_pre (device, the handle's layout) is the field before the assimilation.
 * The forward scales the increment D = w (d - f) by 1/r where D > 0 and by r
 * elsewhere, r = sqrt(|F+/F-|) of get_flux's area-weighted sums; the reverse
 * also differentiates r through both sums (one reduction pass over D and
 * fbar, one pointwise pass).  A one-signed increment (F+ or F- zero, F+ + F-
 * nonzero) is not differentiated (HIPFT_ESTATE).  Without balance_flux, or
 * for the additive form, this is hipft_adj_assimilate (f_pre may be NULL). */
int hipft_adj_assimilate_at(hipft_gpu *h, const double *data3_pt, const hipft_da_opts *o, const double *f_pre,
                            double *fbar);

/* ---- map files ------------------------------------------------------------- */

/* Minimal reader of the reference's HDF5 maps (rdh5, src/hipft.f90:5678):
 * dataset "Data" plus scales "dim1".."dim3".  Sizes first (pass NULL
 * buffers), then data.  dims are Fortran order (fastest first); unused
 * dims are 1.  Data is converted to double. */
int hipft_h5_read(const char *path, int *ndim, int64_t dims[3], double *data, double *s1,
                  double *s2, double *s3);

/* Writer of the reference's HDF5 maps (wrh5, src/hipft.f90:6155-6351):
 * dataset "Data" (float32 when single_precision, else float64) of Fortran
 * dimensions dims[0..ndim-1] (dims[0] varies fastest in `data`) and scale
 * datasets "dim1".."dimN" (s1..s3, converted like the data) attached to it
 * as HDF5 dimension scales.  Returns HIPFT_EIO when the file cannot be
 * written. */
int hipft_h5_write(const char *path, int ndim, const int64_t dims[3], const double *data, const double *s1,
                   const double *s2, const double *s3, int single_precision);

#ifdef __cplusplus
}
#endif
#endif /* HIPFT_GPU_H */
