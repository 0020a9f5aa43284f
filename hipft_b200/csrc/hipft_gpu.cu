// hipft_gpu.cu -- host side of the B200 flux-transport library (C ABI in
// include/hipft_gpu.h).  Owns all device state behind an opaque handle and
// sequences the kernels of kernels.cuh the way HipFT's Fortran routines
// sequence their do-concurrent loops (src/hipft.f90).
#include <cuda_runtime.h>
#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/hipft_gpu.h"
#include "kernels.cuh"
#include "sts_pair_ws.cuh"
#include "sts_quad_ws.cuh"
#include "adjoint.cuh"
#include "graph_step.cuh"

using namespace hipft;

namespace {

// Constants of the reference (src/hipft.f90:83-136).
constexpr double c_pi = 3.1415926535897932;
constexpr double c_pi_i = 0.3183098861837907;
constexpr double c_twopi = 6.2831853071795864;
constexpr double c_pi_two = 1.5707963267948966;
constexpr double c_threepi_two = 4.71238898038469;
constexpr double c_d2r = 0.017453292519943295;
constexpr double c_rsun_cm2 = 4.84416e21;
constexpr double c_km_s_to_rs_hr = 0.005172413793103448;
constexpr double c_m_s_to_rs_hr = 5.172413793103448e-06;
constexpr double c_safety = 0.95;
constexpr double c_three_quarter = 0.75;
constexpr double c_quarter = 0.25;
constexpr double c_sixth = 0.16666666666666666;
constexpr double c_two_third = 0.66666666666666666;
constexpr double c_third = 0.33333333333333333;

constexpr int kNBuf = 8;  // current field + scratch: u0, dty0, two inputs and up to four outputs of a pass

int round_up(int a, int b) { return (a + b - 1) / b * b; }

// Two-stage kernel kinds (see the autotuner) and the plan a handle uses.
enum { PK_SINGLE = 0, PK_WS_ROWS1 = 4, PK_WS_ROWS2 = 5, PK_WS_BULK = 6, PK_WS_QUAD = 7 };
struct PairPlan {
  int kind = -1;    // PK_*; -1: not chosen yet
  int ctas_per_sm = 2;
  double ms = 0.0;  // timed ms per launch pair (0: not timed)
  int candidates = 0;
};

double pow3(double c) { return c * c * c; }
double pow5(double c) { return c * c * c * c * c; }

}  // namespace

// ------------------------------------------------------------- adjoint tape
namespace {
// One RKG2 super-step of the replay.  With q == 0 the tape holds every stage:
// slots t0 = u0, t0+1 = dty0, t0+1+k = Y_k (k = 1..s-1).  With stage
// checkpoints (q > 0, even) it holds u0, dty0 and, for each block start
// c = 1, 1+q, 1+2q, ... (odd, the output of a stage pair), the pair
// (Y_{c-1}, Y_c) in slots t0+2+2b, t0+3+2b (b = block index; Y_0 = u0 is
// not stored twice) and the pole-ring sums of Y_c; the reverse pass
// recomputes the stages of one block at a time from its pair.
struct AdjSub {
  double dtl;
  int64_t s;
  std::vector<double> uj, vj, ubj, gj;
  size_t t0;
  int64_t q = 0;
  std::vector<int64_t> cstart;        // block starts c
  std::vector<size_t> ck_prev, ck_cur;  // tape slots of Y_{c-1} (SIZE_MAX: u0) and Y_c
  size_t ring0 = 0;                   // first ring-checkpoint slot (2*nr doubles each)
};

// One taped (recorded) flux_transport_step: its tape slots sit on the tape's
// stack from `first`, its ring checkpoints from `ring_first`.
struct AdjRec {
  double dt = 0.0;
  size_t first = 0, ring_first = 0;
  size_t ta1[4] = {}, ta2[4] = {};  // SSPRK(4,3) stage inputs of the advection calls
  std::vector<AdjSub> subs;         // RKG2 super-steps
};
}  // namespace

struct hipft_gpu {
  int dev = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int ntm = 0, npm = 0, npm1 = 0, nt = 0, np = 0, nr = 0, ldt = 0, ldv = 0;
  int64_t plane = 0;
  size_t fieldn = 0;
  hipft_params P{};
  std::vector<double> Dc;
  int adv_time = 3, adv_space = 2;
  // host mesh, 1-based (element 0 unused)
  std::vector<double> t, p, th, ph, dt, dth, dp, dph, dt_i, dth_i, dp_i, dph_i, st, sth, ct, cth, st_i, sth_i;
  std::vector<void *> allocs;
  size_t dev_bytes = 0;
  Mesh M{};
  DiffCoef DC{};
  Weno W{};
  Flow FL{};
  double bc_flow_n = 0, bc_flow_s = 0, bc_diff_n = 0, bc_diff_s = 0;
  // fields
  double *buf[kNBuf] = {};
  int nbuf = 6;             // allocated fields (8 once the four-stage path is in use)
  int cur = 0;
  bool field_set = false;
  // flows
  bool have_flow = false, flow_needs_updating = false, flow2d = false;
  bool have_file_flow = false;               // flows from files are the base of vt, vp
  double *d_vtf = nullptr, *d_vpf = nullptr;  // [npm][nt+1], [np][ntm+1]
  double *d_fterms = nullptr;                 // analytic terms applied over the file flow
  hipft_flow_def fdef{};
  std::vector<double> f_p0, f_p2, f_p4, f_p1, f_p3, f_p5, f_att;
  double *d_vt1 = nullptr, *d_vp1 = nullptr, *d_at1 = nullptr, *d_ap1 = nullptr;
  double *d_vt = nullptr, *d_vp = nullptr, *d_at = nullptr, *d_ap = nullptr;
  double *d_trig = nullptr, *d_atten = nullptr;
  // diffusion
  double dt_euler = 0.0;
  bool auto_sc = false;
  int64_t sts_s = 0, n_euler = 0, subcycles_state = 0;
  std::vector<double> sts_uj, sts_vj, sts_ubj, sts_gj, sts_b;
  // scratch
  double *d_ring = nullptr;            // ring sums for kernels that take them from a launch of their own
  double *d_ringbuf[2] = {};           // diffusion ring of a stage's input / output (fused path)
  int ring_cur = 0;
  bool dring_valid = false;            // d_ringbuf[ring_cur] holds the ring of the current field
  double *d_rpart = nullptr;
  unsigned int *d_rcount = nullptr;
  int nkb = 0;
  PairTables ptab{};        // coefficient tables of the warp-specialised two-stage kernel
  PairPlan plan{};          // two-stage kernel chosen for this grid (autotuner)
  std::unordered_map<uint64_t, CUtensorMap> ws_map_cache;  // tensor maps of field buffers, by (pointer, box)
  CUtensorMap ws_rt_map{};               // tensor map of ptab.row
  bool ws_rt_ok = false;
  // four stages per pass on the interior theta blocks
  int q_rb_lo = 0, q_rb_hi = -1;         // interior blocks (none when q_rb_hi < q_rb_lo)
  double *d_qcol = nullptr;              // column table of the quad tiles
  int q_LC = 0, q_nkt = 0;
  CUtensorMap q_rt_map{};
  bool q_rt_ok = false;
  // adjoint: fields of one taped forward step, folded work fields (seam
  // columns stay zero), per-block partial sums and pole sums
  std::vector<double *> tape;             // tape slots (allocated in chunks, see adj_slot)
  std::vector<void *> tape_chunks;
  size_t adj_top = 0;                     // first free tape slot (recorded steps sit below, a stack)
  size_t adj_top_max = 0;                 // most tape slots in use at once since the last release
  std::vector<AdjRec> adj_recs;           // recorded steps, oldest first
  std::vector<double *> adj_block;        // stage fields of one recomputed block
  double *d_adj_rings = nullptr;          // ring sums of the stage checkpoints
  size_t adj_rings_cap = 0, adj_rings_n = 0;
  int64_t adj_tape_limit = 0;             // fields the tape may use (0: half the free memory)
  int64_t adj_force_q = 0;                // stage-checkpoint spacing forced by the caller (0: automatic)
  size_t adj_free_seen = 0;               // free device memory + 1 as seen at the run's first record (0: not yet)
  double *adjw[8] = {};
  double *d_dpart = nullptr, *d_gring = nullptr, *d_gpart[2] = {};
  double *d_dpole = nullptr;  // [nr][adj_nch] D partials of the pole-row chunks
  int adj_nch = 1;            // phi-column chunks of k_adj_pole2
  int dpart_per_r = 0;
  // ragged batches: every realization keeps the schedule it would have if run
  // alone (Euler limit, CFL substeps, PTL subcycles, stage counts)
  bool ragged = false;
  std::vector<double> r_dt_euler, r_dtmax;
  bool r_dtmax_valid = false;
  int *d_rlist_dif = nullptr, *d_rlist_adv = nullptr;  // [nr] realization lists of the launches
  StageCoef *d_rcoef = nullptr;                         // [pairs][nr][2] coefficients of a super-step
  size_t rcoef_pairs = 0;
  StageCoef *d_r1coef = nullptr;                        // [nr] stage-1 coefficients
  double *d_rdt = nullptr;                              // [nr] advection substeps
  unsigned long long *d_rbits = nullptr;                // [2*nr] per-realization reductions
  std::vector<int64_t> r_s, r_cycles, r_substeps;       // the last step's schedule
  int64_t rkg2_cell_stages = 0;  // unique cells x stages k >= 2 advanced (both modes)
  // steps run as one CUDA graph each (hipft_gpu_set_graph)
  bool graph_on = false;
  cudaGraph_t g_graph = nullptr;
  cudaGraphExec_t g_exec = nullptr;
  cudaStream_t g_side[3] = {};      // streams the step (and its loop bodies) are captured on
  GArrays GA{};                     // device schedule arrays
  int g_cur = -1;                   // buffer the capture used as the field
  int g_paircap = 0;                // stage pairs the coefficient tables hold
  bool g_pdl = true;                // programmatic launches inside the captured pair loop
  std::vector<unsigned char> g_key; // launch parameters the capture baked in
  GState g_last{};                  // statistics of the last graph-run step
  bool g_stats_valid = true;        // g_last read back since the last launch
  hipft_allreduce_cb red_cb = nullptr;  // scalar all-reduce over ranks (plain-mode sharding)
  void *red_user = nullptr;
  PoleScratch pole{};       // chunk shares of the ring sums for k_pair_poles
  int pole_nch = 0;
  int *d_err = nullptr;   // set by kernels whose bounded waits gave up
  int num_sms = 148;
  unsigned long long *d_bits = nullptr;
  double *d_part = nullptr;
  size_t part_cap = 0;
  double *h_pin = nullptr;
  // analysis
  double *d_anw = nullptr;
  double *d_adj_delta = nullptr;  // increment of a balanced assimilation, recomputed by its reverse
  unsigned char *d_masks = nullptr;
  std::vector<double> da_t, da_p;
  int vmode = 0;
  double *d_fval_u0 = nullptr, *d_vscale = nullptr, *d_vgauss = nullptr;
  double vwidth = 0.03, vt_const = 0.0, vp_omega = 0.0, vtime_start = 0.0;
  // assimilation
  double *d_da = nullptr, *d_daopt = nullptr;
  double *d_daw = nullptr;                   // mu^power weight planes
  int *d_dawidx = nullptr;                   // [nr+1] plane of each realization
  size_t daw_cap = 0;
  std::vector<double> h_daw;
  // sources: file term (one plane), two RFE frames, the blended source
  double *d_src_file = nullptr, *d_rfe[2] = {}, *d_src = nullptr, *d_rnd = nullptr, *d_rfe_aux = nullptr;
  bool src_set = false;
  int *d_tidx = nullptr;
  std::string err;
  int64_t launches = 0, cell_updates = 0;
  int64_t rkg2_stages = 0;  // RKG2/RKL2 stages k >= 2 run (fused kernels)
  // optional per-kernel event timing
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pending[HIPFT_K_NKINDS];
  double prof_ms[HIPFT_K_NKINDS] = {};
  int64_t prof_n[HIPFT_K_NKINDS] = {};
};

static void graph_release(hipft_gpu *h);

// Event pair around one launch when profiling (returns the stop event).
struct ProfScope {
  hipft_gpu *h;
  int kind;
  cudaEvent_t a = nullptr, b = nullptr;
  static cudaEvent_t take(hipft_gpu *h) {
    if (!h->ev_pool.empty()) {
      cudaEvent_t e = h->ev_pool.back();
      h->ev_pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
  }
  ProfScope(hipft_gpu *hh, int k) : h(hh), kind(k) {
    if (!h->profiling) return;
    a = take(h);
    b = take(h);
    if (a) cudaEventRecord(a, h->stream);
  }
  ~ProfScope() {
    if (!h->profiling || !a || !b) return;
    cudaEventRecord(b, h->stream);
    h->ev_pending[kind].push_back({a, b});
  }
};

// ------------------------------------------------------------------ errors
static int fail(hipft_gpu *h, int code, const char *fmt, ...) {
  char msg[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(msg, sizeof msg, fmt, ap);
  va_end(ap);
  if (h) h->err = msg;
  return code;
}

#define CK(h, call)                                                                         \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return fail((h), HIPFT_ECUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,              \
                  cudaGetErrorString(e_));                                                  \
  } while (0)

#define LAUNCHED(h)                                                                         \
  do {                                                                                      \
    (h)->launches++;                                                                        \
    cudaError_t e_ = cudaPeekAtLastError();                                                 \
    if (e_ != cudaSuccess)                                                                  \
      return fail((h), HIPFT_ECUDA, "%s:%d kernel launch: %s", __FILE__, __LINE__,          \
                  cudaGetErrorString(e_));                                                  \
  } while (0)

// MIN/MAX of a scalar over the ranks sharing a run; a no-op on one process
static int allreduce(hipft_gpu *h, int op, double *v) {
  if (!h->red_cb) return HIPFT_OK;
  if (h->red_cb(h->red_user, op, v) != 0) return fail(h, HIPFT_ECOMM, "all-reduce callback failed");
  return HIPFT_OK;
}

template <typename T>
static int dalloc(hipft_gpu *h, T **p, size_t n) {
  size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
  cudaError_t e = cudaMalloc((void **)p, bytes);
  if (e != cudaSuccess) return fail(h, HIPFT_ENOMEM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
  h->allocs.push_back((void *)*p);
  h->dev_bytes += bytes;
  return HIPFT_OK;
}

template <typename T>
static int upload(hipft_gpu *h, T *d, const std::vector<T> &v) {
  CK(h, cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, h->stream));
  return HIPFT_OK;
}

#define TRY(x)                 \
  do {                         \
    int rc_ = (x);             \
    if (rc_ != HIPFT_OK) return rc_; \
  } while (0)

// ------------------------------------------------------------- set_mesh
// src/hipft.f90:6495-6653, restated on 1-based host vectors.
static int set_mesh(hipft_gpu *h, const double *tin, const double *pin) {
  const double eps = 1.e-5;
  int ntm = h->ntm, npm = h->npm, nt = h->nt, np = h->np, npm1 = h->npm1, ntm1 = h->ntm;
  auto &t = h->t, &p = h->p;
  t.assign(ntm + 1, 0.0);
  p.assign(npm + 1, 0.0);
  for (int j = 1; j <= ntm; ++j) t[j] = tin[j - 1];
  for (int k = 1; k <= npm1; ++k) p[k] = pin[k - 1];
  p[npm1 + 1] = p[2] + c_twopi;
  if (std::fabs(t[1]) > eps || std::fabs(t[ntm] - c_pi) > eps || std::fabs(p[1]) > eps ||
      std::fabs(p[npm - 1] - c_twopi) > eps)
    return fail(h, HIPFT_EINVAL, "set_mesh: the mesh does not cover the sphere (t in [0,pi], p in [0,2pi])");
  h->th.assign(nt + 1, 0); h->dth.assign(nt + 1, 0); h->dth_i.assign(nt + 1, 0);
  h->sth.assign(nt + 1, 0); h->sth_i.assign(nt + 1, 0); h->cth.assign(nt + 1, 0);
  h->dt.assign(ntm + 1, 0); h->dt_i.assign(ntm + 1, 0); h->st.assign(ntm + 1, 0);
  h->st_i.assign(ntm + 1, 0); h->ct.assign(ntm + 1, 0);
  h->ph.assign(np + 1, 0); h->dph.assign(np + 1, 0); h->dph_i.assign(np + 1, 0);
  h->dp.assign(npm + 1, 0); h->dp_i.assign(npm + 1, 0);
  auto &th = h->th, &dth = h->dth, &dt = h->dt, &ph = h->ph, &dph = h->dph, &dp = h->dp;
  for (int i = 2; i <= ntm1; ++i) {
    th[i] = 0.5 * (t[i] + t[i - 1]);
    dth[i] = t[i] - t[i - 1];
  }
  th[1] = th[2] - dth[2];
  th[nt] = th[ntm1] + dth[ntm1];
  dth[1] = dth[2];
  dth[nt] = dth[ntm1];
  for (int i = 1; i <= nt; ++i) h->dth_i[i] = 1.0 / dth[i];
  for (int i = 1; i <= ntm; ++i) {
    dt[i] = th[i + 1] - th[i];
    h->dt_i[i] = 1.0 / dt[i];
  }
  for (int i = 1; i <= ntm; ++i) h->st[i] = std::sin(t[i]);
  h->st[1] = 0.0;
  h->st[ntm] = 0.0;
  for (int i = 1; i <= ntm; ++i) h->ct[i] = std::cos(t[i]);
  h->ct[1] = 1.0;
  h->ct[ntm] = 1.0;
  for (int i = 2; i <= ntm - 1; ++i) h->st_i[i] = 1.0 / h->st[i];
  for (int i = 1; i <= nt; ++i) h->sth[i] = std::sin(std::fabs(th[i]));
  for (int i = 2; i <= ntm1; ++i) h->sth_i[i] = 1.0 / h->sth[i];
  for (int i = 1; i <= nt; ++i) h->cth[i] = std::cos(th[i]);
  for (int i = 2; i <= np; ++i) {
    ph[i] = 0.5 * (p[i] + p[i - 1]);
    dph[i] = p[i] - p[i - 1];
  }
  ph[1] = ph[npm1] - c_twopi;
  dph[1] = dph[npm1];
  for (int i = 1; i <= np; ++i) h->dph_i[i] = 1.0 / dph[i];
  for (int i = 1; i <= npm - 1; ++i) dp[i] = ph[i + 1] - ph[i];
  dp[npm] = dp[2];
  for (int i = 1; i <= npm; ++i) h->dp_i[i] = 1.0 / dp[i];
  return HIPFT_OK;
}

// load_weno grid weights (src/hipft.f90:6893-6932); 7 theta + 7 phi arrays.
static void weno_weights(const hipft_gpu *h, std::vector<double> wt[7], std::vector<double> wp[7]) {
  int nt = h->nt, np = h->np, ntm = h->ntm, npm = h->npm;
  for (int q = 0; q < 7; ++q) {
    wt[q].assign(nt + 2, 0.0);
    wp[q].assign(np + 2, 0.0);
  }
  for (int j = 1; j <= ntm; ++j) wt[6][j] = (h->P.weno_eps <= 0.0) ? h->dt[j] : h->P.weno_eps;
  for (int k = 1; k <= npm; ++k) wp[6][k] = (h->P.weno_eps <= 0.0) ? h->dp[k] : h->P.weno_eps;
  auto fill = [](std::vector<double> *w, const std::vector<double> &d, int lo, int hi) {
    for (int j = lo; j <= hi; ++j) {
      double tot = d[j - 1] + d[j] + d[j + 1];
      w[0][j] = d[j] / (d[j] + d[j + 1]);          // D_C_CP
      w[1][j] = d[j] / (d[j - 1] + d[j]);          // D_C_MC
      w[2][j] = d[j - 1] / tot;                    // D_M_T
      w[3][j] = (d[j] + d[j + 1]) / tot;           // D_CP_T
      w[4][j] = d[j + 1] / tot;                    // D_P_T
      w[5][j] = (d[j - 1] + d[j]) / tot;           // D_MC_T
    }
  };
  fill(wt, h->dt, 2, nt - 2);
  fill(wp, h->dp, 2, np - 1);
  for (int q = 0; q < 6; ++q) {
    wp[q][1] = wp[q][np - 1];
    wp[q][np] = wp[q][2];
  }
}

// Scratch buffer n (0,1,2) other than the current field.
static int scratch(const hipft_gpu *h, int n) {
  int c = 0;
  for (int b = 0; b < h->nbuf; ++b) {
    if (b == h->cur) continue;
    if (c == n) return b;
    ++c;
  }
  return -1;
}

static dim3 stage_grid(const hipft_gpu *h, int tj, int tk) {
  return dim3((unsigned)((h->ntm + tj - 1) / tj), (unsigned)((h->npm - 2 + tk - 1) / tk), (unsigned)h->nr);
}

static int ensure_part(hipft_gpu *h, size_t n) {
  if (n <= h->part_cap) return HIPFT_OK;
  if (h->d_part) {
    cudaFree(h->d_part);
    h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void *)h->d_part), h->allocs.end());
  }
  h->d_part = nullptr;
  TRY(dalloc(h, &h->d_part, n));
  h->part_cap = n;
  return HIPFT_OK;
}

static int sync_read(hipft_gpu *h, const void *dsrc, size_t bytes) {
  CK(h, cudaMemcpyAsync(h->h_pin, dsrc, bytes, cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return HIPFT_OK;
}

// ------------------------------------------------------------- kernels glue
static int ring_diffusion(hipft_gpu *h, const double *x, double *ring) {
  ProfScope ps(h, HIPFT_K_RING);
  k_ring_diffusion<<<h->nr, 256, 0, h->stream>>>(h->M, h->DC, x, ring);
  LAUNCHED(h);
  return HIPFT_OK;
}

// Diffusion ring sums of the current field, reused while the field is
// unchanged (the fused stages leave the ring of their output behind).
static int current_dring(hipft_gpu *h, const double **ring) {
  if (!h->dring_valid) {
    TRY(ring_diffusion(h, h->buf[h->cur], h->d_ringbuf[h->ring_cur]));
    h->dring_valid = true;
  }
  *ring = h->d_ringbuf[h->ring_cur];
  return HIPFT_OK;
}

constexpr int kKPT3 = 4;  // phi columns per thread of the fused single-stage kernel (two rows per thread)

// One fused RKG2/RKL2 (or Euler) stage, k_sts_stage_v3; leaves the ring sums
// of its output for the next stage.
template <int MODE>
static int sts_stage_v2(hipft_gpu *h, const double *x, const double *ykm2, const double *u0, const double *dty0,
                        double *out, double *out2, StageCoef sc) {
  const int nkb = (h->npm - 2 + kKPT3 - 1) / kKPT3;
  RingOut ro{h->d_ringbuf[1 - h->ring_cur], h->d_rpart, h->d_rcount, nkb};
  {
    ProfScope ps(h, MODE == MODE_STSK ? HIPFT_K_STS : HIPFT_K_OTHER);
    // odd ntm: keep the thread owning row ntm off lane 0 (row ntm-1 is its left neighbour)
    const int jshift = (h->ntm % 2 == 1 && ((h->ntm - 1) / 2) % 32 == 0) ? 1 : 0;
    const int nthr = (h->ntm + 2 * jshift + 1) / 2;
    dim3 grd((unsigned)((nthr + 127) / 128), (unsigned)nkb, (unsigned)h->nr);
    k_sts_stage_v3<MODE, kKPT3><<<grd, 128, 0, h->stream>>>(h->M, h->DC.dfac, x, ykm2, u0, dty0, out, out2,
                                                           h->d_ringbuf[h->ring_cur], h->bc_diff_n, h->bc_diff_s, sc,
                                                           ro, jshift);
    LAUNCHED(h);
  }
  h->ring_cur = 1 - h->ring_cur;  // the output's ring is now current
  return HIPFT_OK;
}

// HIPFT_PDL=0 turns off the programmatic (overlapping) launch of the
// two-stage kernel after the previous pair's pole-row kernel.
static bool ws_pdl() {
  static int v = -1;
  if (v < 0) {
    const char *e = std::getenv("HIPFT_PDL");
    v = (e && std::atoi(e) == 0) ? 0 : 1;
  }
  return v == 1;
}

// HIPFT_WS_TMAP=0 turns off the tensor-map tile loads of k_sts_pair_ws (one
// bulk copy per column on every tile instead).
static bool ws_tmap_enabled() {
  static int v = -1;
  if (v < 0) {
    const char *e = std::getenv("HIPFT_WS_TMAP");
    v = (e && std::atoi(e) == 0) ? 0 : 1;
  }
  return v == 1;
}

// cuTensorMapEncodeTiled from the driver, through the runtime (no libcuda link)
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 3-D f64 tensor map (dims d0 x d1 x d2, byte strides s1, s2 of dims 1, 2),
// box b0 x b1 x 1, no swizzle, zero fill outside; false if the driver refuses
// (e.g. a base address or stride that is not a multiple of 16 bytes)
static bool encode_f64_3d(CUtensorMap *m, const void *base, uint64_t d0, uint64_t d1, uint64_t d2, uint64_t s1,
                          uint64_t s2, uint32_t b0, uint32_t b1) {
  PFN_cuTensorMapEncodeTiled_v12000 fn = tmap_encoder();
  if (!fn) return false;
  cuuint64_t dims[3] = {d0, d1, d2};
  cuuint64_t strides[2] = {s1, s2};
  cuuint32_t box[3] = {b0, b1, 1};
  cuuint32_t es[3] = {1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void *>(base), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// a field buffer's map with a box of rows x cols (cached)
static bool field_map(hipft_gpu *h, const double *p, int cols, CUtensorMap *out, int rows = kWR) {
  // key: the address (user-space pointers fit 48 bits) with the box shape above it
  const uint64_t key = (uint64_t)(uintptr_t)p | ((uint64_t)(cols & 0xff) << 48) | ((uint64_t)(rows & 0xff) << 56);
  const auto it = h->ws_map_cache.find(key);
  if (it != h->ws_map_cache.end()) {
    *out = it->second;
    return true;
  }
  CUtensorMap mp;
  if (!encode_f64_3d(&mp, p, (uint64_t)h->ldt, (uint64_t)h->npm, (uint64_t)h->nr, (uint64_t)h->ldt * 8,
                     (uint64_t)h->plane * 8, (uint32_t)rows, (uint32_t)cols))
    return false;
  h->ws_map_cache.emplace(key, mp);
  *out = mp;
  return true;
}

// the tensor maps of one k_sts_pair_ws launch; on = 0 (bulk copies per
// column) when they are turned off or cannot be made
static WsMaps ws_maps(hipft_gpu *h, const double *ykm1, const double *ykm2, const double *u0, const double *dty0) {
  WsMaps tm;
  std::memset(&tm, 0, sizeof(tm));
  if (!ws_tmap_enabled() || !h->ws_rt_ok) return tm;
  if (!field_map(h, ykm1, kWK + 4, &tm.x1) || !field_map(h, ykm2, kWK + 2, &tm.y2) ||
      !field_map(h, u0, kWK + 2, &tm.u) || !field_map(h, dty0, kWK + 2, &tm.d))
    return tm;
  tm.rt = h->ws_rt_map;
  tm.on = 1;
  return tm;
}

// ------------------------------------------------------------ autotuner
// The two-stage launch has several implementations whose speed depends on
// the grid and the batch.  The persistent warp-specialised family shares one
// tile (128 theta rows x 8 phi columns), one ring-sum order and the pole
// kernel, so its members give bitwise the same values: two theta rows per
// consumer thread (PK_WS_ROWS2) at 2 or 1 CTAs per SM, the same with bulk
// stores (PK_WS_BULK), one row per thread (PK_WS_ROWS1).  On the first
// two-stage super-step of a grid size (ntm, npm, nr) on a device the library
// times each of them over a few launches on the handle's own buffers and
// keeps the fastest for the process.  HIPFT_STS_PAIR (0: one stage per
// launch, 4/5/6: the warp-specialised kinds, 7: four stages per pass on the
// interior theta blocks) fixes the choice, and HIPFT_TUNE=0 takes PK_WS_ROWS2
// at 2 CTAs per SM without timing.  The four-stage path (PK_WS_QUAD,
// sts_quad_ws.cuh) computes the same cell values and is a candidate whenever
// the grid has interior blocks.

static const char *pair_kind_name(int k) {
  switch (k) {
    case PK_SINGLE: return "single-stage";
    case PK_WS_ROWS1: return "ws-rows1";
    case PK_WS_ROWS2: return "ws-rows2";
    case PK_WS_BULK: return "ws-bulk";
    case PK_WS_QUAD: return "ws-quad (four stages per pass on interior blocks)";
  }
  return "?";
}

static std::mutex g_plan_mutex;
static std::vector<std::pair<std::array<int, 4>, PairPlan>> g_plans;  // (ntm, npm, nr, device) -> plan

static bool env_plan(PairPlan &p) {
  const char *e = std::getenv("HIPFT_STS_PAIR");
  if (e) {
    const int v = std::atoi(e);
    p.kind = (v == 0 || v == 4 || v == 6 || v == 7) ? v : PK_WS_ROWS2;
    return true;
  }
  const char *t = std::getenv("HIPFT_TUNE");
  if (t && std::atoi(t) == 0) {
    p.kind = PK_WS_ROWS2;
    return true;
  }
  return false;
}

static bool sts_pairs_enabled(const hipft_gpu *h) { return h->plan.kind != PK_SINGLE; }

static int check_wait_flag(hipft_gpu *h, const char *what);

// Two RKG2 stages per launch (stages k, k+1 of diffusion_step_sts_cd,
// src/hipft.f90:5222-5237) with the handle's plan.  overlap_prev: the launch
// before this one on the stream is the previous pair's k_pair_poles (so the
// warp-specialised kernel may start while it runs; everything else it reads
// was finished by the kernels before that one).
static int sts_pair_plan(hipft_gpu *h, const PairPlan &pl, const double *ykm1, const double *ykm2, const double *u0,
                         const double *dty0, double *out_k, double *out_k1, StageCoef ca, StageCoef cb,
                         bool overlap_prev) {
  static_assert(kWK == kPK && kWJ == kPJ, "the two-stage kernels share one tile shape");
  {
    ProfScope ps(h, HIPFT_K_STS);
    const int nkt = (h->npm - 2 + kWK - 1) / kWK;
    RingOut ro{h->d_ringbuf[1 - h->ring_cur], h->d_rpart, h->d_rcount, nkt};
    const int grid = std::min(h->ptab.ntiles, pl.ctas_per_sm * h->num_sms);
    const PairArgs pa{ca, cb, h->d_err};
    const double *rin = h->d_ringbuf[h->ring_cur];
    const WsMaps tmaps = ws_maps(h, ykm1, ykm2, u0, dty0);
    // programmatic dependent launch: may overlap the previous pair's
    // k_pair_poles (the kernel's pole tiles wait for it)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kWThreads);
    cfg.dynamicSmemBytes = kWSmem;
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = (ws_pdl() && overlap_prev) ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t le;
    // bulk stores need 16-byte aligned output columns (ldt and the plane
    // are multiples of 16 elements)
    const bool aligned = ((reinterpret_cast<uintptr_t>(out_k) | reinterpret_cast<uintptr_t>(out_k1)) & 15) == 0;
    if (pl.kind == PK_WS_BULK && aligned)
      le = cudaLaunchKernelEx(&cfg, k_sts_pair_ws<true, true>, h->M, (const double *)h->DC.dfac, ykm1, ykm2, u0,
                              dty0, out_k, out_k1, rin, h->bc_diff_n, h->bc_diff_s, pa, ro, h->ptab, tmaps);
    else if (pl.kind == PK_WS_ROWS1)
      le = cudaLaunchKernelEx(&cfg, k_sts_pair_ws<false>, h->M, (const double *)h->DC.dfac, ykm1, ykm2, u0, dty0,
                              out_k, out_k1, rin, h->bc_diff_n, h->bc_diff_s, pa, ro, h->ptab, tmaps);
    else
      le = cudaLaunchKernelEx(&cfg, k_sts_pair_ws<true>, h->M, (const double *)h->DC.dfac, ykm1, ykm2, u0, dty0,
                              out_k, out_k1, rin, h->bc_diff_n, h->bc_diff_s, pa, ro, h->ptab, tmaps);
    if (le != cudaSuccess) return fail(h, HIPFT_ECUDA, "k_sts_pair_ws launch: %s", cudaGetErrorString(le));
    LAUNCHED(h);
    dim3 pg((unsigned)h->nr, (unsigned)h->pole_nch);
    k_pair_poles<<<pg, kPoleThreads, 0, h->stream>>>(h->M, h->DC.dfac, ykm1, ykm2, u0, dty0, out_k1, rin,
                                                     h->bc_diff_n, h->bc_diff_s, pa, ro, h->pole);
    LAUNCHED(h);
  }
  h->ring_cur = 1 - h->ring_cur;
  return HIPFT_OK;
}

static int sts_pair(hipft_gpu *h, const double *ykm1, const double *ykm2, const double *u0, const double *dty0,
                    double *out_k, double *out_k1, StageCoef ca, StageCoef cb, bool overlap_prev) {
  PairPlan pl = h->plan;
  if (pl.kind == PK_WS_QUAD) pl.kind = PK_WS_ROWS2;  // lone pairs of a four-stage plan
  return sts_pair_plan(h, pl, ykm1, ykm2, u0, dty0, out_k, out_k1, ca, cb, overlap_prev);
}

// ------------------------------------------------ four stages per pass
// The interior theta blocks rb_lo..rb_hi (rows j0-3 .. j0+130 of a block
// inside 2..ntm-1, see sts_quad_ws.cuh); false when there are none.
static bool quad_eligible(const hipft_gpu *h) {
  if (h->DC.grid || !h->ptab.row || h->ntm < kQJ + 132) return false;
  const int rb_hi = (h->ntm - 132) / kQJ;  // largest rb with 128 rb + 132 <= ntm
  return h->ptab.nb - rb_hi <= 6;           // pole blocks: 0 and rb_hi+1 .. nb-1
}

// Tables, tensor map and the two extra fields of the four-stage path.
static int quad_setup(hipft_gpu *h) {
  if (h->d_qcol) return HIPFT_OK;
  h->q_rb_lo = 1;
  h->q_rb_hi = (h->ntm - 132) / kQJ;
  while (h->nbuf < kNBuf) {
    TRY(dalloc(h, &h->buf[h->nbuf], h->fieldn));
    CK(h, cudaMemsetAsync(h->buf[h->nbuf], 0, h->fieldn * sizeof(double), h->stream));
    ++h->nbuf;
  }
  h->q_nkt = (h->npm - 2 + kQK - 1) / kQK;
  h->q_LC = h->q_nkt * kQK + 24;
  TRY(dalloc(h, &h->d_qcol, (size_t)h->nr * h->q_LC * 2));
  k_quad_coltab<<<2 * h->num_sms, 256, 0, h->stream>>>(h->M, h->DC.dfac, h->q_LC, h->d_qcol);
  LAUNCHED(h);
  h->q_rt_ok = encode_f64_3d(&h->q_rt_map, h->ptab.row, (uint64_t)h->ptab.LR, 3, (uint64_t)h->nr,
                             (uint64_t)h->ptab.LR * 8, (uint64_t)h->ptab.LR * 24, kQR, 3);
  CK(h, cudaFuncSetAttribute(k_sts_quad_ws<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kQSmem));
  CK(h, cudaFuncSetAttribute(k_sts_quad_ws<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kQSmem));
  return HIPFT_OK;
}

// The pole blocks (every block outside rb_lo..rb_hi) of `nreal` realizations
// for the two-stage launches of the four-stage path.
static PairTables quad_pole_tables(const hipft_gpu *h, int nreal) {
  PairTables pt = h->ptab;
  pt.nsel = 0;
  for (int rb = 0; rb < pt.nb; ++rb)
    if (rb < h->q_rb_lo || rb > h->q_rb_hi) pt.sel[pt.nsel++] = rb;
  pt.ntiles = pt.nsel * pt.nkt * nreal;
  return pt;
}

// Two-stage launch (k_sts_pair_ws, two rows per consumer) plus k_pair_poles
// over the tiles of `pt`; rlist/rc (may be null): the realizations of a
// ragged batch and their coefficients.  flip: the launch's output ring sums
// become current (a launch that shares its input ring with a following one
// leaves that to the last of them).
static int ws_pair_launch(hipft_gpu *h, const PairTables &pt, int cps, const double *ykm1, const double *ykm2,
                          const double *u0, const double *dty0, double *out_k, double *out_k1, StageCoef ca,
                          StageCoef cb, bool overlap_prev, const int *rlist = nullptr, int nreal = 0,
                          const StageCoef *rc = nullptr, bool flip = true) {
  const int nkt = (h->npm - 2 + kWK - 1) / kWK;
  RingOut ro{h->d_ringbuf[1 - h->ring_cur], h->d_rpart, h->d_rcount, nkt};
  const int grid = std::min(pt.ntiles, cps * h->num_sms);
  PairArgs pa{ca, cb, h->d_err, rlist, rc};
  const double *rin = h->d_ringbuf[h->ring_cur];
  const WsMaps tmaps = ws_maps(h, ykm1, ykm2, u0, dty0);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(kWThreads);
  cfg.dynamicSmemBytes = kWSmem;
  cfg.stream = h->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = (ws_pdl() && overlap_prev) ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaError_t le = rlist ? cudaLaunchKernelEx(&cfg, k_sts_pair_ws<true, false, true>, h->M, (const double *)h->DC.dfac,
                                              ykm1, ykm2, u0, dty0, out_k, out_k1, rin, h->bc_diff_n, h->bc_diff_s,
                                              pa, ro, pt, tmaps)
                         : cudaLaunchKernelEx(&cfg, k_sts_pair_ws<true>, h->M, (const double *)h->DC.dfac, ykm1, ykm2,
                                              u0, dty0, out_k, out_k1, rin, h->bc_diff_n, h->bc_diff_s, pa, ro, pt,
                                              tmaps);
  if (le != cudaSuccess) return fail(h, HIPFT_ECUDA, "k_sts_pair_ws launch: %s", cudaGetErrorString(le));
  LAUNCHED(h);
  dim3 pg((unsigned)(rlist ? nreal : h->nr), (unsigned)h->pole_nch);
  k_pair_poles<<<pg, kPoleThreads, 0, h->stream>>>(h->M, h->DC.dfac, ykm1, ykm2, u0, dty0, out_k1, rin, h->bc_diff_n,
                                                   h->bc_diff_s, pa, ro, h->pole);
  LAUNCHED(h);
  if (flip) h->ring_cur = 1 - h->ring_cur;
  return HIPFT_OK;
}

// The four-stage launch over the interior blocks of all realizations, or of
// the n realizations of rlist with coefficients rcA (stages k, k+1) and rcB
// (k+2, k+3).  It reads nothing the pole blocks' first two-stage launch
// writes, so it may start while that launch's pole kernel runs.
static int quad_launch(hipft_gpu *h, const double *ykm1, const double *ykm2, const double *u0, const double *dty0,
                       double *ok, double *ok1, double *ok2, double *ok3, const StageCoef c[4],
                       const int *rlist = nullptr, int n = 0, const StageCoef *rcA = nullptr,
                       const StageCoef *rcB = nullptr) {
  QuadArgs qa{};
  for (int q = 0; q < 4; ++q) qa.c[q] = c[q];
  qa.err = h->d_err;
  qa.rb_lo = h->q_rb_lo;
  qa.nbi = h->q_rb_hi - h->q_rb_lo + 1;
  qa.nkt = h->q_nkt;
  qa.ntiles = qa.nbi * qa.nkt * (rlist ? n : h->nr);
  qa.edge_lo = (h->q_rb_lo > 0) ? h->q_rb_lo : -1;
  qa.edge_hi = (h->q_rb_hi < h->ptab.nb - 1) ? h->q_rb_hi : -1;
  qa.col = h->d_qcol;
  qa.LC = h->q_LC;
  qa.rlist = rlist;
  qa.rcA = rcA;
  qa.rcB = rcB;
  QuadMaps qm;
  std::memset(&qm, 0, sizeof(qm));
  if (ws_tmap_enabled() && h->q_rt_ok && field_map(h, ykm1, kQX, &qm.x1, kQR) && field_map(h, ykm2, kQI, &qm.y2, kQR) &&
      field_map(h, u0, kQI, &qm.u, kQR) && field_map(h, dty0, kQI, &qm.d, kQR)) {
    qm.rt = h->q_rt_map;
    qm.on = 1;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)std::min(qa.ntiles, h->num_sms));  // one CTA (two tile buffers) per SM
  cfg.blockDim = dim3(kQThreads);
  cfg.dynamicSmemBytes = kQSmem;
  cfg.stream = h->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = ws_pdl() ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  PairTables pt = h->ptab;
  cudaError_t le = rlist ? cudaLaunchKernelEx(&cfg, k_sts_quad_ws<true>, h->M, ykm1, ykm2, u0, dty0, ok, ok1, ok2,
                                              ok3, qa, pt, qm)
                         : cudaLaunchKernelEx(&cfg, k_sts_quad_ws<false>, h->M, ykm1, ykm2, u0, dty0, ok, ok1, ok2,
                                              ok3, qa, pt, qm);
  if (le != cudaSuccess) return fail(h, HIPFT_ECUDA, "k_sts_quad_ws launch: %s", cudaGetErrorString(le));
  LAUNCHED(h);
  return HIPFT_OK;
}

// Stages k..k+3: the pole blocks by two two-stage launches, the interior
// blocks by one four-stage launch between them.  Outputs ok..ok3 hold
// Y_k..Y_{k+3}; Y_k and Y_{k+1} only on the pole blocks and the interior
// blocks' edge rows.
static int quad_pass(hipft_gpu *h, const double *ykm1, const double *ykm2, const double *u0, const double *dty0,
                     double *ok, double *ok1, double *ok2, double *ok3, const StageCoef c[4], bool overlap_prev) {
  const int cps = h->plan.ctas_per_sm;
  const PairTables pp = quad_pole_tables(h, h->nr);
  ProfScope ps(h, HIPFT_K_STS);
  TRY(ws_pair_launch(h, pp, cps, ykm1, ykm2, u0, dty0, ok, ok1, c[0], c[1], overlap_prev));
  TRY(quad_launch(h, ykm1, ykm2, u0, dty0, ok, ok1, ok2, ok3, c));
  TRY(ws_pair_launch(h, pp, cps, ok1, ok, u0, dty0, ok2, ok3, c[2], c[3], false));
  return HIPFT_OK;
}

// Chooses the handle's two-stage plan (see the autotuner above) before the
// first super-step.  Timing runs on four buffers other than the current
// field, with the current field as an input, and leaves the field untouched;
// the ring sums it disturbs are recomputed afterwards.
static int ensure_pair_plan(hipft_gpu *h) {
  if (h->plan.kind >= 0) return HIPFT_OK;
  PairPlan p;
  if (env_plan(p)) {
    if (p.kind == PK_WS_QUAD) {
      if (quad_eligible(h)) TRY(quad_setup(h));
      else p.kind = PK_WS_ROWS2;
    }
    h->plan = p;
    return HIPFT_OK;
  }
  const std::array<int, 4> key{h->ntm, h->npm, h->nr, h->dev};
  {
    std::lock_guard<std::mutex> lk(g_plan_mutex);
    for (const auto &e : g_plans)
      if (e.first == key) {
        h->plan = e.second;
        return HIPFT_OK;
      }
  }
  std::vector<PairPlan> cands;
  for (int c : {2, 1}) {
    PairPlan q;
    q.kind = PK_WS_ROWS2;
    q.ctas_per_sm = c;
    cands.push_back(q);
  }
  for (int k : {PK_WS_BULK, PK_WS_ROWS1}) {
    PairPlan q;
    q.kind = k;
    cands.push_back(q);
  }
  if (quad_eligible(h)) {
    TRY(quad_setup(h));
    PairPlan q;
    q.kind = PK_WS_QUAD;
    cands.push_back(q);
  }
  const bool prof = h->profiling;
  h->profiling = false;
  const double *x = h->buf[h->cur];
  double *bufs[6] = {};
  for (int q = 0; q < 6 && q < h->nbuf - 1; ++q) bufs[q] = h->buf[scratch(h, q)];
  const StageCoef ca{0.5, -0.1, 0.6, 1e-3, 0.0}, cb{0.5, -0.1, 0.6, 1e-3, 0.0};
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CK(h, cudaEventCreate(&e0));
  CK(h, cudaEventCreate(&e1));
  int best = 0;
  const int reps = 3;
  const StageCoef cq[4] = {ca, cb, ca, cb};
  for (size_t c = 0; c < cands.size(); ++c) {
    // time per two stages: a four-stage pass counts as two launch pairs
    const bool quad = cands[c].kind == PK_WS_QUAD;
    const PairPlan saved = h->plan;
    h->plan = cands[c];
    auto once = [&](bool ov) -> int {
      if (quad) return quad_pass(h, x, bufs[0], x, bufs[1], bufs[2], bufs[3], bufs[4], bufs[5], cq, ov);
      return sts_pair_plan(h, cands[c], x, bufs[0], x, bufs[1], bufs[2], bufs[3], ca, cb, ov);
    };
    int rc = once(false);  // warm-up
    CK(h, cudaEventRecord(e0, h->stream));
    for (int r = 0; r < reps && rc == HIPFT_OK; ++r) rc = once(r > 0);
    h->plan = saved;
    TRY(rc);
    CK(h, cudaEventRecord(e1, h->stream));
    CK(h, cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(h, cudaEventElapsedTime(&ms, e0, e1));
    cands[c].ms = ms / reps / (quad ? 2.0 : 1.0);
    if (cands[c].ms < cands[best].ms) best = (int)c;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  h->profiling = prof;
  TRY(check_wait_flag(h, "pair autotuner: a bounded wait for staged tiles gave up"));
  h->plan = cands[best];
  h->plan.candidates = (int)cands.size();
  h->dring_valid = false;
  std::lock_guard<std::mutex> lk(g_plan_mutex);
  g_plans.push_back({key, h->plan});
  return HIPFT_OK;
}

template <int MODE>
static int diffusion_stage(hipft_gpu *h, const double *x, const double *ykm2, const double *u0, const double *dty0,
                           double *out, double *out2, const double *ring, StageCoef sc,
                           unsigned long long *absmax) {
  dim3 blk(32, 8);
  ProfScope ps(h, MODE == MODE_STSK ? HIPFT_K_STS : HIPFT_K_OTHER);
  k_diffusion_stage<MODE><<<stage_grid(h, 32, 8), blk, 0, h->stream>>>(h->M, h->DC, x, ykm2, u0, dty0, out, out2,
                                                                       ring, h->bc_diff_n, h->bc_diff_s, sc,
                                                                       absmax);
  LAUNCHED(h);
  return HIPFT_OK;
}

// HIPFT_ADV_KERNEL selects the WENO3 stage kernel: "tile" the tile kernel
// (k_advection_stage<32, 8, true>), "march" the phi-marching kernel on any
// grid; unset, the library decides by grid size.  Both give bitwise the same
// fields; the tests compare the two.
static int adv_kernel_env() {
  static int v = -1;
  if (v < 0) {
    const char *e = std::getenv("HIPFT_ADV_KERNEL");
    v = (e && std::strcmp(e, "tile") == 0) ? 1 : (e && std::strcmp(e, "march") == 0) ? 2 : 0;
  }
  return v;
}

// One explicit advection stage over nz realization slots (rlist maps slot z
// to a realization when non-null; rdt scales each realization's step).
// WENO3 stages march along phi (k_adv_weno_march) when the grid, in chunks of
// 64 or 32 phi columns, holds 1.5 waves of warps (16 resident per SM): on one
// 1024 x 2048 realization the tile kernel is faster (0.090 against 0.102 ms),
// on 64 of them the marching kernel (3.97 against 5.57 ms).  Upwind stages
// take the tile kernel.
static void launch_adv_stage(const hipft_gpu *h, const Mesh &M, cudaStream_t s, unsigned nz, const double *x,
                             const double *f0, double *out, AdvCombine cb, const int *rlist, const double *rdt) {
  if (h->adv_space == 2 && adv_kernel_env() != 1) {
    const int64_t groups = (h->ntm - 1) / 31 + 1, fill = 24LL * h->num_sms;
    auto warps = [&](int ncol) { return groups * ((h->npm - 2 + ncol - 1) / ncol) * (int64_t)nz; };
    int ncol = kAdvColsMax;
    while (ncol > 8 && warps(ncol) < fill) ncol /= 2;
    if (ncol >= 32 || adv_kernel_env() == 2) {
      const dim3 blk(32, kAdvWarps);
      const dim3 grd((unsigned)((groups + kAdvWarps - 1) / kAdvWarps), (unsigned)((h->npm - 2 + ncol - 1) / ncol),
                     nz);
      auto kern = h->FL.flow2d ? (cb.mode == 0 ? k_adv_weno_march<true, 0> : k_adv_weno_march<true, 1>)
                               : (cb.mode == 0 ? k_adv_weno_march<false, 0> : k_adv_weno_march<false, 1>);
      kern<<<grd, blk, 0, s>>>(M, h->FL, h->W, x, f0, out, h->d_ring, h->bc_flow_n, h->bc_flow_s, cb, rlist, rdt,
                               ncol);
      return;
    }
  }
  const dim3 blk(33, 9);  // (TJ+1) x (TK+1) threads for a 32 x 8 tile
  const dim3 grd((unsigned)((h->ntm + 31) / 32), (unsigned)((h->npm - 2 + 7) / 8), nz);
  if (h->adv_space == 2)
    k_advection_stage<32, 8, true><<<grd, blk, 0, s>>>(M, h->FL, h->W, x, f0, out, h->d_ring, h->bc_flow_n,
                                                        h->bc_flow_s, cb, rlist, rdt);
  else
    k_advection_stage<32, 8, false><<<grd, blk, 0, s>>>(M, h->FL, h->W, x, f0, out, h->d_ring, h->bc_flow_n,
                                                         h->bc_flow_s, cb, rlist, rdt);
}

static int advection_stage(hipft_gpu *h, const double *x, const double *f0, double *out, AdvCombine cb) {
  {
    ProfScope ps(h, HIPFT_K_RING);
    k_ring_advection<<<h->nr, 256, 0, h->stream>>>(h->M, h->FL, x, h->d_ring);
    LAUNCHED(h);
  }
  ProfScope ps(h, HIPFT_K_ADV);
  launch_adv_stage(h, h->M, h->stream, (unsigned)h->nr, x, f0, out, cb, nullptr, nullptr);
  LAUNCHED(h);
  h->cell_updates += (int64_t)h->ntm * (h->npm - 2) * h->nr;
  return HIPFT_OK;
}

// ---------------------------------------------------------------- create
extern "C" int hipft_gpu_create(const hipft_grid *g, const hipft_params *prm, hipft_gpu **out) {
  if (!g || !prm || !out || !g->t || !g->p) return HIPFT_EINVAL;
  *out = nullptr;
  if (g->ntm < 4 || g->npm1 < 5 || g->nr < 1) return HIPFT_EINVAL;
  if (prm->advance_diffusion && !prm->diffusion_coef_constants) return HIPFT_EINVAL;
  if (prm->advance_flow && (prm->flow_num_method < 1 || prm->flow_num_method > 4)) return HIPFT_EINVAL;
  if (prm->advance_diffusion && (prm->diffusion_num_method < 1 || prm->diffusion_num_method > 3))
    return HIPFT_EINVAL;
  hipft_gpu *h = new hipft_gpu();
  h->dev = g->device;
  h->P = *prm;
  h->P.diffusion_coef_constants = nullptr;
  h->ntm = g->ntm;
  h->npm1 = g->npm1;
  h->npm = g->npm1 + 1;
  h->nt = g->ntm + 1;
  h->np = g->npm1 + 1;
  h->nr = g->nr;
  h->ldt = round_up(h->ntm, 16);
  h->ldv = round_up(h->nt, 16);
  h->plane = (int64_t)h->ldt * h->npm;
  h->fieldn = (size_t)h->plane * h->nr;
  // the per-realization constants also set validation run 1's decay rate
  // (src/hipft.f90:3156-3159), diffusion or not
  if (prm->diffusion_coef_constants)
    h->Dc.assign(prm->diffusion_coef_constants, prm->diffusion_coef_constants + g->nr);
  int fm = prm->flow_num_method;
  h->adv_time = (fm == 1) ? 1 : (fm == 4 ? 3 : 2);
  h->adv_space = (fm <= 2) ? 1 : 2;
  h->subcycles_state = prm->diffusion_subcycles;
  auto bail = [&](int rc) {
    std::string e = h->err;
    hipft_gpu_destroy(h);
    (void)e;
    return rc;
  };
  cudaError_t ce = cudaSetDevice(h->dev);
  if (ce != cudaSuccess) {
    fail(h, HIPFT_ECUDA, "cudaSetDevice(%d): %s", h->dev, cudaGetErrorString(ce));
    return bail(HIPFT_ECUDA);
  }
  ce = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (ce != cudaSuccess) return bail(HIPFT_ECUDA);
  h->own_stream = true;
  int rc = set_mesh(h, g->t, g->p);
  if (rc) return bail(rc);
  int ntm = h->ntm, npm = h->npm, nt = h->nt, np = h->np, nr = h->nr;

  // 1-D mesh arrays on the device (one allocation, 1-based slices)
  std::vector<const std::vector<double> *> arrs = {&h->dt_i, &h->dth_i, &h->dp_i, &h->dph_i, &h->st_i,
                                                   &h->sth,  &h->dp,    &h->dth,  &h->dph};
  size_t tot = 0;
  for (auto *a : arrs) tot += a->size();
  double *dm = nullptr;
  if ((rc = dalloc(h, &dm, tot))) return bail(rc);
  std::vector<double> packed;
  packed.reserve(tot);
  std::vector<size_t> offs;
  for (auto *a : arrs) {
    offs.push_back(packed.size());
    packed.insert(packed.end(), a->begin(), a->end());
  }
  if ((rc = upload(h, dm, packed))) return bail(rc);
  h->M.ntm = ntm; h->M.npm = npm; h->M.nt = nt; h->M.np = np; h->M.nr = nr; h->M.ldt = h->ldt;
  h->M.plane = h->plane;
  h->M.dt_i = dm + offs[0]; h->M.dth_i = dm + offs[1]; h->M.dp_i = dm + offs[2]; h->M.dph_i = dm + offs[3];
  h->M.st_i = dm + offs[4]; h->M.sth = dm + offs[5]; h->M.dp = dm + offs[6]; h->M.dth = dm + offs[7];
  h->M.dph = dm + offs[8];

  // fields (the four-stage path adds two more when it is first used)
  for (int b = 0; b < h->nbuf; ++b) {
    if ((rc = dalloc(h, &h->buf[b], h->fieldn))) return bail(rc);
    if (cudaMemsetAsync(h->buf[b], 0, h->fieldn * sizeof(double), h->stream) != cudaSuccess) return bail(HIPFT_ECUDA);
  }
  if ((rc = dalloc(h, &h->d_ring, 2 * (size_t)nr))) return bail(rc);
  h->nkb = (npm - 2 + kKPT3 - 1) / kKPT3;  // partial slots for the smaller phi block
  if ((rc = dalloc(h, &h->d_ringbuf[0], 2 * (size_t)nr))) return bail(rc);
  if ((rc = dalloc(h, &h->d_ringbuf[1], 2 * (size_t)nr))) return bail(rc);
  if ((rc = dalloc(h, &h->d_rpart, 2 * (size_t)nr * h->nkb))) return bail(rc);
  if ((rc = dalloc(h, &h->d_rcount, (size_t)nr))) return bail(rc);
  if ((rc = dalloc(h, &h->d_err, 1))) return bail(rc);
  if (cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream) != cudaSuccess) return bail(HIPFT_ECUDA);
  if (cudaFuncSetAttribute(k_sts_pair_ws<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWSmem) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_sts_pair_ws<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWSmem) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_sts_pair_ws<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kWSmem) !=
          cudaSuccess ||
      cudaFuncSetAttribute(k_sts_pair_ws<true, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kWSmem) != cudaSuccess)
    return bail(fail(h, HIPFT_ECUDA, "cannot reserve shared memory for the two-stage kernels"));
  if (cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->dev) != cudaSuccess || h->num_sms < 1)
    h->num_sms = 148;
  if (cudaMemsetAsync(h->d_rcount, 0, sizeof(unsigned int) * nr, h->stream) != cudaSuccess) return bail(HIPFT_ECUDA);
  if ((rc = dalloc(h, &h->d_bits, 4))) return bail(rc);
  if (cudaMallocHost((void **)&h->h_pin, sizeof(double) * std::max<size_t>(64, (size_t)nr * kNPart)) !=
      cudaSuccess)
    return bail(fail(h, HIPFT_ENOMEM, "cudaMallocHost failed"));

  // diffusion: D constants, Gershgorin dt (load_diffusion, src/hipft.f90:6655-6844)
  std::vector<double> dfac(nr + 1, 0.0);
  if (prm->advance_diffusion)
    for (int i = 1; i <= nr; ++i)
      dfac[i] = prm->diffusion_coef_grid ? h->Dc[i - 1] : prm->diffusion_coef_factor * h->Dc[i - 1];
  double *d_dfac = nullptr;
  if ((rc = dalloc(h, &d_dfac, nr + 1))) return bail(rc);
  if ((rc = upload(h, d_dfac, dfac))) return bail(rc);
  h->DC.dfac = d_dfac;
  h->DC.factor = prm->diffusion_coef_factor;
  h->DC.grid = prm->diffusion_coef_grid;
  if (prm->advance_diffusion && !prm->diffusion_coef_grid) {
    PairTables &pt = h->ptab;
    pt.nb = (ntm + kWJ - 1) / kWJ;
    pt.nkt = (npm - 2 + kWK - 1) / kWK;
    pt.ntiles = pt.nb * pt.nkt * nr;
    pt.LR = pt.nb * kWJ + 4;
    pt.LC = pt.nkt * kWK + 4;
    double *tab = nullptr;
    const size_t nrow = (size_t)nr * pt.LR * 3, ncol = (size_t)nr * pt.LC * 2;
    if ((rc = dalloc(h, &tab, nrow + ncol))) return bail(rc);
    pt.row = tab;
    pt.col = tab + nrow;
    h->ws_rt_ok = encode_f64_3d(&h->ws_rt_map, pt.row, (uint64_t)pt.LR, 3, (uint64_t)nr, (uint64_t)pt.LR * 8,
                                (uint64_t)pt.LR * 24, kWR, 3);
    k_pair_tables<<<2 * h->num_sms, 256, 0, h->stream>>>(h->M, d_dfac, pt.LR, pt.LC, tab, tab + nrow);
    h->launches++;
    if (cudaPeekAtLastError() != cudaSuccess) return bail(fail(h, HIPFT_ECUDA, "k_pair_tables launch failed"));
    h->pole_nch = (npm + kPoleThreads - 1) / kPoleThreads;
    if ((rc = dalloc(h, &h->pole.part, (size_t)nr * h->pole_nch * 2))) return bail(rc);
    if ((rc = dalloc(h, &h->pole.count, (size_t)nr))) return bail(rc);
    if (cudaMemsetAsync(h->pole.count, 0, sizeof(unsigned int) * nr, h->stream) != cudaSuccess)
      return bail(HIPFT_ECUDA);
  }
  h->bc_diff_n = c_pi_i * h->dth_i[2] * h->dth_i[2];
  h->bc_diff_s = c_pi_i * h->dth_i[nt - 1] * h->dth_i[nt - 1];
  h->auto_sc = (prm->diffusion_subcycles == 0);
  if (prm->advance_diffusion) {
    if (cudaMemsetAsync(h->d_bits, 0, sizeof(unsigned long long), h->stream) != cudaSuccess) return bail(HIPFT_ECUDA);
    dim3 blk(32, 8);
    dim3 grd((unsigned)((ntm - 2 + 31) / 32), (unsigned)((npm - 2 + 7) / 8), (unsigned)nr);
    k_gershgorin<<<grd, blk, 0, h->stream>>>(h->M, h->DC, h->d_bits);
    h->launches++;
    if (cudaPeekAtLastError() != cudaSuccess) return bail(fail(h, HIPFT_ECUDA, "k_gershgorin launch failed"));
    if ((rc = sync_read(h, h->d_bits, sizeof(unsigned long long)))) return bail(rc);
    unsigned long long bits;
    std::memcpy(&bits, h->h_pin, 8);
    double max_eig;
    std::memcpy(&max_eig, &bits, 8);
    h->dt_euler = c_safety * (2.0 / max_eig);
  }

  // flows and WENO (load_flows src/hipft.f90:2535-2564, load_weno 6846)
  h->bc_flow_n = 2.0 * h->dth_i[2] * c_pi_i;
  h->bc_flow_s = 2.0 * h->dth_i[nt - 1] * c_pi_i;
  if (prm->advance_flow) {
    std::vector<double> wt[7], wp[7];
    weno_weights(h, wt, wp);
    std::vector<double> pk;
    std::vector<size_t> wo;
    for (int q = 0; q < 7; ++q) { wo.push_back(pk.size()); pk.insert(pk.end(), wt[q].begin(), wt[q].end()); }
    for (int q = 0; q < 7; ++q) { wo.push_back(pk.size()); pk.insert(pk.end(), wp[q].begin(), wp[q].end()); }
    // phi-face rows of the marching advection stage (Weno::ptab): faces
    // 2..npm, face npm with face 2's weights (src/hipft.f90:7882)
    const size_t tab0 = (pk.size() + 1) & ~(size_t)1;  // 16-byte aligned rows
    pk.resize(tab0 + (size_t)(npm - 1) * kPhiTab, 0.0);
    for (int kf = 2; kf <= npm; ++kf) {
      const int kw = (kf >= npm) ? 2 : kf;
      double *row = pk.data() + tab0 + (size_t)(kf - 2) * kPhiTab;
      const double v[10] = {wp[1][kw - 1], wp[1][kw], wp[0][kw - 1], wp[0][kw], wp[4][kw - 1],
                            wp[5][kw - 1], wp[2][kw], wp[3][kw],     wp[6][kw - 1], wp[6][kw]};
      for (int q = 0; q < 10; ++q) row[q] = v[q];
      row[10] = weno_consts_ok(v[4], v[5], v[6], v[7], v[8], v[9]) ? 1.0 : 0.0;
      row[11] = (kf <= npm - 1) ? h->dp_i[kf] : 0.0;
    }
    double *dw = nullptr;
    if ((rc = dalloc(h, &dw, pk.size()))) return bail(rc);
    if ((rc = upload(h, dw, pk))) return bail(rc);
    h->W.cpt = dw + wo[0]; h->W.mct = dw + wo[1]; h->W.mt = dw + wo[2]; h->W.cptt = dw + wo[3];
    h->W.pt = dw + wo[4]; h->W.mctt = dw + wo[5]; h->W.epst = dw + wo[6];
    h->W.cpp = dw + wo[7]; h->W.mcp = dw + wo[8]; h->W.mp = dw + wo[9]; h->W.cptp = dw + wo[10];
    h->W.pp = dw + wo[11]; h->W.mctp = dw + wo[12]; h->W.epsp = dw + wo[13];
    h->W.ptab = dw + tab0;
    if ((rc = dalloc(h, &h->d_vt1, (size_t)nr * (nt + 1)))) return bail(rc);
    if ((rc = dalloc(h, &h->d_vp1, (size_t)nr * (ntm + 1)))) return bail(rc);
    if ((rc = dalloc(h, &h->d_at1, (size_t)nr * (ntm + 1)))) return bail(rc);
    if ((rc = dalloc(h, &h->d_ap1, (size_t)nr * (ntm + 1)))) return bail(rc);
    h->FL.vt1 = h->d_vt1; h->FL.vp1 = h->d_vp1; h->FL.at1 = h->d_at1; h->FL.ap1 = h->d_ap1;
    h->FL.ldv = h->ldv;
    h->FL.vplane = (int64_t)h->ldv * npm;
    h->FL.upwind = prm->upwind;
    // zero flow until set_flow
    std::vector<double> z1((size_t)nr * (nt + 1), 0.0), z2((size_t)nr * (ntm + 1), 0.0);
    if ((rc = upload(h, h->d_vt1, z1)) || (rc = upload(h, h->d_vp1, z2)) || (rc = upload(h, h->d_at1, z2)) ||
        (rc = upload(h, h->d_ap1, z2)))
      return bail(rc);
  }

  // analysis weights (src/hipft.f90:3230-3257; get_flux 8712-8732)
  {
    std::vector<double> w(6 * (size_t)(std::max(ntm, npm) + 1), 0.0);
    size_t L = (size_t)std::max(ntm, npm) + 1;
    double *da_t = &w[0], *sn_t = &w[L], *cs_t = &w[2 * L], *da_p = &w[3 * L], *cs_p = &w[4 * L], *sn_p = &w[5 * L];
    for (int j = 1; j <= ntm; ++j) {
      double tav, sn, cs, d;
      if (j == 1) {
        tav = 0.5 * (h->t[1] + h->t[2]);
        sn = std::sin(tav); cs = std::cos(tav); d = h->dth[2];
        da_t[j] = 0.25 * sn * d;
      } else if (j == ntm) {
        tav = 0.5 * (h->t[ntm] + h->t[ntm - 1]);
        sn = std::sin(tav); cs = std::cos(tav); d = h->dth[ntm];
        da_t[j] = 0.25 * sn * d;
      } else {
        sn = std::sin(h->t[j]); cs = std::cos(h->t[j]); d = h->dt[j];
        da_t[j] = sn * d;
      }
      sn_t[j] = sn;
      cs_t[j] = cs;
    }
    for (int k = 1; k <= npm - 1; ++k) {
      if (k == 1) da_p[k] = 0.5 * h->dph[1];
      else if (k == npm - 1) da_p[k] = 0.5 * h->dph[npm - 1];
      else da_p[k] = h->dp[k];
      cs_p[k] = std::cos(h->p[k]);
      sn_p[k] = std::sin(h->p[k]);
    }
    h->da_t.assign(da_t, da_t + ntm + 1);
    h->da_p.assign(da_p, da_p + npm);
    if ((rc = dalloc(h, &h->d_anw, w.size()))) return bail(rc);
    if ((rc = upload(h, h->d_anw, w))) return bail(rc);
    std::vector<unsigned char> masks(2 * (size_t)(ntm + 1), 0);
    for (int j = 1; j <= ntm; ++j) {
      masks[j] = (h->t[j] <= prm->pole_flux_lat_limit * c_d2r) ? 1 : 0;
      masks[ntm + 1 + j] = (h->t[j] >= c_pi - prm->pole_flux_lat_limit * c_d2r) ? 1 : 0;
    }
    if ((rc = dalloc(h, &h->d_masks, masks.size()))) return bail(rc);
    if (cudaMemcpyAsync(h->d_masks, masks.data(), masks.size(), cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
      return bail(HIPFT_ECUDA);
    if ((rc = dalloc(h, &h->d_vscale, nr + 1))) return bail(rc);
  }
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return bail(fail(h, HIPFT_ECUDA, "create: sync failed"));
  *out = h;
  return HIPFT_OK;
}

extern "C" int hipft_gpu_destroy(hipft_gpu *h) {
  if (!h) return HIPFT_OK;
  cudaSetDevice(h->dev);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (auto &v : h->ev_pending)
    for (auto &pr : v) {
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
  for (auto e : h->ev_pool) cudaEventDestroy(e);
  graph_release(h);
  for (auto s : h->g_side)
    if (s) cudaStreamDestroy(s);
  for (void *p : h->allocs) cudaFree(p);
  if (h->h_pin) cudaFreeHost(h->h_pin);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return HIPFT_OK;
}

extern "C" int hipft_gpu_last_error(const hipft_gpu *h, char *buf, size_t len) {
  if (!buf || !len) return HIPFT_EINVAL;
  const char *m = h ? h->err.c_str() : "no handle";
  std::snprintf(buf, len, "%s", m);
  return HIPFT_OK;
}

extern "C" const char *hipft_gpu_version(void) { return "hipft_b200 0.1.0 (sm_100a, fp64)"; }

// ------------------------------------------------------------- field I/O
extern "C" int hipft_gpu_set_field(hipft_gpu *h, const double *f) {
  if (!h || !f) return HIPFT_EINVAL;
  CK(h, cudaSetDevice(h->dev));
  CK(h, cudaMemcpy2DAsync(h->buf[h->cur], (size_t)h->ldt * sizeof(double), f, (size_t)h->ntm * sizeof(double),
                          (size_t)h->ntm * sizeof(double), (size_t)h->npm * h->nr, cudaMemcpyHostToDevice,
                          h->stream));
  h->field_set = true;
  h->dring_valid = false;
  return HIPFT_OK;
}

extern "C" int hipft_gpu_get_field(hipft_gpu *h, double *f) {
  if (!h || !f) return HIPFT_EINVAL;
  CK(h, cudaSetDevice(h->dev));
  CK(h, cudaMemcpy2DAsync(f, (size_t)h->ntm * sizeof(double), h->buf[h->cur], (size_t)h->ldt * sizeof(double),
                          (size_t)h->ntm * sizeof(double), (size_t)h->npm * h->nr, cudaMemcpyDeviceToHost,
                          h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return HIPFT_OK;
}

// get_flux of a host (ntm,npm) slab (src/hipft.f90:8706-8738).
static void host_flux(const hipft_gpu *h, const double *map, double &fp, double &fm) {
  fp = 0.0;
  fm = 0.0;
  for (int k = 1; k <= h->npm - 1; ++k)
    for (int j = 1; j <= h->ntm; ++j) {
      double fv = map[(size_t)(k - 1) * h->ntm + (j - 1)] * h->da_t[j] * h->da_p[k];
      if (fv > 0.0) fp = fp + fv; else fm = fm + fv;
    }
}

extern "C" int hipft_gpu_load_initial_map(hipft_gpu *h, const double *map_pt, int flux_balance, double mult_fac) {
  if (!h || !map_pt) return HIPFT_EINVAL;
  int ntm = h->ntm, npm = h->npm, npm1 = h->npm1, nr = h->nr;
  std::vector<double> f((size_t)ntm * npm * nr);
  auto F = [&](int j, int k, int i) -> double & { return f[((size_t)(i - 1) * npm + (k - 1)) * ntm + (j - 1)]; };
  for (int i = 1; i <= nr; ++i)
    for (int k = 1; k <= npm1; ++k)
      for (int j = 1; j <= ntm; ++j) F(j, k, i) = map_pt[((size_t)(i - 1) * ntm + (j - 1)) * npm1 + (k - 1)];
  for (int i = 1; i <= nr; ++i)
    for (int j = 1; j <= ntm; ++j) {
      F(j, 1, i) = 0.5 * (F(j, 1, i) + F(j, npm1, i));
      F(j, npm1, i) = F(j, 1, i);
      F(j, npm1 + 1, i) = F(j, 2, i);
    }
  for (int i = 1; i <= nr; ++i) {
    double fn1 = 0.0, fs1 = 0.0;
    for (int k = 2; k <= npm - 1; ++k) {
      fn1 = fn1 + F(1, k, i) * h->dp[k];
      fs1 = fs1 + F(ntm, k, i) * h->dp[k];
    }
    for (int k = 1; k <= npm; ++k) {
      F(1, k, i) = fn1 * 0.15915494309189535;
      F(ntm, k, i) = fs1 * 0.15915494309189535;
    }
  }
  if (flux_balance)
    for (int i = 1; i <= nr; ++i) {
      double *slab = &f[(size_t)(i - 1) * npm * ntm];
      double fp, fm;
      host_flux(h, slab, fp, fm);
      if (fm + fp == 0.0) continue;
      double ratio = std::sqrt(std::fabs(fp / fm));
      for (size_t q = 0; q < (size_t)npm * ntm; ++q) slab[q] = (slab[q] > 0) ? slab[q] / ratio : slab[q] * ratio;
    }
  for (auto &v : f) v = mult_fac * v;
  return hipft_gpu_set_field(h, f.data());
}

// ------------------------------------------------------------------ flows
extern "C" int hipft_gpu_set_flow(hipft_gpu *h, const hipft_flow_def *def) {
  if (!h || !def) return HIPFT_EINVAL;
  if (!h->P.advance_flow) return fail(h, HIPFT_ESTATE, "set_flow: advance_flow is off for this handle");
  int nr = h->nr;
  auto take = [&](std::vector<double> &v, const double *src, double dflt) {
    v.assign(nr, dflt);
    if (src) std::copy(src, src + nr, v.begin());
  };
  if ((def->flow_dr_model == 1 && (!def->dr_p0 || !def->dr_p2 || !def->dr_p4)) ||
      (def->flow_mf_model == 1 && (!def->mf_p1 || !def->mf_p3 || !def->mf_p5)) ||
      (def->flow_attenuate && !def->flow_attenuate_values))
    return fail(h, HIPFT_EINVAL, "set_flow: missing per-realization coefficients");
  take(h->f_p0, def->dr_p0, 0); take(h->f_p2, def->dr_p2, 0); take(h->f_p4, def->dr_p4, 0);
  take(h->f_p1, def->mf_p1, 0); take(h->f_p3, def->mf_p3, 0); take(h->f_p5, def->mf_p5, 0);
  take(h->f_att, def->flow_attenuate_values, 0);
  h->fdef = *def;
  h->have_flow = true;
  h->flow_needs_updating = true;
  // a flow from files, set before or after, stays the base of vt, vp
  h->flow2d = h->have_file_flow || def->flow_attenuate || def->flow_rigid_omega != 0.0;
  return HIPFT_OK;
}

// 1-D analytic parts of vt (theta faces) and vp (phi faces), per
// realization, in the order update_flow adds them (src/hipft.f90:3409-3437).
static void analytic_profiles(const hipft_gpu *h, std::vector<double> &vt1, std::vector<double> &vp1) {
  int nt = h->nt, ntm = h->ntm, nr = h->nr;
  const hipft_flow_def &d = h->fdef;
  vt1.assign((size_t)nr * (nt + 1), 0.0);
  vp1.assign((size_t)nr * (ntm + 1), 0.0);
  for (int i = 1; i <= nr; ++i) {
    double *vt = &vt1[(size_t)(i - 1) * (nt + 1)];
    double *vp = &vp1[(size_t)(i - 1) * (ntm + 1)];
    if (d.flow_mf_model == 1)
      for (int j = 1; j <= nt; ++j) {
        double c = h->cth[j];
        vt[j] = vt[j] - c_m_s_to_rs_hr * h->sth[j] *
                            (h->f_p1[i - 1] * c + h->f_p3[i - 1] * pow3(c) + h->f_p5[i - 1] * pow5(c));
      }
    if (d.flow_dr_model == 1)
      for (int j = 1; j <= ntm; ++j) {
        double c = h->ct[j];
        double c2 = c * c, c4 = c2 * c2;
        vp[j] = vp[j] + c_m_s_to_rs_hr * h->st[j] * (h->f_p0[i - 1] + h->f_p2[i - 1] * c2 + h->f_p4[i - 1] * c4);
      }
    if (d.flow_vp_rigid_omega != 0.0)
      for (int j = 1; j <= ntm; ++j) vp[j] = vp[j] + d.flow_vp_rigid_omega * c_km_s_to_rs_hr * h->st[j];
    if (d.flow_vt_const != 0.0)
      for (int j = 1; j <= nt; ++j) vt[j] = vt[j] + d.flow_vt_const * c_km_s_to_rs_hr;
  }
}

extern "C" int hipft_gpu_set_allreduce(hipft_gpu *h, hipft_allreduce_cb cb, void *user) {
  if (!h) return HIPFT_EINVAL;
  h->red_cb = cb;
  h->red_user = user;
  if (h->P.advance_diffusion) TRY(allreduce(h, HIPFT_RED_MIN, &h->dt_euler));  // src/hipft.f90:5036
  return HIPFT_OK;
}

extern "C" int hipft_gpu_set_flow_from_files(hipft_gpu *h, const double *vt_pt, const double *vp_pt,
                                             int at_load) {
  if (!h || !vt_pt || !vp_pt) return HIPFT_EINVAL;
  if (!h->P.advance_flow) return fail(h, HIPFT_ESTATE, "set_flow_from_files: advance_flow is off for this handle");
  CK(h, cudaSetDevice(h->dev));
  const int nt = h->nt, ntm = h->ntm, npm = h->npm, np = h->np, npm1 = h->npm1;
  std::vector<double> vt((size_t)npm * (nt + 1), 0.0), vp((size_t)np * (ntm + 1), 0.0);
  auto T = [&](int j, int k) -> double & { return vt[(size_t)(k - 1) * (nt + 1) + j]; };
  auto P = [&](int j, int k) -> double & { return vp[(size_t)(k - 1) * (ntm + 1) + j]; };
  for (int k = 1; k <= npm1; ++k)
    for (int j = 1; j <= nt; ++j) T(j, k) = c_m_s_to_rs_hr * vt_pt[(size_t)(j - 1) * npm1 + (k - 1)];
  for (int k = 1; k <= np; ++k)
    for (int j = 1; j <= ntm; ++j) P(j, k) = c_m_s_to_rs_hr * vp_pt[(size_t)(j - 1) * np + (k - 1)];
  if (at_load) {
    for (int j = 1; j <= nt; ++j) T(j, npm) = T(j, 2);  // src/hipft.f90:3789
  } else {                                             // set_periodic_bc_3d, src/hipft.f90:3604, 3634
    for (int j = 1; j <= nt; ++j) { T(j, 1) = T(j, npm - 1); T(j, npm) = T(j, 2); }
    for (int j = 1; j <= ntm; ++j) { P(j, 1) = P(j, np - 1); P(j, np) = P(j, 2); }
  }
  if (!h->d_vtf) {
    TRY(dalloc(h, &h->d_vtf, vt.size()));
    TRY(dalloc(h, &h->d_vpf, vp.size()));
  }
  TRY(upload(h, h->d_vtf, vt));
  TRY(upload(h, h->d_vpf, vp));
  CK(h, cudaStreamSynchronize(h->stream));  // the host staging vectors go out of scope
  h->have_file_flow = true;
  h->flow2d = true;
  h->flow_needs_updating = true;
  return HIPFT_OK;
}

extern "C" int hipft_gpu_update_flow(hipft_gpu *h, int *updated) {
  if (!h) return HIPFT_EINVAL;
  if (updated) *updated = 0;
  if (!(h->have_flow || h->have_file_flow) || !h->flow_needs_updating) return HIPFT_OK;
  CK(h, cudaSetDevice(h->dev));
  h->flow_needs_updating = false;
  int nt = h->nt, ntm = h->ntm, nr = h->nr, npm = h->npm;
  std::vector<double> vt1, vp1;
  analytic_profiles(h, vt1, vp1);
  TRY(upload(h, h->d_vt1, vt1));
  TRY(upload(h, h->d_vp1, vp1));
  if (!h->flow2d) {
    // set_lf_alpha on theta-only profiles (src/hipft.f90:6968-7037)
    std::vector<double> at1((size_t)nr * (ntm + 1), 0.0), ap1((size_t)nr * (ntm + 1), 0.0);
    for (int i = 1; i <= nr; ++i) {
      const double *vt = &vt1[(size_t)(i - 1) * (nt + 1)];
      const double *vp = &vp1[(size_t)(i - 1) * (ntm + 1)];
      double *at = &at1[(size_t)(i - 1) * (ntm + 1)];
      double *ap = &ap1[(size_t)(i - 1) * (ntm + 1)];
      auto A = [&](int j) { return std::fabs(vt[j]); };
      for (int j = 3; j <= nt - 3; ++j)
        at[j] = std::max(std::max(std::max(std::max(std::max(A(j - 2), A(j - 1)), A(j)), A(j + 1)), A(j + 2)), A(j + 3));
      at[1] = std::max(std::max(std::max(A(1), A(2)), A(3)), A(4));
      at[2] = std::max(std::max(std::max(std::max(A(1), A(2)), A(3)), A(4)), A(5));
      { int j = nt - 2; at[j] = std::max(std::max(std::max(std::max(A(j - 2), A(j - 1)), A(j)), A(j + 1)), A(j + 2)); }
      { int j = nt - 1; at[j] = std::max(std::max(std::max(A(j - 2), A(j - 1)), A(j)), A(j + 1)); }
      for (int j = 2; j <= ntm - 1; ++j) ap[j] = std::fabs(vp[j]);
    }
    TRY(upload(h, h->d_at1, at1));
    TRY(upload(h, h->d_ap1, ap1));
    h->FL.flow2d = 0;
  } else {
    if (!h->d_vt) {
      size_t n2 = (size_t)h->ldv * npm * nr;
      TRY(dalloc(h, &h->d_vt, n2));
      TRY(dalloc(h, &h->d_vp, n2));
      TRY(dalloc(h, &h->d_at, n2));
      TRY(dalloc(h, &h->d_ap, n2));
      CK(h, cudaMemsetAsync(h->d_at, 0, n2 * sizeof(double), h->stream));
      CK(h, cudaMemsetAsync(h->d_ap, 0, n2 * sizeof(double), h->stream));
      // cos(p), sin(p), cos(ph), theta metrics (1-based), attenuation factors
      size_t L = (size_t)std::max(npm, nt) + 2;
      std::vector<double> trig(7 * L, 0.0);
      for (int k = 1; k <= npm; ++k) {
        trig[k] = std::cos(h->p[k]);
        trig[L + k] = std::sin(h->p[k]);
        trig[2 * L + k] = std::cos(h->ph[k]);
      }
      for (int j = 1; j <= nt; ++j) { trig[3 * L + j] = h->cth[j]; trig[4 * L + j] = h->sth[j]; }
      for (int j = 1; j <= ntm; ++j) { trig[5 * L + j] = h->ct[j]; trig[6 * L + j] = h->st[j]; }
      TRY(dalloc(h, &h->d_trig, trig.size()));
      TRY(upload(h, h->d_trig, trig));
      std::vector<double> att(nr + 1, 0.0);
      for (int i = 1; i <= nr; ++i)
        att[i] = (h->f_att[i - 1] > 0.0) ? 1.0 / h->f_att[i - 1] : DBL_MAX;
      TRY(dalloc(h, &h->d_atten, nr + 1));
      TRY(upload(h, h->d_atten, att));
    }
    if (h->fdef.flow_attenuate && !h->field_set) return fail(h, HIPFT_ESTATE, "update_flow: attenuation needs the field");
    size_t L = (size_t)std::max(npm, nt) + 2;
    Flow2DBuild b{};
    b.vt1 = h->d_vt1; b.vp1 = h->d_vp1;
    b.cosp = h->d_trig; b.sinp = h->d_trig + L; b.cosph = h->d_trig + 2 * L;
    b.cth = h->d_trig + 3 * L; b.sth = h->d_trig + 4 * L; b.ct = h->d_trig + 5 * L; b.st = h->d_trig + 6 * L;
    b.vrigid = h->fdef.flow_rigid_omega * c_km_s_to_rs_hr;
    b.attenuate = h->fdef.flow_attenuate;
    b.atten_i = h->d_atten;
    if (h->have_file_flow) {
      // the analytic terms one by one, as update_flow adds them over the
      // file flow (src/hipft.f90:3416-3437, 7219-7285)
      const hipft_flow_def &d = h->fdef;
      const size_t nT = (size_t)nr * (nt + 1), nP = (size_t)nr * (ntm + 1);
      std::vector<double> terms(nT + nP + (size_t)(ntm + 1), 0.0);
      double *tmf = terms.data(), *vdr = tmf + nT, *vrg = vdr + nP;
      for (int i = 1; i <= nr; ++i) {
        for (int j = 1; j <= nt; ++j) {
          double c = h->cth[j];
          tmf[(size_t)(i - 1) * (nt + 1) + j] =
              c_m_s_to_rs_hr * h->sth[j] * (h->f_p1[i - 1] * c + h->f_p3[i - 1] * pow3(c) + h->f_p5[i - 1] * pow5(c));
        }
        for (int j = 1; j <= ntm; ++j) {
          double c = h->ct[j];
          double c2 = c * c, c4 = c2 * c2;
          vdr[(size_t)(i - 1) * (ntm + 1) + j] =
              c_m_s_to_rs_hr * h->st[j] * (h->f_p0[i - 1] + h->f_p2[i - 1] * c2 + h->f_p4[i - 1] * c4);
        }
      }
      for (int j = 1; j <= ntm; ++j) vrg[j] = d.flow_vp_rigid_omega * c_km_s_to_rs_hr * h->st[j];
      if (!h->d_fterms) TRY(dalloc(h, &h->d_fterms, terms.size()));
      TRY(upload(h, h->d_fterms, terms));
      b.vtf = h->d_vtf;
      b.vpf = h->d_vpf;
      b.tmf = (d.flow_mf_model == 1) ? h->d_fterms : nullptr;
      b.vdr = (d.flow_dr_model == 1) ? h->d_fterms + nT : nullptr;
      b.vrg = (d.flow_vp_rigid_omega != 0.0) ? h->d_fterms + nT + nP : nullptr;
      b.vtc = (d.flow_vt_const != 0.0) ? d.flow_vt_const * c_km_s_to_rs_hr : 0.0;
    }
    dim3 blk(32, 8), grd((unsigned)((nt + 31) / 32), (unsigned)((npm + 7) / 8), (unsigned)nr);
    k_flow_build<<<grd, blk, 0, h->stream>>>(h->M, b, h->ldv, h->buf[h->cur], h->d_vt, h->d_vp);
    LAUNCHED(h);
    if (h->fdef.flow_attenuate) {
      k_seam<<<dim3((unsigned)((nt + 127) / 128), (unsigned)nr), 128, 0, h->stream>>>(h->M, nt, h->ldv, h->d_vt);
      LAUNCHED(h);
      k_seam<<<dim3((unsigned)((ntm + 127) / 128), (unsigned)nr), 128, 0, h->stream>>>(h->M, ntm, h->ldv, h->d_vp);
      LAUNCHED(h);
      h->flow_needs_updating = true;  // Br changes every step (src/hipft.f90:3514)
    }
    if (h->have_file_flow) h->flow_needs_updating = true;  // src/hipft.f90:3423
    if (h->adv_space == 2) {
      dim3 g2((unsigned)((ntm + 31) / 32), (unsigned)((npm + 7) / 8), (unsigned)nr);
      k_lf_alpha<<<g2, blk, 0, h->stream>>>(h->M, h->ldv, h->d_vt, h->d_vp, h->d_at, h->d_ap);
      LAUNCHED(h);
    }
    h->FL.vt = h->d_vt; h->FL.vp = h->d_vp; h->FL.at = h->d_at; h->FL.ap = h->d_ap;
    h->FL.flow2d = 1;
  }
  h->r_dtmax_valid = false;
  if (updated) *updated = 1;
  return HIPFT_OK;
}

extern "C" int hipft_gpu_flow_dtmax(hipft_gpu *h, double *dtmax) {
  if (!h || !dtmax) return HIPFT_EINVAL;
  if (!h->P.advance_flow) return fail(h, HIPFT_ESTATE, "flow_dtmax: advance_flow is off");
  CK(h, cudaSetDevice(h->dev));
  unsigned long long init = 0x7fefffffffffffffULL;  // DBL_MAX bits
  CK(h, cudaMemcpyAsync(h->d_bits + 1, &init, 8, cudaMemcpyHostToDevice, h->stream));
  dim3 blk(32, 8), grd((unsigned)((h->ntm - 2 + 31) / 32), (unsigned)((h->npm - 2 + 7) / 8), (unsigned)h->nr);
  k_flow_dtmax<<<grd, blk, 0, h->stream>>>(h->M, h->FL, h->d_bits + 1);
  LAUNCHED(h);
  TRY(sync_read(h, h->d_bits + 1, 8));
  double d;
  std::memcpy(&d, h->h_pin, 8);
  d = c_safety * d;
  if (h->P.strang_splitting) d = 2.0 * d;
  if (h->adv_time == 3) d = 2.0 * d;
  TRY(allreduce(h, HIPFT_RED_MIN, &d));  // src/hipft.f90:7345
  *dtmax = d;
  return HIPFT_OK;
}

// ------------------------------------------------------------- advection
static int ragged_advection_step(hipft_gpu *h, double dt);

static int plain_advection_step(hipft_gpu *h, double dt) {
  h->dring_valid = false;
  double *f = h->buf[h->cur];
  int ia = scratch(h, 0), ib = scratch(h, 1);
  double *A = h->buf[ia], *B = h->buf[ib];
  if (h->adv_time == 1) {  // FE (src/hipft.f90:7440-7444)
    TRY(advection_stage(h, f, nullptr, A, AdvCombine{0, 0.0, 0.0, dt}));
    h->cur = ia;
  } else if (h->adv_time == 2) {  // SSPRK(3,3) (7486-7505)
    TRY(advection_stage(h, f, nullptr, A, AdvCombine{0, 0.0, 0.0, dt}));
    TRY(advection_stage(h, A, f, B, AdvCombine{1, c_three_quarter, c_quarter, c_quarter * dt}));
    TRY(advection_stage(h, B, f, f, AdvCombine{1, c_third, c_two_third, c_two_third * dt}));
  } else {  // SSPRK(4,3) (7552-7574)
    TRY(advection_stage(h, f, nullptr, A, AdvCombine{0, 0.0, 0.0, 0.5 * dt}));
    TRY(advection_stage(h, A, nullptr, B, AdvCombine{0, 0.0, 0.0, 0.5 * dt}));
    TRY(advection_stage(h, B, f, A, AdvCombine{1, c_two_third, c_third, c_sixth * dt}));
    TRY(advection_stage(h, A, nullptr, f, AdvCombine{0, 0.0, 0.0, 0.5 * dt}));
  }
  return HIPFT_OK;
}

extern "C" int hipft_gpu_advection_step(hipft_gpu *h, double dt) {
  if (!h) return HIPFT_EINVAL;
  if (!h->field_set) return fail(h, HIPFT_ESTATE, "advection_step before set_field");
  if (!h->P.advance_flow) return fail(h, HIPFT_ESTATE, "advection_step: advance_flow is off");
  CK(h, cudaSetDevice(h->dev));
  if (h->ragged) return ragged_advection_step(h, dt);
  return plain_advection_step(h, dt);
}

// ------------------------------------------------------------- diffusion
// Stage count and coefficients of one RKL2 (method 2) or RKG2 (method 3)
// super-step, load_sts_rkl2 / load_sts_rkg2 (src/hipft.f90:5244-5475).
struct StsTable {
  int64_t s = 0;
  std::vector<double> uj, vj, ubj, gj, b;
};
static void sts_coefs(int method, double dtl, double dt_euler, StsTable &T) {
  const int64_t s = sts_count(method, dtl, dt_euler);
  T.s = s;
  T.b.assign(s + 1, 0); T.uj.assign(s + 1, 0); T.vj.assign(s + 1, 0); T.ubj.assign(s + 1, 0); T.gj.assign(s + 1, 0);
  for (int64_t j = 1; j <= s; ++j) {
    T.b[j] = sts_b(method, j);
    sts_stage(method, s, j, T.uj[j], T.vj[j], T.ubj[j], T.gj[j]);
  }
}

// The stage-k combine coefficients of a super-step of length dtl
// (src/hipft.f90:5224-5235).
static StageCoef sts_stage_coef(const StsTable &T, int64_t k, double dtl) {
  double uj = T.uj[k], vj = T.vj[k];
  return StageCoef{uj, vj, 1.0 - uj - vj, T.ubj[k] * dtl, T.gj[k]};
}

static void load_sts(hipft_gpu *h, double dtl) {
  StsTable T;
  sts_coefs(h->P.diffusion_num_method, dtl, h->dt_euler, T);
  h->sts_s = T.s;
  h->sts_b = std::move(T.b);
  h->sts_uj = std::move(T.uj);
  h->sts_vj = std::move(T.vj);
  h->sts_ubj = std::move(T.ubj);
  h->sts_gj = std::move(T.gj);
}

// diffusion_step_sts_cd (src/hipft.f90:5163-5242): stage 1 then the
// s-1 fused stages, rotating three scratch fields.
static int sts_super_step(hipft_gpu *h, double dtl) {
  if (!h->DC.grid) TRY(ensure_pair_plan(h));
  load_sts(h, dtl);
  int u0 = h->cur, idty = scratch(h, 0), ia = scratch(h, 1), ib = scratch(h, 2);
  const bool fused = !h->DC.grid;
  if (fused) {
    const double *r0;
    TRY(current_dring(h, &r0));
    TRY(sts_stage_v2<MODE_STS1>(h, h->buf[u0], nullptr, nullptr, nullptr, h->buf[ia], h->buf[idty],
                                StageCoef{dtl, h->sts_ubj[1], 0, 0, 0}));
  } else {
    TRY(ring_diffusion(h, h->buf[u0], h->d_ring));
    TRY(diffusion_stage<MODE_STS1>(h, h->buf[u0], nullptr, nullptr, nullptr, h->buf[ia], h->buf[idty], h->d_ring,
                                   StageCoef{dtl, h->sts_ubj[1], 0, 0, 0}, nullptr));
  }
  int ykm1 = ia, ykm2 = u0;
  auto coef = [&](int64_t k) {
    double uj = h->sts_uj[k], vj = h->sts_vj[k];
    return StageCoef{uj, vj, 1.0 - uj - vj, h->sts_ubj[k] * dtl, h->sts_gj[k]};
  };
  // a buffer not holding u0, dty0, Y_{k-1}, Y_{k-2} (or `avoid`)
  auto free_buf = [&](int avoid) {
    for (int b = 0; b < h->nbuf; ++b)
      if (b != u0 && b != idty && b != ykm1 && b != ykm2 && b != avoid) return b;
    return -1;
  };
  (void)ib;
  int64_t k = 2;
  while (k <= h->sts_s) {
    if (fused && h->plan.kind == PK_WS_QUAD && k + 3 <= h->sts_s) {
      int ob[4], no = 0;
      for (int b = 0; b < h->nbuf && no < 4; ++b)
        if (b != u0 && b != idty && b != ykm1 && b != ykm2) ob[no++] = b;
      const StageCoef cq[4] = {coef(k), coef(k + 1), coef(k + 2), coef(k + 3)};
      TRY(quad_pass(h, h->buf[ykm1], h->buf[ykm2], h->buf[u0], h->buf[idty], h->buf[ob[0]], h->buf[ob[1]],
                    h->buf[ob[2]], h->buf[ob[3]], cq, k > 2));
      ykm2 = ob[2];
      ykm1 = ob[3];
      k += 4;
      h->rkg2_stages += 4;
      h->rkg2_cell_stages += 4 * (int64_t)h->ntm * (h->npm - 2) * h->nr;
      continue;
    }
    if (fused && sts_pairs_enabled(h) && k + 1 <= h->sts_s) {
      int bk = free_buf(-1), bk1 = free_buf(bk);
      TRY(sts_pair(h, h->buf[ykm1], h->buf[ykm2], h->buf[u0], h->buf[idty], h->buf[bk], h->buf[bk1], coef(k),
                   coef(k + 1), k > 2));
      ykm2 = bk;
      ykm1 = bk1;
      k += 2;
      h->rkg2_stages += 2;
      h->rkg2_cell_stages += 2 * (int64_t)h->ntm * (h->npm - 2) * h->nr;
      continue;
    }
    int out = (ykm2 == u0) ? free_buf(-1) : ykm2;
    StageCoef sc = coef(k);
    if (fused) {
      TRY(sts_stage_v2<MODE_STSK>(h, h->buf[ykm1], h->buf[ykm2], h->buf[u0], h->buf[idty], h->buf[out], nullptr,
                                  sc));
    } else {
      TRY(ring_diffusion(h, h->buf[ykm1], h->d_ring));
      TRY(diffusion_stage<MODE_STSK>(h, h->buf[ykm1], h->buf[ykm2], h->buf[u0], h->buf[idty], h->buf[out],
                                     nullptr, h->d_ring, sc, nullptr));
    }
    ykm2 = ykm1;
    ykm1 = out;
    k += 1;
    h->rkg2_stages += 1;
    h->rkg2_cell_stages += (int64_t)h->ntm * (h->npm - 2) * h->nr;
  }
  h->cur = ykm1;
  h->dring_valid = fused;  // the last fused stage left the ring of the new field
  h->cell_updates += (int64_t)h->ntm * (h->npm - 2) * h->nr * h->sts_s;
  return HIPFT_OK;
}

// diffusion_step_fe_cd (src/hipft.f90:7352-7407).
static int euler_steps(hipft_gpu *h, double dtl) {
  int64_t n = (int64_t)std::ceil(dtl / h->dt_euler);
  h->n_euler = n;
  double dte = dtl / (double)n;
  for (int64_t c = 0; c < n; ++c) {
    int o = scratch(h, 0);
    if (!h->DC.grid) {
      const double *r0;
      TRY(current_dring(h, &r0));
      TRY(sts_stage_v2<MODE_EULER>(h, h->buf[h->cur], nullptr, nullptr, nullptr, h->buf[o], nullptr,
                                   StageCoef{dte, 0, 0, 0, 0}));
      h->cur = o;
      h->dring_valid = true;
    } else {
      TRY(ring_diffusion(h, h->buf[h->cur], h->d_ring));
      TRY(diffusion_stage<MODE_EULER>(h, h->buf[h->cur], nullptr, nullptr, nullptr, h->buf[o], nullptr, h->d_ring,
                                      StageCoef{dte, 0, 0, 0, 0}, nullptr));
      h->cur = o;
      h->dring_valid = false;
    }
  }
  h->cell_updates += (int64_t)h->ntm * (h->npm - 2) * h->nr * n;
  return HIPFT_OK;
}

// get_dtime_diffusion_ptl (src/hipft.f90:5042-5161).
// Reads and clears the flag that kernels set when a bounded wait gave up;
// HIPFT_ETIMEOUT if it was set (the context stays usable).
static int check_wait_flag(hipft_gpu *h, const char *what) {
  int ev = 0;
  CK(h, cudaMemcpyAsync(&ev, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  if (!ev) return HIPFT_OK;
  CK(h, cudaMemsetAsync(h->d_err, 0, sizeof(int), h->stream));
  CK(h, cudaMemsetAsync(h->d_rcount, 0, sizeof(unsigned int) * h->nr, h->stream));
  return fail(h, HIPFT_ETIMEOUT, "%s", what);
}

static int ptl_dt(hipft_gpu *h, double *dtl) {
  double dtime_in = *dtl;
  double *f = h->buf[h->cur], *af = h->buf[scratch(h, 0)];
  CK(h, cudaMemsetAsync(h->d_bits, 0, 2 * sizeof(unsigned long long), h->stream));
  const double *ring;
  TRY(current_dring(h, &ring));
  TRY(diffusion_stage<MODE_AX>(h, f, nullptr, nullptr, nullptr, af, nullptr, ring, StageCoef{}, h->d_bits));
  TRY(sync_read(h, h->d_bits, 8));
  double axabsmax;
  std::memcpy(&axabsmax, h->h_pin, 8);
  if (h->red_cb) {  // src/hipft.f90:5103: the PTL cells are those at the global maximum
    TRY(allreduce(h, HIPFT_RED_MAX, &axabsmax));
    CK(h, cudaMemcpyAsync(h->d_bits, &axabsmax, 8, cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
  }
  double d = DBL_MAX;
  if (axabsmax > 0.0) {
    unsigned long long init = 0x7fefffffffffffffULL;
    CK(h, cudaMemcpyAsync(h->d_bits + 1, &init, 8, cudaMemcpyHostToDevice, h->stream));
    dim3 blk(32, 8);
    k_ptl<<<stage_grid(h, 32, 8), blk, 0, h->stream>>>(h->M, f, af, h->d_bits, h->d_bits + 1);
    LAUNCHED(h);
    TRY(sync_read(h, h->d_bits + 1, 8));
    std::memcpy(&d, h->h_pin, 8);
    TRY(allreduce(h, HIPFT_RED_MIN, &d));  // src/hipft.f90:5141
    d = 0.95 * d;
    if (d < dtime_in) d = dtime_in;
  }
  *dtl = d;
  return HIPFT_OK;
}

// ================================================================ ragged
// Ragged batches (no counterpart in the reference, which keeps one dt, one
// Euler limit, one stage count and one PTL subcycle sequence for all
// realizations through global MIN/MAX reductions, src/hipft.f90:5036, 5103,
// 5141, 7345).  In a ragged batch every realization gets the schedule it would
// have if it were run alone: its own Gershgorin limit, its own PTL subcycles
// and RKG2/RKL2 stage counts, and, when the step is longer than its own CFL
// limit, its own number of advection substeps.  Launches still cover many
// realizations at once: a launch walks a list of realizations sorted by the
// work they still need, and the realizations that are done drop off its end.

// per-realization Euler limits, get_dtime_diffusion_euler (src/hipft.f90:
// 5019-5025) of each realization alone
static int ragged_gershgorin(hipft_gpu *h) {
  const int nr = h->nr;
  CK(h, cudaMemsetAsync(h->d_rbits, 0, sizeof(unsigned long long) * nr, h->stream));
  dim3 blk(32, 8);
  dim3 grd((unsigned)((h->ntm - 2 + 31) / 32), (unsigned)((h->npm - 2 + 7) / 8), (unsigned)nr);
  k_gershgorin<<<grd, blk, 0, h->stream>>>(h->M, h->DC, h->d_rbits, 1);
  LAUNCHED(h);
  std::vector<unsigned long long> bits(nr);
  CK(h, cudaMemcpyAsync(bits.data(), h->d_rbits, sizeof(unsigned long long) * nr, cudaMemcpyDeviceToHost,
                        h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  h->r_dt_euler.assign(nr, 0.0);
  for (int i = 0; i < nr; ++i) {
    double max_eig;
    std::memcpy(&max_eig, &bits[i], 8);
    h->r_dt_euler[i] = c_safety * (2.0 / max_eig);
  }
  return HIPFT_OK;
}

// per-realization CFL limits, get_flow_dtmax (src/hipft.f90:7287-7350) of each
// realization alone
static int ragged_dtmax(hipft_gpu *h) {
  if (h->r_dtmax_valid) return HIPFT_OK;
  const int nr = h->nr;
  std::vector<unsigned long long> bits(nr, 0x7fefffffffffffffULL);
  CK(h, cudaMemcpyAsync(h->d_rbits, bits.data(), sizeof(unsigned long long) * nr, cudaMemcpyHostToDevice,
                        h->stream));
  dim3 blk(32, 8), grd((unsigned)((h->ntm - 2 + 31) / 32), (unsigned)((h->npm - 2 + 7) / 8), (unsigned)nr);
  k_flow_dtmax<<<grd, blk, 0, h->stream>>>(h->M, h->FL, h->d_rbits, 1);
  LAUNCHED(h);
  CK(h, cudaMemcpyAsync(bits.data(), h->d_rbits, sizeof(unsigned long long) * nr, cudaMemcpyDeviceToHost,
                        h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  h->r_dtmax.assign(nr, 0.0);
  for (int i = 0; i < nr; ++i) {
    double d;
    std::memcpy(&d, &bits[i], 8);
    d = c_safety * d;
    if (h->P.strang_splitting) d = 2.0 * d;
    if (h->adv_time == 3) d = 2.0 * d;
    h->r_dtmax[i] = d;
  }
  h->r_dtmax_valid = true;
  return HIPFT_OK;
}

// realizations `act` ordered by decreasing work (ties by index), uploaded
static int upload_list(hipft_gpu *h, int *dlist, std::vector<int> &act, const std::vector<int64_t> &work) {
  std::stable_sort(act.begin(), act.end(), [&](int a, int b) { return work[a] > work[b]; });
  CK(h, cudaMemcpyAsync(dlist, act.data(), sizeof(int) * act.size(), cudaMemcpyHostToDevice, h->stream));
  return HIPFT_OK;
}

// PTL time steps (src/hipft.f90:5042-5161) of the realizations in `act`,
// each from its own max |Af| and its own argmax cells; dtl[i] is the
// realization's previous subcycle (the floor), replaced by the new one.
static int ragged_ptl(hipft_gpu *h, std::vector<int> act, std::vector<double> &dtl) {
  const int nr = h->nr, na = (int)act.size();
  std::vector<int64_t> none(nr, 0);
  TRY(upload_list(h, h->d_rlist_dif, act, none));
  std::vector<unsigned long long> init(2 * (size_t)nr, 0ULL);
  for (int i = 0; i < nr; ++i) init[nr + i] = 0x7fefffffffffffffULL;
  CK(h, cudaMemcpyAsync(h->d_rbits, init.data(), sizeof(unsigned long long) * 2 * nr, cudaMemcpyHostToDevice,
                        h->stream));
  double *f = h->buf[h->cur], *af = h->buf[scratch(h, 0)];
  const double *ring;
  TRY(current_dring(h, &ring));
  dim3 blk(32, 8);
  dim3 grd((unsigned)((h->ntm + 31) / 32), (unsigned)((h->npm - 2 + 7) / 8), (unsigned)na);
  {
    ProfScope ps(h, HIPFT_K_OTHER);
    k_diffusion_stage<MODE_AX><<<grd, blk, 0, h->stream>>>(h->M, h->DC, f, nullptr, nullptr, nullptr, af, nullptr,
                                                          ring, h->bc_diff_n, h->bc_diff_s, StageCoef{}, h->d_rbits,
                                                          h->d_rlist_dif, 1);
    LAUNCHED(h);
    k_ptl<<<grd, blk, 0, h->stream>>>(h->M, f, af, h->d_rbits, h->d_rbits + nr, h->d_rlist_dif, 1);
    LAUNCHED(h);
  }
  std::vector<unsigned long long> bits(2 * (size_t)nr);
  CK(h, cudaMemcpyAsync(bits.data(), h->d_rbits, sizeof(unsigned long long) * 2 * nr, cudaMemcpyDeviceToHost,
                        h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  for (int i : act) {
    double axabsmax, ptl;
    std::memcpy(&axabsmax, &bits[i], 8);
    std::memcpy(&ptl, &bits[nr + i], 8);
    double d = DBL_MAX;
    if (axabsmax > 0.0) {
      d = 0.95 * ptl;
      if (d < dtl[i]) d = dtl[i];
    }
    dtl[i] = d;
  }
  return HIPFT_OK;
}

// Two-stage launch of a ragged super-step: the first n realizations of the
// list d_rlist_dif, coefficients rc ([nr][2]).
static int sts_pair_ragged(hipft_gpu *h, const double *ykm1, const double *ykm2, const double *u0,
                           const double *dty0, double *out_k, double *out_k1, int n, const StageCoef *rc,
                           bool overlap_prev) {
  const int nkt = (h->npm - 2 + kWK - 1) / kWK;
  RingOut ro{h->d_ringbuf[1 - h->ring_cur], h->d_rpart, h->d_rcount, nkt};
  PairTables pt = h->ptab;
  pt.ntiles = pt.nb * pt.nkt * n;
  const int cps = (h->plan.kind == PK_WS_ROWS2) ? h->plan.ctas_per_sm : 2;
  const int grid = std::min(pt.ntiles, cps * h->num_sms);
  PairArgs pa{StageCoef{}, StageCoef{}, h->d_err, h->d_rlist_dif, rc};
  const double *rin = h->d_ringbuf[h->ring_cur];
  const WsMaps tmaps = ws_maps(h, ykm1, ykm2, u0, dty0);
  {
    ProfScope ps(h, HIPFT_K_STS);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kWThreads);
    cfg.dynamicSmemBytes = kWSmem;
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = (ws_pdl() && overlap_prev) ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t le = cudaLaunchKernelEx(&cfg, k_sts_pair_ws<true, false, true>, h->M,
                                        (const double *)h->DC.dfac, ykm1, ykm2, u0, dty0, out_k, out_k1, rin,
                                        h->bc_diff_n, h->bc_diff_s, pa, ro, pt, tmaps);
    if (le != cudaSuccess) return fail(h, HIPFT_ECUDA, "k_sts_pair_ws (ragged) launch: %s", cudaGetErrorString(le));
    LAUNCHED(h);
    dim3 pg((unsigned)n, (unsigned)h->pole_nch);
    k_pair_poles<<<pg, kPoleThreads, 0, h->stream>>>(h->M, h->DC.dfac, ykm1, ykm2, u0, dty0, out_k1, rin,
                                                     h->bc_diff_n, h->bc_diff_s, pa, ro, h->pole);
    LAUNCHED(h);
  }
  h->ring_cur = 1 - h->ring_cur;
  return HIPFT_OK;
}

// One RKG2/RKL2 super-step of every realization in `act`, realization i over
// dtl[i] with its own stage count s_i (src/hipft.f90:5163-5242 per
// realization).  The launch of stage pair p covers the realizations with
// s_i >= 2p + 3; afterwards every realization's field is gathered into one
// buffer, which becomes the current field.
static int ragged_super_step(hipft_gpu *h, std::vector<int> act, const std::vector<double> &dtl) {
  const int nr = h->nr, method = h->P.diffusion_num_method;
  TRY(ensure_pair_plan(h));
  std::vector<StsTable> T(nr);
  std::vector<int64_t> s(nr, 0);
  int64_t smax = 0;
  for (int i : act) {
    sts_coefs(method, dtl[i], h->r_dt_euler[i], T[i]);
    s[i] = T[i].s;
    h->r_s[i] = T[i].s;
    smax = std::max(smax, s[i]);
  }
  TRY(upload_list(h, h->d_rlist_dif, act, s));
  const int na = (int)act.size();
  const int64_t npairs = (smax - 1) / 2;  // s is odd: stages 2..s are (s-1)/2 pairs
  // stage-1 and pair coefficients, per realization
  std::vector<StageCoef> c1(nr, StageCoef{});
  for (int i : act) c1[i] = StageCoef{dtl[i], T[i].ubj[1], 0, 0, 0};
  CK(h, cudaMemcpyAsync(h->d_r1coef, c1.data(), sizeof(StageCoef) * nr, cudaMemcpyHostToDevice, h->stream));
  if ((size_t)npairs > h->rcoef_pairs) {
    if (h->d_rcoef) {
      CK(h, cudaStreamSynchronize(h->stream));
      cudaFree(h->d_rcoef);
      h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void *)h->d_rcoef), h->allocs.end());
      h->d_rcoef = nullptr;
    }
    const size_t cap = (size_t)npairs + 64;
    TRY(dalloc(h, &h->d_rcoef, cap * nr * 2));
    h->rcoef_pairs = cap;
  }
  std::vector<StageCoef> pc((size_t)npairs * nr * 2, StageCoef{});
  for (int i : act)
    for (int64_t q = 0; q < (s[i] - 1) / 2; ++q) {
      const int64_t k = 2 + 2 * q;
      pc[((size_t)q * nr + i) * 2] = sts_stage_coef(T[i], k, dtl[i]);
      pc[((size_t)q * nr + i) * 2 + 1] = sts_stage_coef(T[i], k + 1, dtl[i]);
    }
  CK(h, cudaMemcpyAsync(h->d_rcoef, pc.data(), sizeof(StageCoef) * pc.size(), cudaMemcpyHostToDevice, h->stream));

  const int u0 = h->cur, idty = scratch(h, 0), ia = scratch(h, 1);
  const double *r0;
  TRY(current_dring(h, &r0));
  {
    // stage 1 (src/hipft.f90:5211-5218) of every realization in the list
    const int nkb = (h->npm - 2 + kKPT3 - 1) / kKPT3;
    RingOut ro{h->d_ringbuf[1 - h->ring_cur], h->d_rpart, h->d_rcount, nkb};
    const int jshift = (h->ntm % 2 == 1 && ((h->ntm - 1) / 2) % 32 == 0) ? 1 : 0;
    const int nthr = (h->ntm + 2 * jshift + 1) / 2;
    dim3 grd((unsigned)((nthr + 127) / 128), (unsigned)nkb, (unsigned)na);
    ProfScope ps(h, HIPFT_K_OTHER);
    k_sts_stage_v3<MODE_STS1, kKPT3><<<grd, 128, 0, h->stream>>>(
        h->M, h->DC.dfac, h->buf[u0], nullptr, nullptr, nullptr, h->buf[ia], h->buf[idty], h->d_ringbuf[h->ring_cur],
        h->bc_diff_n, h->bc_diff_s, StageCoef{}, ro, jshift, h->d_rlist_dif, h->d_r1coef);
    LAUNCHED(h);
    h->ring_cur = 1 - h->ring_cur;
  }
  int ykm1 = ia, ykm2 = u0;
  auto free_buf = [&](int avoid) {
    for (int b = 0; b < h->nbuf; ++b)
      if (b != u0 && b != idty && b != ykm1 && b != ykm2 && b != avoid) return b;
    return -1;
  };
  std::vector<int> fin(nr, u0);  // buffer holding each realization's result
  const int64_t cells = (int64_t)h->ntm * (h->npm - 2);
  const bool quad = h->plan.kind == PK_WS_QUAD && h->d_qcol;
  for (int64_t q = 0; q < npairs;) {
    int n = 0;   // realizations with pair q
    while (n < na && (s[act[n]] - 1) / 2 > q) ++n;
    int nq = 0;  // realizations with pairs q and q+1: four stages in one pass
    while (quad && nq < na && (s[act[nq]] - 1) / 2 >= q + 2) ++nq;
    if (nq > 0) {
      int ob[4], no = 0;
      for (int b = 0; b < h->nbuf && no < 4; ++b)
        if (b != u0 && b != idty && b != ykm1 && b != ykm2) ob[no++] = b;
      const StageCoef *rcA = h->d_rcoef + (size_t)q * nr * 2, *rcB = h->d_rcoef + (size_t)(q + 1) * nr * 2;
      const StageCoef none[4] = {};
      const PairTables pp = quad_pole_tables(h, nq);
      const int cps = h->plan.ctas_per_sm;
      ProfScope ps(h, HIPFT_K_STS);
      // stages k, k+1: the pole blocks of the four-stage realizations and, for
      // the realizations whose last pair this is, every block
      TRY(ws_pair_launch(h, pp, cps, h->buf[ykm1], h->buf[ykm2], h->buf[u0], h->buf[idty], h->buf[ob[0]],
                         h->buf[ob[1]], StageCoef{}, StageCoef{}, q > 0, h->d_rlist_dif, nq, rcA, n == nq));
      if (n > nq) {
        PairTables pt = h->ptab;
        pt.ntiles = pt.nb * pt.nkt * (n - nq);
        TRY(ws_pair_launch(h, pt, cps, h->buf[ykm1], h->buf[ykm2], h->buf[u0], h->buf[idty], h->buf[ob[0]],
                           h->buf[ob[1]], StageCoef{}, StageCoef{}, true, h->d_rlist_dif + nq, n - nq, rcA, true));
      }
      TRY(quad_launch(h, h->buf[ykm1], h->buf[ykm2], h->buf[u0], h->buf[idty], h->buf[ob[0]], h->buf[ob[1]],
                      h->buf[ob[2]], h->buf[ob[3]], none, h->d_rlist_dif, nq, rcA, rcB));
      TRY(ws_pair_launch(h, pp, cps, h->buf[ob[1]], h->buf[ob[0]], h->buf[u0], h->buf[idty], h->buf[ob[2]],
                         h->buf[ob[3]], StageCoef{}, StageCoef{}, false, h->d_rlist_dif, nq, rcB, true));
      for (int e = 0; e < n; ++e) {
        const int64_t P = (s[act[e]] - 1) / 2;
        if (e >= nq && P == q + 1) fin[act[e]] = ob[1];
        if (e < nq && P == q + 2) fin[act[e]] = ob[3];
      }
      ykm2 = ob[2];
      ykm1 = ob[3];
      h->rkg2_stages += 4;
      h->rkg2_cell_stages += 4 * cells * nq + 2 * cells * (n - nq);
      q += 2;
      continue;
    }
    const int bk = free_buf(-1), bk1 = free_buf(bk);
    TRY(sts_pair_ragged(h, h->buf[ykm1], h->buf[ykm2], h->buf[u0], h->buf[idty], h->buf[bk], h->buf[bk1], n,
                        h->d_rcoef + (size_t)q * nr * 2, q > 0));
    for (int e = 0; e < n; ++e)
      if ((s[act[e]] - 1) / 2 == q + 1) fin[act[e]] = bk1;
    ykm2 = bk;
    ykm1 = bk1;
    h->rkg2_stages += 2;
    h->rkg2_cell_stages += 2 * cells * n;
    q += 1;
  }
  // gather: realizations that finished earlier, and those not in this
  // super-step at all (still in u0), into the last pair's output
  const int dst = ykm1;
  const size_t pbytes = (size_t)h->plane * sizeof(double);
  for (int i = 0; i < nr; ++i)
    if (fin[i] != dst)
      CK(h, cudaMemcpyAsync(h->buf[dst] + (size_t)i * h->plane, h->buf[fin[i]] + (size_t)i * h->plane, pbytes,
                            cudaMemcpyDeviceToDevice, h->stream));
  h->cur = dst;
  h->dring_valid = false;  // the ring sums of the finished realizations sit in either buffer
  int64_t tot = 0;
  for (int i : act) tot += s[i];
  h->cell_updates += cells * tot;
  return HIPFT_OK;
}

// diffusion_step (src/hipft.f90:4551-4695) with every realization's own
// subcycle sequence (PTL) and stage counts.
static int ragged_diffusion_step(hipft_gpu *h, double dtl, hipft_diffusion_info *info) {
  const int nr = h->nr, max_sc = 60;
  const int64_t stages0 = h->cell_updates;
  std::vector<double> ts(nr, 0.0), d(nr, h->auto_sc ? 0.0 : dtl / (double)h->P.diffusion_subcycles);
  std::vector<int> act(nr);
  for (int i = 0; i < nr; ++i) act[i] = i;
  h->r_s.assign(nr, 0);
  h->r_cycles.assign(nr, 0);
  int cyc = 1;
  int64_t smax = 0;
  while (!act.empty()) {
    if (h->auto_sc) TRY(ragged_ptl(h, act, d));
    std::vector<int> done;
    for (int i : act) {
      bool fin = false;
      if (h->auto_sc && ts[i] + d[i] >= dtl) {
        d[i] = dtl - ts[i];
        fin = true;
      }
      if (h->auto_sc && cyc == max_sc - 1) {
        d[i] = dtl - ts[i];
        fin = true;
      }
      if (!h->auto_sc && cyc == h->P.diffusion_subcycles) fin = true;
      if (fin) done.push_back(i);
    }
    TRY(ragged_super_step(h, act, d));
    for (int i : act) {
      ts[i] = ts[i] + d[i];
      h->r_cycles[i] = cyc;
      smax = std::max(smax, h->r_s[i]);
    }
    std::vector<int> next;
    for (int i : act)
      if (std::find(done.begin(), done.end(), i) == done.end()) next.push_back(i);
    act.swap(next);
    cyc = cyc + 1;
  }
  TRY(check_wait_flag(h, "diffusion_step: a bounded wait for staged tiles gave up"));
  h->sts_s = smax;
  h->subcycles_state = cyc - 1;
  if (info) {
    info->dtime_diffusion_euler = *std::min_element(h->r_dt_euler.begin(), h->r_dt_euler.end());
    info->sts_s = smax;
    info->subcycles = cyc - 1;
    const int64_t cells = (int64_t)h->ntm * (h->npm - 2) * h->nr;
    info->total_stages = cells ? (h->cell_updates - stages0) / cells : 0;
  }
  return HIPFT_OK;
}

// advection_step (src/hipft.f90:4509-4549) with every realization's own
// substep count: realization i takes n_i = ceil(dt / its own CFL limit)
// substeps of dt / n_i (one substep when dt is within its limit, which is
// the plain step).
static int advection_stage_ragged(hipft_gpu *h, const double *x, const double *f0, double *out, AdvCombine cb,
                                  int n) {
  {
    ProfScope ps(h, HIPFT_K_RING);
    k_ring_advection<<<h->nr, 256, 0, h->stream>>>(h->M, h->FL, x, h->d_ring);
    LAUNCHED(h);
  }
  ProfScope ps(h, HIPFT_K_ADV);
  launch_adv_stage(h, h->M, h->stream, (unsigned)n, x, f0, out, cb, h->d_rlist_adv, h->d_rdt);
  LAUNCHED(h);
  h->cell_updates += (int64_t)h->ntm * (h->npm - 2) * n;
  return HIPFT_OK;
}

static int plain_advection_step(hipft_gpu *h, double dt);

static int ragged_advection_step(hipft_gpu *h, double dt) {
  const int nr = h->nr;
  TRY(ragged_dtmax(h));
  // the CFL limit bounds a whole split step: a Strang half step may use half of it
  const double scale = h->P.strang_splitting ? 2.0 : 1.0;
  std::vector<int64_t> n(nr, 1);
  int64_t nmax = 1;
  for (int i = 0; i < nr; ++i) {
    const double r = dt * scale / h->r_dtmax[i];
    n[i] = (r > 1.0) ? (int64_t)std::ceil(r) : 1;
    nmax = std::max(nmax, n[i]);
  }
  h->r_substeps = n;
  if (nmax == 1) return plain_advection_step(h, dt);
  std::vector<int> act(nr);
  for (int i = 0; i < nr; ++i) act[i] = i;
  TRY(upload_list(h, h->d_rlist_adv, act, n));
  std::vector<double> rdt(nr);
  for (int i = 0; i < nr; ++i) rdt[i] = dt / (double)n[i];
  CK(h, cudaMemcpyAsync(h->d_rdt, rdt.data(), sizeof(double) * nr, cudaMemcpyHostToDevice, h->stream));
  h->dring_valid = false;
  double *f = h->buf[h->cur];
  double *A = h->buf[scratch(h, 0)], *B = h->buf[scratch(h, 1)];
  for (int64_t q = 0; q < nmax; ++q) {
    int na = 0;
    while (na < nr && n[act[na]] > q) ++na;
    if (h->adv_time == 2) {  // SSPRK(3,3) (src/hipft.f90:7486-7505)
      TRY(advection_stage_ragged(h, f, nullptr, A, AdvCombine{0, 0.0, 0.0, 1.0}, na));
      TRY(advection_stage_ragged(h, A, f, B, AdvCombine{1, c_three_quarter, c_quarter, c_quarter}, na));
      TRY(advection_stage_ragged(h, B, f, f, AdvCombine{1, c_third, c_two_third, c_two_third}, na));
    } else {  // SSPRK(4,3) (src/hipft.f90:7552-7574)
      TRY(advection_stage_ragged(h, f, nullptr, A, AdvCombine{0, 0.0, 0.0, 0.5}, na));
      TRY(advection_stage_ragged(h, A, nullptr, B, AdvCombine{0, 0.0, 0.0, 0.5}, na));
      TRY(advection_stage_ragged(h, B, f, A, AdvCombine{1, c_two_third, c_third, c_sixth}, na));
      TRY(advection_stage_ragged(h, A, nullptr, f, AdvCombine{0, 0.0, 0.0, 0.5}, na));
    }
  }
  return HIPFT_OK;
}

extern "C" int hipft_gpu_set_ragged(hipft_gpu *h, int on) {
  if (!h) return HIPFT_EINVAL;
  CK(h, cudaSetDevice(h->dev));
  if (!on) {
    h->ragged = false;
    return HIPFT_OK;
  }
  if (h->red_cb) return fail(h, HIPFT_ESTATE, "set_ragged: a ragged batch has no shared schedule to reduce over ranks");
  if (h->P.advance_diffusion && (h->DC.grid || h->P.diffusion_num_method == 1))
    return fail(h, HIPFT_EINVAL, "set_ragged: needs RKG2 or RKL2 with per-realization constant diffusion coefficients");
  if (h->P.advance_flow && h->adv_time == 1)
    return fail(h, HIPFT_EINVAL, "set_ragged: needs SSPRK(3,3) or SSPRK(4,3) advection");
  const int nr = h->nr;
  if (!h->d_rbits) {
    TRY(dalloc(h, &h->d_rbits, 2 * (size_t)nr));
    TRY(dalloc(h, &h->d_rlist_dif, (size_t)nr));
    TRY(dalloc(h, &h->d_rlist_adv, (size_t)nr));
    TRY(dalloc(h, &h->d_r1coef, (size_t)nr));
    TRY(dalloc(h, &h->d_rdt, (size_t)nr));
  }
  if (h->P.advance_diffusion) TRY(ragged_gershgorin(h));
  h->r_dtmax_valid = false;
  h->r_s.assign(nr, 0);
  h->r_cycles.assign(nr, 0);
  h->r_substeps.assign(nr, 1);
  h->ragged = true;
  return HIPFT_OK;
}

extern "C" int hipft_gpu_flow_dtmax_each(hipft_gpu *h, double *dtmax) {
  if (!h || !dtmax) return HIPFT_EINVAL;
  if (!h->P.advance_flow) return fail(h, HIPFT_ESTATE, "flow_dtmax_each: advance_flow is off");
  CK(h, cudaSetDevice(h->dev));
  if (!h->d_rbits) {
    TRY(dalloc(h, &h->d_rbits, 2 * (size_t)h->nr));
    TRY(dalloc(h, &h->d_rlist_dif, (size_t)h->nr));
    TRY(dalloc(h, &h->d_rlist_adv, (size_t)h->nr));
    TRY(dalloc(h, &h->d_r1coef, (size_t)h->nr));
    TRY(dalloc(h, &h->d_rdt, (size_t)h->nr));
  }
  h->r_dtmax_valid = false;
  TRY(ragged_dtmax(h));
  std::copy(h->r_dtmax.begin(), h->r_dtmax.end(), dtmax);
  return HIPFT_OK;
}

extern "C" int hipft_gpu_ragged_schedule(hipft_gpu *h, int64_t *sts_s, int64_t *subcycles, int64_t *adv_substeps,
                                         double *dt_euler) {
  if (!h) return HIPFT_EINVAL;
  if (!h->ragged) return fail(h, HIPFT_ESTATE, "ragged_schedule: the handle is not in ragged mode");
  if (h->graph_on && h->GA.st) {
    // the device's record of the last graph-run step
    const int nr = h->nr;
    std::vector<long long> s(nr);
    std::vector<int> c(nr), q(nr);
    CK(h, cudaMemcpyAsync(s.data(), h->GA.s_last, sizeof(long long) * nr, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaMemcpyAsync(c.data(), h->GA.cycles_i, sizeof(int) * nr, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaMemcpyAsync(q.data(), h->GA.nsub_i, sizeof(int) * nr, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    for (int i = 0; i < nr; ++i) {
      h->r_s[i] = s[i];
      h->r_cycles[i] = c[i];
      h->r_substeps[i] = q[i] > 0 ? q[i] : 1;
    }
  }
  for (int i = 0; i < h->nr; ++i) {
    if (sts_s) sts_s[i] = h->r_s.empty() ? 0 : h->r_s[i];
    if (subcycles) subcycles[i] = h->r_cycles.empty() ? 0 : h->r_cycles[i];
    if (adv_substeps) adv_substeps[i] = h->r_substeps.empty() ? 1 : h->r_substeps[i];
    if (dt_euler) dt_euler[i] = h->r_dt_euler.empty() ? 0.0 : h->r_dt_euler[i];
  }
  return HIPFT_OK;
}

extern "C" int hipft_gpu_diffusion_step(hipft_gpu *h, double dtl, hipft_cycle_cb cb, void *user,
                                        hipft_diffusion_info *info) {
  if (!h) return HIPFT_EINVAL;
  if (!h->field_set) return fail(h, HIPFT_ESTATE, "diffusion_step before set_field");
  if (!h->P.advance_diffusion) return fail(h, HIPFT_ESTATE, "diffusion_step: advance_diffusion is off");
  CK(h, cudaSetDevice(h->dev));
  if (h->ragged) return ragged_diffusion_step(h, dtl, info);
  // the ring sums of the step's input are summed afresh (as in ragged
  // batches and in a graph-run step), also when the previous step left the
  // fused kernels' ring sums of the same field
  h->dring_valid = false;
  const int max_sc = 60;
  int64_t stages0 = h->cell_updates;
  int i = 1;
  bool done = false;
  double time_stepped = 0.0;
  double dtl2 = h->auto_sc ? 0.0 : dtl / (double)h->P.diffusion_subcycles;
  for (;;) {
    if (h->auto_sc) TRY(ptl_dt(h, &dtl2));
    if (h->auto_sc && time_stepped + dtl2 >= dtl) {
      dtl2 = dtl - time_stepped;
      done = true;
    }
    if (h->auto_sc && i == max_sc - 1) {
      dtl2 = dtl - time_stepped;
      done = true;
    }
    if (h->auto_sc && h->P.verbose > 0) h->subcycles_state = (int64_t)std::ceil((dtl - time_stepped) / dtl2);
    if (h->P.diffusion_num_method == 1) TRY(euler_steps(h, dtl2));
    else TRY(sts_super_step(h, dtl2));
    time_stepped = time_stepped + dtl2;
    if (cb) {
      CK(h, cudaStreamSynchronize(h->stream));
      cb(user, i, time_stepped, dtl2, h->P.diffusion_num_method == 1 ? h->n_euler : h->sts_s, h->subcycles_state);
    }
    if (!h->auto_sc && i == h->P.diffusion_subcycles) done = true;
    if (done) break;
    i = i + 1;
  }
  if (h->auto_sc) h->subcycles_state = i;
  TRY(check_wait_flag(h, "diffusion_step: a bounded wait for staged tiles gave up"));
  if (info) {
    info->dtime_diffusion_euler = h->dt_euler;
    info->sts_s = (h->P.diffusion_num_method == 1) ? h->n_euler : h->sts_s;
    info->subcycles = h->subcycles_state;
    int64_t cells = (int64_t)h->ntm * (h->npm - 2) * h->nr;
    info->total_stages = cells ? (h->cell_updates - stages0) / cells : 0;
  }
  return HIPFT_OK;
}

// ================================================================ graph mode
// hipft_gpu_set_graph: every flux_transport_step runs as one launch of a
// captured CUDA graph.  The schedule decisions that the host-driven step
// makes between launches (PTL subcycles, stage counts, advection substeps)
// are made on the device by the schedule kernels of graph_step.cuh, and the
// loops they size are WHILE nodes.  The capture fixes the buffers: the field
// stays in buffer g_cur; stage outputs rotate through four others with fixed
// roles (an even stage pair reads (R0, R3) and writes (R1, R2), an odd one
// reads (R2, R1) and writes (R3, R0)); each realization's result is gathered
// back into the field buffer after its super-step.

static void graph_release(hipft_gpu *h) {
  if (h->g_exec) cudaGraphExecDestroy(h->g_exec);
  if (h->g_graph) cudaGraphDestroy(h->g_graph);
  h->g_exec = nullptr;
  h->g_graph = nullptr;
}

template <typename T>
static void dfree(hipft_gpu *h, T *&p) {
  if (p) {
    cudaFree((void *)p);
    h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void *)p), h->allocs.end());
  }
  p = nullptr;
}

// Schedule arrays for the handle's realizations and `paircap` stage pairs.
static int graph_alloc(hipft_gpu *h, int paircap) {
  GArrays &g = h->GA;
  const size_t nr = (size_t)h->nr;
  if (!g.st) {
    double *de = nullptr, *dm = nullptr;
    TRY(dalloc(h, &g.st, 1));
    TRY(dalloc(h, &g.ts, nr));
    TRY(dalloc(h, &g.d, nr));
    TRY(dalloc(h, &de, nr));
    TRY(dalloc(h, &dm, nr));
    TRY(dalloc(h, &g.rdt, nr));
    TRY(dalloc(h, &g.act, nr));
    TRY(dalloc(h, &g.fin, nr));
    TRY(dalloc(h, &g.rl_ptl, nr));
    TRY(dalloc(h, &g.rl_dif, nr));
    TRY(dalloc(h, &g.rl_adv, nr));
    TRY(dalloc(h, &g.rl_adv_all, nr));
    TRY(dalloc(h, &g.nsub_i, nr));
    TRY(dalloc(h, &g.cycles_i, nr));
    TRY(dalloc(h, &g.s_i, nr));
    TRY(dalloc(h, &g.s_last, nr));
    TRY(dalloc(h, &g.c1, nr));
    TRY(dalloc(h, &g.bits, 2 * nr));
    g.dt_euler = de;
    g.dtmax = dm;
    CK(h, cudaMemsetAsync(g.st, 0, sizeof(GState), h->stream));
    CK(h, cudaMemsetAsync(g.s_last, 0, nr * sizeof(long long), h->stream));
    CK(h, cudaMemsetAsync(g.cycles_i, 0, nr * sizeof(int), h->stream));
    CK(h, cudaMemsetAsync(g.nsub_i, 0, nr * sizeof(int), h->stream));
    g.nr = h->nr;
  }
  if (paircap > g.paircap) {
    dfree(h, g.nactp);
    dfree(h, g.rc);
    TRY(dalloc(h, &g.nactp, (size_t)paircap));
    TRY(dalloc(h, &g.rc, (size_t)paircap * nr * 2));
    g.paircap = paircap;
  }
  return HIPFT_OK;
}

// Stage pairs (with the pair loop's slack) a step of length dt can need: one
// subcycle over the whole step at the smallest Euler limit bounds every
// realization's stage count.
static int graph_pairs_needed(const hipft_gpu *h, double dt) {
  if (!h->P.advance_diffusion) return kGUnrollMax;
  double dte = h->dt_euler;
  if (h->ragged)
    for (double v : h->r_dt_euler) dte = std::min(dte, v);
  const int64_t s = sts_count(h->P.diffusion_num_method, dt, dte);
  return (int)((s - 1) / 2) + kGUnrollMax;
}

// Launch parameters a capture bakes in besides the buffers; any change (new
// flows, ragged mode, larger tables) means a new capture.
static std::vector<unsigned char> graph_key(const hipft_gpu *h) {
  std::vector<unsigned char> k;
  auto add = [&](const void *p, size_t n) {
    const unsigned char *c = static_cast<const unsigned char *>(p);
    k.insert(k.end(), c, c + n);
  };
  add(&h->FL, sizeof(h->FL));
  add(&h->DC, sizeof(h->DC));
  add(&h->ptab, sizeof(h->ptab));
  const double bc[4] = {h->bc_flow_n, h->bc_flow_s, h->bc_diff_n, h->bc_diff_s};
  add(bc, sizeof(bc));
  const int flags[6] = {h->ragged ? 1 : 0, h->cur, h->GA.paircap, h->g_pdl ? 1 : 0, h->auto_sc ? 1 : 0,
                        (int)h->P.diffusion_subcycles};
  add(flags, sizeof(flags));
  return k;
}

// A conditional handle on the graph that stream s is capturing into.
static cudaError_t g_handle(cudaStream_t s, cudaGraphConditionalHandle *hc) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg = nullptr;
  cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, nullptr, nullptr);
  if (e != cudaSuccess) return e;
  if (cs != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureInvalidated;
  return cudaGraphConditionalHandleCreate(hc, cg, 0, 0);
}

// A WHILE node on handle hc at stream s's capture point; returns its body.
static cudaError_t g_while(cudaStream_t s, cudaGraphConditionalHandle hc, cudaGraph_t *body) {
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd);
  if (e != cudaSuccess) return e;
  if (cs != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureInvalidated;
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = hc;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  e = cudaGraphAddNode(&node, cg, deps, nd, &p);
  if (e != cudaSuccess) return e;
  *body = p.conditional.phGraph_out[0];
  return cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
}

// Captures the split step: the host-driven step's kernels, grids and
// argument values (ragged or plain), with realization lists, coefficients
// and substep lengths read from the schedule arrays.
static int graph_capture(hipft_gpu *h) {
  graph_release(h);
  for (auto &s : h->g_side)
    if (!s) CK(h, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  const int nr = h->nr;
  GArrays &G = h->GA;
  G.method = h->P.diffusion_num_method;
  G.auto_sc = h->auto_sc ? 1 : 0;
  G.subcycles = (int)h->P.diffusion_subcycles;
  G.ragged = h->ragged ? 1 : 0;
  G.strang = h->P.strang_splitting ? 1 : 0;
  G.nadv = (h->adv_time == 1) ? 1 : ((h->adv_time == 2) ? 3 : 4);
  {
    const char *e = std::getenv("HIPFT_GRAPH_UNROLL");
    const int u = e ? std::atoi(e) : kGUnrollMax;  // each iteration boundary costs ~11 us (tick, node relaunch)
    G.unroll = std::max(2, std::min(kGUnrollMax, u - u % 2));
  }
  G.ring0 = h->d_ringbuf[0];
  G.ring1 = h->d_ringbuf[1];
  const GArrays g = G;
  h->g_cur = h->cur;
  double *F = h->buf[h->cur];
  double *Bd = h->buf[scratch(h, 0)];  // dty0
  double *R[4] = {h->buf[scratch(h, 1)], h->buf[scratch(h, 2)], h->buf[scratch(h, 3)], h->buf[scratch(h, 4)]};
  const Mesh M = h->M;
  const int64_t nfield = (int64_t)h->fieldn;
  const int cblocks = 4 * h->num_sms;
  cudaError_t first = cudaSuccess;
  auto ok = [&](cudaError_t e) {
    if (e != cudaSuccess && first == cudaSuccess) first = e;
  };
  auto peek = [&]() { ok(cudaPeekAtLastError()); };
  // captured on a stream of its own (the handle's stream may be the legacy
  // default stream, which cannot capture); launched on the handle's stream
  cudaStream_t s0 = h->g_side[2], s1 = h->g_side[0], s2 = h->g_side[1];
  // the body of a WHILE node at stream s's capture point, captured on stream b
  auto begin_body = [&](cudaStream_t s, cudaGraphConditionalHandle hc, cudaStream_t b) {
    cudaGraph_t body = nullptr;
    ok(g_while(s, hc, &body));
    if (first == cudaSuccess)
      ok(cudaStreamBeginCaptureToGraph(b, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  };
  auto end_body = [&](cudaStream_t b) {
    cudaGraph_t gdone = nullptr;
    ok(cudaStreamEndCapture(b, &gdone));
  };

  // ---- advection_step over frac * dt (src/hipft.f90:4509-4549)
  auto adv_stage = [&](cudaStream_t s, const double *x, const double *f0, double *out, AdvCombine cb) {
    k_ring_advection<<<nr, 256, 0, s>>>(M, h->FL, x, h->d_ring);
    peek();
    launch_adv_stage(h, M, s, (unsigned)nr, x, f0, out, cb, g.rl_adv, g.rdt);
    peek();
  };
  auto advection = [&](double frac) {
    cudaGraphConditionalHandle hc{};
    ok(g_handle(s0, &hc));
    if (first != cudaSuccess) return;
    k_g_adv_plan<<<1, 256, 0, s0>>>(g, frac, hc);
    peek();
    begin_body(s0, hc, s1);
    if (first != cudaSuccess) return;
    double *A = R[0], *B = R[1];
    if (h->adv_time == 1) {  // FE (src/hipft.f90:7440-7444), then back into the field
      adv_stage(s1, F, nullptr, A, AdvCombine{0, 0.0, 0.0, 1.0});
      k_g_copy<<<cblocks, 256, 0, s1>>>(F, A, nfield);
      peek();
    } else if (h->adv_time == 2) {  // SSPRK(3,3) (src/hipft.f90:7486-7505)
      adv_stage(s1, F, nullptr, A, AdvCombine{0, 0.0, 0.0, 1.0});
      adv_stage(s1, A, F, B, AdvCombine{1, c_three_quarter, c_quarter, c_quarter});
      adv_stage(s1, B, F, F, AdvCombine{1, c_third, c_two_third, c_two_third});
    } else {  // SSPRK(4,3) (src/hipft.f90:7552-7574)
      adv_stage(s1, F, nullptr, A, AdvCombine{0, 0.0, 0.0, 0.5});
      adv_stage(s1, A, nullptr, B, AdvCombine{0, 0.0, 0.0, 0.5});
      adv_stage(s1, B, F, A, AdvCombine{1, c_two_third, c_third, c_sixth});
      adv_stage(s1, A, nullptr, F, AdvCombine{0, 0.0, 0.0, 0.5});
    }
    k_g_adv_tick<<<1, 256, 0, s1>>>(g, (h->adv_time == 1) ? 4 : 2 * g.nadv + 1, hc);
    peek();
    end_body(s1);
  };

  // ---- one stage pair of the loop body: pair q of the iteration (q = 0..3)
  const int nkt = (h->npm - 2 + kWK - 1) / kWK;
  auto pair = [&](cudaStream_t s, int q, bool overlap) {
    const bool even = (q % 2) == 0;
    const double *ykm1 = even ? R[0] : R[2], *ykm2 = even ? R[3] : R[1];
    double *ok_ = even ? R[1] : R[3], *ok1 = even ? R[2] : R[0];
    const double *rin = even ? g.ring1 : g.ring0;
    double *rout = even ? g.ring0 : g.ring1;
    RingOut ro{rout, h->d_rpart, h->d_rcount, nkt};
    PairArgs pa{StageCoef{}, StageCoef{}, h->d_err, g.rl_dif, g.rc};
    pa.dctr = &g.st->pctr;
    pa.doff = q;
    pa.dnact = g.nactp;
    pa.dstride = 2 * nr;
    PairTables pt = h->ptab;
    pt.ntiles = pt.nb * pt.nkt * nr;
    const int grid = std::min(pt.ntiles, 2 * h->num_sms);
    const WsMaps tmaps = ws_maps(h, ykm1, ykm2, F, Bd);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kWThreads);
    cfg.dynamicSmemBytes = kWSmem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = (h->g_pdl && overlap) ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    ok(cudaLaunchKernelEx(&cfg, k_sts_pair_ws<true, false, true>, M, (const double *)h->DC.dfac, ykm1, ykm2,
                          (const double *)F, (const double *)Bd, ok_, ok1, rin, h->bc_diff_n, h->bc_diff_s, pa, ro,
                          pt, tmaps));
    const dim3 pg((unsigned)nr, (unsigned)h->pole_nch);
    k_pair_poles<<<pg, kPoleThreads, 0, s>>>(M, h->DC.dfac, ykm1, ykm2, F, Bd, ok1, rin, h->bc_diff_n,
                                             h->bc_diff_s, pa, ro, h->pole);
    peek();
  };

  // ---- diffusion_step over dt (src/hipft.f90:4551-4695)
  auto diffusion = [&]() {
    cudaGraphConditionalHandle hsub{};
    ok(g_handle(s0, &hsub));
    if (first != cudaSuccess) return;
    k_g_dif_begin<<<1, 256, 0, s0>>>(g, h->ragged ? 0 : 1, hsub);
    peek();
    // plain mode: the ring of the field once; later subcycles reuse the ring
    // sums the last stage pair left (the gather moves them to ring0)
    if (!h->ragged) {
      k_ring_diffusion<<<nr, 256, 0, s0>>>(M, h->DC, F, g.ring0);
      peek();
    }
    begin_body(s0, hsub, s1);
    if (first != cudaSuccess) return;
    int body_kernels = 1;  // the subcycle tick itself
    if (h->ragged) {
      k_ring_diffusion<<<nr, 256, 0, s1>>>(M, h->DC, F, g.ring0);
      peek();
      ++body_kernels;
    }
    const dim3 blk(32, 8);
    const dim3 grd((unsigned)((h->ntm + 31) / 32), (unsigned)((h->npm - 2 + 7) / 8), (unsigned)nr);
    if (h->auto_sc) {  // PTL (src/hipft.f90:5042-5161) of the active realizations
      k_g_ptl_reset<<<1, 256, 0, s1>>>(g);
      peek();
      const int pr = h->ragged ? 1 : 0;
      unsigned long long *bmax = g.bits, *bmin = g.bits + (h->ragged ? nr : 1);
      k_diffusion_stage<MODE_AX><<<grd, blk, 0, s1>>>(M, h->DC, F, nullptr, nullptr, nullptr, R[0], nullptr, g.ring0,
                                                      h->bc_diff_n, h->bc_diff_s, StageCoef{}, bmax, g.rl_ptl, pr);
      peek();
      k_ptl<<<grd, blk, 0, s1>>>(M, F, R[0], bmax, bmin, g.rl_ptl, pr);
      peek();
      body_kernels += 2;
    }
    cudaGraphConditionalHandle hpair{};
    ok(g_handle(s1, &hpair));
    if (first != cudaSuccess) return;
    k_g_plan<<<1, 256, 0, s1>>>(g, hpair);
    peek();
    const int64_t ncoef = (int64_t)g.paircap * nr;
    k_g_coefs<<<(unsigned)((ncoef + 255) / 256), 256, 0, s1>>>(g);
    peek();
    // stage 1 (src/hipft.f90:5211-5218): Y_1 into R0, dty0; Y_0 = u0 into R3
    {
      const int nkb = (h->npm - 2 + kKPT3 - 1) / kKPT3;
      RingOut ro{g.ring1, h->d_rpart, h->d_rcount, nkb};
      const int jshift = (h->ntm % 2 == 1 && ((h->ntm - 1) / 2) % 32 == 0) ? 1 : 0;
      const int nthr = (h->ntm + 2 * jshift + 1) / 2;
      const dim3 g1((unsigned)((nthr + 127) / 128), (unsigned)nkb, (unsigned)nr);
      k_sts_stage_v3<MODE_STS1, kKPT3><<<g1, 128, 0, s1>>>(M, h->DC.dfac, F, nullptr, nullptr, nullptr, R[0], Bd,
                                                           g.ring0, h->bc_diff_n, h->bc_diff_s, StageCoef{}, ro,
                                                           jshift, g.rl_dif, g.c1);
      peek();
      k_g_copy<<<cblocks, 256, 0, s1>>>(R[3], F, nfield);
      peek();
      body_kernels += 2;
    }
    begin_body(s1, hpair, s2);
    if (first != cudaSuccess) return;
    for (int q = 0; q < g.unroll; ++q) pair(s2, q, q > 0);
    k_g_pair_tick<<<1, 1, 0, s2>>>(g, hpair);
    peek();
    end_body(s2);
    // the result of each realization back into the field: Y_s is in R2 after
    // an even last pair, in R0 after an odd one
    k_g_gather<<<dim3((unsigned)nr, 64u), 256, 0, s1>>>(g, M, F, R[2], R[0]);
    peek();
    k_g_sub_tick<<<1, 256, 0, s1>>>(g, body_kernels, hsub);
    peek();
    end_body(s1);
  };

  ok(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
  if (first == cudaSuccess) {
    k_g_step_begin<<<1, 32, 0, s0>>>(g);
    peek();
    const double fa = h->P.strang_splitting ? 0.5 : 1.0;
    if (h->P.advance_flow) advection(fa);
    if (h->P.advance_diffusion && first == cudaSuccess) diffusion();
    if (h->P.strang_splitting && h->P.advance_flow && first == cudaSuccess) advection(0.5);
  }
  // a failed body capture may leave a side stream capturing
  for (cudaStream_t s : {s1, s2}) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
      cudaGraph_t gd = nullptr;
      cudaStreamEndCapture(s, &gd);
      if (first == cudaSuccess) first = cudaErrorStreamCaptureInvalidated;
    }
  }
  cudaGraph_t graph = nullptr;
  cudaError_t ee = cudaStreamEndCapture(s0, &graph);
  if (first == cudaSuccess) first = ee;
  if (first == cudaSuccess) first = cudaGraphInstantiate(&h->g_exec, graph, 0);
  if (first != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    h->g_exec = nullptr;
    cudaGetLastError();
    return fail(h, HIPFT_ECUDA, "graph capture of the step: %s", cudaGetErrorString(first));
  }
  h->g_graph = graph;
  h->g_key = graph_key(h);
  return HIPFT_OK;
}

// Statistics of the last graph-run step into the handle's counters.
static int graph_collect(hipft_gpu *h) {
  if (h->g_stats_valid) return HIPFT_OK;
  CK(h, cudaMemcpyAsync(h->h_pin, h->GA.st, sizeof(GState), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  std::memcpy(&h->g_last, h->h_pin, sizeof(GState));
  h->g_stats_valid = true;
  const GState &st = h->g_last;
  const int64_t cells = (int64_t)h->ntm * (h->npm - 2);
  h->cell_updates += cells * (st.stage_sum + st.adv_slices);
  h->rkg2_cell_stages += cells * st.rkg2_sum;
  h->launches += st.kernels;
  if (h->P.advance_diffusion) {
    h->sts_s = st.smax;
    h->subcycles_state = st.cycles;
  }
  if (st.err == 1) return fail(h, HIPFT_ECUDA, "graph-run step: the stage tables were too small");
  if (st.err == 2) return fail(h, HIPFT_ECUDA, "graph-run step: a loop ran past its iteration limit");
  return HIPFT_OK;
}

// One split step as one graph launch.
static int graph_step(hipft_gpu *h, double dt, hipft_diffusion_info *info) {
  TRY(graph_collect(h));
  if (h->P.advance_diffusion) TRY(ensure_pair_plan(h));
  const int need = graph_pairs_needed(h, dt);
  const bool grow = need > h->GA.paircap;
  TRY(graph_alloc(h, grow ? need + need / 4 : need));
  if (h->cur != h->g_cur && h->g_cur >= 0) {
    // another entry point left the field elsewhere: back into the captured buffer
    CK(h, cudaMemcpyAsync(h->buf[h->g_cur], h->buf[h->cur], h->fieldn * sizeof(double), cudaMemcpyDeviceToDevice,
                          h->stream));
    h->cur = h->g_cur;
  }
  // per-realization limits (ragged: each its own; plain: the shared ones)
  const int nr = h->nr;
  std::vector<double> de(nr, h->dt_euler), dm(nr, 0.0);
  if (h->ragged) {
    if (h->P.advance_diffusion) de = h->r_dt_euler;
    if (h->P.advance_flow) {
      TRY(ragged_dtmax(h));
      dm = h->r_dtmax;
    }
  }
  CK(h, cudaMemcpyAsync(const_cast<double *>(h->GA.dt_euler), de.data(), sizeof(double) * nr,
                        cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(const_cast<double *>(h->GA.dtmax), dm.data(), sizeof(double) * nr, cudaMemcpyHostToDevice,
                        h->stream));
  if (!h->g_exec || graph_key(h) != h->g_key) TRY(graph_capture(h));
  CK(h, cudaMemcpyAsync(&h->GA.st->dt, &dt, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaGraphLaunch(h->g_exec, h->stream));
  h->g_stats_valid = false;
  h->dring_valid = false;
  h->ring_cur = 0;
  if (info) {
    TRY(graph_collect(h));
    TRY(check_wait_flag(h, "graph-run step: a bounded wait for staged tiles gave up"));
    info->dtime_diffusion_euler = h->dt_euler;
    if (h->ragged && !h->r_dt_euler.empty())
      info->dtime_diffusion_euler = *std::min_element(h->r_dt_euler.begin(), h->r_dt_euler.end());
    info->sts_s = h->g_last.smax;
    info->subcycles = h->g_last.cycles;
    info->total_stages = nr ? h->g_last.stage_sum / nr : 0;
  }
  return HIPFT_OK;
}

extern "C" int hipft_gpu_set_graph(hipft_gpu *h, int on) {
  if (!h) return HIPFT_EINVAL;
  CK(h, cudaSetDevice(h->dev));
  if (!on) {
    TRY(graph_collect(h));
    h->graph_on = false;
    graph_release(h);
    return HIPFT_OK;
  }
  if (h->red_cb) return fail(h, HIPFT_ESTATE, "set_graph: a step shared over ranks reduces on the host");
  if (h->P.advance_source) return fail(h, HIPFT_EINVAL, "set_graph: sources are not part of a graph-run step");
  if (h->P.advance_diffusion && (h->DC.grid || h->P.diffusion_num_method == 1))
    return fail(h, HIPFT_EINVAL, "set_graph: needs RKG2 or RKL2 with per-realization constant diffusion coefficients");
  if (h->nbuf < 6) return fail(h, HIPFT_ESTATE, "set_graph: needs six field buffers");
  const char *e = std::getenv("HIPFT_GRAPH_PDL");
  h->g_pdl = ws_pdl() && !(e && std::atoi(e) == 0);
  h->graph_on = true;
  return HIPFT_OK;
}

extern "C" int hipft_gpu_flux_transport_step(hipft_gpu *h, double dt, hipft_cycle_cb cb, void *user,
                                             hipft_diffusion_info *info) {
  if (!h) return HIPFT_EINVAL;
  if (h->graph_on) {
    if (cb) return fail(h, HIPFT_ESTATE, "flux_transport_step: subcycle callbacks need the host-driven step");
    if (!h->field_set) return fail(h, HIPFT_ESTATE, "flux_transport_step before set_field");
    CK(h, cudaSetDevice(h->dev));
    return graph_step(h, dt, info);
  }
  if (h->P.strang_splitting) {
    double half = dt * 0.5;
    if (h->P.advance_source) TRY(hipft_gpu_source_step(h, half));
    if (h->P.advance_flow) TRY(hipft_gpu_advection_step(h, half));
    if (h->P.advance_diffusion) TRY(hipft_gpu_diffusion_step(h, dt, cb, user, info));
    if (h->P.advance_flow) TRY(hipft_gpu_advection_step(h, half));
    if (h->P.advance_source) TRY(hipft_gpu_source_step(h, half));
  } else {
    if (h->P.advance_flow) TRY(hipft_gpu_advection_step(h, dt));
    if (h->P.advance_diffusion) TRY(hipft_gpu_diffusion_step(h, dt, cb, user, info));
    if (h->P.advance_source) TRY(hipft_gpu_source_step(h, dt));
  }
  return HIPFT_OK;
}

// ----------------------------------------------------------------- sources
static int ensure_sources(hipft_gpu *h) {
  if (h->d_src) return HIPFT_OK;
  TRY(dalloc(h, &h->d_src, h->fieldn));
  CK(h, cudaMemsetAsync(h->d_src, 0, h->fieldn * sizeof(double), h->stream));
  return HIPFT_OK;
}

extern "C" int hipft_gpu_set_source_file(hipft_gpu *h, const double *data_tp) {
  if (!h || !data_tp) return HIPFT_EINVAL;
  CK(h, cudaSetDevice(h->dev));
  TRY(ensure_sources(h));
  if (!h->d_src_file) TRY(dalloc(h, &h->d_src_file, (size_t)h->ldt * h->npm));
  CK(h, cudaMemcpy2DAsync(h->d_src_file, (size_t)h->ldt * sizeof(double), data_tp, (size_t)h->ntm * sizeof(double),
                          (size_t)h->ntm * sizeof(double), (size_t)h->npm, cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return HIPFT_OK;
}

static int balance_buffer(hipft_gpu *h, double *a);

extern "C" int hipft_gpu_set_rfe_frame(hipft_gpu *h, int slot, int model, const double *rnd_tp, const double *uf) {
  if (!h || !rnd_tp || !uf || slot < 0 || slot > 1 || model < 1 || model > 2) return HIPFT_EINVAL;
  CK(h, cudaSetDevice(h->dev));
  TRY(ensure_sources(h));
  const int ntm = h->ntm, npm = h->npm, nr = h->nr;
  if (!h->d_rfe[slot]) {
    TRY(dalloc(h, &h->d_rfe[slot], h->fieldn));
    CK(h, cudaMemsetAsync(h->d_rfe[slot], 0, h->fieldn * sizeof(double), h->stream));
  }
  if (!h->d_rnd) {
    TRY(dalloc(h, &h->d_rnd, (size_t)ntm * npm));
    TRY(dalloc(h, &h->d_rfe_aux, (size_t)(nr + 1) + (ntm + 1)));
  }
  // da_ti per theta row, model 1 (src/hipft.f90:8840-8853)
  std::vector<double> aux((size_t)(nr + 1) + (ntm + 1), 0.0);
  for (int i = 1; i <= nr; ++i) aux[i] = uf[i - 1];
  double *dati = aux.data() + (nr + 1);
  for (int j = 1; j <= ntm; ++j) {
    if (j == 1 || j == ntm) {
      const double tav = (j == 1) ? 0.5 * (h->t[1] + h->t[2]) : 0.5 * (h->t[ntm] + h->t[ntm - 1]);
      const double sn_t = std::sin(tav), d_t = (j == 1) ? h->dth[2] : h->dth[ntm];
      dati[j] = 1.0 / (0.25 * sn_t * d_t);
    } else {
      dati[j] = h->st_i[j] * h->dt_i[j];
    }
  }
  TRY(upload(h, h->d_rfe_aux, aux));
  CK(h, cudaMemcpyAsync(h->d_rnd, rnd_tp, (size_t)ntm * npm * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  double *fr = h->d_rfe[slot];
  dim3 blk(32, 8), grd((unsigned)((ntm + 31) / 32), (unsigned)((npm - 2 + 7) / 8), (unsigned)nr);
  k_rfe_frame<<<grd, blk, 0, h->stream>>>(h->M, model, h->d_rnd, h->d_rfe_aux, h->d_rfe_aux + (nr + 1), fr);
  LAUNCHED(h);
  k_seam<<<dim3((unsigned)((ntm + 127) / 128), (unsigned)nr), 128, 0, h->stream>>>(h->M, ntm, h->ldt, fr);
  LAUNCHED(h);
  k_rfe_poles<<<nr, 128, 0, h->stream>>>(h->M, fr);
  LAUNCHED(h);
  TRY(balance_buffer(h, fr));
  return HIPFT_OK;
}

extern "C" int hipft_gpu_update_source(hipft_gpu *h, int use_file, int use_rfe, int slot1, int slot2,
                                       double alpha) {
  if (!h || slot1 < 0 || slot1 > 1 || slot2 < 0 || slot2 > 1) return HIPFT_EINVAL;
  if ((use_file && !h->d_src_file) || (use_rfe && (!h->d_rfe[slot1] || !h->d_rfe[slot2])))
    return fail(h, HIPFT_ESTATE, "update_source: source file or RFE frame not set");
  CK(h, cudaSetDevice(h->dev));
  TRY(ensure_sources(h));
  dim3 blk(32, 8), grd((unsigned)((h->ntm + 31) / 32), (unsigned)((h->npm + 7) / 8), (unsigned)h->nr);
  k_source_blend<<<grd, blk, 0, h->stream>>>(h->M, use_file ? h->d_src_file : nullptr,
                                             use_rfe ? h->d_rfe[slot1] : nullptr, use_rfe ? h->d_rfe[slot2] : nullptr,
                                             alpha, h->d_src);
  LAUNCHED(h);
  h->src_set = true;
  return HIPFT_OK;
}

extern "C" int hipft_gpu_source_step(hipft_gpu *h, double dt) {
  if (!h) return HIPFT_EINVAL;
  if (!h->field_set) return fail(h, HIPFT_ESTATE, "source_step before set_field");
  if (!h->src_set) return fail(h, HIPFT_ESTATE, "source_step before update_source");
  CK(h, cudaSetDevice(h->dev));
  dim3 blk(32, 8), grd((unsigned)((h->ntm + 31) / 32), (unsigned)((h->npm + 7) / 8), (unsigned)h->nr);
  k_source_step<<<grd, blk, 0, h->stream>>>(h->M, h->d_src, dt, h->buf[h->cur]);
  LAUNCHED(h);
  h->dring_valid = false;
  return HIPFT_OK;
}

// ------------------------------------------------------------ assimilation
// Uploads one observed map and the per-realization blend options
// (assimilate_new_data's inputs, src/hipft.f90:4083-4146; lat-limit indices
// of load_data_assimilation, 4066-4079) and fills the kernels' arguments.
static int da_args(hipft_gpu *h, const double *data3_pt, const hipft_da_opts *o, DAArgs &a) {
  int ntm = h->ntm, npm1 = h->npm1, nr = h->nr;
  size_t nd = (size_t)npm1 * ntm * 3;
  if (!h->d_da) {
    TRY(dalloc(h, &h->d_da, nd));
    TRY(dalloc(h, &h->d_daopt, 3 * (size_t)(nr + 1)));
    TRY(dalloc(h, &h->d_tidx, 2 * (size_t)(nr + 1)));
  }
  CK(h, cudaMemcpyAsync(h->d_da, data3_pt, nd * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  std::vector<double> opt(3 * (size_t)(nr + 1), 0.0);
  std::vector<int> tidx(2 * (size_t)(nr + 1), -1);
  for (int i = 1; i <= nr; ++i) {
    opt[i] = o->mu_power ? o->mu_power[i - 1] : 0.0;
    opt[(nr + 1) + i] = o->mu_limit ? o->mu_limit[i - 1] : 0.0;
    opt[2 * (nr + 1) + i] = o->lat_limit[i - 1];
    int t0 = -1, t1 = -1;
    for (int j = 1; j <= ntm; ++j)
      if (h->t[j] >= o->lat_limit[i - 1] * c_d2r && t0 == -1) t0 = j;
    for (int j = ntm; j >= 1; --j)
      if (h->t[j] <= (c_pi - o->lat_limit[i - 1] * c_d2r) && t1 == -1) t1 = j;
    tidx[i] = t0;
    tidx[(nr + 1) + i] = t1;
  }
  TRY(upload(h, h->d_daopt, opt));
  CK(h, cudaMemcpyAsync(h->d_tidx, tidx.data(), tidx.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  if (o->custom_from_mu && (!o->mu_power || !o->mu_limit))
    return fail(h, HIPFT_EINVAL, "assimilate: custom_from_mu needs mu_power and mu_limit");
  if (o->custom_from_mu) {
    // mu^power weights (src/hipft.f90:4246-4252) on the host, with the C
    // library's pow: the weights then carry the reference's bits, which the
    // 1e-12 field bar needs (a 2-ulp change of every weight moves the
    // assimilated 1024x2048 fields by 1.8e-12 after 2.5 hours).  One plane
    // per distinct (power, limit).
    const size_t slice = (size_t)npm1 * ntm;
    std::vector<std::pair<double, double>> keys;
    std::vector<int> widx((size_t)nr + 1, 0);
    for (int i = 1; i <= nr; ++i) {
      const std::pair<double, double> key(o->mu_power[i - 1], o->mu_limit[i - 1]);
      size_t u = 0;
      while (u < keys.size() && keys[u] != key) ++u;
      if (u == keys.size()) keys.push_back(key);
      widx[i] = (int)u;
    }
    if (keys.size() * slice > h->daw_cap) {
      if (h->d_daw) {
        CK(h, cudaStreamSynchronize(h->stream));
        cudaFree(h->d_daw);
        h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void *)h->d_daw), h->allocs.end());
        h->d_daw = nullptr;
      }
      TRY(dalloc(h, &h->d_daw, keys.size() * slice));
      TRY(dalloc(h, &h->d_dawidx, (size_t)nr + 1));
      h->daw_cap = keys.size() * slice;
    }
    h->h_daw.resize(keys.size() * slice);
    const double *mu = data3_pt + 2 * slice;
    for (size_t u = 0; u < keys.size(); ++u) {
      double *w = h->h_daw.data() + u * slice;
      const double pw = keys[u].first, lim = keys[u].second;
      for (size_t q = 0; q < slice; ++q) w[q] = (mu[q] > lim) ? std::pow(mu[q], pw) : 0.0;
    }
    CK(h, cudaMemcpyAsync(h->d_daw, h->h_daw.data(), keys.size() * slice * sizeof(double), cudaMemcpyHostToDevice,
                          h->stream));
    CK(h, cudaMemcpyAsync(h->d_dawidx, widx.data(), widx.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));  // h_daw and widx are reused by the next call
  }
  a = DAArgs{};
  a.data = h->d_da;
  a.mu_power = h->d_daopt;
  a.mu_limit = h->d_daopt + (nr + 1);
  a.lat_limit = h->d_daopt + 2 * (nr + 1);
  a.tidx0 = h->d_tidx;
  a.tidx1 = h->d_tidx + (nr + 1);
  a.add = o->add;
  a.custom_from_mu = o->custom_from_mu;
  a.mult_fac = o->mult_fac;
  a.wmap = h->d_daw;
  a.widx = h->d_dawidx;
  return HIPFT_OK;
}

extern "C" int hipft_gpu_assimilate(hipft_gpu *h, const double *data3_pt, const hipft_da_opts *o) {
  if (!h || !data3_pt || !o) return HIPFT_EINVAL;
  if (!h->field_set) return fail(h, HIPFT_ESTATE, "assimilate before set_field");
  if (!o->lat_limit || (o->custom_from_mu && (!o->mu_power || !o->mu_limit)))
    return fail(h, HIPFT_EINVAL, "assimilate: missing per-realization options");
  CK(h, cudaSetDevice(h->dev));
  int ntm = h->ntm, npm1 = h->npm1, nr = h->nr;
  DAArgs a;
  TRY(da_args(h, data3_pt, o, a));
  double *f = h->buf[h->cur], *delta = h->buf[scratch(h, 0)];
  dim3 blk(32, 8), grd((unsigned)((ntm + 31) / 32), (unsigned)((npm1 + 31) / 32), (unsigned)nr);
  k_da_delta<<<grd, blk, 0, h->stream>>>(h->M, a, f, delta);
  LAUNCHED(h);
  const double *ratio = nullptr;
  if (o->balance_flux) {
    int cpb = 16, nb = (h->npm - 1 + cpb - 1) / cpb;
    TRY(ensure_part(h, (size_t)nr * nb * 2 + (nr + 1)));
    double *da_t = h->d_anw, *da_p = h->d_anw + 3 * ((size_t)std::max(ntm, h->npm) + 1);
    k_flux_partial<<<dim3((unsigned)nb, (unsigned)nr), 256, 0, h->stream>>>(h->M, da_t, da_p, delta, 1, h->d_part,
                                                                            cpb);
    LAUNCHED(h);
    std::vector<double> part((size_t)nr * nb * 2);
    CK(h, cudaMemcpyAsync(part.data(), h->d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    std::vector<double> r(nr + 1, 1.0);
    for (int i = 0; i < nr; ++i) {
      double fp = 0.0, fm = 0.0;
      for (int b = 0; b < nb; ++b) {
        fp = fp + part[((size_t)i * nb + b) * 2];
        fm = fm + part[((size_t)i * nb + b) * 2 + 1];
      }
      r[i + 1] = (fm + fp == 0.0) ? 1.0 : std::sqrt(std::fabs(fp / fm));
    }
    double *dr = h->d_part + (size_t)nr * nb * 2;
    TRY(upload(h, dr, r));
    ratio = dr;
  }
  dim3 g2((unsigned)((ntm + 31) / 32), (unsigned)((h->npm + 7) / 8), (unsigned)nr);
  k_da_apply<<<g2, blk, 0, h->stream>>>(h->M, delta, f, ratio);
  LAUNCHED(h);
  h->dring_valid = false;
  return HIPFT_OK;
}

// ------------------------------------------------------------ diagnostics
extern "C" int hipft_gpu_set_validation(hipft_gpu *h, int mode, const double *fval_u0_pt, double width,
                                        double vt_const, double vp_omega, double time_start) {
  if (!h || mode < 0 || mode > 2) return HIPFT_EINVAL;
  CK(h, cudaSetDevice(h->dev));
  h->vmode = mode;
  h->vwidth = width;
  h->vt_const = vt_const;
  h->vp_omega = vp_omega;
  h->vtime_start = time_start;
  if (mode == 1) {
    if (!fval_u0_pt) return HIPFT_EINVAL;
    if ((int)h->Dc.size() != h->nr)
      return fail(h, HIPFT_ESTATE, "validation 1 needs the diffusion coefficient constants");
    size_t n = (size_t)h->npm1 * h->ntm * h->nr;
    if (!h->d_fval_u0) TRY(dalloc(h, &h->d_fval_u0, n));
    CK(h, cudaMemcpyAsync(h->d_fval_u0, fval_u0_pt, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  }
  if (mode == 2 && !h->d_vgauss) {
    // theta scale, phi scale and st_i (1-based) for the analytic Gaussians
    size_t L = (size_t)std::max(h->npm, h->nt) + 2;
    std::vector<double> v(3 * L, 0.0);
    for (int j = 1; j <= h->ntm; ++j) {
      v[j] = h->t[j];
      v[2 * L + j] = h->st_i[j];
    }
    for (int k = 1; k <= h->npm; ++k) v[L + k] = h->p[k];
    TRY(dalloc(h, &h->d_vgauss, v.size()));
    TRY(upload(h, h->d_vgauss, v));
  }
  return HIPFT_OK;
}

// Fortran MODULO for reals.
static double fmodulo(double a, double p) { return a - std::floor(a / p) * p; }

extern "C" int hipft_gpu_analysis(hipft_gpu *h, double time, double *hist) {
  if (!h || !hist) return HIPFT_EINVAL;
  if (!h->field_set) return fail(h, HIPFT_ESTATE, "analysis before set_field");
  CK(h, cudaSetDevice(h->dev));
  int ntm = h->ntm, npm = h->npm, nr = h->nr;
  AnalysisArgs a{};
  size_t L = (size_t)std::max(ntm, npm) + 1;
  a.da_t = h->d_anw; a.sn_t = h->d_anw + L; a.cs_t = h->d_anw + 2 * L;
  a.da_p = h->d_anw + 3 * L; a.cs_p = h->d_anw + 4 * L; a.sn_p = h->d_anw + 5 * L;
  a.pn = h->d_masks; a.ps = h->d_masks + (ntm + 1);
  a.vmode = h->vmode;
  if (h->vmode == 1) {
    // fval = fval_u0 * exp(-42 D factor (time - time_start))  (src/hipft.f90:3156-3159)
    std::vector<double> sc(nr + 1, 0.0);
    for (int i = 1; i <= nr; ++i)
      sc[i] = std::exp(-42.0 * h->Dc[i - 1] * h->P.diffusion_coef_factor * (time - h->vtime_start));
    TRY(upload(h, h->d_vscale, sc));
    a.fval_u0 = h->d_fval_u0;
    a.vscale = h->d_vscale;
  } else if (h->vmode == 2) {
    size_t G = (size_t)std::max(h->npm, h->nt) + 2;
    a.t = h->d_vgauss; a.p = h->d_vgauss + G; a.st_i = h->d_vgauss + 2 * G;
    a.vtt = h->vt_const * c_km_s_to_rs_hr * (time - h->vtime_start);
    a.vpt = h->vp_omega * c_km_s_to_rs_hr * (time - h->vtime_start);
    a.p1 = fmodulo(c_pi_two + a.vpt, c_twopi);
    a.p2 = fmodulo(c_threepi_two + a.vpt, c_twopi);
    a.width = h->vwidth;
  }
  const int cpb = 8;
  int nb = (npm - 1 + cpb - 1) / cpb;
  TRY(ensure_part(h, (size_t)nr * nb * kNPart + (size_t)nr * kNPart));
  double *fin = h->d_part + (size_t)nr * nb * kNPart;
  k_analysis_partial<256><<<dim3((unsigned)nb, (unsigned)nr), 256, 0, h->stream>>>(h->M, a, h->buf[h->cur],
                                                                                    h->d_part, cpb);
  LAUNCHED(h);
  k_analysis_final<<<(nr * kNPart + 127) / 128, 128, 0, h->stream>>>(nb, nr, h->d_part, fin);
  LAUNCHED(h);
  TRY(sync_read(h, fin, (size_t)nr * kNPart * sizeof(double)));
  for (int i = 0; i < nr; ++i) {
    const double *v = h->h_pin + (size_t)i * kNPart;
    double *o = hist + (size_t)i * 14;
    o[0] = v[0]; o[1] = v[1]; o[2] = v[2];
    double verr = v[3], sumfval2 = v[4];
    o[13] = (sumfval2 == 0.0) ? std::sqrt(verr / (double)((int64_t)ntm * (npm - 1))) : std::sqrt(verr / sumfval2);
    o[3] = c_rsun_cm2 * v[5]; o[4] = c_rsun_cm2 * v[6];
    o[5] = c_rsun_cm2 * v[7]; o[6] = c_rsun_cm2 * v[8];
    o[7] = c_rsun_cm2 * v[9]; o[8] = c_rsun_cm2 * v[10];
    o[9] = c_rsun_cm2 * v[11]; o[10] = c_rsun_cm2 * v[12];
    o[12] = c_three_quarter * c_pi_i * v[15];
    double e1 = c_three_quarter * c_pi_i * v[13], e2 = c_three_quarter * c_pi_i * v[14];
    o[11] = std::sqrt(e1 * e1 + e2 * e2);
  }
  return HIPFT_OK;
}

static int flux_of(hipft_gpu *h, const double *a, std::vector<double> &fp, std::vector<double> &fm) {
  int nr = h->nr;
  const int cpb = 16;
  int nb = (h->npm - 1 + cpb - 1) / cpb;
  TRY(ensure_part(h, (size_t)nr * nb * 2 + (nr + 1)));
  size_t L = (size_t)std::max(h->ntm, h->npm) + 1;
  k_flux_partial<<<dim3((unsigned)nb, (unsigned)nr), 256, 0, h->stream>>>(h->M, h->d_anw, h->d_anw + 3 * L, a, 0,
                                                                          h->d_part, cpb);
  LAUNCHED(h);
  std::vector<double> part((size_t)nr * nb * 2);
  CK(h, cudaMemcpyAsync(part.data(), h->d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  fp.assign(nr, 0.0);
  fm.assign(nr, 0.0);
  for (int i = 0; i < nr; ++i)
    for (int b = 0; b < nb; ++b) {
      fp[i] = fp[i] + part[((size_t)i * nb + b) * 2];
      fm[i] = fm[i] + part[((size_t)i * nb + b) * 2 + 1];
    }
  return HIPFT_OK;
}

extern "C" int hipft_gpu_get_flux(hipft_gpu *h, double *flux_p, double *flux_m) {
  if (!h || !flux_p || !flux_m) return HIPFT_EINVAL;
  if (!h->field_set) return fail(h, HIPFT_ESTATE, "get_flux before set_field");
  CK(h, cudaSetDevice(h->dev));
  std::vector<double> fp, fm;
  TRY(flux_of(h, h->buf[h->cur], fp, fm));
  std::copy(fp.begin(), fp.end(), flux_p);
  std::copy(fm.begin(), fm.end(), flux_m);
  return HIPFT_OK;
}

// balance_flux (src/hipft.f90:8752-8807) of every realization of `a`
static int balance_buffer(hipft_gpu *h, double *a) {
  std::vector<double> fp, fm;
  TRY(flux_of(h, a, fp, fm));
  std::vector<double> r(h->nr + 1, 1.0);
  for (int i = 0; i < h->nr; ++i) r[i + 1] = (fm[i] + fp[i] == 0.0) ? 1.0 : std::sqrt(std::fabs(fp[i] / fm[i]));
  size_t L = (size_t)h->nr * ((h->npm - 1 + 15) / 16) * 2;
  double *dr = h->d_part + L;
  TRY(upload(h, dr, r));
  dim3 blk(32, 8), grd((unsigned)((h->ntm + 31) / 32), (unsigned)((h->npm + 7) / 8), (unsigned)h->nr);
  k_scale_balance<<<grd, blk, 0, h->stream>>>(h->M, a, dr);
  LAUNCHED(h);
  CK(h, cudaStreamSynchronize(h->stream));
  return HIPFT_OK;
}

extern "C" int hipft_gpu_balance_flux(hipft_gpu *h) {
  if (!h) return HIPFT_EINVAL;
  if (!h->field_set) return fail(h, HIPFT_ESTATE, "balance_flux before set_field");
  CK(h, cudaSetDevice(h->dev));
  TRY(balance_buffer(h, h->buf[h->cur]));
  h->dring_valid = false;
  return HIPFT_OK;
}

extern "C" int hipft_gpu_info(const hipft_gpu *h, hipft_info *info) {
  if (!h || !info) return HIPFT_EINVAL;
  info->ntm = h->ntm;
  info->npm = h->npm;
  info->nr = h->nr;
  info->ldt = h->ldt;
  info->dtime_diffusion_euler = h->dt_euler;
  info->sts_s = (h->P.diffusion_num_method == 1) ? h->n_euler : h->sts_s;
  info->kernel_launches = h->launches;
  info->cell_stage_updates = h->cell_updates;
  info->device_bytes = h->dev_bytes;
  info->rkg2_stages = h->rkg2_stages;
  info->rkg2_cell_stages = h->rkg2_cell_stages;
  return HIPFT_OK;
}

extern "C" int hipft_gpu_describe(hipft_gpu *h, char *buf, size_t len) {
  if (!h || !buf || !len) return HIPFT_EINVAL;
  const PairPlan &p = h->plan;
  char kind[128];
  if (p.kind < 0)
    std::snprintf(kind, sizeof kind, "not chosen yet");
  else if (p.kind == PK_SINGLE)
    std::snprintf(kind, sizeof kind, "%s", pair_kind_name(p.kind));
  else
    std::snprintf(kind, sizeof kind, "%s, %d CTAs per SM", pair_kind_name(p.kind), p.ctas_per_sm);
  if (p.candidates > 0)
    std::snprintf(buf, len, "schedule=%s; two-stage kernel: %s (tuned over %d candidates, %.4f ms per launch pair)",
                  h->ragged ? "ragged" : "shared", kind, p.candidates, p.ms);
  else
    std::snprintf(buf, len, "schedule=%s; two-stage kernel: %s", h->ragged ? "ragged" : "shared", kind);
  return HIPFT_OK;
}

extern "C" int hipft_gpu_set_stream(hipft_gpu *h, void *s) {
  if (!h) return HIPFT_EINVAL;
  CK(h, cudaStreamSynchronize(h->stream));
  if (s) {
    if (h->own_stream) cudaStreamDestroy(h->stream);
    h->own_stream = false;
    h->stream = (cudaStream_t)s;
  } else if (!h->own_stream) {
    CK(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
  }
  return HIPFT_OK;
}

extern "C" int hipft_gpu_check_bounded_wait(hipft_gpu *h, unsigned int limit) {
  if (!h || limit == 0 || limit > (1u << 22)) return HIPFT_EINVAL;
  CK(h, cudaSetDevice(h->dev));
  k_wait_selftest<<<1, 32, 0, h->stream>>>(limit, h->d_err);
  LAUNCHED(h);
  return check_wait_flag(h, "check_bounded_wait: the wait gave up as intended");
}

extern "C" int hipft_gpu_field_device_ptr(hipft_gpu *h, double **ptr, int *ldt) {
  if (!h || !ptr || !ldt) return HIPFT_EINVAL;
  if (!h->field_set) return fail(h, HIPFT_ESTATE, "field_device_ptr before set_field");
  CK(h, cudaSetDevice(h->dev));
  CK(h, cudaStreamSynchronize(h->stream));  // the field is complete when the pointer is handed out
  *ptr = h->buf[h->cur];
  *ldt = h->ldt;
  return HIPFT_OK;
}

extern "C" int hipft_gpu_synchronize(hipft_gpu *h) {
  if (!h) return HIPFT_EINVAL;
  CK(h, cudaStreamSynchronize(h->stream));
  return HIPFT_OK;
}

// Folds finished event pairs into the per-kind totals.
static int prof_collect(hipft_gpu *h) {
  CK(h, cudaStreamSynchronize(h->stream));
  for (int k = 0; k < HIPFT_K_NKINDS; ++k) {
    for (auto &pr : h->ev_pending[k]) {
      float ms = 0.f;
      CK(h, cudaEventElapsedTime(&ms, pr.first, pr.second));
      h->prof_ms[k] += ms;
      h->prof_n[k] += 1;
      h->ev_pool.push_back(pr.first);
      h->ev_pool.push_back(pr.second);
    }
    h->ev_pending[k].clear();
  }
  return HIPFT_OK;
}

extern "C" int hipft_gpu_set_profiling(hipft_gpu *h, int on) {
  if (!h) return HIPFT_EINVAL;
  TRY(prof_collect(h));
  for (int k = 0; k < HIPFT_K_NKINDS; ++k) {
    h->prof_ms[k] = 0.0;
    h->prof_n[k] = 0;
  }
  h->profiling = on != 0;
  return HIPFT_OK;
}

extern "C" int hipft_gpu_kernel_time(hipft_gpu *h, int kind, int64_t *launches, double *total_ms) {
  if (!h || kind < 0 || kind >= HIPFT_K_NKINDS || !launches || !total_ms) return HIPFT_EINVAL;
  TRY(prof_collect(h));
  *launches = h->prof_n[kind];
  *total_ms = h->prof_ms[kind];
  return HIPFT_OK;
}

// ======================================================================
// hipft_get_flux_noalloc: get_flux (src/hipft.f90:8672) for callers that
// cannot allocate GPU memory.
//
// Some callers own every byte of device memory themselves: a Fortran code
// that keeps its maps device-resident through OpenMP `target enter data`
// mappings (HipFT's own model) and hands over `use_device_ptr` addresses, or
// a host application that runs the GPU from a fixed, pre-reserved arena.
// They cannot let a library call cudaMalloc.  This entry point takes the
// field as a device pointer and keeps all of its scratch -- the mesh scales,
// the cell-area weights, the per-block partial sums and the per-realization
// results -- in one file-scope __device__ array, g_na_scratch, of fixed size
// (kNaScratchDoubles doubles, about 1.6 MB), which every GPU that loads this
// library holds until the process exits.
//
// Limits: ntm <= kNaMaxNtm, npm1 <= kNaMaxNpm1, nr <= kNaMaxNr, and the
// partial sums (2 * nr * ceil((npm1)/16)) must fit kNaMaxPart; larger
// requests return HIPFT_EINVAL.  The array is shared by every call on a
// device and keeps the last call's contents, so calls that overlap on the GPU
// (different streams, or different host threads) race; serialise them.
// The first call on a device looks up the array's device address with
// cudaGetSymbolAddress (with that device current) and caches it; make that
// first call before any stream capture.
// ======================================================================
#include <mutex>

namespace {
constexpr int kNaMaxNtm = 16384;
constexpr int kNaMaxNpm1 = 16384;
constexpr int kNaMaxNr = 2000;
constexpr int kNaMaxPart = 1 << 17;
constexpr int kNaMaxDevices = 64;
// layout (doubles): t[kNaMaxNtm+2] p[kNaMaxNpm1+2] da_t[kNaMaxNtm+2] da_p[kNaMaxNpm1+2] part[kNaMaxPart] out[2*kNaMaxNr]
constexpr size_t kNaOffT = 0;
constexpr size_t kNaOffP = kNaOffT + kNaMaxNtm + 2;
constexpr size_t kNaOffDaT = kNaOffP + kNaMaxNpm1 + 2;
constexpr size_t kNaOffDaP = kNaOffDaT + kNaMaxNtm + 2;
constexpr size_t kNaOffPart = kNaOffDaP + kNaMaxNpm1 + 2;
constexpr size_t kNaOffOut = kNaOffPart + kNaMaxPart;
constexpr size_t kNaScratchDoubles = kNaOffOut + 2 * kNaMaxNr;
std::mutex g_na_mutex;
double *g_na_dev_ptr[kNaMaxDevices] = {};
}  // namespace

static __device__ __align__(256) double g_na_scratch[kNaScratchDoubles];

// Cell-area weights of get_flux (src/hipft.f90:8712-8732) from the raw
// scales, computed with set_mesh's definitions (6579-6641); 1-based.
__global__ void k_na_weights(int ntm, int npm1, const double *t, const double *p, double *da_t, double *da_p) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (n <= ntm) {
    const int j = n;
    double v;
    if (j == 1) {
      v = 0.25 * sin(0.5 * (t[1] + t[2])) * (t[2] - t[1]);
    } else if (j == ntm) {
      v = 0.25 * sin(0.5 * (t[ntm] + t[ntm - 1])) * (t[ntm] - t[ntm - 1]);
    } else {
      double thj = 0.5 * (t[j] + t[j - 1]), thj1 = 0.5 * (t[j + 1] + t[j]);
      v = sin(t[j]) * (thj1 - thj);
    }
    da_t[j] = v;
  }
  if (n <= npm1) {
    const int k = n;
    double v;
    if (k == 1 || k == npm1) {
      v = 0.5 * (p[npm1] - p[npm1 - 1]);
    } else {
      double phk = 0.5 * (p[k] + p[k - 1]), phk1 = 0.5 * (p[k + 1] + p[k]);
      v = phk1 - phk;
    }
    da_p[k] = v;
  }
}

// Per-realization totals of the block partials, in block order.
__global__ void k_na_flux_final(int nb, int nr, const double *part, double *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nr) return;
  double fp = 0.0, fm = 0.0;
  for (int b = 0; b < nb; ++b) {
    fp = fp + part[((int64_t)i * nb + b) * 2];
    fm = fm + part[((int64_t)i * nb + b) * 2 + 1];
  }
  out[2 * i] = fp;
  out[2 * i + 1] = fm;
}

static int na_fail(char *err, size_t len, int code, const char *msg) {
  if (err && len) std::snprintf(err, len, "hipft_get_flux_noalloc: %s", msg);
  return code;
}

extern "C" int hipft_get_flux_noalloc(const double *f_dev, int ntm, int npm1, int nr, int ldt, const double *t,
                                      const double *p, double *flux_p, double *flux_m, void *cuda_stream,
                                      char *err, size_t err_len) {
  if (!f_dev || !t || !p || !flux_p || !flux_m) return na_fail(err, err_len, HIPFT_EINVAL, "null argument");
  if (ntm < 4 || npm1 < 5 || nr < 1 || ldt < ntm)
    return na_fail(err, err_len, HIPFT_EINVAL, "sizes out of range (ntm >= 4, npm1 >= 5, nr >= 1, ldt >= ntm)");
  const int cpb = 16;
  const int npm = npm1 + 1;
  const int nb = (npm - 1 + cpb - 1) / cpb;
  if (ntm > kNaMaxNtm || npm1 > kNaMaxNpm1 || nr > kNaMaxNr || (size_t)2 * nr * nb > (size_t)kNaMaxPart)
    return na_fail(err, err_len, HIPFT_EINVAL,
                   "grid too large for the fixed scratch (ntm <= 16384, npm1 <= 16384, nr <= 2000, "
                   "2*nr*ceil(npm1/16) <= 131072)");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices)
    return na_fail(err, err_len, HIPFT_ECUDA, "no usable current device");
  double *base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_na_mutex);
    if (!g_na_dev_ptr[dev]) {
      double *ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_na_scratch);
      if (e != cudaSuccess || !ptr) return na_fail(err, err_len, HIPFT_ECUDA, cudaGetErrorString(e));
      g_na_dev_ptr[dev] = ptr;
    }
    base = g_na_dev_ptr[dev];
  }
  cudaStream_t s = (cudaStream_t)cuda_stream;
  double *dt = base + kNaOffT, *dp = base + kNaOffP, *dat = base + kNaOffDaT, *dap = base + kNaOffDaP;
  double *part = base + kNaOffPart, *out = base + kNaOffOut;
  // 1-based scales
  if (cudaMemcpyAsync(dt + 1, t, sizeof(double) * ntm, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(dp + 1, p, sizeof(double) * npm1, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return na_fail(err, err_len, HIPFT_ECUDA, "copy of the scales failed");
  int nmax = ntm > npm1 ? ntm : npm1;
  k_na_weights<<<(nmax + 255) / 256, 256, 0, s>>>(ntm, npm1, dt, dp, dat, dap);
  Mesh m{};
  m.ntm = ntm;
  m.npm = npm;
  m.nt = ntm + 1;
  m.np = npm;
  m.nr = nr;
  m.ldt = ldt;
  m.plane = (int64_t)ldt * npm;
  k_flux_partial<<<dim3((unsigned)nb, (unsigned)nr), 256, 0, s>>>(m, dat, dap, f_dev, 0, part, cpb);
  k_na_flux_final<<<(nr + 127) / 128, 128, 0, s>>>(nb, nr, part, out);
  {
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) {
      char msg[256];
      std::snprintf(msg, sizeof msg, "kernel launch failed: %s", cudaGetErrorString(le));
      return na_fail(err, err_len, HIPFT_ECUDA, msg);
    }
  }
  if (cudaMemcpy2DAsync(flux_p, sizeof(double), out, 2 * sizeof(double), sizeof(double), (size_t)nr,
                        cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpy2DAsync(flux_m, sizeof(double), out + 1, 2 * sizeof(double), sizeof(double), (size_t)nr,
                        cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return na_fail(err, err_len, HIPFT_ECUDA, "copy of the results failed");
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return na_fail(err, err_len, HIPFT_ECUDA, cudaGetErrorString(e));
  return HIPFT_OK;
}

// ------------------------------------------------------------------ adjoint
// Discrete adjoint of one flux_transport_step (no reference counterpart):
// the step is replayed from its input with every stage input kept (the
// "tape"), then run backwards through the transposed stages.  The schedule
// of the replay (PTL subcycle dts, RKG2 stage counts) is the forward's own,
// computed by the same routines from the same field, and is held fixed:
// the gradient is that of the discrete map at this schedule.



// Stage spacing of the stage checkpoints for a super-step of s stages:
// 0 (keep every stage) when s + 1 fields fit the tape budget, else an even
// q near sqrt(2 s), which keeps about 2 sqrt(2 s) fields.
static int64_t adj_stage_spacing(hipft_gpu *h, int64_t s) {
  int64_t budget = h->adj_tape_limit;
  if (budget <= 0) {
    if (h->adj_free_seen == 0) {  // once per run (reset by hipft_adj_clear / hipft_adj_release)
      size_t fr = 0, tot = 0;
      if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) fr = 0;
      h->adj_free_seen = fr + 1;
    }
    budget = (int64_t)((h->adj_free_seen - 1) / 2 / (h->fieldn * sizeof(double)));
  }
  if (h->adj_force_q > 0) return h->adj_force_q;
  if (s + 1 <= budget) return 0;
  int64_t q = (int64_t)std::ceil(std::sqrt(2.0 * (double)s));
  if (q % 2) ++q;
  return std::max<int64_t>(q, 2);
}

// Tape slot n; slots are allocated in chunks of up to 32 fields (at most
// 256 MB per chunk), so that taping many steps needs few allocations.
static int adj_slot(hipft_gpu *h, size_t n, double **p) {
  while (h->tape.size() <= n) {
    const size_t fb = h->fieldn * sizeof(double);
    const size_t per = std::max<size_t>(1, std::min<size_t>(32, (size_t)(256u << 20) / fb));
    double *q = nullptr;
    TRY(dalloc(h, &q, h->fieldn * per));
    h->tape_chunks.push_back(q);
    for (size_t e = 0; e < per; ++e) h->tape.push_back(q + e * h->fieldn);
  }
  *p = h->tape[n];
  return HIPFT_OK;
}

static int adj_ensure(hipft_gpu *h) {
  if (h->adjw[0]) return HIPFT_OK;
  for (auto &w : h->adjw) {
    TRY(dalloc(h, &w, h->fieldn));
    CK(h, cudaMemsetAsync(w, 0, h->fieldn * sizeof(double), h->stream));
  }
  dim3 g = stage_grid(h, 32, 8);
  h->dpart_per_r = (int)(g.x * g.y);
  TRY(dalloc(h, &h->d_dpart, (size_t)h->dpart_per_r * h->nr));
  h->adj_nch = (h->npm - 2 + 255) / 256;
  TRY(dalloc(h, &h->d_gring, 2 * (size_t)h->nr * h->adj_nch));
  TRY(dalloc(h, &h->d_dpole, (size_t)h->nr * h->adj_nch));
  for (auto &gp : h->d_gpart) TRY(dalloc(h, &gp, 2 * (size_t)g.y * h->nr));
  return HIPFT_OK;
}

// SSPRK(4,3) with its four stage inputs kept (src/hipft.f90:7552-7574);
// the result replaces the current field.
static int adj_adv_fwd(hipft_gpu *h, double dtl, size_t &nt, size_t t[4]) {
  double *T[4];
  for (int q = 0; q < 4; ++q) {
    t[q] = nt;
    TRY(adj_slot(h, nt++, &T[q]));
  }
  double *f = h->buf[h->cur];
  CK(h, cudaMemcpyAsync(T[0], f, h->fieldn * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  TRY(advection_stage(h, T[0], nullptr, T[1], AdvCombine{0, 0.0, 0.0, 0.5 * dtl}));
  TRY(advection_stage(h, T[1], nullptr, T[2], AdvCombine{0, 0.0, 0.0, 0.5 * dtl}));
  TRY(advection_stage(h, T[2], T[0], T[3], AdvCombine{1, c_two_third, c_third, c_sixth * dtl}));
  TRY(advection_stage(h, T[3], nullptr, f, AdvCombine{0, 0.0, 0.0, 0.5 * dtl}));
  h->dring_valid = false;
  return HIPFT_OK;
}

// diffusion_step (src/hipft.f90:4551-4695) with RKG2 super-steps whose
// stage fields are kept; same subcycle logic as hipft_gpu_diffusion_step.
static int adj_diff_fwd(hipft_gpu *h, double dtl, size_t &nt, std::vector<AdjSub> &subs) {
  const int max_sc = 60;
  TRY(ensure_pair_plan(h));
  int i = 1;
  bool done = false;
  double time_stepped = 0.0;
  double dtl2 = h->auto_sc ? 0.0 : dtl / (double)h->P.diffusion_subcycles;
  for (;;) {
    if (h->auto_sc) TRY(ptl_dt(h, &dtl2));
    if (h->auto_sc && time_stepped + dtl2 >= dtl) {
      dtl2 = dtl - time_stepped;
      done = true;
    }
    if (h->auto_sc && i == max_sc - 1) {
      dtl2 = dtl - time_stepped;
      done = true;
    }
    load_sts(h, dtl2);
    AdjSub S;
    S.dtl = dtl2;
    S.s = h->sts_s;
    S.uj = h->sts_uj;
    S.vj = h->sts_vj;
    S.ubj = h->sts_ubj;
    S.gj = h->sts_gj;
    S.t0 = nt;
    S.q = adj_stage_spacing(h, S.s);
    double *u0, *dty0;
    TRY(adj_slot(h, nt++, &u0));
    TRY(adj_slot(h, nt++, &dty0));
    std::vector<double *> Y((size_t)S.s + 1, nullptr);
    Y[0] = u0;
    if (S.q == 0) {
      for (int64_t k = 1; k <= S.s - 1; ++k) TRY(adj_slot(h, nt++, &Y[k]));
    } else {
      // block starts c = 1, 1+q, ... below s; their pairs (Y_{c-1}, Y_c) are
      // tape slots, the other stages go through a rotating scratch set
      for (int64_t c = 1; c <= S.s - 1; c += S.q) S.cstart.push_back(c);
      for (size_t b = 0; b < S.cstart.size(); ++b) {
        const int64_t c = S.cstart[b];
        S.ck_prev.push_back(SIZE_MAX);
        if (c > 1) {
          S.ck_prev.back() = nt;
          TRY(adj_slot(h, nt++, &Y[c - 1]));
        }
        S.ck_cur.push_back(nt);
        TRY(adj_slot(h, nt++, &Y[c]));
      }
      S.ring0 = h->adj_rings_n;
      h->adj_rings_n += S.cstart.size();
      if (h->adj_rings_n > h->adj_rings_cap) {
        // grown before any ring checkpoint of this step is written
        double *nr_ = nullptr;
        const size_t cap = h->adj_rings_n + 64;
        TRY(dalloc(h, &nr_, cap * 2 * (size_t)h->nr));
        if (h->d_adj_rings) {
          CK(h, cudaMemcpyAsync(nr_, h->d_adj_rings, h->adj_rings_cap * 2 * (size_t)h->nr * sizeof(double),
                                cudaMemcpyDeviceToDevice, h->stream));
          CK(h, cudaStreamSynchronize(h->stream));
          cudaFree(h->d_adj_rings);
          h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void *)h->d_adj_rings), h->allocs.end());
        }
        h->d_adj_rings = nr_;
        h->adj_rings_cap = cap;
      }
      // stages that are not checkpoints rotate through four scratch fields
      // of the block buffer: a stage pair reads Y_{k-1}, Y_{k-2} and writes
      // Y_k, Y_{k+1}, four distinct fields
      while (h->adj_block.size() < 4) {
        double *q = nullptr;
        TRY(dalloc(h, &q, h->fieldn));
        h->adj_block.push_back(q);
      }
      int rot = 0;
      for (int64_t k = 1; k <= S.s - 1; ++k)
        if (!Y[k]) Y[k] = h->adj_block[(rot++) % 4];
    }
    Y[S.s] = h->buf[h->cur];
    CK(h, cudaMemcpyAsync(u0, h->buf[h->cur], h->fieldn * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    // the same kernels, in the same order, as sts_super_step (with its pole
    // sums of the current field), writing every stage into the tape
    const double *r0;
    TRY(current_dring(h, &r0));
    TRY(sts_stage_v2<MODE_STS1>(h, u0, nullptr, nullptr, nullptr, Y[1], dty0, StageCoef{dtl2, S.ubj[1], 0, 0, 0}));
    auto coef = [&](int64_t k) {
      const double uj = S.uj[k], vj = S.vj[k];
      return StageCoef{uj, vj, 1.0 - uj - vj, S.ubj[k] * dtl2, S.gj[k]};
    };
    // ring sums of a block start's Y_c (the ring of the launch's output)
    auto keep_ring = [&](int64_t c) -> int {
      if (S.q == 0) return HIPFT_OK;
      for (size_t b = 0; b < S.cstart.size(); ++b)
        if (S.cstart[b] == c)
          CK(h, cudaMemcpyAsync(h->d_adj_rings + (S.ring0 + b) * 2 * (size_t)h->nr, h->d_ringbuf[h->ring_cur],
                                2 * (size_t)h->nr * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
      return HIPFT_OK;
    };
    TRY(keep_ring(1));
    int64_t k = 2;
    while (k <= S.s) {
      if (sts_pairs_enabled(h) && k + 1 <= S.s) {
        TRY(sts_pair(h, Y[k - 1], Y[k - 2], u0, dty0, Y[k], Y[k + 1], coef(k), coef(k + 1), k > 2));
        TRY(keep_ring(k + 1));
        k += 2;
        continue;
      }
      TRY(sts_stage_v2<MODE_STSK>(h, Y[k - 1], Y[k - 2], u0, dty0, Y[k], nullptr, coef(k)));
      TRY(keep_ring(k));
      k += 1;
    }
    h->dring_valid = true;  // the last fused stage left the ring of the output
    h->cell_updates += (int64_t)h->ntm * (h->npm - 2) * h->nr * S.s;
    subs.push_back(std::move(S));
    time_stepped = time_stepped + dtl2;
    if (!h->auto_sc && i == h->P.diffusion_subcycles) done = true;
    if (done) break;
    i = i + 1;
  }
  return HIPFT_OK;
}

// a work field other than those in `busy`
static double *adj_free(hipft_gpu *h, std::initializer_list<const double *> busy) {
  for (double *w : h->adjw) {
    bool used = false;
    for (const double *b : busy) used = used || (b == w);
    if (!used) return w;
  }
  return nullptr;
}

static int adj_adv_rev(hipft_gpu *h, double dtl, const size_t t[4], double *&W, double *gflow) {
  const dim3 blk(32, 8), grd = stage_grid(h, 32, 8);
  double *g[5];
  for (int q = 0; q < 5; ++q) g[q] = gflow + (size_t)q * h->fieldn;
  auto stage = [&](const double *x, const double *w, double sigma, double alpha, const double *base, double beta,
                   double *out) -> int {
    k_adj_pole_sums<<<h->nr, 256, 0, h->stream>>>(h->M, w, h->d_gring);
    LAUNCHED(h);
    k_adj_adv<<<grd, blk, 0, h->stream>>>(h->M, h->FL, h->W, x, w, base, out, h->d_gring,
                                          AdjAdvArgs{sigma, alpha, beta, h->bc_flow_n, h->bc_flow_s}, g[0], g[1],
                                          g[2], g[3], g[4]);
    LAUNCHED(h);
    return HIPFT_OK;
  };
  double *b3 = adj_free(h, {W});
  double *b2 = adj_free(h, {W, b3});
  double *b1 = adj_free(h, {W, b3, b2});
  const double *T0 = h->tape[t[0]], *T1 = h->tape[t[1]], *T2 = h->tape[t[2]], *T3 = h->tape[t[3]];
  TRY(stage(T3, W, -0.5 * dtl, 1.0, nullptr, 0.0, b3));
  TRY(stage(T2, b3, -c_sixth * dtl, c_third, nullptr, 0.0, b2));
  TRY(stage(T1, b2, -0.5 * dtl, 1.0, nullptr, 0.0, b1));
  TRY(stage(T0, b1, -0.5 * dtl, 1.0, b3, c_two_third, W));
  return HIPFT_OK;
}

// Reverse of one RKG2 super-step: W (cotangent of Y_s) becomes the
// cotangent of u0; dacc[i] += the diffusion-coefficient terms
// sum mu~_k dt <A^T Wbar_k, Y_{k-1}> (+ dt <A^T dbar, u0>).  One launch per
// stage: each leaves the pole-row partials of its output for the next.
// Recomputes the stages Y_{c+1}..Y_e of stage-checkpoint block b (e = the
// block's last stage input, at most s-1) from its pair (Y_{c-1}, Y_c) and the
// ring sums of Y_c, with the replay's kernels and launch grouping, so the
// values are bitwise those of the replay.  Y receives the block's fields.
static int adj_block_recompute(hipft_gpu *h, const AdjSub &S, size_t b, std::vector<const double *> &Y) {
  const int64_t c = S.cstart[b], e = std::min(c + S.q - 1, S.s - 1);
  while ((int64_t)h->adj_block.size() < S.q + 1) {
    double *q = nullptr;
    TRY(dalloc(h, &q, h->fieldn));
    h->adj_block.push_back(q);
  }
  const double *u0 = h->tape[S.t0], *dty0 = h->tape[S.t0 + 1];
  std::vector<double *> Yw((size_t)S.s + 2, nullptr);
  Yw[c - 1] = (S.ck_prev[b] == SIZE_MAX) ? const_cast<double *>(u0) : h->tape[S.ck_prev[b]];
  Yw[c] = h->tape[S.ck_cur[b]];
  for (int64_t k = c + 1; k <= std::min(e + 1, S.s); ++k) Yw[k] = h->adj_block[k - c - 1];
  CK(h, cudaMemcpyAsync(h->d_ringbuf[h->ring_cur], h->d_adj_rings + (S.ring0 + b) * 2 * (size_t)h->nr,
                        2 * (size_t)h->nr * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  auto coef = [&](int64_t k) {
    const double uj = S.uj[k], vj = S.vj[k];
    return StageCoef{uj, vj, 1.0 - uj - vj, S.ubj[k] * S.dtl, S.gj[k]};
  };
  int64_t k = c + 1;
  while (k <= e) {
    if (sts_pairs_enabled(h) && k + 1 <= S.s) {
      TRY(sts_pair(h, Yw[k - 1], Yw[k - 2], u0, dty0, Yw[k], Yw[k + 1], coef(k), coef(k + 1), k > c + 1));
      k += 2;
      continue;
    }
    TRY(sts_stage_v2<MODE_STSK>(h, Yw[k - 1], Yw[k - 2], u0, dty0, Yw[k], nullptr, coef(k)));
    k += 1;
  }
  for (int64_t q = c - 1; q <= e; ++q) Y[q] = Yw[q];
  h->dring_valid = false;
  return HIPFT_OK;
}

// HIPFT_ADJ_PAIR=0 runs the reverse RKG2 stages one per launch (A/B timing).
static bool adj_pairs_enabled() {
  static int v = -1;
  if (v < 0) {
    const char *e = std::getenv("HIPFT_ADJ_PAIR");
    v = (e && std::atoi(e) == 0) ? 0 : 1;
  }
  return v == 1;
}

static int adj_diff_rev(hipft_gpu *h, const AdjSub &S, double *&W, double *dacc) {
  const dim3 blk(32, 8), grd = stage_grid(h, 32, 8);
  const double dtl = S.dtl;
  double *ub = adj_free(h, {W});
  double *db = adj_free(h, {W, ub});
  CK(h, cudaMemsetAsync(ub, 0, h->fieldn * sizeof(double), h->stream));
  CK(h, cudaMemsetAsync(db, 0, h->fieldn * sizeof(double), h->stream));
  CK(h, cudaMemsetAsync(h->d_dpart, 0, (size_t)h->dpart_per_r * h->nr * sizeof(double), h->stream));
  CK(h, cudaMemsetAsync(h->d_dpole, 0, (size_t)h->adj_nch * h->nr * sizeof(double), h->stream));
  // stage inputs Y_k: all on the tape (q == 0) or one recomputed block at a time
  std::vector<const double *> Yr((size_t)S.s + 1, nullptr);
  Yr[0] = h->tape[S.t0];
  if (S.q == 0)
    for (int64_t k = 1; k <= S.s - 1; ++k) Yr[k] = h->tape[S.t0 + 1 + k];
  int64_t curb = -1;
  auto Yt = [&](int64_t k) -> const double * { return Yr[k]; };
  const double *gin = h->d_gring;
  int npin = 1, pp = 0;
  auto pole_sums = [&](const double *w) -> int {
    k_adj_pole_sums<<<h->nr, 256, 0, h->stream>>>(h->M, w, h->d_gring);
    LAUNCHED(h);
    gin = h->d_gring;
    npin = 1;
    return HIPFT_OK;
  };
  auto stage = [&](const double *w, const double *wp, const double *y, double *out, double *u, double *d,
                   AdjDiffCoef ac) -> int {
    double *gout = h->d_gpart[pp];
    k_adj_diff<<<grd, blk, 0, h->stream>>>(h->M, h->DC, w, wp, y, out, u, d, gin, npin, gout, h->bc_diff_n,
                                           h->bc_diff_s, ac, h->d_dpart, h->ptab);
    LAUNCHED(h);
    gin = gout;
    npin = (int)grd.y;
    pp ^= 1;
    return HIPFT_OK;
  };
  TRY(pole_sums(W));
  double *Wk = W, *Wk1 = nullptr;
  int64_t k = S.s;
  // two reverse stages per launch (k_adj_diff2 + k_adj_pole2) while both of
  // their stage inputs Y_{k-1}, Y_{k-2} lie in one stage-checkpoint block
  // A pair launch follows the previous pair's k_adj_pole2 programmatically
  // (its interior tiles start while that kernel runs); its outputs then avoid
  // the previous pair's W_k as well, which that kernel still reads.
  double *Wprev = nullptr;
  bool after_pole2 = false;
  const dim3 grd2((unsigned)((h->ntm + kA2J - 1) / kA2J), (unsigned)((h->npm - 2 + kA2K - 1) / kA2K), (unsigned)h->nr);
  while (adj_pairs_enabled() && k >= 3 && (S.q == 0 || (k - 2) / S.q == (k - 3) / S.q)) {
    if (S.q > 0 && (k - 3) / S.q != curb) {
      curb = (k - 3) / S.q;
      TRY(adj_block_recompute(h, S, (size_t)curb, Yr));
      after_pole2 = false;
    }
    double *Wm1 = adj_free(h, {Wk, Wk1, ub, db, Wprev});
    double *Wm2 = adj_free(h, {Wk, Wk1, ub, db, Wprev, Wm1});
    const double u1 = S.uj[k], v1 = S.vj[k], u2 = S.uj[k - 1], v2 = S.vj[k - 1];
    const double nu1 = (k < S.s) ? S.vj[k + 1] : 0.0;
    const AdjDiff2Coef ac{u1, nu1, S.ubj[k] * dtl, 1.0 - u1 - v1, S.gj[k], S.ubj[k] * dtl,
                          u2, v1, S.ubj[k - 1] * dtl, 1.0 - u2 - v2, S.gj[k - 1], S.ubj[k - 1] * dtl};
    double *gpart = h->d_gpart[pp];
    {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = grd2;
      cfg.blockDim = dim3(kA2J, kA2K);
      cfg.stream = h->stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      attr[0].val.programmaticStreamSerializationAllowed = (ws_pdl() && after_pole2) ? 1 : 0;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      const double *y1 = Yt(k - 1), *y2 = Yt(k - 2);
      CK(h, cudaLaunchKernelEx(&cfg, k_adj_diff2, h->M, h->DC, (const double *)Wk, (const double *)Wk1, y1, y2, Wm1,
                               Wm2, ub, db, gin, npin, gpart, h->bc_diff_n, h->bc_diff_s, ac, h->d_dpart,
                               h->dpart_per_r, h->ptab));
      LAUNCHED(h);
    }
    k_adj_pole2<<<dim3((unsigned)h->nr, (unsigned)h->adj_nch), 256, 0, h->stream>>>(
        h->M, h->DC, Wk, Wm1, Yt(k - 2), Wm2, gpart, (int)grd2.y, h->d_gring, h->bc_diff_n, h->bc_diff_s, ac, h->d_dpole,
        h->ptab);
    LAUNCHED(h);
    after_pole2 = true;
    gin = h->d_gring;
    npin = h->adj_nch;
    pp ^= 1;
    Wprev = Wk;
    Wk1 = Wm1;
    Wk = Wm2;
    k -= 2;
  }
  for (; k >= 2; --k) {
    if (S.q > 0 && (k - 2) / S.q != curb) {
      curb = (k - 2) / S.q;  // the block holding Y_{k-1}
      TRY(adj_block_recompute(h, S, (size_t)curb, Yr));
    }
    double *Wm = adj_free(h, {Wk, Wk1, ub, db});
    const double uj = S.uj[k], vj = S.vj[k];
    const double nu1 = (k < S.s) ? S.vj[k + 1] : 0.0;
    TRY(stage(Wk, Wk1, Yt(k - 1), Wm, ub, db,
              AdjDiffCoef{uj, nu1, S.ubj[k] * dtl, 1.0 - uj - vj, S.gj[k], S.ubj[k] * dtl}));
    Wk1 = Wk;
    Wk = Wm;
  }
  // Y_1 = u0 + mu~_1 dty0 and Y_0 = u0 (read by stage 2 with nu_2)
  k_adj_axpy2<<<grd, blk, 0, h->stream>>>(h->M, ub, 1.0, Wk, S.vj[2], Wk1);
  LAUNCHED(h);
  k_adj_axpy2<<<grd, blk, 0, h->stream>>>(h->M, db, S.ubj[1], Wk, 0.0, nullptr);
  LAUNCHED(h);
  // dty0 = dt A u0
  TRY(pole_sums(db));
  TRY(stage(db, ub, Yt(0), ub, nullptr, nullptr, AdjDiffCoef{0.0, 1.0, dtl, 0.0, 0.0, dtl}));
  k_adj_dsum<<<h->nr, 256, 0, h->stream>>>(h->d_dpart, h->dpart_per_r, h->d_dpole, h->adj_nch, 1.0, dacc);
  LAUNCHED(h);
  W = ub;
  return HIPFT_OK;
}

static int adj_check(hipft_gpu *h) {
  if (!h->field_set) return fail(h, HIPFT_ESTATE, "adjoint step before set_field");
  if (h->P.advance_flow && (h->adv_time != 3 || h->adv_space != 2))
    return fail(h, HIPFT_ESTATE, "adjoint: advection must be WENO3+SSPRK(4,3)");
  // flows from files (with or without analytic parts) do not depend on the
  // field; attenuated flows do (through |Br|), and the rotated rigid rotation
  // is NaN on most grids
  if (h->P.advance_flow && h->have_flow && (h->fdef.flow_attenuate || h->fdef.flow_rigid_omega != 0.0))
    return fail(h, HIPFT_ESTATE, "adjoint: attenuated or rotated flows are not differentiated");
  if (h->P.advance_diffusion && (h->P.diffusion_num_method != 3 || h->DC.grid))
    return fail(h, HIPFT_ESTATE, "adjoint: diffusion must be RKG2 with per-realization constant coefficients");
  if (h->P.advance_source) return fail(h, HIPFT_ESTATE, "adjoint: sources are not differentiated");
  if (h->ragged) return fail(h, HIPFT_ESTATE, "adjoint: replays the shared (plain) schedule only");
  return HIPFT_OK;
}

// One flux_transport_step of the current field with its tape pushed on the
// tape stack (the field becomes the step's output).
static int adj_record(hipft_gpu *h, double dt) {
  TRY(adj_ensure(h));
  h->dring_valid = false;
  AdjRec R;
  R.dt = dt;
  R.first = h->adj_top;
  R.ring_first = h->adj_rings_n;
  size_t nt = h->adj_top;
  const bool strang = h->P.strang_splitting != 0;
  const double da = strang ? 0.5 * dt : dt;
  if (h->P.advance_flow) TRY(adj_adv_fwd(h, da, nt, R.ta1));
  if (h->P.advance_diffusion) TRY(adj_diff_fwd(h, dt, nt, R.subs));
  if (strang && h->P.advance_flow) TRY(adj_adv_fwd(h, da, nt, R.ta2));
  h->adj_top = nt;
  h->adj_top_max = std::max(h->adj_top_max, nt);
  h->adj_recs.push_back(std::move(R));
  return HIPFT_OK;
}

// Reverse of the most recently recorded step (popped from the stack).
static int adj_reverse(hipft_gpu *h, double *fbar, double *dacc, double *gflow) {
  if (h->adj_recs.empty()) return fail(h, HIPFT_ESTATE, "adjoint reverse: no recorded step");
  const AdjRec &R = h->adj_recs.back();
  const size_t bytes = h->fieldn * sizeof(double);
  const bool strang = h->P.strang_splitting != 0;
  const double da = strang ? 0.5 * R.dt : R.dt;
  double *W = h->adjw[0];
  CK(h, cudaMemcpyAsync(W, fbar, bytes, cudaMemcpyDeviceToDevice, h->stream));
  if (strang && h->P.advance_flow) TRY(adj_adv_rev(h, da, R.ta2, W, gflow));
  for (size_t q = R.subs.size(); q-- > 0;) TRY(adj_diff_rev(h, R.subs[q], W, dacc));
  if (h->P.advance_flow) TRY(adj_adv_rev(h, da, R.ta1, W, gflow));
  CK(h, cudaMemcpyAsync(fbar, W, bytes, cudaMemcpyDeviceToDevice, h->stream));
  h->adj_top = R.first;
  h->adj_rings_n = R.ring_first;
  h->adj_recs.pop_back();
  h->dring_valid = false;
  return HIPFT_OK;
}

extern "C" int hipft_adj_step(hipft_gpu *h, double dt, const double *f_in, double *fbar, double *dacc,
                              double *gflow) {
  if (!h || !f_in || !fbar || !dacc || !gflow) return HIPFT_EINVAL;
  TRY(adj_check(h));
  CK(h, cudaSetDevice(h->dev));
  CK(h, cudaMemcpyAsync(h->buf[h->cur], f_in, h->fieldn * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  TRY(adj_record(h, dt));
  TRY(adj_reverse(h, fbar, dacc, gflow));
  CK(h, cudaStreamSynchronize(h->stream));
  CK(h, cudaGetLastError());
  return HIPFT_OK;
}

extern "C" int hipft_adj_record(hipft_gpu *h, double dt) {
  if (!h) return HIPFT_EINVAL;
  TRY(adj_check(h));
  CK(h, cudaSetDevice(h->dev));
  TRY(adj_record(h, dt));
  CK(h, cudaGetLastError());
  return HIPFT_OK;
}

extern "C" int hipft_adj_reverse(hipft_gpu *h, double *fbar, double *dacc, double *gflow) {
  if (!h || !fbar || !dacc || !gflow) return HIPFT_EINVAL;
  CK(h, cudaSetDevice(h->dev));
  TRY(adj_reverse(h, fbar, dacc, gflow));  // asynchronous on the handle's stream
  CK(h, cudaGetLastError());
  return HIPFT_OK;
}

extern "C" int hipft_adj_clear(hipft_gpu *h) {
  if (!h) return HIPFT_EINVAL;
  h->adj_recs.clear();
  h->adj_top = 0;
  h->adj_rings_n = 0;
  h->adj_free_seen = 0;
  return HIPFT_OK;
}

extern "C" int hipft_adj_recorded(hipft_gpu *h, int64_t *n, int64_t *slots_used) {
  if (!h || !n) return HIPFT_EINVAL;
  *n = (int64_t)h->adj_recs.size();
  if (slots_used) *slots_used = (int64_t)h->adj_top;
  return HIPFT_OK;
}

extern "C" int hipft_adj_tape_fields(hipft_gpu *h, int64_t *n) {
  if (!h || !n) return HIPFT_EINVAL;
  *n = (int64_t)(h->adj_top_max + h->adj_block.size());
  return HIPFT_OK;
}

extern "C" int hipft_adj_set_tape_limit(hipft_gpu *h, int64_t max_fields, int64_t stage_spacing) {
  if (!h || max_fields < 0 || stage_spacing < 0 || stage_spacing % 2) return HIPFT_EINVAL;
  h->adj_tape_limit = max_fields;
  h->adj_force_q = stage_spacing;
  return HIPFT_OK;
}

extern "C" int hipft_adj_release(hipft_gpu *h) {
  if (!h) return HIPFT_EINVAL;
  CK(h, cudaSetDevice(h->dev));
  CK(h, cudaStreamSynchronize(h->stream));
  auto drop = [&](void *p) {
    if (!p) return;
    cudaFree(p);
    h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), p), h->allocs.end());
    h->dev_bytes -= h->fieldn * sizeof(double);
  };
  {
    const size_t fb = h->fieldn * sizeof(double);
    const size_t per = std::max<size_t>(1, std::min<size_t>(32, (size_t)(256u << 20) / fb));
    for (void *q : h->tape_chunks) {
      if (!q) continue;
      cudaFree(q);
      h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), q), h->allocs.end());
      h->dev_bytes -= per * fb;
    }
  }
  for (double *q : h->adj_block) drop(q);
  h->tape.clear();
  h->tape_chunks.clear();
  h->adj_block.clear();
  h->adj_recs.clear();
  h->adj_top = 0;
  h->adj_top_max = 0;
  h->adj_free_seen = 0;
  h->adj_rings_n = 0;
  return HIPFT_OK;
}

extern "C" int hipft_adj_assimilate(hipft_gpu *h, const double *data3_pt, const hipft_da_opts *o, double *fbar) {
  if (!h || !data3_pt || !o || !fbar) return HIPFT_EINVAL;
  if (!o->lat_limit || (o->custom_from_mu && (!o->mu_power || !o->mu_limit)))
    return fail(h, HIPFT_EINVAL, "adj_assimilate: missing per-realization options");
  if (o->balance_flux) return fail(h, HIPFT_ESTATE, "adj_assimilate: the balanced increment is not differentiated");
  CK(h, cudaSetDevice(h->dev));
  DAArgs a;
  TRY(da_args(h, data3_pt, o, a));
  dim3 blk(32, 8), grd((unsigned)((h->ntm + 31) / 32), (unsigned)((h->npm - 2 + 7) / 8), (unsigned)h->nr);
  k_adj_da<<<grd, blk, 0, h->stream>>>(h->M, a, fbar);
  LAUNCHED(h);
  CK(h, cudaStreamSynchronize(h->stream));
  return HIPFT_OK;
}

extern "C" int hipft_adj_assimilate_at(hipft_gpu *h, const double *data3_pt, const hipft_da_opts *o,
                                       const double *f_pre, double *fbar) {
  if (!h || !data3_pt || !o || !fbar) return HIPFT_EINVAL;
  if (!o->balance_flux || o->add) {
    // the plain blend, or an increment that does not depend on f
    hipft_da_opts o2 = *o;
    o2.balance_flux = 0;
    return hipft_adj_assimilate(h, data3_pt, &o2, fbar);
  }
  if (!f_pre) return fail(h, HIPFT_EINVAL, "adj_assimilate_at: the balanced increment needs the field it was applied to");
  if (!o->lat_limit || (o->custom_from_mu && (!o->mu_power || !o->mu_limit)))
    return fail(h, HIPFT_EINVAL, "adj_assimilate_at: missing per-realization options");
  CK(h, cudaSetDevice(h->dev));
  const int ntm = h->ntm, npm1 = h->npm1, nr = h->nr;
  DAArgs a;
  TRY(da_args(h, data3_pt, o, a));
  if (!h->d_adj_delta) TRY(dalloc(h, &h->d_adj_delta, h->fieldn));
  double *delta = h->d_adj_delta;
  dim3 blk(32, 8), grd((unsigned)((ntm + 31) / 32), (unsigned)((npm1 + 31) / 32), (unsigned)nr);
  k_da_delta<<<grd, blk, 0, h->stream>>>(h->M, a, f_pre, delta);
  LAUNCHED(h);
  // F+, F- exactly as the forward's balance (same kernel, same block order),
  // then SP, SN over the core columns
  const int cpb = 16, nb = (h->npm - 1 + cpb - 1) / cpb, nb2 = (h->npm - 2 + cpb - 1) / cpb;
  TRY(ensure_part(h, (size_t)nr * (nb + nb2) * 2 + 4 * (size_t)nr));
  const double *da_t = h->d_anw, *da_p = h->d_anw + 3 * ((size_t)std::max(ntm, h->npm) + 1);
  double *pf = h->d_part, *ps = h->d_part + (size_t)nr * nb * 2, *dcoef = ps + (size_t)nr * nb2 * 2;
  k_flux_partial<<<dim3((unsigned)nb, (unsigned)nr), 256, 0, h->stream>>>(h->M, da_t, da_p, delta, 1, pf, cpb);
  LAUNCHED(h);
  k_adj_bal_partial<<<dim3((unsigned)nb2, (unsigned)nr), 256, 0, h->stream>>>(h->M, delta, fbar, cpb, ps);
  LAUNCHED(h);
  std::vector<double> part((size_t)nr * (nb + nb2) * 2);
  CK(h, cudaMemcpyAsync(part.data(), h->d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  std::vector<double> coef(4 * (size_t)nr);
  for (int i = 0; i < nr; ++i) {
    double fp = 0.0, fm = 0.0, sp = 0.0, sn = 0.0;
    for (int q = 0; q < nb; ++q) {
      fp = fp + part[((size_t)i * nb + q) * 2];
      fm = fm + part[((size_t)i * nb + q) * 2 + 1];
    }
    const double *p2 = part.data() + (size_t)nr * nb * 2;
    for (int q = 0; q < nb2; ++q) {
      sp = sp + p2[((size_t)i * nb2 + q) * 2];
      sn = sn + p2[((size_t)i * nb2 + q) * 2 + 1];
    }
    double *c = coef.data() + 4 * (size_t)i;
    if (fm + fp == 0.0) {  // the forward leaves the increment as it is
      c[0] = c[1] = 1.0;
      c[2] = c[3] = 0.0;
      continue;
    }
    if (fp == 0.0 || fm == 0.0)
      return fail(h, HIPFT_ESTATE, "adj_assimilate_at: realization %d: one-signed balanced increment", i + 1);
    const double r = std::sqrt(std::fabs(fp / fm));
    const double S = -sp / (r * r) + sn;
    c[0] = 1.0 / r;
    c[1] = r;
    c[2] = S * r / (2.0 * fp);
    c[3] = -S * r / (2.0 * fm);
  }
  TRY(upload(h, dcoef, coef));
  dim3 g2((unsigned)((ntm + 31) / 32), (unsigned)((h->npm - 2 + 7) / 8), (unsigned)nr);
  k_adj_da_bal<<<g2, blk, 0, h->stream>>>(h->M, a, delta, da_t, da_p, dcoef, fbar);
  LAUNCHED(h);
  CK(h, cudaStreamSynchronize(h->stream));
  return HIPFT_OK;
}

extern "C" int hipft_gpu_set_field_device(hipft_gpu *h, const double *f_dev) {
  if (!h || !f_dev) return HIPFT_EINVAL;
  if (!h->field_set) return fail(h, HIPFT_ESTATE, "set_field_device before set_field");
  CK(h, cudaSetDevice(h->dev));
  CK(h, cudaMemcpyAsync(h->buf[h->cur], f_dev, h->fieldn * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  h->dring_valid = false;
  CK(h, cudaStreamSynchronize(h->stream));
  return HIPFT_OK;
}
