// graph_step.cuh -- device-side scheduling of a flux-transport step that runs
// as one CUDA graph.
//
// The host-driven step (hipft_gpu.cu) reads small results back between
// launches: the PTL limit of every subcycle (get_dtime_diffusion_ptl,
// src/hipft.f90:5042-5161), from which the subcycle length and the RKG2/RKL2
// stage count follow (src/hipft.f90:4551-4695, 5361-5475).  Here those
// decisions are made by one-block "schedule" kernels that leave their results
// in device memory, and the loops whose trip counts they decide (subcycles,
// stage pairs, advection substeps) are conditional WHILE nodes of the graph,
// continued or ended by cudaGraphSetConditional from the kernel that closes
// each iteration.  The arithmetic of every decision is the host path's (same
// expressions, same order), so a graph-run step and a host-driven step give
// the same bits.
#pragma once

#include <cfloat>

namespace hipft {

constexpr int kGUnrollMax = 16;      // most stage pairs per iteration of the pair loop (an even number: buffer roles repeat)
constexpr int kGMaxCycles = 60;      // max_sc of diffusion_step (src/hipft.f90:4565)
constexpr int kGAdvLimit = 100000;   // advection substeps after which the loop stops and reports an error
constexpr int kGSubLimit = 1000;     // subcycles likewise (PTL forces the last one at kGMaxCycles - 1)

// Scalars of one graph-run step (device memory).  The host writes dt before
// each launch and reads the statistics afterwards.
struct GState {
  double dt;                // the split step
  int cyc;                  // diffusion subcycle (1-based)
  int nact;                 // realizations still subcycling
  int npairs;               // stage pairs of the longest super-step of this subcycle
  int pctr;                 // first stage pair of the current pair-loop iteration
  int nsub;                 // advection substeps of the slowest realization
  int qctr;                 // current advection substep
  int err;                  // 1: a table was too small, 2: a loop hit its iteration limit
  int cycles;               // subcycles of the step
  long long stage_sum;      // sum over super-steps and realizations of s_i
  long long rkg2_sum;       // the same for stages k >= 2
  long long smax;           // largest s of the step
  long long adv_slices;     // realization-stages of advection
  long long kernels;        // kernels the step ran
};

// Per-realization and per-pair arrays of the schedule, and the mode.
struct GArrays {
  GState *st;
  double *ts, *d;                 // [nr] time subcycled so far, current subcycle length
  const double *dt_euler;         // [nr] Euler limits (one shared value in plain mode)
  const double *dtmax;            // [nr] flow CFL limits (ragged advection)
  double *rdt;                    // [nr] advection substep length
  int *act, *fin;                 // [nr] still subcycling / finishing this subcycle
  int *rl_ptl;                    // [nr] active realizations, -1 after the last
  int *rl_dif;                    // [nr] active realizations by stage count (descending), -1 after the last
  int *rl_adv, *rl_adv_all;       // [nr] realizations of the current advection substep (-1 padded), all by substeps
  int *nsub_i, *cycles_i;         // [nr] advection substeps, subcycles run
  int *nactp;                     // [paircap] realizations taking part in stage pair p
  long long *s_i, *s_last;        // [nr] stage count of the current / last super-step
  StageCoef *c1;                  // [nr] stage-1 coefficients
  StageCoef *rc;                  // [paircap][nr][2] stage-pair coefficients
  unsigned long long *bits;       // PTL reductions: [2 nr] ragged, [2] plain
  double *ring0, *ring1;          // diffusion ring sums of stage inputs / outputs
  int nr, paircap;
  int method, auto_sc, subcycles, ragged, strang, nadv;  // nadv: advection stages per substep
  int unroll;                     // stage pairs per pair-loop iteration (even)
};

__device__ __forceinline__ double bits_to_double(unsigned long long b) { return __longlong_as_double((long long)b); }

// Start of a step: statistics reset.
__global__ void k_g_step_begin(GArrays g) {
  if (threadIdx.x == 0) {
    GState &s = *g.st;
    s.err = 0;
    s.cycles = 0;
    s.stage_sum = 0;
    s.rkg2_sum = 0;
    s.smax = 0;
    s.adv_slices = 0;
    s.kernels = 1;
  }
}

// Rank of realization i in the order (key descending, index ascending) among
// the realizations with on[j] != 0.
template <typename K>
__device__ __forceinline__ int g_rank(const K *key, const int *on, int nr, int i) {
  const K ki = key[i];
  int r = 0;
  for (int j = 0; j < nr; ++j)
    if (on[j]) r += (key[j] > ki || (key[j] == ki && j < i)) ? 1 : 0;
  return r;
}

// Advection substeps of every realization (advection_step, src/hipft.f90:
// 4509-4549; a ragged batch gives realization i ceil(dt / its CFL limit)
// substeps), their lengths, and the list of the first substep.  One block.
__global__ void k_g_adv_plan(GArrays g, double frac, cudaGraphConditionalHandle hc) {
  GState &st = *g.st;
  const int nr = g.nr, tid = threadIdx.x;
  const double dta = frac * st.dt;
  __shared__ int s_max;
  __shared__ long long s_sum;
  if (tid == 0) {
    s_max = 1;
    s_sum = 0;
  }
  __syncthreads();
  for (int i = tid; i < nr; i += blockDim.x) {
    int n = 1;
    if (g.ragged) {
      const double r = dta * (g.strang ? 2.0 : 1.0) / g.dtmax[i];
      n = (r > 1.0) ? (int)ceil(r) : 1;
    }
    g.nsub_i[i] = n;
    g.rdt[i] = dta / (double)n;
    g.act[i] = 1;
    atomicMax(&s_max, n);
    atomicAdd((unsigned long long *)&s_sum, (unsigned long long)n);
  }
  __syncthreads();
  for (int i = tid; i < nr; i += blockDim.x) {
    const int r = g_rank(g.nsub_i, g.act, nr, i);
    g.rl_adv_all[r] = i;
    g.rl_adv[r] = i;
  }
  if (tid == 0) {
    st.nsub = s_max;
    st.qctr = 0;
    st.adv_slices += s_sum * g.nadv;
    st.kernels += 1;
    cudaGraphSetConditional(hc, 1u);
  }
}

// End of an advection substep (body_kernels: the kernels of one substep,
// this one included): the next substep's list, or the loop's end.
__global__ void k_g_adv_tick(GArrays g, int body_kernels, cudaGraphConditionalHandle hc) {
  GState &st = *g.st;
  const int q = st.qctr + 1;
  for (int e = threadIdx.x; e < g.nr; e += blockDim.x) {
    const int i = g.rl_adv_all[e];
    g.rl_adv[e] = (g.nsub_i[i] > q) ? i : -1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    st.qctr = q;
    st.kernels += body_kernels;
    bool more = q < st.nsub;
    if (more && q >= kGAdvLimit) {
      st.err = 2;
      more = false;
    }
    cudaGraphSetConditional(hc, more ? 1u : 0u);
  }
}

// Start of a diffusion step (src/hipft.f90:4551-4570): every realization
// subcycles, from time 0, with the fixed subcycle length or (PTL) a floor of 0.
// extra_kernels: kernels of the step outside the loops, counted here.
__global__ void k_g_dif_begin(GArrays g, int extra_kernels, cudaGraphConditionalHandle hc) {
  GState &st = *g.st;
  const double dtl = st.dt;
  for (int i = threadIdx.x; i < g.nr; i += blockDim.x) {
    g.ts[i] = 0.0;
    g.act[i] = 1;
    g.d[i] = g.auto_sc ? 0.0 : dtl / (double)g.subcycles;
    g.rl_ptl[i] = i;
  }
  if (threadIdx.x == 0) {
    st.cyc = 1;
    st.nact = g.nr;
    st.kernels += 1 + extra_kernels;
    cudaGraphSetConditional(hc, 1u);
  }
}

// Initial values of the PTL reductions (max |Af| from 0, the minimum from the
// largest finite double).
__global__ void k_g_ptl_reset(GArrays g) {
  const int n = g.ragged ? g.nr : 1;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    g.bits[i] = 0ULL;
    g.bits[n + i] = 0x7fefffffffffffffULL;
  }
  if (threadIdx.x == 0) g.st->kernels += 1;
}

// One subcycle's schedule (one block): each active realization's subcycle
// length from its PTL limit or the fixed count (the decisions of
// hipft_gpu_diffusion_step / ragged_diffusion_step in their order), its stage
// count and stage-1 coefficients, the realizations sorted by stage count, and
// how many take part in each stage pair.  Plain mode reads one shared PTL
// limit and one Euler limit, so every realization gets the same schedule.
__global__ void __launch_bounds__(256) k_g_plan(GArrays g, cudaGraphConditionalHandle hpair) {
  GState &st = *g.st;
  const int nr = g.nr, tid = threadIdx.x;
  const double dtl = st.dt;
  const int cyc = st.cyc;
  __shared__ int s_na, s_pmax;
  __shared__ long long s_ssum, s_smax;
  if (tid == 0) {
    s_na = 0;
    s_pmax = 0;
    s_ssum = 0;
    s_smax = 0;
  }
  __syncthreads();
  for (int i = tid; i < nr; i += blockDim.x) {
    if (!g.act[i]) {
      g.s_i[i] = 0;
      continue;
    }
    double d = g.d[i];
    if (g.auto_sc) {
      const double axm = bits_to_double(g.ragged ? g.bits[i] : g.bits[0]);
      const double ptl = bits_to_double(g.ragged ? g.bits[nr + i] : g.bits[1]);
      double dd = DBL_MAX;
      if (axm > 0.0) {
        dd = 0.95 * ptl;
        if (dd < d) dd = d;
      }
      d = dd;
    }
    int fin = 0;
    if (g.auto_sc && g.ts[i] + d >= dtl) {
      d = dtl - g.ts[i];
      fin = 1;
    }
    if (g.auto_sc && cyc == kGMaxCycles - 1) {
      d = dtl - g.ts[i];
      fin = 1;
    }
    if (!g.auto_sc && cyc == g.subcycles) fin = 1;
    g.d[i] = d;
    g.fin[i] = fin;
    const long long s = sts_count(g.method, d, g.dt_euler[i]);
    g.s_i[i] = s;
    g.s_last[i] = s;
    g.cycles_i[i] = cyc;
    double uj, vj, ubj, gj;
    sts_stage(g.method, s, 1, uj, vj, ubj, gj);
    g.c1[i] = StageCoef{d, ubj, 0.0, 0.0, 0.0};
    atomicAdd(&s_na, 1);
    atomicMax(&s_pmax, (int)((s - 1) / 2));
    atomicAdd((unsigned long long *)&s_ssum, (unsigned long long)s);
    atomicMax((unsigned long long *)&s_smax, (unsigned long long)s);
  }
  __syncthreads();
  for (int i = tid; i < nr; i += blockDim.x)
    if (g.act[i]) g.rl_dif[g_rank(g.s_i, g.act, nr, i)] = i;
  __syncthreads();
  const int na = s_na;
  for (int e = na + tid; e < nr; e += blockDim.x) g.rl_dif[e] = -1;
  int np = s_pmax;
  const bool fits = np + g.unroll <= g.paircap;
  if (!fits) np = 0;
  for (int p = tid; p < np + g.unroll; p += blockDim.x) {
    int c = 0;
    for (int e = 0; e < na; ++e) c += ((g.s_i[g.rl_dif[e]] - 1) / 2 > p) ? 1 : 0;
    g.nactp[p] = c;
  }
  if (tid == 0) {
    st.npairs = np;
    st.pctr = 0;
    if (!fits) st.err = 1;
    st.stage_sum += s_ssum;
    st.rkg2_sum += s_ssum - na;
    if (s_smax > st.smax) st.smax = s_smax;
    st.cycles = cyc;
    st.kernels += 1;
    cudaGraphSetConditional(hpair, np > 0 ? 1u : 0u);
  }
}

// Stage-pair coefficients of the subcycle (src/hipft.f90:5224-5235): entry
// (p, i) holds stages 2p+2 and 2p+3 of realization i.  Grid over paircap x nr.
__global__ void k_g_coefs(GArrays g) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx == 0) g.st->kernels += 1;
  const int nr = g.nr;
  const int p = (int)(idx / nr), i = (int)(idx % nr);
  if (p >= g.st->npairs || !g.act[i]) return;
  const long long s = g.s_i[i];
  if (p >= (s - 1) / 2) return;
  const long long k = 2 + 2 * (long long)p;
  g.rc[idx * 2] = sts_combine(g.method, s, k, g.d[i]);
  g.rc[idx * 2 + 1] = sts_combine(g.method, s, k + 1, g.d[i]);
}

// End of a pair-loop iteration (one thread).
__global__ void k_g_pair_tick(GArrays g, cudaGraphConditionalHandle hc) {
  GState &st = *g.st;
  const int p = st.pctr + g.unroll;
  st.pctr = p;
  st.kernels += 2 * g.unroll + 1;
  // npairs fits the tables (k_g_plan), so the loop ends within paircap / unroll iterations
  cudaGraphSetConditional(hc, p < st.npairs ? 1u : 0u);
}

// After the pair loop: each realization of the super-step has Y_s in y_even
// (its last pair had an even index) or y_odd; the plane goes back into the
// field buffer.  In plain mode the ring sums of Y_s move to ring0 as well
// (the host path reuses the fused kernels' ring sums in the next subcycle;
// ragged batches recompute them).  Grid (nr, chunks).
__global__ void k_g_gather(GArrays g, Mesh m, double *f, const double *__restrict__ y_even,
                           const double *__restrict__ y_odd) {
  const int i = blockIdx.x;
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) g.st->kernels += 1;
  if (!g.act[i]) return;
  const long long P = (g.s_i[i] - 1) / 2;
  const bool odd = ((P - 1) & 1) != 0;
  const double *src = (odd ? y_odd : y_even) + (int64_t)i * m.plane;
  double *dst = f + (int64_t)i * m.plane;
  const int64_t n2 = m.plane / 2;
  const double2 *s2 = reinterpret_cast<const double2 *>(src);
  double2 *d2 = reinterpret_cast<double2 *>(dst);
  for (int64_t e = (int64_t)blockIdx.y * blockDim.x + threadIdx.x; e < n2; e += (int64_t)gridDim.y * blockDim.x)
    d2[e] = s2[e];
  if (!g.ragged && odd && blockIdx.y == 0 && threadIdx.x < 2) g.ring0[2 * i + threadIdx.x] = g.ring1[2 * i + threadIdx.x];
}

// dst = src over whole fields (n doubles, n even; 16-byte aligned).
__global__ void k_g_copy(double *__restrict__ dst, const double *__restrict__ src, int64_t n) {
  const int64_t n2 = n / 2;
  const double2 *s2 = reinterpret_cast<const double2 *>(src);
  double2 *d2 = reinterpret_cast<double2 *>(dst);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n2; e += (int64_t)gridDim.x * blockDim.x)
    d2[e] = s2[e];
}

// End of a subcycle (one block): time stepped, finished realizations leave,
// the next subcycle's list; the loop ends when none is left.
__global__ void k_g_sub_tick(GArrays g, int body_kernels, cudaGraphConditionalHandle hc) {
  GState &st = *g.st;
  const int nr = g.nr, tid = threadIdx.x;
  __shared__ int s_na;
  if (tid == 0) s_na = 0;
  __syncthreads();
  for (int i = tid; i < nr; i += blockDim.x) {
    if (g.act[i]) {
      g.ts[i] = g.ts[i] + g.d[i];
      if (g.fin[i]) g.act[i] = 0;
    }
    if (g.act[i]) atomicAdd(&s_na, 1);
  }
  __syncthreads();
  for (int i = tid; i < nr; i += blockDim.x)
    if (g.act[i]) {
      int r = 0;
      for (int j = 0; j < i; ++j) r += g.act[j] ? 1 : 0;
      g.rl_ptl[r] = i;
    }
  for (int e = s_na + tid; e < nr; e += blockDim.x) g.rl_ptl[e] = -1;
  if (tid == 0) {
    const int c = st.cyc + 1;
    st.cyc = c;
    st.nact = s_na;
    st.kernels += body_kernels;
    bool more = s_na > 0;
    if (more && c >= kGSubLimit) {
      st.err = 2;
      more = false;
    }
    cudaGraphSetConditional(hc, more ? 1u : 0u);
  }
}

}  // namespace hipft
