// kernels.cuh -- device code of the flux-transport step (sm_100a, FP64).
//
// Layout: a field is f(j,k,i) with j = theta (1..ntm), k = phi (1..npm,
// two-point periodic overlap), i = realization (1..nr), stored theta-fastest
// with a padded theta stride `ldt` (a multiple of 16 doubles, 128 B) so every
// phi column starts on a 128-byte boundary.  Index formulas below keep the
// reference's 1-based j,k,i so each expression can be read against
// src/hipft.f90 line by line; 1-D mesh arrays are stored with an unused
// element 0 for the same reason.
//
// Every arithmetic expression is written in the reference's left-to-right
// order and the library is compiled with --fmad=false, so stencil values are
// bit-identical to the CPU restatement given identical inputs.  The only
// order-dependent operations are the ring sums at the poles and the
// diagnostic sums; both use a fixed reduction tree (deterministic run to run).
#pragma once
#include <cstdint>

namespace hipft {

constexpr double kHalf = 0.5;
constexpr double kOne = 1.0;
constexpr double kTwoPiI = 0.15915494309189535;  // twopi_i, src/hipft.f90:111
constexpr double kTwo = 2.0;
constexpr double kFour = 4.0;

// ---------------------------------------------------------------- meshes
struct Mesh {
  int ntm, npm, nt, np, nr, ldt;
  int64_t plane;  // ldt * npm
  // 1-based device arrays (element 0 unused)
  const double *dt_i, *dth_i, *dp_i, *dph_i, *st_i, *sth, *dp, *dth, *dph;
};

__device__ __forceinline__ int64_t fidx(const Mesh &m, int j, int k, int i) {
  return (int64_t)(i - 1) * m.plane + (int64_t)(k - 1) * m.ldt + (j - 1);
}

// ------------------------------------------------------------ diffusion
// Diffusion coefficient on the half-half mesh, load_diffusion
// (src/hipft.f90:6687-6820): factor * (constant [+ grid term]).
struct DiffCoef {
  const double *dfac;  // [nr+1] factor*constant (no grid) or constant (grid)
  double factor;
  int grid;
};

__device__ __forceinline__ double dcoef(const Mesh &m, const DiffCoef &c, int j, int k, int i) {
  if (!c.grid) return c.dfac[i];
  double a = m.dth[j], b = m.dph[k] * m.sth[j];
  return c.factor * (c.dfac[i] + (a * a + b * b));
}

// 5-point coefficients, load_diffusion_matrix (src/hipft.f90:4958-4980).
struct Coef5 {
  double c1, c2, c3, c4, c5;
};

__device__ __forceinline__ Coef5 coef5(const Mesh &m, const DiffCoef &c, int j, int k, int i) {
  double Djk = dcoef(m, c, j, k, i), Dj1k = dcoef(m, c, j + 1, k, i);
  double Djk1 = dcoef(m, c, j, k + 1, i), Dj1k1 = dcoef(m, c, j + 1, k + 1, i);
  Coef5 r;
  r.c1 = kHalf * (Djk + Dj1k) * m.dph_i[k] * m.dp_i[k] * m.st_i[j] * m.st_i[j];
  r.c2 = kHalf * (Djk + Djk1) * m.dth_i[j] * m.dt_i[j] * m.st_i[j] * m.sth[j];
  r.c4 = kHalf * (Dj1k + Dj1k1) * m.dth_i[j + 1] * m.dt_i[j] * m.st_i[j] * m.sth[j + 1];
  r.c5 = kHalf * (Djk1 + Dj1k1) * m.dph_i[k + 1] * m.dp_i[k] * m.st_i[j] * m.st_i[j];
  r.c3 = -(r.c1 + r.c2 + r.c4 + r.c5);
  return r;
}

// Deterministic block sum of two values (blockDim.x*blockDim.y threads,
// multiple of 32, at most 1024).  Result valid in thread 0.
__device__ __forceinline__ void block_sum2(double &a, double &b, double *sh) {
  const int tid = threadIdx.x + threadIdx.y * blockDim.x;
  const int nthr = blockDim.x * blockDim.y;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int w = tid >> 5, l = tid & 31, nw = nthr >> 5;
  if (l == 0) {
    sh[2 * w] = a;
    sh[2 * w + 1] = b;
  }
  __syncthreads();
  if (w == 0) {
    a = (l < nw) ? sh[2 * l] : 0.0;
    b = (l < nw) ? sh[2 * l + 1] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
  }
  __syncthreads();
}

// Pole ring sums of the diffusion operator, diffusion_operator_cd
// (src/hipft.f90:7969-7979).  One block per realization; ring[2(i-1)] = fn,
// ring[2(i-1)+1] = fs.
__global__ void k_ring_diffusion(Mesh m, DiffCoef c, const double *__restrict__ x,
                                 double *__restrict__ ring) {
  __shared__ double sh[64];
  const int i = blockIdx.x + 1;
  double fn = 0.0, fs = 0.0;
  for (int k = 2 + threadIdx.x; k <= m.npm - 1; k += blockDim.x) {
    double x1 = x[fidx(m, 1, k, i)], x2 = x[fidx(m, 2, k, i)];
    double xa = x[fidx(m, m.ntm - 1, k, i)], xb = x[fidx(m, m.ntm, k, i)];
    fn = fn + (dcoef(m, c, 1, k, i) + dcoef(m, c, 2, k, i)) * (x2 - x1) * m.dp[k];
    fs = fs + (dcoef(m, c, m.nt - 1, k, i) + dcoef(m, c, m.nt, k, i)) * (xb - xa) * m.dp[k];
  }
  block_sum2(fn, fs, sh);
  if (threadIdx.x == 0) {
    ring[2 * (i - 1)] = fn;
    ring[2 * (i - 1) + 1] = fs;
  }
}

// One diffusion stage: y = A x at (j,k,i) fused with the stage combine.
//   MODE_AX    : out = A x                          (PTL's Af, F:5097)
//   MODE_STS1  : out2 = dt*(A x); out = x + ubj1*out2 (F:5211-5218)
//   MODE_STSK  : out = uj*x + vj*ykm2 + c*u0 + ubjdt*(A x) + gj*dty0, written
//                over ykm2 (F:5224-5235)
//   MODE_EULER : out = x + dte*(A x)                  (F:7396-7399)
enum { MODE_AX = 0, MODE_STS1 = 1, MODE_STSK = 2, MODE_EULER = 3 };

struct StageCoef {
  double a, b, c, d, e;  // meaning depends on the mode
};

// RKL2 (method 2) / RKG2 (method 3) super-step recurrences, load_sts_rkl2 /
// load_sts_rkg2 (src/hipft.f90:5244-5475).  Host and device evaluate the same
// expressions (no contraction), so a schedule built on either side has the
// same bits.
__host__ __device__ inline int64_t sts_count(int method, double dtl, double dt_euler) {
  int64_t s;
  if (method == 2)
    s = (int64_t)ceil(0.5 * (sqrt(9.0 + 16.0 * (dtl / dt_euler)) - 1.0));
  else
    s = (int64_t)ceil(0.5 * (sqrt(25.0 + 24.0 * (dtl / dt_euler)) - 3.0));
  if (s < 3) s = 3;
  if (s % 2 == 0) s = s + 1;
  return s;
}

__host__ __device__ inline double sts_b(int method, int64_t j) {
  if (method == 2) {
    if (j <= 2) return 1.0 / 3.0;
    return ((double)(j * j + j) - 2.0) / (2.0 * (double)j * (double)(j + 1));
  }
  if (j <= 1) return 1.0 / 3.0;
  if (j == 2) return 1.0 / 15.0;
  return (4.0 * (double)(j - 1) * (double)(j + 4)) /
         (3.0 * (double)j * (double)(j + 1) * (double)(j + 2) * (double)(j + 3));
}

// mu_j, nu_j, mu~_j, gamma~_j of stage j of an s-stage super-step; j = 1
// gives mu~_1 (the others are unused there).
__host__ __device__ inline void sts_stage(int method, int64_t s, int64_t j, double &uj, double &vj, double &ubj,
                                          double &gj) {
  if (method == 2) {
    const double w = 4.0 / (double)(s * s + s - 2);
    if (j == 1) {
      uj = -9999.0; vj = -9999.0; ubj = 4.0 / (3.0 * (double)(s * s + s - 2)); gj = -9999.0;
    } else if (j == 2) {
      uj = 3.0 / 2.0; vj = -0.5; ubj = uj * w; gj = -w;
    } else {
      const double b = sts_b(2, j), r1 = b / sts_b(2, j - 1), r2 = b / sts_b(2, j - 2);
      uj = r1 * (2.0 - 1.0 / (double)j);
      vj = r2 * (1.0 / (double)j - 1.0);
      ubj = uj * w;
      gj = (sts_b(2, j - 1) - 1.0) * ubj;
    }
    return;
  }
  const double w = 6.0 / (double)((s + 4) * (s - 1));
  if (j == 1) {
    uj = 1.0; vj = -9999.0; ubj = w; gj = -9999.0;
  } else if (j == 2) {
    uj = 1.0 / 2.0; vj = -1.0 / 10.0; ubj = uj * w; gj = 0.0;
  } else {
    const double b = sts_b(3, j), r1 = b / sts_b(3, j - 1), r2 = b / sts_b(3, j - 2);
    uj = r1 * (2.0 + 1.0 / (double)j);
    vj = -r2 * (1.0 / (double)j + 1.0);
    ubj = uj * w;
    gj = (0.5 * (double)j * ((double)j + 1.0) * sts_b(3, j - 1) - 1.0) * ubj;
  }
}

// The stage-k combine of a super-step of length dtl (src/hipft.f90:5224-5235).
__host__ __device__ inline StageCoef sts_combine(int method, int64_t s, int64_t k, double dtl) {
  double uj, vj, ubj, gj;
  sts_stage(method, s, k, uj, vj, ubj, gj);
  return StageCoef{uj, vj, 1.0 - uj - vj, ubj * dtl, gj};
}

// rlist (may be null): realization (0-based) of grid slice z, for ragged
// batches that advance a subset (a negative entry: the slice does nothing);
// per_real: one max |Af| per realization.
template <int MODE>
__global__ void __launch_bounds__(256) k_diffusion_stage(
    Mesh m, DiffCoef dc, const double *__restrict__ x, const double *ykm2, const double *__restrict__ u0,
    const double *__restrict__ dty0, double *out, double *out2, const double *__restrict__ ring, double bcn,
    double bcs, StageCoef sc, unsigned long long *absmax_bits, const int *__restrict__ rlist = nullptr,
    int per_real = 0) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 2;
  if (rlist && rlist[blockIdx.z] < 0) return;  // slot past the list's end
  const int i = (rlist ? rlist[blockIdx.z] : (int)blockIdx.z) + 1;
  double ax = 0.0;
  bool active = (j <= m.ntm && k <= m.npm - 1);
  int64_t q = 0;
  if (active) {
    q = fidx(m, j, k, i);
    if (j == 1) {
      ax = ring[2 * (i - 1)] * bcn;
    } else if (j == m.ntm) {
      ax = -ring[2 * (i - 1) + 1] * bcs;
    } else {
      Coef5 cf = coef5(m, dc, j, k, i);
      ax = cf.c1 * x[q - m.ldt] + cf.c2 * x[q - 1] + cf.c3 * x[q] + cf.c4 * x[q + 1] + cf.c5 * x[q + m.ldt];
    }
    double y;
    if (MODE == MODE_AX) {
      y = ax;
    } else if (MODE == MODE_STS1) {
      double d0 = sc.a * ax;  // dt * (A f)
      y = x[q] + sc.b * d0;   // f + ubj(1)*dty0
      out2[q] = d0;
      if (k == 2) out2[q + (int64_t)(m.npm - 2) * m.ldt] = d0;
      if (k == m.npm - 1) out2[q - (int64_t)(m.npm - 2) * m.ldt] = d0;
    } else if (MODE == MODE_STSK) {
      y = sc.a * x[q] + sc.b * ykm2[q] + sc.c * u0[q] + sc.d * ax + sc.e * dty0[q];
    } else {
      y = x[q] + sc.a * ax;
    }
    out[q] = y;
    if (k == 2) out[q + (int64_t)(m.npm - 2) * m.ldt] = y;
    if (k == m.npm - 1) out[q - (int64_t)(m.npm - 2) * m.ldt] = y;
  }
  if (MODE == MODE_AX && absmax_bits) {
    // max |Af| over |f| > fmin (src/hipft.f90:5097-5102): non-negative
    // doubles order like their bit patterns.
    double v = (active && fabs(x[q]) > 1e-14) ? fabs(ax) : 0.0;
    unsigned long long b = __double_as_longlong(v);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      unsigned long long t = __shfl_down_sync(0xffffffffu, b, o);
      b = t > b ? t : b;
    }
    if ((threadIdx.x & 31) == 0 && b) atomicMax(absmax_bits + (per_real ? i - 1 : 0), b);
  }
}

// PTL candidates at the argmax cells (src/hipft.f90:5108-5135).  With
// per_real, each realization has its own maximum and its own minimum (ragged
// batches); rlist as in k_diffusion_stage.
__global__ void k_ptl(Mesh m, const double *__restrict__ f, const double *__restrict__ af,
                      const unsigned long long *absmax_bits, unsigned long long *ptl_bits,
                      const int *__restrict__ rlist = nullptr, int per_real = 0) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 2;
  if (rlist && rlist[blockIdx.z] < 0) return;  // slot past the list's end
  const int i = (rlist ? rlist[blockIdx.z] : (int)blockIdx.z) + 1;
  if (j < 2 || j > m.ntm - 1 || k > m.npm - 1) return;
  const double fmin_v = 1e-14;
  if (per_real) {
    absmax_bits += i - 1;
    ptl_bits += i - 1;
  }
  double axabsmax = __longlong_as_double(*absmax_bits);
  int64_t q = fidx(m, j, k, i);
  if (!(axabsmax == fabs(af[q]) && fabs(f[q]) > fmin_v)) return;
  double best = 1.7976931348623157e308;
  const int64_t nb[4] = {-1, 1, -(int64_t)m.ldt, (int64_t)m.ldt};
#pragma unroll
  for (int n = 0; n < 4; ++n) {
    double du = f[q] - f[q + nb[n]];
    double df = af[q] - af[q + nb[n]];
    if (du * df < -fmin_v) best = fmin(-du / df, best);
  }
  if (best < 1.7976931348623157e308) atomicMin(ptl_bits, (unsigned long long)__double_as_longlong(best));
}

// Gershgorin bound, get_dtime_diffusion_euler (src/hipft.f90:5019-5025);
// per_real: one bound per realization (ragged batches).
__global__ void k_gershgorin(Mesh m, DiffCoef dc, unsigned long long *max_bits, int per_real = 0) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int i = blockIdx.z + 1;
  double g = 0.0;
  if (j <= m.ntm - 1 && k <= m.npm - 1) {
    Coef5 c = coef5(m, dc, j, k, i);
    g = 0.0;
    g = g + fabs(c.c1);
    g = g + fabs(c.c2);
    g = g + fabs(c.c3);
    g = g + fabs(c.c4);
    g = g + fabs(c.c5);
  }
  unsigned long long b = __double_as_longlong(g);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long t = __shfl_down_sync(0xffffffffu, b, o);
    b = t > b ? t : b;
  }
  if ((threadIdx.x & 31) == 0 && b) atomicMax(max_bits + (per_real ? i - 1 : 0), b);
}

// ------------------------------------------------------------ advection
// Velocities either as 1-D theta profiles per realization (analytic flows,
// identical in every phi column) or as full 2-D arrays (attenuated or rotated
// flows).  vt lives on theta faces (nt per column), vp on phi faces (np).
struct Flow {
  int flow2d;
  // 1-D: [nr][nt+1] / [nr][ntm+1], 1-based inside each row
  const double *vt1, *vp1, *at1, *ap1;
  // 2-D: vt(nt,npm,nr), vp(ntm,np,nr), at/ap(ntm,npm,nr), all with theta
  // stride ldv >= nt (np == npm, so one plane size serves all four)
  const double *vt, *vp, *at, *ap;
  int ldv;
  int64_t vplane;  // ldv * npm
  double upwind;
};

__device__ __forceinline__ double vt_at(const Mesh &m, const Flow &fl, int j, int k, int i) {
  if (fl.flow2d) return fl.vt[(int64_t)(i - 1) * fl.vplane + (int64_t)(k - 1) * fl.ldv + (j - 1)];
  return fl.vt1[(int64_t)(i - 1) * (m.nt + 1) + j];
}
__device__ __forceinline__ double vp_at(const Mesh &m, const Flow &fl, int j, int k, int i) {
  if (fl.flow2d) return fl.vp[(int64_t)(i - 1) * fl.vplane + (int64_t)(k - 1) * fl.ldv + (j - 1)];
  return fl.vp1[(int64_t)(i - 1) * (m.ntm + 1) + j];
}
__device__ __forceinline__ double at_at(const Mesh &m, const Flow &fl, int j, int k, int i) {
  if (fl.flow2d) return fl.at[(int64_t)(i - 1) * fl.vplane + (int64_t)(k - 1) * fl.ldv + (j - 1)];
  return fl.at1[(int64_t)(i - 1) * (m.ntm + 1) + j];
}
__device__ __forceinline__ double ap_at(const Mesh &m, const Flow &fl, int j, int k, int i) {
  if (fl.flow2d) return fl.ap[(int64_t)(i - 1) * fl.vplane + (int64_t)(k - 1) * fl.ldv + (j - 1)];
  return fl.ap1[(int64_t)(i - 1) * (m.ntm + 1) + j];
}

// 1-D WENO weights (load_weno, src/hipft.f90:6905-6932), 1-based.
struct Weno {
  const double *cpt, *mct, *mt, *cptt, *pt, *mctt, *epst;  // theta: D_C_CPt, D_C_MCt, D_M_Tt, D_CP_Tt, D_P_Tt, D_MC_Tt, eps
  const double *cpp, *mcp, *mp, *cptp, *pp, *mctp, *epsp;  // phi
  // Phi faces k = 2..npm, kPhiTab doubles each at ptab[(k-2)*kPhiTab]: the ten
  // weights in weno_face's argument order (face npm takes face 2's), a flag
  // (1.0 when the linear weights and eps lie in weno_face_nr's range) and
  // dp_i(k) (the cell divergence factor of column k).
  const double *ptab;
};
constexpr int kPhiTab = 12;

// WENO3 face flux (src/hipft.f90:7775-7801).  LN*: LN(j-2), LN(j-1), LN(j);
// LP*: LP(j-1), LP(j), LP(j+1); weights at indices j-1 (m1) and j (0).
// The nonlinear weights are normalised in the reference's order,
// OM = w / (w0 + w1) with w0m = D_P_T(j-1)/e0^2, w1m = D_MC_T(j-1)/e1^2, and
// the face value is sum(OM*p): six divisions per face.  A form with one
// division per side (numerator and denominator multiplied by e0^2 e1^2) is
// the same value in exact arithmetic, but its rounding drifts the 24-hour
// 1024x2048 field by 1.5e-12 relative, above the 1e-12 parity bar.
__device__ __forceinline__ double weno_face(double LNm2, double LNm1, double LN0, double LPm1, double LP0,
                                            double LPp1, double DCMC_m1, double DCMC_0, double DCCP_m1,
                                            double DCCP_0, double DPT_m1, double DMCT_m1, double DMT_0,
                                            double DCPT_0, double eps_m1, double eps_0) {
  double p0m = (kOne + DCMC_m1) * LNm1 - DCMC_m1 * LNm2;
  double p1m = DCMC_0 * LNm1 + DCCP_m1 * LN0;
  double p0p = (kOne + DCCP_0) * LP0 - DCCP_0 * LPp1;
  double p1p = DCCP_m1 * LP0 + DCMC_0 * LPm1;
  double t0 = DCMC_m1 * (LNm1 - LNm2), t1 = DCCP_m1 * (LN0 - LNm1);
  double t2 = DCCP_0 * (LPp1 - LP0), t3 = DCMC_0 * (LP0 - LPm1);
  double e0 = eps_m1 + kFour * (t0 * t0), e1 = eps_m1 + kFour * (t1 * t1);
  double e2 = eps_0 + kFour * (t2 * t2), e3 = eps_0 + kFour * (t3 * t3);
  double w0m = DPT_m1 / (e0 * e0), w1m = DMCT_m1 / (e1 * e1);
  double w0p = DMT_0 / (e2 * e2), w1p = DCPT_0 / (e3 * e3);
  double sm = w0m + w1m, sp = w0p + w1p;
  double um = (w0m / sm) * p0m + (w1m / sm) * p1m;
  double up = (w0p / sp) * p0p + (w1p / sp) * p1p;
  return up + um;
}

// Division by Newton-Raphson refinement, for the marching advection stage.
// recip_nr(b): 1/b rounded to nearest, from the hardware reciprocal estimate
// and three steps y' = y + y (1 - b y), the last of which is Markstein's
// correctly rounding step; quot_nr(a, b, y): a/b rounded to nearest, from
// q = a y and two corrections q' = q + (a - b q) y whose residuals the fused
// multiply-add computes exactly (P. Markstein, IBM J. Res. Dev. 34(1), 1990;
// J.-M. Muller et al., Handbook of Floating-Point Arithmetic, ch. 4).  The
// quotient of two doubles is never a rounding midpoint, so the result is the
// IEEE quotient whenever operands, reciprocals and quotients stay well inside
// the normal range; weno_face_nr checks that range and its caller falls back
// to weno_face otherwise.  Compared bit for bit with the IEEE division by the
// tile-kernel comparison in tests/test_gpu_adv_march.py.
__device__ __forceinline__ double recip_nr(double b) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
  double e = fma(-b, y, kOne);
  y = fma(y, e, y);
  e = fma(-b, y, kOne);
  y = fma(y, e, y);
  e = fma(-b, y, kOne);
  return fma(y, e, y);
}
__device__ __forceinline__ double quot_nr(double a, double b, double y) {
  double q = a * y;
  double r = fma(-b, q, a);
  q = fma(r, y, q);
  r = fma(-b, q, a);
  return fma(r, y, q);
}

// weno_face with the divisions of quot_nr (the two normalising divisions of
// each side share one reciprocal).  The smoothness denominators are
// e = eps + 4 t^2 >= eps; ok is cleared unless every e is at most 2^100.  With
// eps and the linear weights in [2^-100, 2^100] (weno_consts_ok, checked by
// the caller) every operand, reciprocal and quotient is then a normal double
// and the face equals weno_face's bit for bit.
__device__ __forceinline__ double weno_face_nr(double LNm2, double LNm1, double LN0, double LPm1, double LP0,
                                               double LPp1, double DCMC_m1, double DCMC_0, double DCCP_m1,
                                               double DCCP_0, double DPT_m1, double DMCT_m1, double DMT_0,
                                               double DCPT_0, double eps_m1, double eps_0, bool &ok) {
  double p0m = (kOne + DCMC_m1) * LNm1 - DCMC_m1 * LNm2;
  double p1m = DCMC_0 * LNm1 + DCCP_m1 * LN0;
  double p0p = (kOne + DCCP_0) * LP0 - DCCP_0 * LPp1;
  double p1p = DCCP_m1 * LP0 + DCMC_0 * LPm1;
  double t0 = DCMC_m1 * (LNm1 - LNm2), t1 = DCCP_m1 * (LN0 - LNm1);
  double t2 = DCCP_0 * (LPp1 - LP0), t3 = DCMC_0 * (LP0 - LPm1);
  double e0 = eps_m1 + kFour * (t0 * t0), e1 = eps_m1 + kFour * (t1 * t1);
  double e2 = eps_0 + kFour * (t2 * t2), e3 = eps_0 + kFour * (t3 * t3);
  ok = fmax(fmax(e0, e1), fmax(e2, e3)) <= 0x1p100;
  const double s0 = e0 * e0, s1 = e1 * e1, s2 = e2 * e2, s3 = e3 * e3;
  double w0m = quot_nr(DPT_m1, s0, recip_nr(s0)), w1m = quot_nr(DMCT_m1, s1, recip_nr(s1));
  double w0p = quot_nr(DMT_0, s2, recip_nr(s2)), w1p = quot_nr(DCPT_0, s3, recip_nr(s3));
  double sm = w0m + w1m, sp = w0p + w1p;
  const double ym = recip_nr(sm), yp = recip_nr(sp);
  double um = quot_nr(w0m, sm, ym) * p0m + quot_nr(w1m, sm, ym) * p1m;
  double up = quot_nr(w0p, sp, yp) * p0p + quot_nr(w1p, sp, yp) * p1p;
  return up + um;
}

// A face's linear weights (DPT_m1, DMCT_m1, DMT_0, DCPT_0) and epsilons within
// [2^-100, 2^100], weno_face_nr's range.
__host__ __device__ inline bool weno_consts_ok(double a, double b, double c, double d, double e, double f) {
  const double lo = 0x1p-100, hi = 0x1p100;
  return a >= lo && a <= hi && b >= lo && b <= hi && c >= lo && c <= hi && d >= lo && d <= hi && e >= lo &&
         e <= hi && f >= lo && f <= hi;
}

// First-order upwind face flux (src/hipft.f90:7649-7651, 7809-7815).
__device__ __forceinline__ double upwind_flux(double v, double upw, double xhi, double xlo) {
  double cct = copysign(upw, v);
  return v * kHalf * ((kOne - cct) * xhi + (kOne + cct) * xlo);
}

// Pole ring sums of the advection operator (src/hipft.f90:7902-7915): theta
// fluxes through faces 2 and nt-1 (upwind in both operators).
__global__ void k_ring_advection(Mesh m, Flow fl, const double *__restrict__ x, double *__restrict__ ring) {
  __shared__ double sh[64];
  const int i = blockIdx.x + 1;
  double fn = 0.0, fs = 0.0;
  for (int k = 2 + threadIdx.x; k <= m.npm - 1; k += blockDim.x) {
    double ftn = upwind_flux(vt_at(m, fl, 2, k, i), fl.upwind, x[fidx(m, 2, k, i)], x[fidx(m, 1, k, i)]);
    double fts = upwind_flux(vt_at(m, fl, m.nt - 1, k, i), fl.upwind, x[fidx(m, m.ntm, k, i)],
                             x[fidx(m, m.ntm - 1, k, i)]);
    fn = fn + ftn * m.dp[k];
    fs = fs + fts * m.dp[k];
  }
  block_sum2(fn, fs, sh);
  if (threadIdx.x == 0) {
    ring[2 * (i - 1)] = fn;
    ring[2 * (i - 1) + 1] = fs;
  }
}

// Stage combine of the explicit integrators (src/hipft.f90:7440-7578):
//   mode 0: out = x - C*aop
//   mode 1: out = A*f0 + B*x - C*aop
struct AdvCombine {
  int mode;
  double A, B, C;
};

// Phi cell index with the reference's periodic pad (LP(j,0) = LP(j,npm-2),
// LP(j,npm) = LP(j,2), src/hipft.f90:7840-7845).
__device__ __forceinline__ int wrap_cell(const Mesh &m, int c) {
  if (c < 1) return c + (m.npm - 2);
  if (c > m.npm - 1) return c - (m.npm - 2);
  return c;
}

// One explicit advection stage over a tile of TJ x TK cells: face fluxes
// (WENO3 or upwind), divergence (src/hipft.f90:7890-7898), pole rows from the
// ring sums, seam, and the integrator's combine.  The block is (TJ+1) x
// (TK+1) threads: thread (a, b) computes the theta face j0+a of column k0+b
// (b < TK) and the phi face k0+b of row j0+a (a < TJ), then the cell (a, b)
// (a < TJ, b < TK); no thread computes more than two faces.  The input tile
// (halo 2, phi wrapped with the reference's periodic pad), the WENO weights of
// the tile's faces and, for 1-D flows, the per-row flow terms v +/- alpha
// are staged in shared memory first.
// Ragged batches: rlist (may be null) maps grid slice z to a realization, and
// rdt (may be null) holds each realization's substep, which multiplies cb.C.
template <int TJ, int TK>
struct AdvSmem {
  double x[TK + 4][TJ + 4];   // column k0-2+b, row j0-2+a
  double ft[TK][TJ + 1];      // theta faces j0..j0+TJ of column k0+b
  double fp[TK + 1][TJ];      // phi faces k0..k0+TK of row j0+a
  double wt[10][TJ + 1];      // theta weights of face j0+a, in weno_face's argument order
  double wp[10][TK + 1];      // phi weights of face k0+b
  double tn[TJ + 4], tp[TJ + 4];  // 1-D flows: vt(c)+at(c), vt(c+1)-at(c) at row c = j0-2+a
  double pn[TJ], pp[TJ];          // 1-D flows: vp(j)+ap(j), vp(j)-ap(j) at row j = j0+a
};

template <int TJ, int TK, bool WENO>
__global__ void __launch_bounds__((TJ + 1) * (TK + 1)) k_advection_stage(
    Mesh m, Flow fl, Weno wn, const double *__restrict__ x, const double *__restrict__ f0, double *out,
    const double *__restrict__ ring, double bcn, double bcs, AdvCombine cb, const int *__restrict__ rlist = nullptr,
    const double *__restrict__ rdt = nullptr) {
  __shared__ AdvSmem<TJ, TK> s;
  constexpr int NT = (TJ + 1) * (TK + 1);
  static_assert(TJ + 1 <= 64 && TK + 1 <= 64 && TJ + 4 <= 64 && TJ <= 64 && NT >= 192 + TJ,
                "staging thread ranges 0.., 64.., 128.., 192..");
  const int a = threadIdx.x, b = threadIdx.y;
  const int tid = a + b * (TJ + 1);
  const int j0 = blockIdx.x * TJ + 1;
  const int k0 = blockIdx.y * TK + 2;
  if (rlist && rlist[blockIdx.z] < 0) return;  // slot past the list's end
  const int i = (rlist ? rlist[blockIdx.z] : (int)blockIdx.z) + 1;
  if (rdt) cb.C = cb.C * rdt[i - 1];
  const int ntm = m.ntm, npm = m.npm;
  const int64_t pbase = (int64_t)(i - 1) * m.plane;
  const bool oned = !fl.flow2d;

  // input tile with halo 2 (theta clipped to 1..ntm, phi wrapped periodically)
  for (int e = tid; e < (TJ + 4) * (TK + 4); e += NT) {
    const int r = e % (TJ + 4), c = e / (TJ + 4);
    const int j = j0 - 2 + r, k = wrap_cell(m, k0 - 2 + c);
    s.x[c][r] = (j >= 1 && j <= ntm) ? x[pbase + (int64_t)(k - 1) * m.ldt + (j - 1)] : 0.0;
  }
  if (WENO) {
    if (tid < TJ + 1) {
      const int r = tid, jf = min(max(j0 + r, 2), m.nt - 1);
      s.wt[0][r] = wn.mct[jf - 1];
      s.wt[1][r] = wn.mct[jf];
      s.wt[2][r] = wn.cpt[jf - 1];
      s.wt[3][r] = wn.cpt[jf];
      s.wt[4][r] = wn.pt[jf - 1];
      s.wt[5][r] = wn.mctt[jf - 1];
      s.wt[6][r] = wn.mt[jf];
      s.wt[7][r] = wn.cptt[jf];
      s.wt[8][r] = wn.epst[jf - 1];
      s.wt[9][r] = wn.epst[jf];
    } else if (tid >= 64 && tid < 64 + TK + 1) {
      const int c = tid - 64;
      const int kw = (k0 + c >= npm) ? 2 : k0 + c;  // face npm copies face 2 (src/hipft.f90:7882)
      s.wp[0][c] = wn.mcp[kw - 1];
      s.wp[1][c] = wn.mcp[kw];
      s.wp[2][c] = wn.cpp[kw - 1];
      s.wp[3][c] = wn.cpp[kw];
      s.wp[4][c] = wn.pp[kw - 1];
      s.wp[5][c] = wn.mctp[kw - 1];
      s.wp[6][c] = wn.mp[kw];
      s.wp[7][c] = wn.cptp[kw];
      s.wp[8][c] = wn.epsp[kw - 1];
      s.wp[9][c] = wn.epsp[kw];
    }
  }
  if (oned) {
    const double *vt = fl.vt1 + (int64_t)(i - 1) * (m.nt + 1), *at = fl.at1 + (int64_t)(i - 1) * (m.ntm + 1);
    const double *vp = fl.vp1 + (int64_t)(i - 1) * (m.ntm + 1), *ap = fl.ap1 + (int64_t)(i - 1) * (m.ntm + 1);
    const int e = tid - 128;  // threads 128.. (the weight loads use 0..63, 64..)
    if (e >= 0 && e < TJ + 4) {
      const int c = j0 - 2 + e;
      const bool ok = (c >= 1 && c <= ntm);
      s.tn[e] = ok ? vt[c] + at[c] : 0.0;
      s.tp[e] = ok ? vt[c + 1] - at[c] : 0.0;
    }
    const int f = tid - 192;
    if (f >= 0 && f < TJ) {
      const int j = j0 + f;
      const bool ok = (j >= 1 && j <= ntm);
      s.pn[f] = ok ? vp[j] + ap[j] : 0.0;
      s.pp[f] = ok ? vp[j] - ap[j] : 0.0;
    }
  }
  __syncthreads();

  // theta face jf = j0 + a of column k = k0 + b
  if (b < TK) {
    const int jf = j0 + a, k = k0 + b;
    double F = 0.0;
    if (k <= npm - 1 && jf >= 2 && jf <= ntm) {
      const double *xc = &s.x[b + 2][0];
      const double xa = xc[a + 2], xb = xc[a + 1];  // x(jf), x(jf-1)
      if (!WENO || jf == 2 || jf == ntm) {
        F = upwind_flux(vt_at(m, fl, jf, k, i), fl.upwind, xa, xb);
      } else {
        // LN(c) = half*x(c)*(vt(c)+alpha_t(c)), LP(c) = half*x(c)*(vt(c+1)-alpha_t(c))
        double LN[3], LP[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const int c = jf - 2 + d;  // LN at jf-2, jf-1, jf (shared row a + d)
          const double v = oned ? s.tn[a + d] : vt_at(m, fl, c, k, i) + at_at(m, fl, c, k, i);
          LN[d] = kHalf * xc[a + d] * v;
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const int c = jf - 1 + d;  // LP at jf-1, jf, jf+1 (shared row a + 1 + d)
          const double v = oned ? s.tp[a + 1 + d] : vt_at(m, fl, c + 1, k, i) - at_at(m, fl, c, k, i);
          LP[d] = kHalf * xc[a + 1 + d] * v;
        }
        F = weno_face(LN[0], LN[1], LN[2], LP[0], LP[1], LP[2], s.wt[0][a], s.wt[1][a], s.wt[2][a], s.wt[3][a],
                      s.wt[4][a], s.wt[5][a], s.wt[6][a], s.wt[7][a], s.wt[8][a], s.wt[9][a]);
      }
    }
    s.ft[b][a] = F;
  }
  // phi face kf = k0 + b of row j = j0 + a (interior rows only).  Face npm is
  // the seam copy of face 2 (src/hipft.f90:7882): its stencil cells are the
  // seam copies of face 2's cells, and it takes face 2's weights.
  if (a < TJ) {
    const int j = j0 + a, kf = k0 + b;
    double F = 0.0;
    if (j >= 2 && j <= ntm - 1 && kf <= npm) {
      const int kw = (kf == npm) ? 2 : kf;
      const int bb = b + 2;  // shared column of cell kf
      if (!WENO) {
        F = upwind_flux(vp_at(m, fl, j, kw, i), fl.upwind, s.x[bb][a + 2], s.x[bb - 1][a + 2]);
      } else {
        double LN[3], LP[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const int c = wrap_cell(m, kf - 2 + d);
          const double v = oned ? s.pn[a] : vp_at(m, fl, j, c, i) + ap_at(m, fl, j, c, i);
          LN[d] = kHalf * s.x[bb - 2 + d][a + 2] * v;
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const int c = wrap_cell(m, kf - 1 + d);
          const double v = oned ? s.pp[a] : vp_at(m, fl, j, c + 1, i) - ap_at(m, fl, j, c, i);
          LP[d] = kHalf * s.x[bb - 1 + d][a + 2] * v;
        }
        F = weno_face(LN[0], LN[1], LN[2], LP[0], LP[1], LP[2], s.wp[0][b], s.wp[1][b], s.wp[2][b], s.wp[3][b],
                      s.wp[4][b], s.wp[5][b], s.wp[6][b], s.wp[7][b], s.wp[8][b], s.wp[9][b]);
      }
    }
    s.fp[b][a] = F;
  }
  __syncthreads();

  if (a >= TJ || b >= TK) return;
  const int j = j0 + a, k = k0 + b;
  if (j > ntm || k > npm - 1) return;
  double aop;
  if (j == 1) {
    aop = ring[2 * (i - 1)] * bcn;
  } else if (j == ntm) {
    aop = -ring[2 * (i - 1) + 1] * bcs;
  } else {
    aop = ((m.sth[j + 1] * s.ft[b][a + 1] - m.sth[j] * s.ft[b][a]) * m.st_i[j] * m.dt_i[j] +
           (s.fp[b + 1][a] - s.fp[b][a]) * m.st_i[j] * m.dp_i[k]);
  }
  const int64_t q = pbase + (int64_t)(k - 1) * m.ldt + (j - 1);
  const double xv = s.x[b + 2][a + 2];
  double y;
  if (cb.mode == 0) {
    y = xv - cb.C * aop;
  } else {
    y = cb.A * f0[q] + cb.B * xv - cb.C * aop;
  }
  out[q] = y;
  if (k == 2) out[q + (int64_t)(npm - 2) * m.ldt] = y;
  if (k == npm - 1) out[q - (int64_t)(npm - 2) * m.ldt] = y;
}

// One WENO3 advection stage that marches along phi (the same faces,
// divergence, pole rows, seam and combine as k_advection_stage<., ., true>,
// with the same values: bitwise the same results).  The eight divisions per
// face bound this stage; the faces divide by Newton-Raphson refinement
// (weno_face_nr: correctly rounded, so the IEEE quotients; weno_face where
// its range check fails), which ran at 1.8x the IEEE routine's throughput.
//
// Each warp owns a group of theta rows and a chunk of ncol phi columns:
// lane l holds row r = j0 - 1 + l (j0 = 1 + 31 g for row group g), so lanes
// 1..31 own the cells of rows j0..j0+30 and lane 0's row, which belongs to the
// group below, only supplies the theta face between rows j0-1 and j0.  Per
// column k every lane computes one theta face (the face between its row and
// the next) and one phi face (between columns k and k+1 of its row): each face
// once, two per cell.  The theta face's LN/LP terms of the neighbouring rows
// come by warp shuffles (lanes 31, 0 and 1 also load the halo rows j0-2,
// j0+31 and j0+32), the phi face's from a sliding window of the row's last
// columns, and the cell takes the lower theta face from lane l-1 and the
// lower phi face from the previous column.  Both faces are evaluated before
// either range check, so the scheduler has two independent chains.  The phi
// face's weights and the column's dp_i come as six 16-byte loads of one
// table row (Weno::ptab), the same address across the warp.  The next
// column's inputs are loaded one column ahead.  No block barrier: warps are
// independent.
constexpr int kAdvColsMax = 64;  // phi columns per warp (fewer when the grid would not fill the GPU)
constexpr int kAdvWarps = 2;   // row groups per block (8 blocks per SM: at most 128 registers)

template <bool FLOW2D, int MODE>
__global__ void __launch_bounds__(32 * kAdvWarps, 8) k_adv_weno_march(
    Mesh m, Flow fl, Weno wn, const double *__restrict__ x, const double *__restrict__ f0, double *out,
    const double *__restrict__ ring, double bcn, double bcs, AdvCombine cb, const int *__restrict__ rlist,
    const double *__restrict__ rdt, int ncol) {
  const int l = threadIdx.x;
  const int ntm = m.ntm, npm = m.npm;
  const int j0 = 1 + 31 * (int)(blockIdx.x * kAdvWarps + threadIdx.y);
  const int kc0 = 2 + (int)blockIdx.y * ncol;
  if (j0 > ntm || kc0 > npm - 1) return;  // uniform per warp
  if (rlist && rlist[blockIdx.z] < 0) return;
  const int i = (rlist ? rlist[blockIdx.z] : (int)blockIdx.z) + 1;
  if (rdt) cb.C = cb.C * rdt[i - 1];
  const int kc1 = min(kc0 + ncol - 1, npm - 1);
  const int r = j0 - 1 + l;
  const int hr = (l == 31) ? j0 - 2 : (l == 0) ? j0 + 31 : (l == 1) ? j0 + 32 : 0;  // halo row (0: none)
  const bool rin = r >= 1 && r <= ntm, hin = hr >= 1 && hr <= ntm;
  const int64_t pbase = (int64_t)(i - 1) * m.plane;
  const int ldt = m.ldt, ldv = fl.ldv;
  // this lane's row and halo row of realization i (clamped into the plane
  // when out of range; such lanes use zeros instead of their loads)
  const double *xr = x + pbase + (rin ? r - 1 : 0);
  const double *xh = x + pbase + (hin ? hr - 1 : 0);

  // theta face jf = r + 1: none, first-order upwind (faces 2 and ntm) or WENO3
  const int jf = r + 1;
  const bool tface = jf >= 2 && jf <= ntm;
  const bool tup = tface && (jf == 2 || jf == ntm);
  const bool wup = __any_sync(0xffffffffu, tup);
  const int jw = min(max(jf, 2), m.nt - 1);
  const double w0 = wn.mct[jw - 1], w1 = wn.mct[jw], w2 = wn.cpt[jw - 1], w3 = wn.cpt[jw], w4 = wn.pt[jw - 1];
  const double w5 = wn.mctt[jw - 1], w6 = wn.mt[jw], w7 = wn.cptt[jw], w8 = wn.epst[jw - 1], w9 = wn.epst[jw];
  const bool tok = weno_consts_ok(w4, w5, w6, w7, w8, w9);
  // divergence factors of row r
  const int rc = min(max(r, 1), ntm);
  const double sth0 = m.sth[rc], sth1 = m.sth[rc + 1], sti = m.st_i[rc], dti = m.dt_i[rc];
  const bool cell = l >= 1 && rin;
  const bool pface = r >= 2 && r <= ntm - 1;
  const double apole = (r == 1) ? ring[2 * (i - 1)] * bcn : -ring[2 * (i - 1) + 1] * bcs;
  const bool pole = r == 1 || r == ntm;

  // LN(c) = half x(c) (vt(c)+at(c)) and LP(c) = half x(c) (vt(c+1)-at(c)) are
  // formed as x(c) * (half (vt(c)+at(c))) etc.: halving is exact, so the
  // products are the reference's (for |x| above 2^-1021, i.e. any map).
  // 1-D flows: the halved theta terms of the row and the halo row, and the
  // halved phi terms vp(j)+ap(j), vp(j)-ap(j), per row.
  double tn = 0.0, tp = 0.0, htn = 0.0, htp = 0.0, pn = 0.0, pp = 0.0, vtu = 0.0;
  if (!FLOW2D) {
    const double *vt = fl.vt1 + (int64_t)(i - 1) * (m.nt + 1), *at = fl.at1 + (int64_t)(i - 1) * (m.ntm + 1);
    const double *vp = fl.vp1 + (int64_t)(i - 1) * (m.ntm + 1), *ap = fl.ap1 + (int64_t)(i - 1) * (m.ntm + 1);
    if (rin) {
      tn = kHalf * (vt[r] + at[r]);
      tp = kHalf * (vt[r + 1] - at[r]);
      pn = kHalf * (vp[r] + ap[r]);
      pp = kHalf * (vp[r] - ap[r]);
    }
    if (hin) {
      htn = kHalf * (vt[hr] + at[hr]);
      htp = kHalf * (vt[hr + 1] - at[hr]);
    }
    if (tup) vtu = vt[jf];
  }
  // 2-D flows: this lane's row of the planes of realization i (theta stride ldv)
  const int64_t vbase = (int64_t)(i - 1) * fl.vplane;
  const double *vtr = fl.vt + vbase + (rin ? r - 1 : 0), *atr = fl.at + vbase + (rin ? r - 1 : 0);
  const double *vth = fl.vt + vbase + (hin ? hr - 1 : 0), *ath = fl.at + vbase + (hin ? hr - 1 : 0);
  const double *vpr = fl.vp + vbase + (rin ? r - 1 : 0), *apr = fl.ap + vbase + (rin ? r - 1 : 0);

  // column c (wrapped onto 1..npm-1) of the row: x, and the halved phi terms
  auto xload = [&](int c) -> double {
    const int cw = wrap_cell(m, c);
    return rin ? xr[(int64_t)(cw - 1) * ldt] : 0.0;
  };
  auto vN = [&](int c) -> double {
    if (!FLOW2D) return pn;
    const int cw = wrap_cell(m, c);
    return rin ? kHalf * (vpr[(int64_t)(cw - 1) * ldv] + apr[(int64_t)(cw - 1) * ldv]) : 0.0;
  };
  auto vP = [&](int c) -> double {
    if (!FLOW2D) return pp;
    const int cw = wrap_cell(m, c);
    return rin ? kHalf * (vpr[(int64_t)cw * ldv] - apr[(int64_t)(cw - 1) * ldv]) : 0.0;
  };
  // the phi-face table row of face kf (2..npm)
  auto ptab = [&](int kf) -> const double2 * {
    return reinterpret_cast<const double2 *>(wn.ptab + (int64_t)(kf - 2) * kPhiTab);
  };

  // window: LN at k-1, k, k+1; LP at k, k+1; x at k, k+1; the lower phi face
  // of column k and dp_i(k)
  double LN0, LN1, LN2, LP0, LP1, xk, xk1, Fplo, dpk;
  {
    const double xm2 = xload(kc0 - 2), xm1 = xload(kc0 - 1), x0 = xload(kc0), x1 = xload(kc0 + 1);
    const double LNm2 = xm2 * vN(kc0 - 2);
    LN0 = xm1 * vN(kc0 - 1);
    LN1 = x0 * vN(kc0);
    LN2 = x1 * vN(kc0 + 1);
    const double LPm1 = xm1 * vP(kc0 - 1);
    LP0 = x0 * vP(kc0);
    LP1 = x1 * vP(kc0 + 1);
    const double2 *T = ptab(kc0);
    const double2 q0 = T[0], q1 = T[1], q2 = T[2], q3 = T[3], q4 = T[4], q5 = T[5];
    bool ok;
    double F = weno_face_nr(LNm2, LN0, LN1, LPm1, LP0, LP1, q0.x, q0.y, q1.x, q1.y, q2.x, q2.y, q3.x, q3.y, q4.x,
                            q4.y, ok);
    if (!(ok && q5.x != 0.0))
      F = weno_face(LNm2, LN0, LN1, LPm1, LP0, LP1, q0.x, q0.y, q1.x, q1.y, q2.x, q2.y, q3.x, q3.y, q4.x, q4.y);
    Fplo = pface ? F : 0.0;
    dpk = q5.y;
    xk = x0;
    xk1 = x1;
  }
  // loads one column ahead: x(r, k+2) for the phi window, the halo row at
  // column k, f0 at column k, and the 2-D flows (theta at column k, phi at
  // column k+2); the last iteration's loads reach column npm at most, which
  // is inside the planes
  double xn = xload(kc0 + 2);
  double xhn = hin ? xh[(int64_t)(kc0 - 1) * ldt] : 0.0;
  double fv = (MODE != 0 && cell) ? f0[pbase + (int64_t)(kc0 - 1) * ldt + (r - 1)] : 0.0;
  double vt0 = 0.0, vt1 = 0.0, at0 = 0.0, vh0 = 0.0, vh1 = 0.0, ah0 = 0.0, vNn = pn, vPn = pp;
  if (FLOW2D) {
    const int64_t o = (int64_t)(kc0 - 1) * ldv;
    vt0 = rin ? vtr[o] : 0.0;
    vt1 = rin ? vtr[o + 1] : 0.0;
    at0 = rin ? atr[o] : 0.0;
    vh0 = hin ? vth[o] : 0.0;
    vh1 = hin ? vth[o + 1] : 0.0;
    ah0 = hin ? ath[o] : 0.0;
    vNn = vN(kc0 + 2);
    vPn = vP(kc0 + 2);
  }

  for (int k = kc0; k <= kc1; ++k) {
    const double xc2 = xn, xhc = xhn, fc = fv;
    double ctn = tn, ctp = tp, chn = htn, chp = htp, cvu = vtu;
    const double cN = vNn, cP = vPn;
    if (FLOW2D) {
      ctn = kHalf * (vt0 + at0);
      ctp = kHalf * (vt1 - at0);
      chn = kHalf * (vh0 + ah0);
      chp = kHalf * (vh1 - ah0);
      cvu = vt1;
    }
    xn = xload(k + 3);
    xhn = hin ? xh[(int64_t)k * ldt] : 0.0;
    if (MODE != 0 && cell) fv = f0[pbase + (int64_t)k * ldt + (r - 1)];
    if (FLOW2D) {
      const int64_t o = (int64_t)k * ldv;
      vt0 = rin ? vtr[o] : 0.0;
      vt1 = rin ? vtr[o + 1] : 0.0;
      at0 = rin ? atr[o] : 0.0;
      vh0 = hin ? vth[o] : 0.0;
      vh1 = hin ? vth[o + 1] : 0.0;
      ah0 = hin ? ath[o] : 0.0;
      vNn = vN(k + 3);
      vPn = vP(k + 3);
    }
    const double2 *T = ptab(k + 1);
    const double2 q0 = T[0], q1 = T[1], q2 = T[2], q3 = T[3], q4 = T[4], q5 = T[5];
    // phi face k+1: LN at k-1, k, k+1; LP at k, k+1, k+2
    const double LN3 = xc2 * cN, LP2 = xc2 * cP;
    // theta face r+1 of column k: LN at r-1, r, r+1; LP at r, r+1, r+2
    const double LNt = xk * ctn, LPt = xk * ctp;
    const double LNh = xhc * chn, LPh = xhc * chp;
    const double LNrm = __shfl_sync(0xffffffffu, l == 31 ? LNh : LNt, (l + 31) & 31);
    const double LNrp = __shfl_sync(0xffffffffu, l == 0 ? LNh : LNt, (l + 1) & 31);
    const double LPrp = __shfl_sync(0xffffffffu, l == 0 ? LPh : LPt, (l + 1) & 31);
    const double LPrpp = __shfl_sync(0xffffffffu, l <= 1 ? LPh : LPt, (l + 2) & 31);
    // both faces first (independent work for the scheduler), then the rare
    // IEEE-division recomputations
    bool okp, okt;
    double Fphi = weno_face_nr(LN0, LN1, LN2, LP0, LP1, LP2, q0.x, q0.y, q1.x, q1.y, q2.x, q2.y, q3.x, q3.y, q4.x,
                               q4.y, okp);
    double Ft = weno_face_nr(LNrm, LNt, LNrp, LPt, LPrp, LPrpp, w0, w1, w2, w3, w4, w5, w6, w7, w8, w9, okt);
    if (!(okp && q5.x != 0.0))
      Fphi = weno_face(LN0, LN1, LN2, LP0, LP1, LP2, q0.x, q0.y, q1.x, q1.y, q2.x, q2.y, q3.x, q3.y, q4.x, q4.y);
    if (!(okt && tok)) Ft = weno_face(LNrm, LNt, LNrp, LPt, LPrp, LPrpp, w0, w1, w2, w3, w4, w5, w6, w7, w8, w9);
    if (!pface) Fphi = 0.0;
    if (wup) {  // x(r+1) for the upwind faces 2 and ntm
      const double xr1 = __shfl_sync(0xffffffffu, l == 0 ? xhc : xk, (l + 1) & 31);
      if (tup) Ft = upwind_flux(cvu, fl.upwind, xr1, xk);
    }
    if (!tface) Ft = 0.0;
    const double Ftlo = __shfl_sync(0xffffffffu, Ft, (l + 31) & 31);
    const double aop = pole ? apole : ((sth1 * Ft - sth0 * Ftlo) * sti * dti + (Fphi - Fplo) * sti * dpk);
    const double y = MODE == 0 ? xk - cb.C * aop : cb.A * fc + cb.B * xk - cb.C * aop;
    if (cell) {
      double *o = out + pbase + (int64_t)(k - 1) * ldt + (r - 1);
      *o = y;
      if (k == 2) o[(int64_t)(npm - 2) * ldt] = y;
      if (k == npm - 1) o[-(int64_t)(npm - 2) * ldt] = y;
    }
    // slide the window
    Fplo = Fphi;
    dpk = q5.y;
    LN0 = LN1;
    LN1 = LN2;
    LN2 = LN3;
    LP0 = LP1;
    LP1 = LP2;
    xk = xk1;
    xk1 = xc2;
  }
}

// CFL limit, get_flow_dtmax (src/hipft.f90:7321-7327): min over interior
// cells of half/max(kdotv, tiny); positive doubles order like their bits.
// per_real: one limit per realization (ragged batches).
__global__ void k_flow_dtmax(Mesh m, Flow fl, unsigned long long *min_bits, int per_real = 0) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 2;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int i = blockIdx.z + 1;
  double dtv = 1.7976931348623157e308;
  if (j <= m.ntm - 1 && k <= m.npm - 1) {
    double kdotv = fmax(fabs(vt_at(m, fl, j, k, i)), fabs(vt_at(m, fl, j + 1, k, i))) * m.dt_i[j] +
                   fmax(fabs(vp_at(m, fl, j, k, i)), fabs(vp_at(m, fl, j, k + 1, i))) * m.st_i[j] * m.dp_i[k];
    dtv = kHalf / fmax(kdotv, 2.2250738585072014e-308);
  }
  unsigned long long b = __double_as_longlong(dtv);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long t = __shfl_down_sync(0xffffffffu, b, o);
    b = t < b ? t : b;
  }
  if ((threadIdx.x & 31) == 0) atomicMin(min_bits + (per_real ? i - 1 : 0), b);
}

// 2-D flow build (update_flow, src/hipft.f90:3393-3519): theta/phi profiles
// from the analytic models (1-D, computed on the host), the rotated rigid
// rotation, and Br attenuation.  One thread per (j,k,i) of the larger of
// the vt (nt x npm) and vp (ntm x np) grids.
struct Flow2DBuild {
  const double *vt1, *vp1;  // analytic 1-D parts, [nr][nt+1], [nr][ntm+1]
  // flows from files (shared by all realizations): when vtf is set, v starts
  // from vtf[k][j] ([npm][nt+1]) / vpf[k][j] ([np][ntm+1]) and the analytic
  // terms are applied one by one in update_flow's order instead of vt1/vp1
  const double *vtf, *vpf;
  const double *tmf;   // meridional term to subtract, [nr][nt+1] (NULL: model off)
  const double *vdr;   // differential rotation term to add, [nr][ntm+1] (NULL: off)
  const double *vrg;   // rigid rotation term to add, [ntm+1] (NULL: off)
  double vtc;          // constant theta velocity (0: off)
  const double *cth, *sth, *ct, *st;  // 1-based
  const double *cosp, *sinp, *cosph;  // cos(p(k)), sin(p(k)), cos(ph(k)), 1-based
  double vrigid;      // flow_rigid_omega * km_s_to_rs_hr (0: off)
  int attenuate;
  const double *atten_i;  // [nr+1]
};

__device__ __forceinline__ double sgn1(double b) { return copysign(1.0, b); }

__global__ void k_flow_build(Mesh m, Flow2DBuild b, int ldv, const double *__restrict__ f, double *vt,
                             double *vp) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int i = blockIdx.z + 1;
  const int64_t base = ((int64_t)(i - 1) * m.npm + (k - 1)) * ldv + (j - 1);
  if (j <= m.nt && k <= m.npm) {
    double v;
    if (b.vtf) {
      v = b.vtf[(int64_t)(k - 1) * (m.nt + 1) + j];
      if (b.tmf) v = v - b.tmf[(int64_t)(i - 1) * (m.nt + 1) + j];
      if (b.vtc != 0.0) v = v + b.vtc;
    } else {
      v = b.vt1[(int64_t)(i - 1) * (m.nt + 1) + j];
    }
    if (b.vrigid != 0.0) {
      double cp = b.cosp[k], c = b.cth[j], sv = b.sth[j];
      double acp = fabs(cp);
      double p1 = -2 * c * fabs(sv * cp);
      double p2 = (cp * c * c - cp) * acp * acp * acp;
      double p3 = (-3 * cp * c * c + 2 * cp) * acp;
      double p4 = sgn1(cp) * c * c;
      double p5 = 2 * acp * acp * acp * c * fabs(sv);
      double p6 = (-cp * cp * cp * cp + 3 * cp * cp - 1) * c * c;
      double p7 = (-2 * cp * cp * cp * sv + 2 * sv * cp) * c;
      double p8 = cp * cp * cp * cp - 2 * cp * cp + 1;
      double p9 = fabs(sv * cp) * b.sinp[k] * b.vrigid;
      double p10 = (cp * cp * cp * cp - 3 * cp * cp + 1) * c * c;
      double p11 = (2 * cp * cp * cp * sv - 2 * sv * cp) * c;
      double p12 = cp * cp * cp * cp + 2 * cp * cp;
      v = v + (-((p1 + (p2 + p3 + p4) * sgn1(sv) + p5 + p6 + p7 + p8) * p9) / sqrt(p10 + p11 - p12));
      if (fabs(v) > 1.0e5 || fabs(v) < -1.0e-5) v = 0;
    }
    if (b.attenuate && k >= 2 && k <= m.npm - 1 && j >= 2 && j <= m.nt - 1) {
      double ba = fmax(fabs(f[fidx(m, j - 1, k, i)]), fabs(f[fidx(m, j, k, i)]));
      v = v * (kOne - tanh(ba * b.atten_i[i]));
    }
    vt[base] = v;
  }
  if (j <= m.ntm && k <= m.np) {
    double v;
    if (b.vpf) {
      v = b.vpf[(int64_t)(k - 1) * (m.ntm + 1) + j];
      if (b.vdr) v = v + b.vdr[(int64_t)(i - 1) * (m.ntm + 1) + j];
      if (b.vrg) v = v + b.vrg[j];
    } else {
      v = b.vp1[(int64_t)(i - 1) * (m.ntm + 1) + j];
    }
    if (b.vrigid != 0.0) {
      double cph = b.cosph[k], c = b.ct[j], sv = b.st[j];
      double p1 = b.vrigid * (cph * cph * c + sv * cph - c) * sgn1(cph) * fabs(sv);
      double p2 = (cph * cph * cph * cph - 3 * cph * cph + 1) * c * c;
      double p3 = (2 * cph * cph * cph * sv - 2 * sv * cph) * c;
      double p4 = cph * cph * cph * cph + 2 * cph * cph;
      v = v - p1 / sqrt(p2 + p3 - p4);
      if (fabs(v) > 1.0e5 || fabs(v) < -1.0e-5) v = 0;
    }
    if (b.attenuate && k >= 2 && k <= m.np - 1) {
      double ba = fmax(fabs(f[fidx(m, j, k - 1, i)]), fabs(f[fidx(m, j, k, i)]));
      v = v * (kOne - tanh(ba * b.atten_i[i]));
    }
    vp[base] = v;
  }
}

// Periodic seam of a (n1 rows) x npm x nr array with stride ldt
// (set_periodic_bc_3d, src/hipft.f90:4920-4923).
__global__ void k_seam(Mesh m, int n1, int ld, double *a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int i = blockIdx.y + 1;
  if (j > n1) return;
  int64_t b = (int64_t)(i - 1) * m.npm * ld + (j - 1);
  a[b] = a[b + (int64_t)(m.npm - 2) * ld];
  a[b + (int64_t)(m.npm - 1) * ld] = a[b + (int64_t)ld];
}

// ------------------------------------------------------------------ sources
// generate_rfe (src/hipft.f90:8854-8873) on the interior columns of one
// frame: rfe = rnd(j,k) * uf(i) * da_ti(j) * dp_i(k) (model 1) or
// rnd(j,k) * uf(i) (model 2).  rnd is (ntm, npm), theta fastest.
__global__ void k_rfe_frame(Mesh m, int model, const double *__restrict__ rnd, const double *__restrict__ uf,
                            const double *__restrict__ dati, double *rfe) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int i = blockIdx.z + 1;
  if (j > m.ntm || k > m.npm - 1) return;
  const double r = rnd[(int64_t)(k - 1) * m.ntm + (j - 1)];
  rfe[fidx(m, j, k, i)] = (model == 1) ? r * uf[i] * dati[j] * m.dp_i[k] : r * uf[i];
}

// The frame's pole rows: the mean over phi of rows 1 and ntm, summed in the
// reference's sequential order (src/hipft.f90:8880-8894).  One block per
// realization.
__global__ void k_rfe_poles(Mesh m, double *rfe) {
  const int i = blockIdx.x + 1;
  __shared__ double s[2];
  if (threadIdx.x == 0) {
    double fn = 0.0, fs = 0.0;
    for (int k = 1; k <= m.npm - 2; ++k) {
      fn = fn + rfe[fidx(m, 1, k, i)] * m.dp[k];
      fs = fs + rfe[fidx(m, m.ntm, k, i)] * m.dp[k];
    }
    s[0] = fn * kTwoPiI;
    s[1] = fs * kTwoPiI;
  }
  __syncthreads();
  for (int k = 1 + threadIdx.x; k <= m.npm; k += blockDim.x) {
    rfe[fidx(m, 1, k, i)] = s[0];
    rfe[fidx(m, m.ntm, k, i)] = s[1];
  }
}

// update_source (src/hipft.f90:3898-3945): source = 0 [+ file]
// [+ (1-alpha) frame1 + alpha frame2], in that order.
__global__ void k_source_blend(Mesh m, const double *__restrict__ file, const double *__restrict__ r1,
                               const double *__restrict__ r2, double alpha, double *src) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int i = blockIdx.z + 1;
  if (j > m.ntm || k > m.npm) return;
  const int64_t q = fidx(m, j, k, i);
  double v = 0.0;
  if (file) v = v + file[(int64_t)(k - 1) * m.ldt + (j - 1)];
  if (r1) v = v + (kOne - alpha) * r1[q] + alpha * r2[q];
  src[q] = v;
}

// source_step (src/hipft.f90:4719-4721): f = f + dt * source.
__global__ void k_source_step(Mesh m, const double *__restrict__ src, double dt, double *f) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int i = blockIdx.z + 1;
  if (j > m.ntm || k > m.npm) return;
  const int64_t q = fidx(m, j, k, i);
  f[q] = f[q] + dt * src[q];
}

// Local Lax-Friedrichs alpha from 2-D velocities (set_lf_alpha,
// src/hipft.f90:6968-7046).
__global__ void k_lf_alpha(Mesh m, int ldv, const double *__restrict__ vt, const double *__restrict__ vp,
                           double *at, double *ap) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int i = blockIdx.z + 1;
  const int nt = m.nt, np = m.np;
  if (j > m.ntm || k > m.npm) return;
  const int64_t col = ((int64_t)(i - 1) * m.npm + (k - 1)) * ldv;
  auto VT = [&](int jj) { return fabs(vt[col + (jj - 1)]); };
  double a;
  if (j >= 3 && j <= nt - 3)
    a = fmax(fmax(fmax(fmax(fmax(VT(j - 2), VT(j - 1)), VT(j)), VT(j + 1)), VT(j + 2)), VT(j + 3));
  else if (j == 1)
    a = fmax(fmax(fmax(VT(j), VT(j + 1)), VT(j + 2)), VT(j + 3));
  else if (j == 2)
    a = fmax(fmax(fmax(fmax(VT(j - 1), VT(j)), VT(j + 1)), VT(j + 2)), VT(j + 3));
  else if (j == nt - 2)
    a = fmax(fmax(fmax(fmax(VT(j - 2), VT(j - 1)), VT(j)), VT(j + 1)), VT(j + 2));
  else
    a = fmax(fmax(fmax(VT(j - 2), VT(j - 1)), VT(j)), VT(j + 1));
  at[col + (j - 1)] = a;
  // alpha_p on interior rows and columns 2..np-1; columns 1 and npm by seam.
  double b = 0.0;
  if (j >= 2 && j <= m.ntm - 1) {
    const int64_t rb = (int64_t)(i - 1) * m.npm * ldv + (j - 1);
    auto VP = [&](int kk) { return fabs(vp[rb + (int64_t)(kk - 1) * ldv]); };
    int kk = k;
    if (kk == 1) kk = np - 1;
    if (kk == np) kk = 2;
    if (kk >= 3 && kk <= np - 3)
      b = fmax(fmax(fmax(fmax(fmax(VP(kk - 2), VP(kk - 1)), VP(kk)), VP(kk + 1)), VP(kk + 2)), VP(kk + 3));
    else if (kk == 2)
      b = fmax(fmax(fmax(fmax(fmax(VP(np - 2), VP(kk - 1)), VP(kk)), VP(kk + 1)), VP(kk + 2)), VP(kk + 3));
    else if (kk == np - 2)
      b = fmax(fmax(fmax(fmax(fmax(VP(kk - 2), VP(kk - 1)), VP(kk)), VP(kk + 1)), VP(kk + 2)), VP(3));
    else
      b = fmax(fmax(fmax(fmax(fmax(VP(kk - 2), VP(kk - 1)), VP(kk)), VP(kk + 1)), VP(3)), VP(4));
  }
  ap[col + (j - 1)] = b;
}

// ------------------------------------------------------------- analysis
// Per-realization diagnostics of analysis_step (src/hipft.f90:3183-3325).
// Stage 1: each block reduces a slab of phi columns into 15 partials
// (min, max, min|.|, verr, sumfval2, fluxp, fluxm, fluxp_pn, fluxm_pn,
// fluxp_ps, fluxm_ps, area_pn, area_ps, eqd1, eqd2, axd -> 16 slots).
constexpr int kNPart = 16;

struct AnalysisArgs {
  const double *da_t, *sn_t, *cs_t;        // [ntm+1], 1-based
  const double *da_p, *cs_p, *sn_p;        // [npm+1], 1-based
  const unsigned char *pn, *ps;            // [ntm+1] polar-cap masks
  int vmode;                               // validation mode 0/1/2
  const double *fval_u0;                   // PT (npm1, ntm, nr)
  const double *vscale;                    // [nr+1] mode-1 decay factors
  const double *t, *p, *st_i;              // 1-based, mode 2
  double vtt, vpt, width, p1, p2;
};

__device__ __forceinline__ double fval_at(const Mesh &m, const AnalysisArgs &a, int jphi, int jth, int i) {
  if (a.vmode == 1) {
    int npm1 = m.npm - 1;
    return a.fval_u0[((int64_t)(i - 1) * m.ntm + (jth - 1)) * npm1 + (jphi - 1)] * a.vscale[i];
  }
  // mode 2: two Gaussians (src/hipft.f90:3162-3174)
  double tt = a.t[jth] - 0.7853981633974483 - a.vtt;
  double b1 = a.p[jphi] - a.p1, b2 = a.p[jphi] - a.p2;
  return -a.st_i[jth] * exp(-(tt * tt) / a.width - (b1 * b1) / a.width) +
         a.st_i[jth] * exp(-(tt * tt) / a.width - (b2 * b2) / a.width);
}

template <int NT>
__global__ void __launch_bounds__(NT) k_analysis_partial(Mesh m, AnalysisArgs a, const double *__restrict__ f,
                                                         double *part, int cols_per_block) {
  __shared__ double sh[kNPart][NT / 32];
  const int i = blockIdx.y + 1;
  const int kb = blockIdx.x * cols_per_block + 1;
  const int ke = min(kb + cols_per_block - 1, m.npm - 1);
  double v[kNPart];
  v[0] = 1.7976931348623157e308;  // min
  v[1] = 2.2250738585072014e-308; // max starts at tiny (small_value)
  v[2] = 1.7976931348623157e308;  // min |f|
#pragma unroll
  for (int q = 3; q < kNPart; ++q) v[q] = 0.0;
  const int ncell = (ke - kb + 1) * m.ntm;
  for (int e = threadIdx.x; e < ncell; e += NT) {
    int k = kb + e / m.ntm, j = 1 + e % m.ntm;
    double fj = f[fidx(m, j, k, i)];
    if (k <= m.npm - 2) {
      v[0] = fmin(fj, v[0]);
      v[1] = fmax(fj, v[1]);
      v[2] = fmin(fabs(fj), v[2]);
      double fv = 0.0, fval;
      if (a.vmode == 0) {
        fval = fj;
      } else {
        fval = fval_at(m, a, k, j, i);
      }
      double d = fj - fval;
      v[3] = v[3] + d * d;
      v[4] = v[4] + fabs(fj) * fabs(fval);
      (void)fv;
    }
    double dat = a.da_t[j], dap = a.da_p[k];
    double fv = fj * dat * dap;
    if (fv > 0.) v[5] = v[5] + fv; else v[6] = v[6] + fv;
    if (a.pn[j]) {
      if (fv > 0.) v[7] = v[7] + fv; else v[8] = v[8] + fv;
      v[11] = v[11] + dat * dap;
    }
    if (a.ps[j]) {
      if (fv > 0.) v[9] = v[9] + fv; else v[10] = v[10] + fv;
      v[12] = v[12] + dat * dap;
    }
    v[13] = v[13] + fj * a.sn_t[j] * a.cs_p[k] * dat * dap;
    v[14] = v[14] + fj * a.sn_t[j] * a.sn_p[k] * dat * dap;
    v[15] = v[15] + fj * a.cs_t[j] * dat * dap;
  }
  const int l = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < kNPart; ++q) {
    double x = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double y = __shfl_down_sync(0xffffffffu, x, o);
      if (q == 0 || q == 2) x = fmin(x, y);
      else if (q == 1) x = fmax(x, y);
      else x = x + y;
    }
    if (l == 0) sh[q][w] = x;
  }
  __syncthreads();
  if (threadIdx.x < kNPart) {
    int q = threadIdx.x;
    double x = sh[q][0];
    for (int ww = 1; ww < NT / 32; ++ww) {
      double y = sh[q][ww];
      if (q == 0 || q == 2) x = fmin(x, y);
      else if (q == 1) x = fmax(x, y);
      else x = x + y;
    }
    part[((int64_t)(i - 1) * gridDim.x + blockIdx.x) * kNPart + q] = x;
  }
}

// Stage 2: one thread per (realization, slot) reduces the block partials in
// block order (deterministic).
__global__ void k_analysis_final(int nblocks, int nr, const double *__restrict__ part, double *out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nr * kNPart) return;
  const int i = t / kNPart, q = t % kNPart;
  double x = part[((int64_t)i * nblocks) * kNPart + q];
  for (int b = 1; b < nblocks; ++b) {
    double y = part[((int64_t)i * nblocks + b) * kNPart + q];
    if (q == 0 || q == 2) x = fmin(x, y);
    else if (q == 1) x = fmax(x, y);
    else x = x + y;
  }
  out[(int64_t)i * kNPart + q] = x;
}

// -------------------------------------------------------- assimilation
// Increment of assimilate_new_data (src/hipft.f90:4111-4120) with the mu
// weights, latitude caps and scaling of apply_data_assimilation
// (4242-4271).  The PT map (phi fastest) is read through a 32x32 shared
// tile so both the map and the field are accessed coalesced.
struct DAArgs {
  const double *data;   // (npm1, ntm, 3) PT
  const double *mu_power, *mu_limit, *lat_limit;  // [nr+1]
  const int *tidx0, *tidx1;                        // [nr+1]
  int add, custom_from_mu;
  double mult_fac;
  // custom_from_mu: weight planes (npm1, ntm) PT, mu^power where mu >
  // mu_limit, one per distinct (power, limit), and realization i's plane
  const double *wmap;
  const int *widx;                                 // [nr+1]
};

// Blend weight of PT cell (theta jt, phi kp) for realization i
// (src/hipft.f90:4242-4271): the map's weight slice, or the mu^power plane
// (evaluated on the host with the C library's pow, the function the
// reference's real-exponent ** calls, so the weights carry its bits); zero
// inside the latitude caps.
__device__ __forceinline__ double da_weight(const Mesh &m, const DAArgs &a, int jt, int kp, int i) {
  const int npm1 = m.npm - 1;
  const int64_t slice = (int64_t)npm1 * m.ntm;
  const int64_t q = (int64_t)(jt - 1) * npm1 + (kp - 1);
  double w;
  if (a.custom_from_mu) {
    w = a.wmap[(int64_t)a.widx[i] * slice + q];
  } else {
    w = a.data[slice + q];
  }
  if (a.lat_limit[i] > 0 && (jt <= a.tidx0[i] || jt >= a.tidx1[i])) w = 0.0;
  return w;
}

__global__ void k_da_delta(Mesh m, DAArgs a, const double *__restrict__ f, double *delta) {
  __shared__ double sd[32][33], sw[32][33];
  const int npm1 = m.npm - 1;
  const int i = blockIdx.z + 1;
  const int j0 = blockIdx.x * 32 + 1;   // theta tile start
  const int k0 = blockIdx.y * 32 + 1;   // phi tile start
  // load: thread (tx,ty) reads phi = k0+tx, theta = j0+ty+8r
  for (int r = 0; r < 4; ++r) {
    int jt = j0 + threadIdx.y + 8 * r, kp = k0 + threadIdx.x;
    double d = 0.0, w = 0.0;
    if (jt <= m.ntm && kp <= npm1) {
      int64_t q = (int64_t)(jt - 1) * npm1 + (kp - 1);
      d = a.data[q];
      w = da_weight(m, a, jt, kp, i);
      d = a.mult_fac * d;
    }
    sd[threadIdx.y + 8 * r][threadIdx.x] = d;
    sw[threadIdx.y + 8 * r][threadIdx.x] = w;
  }
  __syncthreads();
  // compute: thread (tx,ty) handles theta = j0+tx, phi = k0+ty+8r
  for (int r = 0; r < 4; ++r) {
    int jt = j0 + threadIdx.x, kp = k0 + threadIdx.y + 8 * r;
    if (jt > m.ntm || kp > npm1) continue;
    double d = sd[threadIdx.x][threadIdx.y + 8 * r], w = sw[threadIdx.x][threadIdx.y + 8 * r];
    int64_t q = fidx(m, jt, kp, i);
    double dv = a.add ? w * d : w * (d - f[q]);
    delta[q] = dv;
  }
}

// f += delta (src/hipft.f90:4138-4141) over every point including the seam,
// with the delta's seam taken first (4121) -- both done by reading the seam
// source columns directly; an optional per-realization scale implements
// balance_flux of the increment (8794-8801).
__global__ void k_da_apply(Mesh m, const double *__restrict__ delta, double *f, const double *ratio) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int i = blockIdx.z + 1;
  if (j > m.ntm || k > m.npm) return;
  int ks = k;
  if (k == 1) ks = m.npm - 1;
  if (k == m.npm) ks = 2;
  double d = delta[fidx(m, j, ks, i)];
  if (ratio) {
    double r = ratio[i];
    d = (d > 0) ? d / r : d * r;
  }
  int64_t q = fidx(m, j, k, i);
  f[q] = f[q] + d;
}

// get_flux (src/hipft.f90:8706-8738) partial sums per block; the host
// finishes the per-realization sums in block order.
__global__ void k_flux_partial(Mesh m, const double *__restrict__ da_t, const double *__restrict__ da_p,
                               const double *__restrict__ a, int seam_src, double *part, int cols_per_block) {
  __shared__ double sh[64];
  const int i = blockIdx.y + 1;
  const int kb = blockIdx.x * cols_per_block + 1;
  const int ke = min(kb + cols_per_block - 1, m.npm - 1);
  double fp = 0.0, fm = 0.0;
  const int ncell = (ke - kb + 1) * m.ntm;
  for (int e = threadIdx.x; e < ncell; e += blockDim.x) {
    int k = kb + e / m.ntm, j = 1 + e % m.ntm;
    int ks = k;
    if (seam_src && k == 1) ks = m.npm - 1;
    double fv = a[fidx(m, j, ks, i)] * da_t[j] * da_p[k];
    if (fv > 0.0) fp = fp + fv; else fm = fm + fv;
  }
  block_sum2(fp, fm, sh);
  if (threadIdx.x == 0) {
    part[((int64_t)(i - 1) * gridDim.x + blockIdx.x) * 2] = fp;
    part[((int64_t)(i - 1) * gridDim.x + blockIdx.x) * 2 + 1] = fm;
  }
}

// Multiplicative balance (src/hipft.f90:8794-8801) of the whole array.
__global__ void k_scale_balance(Mesh m, double *a, const double *ratio) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 1;
  const int i = blockIdx.z + 1;
  if (j > m.ntm || k > m.npm) return;
  double r = ratio[i];
  int64_t q = fidx(m, j, k, i);
  double br = a[q];
  a[q] = (br > 0) ? br / r : br * r;
}

}  // namespace hipft

namespace hipft {

// ---------------------------------------------- fused RKG2 stage (ring out)
// The fused single-stage kernel below is for a diffusion coefficient that is
// constant per realization (the diffusion_coef_constant path of
// load_diffusion).  Its 5-point coefficients are assembled from per-row and
// per-column factors in exactly the operation order of load_diffusion_matrix
// (src/hipft.f90:4962-4979), so values are bit-identical to the general
// kernel.
//
// The pole-ring sums of the *output* (needed by the next stage's pole rows,
// src/hipft.f90:7969-7979) are fused: the threads owning rows 2 and ntm-1
// add their KPT terms in column order, write one partial per phi block, and
// the last contributor of each realization (atomic counter, no waiting)
// reduces the partials in block order with a fixed shuffle tree and writes
// ring_out.  Nothing spins, so no wait needs a bound.
struct RingOut {
  double *ring;          // [2*nr] (fn, fs) of the output field
  double *part;          // [2][nr][nkb] partial sums
  unsigned int *count;   // [nr] contribution counters (left at 0)
  int nkb;               // phi blocks per realization
};


}  // namespace hipft

namespace hipft {

// ------------------------------------------------------ RKG2 stage, v3
// Every thread owns two adjacent theta rows and marches over KPT phi
// columns, moving the rows with 16-byte loads and stores (a warp touches 512
// contiguous bytes per array and column); all of its loads are issued
// before any arithmetic.  Row pairs start at an odd row (j = 2t+1, 2t+2) so the pole
// pairs (1,2) and (ntm-1,ntm) stay inside one thread when ntm is even, and
// inside one warp otherwise (handled with shuffles).  Requires ldt even.
// Ragged batches: rlist (may be null) maps grid slice z to a realization and
// rc (may be null) holds each realization's stage coefficients.
template <int MODE, int KPT>
__global__ void __launch_bounds__(128, 4) k_sts_stage_v3(Mesh m, const double *__restrict__ dfac,
                                                        const double *__restrict__ x, const double *ykm2,
                                                        const double *__restrict__ u0,
                                                        const double *__restrict__ dty0, double *out, double *out2,
                                                        const double *__restrict__ ring_in, double bcn, double bcs,
                                                        StageCoef sc, RingOut ro, int jshift,
                                                        const int *__restrict__ rlist = nullptr,
                                                        const StageCoef *__restrict__ rc = nullptr) {
  const int lane = threadIdx.x & 31;
  // thread t owns rows ja = 2t+1-2*jshift and ja+1; for odd ntm, jshift moves
  // the thread owning row ntm off lane 0 so row ntm-1 is in the same warp
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int ja = 2 * t + 1 - 2 * jshift;
  const int kb = blockIdx.y;
  const int k0 = kb * KPT + 2;
  if (rlist && rlist[blockIdx.z] < 0) return;  // slot past the list's end
  const int i = (rlist ? rlist[blockIdx.z] : (int)blockIdx.z) + 1;
  if (rc) sc = rc[i - 1];
  const int ntm = m.ntm, npm = m.npm;
  const int nk = min(KPT, npm - 1 - k0 + 1);
  const bool rowa = (ja >= 1 && ja <= ntm), rowb = (ja + 1 >= 1 && ja + 1 <= ntm);
  const bool any = rowa || rowb;
  const int64_t ld = m.ldt;
  // 16-byte aligned pair offset (ja-1 is even)
  const int64_t q0 = (int64_t)(i - 1) * m.plane + (int64_t)(k0 - 1) * ld + (ja - 1);
  const double Dr = dfac[i];
  const double Dh = kHalf * (Dr + Dr);

  double2 xv[KPT + 2], y2[KPT], uu[KPT], dd[KPT];
  double xe[KPT];
#pragma unroll
  for (int c = 0; c < KPT + 2; ++c) {
    int kc = k0 - 1 + c;
    xv[c] = (any && ja >= 1 && kc <= npm) ? *reinterpret_cast<const double2 *>(&x[q0 + (int64_t)(c - 1) * ld])
                                          : make_double2(0.0, 0.0);
  }
#pragma unroll
  for (int c = 0; c < KPT; ++c) {
    bool ok = any && ja >= 1 && c < nk;
    int64_t q = q0 + (int64_t)c * ld;
    double e = 0.0;
    // lane 0 needs x(ja-1), lane 31 needs x(ja+2)
    if (ok && lane == 0 && ja >= 2) e = x[q - 1];
    if (ok && lane == 31 && ja + 2 <= ntm) e = x[q + 2];
    xe[c] = e;
    if (MODE == MODE_STSK) {
      y2[c] = ok ? *reinterpret_cast<const double2 *>(&ykm2[q]) : make_double2(0.0, 0.0);
      uu[c] = ok ? *reinterpret_cast<const double2 *>(&u0[q]) : make_double2(0.0, 0.0);
      dd[c] = ok ? *reinterpret_cast<const double2 *>(&dty0[q]) : make_double2(0.0, 0.0);
    }
  }
  // per-row factors for rows ja (a) and ja+1 (b)
  const int jb = ja + 1;
  const bool ia = rowa && ja >= 2 && ja <= ntm - 1, ib = rowb && jb >= 2 && jb <= ntm - 1;
  double sta = 0, c2a = 0, c4a = 0, stb = 0, c2b = 0, c4b = 0;
  if (ia) {
    sta = m.st_i[ja];
    c2a = Dh * m.dth_i[ja] * m.dt_i[ja] * sta * m.sth[ja];
    c4a = Dh * m.dth_i[ja + 1] * m.dt_i[ja] * sta * m.sth[ja + 1];
  }
  if (ib) {
    stb = m.st_i[jb];
    c2b = Dh * m.dth_i[jb] * m.dt_i[jb] * stb * m.sth[jb];
    c4b = Dh * m.dth_i[jb + 1] * m.dt_i[jb] * stb * m.sth[jb + 1];
  }
  double rn_acc = 0.0;
  const double ax_n = ring_in[2 * (i - 1)] * bcn;
  const double ax_s = -ring_in[2 * (i - 1) + 1] * bcs;
#pragma unroll
  for (int c = 0; c < KPT; ++c) {
    const int k = k0 + c;
    const bool active = any && c < nk;
    double2 xc = xv[c + 1];
    double left = __shfl_up_sync(0xffffffffu, xc.y, 1);    // x(ja-1)
    double right = __shfl_down_sync(0xffffffffu, xc.x, 1); // x(jb+1)
    double xjm_a = (lane == 0) ? xe[c] : left;
    double xjp_b = (lane == 31) ? xe[c] : right;
    double pk = m.dph_i[min(k, npm)], pk1 = m.dph_i[min(k + 1, npm)], dpi = m.dp_i[min(k, npm)];
    double axa, axb;
    if (ja == 1) {
      axa = ax_n;
    } else if (ja == ntm) {
      axa = ax_s;
    } else {
      double c1 = Dh * pk * dpi * sta * sta;
      double c5 = Dh * pk1 * dpi * sta * sta;
      double c3 = -(c1 + c2a + c4a + c5);
      axa = c1 * xv[c].x + c2a * xjm_a + c3 * xc.x + c4a * xc.y + c5 * xv[c + 2].x;
    }
    if (jb == 1) {
      axb = ax_n;
    } else if (jb == ntm) {
      axb = ax_s;
    } else {
      double c1 = Dh * pk * dpi * stb * stb;
      double c5 = Dh * pk1 * dpi * stb * stb;
      double c3 = -(c1 + c2b + c4b + c5);
      axb = c1 * xv[c].y + c2b * xc.x + c3 * xc.y + c4b * xjp_b + c5 * xv[c + 2].y;
    }
    double ya, yb, da = 0.0, db = 0.0;
    if (MODE == MODE_STS1) {
      da = sc.a * axa;
      ya = xc.x + sc.b * da;
      db = sc.a * axb;
      yb = xc.y + sc.b * db;
    } else if (MODE == MODE_STSK) {
      ya = sc.a * xc.x + sc.b * y2[c].x + sc.c * uu[c].x + sc.d * axa + sc.e * dd[c].x;
      yb = sc.a * xc.y + sc.b * y2[c].y + sc.c * uu[c].y + sc.d * axb + sc.e * dd[c].y;
    } else {
      ya = xc.x + sc.a * axa;
      yb = xc.y + sc.a * axb;
    }
    // ring terms of the output: rows (1,2) and (ntm-1,ntm)
    double yb_prev = __shfl_up_sync(0xffffffffu, yb, 1);  // y(ja-1), for odd ntm
    if (!active) continue;
    if (ja == 1) rn_acc = rn_acc + (Dr + Dr) * (yb - ya) * m.dp[k];
    if (jb == ntm) rn_acc = rn_acc + (Dr + Dr) * (yb - ya) * m.dp[k];
    if (ja == ntm) rn_acc = rn_acc + (Dr + Dr) * (ya - yb_prev) * m.dp[k];
    const int64_t q = q0 + (int64_t)c * ld;
    double2 yv = make_double2(ya, yb);
    // rows beyond ntm (padding) are written too: they lie inside the padded column
    *reinterpret_cast<double2 *>(&out[q]) = yv;
    if (k == 2) *reinterpret_cast<double2 *>(&out[q + (int64_t)(npm - 2) * ld]) = yv;
    if (k == npm - 1) *reinterpret_cast<double2 *>(&out[q - (int64_t)(npm - 2) * ld]) = yv;
    if (MODE == MODE_STS1) {
      double2 dv = make_double2(da, db);
      *reinterpret_cast<double2 *>(&out2[q]) = dv;
      if (k == 2) *reinterpret_cast<double2 *>(&out2[q + (int64_t)(npm - 2) * ld]) = dv;
      if (k == npm - 1) *reinterpret_cast<double2 *>(&out2[q - (int64_t)(npm - 2) * ld]) = dv;
    }
  }
  // contributors: the thread owning row 1 (north) and the one owning row ntm (south)
  const bool north = (ja == 1), south = (jb == ntm) || (ja == ntm);
  unsigned int last = 0;
  if ((north || south) && any) {
    // a thread owning both poles (ntm == 2) cannot occur: ntm >= 4
    ro.part[((int64_t)(south ? 1 : 0) * m.nr + (i - 1)) * ro.nkb + kb] = rn_acc;
    __threadfence();
    unsigned int old = atomicAdd(&ro.count[i - 1], 1u);
    last = (old == 2u * (unsigned)ro.nkb - 1u) ? 1u : 0u;
  }
  unsigned int src_mask = __ballot_sync(0xffffffffu, last != 0);
  if (src_mask) {
    __threadfence();
    double sn = 0.0, ss = 0.0;
    for (int b = lane; b < ro.nkb; b += 32) {
      sn = sn + __ldcg(&ro.part[((int64_t)0 * m.nr + (i - 1)) * ro.nkb + b]);
      ss = ss + __ldcg(&ro.part[((int64_t)1 * m.nr + (i - 1)) * ro.nkb + b]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sn += __shfl_down_sync(0xffffffffu, sn, o);
      ss += __shfl_down_sync(0xffffffffu, ss, o);
    }
    if (lane == 0) {
      ro.ring[2 * (i - 1)] = sn;
      ro.ring[2 * (i - 1) + 1] = ss;
      ro.count[i - 1] = 0u;
    }
  }
}

}  // namespace hipft

namespace hipft {

// ---------------------------------------------------- bulk-copy helpers
// 1-D TMA (cp.async.bulk) global -> shared copies completed on an mbarrier.
// Every copy is 16-byte aligned at both ends and a multiple of 16 bytes.
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
// 3-D tensor tile load (global -> shared) completing on an mbarrier; the map
// is a kernel parameter (__grid_constant__), x the innermost coordinate
__device__ __forceinline__ void tma_load_3d(void *dst, const void *map, int x, int y, int z, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}
// shared -> global bulk copy in this thread's bulk async-group (both
// addresses 16-byte aligned, bytes a multiple of 16)
__device__ __forceinline__ void bulk_store(void *gdst, const void *ssrc, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_addr(ssrc)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// this thread's bulk stores have read their shared sources
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// this thread's bulk stores are complete
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// this thread's shared-memory writes become visible to later bulk copies
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
// Bounded wait: false if the copies did not land within the limit.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t phase, uint32_t limit) {
  for (uint32_t it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, phase)) return true;
  return false;
}

// ------------------------------------------- two RKG2 stages per launch
// Launch arguments of the two-stage kernel k_sts_pair_ws (sts_pair_ws.cuh):
// temporal blocking of stages k and k+1 (src/hipft.f90:5222-5237) over tiles
// of kPJ theta rows x kPK phi columns.
constexpr int kPJ = 128;          // theta rows per tile
constexpr int kPK = 8;            // phi columns per tile

struct PairArgs {
  StageCoef ca, cb;     // stages k and k+1
  int *err;             // set to 1 when a bounded wait gives up
  // ragged batches (null otherwise): the realizations (0-based) this launch
  // advances, and per realization the coefficients of its stages k, k+1
  // ([nr][2])
  const int *rlist = nullptr;
  const StageCoef *rc = nullptr;
  // steps run as a CUDA graph (with rlist and rc): the launch's stage pair is
  // *dctr + doff, read on the device; dnact[pair] realizations of rlist take
  // part and rc holds dstride coefficients per pair
  const int *dctr = nullptr;
  int doff = 0;
  const int *dnact = nullptr;
  int dstride = 0;
};

}  // namespace hipft
