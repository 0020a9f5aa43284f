// adjoint.cuh -- discrete adjoint (vector-Jacobian products) of the
// flux-transport step's two operators, for gradients of a map misfit with
// respect to the initial map, the diffusion coefficient and the analytic flow
// profiles (no reference counterpart; the forward operators are
// diffusion_operator_cd, src/hipft.f90:7927-7990, and
// advection_operator_weno3, src/hipft.f90:7711-7925).
//
// Cotangent fields are "folded": their phi seam columns 1 and npm hold zero,
// and the dependence of a forward field's seam columns (copies of columns
// npm-1 and 2) is carried by the columns they copy.  Every kernel here reads
// and writes core columns 2..npm-1 only.
#pragma once

#include "kernels.cuh"
#include "sts_pair_ws.cuh"  // PairTables (coefficient tables of k_pair_tables)

namespace hipft {

// neighbour of core column k on the periodic core ring 2..npm-1
__device__ __forceinline__ int core_wrap(const Mesh &m, int k) {
  if (k < 2) return k + (m.npm - 2);
  if (k > m.npm - 1) return k - (m.npm - 2);
  return k;
}

// Sums of a folded field over the core columns of the pole rows, one block
// per realization: g[2(i-1)] = sum_k w(1,k), g[2(i-1)+1] = sum_k w(ntm,k).
__global__ void k_adj_pole_sums(Mesh m, const double *__restrict__ w, double *__restrict__ g) {
  __shared__ double sh[64];
  const int i = blockIdx.x + 1;
  double a = 0.0, b = 0.0;
  for (int k = 2 + threadIdx.x; k <= m.npm - 1; k += blockDim.x) {
    a = a + w[fidx(m, 1, k, i)];
    b = b + w[fidx(m, m.ntm, k, i)];
  }
  block_sum2(a, b, sh);
  if (threadIdx.x == 0) {
    g[2 * (i - 1)] = a;
    g[2 * (i - 1) + 1] = b;
  }
}

// (A^T w)(j,k) at core cell (j,k) for the diffusion operator with its pole
// rows and periodic seam; gn, gs are w's pole sums.  Each term is one output
// of A that reads x(j,k): (j,k) [c3], (j,k+1) [c1], (j,k-1) [c5], (j+1,k)
// [c2], (j-1,k) [c4], and the pole rows through the ring sums.
__device__ __forceinline__ double adj_diff_at(const Mesh &m, const DiffCoef &dc, const double *__restrict__ w, int j,
                                              int k, int i, double gn, double gs, double bcn, double bcs) {
  const int ntm = m.ntm;
  double r = 0.0;
  if (j >= 2 && j <= ntm - 1) {
    const int kp = core_wrap(m, k + 1), km = core_wrap(m, k - 1);
    r += coef5(m, dc, j, k, i).c3 * w[fidx(m, j, k, i)];
    r += coef5(m, dc, j, kp, i).c1 * w[fidx(m, j, kp, i)];
    r += coef5(m, dc, j, km, i).c5 * w[fidx(m, j, km, i)];
    if (j + 1 <= ntm - 1) r += coef5(m, dc, j + 1, k, i).c2 * w[fidx(m, j + 1, k, i)];
    if (j - 1 >= 2) r += coef5(m, dc, j - 1, k, i).c4 * w[fidx(m, j - 1, k, i)];
    if (j == 2) r += (dcoef(m, dc, 1, k, i) + dcoef(m, dc, 2, k, i)) * m.dp[k] * bcn * gn;
    if (j == ntm - 1) r += (dcoef(m, dc, m.nt - 1, k, i) + dcoef(m, dc, m.nt, k, i)) * m.dp[k] * bcs * gs;
  } else if (j == 1) {
    r += coef5(m, dc, 2, k, i).c2 * w[fidx(m, 2, k, i)];
    r -= (dcoef(m, dc, 1, k, i) + dcoef(m, dc, 2, k, i)) * m.dp[k] * bcn * gn;
  } else {
    r += coef5(m, dc, ntm - 1, k, i).c4 * w[fidx(m, ntm - 1, k, i)];
    r -= (dcoef(m, dc, m.nt - 1, k, i) + dcoef(m, dc, m.nt, k, i)) * m.dp[k] * bcs * gs;
  }
  return r;
}

// The same, from the coefficient tables of k_pair_tables (per-realization
// constant D): row j's st_i, c2, c4 and column k's {P1, P5}, with
// c1 = P1 st_i^2, c5 = P5 st_i^2 and c3 = -(c1+c2+c4+c5) as in the forward
// two-stage kernel; five table rows and columns instead of five coef5().
__device__ __forceinline__ double adj_diff_at_tab(const Mesh &m, const DiffCoef &dc, const PairTables &pt,
                                                  const double *__restrict__ w, int j, int k, int i, double gn,
                                                  double gs, double bcn, double bcs) {
  const int ntm = m.ntm;
  const double *R = pt.row + (int64_t)(i - 1) * 3 * pt.LR;  // entry jj holds row jj-1
  const double2 *P = reinterpret_cast<const double2 *>(pt.col) + (int64_t)(i - 1) * pt.LC;
  double r = 0.0;
  if (j >= 2 && j <= ntm - 1) {
    const int kp = core_wrap(m, k + 1), km = core_wrap(m, k - 1);
    const double sj = R[j + 1], c2 = R[pt.LR + j + 1], c4 = R[2 * pt.LR + j + 1];
    const double2 Pk = P[k];
    const double c1 = Pk.x * sj * sj, c5 = Pk.y * sj * sj;
    const double c3 = -(c1 + c2 + c4 + c5);
    r += c3 * w[fidx(m, j, k, i)];
    r += (P[kp].x * sj * sj) * w[fidx(m, j, kp, i)];
    r += (P[km].y * sj * sj) * w[fidx(m, j, km, i)];
    if (j + 1 <= ntm - 1) r += R[pt.LR + j + 2] * w[fidx(m, j + 1, k, i)];
    if (j - 1 >= 2) r += R[2 * pt.LR + j] * w[fidx(m, j - 1, k, i)];
    if (j == 2) r += (dcoef(m, dc, 1, k, i) + dcoef(m, dc, 2, k, i)) * m.dp[k] * bcn * gn;
    if (j == ntm - 1) r += (dcoef(m, dc, m.nt - 1, k, i) + dcoef(m, dc, m.nt, k, i)) * m.dp[k] * bcs * gs;
  } else if (j == 1) {
    r += R[pt.LR + 3] * w[fidx(m, 2, k, i)];
    r -= (dcoef(m, dc, 1, k, i) + dcoef(m, dc, 2, k, i)) * m.dp[k] * bcn * gn;
  } else {
    r += R[2 * pt.LR + ntm] * w[fidx(m, ntm - 1, k, i)];
    r -= (dcoef(m, dc, m.nt - 1, k, i) + dcoef(m, dc, m.nt, k, i)) * m.dp[k] * bcs * gs;
  }
  return r;
}

// One reverse RKG2 stage (or a plain A^T application), per core cell:
//   out = a*w + b*wp + c*(A^T w);   ub += c0*w;   db += g*w;
// dpart[block] += dscale * (block sum of (A^T w)*y) (the diffusion-
// coefficient term, summed per realization by k_adj_dsum).  wp, y, ub, db
// may be null; out may alias wp (each cell reads wp before writing out).
// w's pole sums come as npin partials per realization, gin[(i-1)][q][2]
// (summed in order by the blocks that need them); the kernel leaves the
// pole sums of `out` as gridDim.y partials in gout, for the next stage.
struct AdjDiffCoef {
  double a, b, c, c0, g, dscale;
};

__global__ void __launch_bounds__(256) k_adj_diff(Mesh m, DiffCoef dc, const double *__restrict__ w, const double *wp,
                                                  const double *__restrict__ y, double *out, double *ub, double *db,
                                                  const double *__restrict__ gin, int npin, double *__restrict__ gout,
                                                  double bcn, double bcs, AdjDiffCoef ac, double *__restrict__ dpart,
                                                  PairTables pt) {
  __shared__ double sh[64];
  __shared__ double s_g[2];
  __shared__ double s_n[8], s_s[8];
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int i = blockIdx.z + 1;
  const int j0 = blockIdx.x * blockDim.x + 1, j1 = j0 + blockDim.x - 1;
  const bool need = (j0 <= 2) || (j1 >= m.ntm - 1);  // rows 1, 2, ntm-1, ntm use the pole sums
  if (need) {
    if (threadIdx.y == 0) {  // one warp: lane-strided sums, then a fixed shuffle tree
      double a = 0.0, b = 0.0;
      const double *g = gin + (int64_t)(i - 1) * npin * 2;
      for (int q = threadIdx.x; q < npin; q += 32) {
        a = a + g[2 * q];
        b = b + g[2 * q + 1];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
      }
      if (threadIdx.x == 0) {
        s_g[0] = a;
        s_g[1] = b;
      }
    }
    __syncthreads();
  }
  double dsum = 0.0, o = 0.0;
  const bool active = (j <= m.ntm && k <= m.npm - 1);
  if (active) {
    const int64_t q = fidx(m, j, k, i);
    const double gn = need ? s_g[0] : 0.0, gs = need ? s_g[1] : 0.0;
    const double aw = pt.row ? adj_diff_at_tab(m, dc, pt, w, j, k, i, gn, gs, bcn, bcs)
                             : adj_diff_at(m, dc, w, j, k, i, gn, gs, bcn, bcs);
    const double wq = w[q];
    o = ac.a * wq + ac.c * aw;
    if (wp) o += ac.b * wp[q];
    out[q] = o;
    if (ub) ub[q] += ac.c0 * wq;
    if (db) db[q] += ac.g * wq;
    if (y) dsum = aw * y[q];
  }
  // pole-row partials of out over this block's columns (fixed order)
  const bool has_n = (j0 == 1), has_s = (j0 <= m.ntm && j1 >= m.ntm);
  if (has_n || has_s) {
    if (threadIdx.x == 0) s_n[threadIdx.y] = active ? o : 0.0;
    if (j == m.ntm) s_s[threadIdx.y] = active ? o : 0.0;
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      double a = 0.0, b = 0.0;
      for (int t = 0; t < (int)blockDim.y; ++t) {
        a = a + s_n[t];
        b = b + s_s[t];
      }
      double *go = gout + ((int64_t)(i - 1) * gridDim.y + blockIdx.y) * 2;
      if (has_n) go[0] = a;
      if (has_s) go[1] = b;
    }
  }
  if (dpart && y) {
    double z = 0.0;
    block_sum2(dsum, z, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0)
      dpart[((int64_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] += ac.dscale * dsum;
  }
}

// ---------------------------------------------- two reverse stages per launch
// Stages k and k-1 of the reverse RKG2 recurrence in one pass over the field:
//   W_{k-1} = a1 W_k + b1 W_{k+1} + c1 A^T W_k,
//   W_{k-2} = a2 W_{k-1} + b2 W_k + c2 A^T W_{k-1},
//   ub += c01 W_k + c02 W_{k-1},  db += g1 W_k + g2 W_{k-1},
//   dpart += ds1 <A^T W_k, Y_{k-1}> + ds2 <A^T W_{k-1}, Y_{k-2}> (block partials).
// A tile of 32 theta rows x 16 core columns stages W_k with a halo of 2 in
// shared memory, computes W_{k-1} on the tile plus a halo of 1 there, then
// W_{k-2} on the tile: per cell and two stages W_k, W_{k+1}, Y_{k-1}, Y_{k-2},
// ub, db are read and W_{k-1}, W_{k-2}, ub, db written (80 B) where two
// one-stage launches move 128 B.  A^T at rows 1, 2, ntm-1, ntm needs the pole
// sums of its input over every column, which for W_{k-1} exist only after the
// whole grid; k_adj_pole2 finishes W_{k-2} (and its D partials) there and
// leaves the pole sums of W_{k-2} for the next launch.  Tiles holding rows 1 /
// ntm write per-tile partials of W_{k-1}'s pole sums.  Operation order per
// cell as adj_diff_at_tab.
struct AdjDiff2Coef {
  double a1, b1, c1, c01, g1, ds1;  // stage k
  double a2, b2, c2, c02, g2, ds2;  // stage k-1
};

constexpr int kA2J = 32, kA2K = 16;  // tile: theta rows x core columns (block 32 x 16 threads)

// A^T w at (j, k) from a shared tile ws (column stride ld) at shared (r, c),
// gn, gs: w's pole sums, with the tile's coefficient tables in shared memory
// (same expression order as adj_diff_at_tab): sR[a*36 +
// (jj - jbase)] holds table row jj of array a (st_i, c2, c4; jj = row + 1) for
// jj in jbase .. jbase+35, and sP[pc] the column entry of the cell's column k
// (sP[pc+1] of k+1, sP[pc-1] of k-1).  Same expressions, same order.
constexpr int kA2R = kA2J + 4;  // table rows of a k_adj_diff2 tile
__device__ __forceinline__ double adj_at_tile_s(const Mesh &m, const DiffCoef &dc, int i, int j, int k,
                                                const double *ws, int ld, int r, int c, const double *sR, int jbase,
                                                const double2 *sP, int pc, double gn, double gs, double bcn,
                                                double bcs) {
  const int ntm = m.ntm;
  auto R = [&](int a, int jj) { return sR[a * kA2R + (jj - jbase)]; };
  auto W = [&](int dr, int dcl) { return ws[(c + dcl) * ld + (r + dr)]; };
  double res = 0.0;
  if (j >= 2 && j <= ntm - 1) {
    const double sj = R(0, j + 1), c2 = R(1, j + 1), c4 = R(2, j + 1);
    const double2 Pk = sP[pc];
    const double c1 = Pk.x * sj * sj, c5 = Pk.y * sj * sj;
    const double c3 = -(c1 + c2 + c4 + c5);
    res += c3 * W(0, 0);
    res += (sP[pc + 1].x * sj * sj) * W(0, 1);
    res += (sP[pc - 1].y * sj * sj) * W(0, -1);
    if (j + 1 <= ntm - 1) res += R(1, j + 2) * W(1, 0);
    if (j - 1 >= 2) res += R(2, j) * W(-1, 0);
    if (j == 2) res += (dcoef(m, dc, 1, k, i) + dcoef(m, dc, 2, k, i)) * m.dp[k] * bcn * gn;
    if (j == ntm - 1) res += (dcoef(m, dc, m.nt - 1, k, i) + dcoef(m, dc, m.nt, k, i)) * m.dp[k] * bcs * gs;
  } else if (j == 1) {
    res += R(1, 3) * W(1, 0);
    res -= (dcoef(m, dc, 1, k, i) + dcoef(m, dc, 2, k, i)) * m.dp[k] * bcn * gn;
  } else {
    res += R(2, ntm) * W(-1, 0);
    res -= (dcoef(m, dc, m.nt - 1, k, i) + dcoef(m, dc, m.nt, k, i)) * m.dp[k] * bcs * gs;
  }
  return res;
}

__global__ void __launch_bounds__(kA2J * kA2K, 3) k_adj_diff2(Mesh m, DiffCoef dc, const double *__restrict__ w,
                                                   const double *__restrict__ wp, const double *__restrict__ y1,
                                                   const double *__restrict__ y2, double *out1, double *out2,
                                                   double *ub, double *db, const double *__restrict__ gin, int npin,
                                                   double *__restrict__ gpart, double bcn, double bcs,
                                                   AdjDiff2Coef ac, double *__restrict__ dpart, int dstride,
                                                   PairTables pt) {
  constexpr int LW = kA2J + 4, LM = kA2J + 2;
  __shared__ double sw[(kA2K + 4) * LW];  // W_k, halo 2: sw(r, c) = row j0-2+r, core column k0-2+c
  __shared__ double sm[(kA2K + 2) * LM];  // W_{k-1}, halo 1: sm(r, c) = row j0-1+r, core column k0-1+c
  __shared__ double sh[64];
  __shared__ double s_g[2];
  __shared__ double s_n[kA2K], s_s[kA2K];
  __shared__ double sR[3 * kA2R];      // row tables, rows j0-2 .. j0+33 (entries jj = j0-1 .. j0+34)
  __shared__ double2 sP[kA2K + 4];     // column table, core columns k0-2 .. k0+9
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + ty * kA2J;
  const int j0 = blockIdx.x * kA2J + 1, k0 = blockIdx.y * kA2K + 2;
  const int i = blockIdx.z + 1;
  const int ntm = m.ntm, npm = m.npm;
  const int jbase = j0 - 1;
  if (tid < 3 * kA2R) {
    const int a = tid / kA2R, jj = jbase + tid % kA2R;
    sR[tid] = (jj < pt.LR) ? pt.row[((int64_t)(i - 1) * 3 + a) * pt.LR + jj] : 0.0;
  } else if (tid >= 128 && tid < 128 + kA2K + 4) {
    const int q = tid - 128;
    sP[q] = reinterpret_cast<const double2 *>(pt.col)[(int64_t)(i - 1) * pt.LC + core_wrap(m, k0 - 2 + q)];
  }
  // Launched programmatically after the previous pair's k_adj_pole2, this
  // kernel may start while that one still writes W_k's pole rows (1, 2,
  // ntm-1, ntm) and pole sums: the tiles whose rows (with halo) reach them
  // wait for it; the others read neither.  (Without such a launch the wait
  // returns at once.)
  const bool edge = (j0 - 2 <= 2) || (j0 + kA2J + 1 >= ntm - 1);
  if (edge) asm volatile("griddepcontrol.wait;" ::: "memory");
  // pole sums of W_k, summed in order by every block that uses them (a fixed tree)
  if (ty == 0) {
    double a = 0.0, b = 0.0;
    const double *g = gin + (int64_t)(i - 1) * npin * 2;
    for (int q = tx; edge && q < npin; q += 32) {
      a = a + g[2 * q];
      b = b + g[2 * q + 1];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if (tx == 0) {
      s_g[0] = a;
      s_g[1] = b;
    }
  }
  // Every global operand of the thread's cells is requested here, before
  // the first barrier, so that the loads' latencies overlap: W_{k+1} of its
  // (at most two) stage-k cells, Y_{k-1} of those it owns, and ub, db,
  // Y_{k-2} of its stage-(k-1) cell.
  constexpr int NT = kA2J * kA2K, NE = (kA2K + 2) * LM, NPER = (NE + NT - 1) / NT;
  double wpv[NPER], y1v[NPER];
#pragma unroll
  for (int n = 0; n < NPER; ++n) {
    const int e = tid + n * NT, r = e % LM, c = e / LM;
    const int jj = j0 - 1 + r, kk = core_wrap(m, k0 - 1 + c);
    const bool in = e < NE && jj >= 1 && jj <= ntm;
    const bool own = (r >= 1 && r <= kA2J && c >= 1 && c <= kA2K && k0 - 1 + c <= npm - 1);
    const int64_t q = in ? fidx(m, jj, kk, i) : 0;
    wpv[n] = (in && wp) ? wp[q] : 0.0;
    y1v[n] = (in && own && y1) ? y1[q] : 0.0;
  }
  const int j = j0 + tx, k = k0 + ty;
  const bool active = (j <= ntm && k <= npm - 1);
  const int64_t qa = active ? fidx(m, j, k, i) : 0;
  const double ubv = (active && ub) ? ub[qa] : 0.0, dbv = (active && db) ? db[qa] : 0.0;
  const double y2v = (active && y2 && j >= 3 && j <= ntm - 2) ? y2[qa] : 0.0;
  for (int e = tid; e < (kA2K + 4) * LW; e += NT) {
    const int r = e % LW, c = e / LW;
    const int jj = j0 - 2 + r, kk = core_wrap(m, k0 - 2 + c);
    sw[e] = (jj >= 1 && jj <= ntm) ? w[fidx(m, jj, kk, i)] : 0.0;
  }
  __syncthreads();
  const double gn = s_g[0], gs = s_g[1];
  double dsum = 0.0;
  // stage k on the tile plus a halo of 1: W_{k-1} into shared memory
#pragma unroll
  for (int n = 0; n < NPER; ++n) {
    const int e = tid + n * NT;
    if (e >= NE) break;
    const int r = e % LM, c = e / LM;
    const int jj = j0 - 1 + r, kk = core_wrap(m, k0 - 1 + c);
    double o = 0.0;
    if (jj >= 1 && jj <= ntm) {
      const double aw =
          adj_at_tile_s(m, dc, i, jj, kk, sw, LW, r + 1, c + 1, sR, jbase, sP, c + 1, gn, gs, bcn, bcs);
      const int64_t q = fidx(m, jj, kk, i);
      const double wq = sw[(c + 1) * LW + r + 1];
      o = ac.a1 * wq + ac.c1 * aw;
      if (wp) o += ac.b1 * wpv[n];
      const bool own = (r >= 1 && r <= kA2J && c >= 1 && c <= kA2K && k0 - 1 + c <= npm - 1);
      if (own) {
        out1[q] = o;
        if (y1) dsum += ac.ds1 * (aw * y1v[n]);
      }
    }
    sm[e] = o;
  }
  __syncthreads();
  // stage k-1 on the tile, except the rows that need W_{k-1}'s pole sums
  double wm = 0.0;
  if (active) {
    const int64_t q = qa;
    const double wk = sw[(ty + 2) * LW + tx + 2];
    wm = sm[(ty + 1) * LM + tx + 1];
    if (ub) ub[q] = ubv + ac.c01 * wk + ac.c02 * wm;
    if (db) db[q] = dbv + ac.g1 * wk + ac.g2 * wm;
    if (j >= 3 && j <= ntm - 2) {
      const double aw =
          adj_at_tile_s(m, dc, i, j, k, sm, LM, tx + 1, ty + 1, sR, jbase, sP, ty + 2, 0.0, 0.0, bcn, bcs);
      out2[q] = ac.a2 * wm + ac.b2 * wk + ac.c2 * aw;
      if (y2) dsum += ac.ds2 * (aw * y2v);
    }
  }
  // per-tile partials of W_{k-1}'s pole sums (fixed order over the tile's columns)
  const bool has_n = (j0 == 1), has_s = (j0 <= ntm && j0 + kA2J - 1 >= ntm);
  if (has_n || has_s) {
    if (tx == 0) s_n[ty] = active ? wm : 0.0;
    if (j == ntm) s_s[ty] = active ? wm : 0.0;
    __syncthreads();
    if (tid == 0) {
      double a = 0.0, b = 0.0;
      for (int t = 0; t < kA2K; ++t) {
        a = a + s_n[t];
        b = b + s_s[t];
      }
      double *go = gpart + ((int64_t)(i - 1) * gridDim.y + blockIdx.y) * 2;
      if (has_n) go[0] = a;
      if (has_s) go[1] = b;
    }
  }
  if (dpart) {
    double z = 0.0;
    block_sum2(dsum, z, sh);
    if (tid == 0) dpart[(int64_t)blockIdx.z * dstride + blockIdx.y * gridDim.x + blockIdx.x] += dsum;
  }
}

// Stage k-1 at rows 1, 2, ntm-1, ntm (after k_adj_diff2); grid (realization,
// chunk of blockDim.x phi columns): W_{k-1}'s pole sums from the tiles'
// partials (fixed order, the same in every block), W_{k-2} = a2 W_{k-1} +
// b2 W_k + c2 A^T W_{k-1} there, the chunk's D partials of those rows (added
// to its own slot of dpole), and the chunk's partial pole sums of W_{k-2} for
// the next launch (gout[(i-1)][chunk][0..1]; the consumer sums the chunks in
// order).
__global__ void __launch_bounds__(256) k_adj_pole2(Mesh m, DiffCoef dc, const double *__restrict__ w,
                                                   const double *__restrict__ wm1, const double *__restrict__ y2,
                                                   double *out2, const double *__restrict__ gpart, int npart,
                                                   double *__restrict__ gout, double bcn, double bcs,
                                                   AdjDiff2Coef ac, double *__restrict__ dpole, PairTables pt) {
  __shared__ double sh[64];
  __shared__ double s_g[2];
  // the next pair's k_adj_diff2 may launch now; its pole tiles wait for this grid
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int i = blockIdx.x + 1, ch = blockIdx.y, nch = gridDim.y, tid = threadIdx.x, ntm = m.ntm;
  if (tid < 32) {
    double a = 0.0, b = 0.0;
    const double *g = gpart + (int64_t)(i - 1) * npart * 2;
    for (int q = tid; q < npart; q += 32) {
      a = a + g[2 * q];
      b = b + g[2 * q + 1];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if (tid == 0) {
      s_g[0] = a;
      s_g[1] = b;
    }
  }
  __syncthreads();
  const double gn = s_g[0], gs = s_g[1];
  double dsum = 0.0, pn = 0.0, ps = 0.0;
  for (int k = 2 + ch * blockDim.x + tid; k <= m.npm - 1; k += nch * blockDim.x) {
    for (int q = 0; q < 4; ++q) {
      const int j = (q == 0) ? 1 : ((q == 1) ? 2 : ((q == 2) ? ntm - 1 : ntm));
      const double aw = adj_diff_at_tab(m, dc, pt, wm1, j, k, i, gn, gs, bcn, bcs);
      const int64_t x = fidx(m, j, k, i);
      const double v = ac.a2 * wm1[x] + ac.b2 * w[x] + ac.c2 * aw;
      out2[x] = v;
      if (y2) dsum += ac.ds2 * (aw * y2[x]);
      if (j == 1) pn = pn + v;
      if (j == ntm) ps = ps + v;
    }
  }
  block_sum2(pn, ps, sh);
  if (tid == 0) {
    gout[((int64_t)(i - 1) * nch + ch) * 2] = pn;
    gout[((int64_t)(i - 1) * nch + ch) * 2 + 1] = ps;
  }
  if (dpole) {
    double z = 0.0;
    block_sum2(dsum, z, sh);
    if (tid == 0) dpole[(int64_t)(i - 1) * nch + ch] += dsum;
  }
}

// Reverse of the assimilation blend f += w (d - f) (src/hipft.f90:4116-4141):
// on the core columns the blend is f_new = (1 - w) f + w d, so the folded
// cotangent becomes (1 - w) fbar; the additive form f += w d leaves it
// unchanged.  One thread per core cell.
__global__ void k_adj_da(Mesh m, DAArgs a, double *fbar) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int i = blockIdx.z + 1;
  if (j > m.ntm || k > m.npm - 1 || a.add) return;
  const double w = da_weight(m, a, j, k, i);
  const int64_t q = fidx(m, j, k, i);
  fbar[q] = (kOne - w) * fbar[q];
}

// Reverse of the balanced increment (balance_flux of D = w (d - f),
// src/hipft.f90:8752-8807, applied at 4125-4141).  Forward: B(D) = D / r where
// D > 0, D r elsewhere, r = sqrt(|F+ / F-|), F+- get_flux's area-weighted
// sums of the positive and the other cells (columns 1..npm-1, column 1 the
// seam copy of npm-1).  With b the folded cotangent of f after the step,
//   Dbar = g b + S dr/dD,  g = 1/r (D > 0) or r,
//   S = sum b D dg/dr = -SP / r^2 + SN,  SP, SN = sum of b D over D > 0, D <= 0,
//   dr/dD = A r / (2 F+) (D > 0) or -A r / (2 F-),
// A the cell's get_flux area (column npm-1 twice: itself and its seam copy),
// and fbar = b - w Dbar.  k_adj_bal_partial: per-block partials of SP, SN
// over core columns (the host sums them in block order); k_adj_da_bal: the
// pointwise pass with coef[i] = {1/r, r, S r / (2 F+), -S r / (2 F-)}.
__global__ void k_adj_bal_partial(Mesh m, const double *__restrict__ delta, const double *__restrict__ fbar,
                                  int cols_per_block, double *part) {
  __shared__ double sh[64];
  const int i = blockIdx.y + 1;
  const int kb = 2 + blockIdx.x * cols_per_block;
  const int ke = min(kb + cols_per_block - 1, m.npm - 1);
  double sp = 0.0, sn = 0.0;
  const int ncell = (ke - kb + 1) * m.ntm;
  for (int e = threadIdx.x; e < ncell; e += blockDim.x) {
    const int k = kb + e / m.ntm, j = 1 + e % m.ntm;
    const int64_t q = fidx(m, j, k, i);
    const double d = delta[q], v = fbar[q] * d;
    if (d > 0.0) sp = sp + v; else sn = sn + v;
  }
  block_sum2(sp, sn, sh);
  if (threadIdx.x == 0) {
    part[((int64_t)(i - 1) * gridDim.x + blockIdx.x) * 2] = sp;
    part[((int64_t)(i - 1) * gridDim.x + blockIdx.x) * 2 + 1] = sn;
  }
}

__global__ void k_adj_da_bal(Mesh m, DAArgs a, const double *__restrict__ delta, const double *__restrict__ da_t,
                             const double *__restrict__ da_p, const double *__restrict__ coef, double *fbar) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int i = blockIdx.z + 1;
  if (j > m.ntm || k > m.npm - 1) return;
  const double *c = coef + 4 * (i - 1);
  const int64_t q = fidx(m, j, k, i);
  const double d = delta[q], b = fbar[q];
  double A = da_t[j] * da_p[k];
  if (k == m.npm - 1) A = A + da_t[j] * da_p[1];
  const double dbar = (d > 0.0) ? c[0] * b + c[2] * A : c[1] * b + c[3] * A;
  fbar[q] = b - da_weight(m, a, j, k, i) * dbar;
}

// dacc[i] += scale * (sum of realization i's block partials and pole-row
// chunk partials), fixed order.
__global__ void k_adj_dsum(const double *__restrict__ dpart, int nblk, const double *__restrict__ dpole, int nch,
                           double scale, double *dacc) {
  __shared__ double sh[64];
  const int i = blockIdx.x;
  double a = 0.0, b = 0.0;
  for (int q = threadIdx.x; q < nblk; q += blockDim.x) a = a + dpart[(int64_t)i * nblk + q];
  for (int q = threadIdx.x; q < nch; q += blockDim.x) b = b + dpole[(int64_t)i * nch + q];
  block_sum2(a, b, sh);
  a = a + b;
  if (threadIdx.x == 0) dacc[i] += scale * a;
}

// y += a*x1 + b*x2 on core cells (x2 may be null)
__global__ void k_adj_axpy2(Mesh m, double *y, double a, const double *__restrict__ x1, double b,
                            const double *__restrict__ x2) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.y * blockDim.y + threadIdx.y + 2;
  const int i = blockIdx.z + 1;
  if (j > m.ntm || k > m.npm - 1) return;
  const int64_t q = fidx(m, j, k, i);
  double v = y[q] + a * x1[q];
  if (x2) v += b * x2[q];
  y[q] = v;
}

// Partial derivatives of weno_face (kernels.cuh) with respect to its six
// inputs LN(j-2), LN(j-1), LN(j), LP(j-1), LP(j), LP(j+1): d[0..5].  The
// nonlinear weights are differentiated through: with w = D/(eps+4t^2)^2,
// d(sum OM*p)/dt = -16 OM (p - u) t / (eps + 4t^2) for each candidate.
__device__ __forceinline__ void weno_face_vjp(double LNm2, double LNm1, double LN0, double LPm1, double LP0,
                                              double LPp1, double DCMC_m1, double DCMC_0, double DCCP_m1,
                                              double DCCP_0, double DPT_m1, double DMCT_m1, double DMT_0,
                                              double DCPT_0, double eps_m1, double eps_0, double d[6]) {
  // minus side
  const double p0m = (kOne + DCMC_m1) * LNm1 - DCMC_m1 * LNm2;
  const double p1m = DCMC_0 * LNm1 + DCCP_m1 * LN0;
  const double t0 = DCMC_m1 * (LNm1 - LNm2), t1 = DCCP_m1 * (LN0 - LNm1);
  const double e0 = eps_m1 + kFour * (t0 * t0), e1 = eps_m1 + kFour * (t1 * t1);
  const double w0m = DPT_m1 / (e0 * e0), w1m = DMCT_m1 / (e1 * e1);
  const double sm = w0m + w1m;
  const double O0m = w0m / sm, O1m = w1m / sm;
  const double um = O0m * p0m + O1m * p1m;
  const double dt0 = -16.0 * O0m * (p0m - um) * t0 / e0;
  const double dt1 = -16.0 * O1m * (p1m - um) * t1 / e1;
  d[0] = -DCMC_m1 * O0m - DCMC_m1 * dt0;
  d[1] = (kOne + DCMC_m1) * O0m + DCMC_0 * O1m + DCMC_m1 * dt0 - DCCP_m1 * dt1;
  d[2] = DCCP_m1 * O1m + DCCP_m1 * dt1;
  // plus side
  const double p0p = (kOne + DCCP_0) * LP0 - DCCP_0 * LPp1;
  const double p1p = DCCP_m1 * LP0 + DCMC_0 * LPm1;
  const double t2 = DCCP_0 * (LPp1 - LP0), t3 = DCMC_0 * (LP0 - LPm1);
  const double e2 = eps_0 + kFour * (t2 * t2), e3 = eps_0 + kFour * (t3 * t3);
  const double w0p = DMT_0 / (e2 * e2), w1p = DCPT_0 / (e3 * e3);
  const double sp = w0p + w1p;
  const double O0p = w0p / sp, O1p = w1p / sp;
  const double up = O0p * p0p + O1p * p1p;
  const double dt2 = -16.0 * O0p * (p0p - up) * t2 / e2;
  const double dt3 = -16.0 * O1p * (p1p - up) * t3 / e3;
  d[3] = DCMC_0 * O1p - DCMC_0 * dt3;
  d[4] = (kOne + DCCP_0) * O0p + DCCP_m1 * O1p - DCCP_0 * dt2 + DCMC_0 * dt3;
  d[5] = -DCCP_0 * O0p + DCCP_0 * dt2;
}

// Reverse of one explicit advection stage at core cell (j,k):
//   out = alpha*w + beta*base + L_x^T(sigma*w)
// where L is advection_operator_weno3 linearised at x (analytic 1-D flows,
// WENO3 faces, upwind faces next to the poles, pole rings, periodic seam).
// gring holds w's pole sums.  The flow cotangents are accumulated per cell:
//   gln_t += LNbar*x/2 (for vt(j)+at(j)),  glp_t += LPbar*x/2 (vt(j+1)-at(j)),
//   gup_t += the upwind faces' vt cotangent (face j), and the same for phi
//   (gln_p, glp_p: vp(j) + ap(j), vp(j) - ap(j)).
struct AdjAdvArgs {
  double sigma, alpha, beta, bcfn, bcfs;
};

constexpr int kAAJ = 32, kAAK = 8;  // tile of k_adj_adv: theta rows x core columns (block 32 x 8)

// The reverse of one SSPRK stage on a tile of kAAJ x kAAK cells.  Each WENO3
// face's cotangent-weighted derivatives (Fb * d[0..5]) are computed once per
// tile into shared memory -- theta faces j0-1 .. j0+kAAJ+1 of the tile's
// columns, phi faces k0-1 .. k0+kAAK+1 of its interior rows -- and every cell
// then gathers the four faces on each axis that read it, in the order
// jf = j-1 .. j+2 (kf = k-1 .. k+2), so each sum has the operation order of
// one cell computing its faces itself.  Upwind pole faces and the phi faces
// that reach a cell through the periodic seam aliases are computed by the
// cell.
__global__ void __launch_bounds__(256, 3) k_adj_adv(Mesh m, Flow fl, Weno wn, const double *__restrict__ x,
                                                 const double *__restrict__ w, const double *__restrict__ base,
                                                 double *__restrict__ out, const double *__restrict__ gring,
                                                 AdjAdvArgs a, double *gln_t, double *glp_t, double *gup_t,
                                                 double *gln_p, double *glp_p) {
  __shared__ double tf[kAAK][kAAJ + 3][6];  // theta face jf = j0-1+e of column k0+c
  __shared__ double pf[kAAJ][kAAK + 3][6];  // phi face kf = k0-1+e of row j0+r
  const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + ty * kAAJ;
  const int j0 = blockIdx.x * kAAJ + 1, k0 = blockIdx.y * kAAK + 2;
  const int i = blockIdx.z + 1;
  const int ntm = m.ntm, npm = m.npm;
  const double gn = a.sigma * gring[2 * (i - 1)], gs = a.sigma * gring[2 * (i - 1) + 1];
  auto abar = [&](int jj, int kk) { return a.sigma * w[fidx(m, jj, kk, i)]; };
  auto X = [&](int jj, int kk) { return x[fidx(m, jj, kk, i)]; };
  // cotangent of flux_t(jf,k): divergence of cells jf-1 and jf, pole rings
  auto ftbar = [&](int jf, int k) {
    double v = 0.0;
    if (jf - 1 >= 2 && jf - 1 <= ntm - 1) v += abar(jf - 1, k) * m.sth[jf] * m.st_i[jf - 1] * m.dt_i[jf - 1];
    if (jf >= 2 && jf <= ntm - 1) v -= abar(jf, k) * m.sth[jf] * m.st_i[jf] * m.dt_i[jf];
    if (jf == 2) v += a.bcfn * m.dp[k] * gn;
    if (jf == ntm) v -= a.bcfs * m.dp[k] * gs;
    return v;
  };
  // cotangent of flux_p(j,kf): divergence of cells kf-1 (npm-1 for kf = 2) and kf
  auto fpbar = [&](int j, int kf) {
    double v = 0.0;
    if (kf >= 3) v += abar(j, kf - 1) * m.st_i[j] * m.dp_i[kf - 1];
    else v += abar(j, npm - 1) * m.st_i[j] * m.dp_i[npm - 1];
    v -= abar(j, kf) * m.st_i[j] * m.dp_i[kf];
    return v;
  };
  // Fb * d of the WENO theta face jf of column k (zeros where Fb is zero)
  auto theta_face = [&](int jf, int k, double *o) {
    const double Fb = ftbar(jf, k);
    if (Fb == 0.0) return;
    double LN[3], LP[3], d[6];
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const int c = jf - 2 + e;
      LN[e] = kHalf * X(c, k) * (vt_at(m, fl, c, k, i) + at_at(m, fl, c, k, i));
    }
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const int c = jf - 1 + e;
      LP[e] = kHalf * X(c, k) * (vt_at(m, fl, c + 1, k, i) - at_at(m, fl, c, k, i));
    }
    weno_face_vjp(LN[0], LN[1], LN[2], LP[0], LP[1], LP[2], wn.mct[jf - 1], wn.mct[jf], wn.cpt[jf - 1],
                  wn.cpt[jf], wn.pt[jf - 1], wn.mctt[jf - 1], wn.mt[jf], wn.cptt[jf], wn.epst[jf - 1],
                  wn.epst[jf], d);
#pragma unroll
    for (int q = 0; q < 6; ++q) o[q] = Fb * d[q];
  };
  // Fb * d of the phi face kf of row j
  auto phi_face = [&](int j, int kf, double *o) {
    const double Fb = fpbar(j, kf);
    if (Fb == 0.0) return;
    double LN[3], LP[3], d[6];
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const int c = wrap_cell(m, kf - 2 + e);
      LN[e] = kHalf * X(j, c) * (vp_at(m, fl, j, c, i) + ap_at(m, fl, j, c, i));
    }
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      const int c = wrap_cell(m, kf - 1 + e);
      LP[e] = kHalf * X(j, c) * (vp_at(m, fl, j, c + 1, i) - ap_at(m, fl, j, c, i));
    }
    weno_face_vjp(LN[0], LN[1], LN[2], LP[0], LP[1], LP[2], wn.mcp[kf - 1], wn.mcp[kf], wn.cpp[kf - 1],
                  wn.cpp[kf], wn.pp[kf - 1], wn.mctp[kf - 1], wn.mp[kf], wn.cptp[kf], wn.epsp[kf - 1],
                  wn.epsp[kf], d);
#pragma unroll
    for (int q = 0; q < 6; ++q) o[q] = Fb * d[q];
  };
  for (int e = tid; e < kAAK * (kAAJ + 3); e += kAAJ * kAAK) {
    const int c = e / (kAAJ + 3), f = e % (kAAJ + 3);
    const int k = k0 + c, jf = j0 - 1 + f;
    double *o = tf[c][f];
#pragma unroll
    for (int q = 0; q < 6; ++q) o[q] = 0.0;
    if (k <= npm - 1 && jf >= 3 && jf <= ntm - 1) theta_face(jf, k, o);
  }
  for (int e = tid; e < kAAJ * (kAAK + 3); e += kAAJ * kAAK) {
    const int r = e / (kAAK + 3), f = e % (kAAK + 3);
    const int j = j0 + r, kf = k0 - 1 + f;
    double *o = pf[r][f];
#pragma unroll
    for (int q = 0; q < 6; ++q) o[q] = 0.0;
    if (j >= 2 && j <= ntm - 1 && kf >= 2 && kf <= npm - 1) phi_face(j, kf, o);
  }
  __syncthreads();
  const int j = j0 + tx, k = k0 + ty;
  if (j > ntm || k > npm - 1) return;

  // ---- theta faces jf = j-1 .. j+2 of column k
  double lnb = 0.0, lpb = 0.0, xb = 0.0, upv = 0.0;
  for (int jf = j - 1; jf <= j + 2; ++jf) {
    if (jf < 2 || jf > ntm) continue;
    if (jf == 2 || jf == ntm) {  // upwind face: x(jf) high side, x(jf-1) low side
      const double Fb = ftbar(jf, k);
      if (Fb == 0.0) continue;
      const double v = vt_at(m, fl, jf, k, i), cct = copysign(fl.upwind, v);
      if (j == jf) {
        xb += Fb * v * kHalf * (kOne - cct);
        upv += Fb * kHalf * ((kOne - cct) * X(jf, k) + (kOne + cct) * X(jf - 1, k));
      }
      if (j == jf - 1) xb += Fb * v * kHalf * (kOne + cct);
    } else {
      const double *o = tf[ty][jf - (j0 - 1)];
      const int pos = j - jf;  // -2, -1, 0, 1
      if (pos == -2) lnb += o[0];
      if (pos == -1) {
        lnb += o[1];
        lpb += o[3];
      }
      if (pos == 0) {
        lnb += o[2];
        lpb += o[4];
      }
      if (pos == 1) lpb += o[5];
    }
  }
  const double xj = X(j, k);
  xb += lnb * kHalf * (vt_at(m, fl, j, k, i) + at_at(m, fl, j, k, i)) +
        lpb * kHalf * (vt_at(m, fl, j + 1, k, i) - at_at(m, fl, j, k, i));
  const int64_t q = fidx(m, j, k, i);
  gln_t[q] += lnb * kHalf * xj;
  glp_t[q] += lpb * kHalf * xj;
  gup_t[q] += upv;

  // ---- phi faces (interior rows): core faces kf = 2..npm-1, face npm is
  // the seam copy of face 2; cell index c' of the padded row (0..npm)
  // aliases core cell k when c' = k (faces from the tile), or c' = 0
  // (k = npm-2), 1 (k = npm-1), npm (k = 2) (faces computed here)
  if (j >= 2 && j <= ntm - 1) {
    double lnbp = 0.0, lpbp = 0.0;
    auto add = [&](const double *o, int pos) {
      if (pos == -2) lnbp += o[0];
      if (pos == -1) {
        lnbp += o[1];
        lpbp += o[3];
      }
      if (pos == 0) {
        lnbp += o[2];
        lpbp += o[4];
      }
      if (pos == 1) lpbp += o[5];
    };
    for (int kf = k - 1; kf <= k + 2; ++kf)
      if (kf >= 2 && kf <= npm - 1) add(pf[tx][kf - (k0 - 1)], k - kf);
    int cp = -1;
    if (k == npm - 2) cp = 0;
    if (k == npm - 1) cp = 1;
    if (k == 2) cp = npm;
    if (cp >= 0) {
      for (int kf = cp - 1; kf <= cp + 2; ++kf) {
        if (kf < 2 || kf > npm - 1) continue;
        double o[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        phi_face(j, kf, o);
        add(o, cp - kf);
      }
    }
    xb += lnbp * kHalf * (vp_at(m, fl, j, k, i) + ap_at(m, fl, j, k, i)) +
          lpbp * kHalf * (vp_at(m, fl, j, k + 1, i) - ap_at(m, fl, j, k, i));
    gln_p[q] += lnbp * kHalf * xj;
    glp_p[q] += lpbp * kHalf * xj;
  }
  double o = a.alpha * w[q] + xb;
  if (base) o += a.beta * base[q];
  out[q] = o;
}

}  // namespace hipft
