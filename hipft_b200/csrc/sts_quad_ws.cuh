// Four RKG2 stages per HBM pass on the interior theta blocks.
//
// Stages k..k+3 of diffusion_step_sts_cd (src/hipft.f90:5222-5237) with the
// 5-point operator of diffusion_operator_cd (src/hipft.f90:7927-7984).  A
// theta block is "interior" when the rows that its four stages compute, with
// their halos, stay clear of the pole rows 1 and ntm: then no stage of the
// block needs the pole-ring sums, which couple every phi column, and the
// block can advance four stages from one load of its inputs.  The pole blocks
// take the two-stage path twice (k_sts_pair_ws + k_pair_poles for stages
// k, k+1, then for k+2, k+3), which supplies the ring sums.
//
// A tile is 128 theta rows x 16 phi columns.  Its inputs are staged once:
// Y_{k-1} with a halo of 4 (136 rows x 24 columns) and Y_{k-2}, u0, dty0 with
// a halo of 3 (22 columns), together with the tile's rows of the row table
// (st_i, c2, c4) and columns of a column table ({P1, P5}).  The consumers then
// compute, in shared memory and in place,
//   stage k   on the tile plus 3 (over Y_{k-2}),
//   stage k+1 on the tile plus 2 (over Y_{k-1}),
//   stage k+2 on the tile plus 1 (over Y_k),
//   stage k+3 on the tile,
// and store Y_{k+2} and Y_{k+3} (the next pass's Y_{k-2}, Y_{k-1}) to HBM:
// per cell and four stages 4 reads + 2 writes = 48 B instead of 4 x 40 B
// (2 x 48 B on the two-stage path).  Every cell value is computed by the same
// expressions, in the same order, as on the two-stage path, so the results
// are bitwise the same.  The blocks next to a pole block also store the rows
// of Y_k (one) and Y_{k+1} (two) at their edge, which the pole block's second
// two-stage launch reads as its halo.
//
// Shared row r is theta row j0-4+r (r = 0..135; the stage-k pass also runs
// the unused rows 0 and 135 so that every row pair starts on a 16-byte
// boundary); shared column c of Y_{k-1} is phi column k0-4+c (c = 0..23) and
// column c-1 of the other arrays holds phi column k0-4+c.  One CTA per SM
// holds two tile buffers: one producer warp stages the next tile (five tensor
// copies and one bulk copy per tile, or one bulk copy per column at the phi
// seams) while sixteen consumer warps compute the current one; every wait is
// bounded and reports through the error flag.
#pragma once

#include "sts_pair_ws.cuh"

namespace hipft {

constexpr int kQJ = 128;                 // theta rows per tile
constexpr int kQK = 16;                  // phi columns per tile
constexpr int kQR = kQJ + 8;             // shared rows per column (halo 4)
constexpr int kQX = kQK + 8;             // shared columns of Y_{k-1} (halo 4)
constexpr int kQI = kQK + 6;             // shared columns of Y_{k-2}, u0, dty0 (halo 3)
constexpr int kQCons = 512;              // consumer threads (64 row pairs x 8 column groups)
constexpr int kQThreads = kQCons + 32;   // + the producer warp
constexpr int kQNB = 2;                  // tile buffers: the next tile loads while one is computed
constexpr int kQX1 = 0;                              // Y_{k-1}
constexpr int kQY2 = al16(kQX1 + kQX * kQR);         // Y_{k-2}
constexpr int kQU = al16(kQY2 + kQI * kQR);          // u0
constexpr int kQD = al16(kQU + kQI * kQR);           // dty0
constexpr int kQRT = al16(kQD + kQI * kQR);          // rows: st_i, c2, c4, kQR each
constexpr int kQCT = kQRT + 3 * kQR;                 // columns: {P1, P5} per shared column of Y_{k-1}
constexpr int kQInfo = kQCT + 2 * kQX;               // tile record: (kt, rb, i, nk)
constexpr int kQInfoCoef = kQInfo + 4;               // ragged batches: the tile's four StageCoef (20 doubles)
constexpr int kQBuf = al16(kQInfoCoef + 20);
constexpr size_t kQSmem = (size_t)kQNB * kQBuf * sizeof(double) + 2 * kQNB * sizeof(uint64_t);
static_assert(kQX1 % 16 == 0 && kQY2 % 16 == 0 && kQU % 16 == 0 && kQD % 16 == 0 && kQRT % 16 == 0 &&
                  kQCT % 2 == 0 && kQR % 2 == 0,
              "tensor-copy destinations 128-byte aligned, row pairs 16-byte aligned");
static_assert(kQSmem + 1024 <= 227 * 1024, "two tile buffers in one CTA per SM");

// Barriers of the quad kernel's consumer threads (named barrier 1).
__device__ __forceinline__ void qcons_sync() { asm volatile("bar.sync 1, 512;" ::: "memory"); }
__device__ __forceinline__ bool qcons_any(bool p) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred q, o;\n setp.ne.u32 q, %1, 0;\n bar.red.or.pred o, 1, 512, q;\n selp.u32 %0, 1, 0, o;\n}"
      : "=r"(r)
      : "r"((uint32_t)p)
      : "memory");
  return r != 0;
}

// Tensor maps of the quad tiles: fields with boxes of kQR rows x kQX (x1) or
// kQI (y2, u, d) columns, the row table with kQR x 3.
struct QuadMaps {
  CUtensorMap x1, y2, u, d, rt;
  int on;
};

struct QuadArgs {
  StageCoef c[4];        // stages k..k+3
  int *err;              // set to 1 when a bounded wait gives up
  int rb_lo, nbi;        // interior theta blocks rb_lo .. rb_lo+nbi-1
  int nkt;               // phi tiles of kQK columns
  int ntiles;            // nbi * nkt * realizations
  int edge_lo, edge_hi;  // blocks whose first / last rows of Y_k, Y_{k+1} the pole blocks read
  const double *col;     // column table: entry kk holds phi column kk-2 (mapped onto 2..npm-1)
  int LC;                // column-table entries per realization
  // ragged batches: realizations (0-based) of the launch, and per
  // realization the coefficients of stages k, k+1 (rcA[2(i-1)], rcA[2(i-1)+1])
  // and k+2, k+3 (rcB)
  const int *rlist;
  const StageCoef *rcA, *rcB;
};

// Column table of the quad tiles: entry kk (0..LC-1) of realization i holds
// {Dh dph_i(kw) dp_i(kw), Dh dph_i(kw+1) dp_i(kw)} for the interior column kw
// that phi column kk-2 duplicates (load_diffusion_matrix's order, src/hipft.f90:
// 6880-6920, as in k_pair_tables).
__global__ void k_quad_coltab(Mesh m, const double *__restrict__ dfac, int LC, double *coltab) {
  const int64_t ncol = (int64_t)m.nr * LC;
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < ncol; f += (int64_t)gridDim.x * blockDim.x) {
    const int i = (int)(f / LC) + 1, kk = (int)(f % LC);
    const int n2 = m.npm - 2;
    const int kw = ((kk - 2 - 2) % n2 + n2) % n2 + 2;
    const double Dr = dfac[i];
    const double Dh = kHalf * (Dr + Dr);
    coltab[2 * f] = Dh * m.dph_i[kw] * m.dp_i[kw];
    coltab[2 * f + 1] = Dh * m.dph_i[kw + 1] * m.dp_i[kw];
  }
}

__device__ __forceinline__ void quad_tile(const QuadArgs &qa, int t, int &kt, int &rb, int &i, bool ragged) {
  kt = t % qa.nkt;
  const int rest = t / qa.nkt;
  rb = qa.rb_lo + rest % qa.nbi;
  i = (ragged ? qa.rlist[rest / qa.nbi] : rest / qa.nbi) + 1;
}

// One stage over a rectangle of row pairs p in [p0, p0+np) and shared columns
// c in [c0, c0+nc) (columns of Y_{k-1}'s indexing).  S: the stencil input,
// O2: the combine's second input, OUT: the output (all in shared memory; an
// array with soff = 1 holds shared column c at index c-1).  store(r, c, y) is
// called for every computed pair (r = 2p).
template <typename Store>
__device__ __forceinline__ void quad_stage(int tid, int p0, int np, int c0, int nc, const double *S, int soff,
                                           const double *O2, int ooff, double *OUT, int woff, const double *U,
                                           const double *D, const double *RT, const double2 *CT,
                                           const StageCoef &sc, Store store) {
  const int n = np * nc;
  for (int e = tid; e < n; e += kQCons) {
    const int r = 2 * (p0 + e % np), c = c0 + e / np;
    const double *s = S + (c - soff) * kQR + r;
    const double2 xl = *reinterpret_cast<const double2 *>(s - kQR);
    const double2 xc = *reinterpret_cast<const double2 *>(s);
    const double2 xr = *reinterpret_cast<const double2 *>(s + kQR);
    const double up = s[-1], dn = s[2];
    const double2 st2 = *reinterpret_cast<const double2 *>(RT + r);
    const double2 c22 = *reinterpret_cast<const double2 *>(RT + kQR + r);
    const double2 c42 = *reinterpret_cast<const double2 *>(RT + 2 * kQR + r);
    const double2 o2 = *reinterpret_cast<const double2 *>(O2 + (c - ooff) * kQR + r);
    const double2 u = *reinterpret_cast<const double2 *>(U + (c - 1) * kQR + r);
    const double2 d = *reinterpret_cast<const double2 *>(D + (c - 1) * kQR + r);
    const double2 y = pair_rows_step(xl, xc, xr, up, dn, st2, c22, c42, CT[c], false, false, 0.0, 0.0, o2, u, d, sc);
    *reinterpret_cast<double2 *>(OUT + (c - woff) * kQR + r) = y;
    store(r, c, y);
  }
}

// The same stage over row pairs 2..65 (rows 4..131) and shared columns
// c0 .. c0+nc-1, by column marching: consumer thread t owns row pair
// 2 + (t % 64) and a quarter of the columns (t / 64), keeps the pair's row
// table (st2, c22, c42) and its stencil window (columns c-1, c, c+1) in
// registers, and takes the rows above and below from its warp neighbours
// (lanes 0 and 31 read theirs from shared memory).  Per cell pair it loads
// the next window column, the combine inputs and the column table: half the
// shared-memory reads of quad_stage.  O2 is read through OUT (the same array
// when the stage works in place; each unit reads only its own cell there).
template <typename Store>
__device__ __forceinline__ void quad_march(int tid, int c0, int nc, const double *__restrict__ S, int soff,
                                           double *OUT, int ooff, int woff, const double *__restrict__ U,
                                           const double *__restrict__ D, const double2 *__restrict__ CT,
                                           double2 st2, double2 c22, double2 c42, const StageCoef &sc, Store store) {
  constexpr int NG = kQCons / 64;  // column groups
  const int lane = tid & 31, g = tid >> 6;
  const int r = 4 + 2 * (tid & 63);
  const int cs = c0 + (g * nc) / NG, ce = c0 + ((g + 1) * nc) / NG;  // columns cs .. ce-1 (warp-uniform)
  if (cs >= ce) return;
  double2 xl = *reinterpret_cast<const double2 *>(S + (cs - 1 - soff) * kQR + r);
  double2 xc = *reinterpret_cast<const double2 *>(S + (cs - soff) * kQR + r);
  for (int c = cs; c < ce; ++c) {
    const double2 xr = *reinterpret_cast<const double2 *>(S + (c + 1 - soff) * kQR + r);
    double up = __shfl_up_sync(0xffffffffu, xc.y, 1);
    double dn = __shfl_down_sync(0xffffffffu, xc.x, 1);
    if (lane == 0) up = S[(c - soff) * kQR + r - 1];
    if (lane == 31) dn = S[(c - soff) * kQR + r + 2];
    const double2 o2 = *reinterpret_cast<const double2 *>(OUT + (c - ooff) * kQR + r);
    const double2 u = *reinterpret_cast<const double2 *>(U + (c - 1) * kQR + r);
    const double2 d = *reinterpret_cast<const double2 *>(D + (c - 1) * kQR + r);
    const double2 y = pair_rows_step(xl, xc, xr, up, dn, st2, c22, c42, CT[c], false, false, 0.0, 0.0, o2, u, d, sc);
    *reinterpret_cast<double2 *>(OUT + (c - woff) * kQR + r) = y;
    store(r, c, y);
    xl = xc;
    xc = xr;
  }
}

// Four RKG2 stages on the interior blocks (see the file comment).  Outputs:
// out_k2 = Y_{k+2}, out_k3 = Y_{k+3} on the tiles, and the edge rows of
// out_k = Y_k, out_k1 = Y_{k+1} on the blocks edge_lo / edge_hi.  RAGGED:
// the tiles of the realizations in qa.rlist, each with its own coefficients,
// which the producer copies into the tile record.
template <bool RAGGED>
__global__ void __launch_bounds__(kQThreads, 1) k_sts_quad_ws(Mesh m, const double *__restrict__ ykm1,
                                                             const double *__restrict__ ykm2,
                                                             const double *__restrict__ u0,
                                                             const double *__restrict__ dty0, double *out_k,
                                                             double *out_k1, double *out_k2, double *out_k3,
                                                             QuadArgs qa, PairTables pt,
                                                             const __grid_constant__ QuadMaps tm) {
  extern __shared__ __align__(128) double qsm[];
  uint64_t *full = reinterpret_cast<uint64_t *>(qsm + kQNB * kQBuf);
  uint64_t *empty = full + kQNB;
  const int tid = threadIdx.x;
  const int npm = m.npm;
  const int64_t ld = m.ldt;
  if (tid == 0) {
    for (int b = 0; b < kQNB; ++b) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], kQCons);
    }
    fence_mbar_init();
  }
  __syncthreads();

  if (tid >= kQCons) {
    // ------------------------------------------------------------ producer
    const int lane = tid - kQCons;
    const bool maps_ok = tm.on && (smem_addr(qsm) & 127u) == 0;
    int n = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < qa.ntiles; t += gridDim.x, ++n) {
      int kt, rb, i;
      quad_tile(qa, t, kt, rb, i, RAGGED);
      StageCoef rc[4] = {};
      if (RAGGED && lane == 0) {
        rc[0] = qa.rcA[2 * (i - 1)];
        rc[1] = qa.rcA[2 * (i - 1) + 1];
        rc[2] = qa.rcB[2 * (i - 1)];
        rc[3] = qa.rcB[2 * (i - 1) + 1];
      }
      const int j0 = rb * kQJ + 1, k0 = kt * kQK + 2;
      const int nk = min(kQK, npm - 1 - k0 + 1);
      const int64_t pbase = (int64_t)(i - 1) * m.plane;
      const int b = n % kQNB, u = n / kQNB;
      double *B = qsm + b * kQBuf;
      uint64_t *fb = &full[b];
      // buffer b is free once the consumers are done with its previous tile
      if (u >= 1 && !mbar_wait_bounded(&empty[b], (uint32_t)((u - 1) & 1), 1u << 22)) {
        ok = false;
        break;
      }
      const bool boxed = maps_ok && nk == kQK && k0 - 4 >= 1 && k0 + kQK + 3 <= npm;
      const uint32_t run = kQR * 8u;  // rows j0-4 .. j0+131, all inside 1..ntm for an interior block
      if (lane == 0) {
        int *Ii = reinterpret_cast<int *>(B + kQInfo);
        Ii[0] = kt;
        Ii[1] = rb;
        Ii[2] = i;
        Ii[3] = nk;
        if (RAGGED) {
          double *C = B + kQInfoCoef;
          for (int q = 0; q < 4; ++q) {
            C[5 * q] = rc[q].a;
            C[5 * q + 1] = rc[q].b;
            C[5 * q + 2] = rc[q].c;
            C[5 * q + 3] = rc[q].d;
            C[5 * q + 4] = rc[q].e;
          }
        }
        mbar_expect_tx(fb, (uint32_t)((kQX + 3 * kQI) * kQR * 8 + 3 * kQR * 8 + kQX * 16));
        if (boxed) {
          tma_load_3d(B + kQX1, &tm.x1, j0 - 5, k0 - 5, i - 1, fb);
          tma_load_3d(B + kQY2, &tm.y2, j0 - 5, k0 - 4, i - 1, fb);
          tma_load_3d(B + kQU, &tm.u, j0 - 5, k0 - 4, i - 1, fb);
          tma_load_3d(B + kQD, &tm.d, j0 - 5, k0 - 4, i - 1, fb);
          tma_load_3d(B + kQRT, &tm.rt, rb * kQJ - 2, 0, i - 1, fb);
          bulk_load(B + kQCT, qa.col + ((int64_t)(i - 1) * qa.LC + (int64_t)kt * kQK) * 2, kQX * 16, fb);
        }
      }
      __syncwarp();
      if (!boxed) {
        // one bulk copy per column (phi seam tiles, or no tensor maps)
        const int ncp = kQX + 3 * kQI + 4;
        for (int q = lane; q < ncp; q += 32) {
          const double *src;
          double *dst;
          uint32_t bytes = run;
          if (q < kQX) {
            const int kg = wrap_col(k0 - 4 + q, npm);
            src = ykm1 + pbase + (int64_t)(kg - 1) * ld + (j0 - 5);
            dst = B + kQX1 + q * kQR;
          } else if (q < kQX + 3 * kQI) {
            const int qq = q - kQX, a = qq / kQI, c = qq % kQI;
            const int kg = wrap_col(k0 - 3 + c, npm);
            src = (a == 0 ? ykm2 : (a == 1 ? u0 : dty0)) + pbase + (int64_t)(kg - 1) * ld + (j0 - 5);
            dst = B + (a == 0 ? kQY2 : (a == 1 ? kQU : kQD)) + c * kQR;
          } else if (q < kQX + 3 * kQI + 3) {
            const int a = q - (kQX + 3 * kQI);
            src = pt.row + ((int64_t)(i - 1) * 3 + a) * pt.LR + (int64_t)(rb * kQJ - 2);
            dst = B + kQRT + a * kQR;
          } else {
            src = qa.col + ((int64_t)(i - 1) * qa.LC + (int64_t)kt * kQK) * 2;
            dst = B + kQCT;
            bytes = kQX * 16;
          }
          bulk_load(dst, src, bytes, fb);
        }
      }
    }
    if (!ok && lane == 0) atomicExch(qa.err, 1);
    // every issued copy lands before this warp exits (tiles 0..n-1 were issued)
    for (int b = 0; b < kQNB; ++b) {
      int last = n - 1;
      while (last >= 0 && last % kQNB != b) --last;
      if (last >= 0) mbar_wait_bounded(&full[b], (uint32_t)((last / kQNB) & 1), 1u << 22);
    }
    return;
  }

  // -------------------------------------------------------------- consumers
  StageCoef s0 = qa.c[0], s1 = qa.c[1], s2 = qa.c[2], s3 = qa.c[3];
  const int64_t seam = (int64_t)(npm - 2) * ld;
  int n = 0;
  for (int t = blockIdx.x; t < qa.ntiles; t += gridDim.x, ++n) {
    const int bq = n % kQNB, uq = n / kQNB;
    const bool landed = mbar_wait_bounded(&full[bq], (uint32_t)(uq & 1), 1u << 22);
    if (qcons_any(!landed)) {
      if (tid == 0) atomicExch(qa.err, 1);
      break;
    }
    double *B = qsm + bq * kQBuf;
    const int *Ii = reinterpret_cast<const int *>(B + kQInfo);
    const int kt = Ii[0], rb = Ii[1], i = Ii[2], nk = Ii[3];
    if (RAGGED) {
      const double *C = B + kQInfoCoef;
      s0 = StageCoef{C[0], C[1], C[2], C[3], C[4]};
      s1 = StageCoef{C[5], C[6], C[7], C[8], C[9]};
      s2 = StageCoef{C[10], C[11], C[12], C[13], C[14]};
      s3 = StageCoef{C[15], C[16], C[17], C[18], C[19]};
    }
    const int j0 = rb * kQJ + 1, k0 = kt * kQK + 2;
    const int64_t pbase = (int64_t)(i - 1) * m.plane;
    double *X = B + kQX1, *Y2 = B + kQY2;
    const double *U = B + kQU, *D = B + kQD, *RT = B + kQRT;
    const double2 *CT = reinterpret_cast<const double2 *>(B + kQCT);
    const bool elo = (rb == qa.edge_lo), ehi = (rb == qa.edge_hi);
    // a value of shared cell (r, c) to HBM (with its seam copy), for the
    // tile's own columns c = 4 .. 3+nk
    auto put = [&](double *g, int r, int c, double2 y) {
      const int k = k0 - 4 + c;
      double *q = g + pbase + (int64_t)(k - 1) * ld + (j0 - 5 + r);
      *reinterpret_cast<double2 *>(q) = y;
      if (k == 2) *reinterpret_cast<double2 *>(q + seam) = y;
      if (k == npm - 1) *reinterpret_cast<double2 *>(q - seam) = y;
    };
    const int cend = 4 + nk;  // one past the tile's last shared column
    // the row pair of this thread's column march (rows 4..131), for all four stages
    const int rm = 4 + 2 * (tid & 63);
    const double2 st2 = *reinterpret_cast<const double2 *>(RT + rm);
    const double2 c22 = *reinterpret_cast<const double2 *>(RT + kQR + rm);
    const double2 c42 = *reinterpret_cast<const double2 *>(RT + 2 * kQR + rm);
    // stage k on rows 0..135 (1..134 valid), columns 1..cend+2, over Y_{k-2}
    auto st_k = [&](int r, int c, double2 y) {
      // Y_k at the edge row a neighbouring pole block reads (rows j0 or j0+127)
      if (c >= 4 && c < cend && ((elo && r == 4) || (ehi && r == 130))) {
        const int k = k0 - 4 + c;
        double *q = out_k + pbase + (int64_t)(k - 1) * ld + (j0 - 5 + r);
        const int rr = (r == 4) ? 0 : 1;  // row j0 is the pair's first row, row j0+127 its second
        const double v = rr ? y.y : y.x;
        q[rr] = v;
        if (k == 2) q[rr + seam] = v;
        if (k == npm - 1) q[rr - seam] = v;
      }
    };
    quad_march(tid, 1, nk + 6, X, 0, Y2, 1, 1, U, D, CT, st2, c22, c42, s0, st_k);
    quad_stage(tid, 0, 2, 1, nk + 6, X, 0, Y2, 1, Y2, 1, U, D, RT, CT, s0, st_k);
    quad_stage(tid, 66, 2, 1, nk + 6, X, 0, Y2, 1, Y2, 1, U, D, RT, CT, s0, st_k);
    qcons_sync();
    // stage k+1 on rows 2..133, columns 2..cend+1, stencil Y_k, over Y_{k-1}
    auto st_k1 = [&](int r, int c, double2 y) {
      // Y_{k+1} at the two edge rows (j0, j0+1 or j0+126, j0+127)
      if (c >= 4 && c < cend && ((elo && r == 4) || (ehi && r == 130))) put(out_k1, r, c, y);
    };
    quad_march(tid, 2, nk + 4, Y2, 1, X, 0, 0, U, D, CT, st2, c22, c42, s1, st_k1);
    quad_stage(tid, 1, 1, 2, nk + 4, Y2, 1, X, 0, X, 0, U, D, RT, CT, s1, st_k1);
    quad_stage(tid, 66, 1, 2, nk + 4, Y2, 1, X, 0, X, 0, U, D, RT, CT, s1, st_k1);
    qcons_sync();
    // stage k+2 on rows 2..133 (3..132 valid), columns 3..cend, stencil Y_{k+1}, over Y_k
    auto st_k2 = [&](int r, int c, double2 y) {
      if (c >= 4 && c < cend && r >= 4 && r <= 130) put(out_k2, r, c, y);
    };
    quad_march(tid, 3, nk + 2, X, 0, Y2, 1, 1, U, D, CT, st2, c22, c42, s2, st_k2);
    quad_stage(tid, 1, 1, 3, nk + 2, X, 0, Y2, 1, Y2, 1, U, D, RT, CT, s2, st_k2);
    quad_stage(tid, 66, 1, 3, nk + 2, X, 0, Y2, 1, Y2, 1, U, D, RT, CT, s2, st_k2);
    qcons_sync();
    // stage k+3 on the tile: rows 4..131, columns 4..cend-1, stencil Y_{k+2},
    // second input Y_{k+1} (the shared copy of Y_{k+3} is not read again)
    quad_march(tid, 4, nk, Y2, 1, X, 0, 0, U, D, CT, st2, c22, c42, s3,
               [&](int r, int c, double2 y) { put(out_k3, r, c, y); });
    qcons_sync();              // all reads of the buffer are done
    mbar_arrive(&empty[bq]);   // the producer may refill it
  }
}

}  // namespace hipft
