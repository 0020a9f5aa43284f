// Two RKG2 stages per launch, persistent and warp-specialised.
//
// Same tiles and the same arithmetic as k_sts_pair (stages k and k+1 of
// diffusion_step_sts_cd, src/hipft.f90:5222-5237, with the 5-point operator of
// diffusion_operator_cd, src/hipft.f90:7927-7984), organised so that HBM is
// busy while the SMs compute:
//
//  * one producer warp walks the CTA's tiles and fills a ring of two tile
//    buffers: Y_{k-1} on the tile plus a halo of 2, Y_{k-2}, u0 and dty0 plus
//    a halo of 1, and the tile's rows and columns of two coefficient tables
//    precomputed in HBM (k_pair_tables).  A tile whose halo columns need no
//    phi wrap takes five 3-D tensor copies (cp.async.bulk.tensor, one box per
//    array) and one bulk copy; the seam tiles take one 1-D bulk copy
//    (cp.async.bulk) per column.  The number of copies per tile, not their
//    bytes, had bounded the load rate: 46 copies per tile ran 20% slower per
//    clock than 6;
//    each buffer has a "full" mbarrier (copies landed) and an "empty" one (all
//    consumers done reading it); every wait is bounded and reports through the
//    error flag;
//  * eight consumer warps compute Y_k on the tile plus a halo of 1 into a
//    shared array of their own, then Y_{k+1} on the tile.  A consumer thread
//    owns one theta row and half of the tile's phi columns and marches along
//    phi with a three-value register window, so a cell costs six shared loads
//    per stage.  The consumers synchronise with named barrier 1 only.
//
// Tiles are walked phi tile fastest, so every CTA sees every theta block.
// Each buffer also carries a small tile record (realization, tile indices,
// D and the pole terms of the input's ring sums) that the producer writes
// before its arrival, so consumers start a tile without global loads or
// index division.  Shared memory per CTA: 2 x 48.8 KB buffers + 10.6 KB for
// Y_k = 108 KB, two CTAs per SM.  Tiles holding rows 2 / ntm-1 publish ring partials of Y_k; the
// pole rows of Y_{k+1} and its ring sums are finished by k_pair_poles in a
// launch of its own.
#pragma once

#include <cuda.h>  // CUtensorMap

#include "kernels.cuh"

namespace hipft {

constexpr int kWJ = 128;                  // theta rows per tile
constexpr int kWK = 8;                    // phi columns per tile
constexpr int kWR = kWJ + 4;              // shared rows per column (theta halo 2)
constexpr int kWNB = 2;                   // tile buffers
constexpr int kWCons = 256;               // consumer threads
constexpr int kWThreads = kWCons + 32;    // + the producer warp
// doubles, offsets within one tile buffer; the destinations of tensor copies
// start on 128-byte boundaries
constexpr int al16(int x) { return (x + 15) / 16 * 16; }
constexpr int kWX1 = 0;                             // Y_{k-1}: kWK+4 columns (shared columns 0..kWK+3)
constexpr int kWY2 = al16(kWX1 + (kWK + 4) * kWR);  // Y_{k-2}: kWK+2 columns (shared columns 1..kWK+2)
constexpr int kWU = al16(kWY2 + (kWK + 2) * kWR);   // u0
constexpr int kWD = al16(kWU + (kWK + 2) * kWR);    // dty0
constexpr int kWRT = al16(kWD + (kWK + 2) * kWR);   // rows: st_i, c2, c4, each kWR long
constexpr int kWCT = kWRT + 3 * kWR;                // columns: {P1, P5} per shared column
constexpr int kWInfo = kWCT + 2 * (kWK + 4);       // tile record: D, pole terms, (kt, rb, i), stage coefficients
constexpr int kWInfoCoef = kWInfo + 5;              // ragged batches: the tile's two StageCoef (10 doubles)
constexpr int kWBuf = al16(kWInfo + 16);
constexpr int kWYk = kWNB * kWBuf;                  // Y_k: kWK+2 columns, consumers only
constexpr int kWEnd = kWYk + (kWK + 2) * kWR;
constexpr size_t kWSmem = (size_t)kWEnd * sizeof(double) + 2 * kWNB * sizeof(uint64_t);
static_assert(kWX1 % 16 == 0 && kWY2 % 16 == 0 && kWU % 16 == 0 && kWD % 16 == 0 && kWRT % 16 == 0 &&
                  kWCT % 2 == 0 && kWBuf % 16 == 0 && kWYk % 2 == 0 && kWEnd % 2 == 0,
              "tensor-copy destinations 128-byte aligned, bulk-copy destinations 16-byte aligned");
static_assert(2 * (kWSmem + 1024 + 256) <= 228 * 1024, "two CTAs per SM");

// Tensor maps of the tile loads (3-D: theta row, phi column, realization;
// f64, no swizzle, zero fill outside): x1 with a box of kWR x (kWK+4) x 1,
// y2, u and d with kWR x (kWK+2) x 1, and the row table ([nr][3][LR]) with
// kWR x 3 x 1.  With `on` set, a tile whose halo columns need no phi wrap
// takes five tensor copies instead of one bulk copy per column.
struct WsMaps {
  CUtensorMap x1, y2, u, d, rt;
  int on;
};
static_assert((kWR * 8) % 16 == 0, "column stride must keep 16-byte alignment");

// Coefficient tables of the two-stage kernels, in load_diffusion_matrix's
// operation order (src/hipft.f90:6880-6920) for a per-realization constant D:
//   rows    [nr][3][LR]: entry jj of the three arrays holds theta row j = jj-1:
//           st_i(j), Dh dth_i(j) dt_i(j) st_i(j) sth(j), Dh dth_i(j+1) dt_i(j) st_i(j) sth(j+1)
//           for 2 <= j <= ntm-1, zeros elsewhere (separate arrays, so that
//           consecutive rows are consecutive in shared memory);
//   columns [nr][LC][2]: entry kk holds phi column kk mapped onto the interior
//           column kw in 2..npm-1 it duplicates: {Dh dph_i(kw) dp_i(kw), Dh dph_i(kw+1) dp_i(kw)}.
__global__ void k_pair_tables(Mesh m, const double *__restrict__ dfac, int LR, int LC, double *rowtab,
                              double *coltab) {
  const int64_t nrow = (int64_t)m.nr * LR, ncol = (int64_t)m.nr * LC;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nrow + ncol;
       e += (int64_t)gridDim.x * blockDim.x) {
    if (e < nrow) {
      const int i = (int)(e / LR) + 1, j = (int)(e % LR) - 1;
      const double Dr = dfac[i];
      const double Dh = kHalf * (Dr + Dr);
      double st = 0.0, c2 = 0.0, c4 = 0.0;
      if (j >= 2 && j <= m.ntm - 1) {
        st = m.st_i[j];
        c2 = Dh * m.dth_i[j] * m.dt_i[j] * st * m.sth[j];
        c4 = Dh * m.dth_i[j + 1] * m.dt_i[j] * st * m.sth[j + 1];
      }
      double *o = rowtab + (int64_t)(i - 1) * 3 * LR + (e % LR);
      o[0] = st;
      o[LR] = c2;
      o[2 * LR] = c4;
    } else {
      const int64_t f = e - nrow;
      const int i = (int)(f / LC) + 1, kk = (int)(f % LC);
      const int n2 = m.npm - 2;
      const int kw = ((kk - 2) % n2 + n2) % n2 + 2;
      const double Dr = dfac[i];
      const double Dh = kHalf * (Dr + Dr);
      coltab[2 * f] = Dh * m.dph_i[kw] * m.dp_i[kw];
      coltab[2 * f + 1] = Dh * m.dph_i[kw + 1] * m.dp_i[kw];
    }
  }
}

// Exercises the error path of the bounded waits: waits for phase 0 of an
// mbarrier that expects one arrival nobody makes, gives up after `limit`
// polls, sets the error flag and returns (no copy is in flight).
__global__ void k_wait_selftest(uint32_t limit, int *err) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (!mbar_wait_bounded(&bar, 0, limit) && threadIdx.x == 0) atomicExch(err, 1);
}

__device__ __forceinline__ void cons_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

// true on every consumer thread if p is true on any of them (named barrier 1)
__device__ __forceinline__ bool cons_any(bool p) {
  uint32_t r;
  asm volatile(
      "{\n .reg .pred q, o;\n setp.ne.u32 q, %1, 0;\n bar.red.or.pred o, 1, 256, q;\n selp.u32 %0, 1, 0, o;\n}"
      : "=r"(r)
      : "r"((uint32_t)p)
      : "memory");
  return r != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ int wrap_col(int c, int npm) {
  if (c < 1) return c + (npm - 2);
  if (c > npm) return c - (npm - 2);
  return c;
}

struct PairTables {
  const double *row, *col;  // k_pair_tables output
  int LR, LC;               // entries per realization
  int nb, nkt, ntiles;      // theta blocks, phi tiles, all tiles
  // nsel > 0: the launch covers only theta blocks sel[0..nsel-1] (the pole
  // blocks, when the interior blocks take four stages per pass)
  int nsel = 0;
  int sel[6] = {};
};

// One stencil-and-combine step for a theta-row pair (a, b = a+1) of one
// column, in the single-row kernels' operation order: xl, xc, xr the pair in
// columns c-1, c, c+1 of the stage input; up = row a-1 and dn = row b+1 of
// column c; st2, c22, c42 the rows' st_i, c2, c4; P the column's {P1, P5};
// pole rows take ax from the ring sums; o2 the second input (Y_{k-2} for
// stage k, Y_{k-1} for stage k+1), u = u0, d = dty0.
__device__ __forceinline__ double2 pair_rows_step(double2 xl, double2 xc, double2 xr, double up, double dn,
                                                  double2 st2, double2 c22, double2 c42, double2 P, bool pola,
                                                  bool polb, double axpa, double axpb, double2 o2, double2 u,
                                                  double2 d, const StageCoef &sc) {
  double axa, axb;
  if (pola) {
    axa = axpa;
  } else {
    const double st = st2.x, c2 = c22.x, c4 = c42.x;
    const double c1 = P.x * st * st;
    const double c5 = P.y * st * st;
    const double c3 = -(c1 + c2 + c4 + c5);
    axa = c1 * xl.x + c2 * up + c3 * xc.x + c4 * xc.y + c5 * xr.x;
  }
  if (polb) {
    axb = axpb;
  } else {
    const double st = st2.y, c2 = c22.y, c4 = c42.y;
    const double c1 = P.x * st * st;
    const double c5 = P.y * st * st;
    const double c3 = -(c1 + c2 + c4 + c5);
    axb = c1 * xl.y + c2 * xc.x + c3 * xc.y + c4 * dn + c5 * xr.y;
  }
  return make_double2(sc.a * xc.x + sc.b * o2.x + sc.c * u.x + sc.d * axa + sc.e * d.x,
                      sc.a * xc.y + sc.b * o2.y + sc.c * u.y + sc.d * axb + sc.e * d.y);
}

// The pair's value to HBM (16-byte store when both rows are kept) and to the
// seam column it duplicates.
__device__ __forceinline__ void store_pair(double *g, double2 y, bool va, bool vb, int64_t seam_off) {
  if (va && vb) {
    *reinterpret_cast<double2 *>(g) = y;
    if (seam_off) *reinterpret_cast<double2 *>(g + seam_off) = y;
  } else {
    if (va) g[0] = y.x;
    if (vb) g[1] = y.y;
    if (seam_off) {
      if (va) g[seam_off] = y.x;
      if (vb) g[seam_off + 1] = y.y;
    }
  }
}

// Tile t of a launch: phi tile kt, theta block rb, realization i.  Theta
// blocks go in the order 1..nb-2, 0, nb-1: interior tiles first, so that the
// wait for the previous pole kernel comes as late as possible.  In a ragged
// batch the launch covers only the realizations in rlist (pt.ntiles counts
// their tiles).
__device__ __forceinline__ void ws_tile(const PairTables &pt, int t, int &kt, int &rb, int &i,
                                        const int *rlist) {
  kt = t % pt.nkt;
  const int rest = t / pt.nkt;
  if (pt.nsel > 0) {
    rb = pt.sel[rest % pt.nsel];
    i = (rlist ? rlist[rest / pt.nsel] : rest / pt.nsel) + 1;
    return;
  }
  const int q = rest % pt.nb;
  i = (rlist ? rlist[rest / pt.nb] : rest / pt.nb) + 1;
  rb = (pt.nb <= 2) ? q : ((q < pt.nb - 2) ? q + 1 : ((q == pt.nb - 2) ? 0 : pt.nb - 1));
}

// Bulk stores of one tile column set: lane q < kWK writes column k0+q (theta
// rows j0..j0+kWJ-1, kWJ*8 bytes) from src0 + q*kWR; lanes kWK and kWK+1 write
// the seam columns (npm duplicates column 2, column 1 duplicates npm-1).
// Each issuing lane commits its own bulk async-group.
__device__ __forceinline__ void ws_store_cols(double *out, int64_t pbase, int k0, int j0, const double *src0, int lane,
                                              int npm, int64_t ld) {
  int c = -1, kg = 0;
  if (lane < kWK) {
    c = lane;
    kg = k0 + lane;
  } else if (lane == kWK && k0 == 2) {
    c = 0;
    kg = npm;
  } else if (lane == kWK + 1 && k0 + kWK - 1 == npm - 1) {
    c = kWK - 1;
    kg = 1;
  }
  if (c >= 0) {
    bulk_store(out + pbase + (int64_t)(kg - 1) * ld + (j0 - 1), src0 + c * kWR, kWJ * 8u);
    bulk_commit();
  }
}

// BULKST (with ROWPAIRS and a separate pole kernel): on tiles of kWK full
// columns and kWJ rows inside 1..ntm, Y_k goes to HBM by bulk stores from
// its shared array and Y_{k+1} by bulk stores from the tile buffer's Y_{k-2}
// region (free after stage k), issued by the producer when the consumers
// release the buffer; no consumer thread stores to global memory there.
// Those stores also write the pole rows 1 / ntm of Y_{k+1} with unused
// values; k_pair_poles, launched after this kernel, overwrites them.
//
// RAGGED: the launch advances the realizations of pa.rlist, each with its
// own stage coefficients pa.rc[2(i-1)], pa.rc[2(i-1)+1]; the producer copies
// them into the tile record, so the consumers read them from shared memory.
template <bool ROWPAIRS, bool BULKST = false, bool RAGGED = false>
__global__ void __launch_bounds__(kWThreads, 2) k_sts_pair_ws(Mesh m, const double *__restrict__ dfac,
                                                             const double *__restrict__ ykm1,
                                                             const double *__restrict__ ykm2,
                                                             const double *__restrict__ u0,
                                                             const double *__restrict__ dty0, double *out_k,
                                                             double *out_k1, const double *__restrict__ ring_in,
                                                             double bcn, double bcs, PairArgs pa, RingOut ro,
                                                             PairTables pt, const __grid_constant__ WsMaps tm) {
  extern __shared__ __align__(128) double wsm[];
  uint64_t *full = reinterpret_cast<uint64_t *>(wsm + kWEnd);
  uint64_t *empty = full + kWNB;
  static_assert(!BULKST || ROWPAIRS, "bulk stores need the row-pair consumers");

  const int tid = threadIdx.x;
  const int ntm = m.ntm, npm = m.npm;
  const int64_t ld = m.ldt;
  // tiles and coefficients of this launch: from the launch arguments, or in a
  // graph-run step from the device's pair counter
  int ntiles = pt.ntiles;
  const StageCoef *rcp = pa.rc;
  if (RAGGED && pa.dctr) {
    const int pq = *pa.dctr + pa.doff;
    ntiles = (pt.nsel > 0 ? pt.nsel : pt.nb) * pt.nkt * pa.dnact[pq];
    rcp = pa.rc + (int64_t)pq * pa.dstride;
  }
  if (tid == 0) {
    for (int b = 0; b < kWNB; ++b) {
      mbar_init(&full[b], 1);
      mbar_init(&empty[b], kWCons);
    }
    fence_mbar_init();
  }
  __syncthreads();

  if (tid >= kWCons) {
    // ------------------------------------------------------------ producer
    const int lane = tid - kWCons;
    int n = 0;
    bool ok = true, dep_done = false;
    const bool maps_ok = tm.on && (smem_addr(wsm) & 127u) == 0;
    auto store_prev_k1 = [&](int tp, const double *Bp) {
      int ktp, rbp, ip;
      ws_tile(pt, tp, ktp, rbp, ip, RAGGED ? pa.rlist : nullptr);
      const int j0p = rbp * kWJ + 1, k0p = ktp * kWK + 2;
      if (k0p + kWK - 1 <= npm - 1 && j0p + kWJ - 1 <= ntm)
        ws_store_cols(out_k1, (int64_t)(ip - 1) * m.plane, k0p, j0p, Bp + kWY2, lane, npm, ld);
    };
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++n) {
      const int b = n % kWNB, u = n / kWNB;
      int kt, rb, i;
      ws_tile(pt, t, kt, rb, i, RAGGED ? pa.rlist : nullptr);
      const int j0 = rb * kWJ + 1, k0 = kt * kWK + 2;
      const int nk = min(kWK, npm - 1 - k0 + 1);
      const int rs = max(1, j0 - 2), re = min((int)ld, j0 + kWJ + 1);
      const uint32_t run = (uint32_t)(re - rs + 1) * 8u;
      const int roff = rs - (j0 - 2);
      const int64_t pbase = (int64_t)(i - 1) * m.plane;
      double *B = wsm + b * kWBuf;
      const int nx = nk + 4, ny = nk + 2, ncp = nx + 3 * ny + 4;
      // tensor copies when every halo column lies in 1..npm (no phi wrap)
      const bool boxed = maps_ok && nk == kWK && k0 - 2 >= 1 && k0 + kWK + 1 <= npm;
      // Launched programmatically after the previous pair's k_pair_poles,
      // this kernel may start while that one still runs; it reads and writes
      // the pole rows 1, ntm, the rows 2, ntm-1 next to them and the ring
      // sums.  Tiles whose rows (with halo) reach those rows wait for it to
      // finish first; the other tiles touch none of them.  (Without such a
      // launch the wait returns at once.)
      if (!dep_done && (j0 - 2 <= 2 || j0 + kWJ + 1 >= ntm - 1)) {
        asm volatile("griddepcontrol.wait;" ::: "memory");
        dep_done = true;
      }
      // the tile record's global loads go out before the wait for the
      // buffer, so their latency hides behind it
      double rd = 0.0, rn = 0.0, rsv = 0.0;
      StageCoef rca{}, rcb{};
      if (RAGGED && lane == 0) {
        rca = rcp[2 * (i - 1)];
        rcb = rcp[2 * (i - 1) + 1];
      }
      if (lane == 0) {
        rd = dfac[i];
        if (dep_done) {  // used by pole tiles only
          rn = ring_in[2 * (i - 1)] * bcn;
          rsv = -ring_in[2 * (i - 1) + 1] * bcs;
        }
      }
      if (u >= 1 && !mbar_wait_bounded(&empty[b], (uint32_t)((u - 1) & 1), 1u << 22)) {
        ok = false;
        break;
      }
      if (BULKST && u >= 1) {
        // Y_{k+1} of the tile that used this buffer before, from its
        // Y_{k-2} region; read out before the buffer is refilled
        store_prev_k1(t - kWNB * (int)gridDim.x, B);
        bulk_wait_read();
        __syncwarp();
      }
      if (lane == 0) {
        // the tile record, written before the arrival that releases it
        double *I = B + kWInfo;
        I[0] = rd;
        I[1] = rn;
        I[2] = rsv;
        int *Ii = reinterpret_cast<int *>(I + 3);
        Ii[0] = kt;
        Ii[1] = rb;
        Ii[2] = i;
        if (RAGGED) {
          double *C = B + kWInfoCoef;
          C[0] = rca.a; C[1] = rca.b; C[2] = rca.c; C[3] = rca.d; C[4] = rca.e;
          C[5] = rcb.a; C[6] = rcb.b; C[7] = rcb.c; C[8] = rcb.d; C[9] = rcb.e;
        }
        if (boxed) {
          // five tensor copies (halo rows outside the field read as zeros;
          // x = j0-3 keeps the innermost offset a multiple of 16 bytes) and
          // the column table
          mbar_expect_tx(&full[b], (uint32_t)((nx + 3 * ny) * kWR * 8 + 3 * kWR * 8 + (kWK + 4) * 16));
          tma_load_3d(B + kWX1, &tm.x1, j0 - 3, k0 - 3, i - 1, &full[b]);
          tma_load_3d(B + kWY2, &tm.y2, j0 - 3, k0 - 2, i - 1, &full[b]);
          tma_load_3d(B + kWU, &tm.u, j0 - 3, k0 - 2, i - 1, &full[b]);
          tma_load_3d(B + kWD, &tm.d, j0 - 3, k0 - 2, i - 1, &full[b]);
          tma_load_3d(B + kWRT, &tm.rt, rb * kWJ, 0, i - 1, &full[b]);
          bulk_load(B + kWCT, pt.col + ((int64_t)(i - 1) * pt.LC + (int64_t)kt * kWK) * 2, (kWK + 4) * 16,
                    &full[b]);
        } else {
          mbar_expect_tx(&full[b], (uint32_t)(nx + 3 * ny) * run + (uint32_t)(3 * kWR * 8 + (kWK + 4) * 16));
        }
      }
      __syncwarp();
      for (int q = lane; q < (boxed ? 0 : ncp); q += 32) {
        const double *src;
        double *dst;
        uint32_t bytes = run;
        if (q < nx) {
          const int kg = wrap_col(k0 - 2 + q, npm);
          src = ykm1 + pbase + (int64_t)(kg - 1) * ld + (rs - 1);
          dst = B + kWX1 + q * kWR + roff;
        } else if (q < nx + 3 * ny) {
          const int qq = q - nx, a = qq / ny, c = 1 + qq % ny;
          const int kg = wrap_col(k0 - 2 + c, npm);
          const int64_t g = pbase + (int64_t)(kg - 1) * ld + (rs - 1);
          src = (a == 0 ? ykm2 : (a == 1 ? u0 : dty0)) + g;
          dst = B + (a == 0 ? kWY2 : (a == 1 ? kWU : kWD)) + (c - 1) * kWR + roff;
        } else if (q < nx + 3 * ny + 3) {
          const int a = q - (nx + 3 * ny);
          src = pt.row + ((int64_t)(i - 1) * 3 + a) * pt.LR + (int64_t)rb * kWJ;
          dst = B + kWRT + a * kWR;
          bytes = kWR * 8;
        } else {
          src = pt.col + ((int64_t)(i - 1) * pt.LC + (int64_t)kt * kWK) * 2;
          dst = B + kWCT;
          bytes = (kWK + 4) * 16;
        }
        bulk_load(dst, src, bytes, &full[b]);
      }
    }
    if (BULKST && ok) {
      // Y_{k+1} of the last tile of each buffer, once the consumers are done
      for (int nn = max(0, n - kWNB); nn < n; ++nn) {
        const int bb = nn % kWNB;
        if (!mbar_wait_bounded(&empty[bb], (uint32_t)((nn / kWNB) & 1), 1u << 22)) {
          ok = false;
          break;
        }
        store_prev_k1(blockIdx.x + nn * (int)gridDim.x, wsm + bb * kWBuf);
      }
    }
    if (BULKST) bulk_wait_all();
    if (!ok && lane == 0) atomicExch(pa.err, 1);
    // every issued copy lands before this warp exits (tiles 0..n-1 were issued)
    for (int b = 0; b < kWNB; ++b) {
      int last = n - 1;
      while (last >= 0 && last % kWNB != b) --last;
      if (last >= 0) mbar_wait_bounded(&full[b], (uint32_t)((last / kWNB) & 1), 1u << 22);
    }
    return;
  }

  // -------------------------------------------------------------- consumers
  const int lane = tid & 31, w = tid >> 5;
  const int h = tid >> 7;            // column half of the tile
  const int r2 = 1 + (tid & 127);    // stage-k shared row (rows 129, 130 by the last 20 threads)
  const int r3 = r2 + 1;             // stage-k+1 shared row
  StageCoef sa = pa.ca, sb = pa.cb;
  double *sYk = wsm + kWYk;          // column c of the tile at (c-1)*kWR
  int n = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++n) {
    const int b = n % kWNB, u = n / kWNB;
    const bool landed = mbar_wait_bounded(&full[b], (uint32_t)(u & 1), 1u << 22);
    if (BULKST && w == 0) bulk_wait_read();  // the previous tile's Y_k stores have read sYk
    // one vote: every consumer stops together; also orders the previous
    // tile's reads of sYk before this tile's writes
    if (cons_any(!landed)) {
      if (tid == 0) atomicExch(pa.err, 1);
      break;
    }
    double *Bw = wsm + b * kWBuf;
    const double *B = Bw;
    const double Dr = B[kWInfo], ax_n = B[kWInfo + 1], ax_s = B[kWInfo + 2];
    const int *Ii = reinterpret_cast<const int *>(B + kWInfo + 3);
    const int kt = Ii[0], rb = Ii[1], i = Ii[2];
    if (RAGGED) {
      const double *C = B + kWInfoCoef;
      sa = StageCoef{C[0], C[1], C[2], C[3], C[4]};
      sb = StageCoef{C[5], C[6], C[7], C[8], C[9]};
    }
    const int j0 = rb * kWJ + 1, k0 = kt * kWK + 2;
    const int nk = min(kWK, npm - 1 - k0 + 1);
    const int64_t pbase = (int64_t)(i - 1) * m.plane;
    const double *X1 = B + kWX1, *Y2 = B + kWY2, *U = B + kWU, *D = B + kWD, *RT = B + kWRT;
    const double2 *CT = reinterpret_cast<const double2 *>(B + kWCT);
    const int64_t seam = (int64_t)(npm - 2) * ld;
    const bool bulk = BULKST && nk == kWK && j0 + kWJ - 1 <= ntm;

    // ---------------------------------------------- stage k: Y_k into sYk
    if (ROWPAIRS && nk == kWK) {
      // thread: theta-row pair (r0, r0+1), r0 = 2(tid % 64), and a group of
      // columns 1-3, 4-6, 7-8 or 9-10; the pairs of rows 128-131 are units of
      // their own for 20 threads of the two-column groups
      auto rowf = [&](int r0, double2 &st2, double2 &c22, double2 &c42) {
        st2 = *reinterpret_cast<const double2 *>(RT + r0);
        c22 = *reinterpret_cast<const double2 *>(RT + kWR + r0);
        c42 = *reinterpret_cast<const double2 *>(RT + 2 * kWR + r0);
      };
      auto unit = [&](int r0, int c, double2 xl, double2 xc, double2 xr, double2 st2, double2 c22,
                      double2 c42) -> double2 {
        const int ja = j0 - 2 + r0, jb = ja + 1;
        const double up = X1[c * kWR + r0 - 1], dn = X1[c * kWR + r0 + 2];
        const double2 o2 = *reinterpret_cast<const double2 *>(Y2 + (c - 1) * kWR + r0);
        const double2 u = *reinterpret_cast<const double2 *>(U + (c - 1) * kWR + r0);
        const double2 d = *reinterpret_cast<const double2 *>(D + (c - 1) * kWR + r0);
        const double2 y = pair_rows_step(xl, xc, xr, up, dn, st2, c22, c42, CT[c],
                                         ja == 1 || ja == ntm, jb == 1 || jb == ntm, ja == 1 ? ax_n : ax_s,
                                         jb == 1 ? ax_n : ax_s, o2, u, d, sa);
        return y;
      };
      auto put = [&](int r0, int c, double2 y) {
        *reinterpret_cast<double2 *>(sYk + (c - 1) * kWR + r0) = y;
        if (!bulk && c >= 2 && c <= kWK + 1 && r0 >= 2 && r0 <= kWJ) {
          const int ja = j0 - 2 + r0, k = k0 - 2 + c;
          const bool va = (ja >= 1 && ja <= ntm), vb = (ja + 1 >= 1 && ja + 1 <= ntm);
          const int64_t so = (k == 2) ? seam : ((k == npm - 1) ? -seam : 0);
          store_pair(out_k + pbase + (int64_t)(k - 1) * ld + (ja - 1), y, va, vb, so);
        }
      };
      const int g = tid >> 6, r0 = 2 * (tid & 63);
      const int cb = (g == 0) ? 1 : ((g == 1) ? 4 : ((g == 2) ? 7 : 9));
      const int nc = (g < 2) ? 3 : 2;
      double2 st2, c22, c42;
      rowf(r0, st2, c22, c42);
      double2 xl = *reinterpret_cast<const double2 *>(X1 + (cb - 1) * kWR + r0);
      double2 xc = *reinterpret_cast<const double2 *>(X1 + cb * kWR + r0);
      double2 y[3];
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        if (s < nc) {
          const double2 xr = *reinterpret_cast<const double2 *>(X1 + (cb + s + 1) * kWR + r0);
          y[s] = unit(r0, cb + s, xl, xc, xr, st2, c22, c42);
          xl = xc;
          xc = xr;
        }
      }
#pragma unroll
      for (int s = 0; s < 3; ++s)
        if (s < nc) put(r0, cb + s, y[s]);
      const int e = tid - 2 * 64;  // units of the pairs at rows 128 and 130
      if (e >= 0 && e < 2 * (kWK + 2)) {
        const int rr = kWJ + 2 * (e & 1), c = 1 + (e >> 1);
        const double2 a = *reinterpret_cast<const double2 *>(X1 + (c - 1) * kWR + rr);
        const double2 b = *reinterpret_cast<const double2 *>(X1 + c * kWR + rr);
        const double2 z = *reinterpret_cast<const double2 *>(X1 + (c + 1) * kWR + rr);
        double2 sx, cx2, cx4;
        rowf(rr, sx, cx2, cx4);
        put(rr, c, unit(rr, c, a, b, z, sx, cx2, cx4));
      }
    } else if (nk == kWK) {
      {
        const int r = r2, j = j0 - 2 + r;
        const bool rowst = (j >= 1 && j <= ntm) && r >= 2;
        const bool pole = (j == 1 || j == ntm);
        const double axp = (j == 1) ? ax_n : ax_s;
        const double sti = RT[r], c2 = RT[kWR + r], c4 = RT[2 * kWR + r];
        const int cb = 1 + 5 * h;  // columns cb..cb+4
        const double *x = X1 + cb * kWR + r;
        const double *y2 = Y2 + (cb - 1) * kWR + r, *uu = U + (cb - 1) * kWR + r, *dd = D + (cb - 1) * kWR + r;
        double *yk = sYk + (cb - 1) * kWR + r;
        const double2 *ct = CT + cb;
        double *g = out_k + pbase + (int64_t)(k0 - 3 + cb) * ld + (j - 1);
        // all five cells before any shared store, so that the five
        // arithmetic chains can overlap (a store to sYk would otherwise
        // order every later shared load after it)
        double y[5];
        double xl = x[-kWR], xc = x[0];
#pragma unroll
        for (int s = 0; s < 5; ++s) {
          const double xr = x[(s + 1) * kWR];
          const double up = x[s * kWR - 1], dn = x[s * kWR + 1];
          double ax;
          if (pole) {
            ax = axp;
          } else {
            const double2 P = ct[s];
            const double c1 = P.x * sti * sti;
            const double c5 = P.y * sti * sti;
            const double c3 = -(c1 + c2 + c4 + c5);
            ax = c1 * xl + c2 * up + c3 * xc + c4 * dn + c5 * xr;
          }
          y[s] = sa.a * xc + sa.b * y2[s * kWR] + sa.c * uu[s * kWR] + sa.d * ax + sa.e * dd[s * kWR];
          xl = xc;
          xc = xr;
        }
#pragma unroll
        for (int s = 0; s < 5; ++s) {
          const int c = cb + s;
          yk[s * kWR] = y[s];
          if (rowst && c >= 2 && c <= kWK + 1) {
            double *gq = g + (int64_t)s * ld;
            *gq = y[s];
            const int k = k0 - 2 + c;
            if (k == 2) gq[seam] = y[s];
            if (k == npm - 1) gq[-seam] = y[s];
          }
        }
      }
      if (tid >= kWCons - 2 * (kWK + 2)) {  // shared rows kWJ+1, kWJ+2 (one cell each)
        const int e = tid - (kWCons - 2 * (kWK + 2));
        const int r = kWJ + 1 + (e & 1), c = 1 + (e >> 1);
        const int j = j0 - 2 + r;
        if (j >= 1 && j <= ntm) {
          double ax;
          if (j == 1) {
            ax = ax_n;
          } else if (j == ntm) {
            ax = ax_s;
          } else {
            const double sti = RT[r], c2 = RT[kWR + r], c4 = RT[2 * kWR + r];
            const double2 P = CT[c];
            const double c1 = P.x * sti * sti;
            const double c5 = P.y * sti * sti;
            const double c3 = -(c1 + c2 + c4 + c5);
            ax = c1 * X1[(c - 1) * kWR + r] + c2 * X1[c * kWR + r - 1] + c3 * X1[c * kWR + r] +
                 c4 * X1[c * kWR + r + 1] + c5 * X1[(c + 1) * kWR + r];
          }
          const double y = sa.a * X1[c * kWR + r] + sa.b * Y2[(c - 1) * kWR + r] + sa.c * U[(c - 1) * kWR + r] +
                           sa.d * ax + sa.e * D[(c - 1) * kWR + r];
          sYk[(c - 1) * kWR + r] = y;
          if (r == kWJ + 1 && c >= 2 && c <= kWK + 1) {
            const int k = k0 - 2 + c;
            double *gq = out_k + pbase + (int64_t)(k - 1) * ld + (j - 1);
            *gq = y;
            if (k == 2) gq[seam] = y;
            if (k == npm - 1) gq[-seam] = y;
          }
        }
      }
    } else {
      const int nr2 = kWJ + 2, nc2 = nk + 2;
      for (int e = tid; e < nr2 * nc2; e += kWCons) {
        const int r = 1 + e % nr2, c = 1 + e / nr2;
        const int j = j0 - 2 + r;
        if (j < 1 || j > ntm) continue;
        double ax;
        if (j == 1) {
          ax = ax_n;
        } else if (j == ntm) {
          ax = ax_s;
        } else {
          const double sti = RT[r], c2 = RT[kWR + r], c4 = RT[2 * kWR + r];
          const double2 P = CT[c];
          const double c1 = P.x * sti * sti;
          const double c5 = P.y * sti * sti;
          const double c3 = -(c1 + c2 + c4 + c5);
          ax = c1 * X1[(c - 1) * kWR + r] + c2 * X1[c * kWR + r - 1] + c3 * X1[c * kWR + r] +
               c4 * X1[c * kWR + r + 1] + c5 * X1[(c + 1) * kWR + r];
        }
        const double y = sa.a * X1[c * kWR + r] + sa.b * Y2[(c - 1) * kWR + r] + sa.c * U[(c - 1) * kWR + r] +
                         sa.d * ax + sa.e * D[(c - 1) * kWR + r];
        sYk[(c - 1) * kWR + r] = y;
        if (r >= 2 && r < 2 + kWJ && c >= 2 && c < 2 + nk) {
          const int k = k0 - 2 + c;
          double *gq = out_k + pbase + (int64_t)(k - 1) * ld + (j - 1);
          *gq = y;
          if (k == 2) gq[seam] = y;
          if (k == npm - 1) gq[-seam] = y;
        }
      }
    }
    if (bulk) fence_proxy_async_smem();  // sYk, as written, for the bulk stores
    cons_sync();
    if (bulk && w == 0)  // Y_k rows j0..j0+kWJ-1 are shared rows 2..kWJ+1
      ws_store_cols(out_k, pbase, k0, j0, sYk + kWR + 2, lane, npm, ld);

    // ---- ring partials of Y_k over this tile's columns (fixed tree over columns)
    const bool has_n = (j0 == 1);
    const bool has_s = (ntm - 1 >= j0 && ntm - 1 <= j0 + kWJ - 1);
    if ((w == 0 && has_n) || (w == 1 && has_s)) {
      const int ra = (w == 0) ? 3 : ntm - (j0 - 2);  // (row 2 - row 1) or (row ntm - row ntm-1)
      double v = 0.0;
      if (lane < nk) {
        const int c = 2 + lane;
        v = (Dr + Dr) * (sYk[(c - 1) * kWR + ra] - sYk[(c - 1) * kWR + ra - 1]) * m.dp[k0 - 2 + c];
      }
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if (lane == 0) ro.part[((int64_t)w * m.nr + (i - 1)) * ro.nkb + kt] = v;
    }

    // -------------------------------------- stage k+1: Y_{k+1} to HBM
    if (ROWPAIRS && nk == kWK) {
      // thread: theta-row pair (r0, r0+1), r0 = 2 + 2(tid % 64), columns
      // 2 + 2(tid / 64) and the next one
      const int r0 = 2 + 2 * (tid & 63), cb = 2 + 2 * (tid >> 6);
      const int ja = j0 - 2 + r0;
      const double2 st2 = *reinterpret_cast<const double2 *>(RT + r0);
      const double2 c22 = *reinterpret_cast<const double2 *>(RT + kWR + r0);
      const double2 c42 = *reinterpret_cast<const double2 *>(RT + 2 * kWR + r0);
      const bool va = (ja >= 2 && ja <= ntm - 1), vb = (ja + 1 >= 2 && ja + 1 <= ntm - 1);
      double2 xl = *reinterpret_cast<const double2 *>(sYk + (cb - 2) * kWR + r0);
      double2 xc = *reinterpret_cast<const double2 *>(sYk + (cb - 1) * kWR + r0);
      double2 y[2];
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        const int c = cb + s;
        const double2 xr = *reinterpret_cast<const double2 *>(sYk + c * kWR + r0);
        const double up = sYk[(c - 1) * kWR + r0 - 1], dn = sYk[(c - 1) * kWR + r0 + 2];
        const double2 o2 = *reinterpret_cast<const double2 *>(X1 + c * kWR + r0);
        const double2 u = *reinterpret_cast<const double2 *>(U + (c - 1) * kWR + r0);
        const double2 d = *reinterpret_cast<const double2 *>(D + (c - 1) * kWR + r0);
        y[s] = pair_rows_step(xl, xc, xr, up, dn, st2, c22, c42, CT[c], false, false, 0.0, 0.0, o2,
                              u, d, sb);
        xl = xc;
        xc = xr;
      }
      if (bulk) {
        // staged in the Y_{k-2} region (column c at (c-2)*kWR, row j at
        // j-j0) for the producer's bulk stores; fenced before the release
#pragma unroll
        for (int s = 0; s < 2; ++s)
          *reinterpret_cast<double2 *>(Bw + kWY2 + (cb + s - 2) * kWR + (r0 - 2)) = y[s];
        fence_proxy_async_smem();
      } else {
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          const int k = k0 - 2 + cb + s;
          const int64_t so = (k == 2) ? seam : ((k == npm - 1) ? -seam : 0);
          store_pair(out_k1 + pbase + (int64_t)(k - 1) * ld + (ja - 1), y[s], va, vb, so);
        }
      }
    } else if (nk == kWK) {
      const int r = r3, j = j0 - 2 + r;
      const bool rowok = (j >= 2 && j <= ntm - 1);
      const double sti = RT[r], c2 = RT[kWR + r], c4 = RT[2 * kWR + r];
      const int cb = 2 + 4 * h;  // columns cb..cb+3
      const double *yk = sYk + (cb - 1) * kWR + r;
      const double *x1 = X1 + cb * kWR + r, *uu = U + (cb - 1) * kWR + r, *dd = D + (cb - 1) * kWR + r;
      const double2 *ct = CT + cb;
      double *g = out_k1 + pbase + (int64_t)(k0 - 3 + cb) * ld + (j - 1);
      double xl = yk[-kWR], xc = yk[0];
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const int c = cb + s;
        const double xr = yk[(s + 1) * kWR];
        const double up = yk[s * kWR - 1], dn = yk[s * kWR + 1];
        const double2 P = ct[s];
        const double c1 = P.x * sti * sti;
        const double c5 = P.y * sti * sti;
        const double c3 = -(c1 + c2 + c4 + c5);
        const double ax = c1 * xl + c2 * up + c3 * xc + c4 * dn + c5 * xr;
        const double y = sb.a * xc + sb.b * x1[s * kWR] + sb.c * uu[s * kWR] + sb.d * ax + sb.e * dd[s * kWR];
        if (rowok) {
          double *gq = g + (int64_t)s * ld;
          *gq = y;
          const int k = k0 - 2 + c;
          if (k == 2) gq[seam] = y;
          if (k == npm - 1) gq[-seam] = y;
        }
        xl = xc;
        xc = xr;
      }
    } else {
      for (int e = tid; e < kWJ * nk; e += kWCons) {
        const int r = 2 + e % kWJ, c = 2 + e / kWJ;
        const int j = j0 - 2 + r;
        if (j < 2 || j > ntm - 1) continue;
        const double sti = RT[r], c2 = RT[kWR + r], c4 = RT[2 * kWR + r];
        const double2 P = CT[c];
        const double c1 = P.x * sti * sti;
        const double c5 = P.y * sti * sti;
        const double c3 = -(c1 + c2 + c4 + c5);
        const double ax = c1 * sYk[(c - 2) * kWR + r] + c2 * sYk[(c - 1) * kWR + r - 1] +
                          c3 * sYk[(c - 1) * kWR + r] + c4 * sYk[(c - 1) * kWR + r + 1] + c5 * sYk[c * kWR + r];
        const double y = sb.a * sYk[(c - 1) * kWR + r] + sb.b * X1[c * kWR + r] + sb.c * U[(c - 1) * kWR + r] +
                         sb.d * ax + sb.e * D[(c - 1) * kWR + r];
        const int k = k0 - 2 + c;
        double *gq = out_k1 + pbase + (int64_t)(k - 1) * ld + (j - 1);
        *gq = y;
        if (k == 2) gq[seam] = y;
        if (k == npm - 1) gq[-seam] = y;
      }
    }
    mbar_arrive(&empty[b]);  // this thread is done with buffer b
  }
  if (BULKST && w == 0) bulk_wait_all();  // this warp's Y_k stores, before the CTA exits
}

// Pole rows of Y_{k+1} and the ring sums of Y_{k+1}, after
// k_sts_pair_ws<false>.  Grid (realization, chunk of kPoleThreads phi
// columns); in a ragged batch grid x walks pa.rlist and the coefficients are
// the realization's own (pa.rc).  Every block sums the ring partials of Y_k that the pole tiles
// wrote (tile order, the same fixed tree in every block), computes the pole
// rows of Y_{k+1} for its columns by stage k+1's combine (src/hipft.f90:
// 5224-5235) with Y_k at the poles recomputed from the inputs, and writes its
// chunk's share of the ring sums of Y_{k+1} (src/hipft.f90:7969-7979); the
// last block of a realization (atomic counter, no waiting) adds the chunks in
// order and leaves the ring sums for the next launch.
constexpr int kPoleThreads = 256;
struct PoleScratch {
  double *part;          // [nr][nch][2] chunk shares of the ring sums
  unsigned int *count;   // [nr] blocks done, reset by the last one
};
__global__ void __launch_bounds__(kPoleThreads) k_pair_poles(Mesh m, const double *__restrict__ dfac,
                                                            const double *__restrict__ ykm1,
                                                            const double *__restrict__ ykm2,
                                                            const double *__restrict__ u0,
                                                            const double *__restrict__ dty0, double *out_k1,
                                                            const double *__restrict__ ring_in, double bcn,
                                                            double bcs, PairArgs pa, RingOut ro, PoleScratch ps) {
  __shared__ double sh[2 * (kPoleThreads / 32)];
  __shared__ double s_ring[2];
  __shared__ int s_last;
  // the next pair's kernel may launch now; its tiles at the poles wait for
  // this grid to finish (griddepcontrol.wait)
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  const int tid = threadIdx.x, ch = blockIdx.y, nch = gridDim.y;
  const StageCoef *rcp = pa.rc;
  if (pa.dctr) {  // graph-run step: the grid covers every realization
    const int pq = *pa.dctr + pa.doff;
    if ((int)blockIdx.x >= pa.dnact[pq]) return;
    rcp = pa.rc + (int64_t)pq * pa.dstride;
  }
  const int i = (pa.rlist ? pa.rlist[blockIdx.x] : (int)blockIdx.x) + 1;
  const int ntm = m.ntm, npm = m.npm;
  const int64_t ld = m.ldt, pbase = (int64_t)(i - 1) * m.plane;
  const StageCoef sa = rcp ? rcp[2 * (i - 1)] : pa.ca, sb = rcp ? rcp[2 * (i - 1) + 1] : pa.cb;
  const double Dr = dfac[i];
  const double ax_n = ring_in[2 * (i - 1)] * bcn;
  const double ax_s = -ring_in[2 * (i - 1) + 1] * bcs;
  // this block's column: its inputs are loaded before the ring reduction
  const int k = 1 + ch * kPoleThreads + tid;
  const bool kin = (k <= npm);
  const int64_t qn = pbase + (int64_t)(kin ? k - 1 : 0) * ld;  // row 1
  const int64_t qs = qn + (ntm - 1);                           // row ntm
  double a1n = 0, a2n = 0, aun = 0, adn = 0, a1s = 0, a2s = 0, aus = 0, ads = 0, y2 = 0, ym = 0, dpk = 0;
  if (kin) {
    a1n = ykm1[qn]; a2n = ykm2[qn]; aun = u0[qn]; adn = dty0[qn];
    a1s = ykm1[qs]; a2s = ykm2[qs]; aus = u0[qs]; ads = dty0[qs];
    y2 = out_k1[qn + 1];
    ym = out_k1[qs - 1];
    dpk = m.dp[k];
  }
  double sn = 0.0, ss = 0.0;
  for (int q = tid; q < ro.nkb; q += kPoleThreads) {
    sn = sn + ro.part[((int64_t)0 * m.nr + (i - 1)) * ro.nkb + q];
    ss = ss + ro.part[((int64_t)1 * m.nr + (i - 1)) * ro.nkb + q];
  }
  block_sum2(sn, ss, sh);
  if (tid == 0) {
    s_ring[0] = sn;
    s_ring[1] = ss;
  }
  __syncthreads();
  const double axn1 = s_ring[0] * bcn, axs1 = -s_ring[1] * bcs;
  double rn = 0.0, rsum = 0.0;
  if (kin) {
    const double ykn = sa.a * a1n + sa.b * a2n + sa.c * aun + sa.d * ax_n + sa.e * adn;
    const double yks = sa.a * a1s + sa.b * a2s + sa.c * aus + sa.d * ax_s + sa.e * ads;
    const double yn = sb.a * ykn + sb.b * a1n + sb.c * aun + sb.d * axn1 + sb.e * adn;
    const double ys = sb.a * yks + sb.b * a1s + sb.c * aus + sb.d * axs1 + sb.e * ads;
    out_k1[qn] = yn;
    out_k1[qs] = ys;
    if (k >= 2 && k <= npm - 1) {
      rn = (Dr + Dr) * (y2 - yn) * dpk;
      rsum = (Dr + Dr) * (ys - ym) * dpk;
    }
  }
  block_sum2(rn, rsum, sh);
  if (tid == 0) {
    double *pp = ps.part + ((int64_t)(i - 1) * nch + ch) * 2;
    pp[0] = rn;
    pp[1] = rsum;
    __threadfence();
    const unsigned int old = atomicAdd(&ps.count[i - 1], 1u);
    s_last = (old == (unsigned)nch - 1u) ? 1 : 0;
  }
  __syncthreads();
  if (!s_last) return;
  if (tid == 0) {
    __threadfence();
    double tn = 0.0, ts = 0.0;
    for (int c = 0; c < nch; ++c) {
      tn = tn + __ldcg(&ps.part[((int64_t)(i - 1) * nch + c) * 2]);
      ts = ts + __ldcg(&ps.part[((int64_t)(i - 1) * nch + c) * 2 + 1]);
    }
    ro.ring[2 * (i - 1)] = tn;
    ro.ring[2 * (i - 1) + 1] = ts;
    ps.count[i - 1] = 0u;
  }
}

}  // namespace hipft
