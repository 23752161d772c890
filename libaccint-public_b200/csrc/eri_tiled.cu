// Warp-per-quartet Rys ERI kernel with the lanes spread over the quartet's output
// integrals -- the path for the classes too large for the register-resident
// kernels (f and g shells, (dd|..) blocks).
//
// Per quartet (one warp), for every primitive quartet and batch of Rys roots:
//   1. table phase: lane t < 3*rb owns (root r = t/3, direction x = t%3); it builds
//      the 2D integrals V[e][f] (e <= la+lb, f <= lc+ld) by the vertical recurrence
//      of eri_device.cuh, then the transferred table H[a][b][c][d] by the
//      horizontal recurrence I(a, b+1) = I(a+1, b) + AB I(a, b) on the bra and the
//      same on the ket (eri_kernel.cpp:143-163), per direction, all in shared
//      memory;
//   2. output phase: lane l owns outputs j = l + 32 m of the current pass and adds
//      sum_r Hx[r][..] Hy[r][..] Hz[r][..] to them (w pref folded into z), with the
//      three table offsets of each output precomputed once per pass.
// Outputs stay in registers over the primitive and root loops; after the last
// primitive they are normalized and digested: the six Fock blocks of the 8-fold
// scatter (J'_ab, J'_cd, K'_ac, K'_ad, K'_bc, K'_bd) are summed per warp in shared
// memory and added to global J'/K' with one atomic per element.  Classes with more
// outputs than 32 x kOut run several passes, each repeating the table phase.
// The reference counterparts are eri_kernel<La,Lb,Lc,Ld> (thread per quartet,
// src/device/cuda/kernels/eri_kernel.cu:227-461) and eri_warp_kernel_runtime
// (warp per quartet, eri_kernel_warp.cu:140-344) followed by the separate
// fock_accumulate_batch_kernel; here no integral reaches global memory.
#include <cuda_runtime.h>

#include <algorithm>

#include "eri_device.cuh"
#include "eri_kernels.h"

namespace lai {

namespace {

constexpr int kOut = 16;     // outputs per lane per pass
constexpr int kWarps = 4;    // warps per block

struct TiledGeom {
  int la, lb, lc, ld;
  int na, nb, nc, nd, nout;
  int LAB, LCD;
  int EA, EB, EC, ED;        // la+1, lb+1, lc+1, ld+1
  int n;                     // roots
  int rb;                    // roots per batch (3*rb <= 32 table lanes)
  int vsz, xsz, hsz;         // (LAB+1)(LCD+1), EA*EB*(LCD+1), EA*EB*EC*ED
  int npass;
  // per-warp shared memory (doubles)
  int off_v, off_x, off_h, off_d, off_acc, off_o, per_warp;
  int nDab, nDcd, nDac, nDad, nDbc, nDbd, nacc;
};

TiledGeom make_tiled_geom(int la, int lb, int lc, int ld, size_t smem_per_warp_max) {
  TiledGeom g{};
  g.la = la; g.lb = lb; g.lc = lc; g.ld = ld;
  g.na = ncart(la); g.nb = ncart(lb); g.nc = ncart(lc); g.nd = ncart(ld);
  g.nout = g.na * g.nb * g.nc * g.nd;
  g.LAB = la + lb; g.LCD = lc + ld;
  g.EA = la + 1; g.EB = lb + 1; g.EC = lc + 1; g.ED = ld + 1;
  g.n = (la + lb + lc + ld) / 2 + 1;
  g.vsz = (g.LAB + 1) * (g.LCD + 1);
  g.xsz = g.EA * g.EB * (g.LCD + 1);
  g.hsz = g.EA * g.EB * g.EC * g.ED;
  g.npass = (g.nout + 32 * kOut - 1) / (32 * kOut);
  g.nDab = g.na * g.nb; g.nDcd = g.nc * g.nd; g.nDac = g.na * g.nc;
  g.nDad = g.na * g.nd; g.nDbc = g.nb * g.nc; g.nDbd = g.nb * g.nd;
  g.nacc = g.nDab + g.nDcd + g.nDac + g.nDad + g.nDbc + g.nDbd;
  for (int rb = std::min(g.n, 10); rb >= 1; --rb) {
    g.rb = rb;
    int o = 0;
    g.off_v = o; o += 3 * rb * g.vsz;
    g.off_x = o; o += 3 * rb * g.xsz;
    g.off_h = o; o += 3 * rb * g.hsz;
    g.off_d = o; o += g.nacc;
    g.off_acc = o; o += g.nacc;
    g.off_o = o; o += 32 * kOut;
    g.per_warp = (o + 1) & ~1;
    if ((size_t)g.per_warp * 8 <= smem_per_warp_max) return g;
  }
  g.per_warp = -1;
  return g;
}

__global__ void __launch_bounds__(kWarps * 32) eri_tiled_kernel(QuartetBlock blk, JKArgs args,
                                                                RysTablesView tab, TiledGeom g) {
  extern __shared__ __align__(16) double smem_t[];
  // class tables: Cartesian components and normalization factors of the four shells
  __shared__ int s_comp[4][kNCartMax];
  __shared__ double s_norm[4][kNCartMax];
  for (int i = threadIdx.x; i < 4 * kNCartMax; i += blockDim.x) {
    const int sh = i / kNCartMax, k = i - sh * kNCartMax;
    const int l = sh == 0 ? g.la : sh == 1 ? g.lb : sh == 2 ? g.lc : g.ld;
    if (k < ncart(l)) {
      s_comp[sh][k] = cart_comp(l, k);
      s_norm[sh][k] = norm_factor(l, k);
    }
  }
  // output tables of a one-pass class (output j -> packed table offsets and packed
  // a|b|c|d), built once per block: the integer divisions stay out of the loops
  __shared__ int s_off[32 * kOut];
  __shared__ int s_idx[32 * kOut];
  const bool one_pass = g.npass == 1;
  const int ncd0 = ncart(g.lc) * ncart(g.ld), nbcd0 = ncart(g.lb) * ncd0;
  auto out_off = [&](int j, int& off, int& idx) {
    const int a = j / nbcd0, b = (j / ncd0) % g.nb, c = (j / g.nd) % g.nc, d = j % g.nd;
    const int ca = s_comp[0][a], cb = s_comp[1][b], cc = s_comp[2][c], cd = s_comp[3][d];
    const int ox = ((comp_x(ca) * g.EB + comp_x(cb)) * g.EC + comp_x(cc)) * g.ED + comp_x(cd);
    const int oy = ((comp_y(ca) * g.EB + comp_y(cb)) * g.EC + comp_y(cc)) * g.ED + comp_y(cd);
    const int oz = ((comp_z(ca) * g.EB + comp_z(cb)) * g.EC + comp_z(cc)) * g.ED + comp_z(cd);
    off = ox | (oy << 10) | (oz << 20);
    idx = a | (b << 8) | (c << 16) | (d << 24);
  };
  if (one_pass) {
    __syncthreads();
    for (int j = threadIdx.x; j < g.nout; j += blockDim.x) out_off(j, s_off[j], s_idx[j]);
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  double* ws = smem_t + (size_t)warp * g.per_warp;
  double* Vt = ws + g.off_v;   // [rb][3][vsz]
  double* Xt = ws + g.off_x;   // [rb][3][xsz]
  double* Ht = ws + g.off_h;   // [rb][3][hsz]
  double* Ds = ws + g.off_d;   // D_ab, D_cd, D_ac, D_ad, D_bc, D_bd
  double* Acc = ws + g.off_acc;  // J'_ab, J'_cd, K'_ac, K'_ad, K'_bc, K'_bd (same layout)
  double* Ob = ws + g.off_o;     // this pass's normalized outputs
  const int oDab = 0, oDcd = g.nDab, oDac = oDcd + g.nDcd, oDad = oDac + g.nDac, oDbc = oDad + g.nDad,
            oDbd = oDbc + g.nDbc;

  const int nbra = blk.bra.npairs, nket = blk.ket.npairs;
  const int Kab = blk.bra.Ka * blk.bra.Kb, Kcd = blk.ket.Ka * blk.ket.Kb;
  (void)nbra; (void)nket;
  const int W = g.LCD + 1;
  const int ncd = g.nc * g.nd, nbcd = g.nb * ncd;
  // one quartet's geometry, set per quartet below and read by the phases
  double AB[3] = {0.0, 0.0, 0.0}, CD[3] = {0.0, 0.0, 0.0};
  // primitive-quartet quantities
  struct PrimQ {
    double hz, he, inv, rz, re, T, pref;
    double PA[3], QC[3], PQ[3];
  };
  // pb, pk: the bra and ket primitive pairs' per-pair records (BraRecField); the
  // whole warp reads the same record, a few contiguous lines
  auto prim_quartet = [&](const double* pb, const double* pk, PrimQ& o) {
    const double zeta = __ldg(pb + BR_ZETA);
    o.hz = __ldg(pb + BR_HZ);
    const double P[3] = {__ldg(pb + BR_PX), __ldg(pb + BR_PY), __ldg(pb + BR_PZ)};
    o.PA[0] = __ldg(pb + BR_PAX); o.PA[1] = __ldg(pb + BR_PAY); o.PA[2] = __ldg(pb + BR_PAZ);
    const double cab = __ldg(pb + BR_C);
    const double eta = __ldg(pk + BR_ZETA);
    o.he = __ldg(pk + BR_HZ);
    o.QC[0] = __ldg(pk + BR_PAX); o.QC[1] = __ldg(pk + BR_PAY); o.QC[2] = __ldg(pk + BR_PAZ);
    o.PQ[0] = P[0] - __ldg(pk + BR_PX);
    o.PQ[1] = P[1] - __ldg(pk + BR_PY);
    o.PQ[2] = P[2] - __ldg(pk + BR_PZ);
    const double ccd = __ldg(pk + BR_C);
    const double rs = rsqrt(zeta + eta);
    o.inv = rs * rs;
    o.rz = eta * o.inv;
    o.re = zeta * o.inv;
    o.T = zeta * o.rz * (o.PQ[0] * o.PQ[0] + o.PQ[1] * o.PQ[1] + o.PQ[2] * o.PQ[2]);
    o.pref = cab * ccd * rs;
  };
  // table phase: lane t < 3*nr owns (root r0 + t/3, direction t%3); builds V by the
  // vertical recurrence, then in place the bra transfer into X and the ket
  // transfer into H
  auto table_phase = [&](int r0, int nr, const PrimQ& o) {
    if (lane >= 3 * nr) return;
    const int rr = lane / 3, x = lane - 3 * rr;
    double u, w;
    rys_root_one<double>(g.n, r0 + rr, o.T, tab, u, w);
    double* V = Vt + (rr * 3 + x) * g.vsz;
    const double b00 = 0.5 * o.inv * u, b10 = o.hz - o.hz * o.rz * u, b01 = o.he - o.he * o.re * u;
    // direction-x components (selects, not runtime-indexed arrays, which would
    // live in local memory)
    const double pqx = x == 0 ? o.PQ[0] : x == 1 ? o.PQ[1] : o.PQ[2];
    const double pax = x == 0 ? o.PA[0] : x == 1 ? o.PA[1] : o.PA[2];
    const double qcx = x == 0 ? o.QC[0] : x == 1 ? o.QC[1] : o.QC[2];
    const double pa = pax - o.rz * u * pqx;
    const double qc = qcx + o.re * u * pqx;
    V[0] = (x == 2) ? w * o.pref : 1.0;
    if (g.LAB > 0) V[W] = pa * V[0];
    for (int e = 1; e < g.LAB; ++e) V[(e + 1) * W] = pa * V[e * W] + e * b10 * V[(e - 1) * W];
    for (int f = 0; f < g.LCD; ++f)
      for (int e = 0; e <= g.LAB; ++e) {
        double v = qc * V[e * W + f];
        if (f) v += f * b01 * V[e * W + f - 1];
        if (e) v += e * b00 * V[(e - 1) * W + f];
        V[e * W + f + 1] = v;
      }
    // horizontal transfer, in place: bra levels b = 0..lb of each column f of V
    // (I(a, b+1) = I(a+1, b) + AB I(a, b)) into X[a][b][f], then ket levels of
    // each X[a][b][.] into H[a][b][c][d]
    double* X = Xt + (rr * 3 + x) * g.xsz;
    double* H = Ht + (rr * 3 + x) * g.hsz;
    const double ab = x == 0 ? AB[0] : x == 1 ? AB[1] : AB[2];
    const double cdv = x == 0 ? CD[0] : x == 1 ? CD[1] : CD[2];
    for (int f = 0; f <= g.LCD; ++f) {
      for (int a = 0; a < g.EA; ++a) X[(a * g.EB) * W + f] = V[a * W + f];
      for (int b = 1; b < g.EB; ++b) {
        for (int a = 0; a + b <= g.LAB; ++a) V[a * W + f] = V[(a + 1) * W + f] + ab * V[a * W + f];
        for (int a = 0; a < g.EA; ++a) X[(a * g.EB + b) * W + f] = V[a * W + f];
      }
    }
    for (int a = 0; a < g.EA; ++a)
      for (int b = 0; b < g.EB; ++b) {
        double* col = X + (a * g.EB + b) * W;
        double* h = H + (a * g.EB + b) * g.EC * g.ED;
        for (int c = 0; c < g.EC; ++c) h[c * g.ED] = col[c];
        for (int d = 1; d < g.ED; ++d) {
          for (int c = 0; c + d <= g.LCD; ++c) col[c] = col[c + 1] + cdv * col[c];
          for (int c = 0; c < g.EC; ++c) h[c * g.ED + d] = col[c];
        }
      }
  };
  // output phase: acc[m] += sum over the batch's roots of Hx Hy Hz at the lane's
  // output offsets
  auto output_phase = [&](int nr, const int (&off)[kOut], double (&acc)[kOut]) {
    for (int rr = 0; rr < nr; ++rr) {
      const double* Hx = Ht + (rr * 3 + 0) * g.hsz;
      const double* Hy = Ht + (rr * 3 + 1) * g.hsz;
      const double* Hz = Ht + (rr * 3 + 2) * g.hsz;
#pragma unroll
      for (int m = 0; m < kOut; ++m) {
        const int o = off[m];
        if (o >= 0) acc[m] += Hx[o & 1023] * Hy[(o >> 10) & 1023] * Hz[o >> 20];
      }
    }
  };

  const int64_t gw = (int64_t)blockIdx.x * kWarps + warp;
  const int64_t nw = (int64_t)gridDim.x * kWarps;
  const int64_t nq_all = blk.total - blk.t_begin;
  const int64_t per = (nq_all + nw - 1) / nw;
  const int64_t tbeg = blk.t_begin + gw * per;
  const int64_t tend = min(blk.total, tbeg + per);
  // a single primitive quartet per quartet and all roots in one batch: the tables
  // are built once and serve every output pass
  const bool single = Kab * Kcd == 1 && g.rb >= g.n && g.npass > 1;
  int p = -1;
  for (int64_t t = tbeg; t < tend; ++t) {
    if (p < 0) {
      if (lane == 0) p = find_bra(blk.offsets, nbra, t);
      p = __shfl_sync(0xffffffffu, p, 0);
    } else {
      while (t >= __ldg(blk.offsets + p + 1)) ++p;
    }
    const int q = (blk.qbegin ? __ldg(blk.qbegin + p) : 0) + (int)(t - __ldg(blk.offsets + p));
    AB[0] = __ldg(blk.bra.AB + p); AB[1] = __ldg(blk.bra.AB + nbra + p); AB[2] = __ldg(blk.bra.AB + 2 * nbra + p);
    CD[0] = __ldg(blk.ket.AB + q); CD[1] = __ldg(blk.ket.AB + nket + q); CD[2] = __ldg(blk.ket.AB + 2 * nket + q);
    const int fa = __ldg(blk.bra.func_a + p), fb = __ldg(blk.bra.func_b + p);
    const int fc = __ldg(blk.ket.func_a + q), fd = __ldg(blk.ket.func_b + q);
    const double sym = args.mode == MODE_JK ? quartet_weight(blk, p, q) : 0.0;
    const SysMats mats = sys_mats(args, blk, p);
    if (args.mode == MODE_JK) {  // density sub-blocks of the six scatter targets
      const size_t n = (size_t)mats.nbf;
      const double* D = mats.D;
      for (int i = lane; i < g.nacc; i += 32) {
        int r0, r1, c0, c1, k;
        if (i < oDcd) { k = i; r0 = fa; c0 = fb; r1 = g.na; c1 = g.nb; }
        else if (i < oDac) { k = i - oDcd; r0 = fc; c0 = fd; r1 = g.nc; c1 = g.nd; }
        else if (i < oDad) { k = i - oDac; r0 = fa; c0 = fc; r1 = g.na; c1 = g.nc; }
        else if (i < oDbc) { k = i - oDad; r0 = fa; c0 = fd; r1 = g.na; c1 = g.nd; }
        else if (i < oDbd) { k = i - oDbc; r0 = fb; c0 = fc; r1 = g.nb; c1 = g.nc; }
        else { k = i - oDbd; r0 = fb; c0 = fd; r1 = g.nb; c1 = g.nd; }
        (void)r1;
        Ds[i] = __ldg(D + (size_t)(r0 + k / c1) * n + c0 + k % c1);
        Acc[i] = 0.0;
      }
    }
    double smax = 0.0;
    unsigned int nprim_done = 0;
    bool have_tables = false;

    for (int pass = 0; pass < g.npass; ++pass) {
      // packed table offsets of this lane's outputs (x | y << 10 | z << 20), -1 = none
      int off[kOut];
      double acc[kOut];
#pragma unroll
      for (int m = 0; m < kOut; ++m) {
        const int j = pass * 32 * kOut + lane + 32 * m;
        acc[m] = 0.0;
        off[m] = -1;
        if (j < g.nout) {
          if (one_pass) {
            off[m] = s_off[j];
          } else {
            int idx;
            out_off(j, off[m], idx);
          }
        }
      }

      if (single) {
        // one primitive quartet and one root batch: its tables, built in the first
        // pass, stay in shared memory for the later passes
        if (pass == 0) {
          const double* pb = blk.bra.primb + (size_t)p * Kab * kBraRec;
          const double* pk = blk.ket.primb + (size_t)q * Kcd * kBraRec;
          const double qab = __ldg(pb + BR_Q), qcd = __ldg(pk + BR_Q);
          have_tables = !(qab * qcd < args.prim_eps);
          if (have_tables) {
            ++nprim_done;
            PrimQ pq;
            prim_quartet(pb, pk, pq);
            table_phase(0, g.n, pq);
          }
          __syncwarp();
        }
        if (have_tables) output_phase(g.n, off, acc);
      } else {
        for (int ib = 0; ib < Kab; ++ib) {
          const double* pb = blk.bra.primb + ((size_t)p * Kab + ib) * kBraRec;
          const double qab = __ldg(pb + BR_Q);
          if (qab * blk.ket.qprim_max < args.prim_eps) break;
          for (int ik = 0; ik < Kcd; ++ik) {
            const double* pk = blk.ket.primb + ((size_t)q * Kcd + ik) * kBraRec;
            const double qcd = __ldg(pk + BR_Q);
            if (qab * qcd < args.prim_eps) break;
            if (pass == 0) ++nprim_done;
            PrimQ pq;
            prim_quartet(pb, pk, pq);
            for (int r0 = 0; r0 < g.n; r0 += g.rb) {
              const int nr = min(g.rb, g.n - r0);
              table_phase(r0, nr, pq);
              __syncwarp();
              output_phase(nr, off, acc);
              __syncwarp();
            }
          }
        }
      }

      // ---- normalization and consumption of this pass's outputs ----
      const int j0 = pass * 32 * kOut, j1 = min(g.nout, j0 + 32 * kOut);
#pragma unroll
      for (int m = 0; m < kOut; ++m) {
        const int j = j0 + lane + 32 * m;
        if (j >= j1) continue;
        int idx;
        if (one_pass) {
          idx = s_idx[j];
        } else {
          int o;
          out_off(j, o, idx);
        }
        const int a = idx & 255, b = (idx >> 8) & 255, c = (idx >> 16) & 255, d = idx >> 24;
        const double v = acc[m] * s_norm[0][a] * s_norm[1][b] * s_norm[2][c] * s_norm[3][d];
        if (args.mode == MODE_RAW) {
          args.raw_out[(size_t)(t - blk.t_begin) * g.nout + j] = v;
        } else if (args.mode == MODE_SCHWARZ) {
          if (a == c && b == d) smax = fmax(smax, fabs(v));
        } else {
          Ob[j - j0] = v;
        }
      }
      if (args.mode == MODE_JK) {
        // every lane owns whole Fock elements and sums their contributions from
        // this pass (no atomics): J'_ab = 2s sum_cd V D_cd, J'_cd = 2s sum_ab V D_ab,
        // K'_ac = s sum_bd V D_bd, K'_ad = s sum_bc V D_bc, K'_bc = s sum_ad V D_ad,
        // K'_bd = s sum_ac V D_ac
        __syncwarp();
        const int nab = g.na * g.nb;
        for (int i = lane; i < g.nacc; i += 32) {
          double sacc = 0.0;
          if (i < oDcd) {
            const int base = i * ncd;
            const int jb = max(base, j0), je = min(base + ncd, j1);
            for (int j = jb; j < je; ++j) sacc += Ob[j - j0] * Ds[oDcd + (j - base)];
            sacc *= 2.0 * sym;
          } else if (i < oDac) {
            const int k = i - oDcd;
            for (int ab = 0; ab < nab; ++ab) {
              const int j = ab * ncd + k;
              if (j >= j0 && j < j1) sacc += Ob[j - j0] * Ds[oDab + ab];
            }
            sacc *= 2.0 * sym;
          } else if (i < oDad) {
            const int k = i - oDac, a = k / g.nc, c = k - a * g.nc;
            for (int b = 0; b < g.nb; ++b) {
              const int base = a * nbcd + b * ncd + c * g.nd;
              const int jb = max(base, j0), je = min(base + g.nd, j1);
              for (int j = jb; j < je; ++j) sacc += Ob[j - j0] * Ds[oDbd + b * g.nd + (j - base)];
            }
            sacc *= sym;
          } else if (i < oDbc) {
            const int k = i - oDad, a = k / g.nd, d = k - a * g.nd;
            for (int b = 0; b < g.nb; ++b)
              for (int c = 0; c < g.nc; ++c) {
                const int j = a * nbcd + b * ncd + c * g.nd + d;
                if (j >= j0 && j < j1) sacc += Ob[j - j0] * Ds[oDbc + b * g.nc + c];
              }
            sacc *= sym;
          } else if (i < oDbd) {
            const int k = i - oDbc, b = k / g.nc, c = k - b * g.nc;
            for (int a = 0; a < g.na; ++a) {
              const int base = a * nbcd + b * ncd + c * g.nd;
              const int jb = max(base, j0), je = min(base + g.nd, j1);
              for (int j = jb; j < je; ++j) sacc += Ob[j - j0] * Ds[oDad + a * g.nd + (j - base)];
            }
            sacc *= sym;
          } else {
            const int k = i - oDbd, b = k / g.nd, d = k - b * g.nd;
            for (int a = 0; a < g.na; ++a)
              for (int c = 0; c < g.nc; ++c) {
                const int j = a * nbcd + b * ncd + c * g.nd + d;
                if (j >= j0 && j < j1) sacc += Ob[j - j0] * Ds[oDac + a * g.nc + c];
              }
            sacc *= sym;
          }
          Acc[i] += sacc;
        }
        __syncwarp();
      }
    }
    count_prims(args.prim_count, lane == 0 ? nprim_done : 0u);
    __syncwarp();
    if (args.mode == MODE_RAW) {
      if (lane == 0) {
        int* mt = args.raw_meta + 4 * (t - blk.t_begin);
        mt[0] = fa; mt[1] = fb; mt[2] = fc; mt[3] = fd;
      }
    } else if (args.mode == MODE_SCHWARZ) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
      if (lane == 0) args.schwarz_out[p] = sqrt(smax);
    } else {
      const size_t n = (size_t)mats.nbf;
      for (int i = lane; i < g.nacc; i += 32) {
        int r0, c0, c1, k;
        double* M;
        if (i < oDcd) { k = i; r0 = fa; c0 = fb; c1 = g.nb; M = mats.J; }
        else if (i < oDac) { k = i - oDcd; r0 = fc; c0 = fd; c1 = g.nd; M = mats.J; }
        else if (i < oDad) { k = i - oDac; r0 = fa; c0 = fc; c1 = g.nc; M = mats.K; }
        else if (i < oDbc) { k = i - oDad; r0 = fa; c0 = fd; c1 = g.nd; M = mats.K; }
        else if (i < oDbd) { k = i - oDbc; r0 = fb; c0 = fc; c1 = g.nc; M = mats.K; }
        else { k = i - oDbd; r0 = fb; c0 = fd; c1 = g.nd; M = mats.K; }
        const double v = Acc[i];
        if (v != 0.0) atomicAdd(M + (size_t)(r0 + k / c1) * n + c0 + k % c1, v);
      }
    }
    __syncwarp();
  }
}

}  // namespace

int launch_tiled(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab, cudaStream_t stream,
                 int num_sms) {
  if (blk.total - blk.t_begin <= 0) return 0;
  // dynamic shared memory available next to the kernel's static class tables
  static size_t smem_max = 0;
  if (!smem_max) {
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, eri_tiled_kernel) != cudaSuccess) return -3;
    const size_t dyn = 227 * 1024 - fa.sharedSizeBytes;
    if (cudaFuncSetAttribute(eri_tiled_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn) !=
        cudaSuccess)
      return -3;
    smem_max = dyn;
  }
  const TiledGeom g = make_tiled_geom(blk.bra.la, blk.bra.lb, blk.ket.la, blk.ket.lb, smem_max / kWarps);
  if (g.per_warp < 0) return -1;
  const size_t smem = (size_t)g.per_warp * 8 * kWarps;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, eri_tiled_kernel, kWarps * 32, smem) != cudaSuccess)
    return -3;
  const int64_t want = (blk.total - blk.t_begin + kWarps - 1) / kWarps;
  const int64_t cap = (int64_t)num_sms * std::max(per_sm, 1) * 4;
  const int grid = (int)std::min<int64_t>(want, cap);
  eri_tiled_kernel<<<grid, kWarps * 32, smem, stream>>>(blk, args, tab, g);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

}  // namespace lai
