// Generic warp-per-quartet Rys ERI kernel (any la..ld <= 4, run-time angular
// momenta), fused with J/K digestion -- the path for the large classes that the
// register-resident (eri_small.cu) and bra-sliced (eri_sliced.cu) kernels do not
// cover.
//
// Per block, class-constant tables are built once in shared memory: the
// Cartesian components of the (e0| and |f0) lists, and for the closed-form
// transfer the row of (e0| needed by every (a, b, k) term with its binomial
// weight and the exponents of (A-B).  Each warp then owns one canonical quartet
// at a time (a contiguous run of quartets per warp):
//   1. items = (primitive quartet x root); lanes build one item's three 2D tables
//      each into shared memory (batches of up to 32 items);
//   2. lanes sweep the (e0|f0) block G in tiles of 32 x kR entries held in
//      registers, summing Ix*Iy*Iz over the staged items (G kept in shared memory
//      or, for the largest classes, a per-warp slab of global scratch);
//   3. per Cartesian component a of the bra's first shell: bra transfer into
//      tmp[b][f], ket transfer + normalization into O[b][c][d], digestion:
//      J_ij[a][:], K_ik[a][:], K_il[a][:] per tile, J_kl, K_jk, K_jl accumulated
//      in shared memory over the tiles.
// The reference counterpart is eri_kernel<La,Lb,Lc,Ld> (thread per quartet,
// src/device/cuda/kernels/eri_kernel.cu:227-461) followed by the separate
// fock_accumulate_batch_kernel (src/device/cuda/consumers/fock_builder_gpu.cu:116-180);
// here no integral is written to HBM.
#include <cuda_runtime.h>

#include "eri_device.cuh"
#include "eri_kernels.h"

namespace lai {

namespace {

constexpr int kR = 8;          // G entries per lane per tile
constexpr int kMaxTerms = 12;  // max prod_x (b_x + 1) over components b with |b| <= 4

struct GenericGeom {
  int la, lb, lc, ld;
  int LAB, LCD;
  int na, nb, nc, nd;
  int NE, NF, NEF;
  int n;          // roots
  int nbt;        // items staged per batch
  int tsz;        // (LAB+1)*(LCD+1)
  // class tables (shared by the block), ints
  int off_ecomp, off_fcomp, off_brow, off_bexp, off_krow, off_kexp, class_ints;
  // per-warp region (doubles)
  int off_tab, off_G, off_tmp, off_O, off_D, off_acc, off_bcoef, off_kcoef, per_warp;
  int G_in_global;
  __host__ __device__ size_t smem_bytes(int warps) const {
    return (size_t)class_ints * 4 + (size_t)per_warp * 8 * warps;
  }
};

__host__ GenericGeom make_geom(int la, int lb, int lc, int ld, size_t smem_limit, int warps) {
  GenericGeom g{};
  g.la = la; g.lb = lb; g.lc = lc; g.ld = ld;
  g.LAB = la + lb; g.LCD = lc + ld;
  g.na = ncart(la); g.nb = ncart(lb); g.nc = ncart(lc); g.nd = ncart(ld);
  g.NE = ncart_range(la, la + lb);
  g.NF = ncart_range(lc, lc + ld);
  g.NEF = g.NE * g.NF;
  g.n = (la + lb + lc + ld) / 2 + 1;
  g.tsz = (g.LAB + 1) * (g.LCD + 1);
  int o = 0;
  g.off_ecomp = o; o += g.NE;
  g.off_fcomp = o; o += g.NF;
  g.off_brow = o; o += g.na * g.nb * kMaxTerms;   // row of (e0| for (a, b, term)
  g.off_bexp = o; o += g.nb * kMaxTerms;          // packed (A-B) exponents | binomial
  g.off_krow = o; o += g.nc * g.nd * kMaxTerms;   // column of |f0) for (c, d, term)
  g.off_kexp = o; o += g.nd * kMaxTerms;
  g.class_ints = (o + 3) & ~3;                    // keeps the double region 16-byte aligned
  const int nD = g.na * g.nb + g.nc * g.nd + g.na * g.nc + g.na * g.nd + g.nb * g.nc + g.nb * g.nd;
  const int nacc = g.nc * g.nd + g.nb * g.nc + g.nb * g.nd;
  for (int nbt = 32; nbt >= 1; nbt >>= 1) {
    for (int gglob = 0; gglob <= 1; ++gglob) {
      g.nbt = nbt;
      g.G_in_global = gglob;
      int w = 0;
      g.off_tab = w; w += nbt * 3 * g.tsz;
      g.off_G = w; w += gglob ? 0 : g.NEF;
      g.off_tmp = w; w += g.nb * g.NF;
      g.off_O = w; w += g.nb * g.nc * g.nd;
      g.off_D = w; w += nD;
      g.off_acc = w; w += nacc;
      g.off_bcoef = w; w += g.nb * kMaxTerms;
      g.off_kcoef = w; w += g.nd * kMaxTerms;
      g.per_warp = (w + 1) & ~1;
      if (g.smem_bytes(warps) <= smem_limit) return g;
    }
  }
  g.per_warp = -1;
  return g;
}

// Build the 2D tables of one (primitive quartet, root) item into tab[3][LAB+1][LCD+1].
__device__ __forceinline__ void vrr_item(const GenericGeom& g, double* __restrict__ tab, double u,
                                         double wp, const double PA[3], const double QC[3],
                                         const double PQ[3], double rz, double re, double hz,
                                         double he, double hinv) {
  const double b00 = hinv * u;
  const double b10 = hz - hz * rz * u;
  const double b01 = he - he * re * u;
  const int W = g.LCD + 1;
  for (int x = 0; x < 3; ++x) {
    double* I = tab + x * g.tsz;
    const double pa = PA[x] - rz * u * PQ[x];
    const double qc = QC[x] + re * u * PQ[x];
    I[0] = (x == 2) ? wp : 1.0;
    if (g.LAB > 0) I[W] = pa * I[0];
    for (int e = 1; e < g.LAB; ++e) I[(e + 1) * W] = pa * I[e * W] + e * b10 * I[(e - 1) * W];
    for (int f = 0; f < g.LCD; ++f) {
      for (int e = 0; e <= g.LAB; ++e) {
        double v = qc * I[e * W + f];
        if (f) v += f * b01 * I[e * W + f - 1];
        if (e) v += e * b00 * I[(e - 1) * W + f];
        I[e * W + f + 1] = v;
      }
    }
  }
}

// Class tables: component lists and the transfer terms.  brow[(a*nb+b)*T + m] is
// the row in (e0| of a+k for the m-th shift k <= b (-1 past the last term);
// bexp[b*T + m] packs the exponents of (A-B) with the binomial product in the
// high bits.  krow / kexp are the same for the ket.
__device__ void build_class_tables(const GenericGeom& g, int* __restrict__ ci) {
  int* ecomp = ci + g.off_ecomp;
  int* fcomp = ci + g.off_fcomp;
  int* brow = ci + g.off_brow;
  int* bexp = ci + g.off_bexp;
  int* krow = ci + g.off_krow;
  int* kexp = ci + g.off_kexp;
  for (int i = threadIdx.x; i < g.NE; i += blockDim.x) {
    int l = g.la, r = i;
    while (r >= ncart(l)) { r -= ncart(l); ++l; }
    ecomp[i] = cart_comp(l, r);
  }
  for (int i = threadIdx.x; i < g.NF; i += blockDim.x) {
    int l = g.lc, r = i;
    while (r >= ncart(l)) { r -= ncart(l); ++l; }
    fcomp[i] = cart_comp(l, r);
  }
  for (int side = 0; side < 2; ++side) {
    const int lt = side ? g.ld : g.lb;
    const int nt = side ? g.nd : g.nb;
    int* ex = side ? kexp : bexp;
    for (int i = threadIdx.x; i < nt; i += blockDim.x) {
      const int cb = cart_comp(lt, i);
      int m = 0;
      for (int kx = 0; kx <= comp_x(cb); ++kx)
        for (int ky = 0; ky <= comp_y(cb); ++ky)
          for (int kz = 0; kz <= comp_z(cb); ++kz, ++m) {
            const int bi = (int)(binom(comp_x(cb), kx) * binom(comp_y(cb), ky) * binom(comp_z(cb), kz));
            ex[i * kMaxTerms + m] = (comp_x(cb) - kx) | ((comp_y(cb) - ky) << 4) |
                                    ((comp_z(cb) - kz) << 8) | (bi << 12);
          }
      for (; m < kMaxTerms; ++m) ex[i * kMaxTerms + m] = -1;
    }
  }
  for (int side = 0; side < 2; ++side) {
    const int l1 = side ? g.lc : g.la, l2 = side ? g.ld : g.lb;
    const int n1 = ncart(l1), n2 = ncart(l2);
    int* rows = side ? krow : brow;
    for (int i = threadIdx.x; i < n1 * n2; i += blockDim.x) {
      const int a = i / n2, b = i - a * n2;
      const int ca = cart_comp(l1, a), cb = cart_comp(l2, b);
      int m = 0;
      for (int kx = 0; kx <= comp_x(cb); ++kx)
        for (int ky = 0; ky <= comp_y(cb); ++ky)
          for (int kz = 0; kz <= comp_z(cb); ++kz, ++m) {
            const int ex = comp_x(ca) + kx, ey = comp_y(ca) + ky, ez = comp_z(ca) + kz;
            rows[i * kMaxTerms + m] = ncart_before(l1, ex + ey + ez) + cart_index(ex, ey, ez);
          }
      for (; m < kMaxTerms; ++m) rows[i * kMaxTerms + m] = -1;
    }
  }
}

__device__ __forceinline__ double pow_small(double x, int m) {
  double r = 1.0;
  for (int i = 0; i < m; ++i) r *= x;
  return r;
}

__device__ __forceinline__ double comp_norm(int c) {
  return rsqrt(dfact_odd(comp_x(c)) * dfact_odd(comp_y(c)) * dfact_odd(comp_z(c)));
}

__global__ void __launch_bounds__(128) eri_generic_kernel(QuartetBlock blk, JKArgs args,
                                                          RysTablesView tab, GenericGeom g,
                                                          double* __restrict__ gscratch) {
  extern __shared__ double smem[];
  int* ci = reinterpret_cast<int*>(smem);
  build_class_tables(g, ci);
  __syncthreads();
  const int* ecomp = ci + g.off_ecomp;
  const int* fcomp = ci + g.off_fcomp;
  const int* brow = ci + g.off_brow;
  const int* bexp = ci + g.off_bexp;
  const int* krow = ci + g.off_krow;
  const int* kexp = ci + g.off_kexp;

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps_blk = blockDim.x >> 5;
  double* ws = smem + (size_t)g.class_ints / 2 + (size_t)warp * g.per_warp;
  double* tabs = ws + g.off_tab;
  const int64_t gwarp = (int64_t)blockIdx.x * nwarps_blk + warp;
  const int64_t nwarps = (int64_t)gridDim.x * nwarps_blk;
  double* G = g.G_in_global ? gscratch + (size_t)gwarp * g.NEF : ws + g.off_G;
  double* tmp = ws + g.off_tmp;
  double* O = ws + g.off_O;
  double* Dij = ws + g.off_D;
  double* Dkl = Dij + g.na * g.nb;
  double* Dik = Dkl + g.nc * g.nd;
  double* Dil = Dik + g.na * g.nc;
  double* Djk = Dil + g.na * g.nd;
  double* Djl = Djk + g.nb * g.nc;
  double* Akl = ws + g.off_acc;
  double* Ajk = Akl + g.nc * g.nd;
  double* Ajl = Ajk + g.nb * g.nc;
  double* bcoef = ws + g.off_bcoef;
  double* kcoef = ws + g.off_kcoef;

  const int Kab = blk.bra.Ka * blk.bra.Kb;
  const int Kcd = blk.ket.Ka * blk.ket.Kb;
  const int nitems = Kab * Kcd * g.n;
  const int nbra = blk.bra.npairs, nket = blk.ket.npairs;
  const int W = g.LCD + 1;
  const int ncd = g.nc * g.nd;
  const size_t sb = (size_t)Kab * nbra, sk = (size_t)Kcd * nket;

  const int64_t nq_all = blk.total - blk.t_begin;
  const int64_t per = (nq_all + nwarps - 1) / nwarps;
  const int64_t tbeg = blk.t_begin + gwarp * per;
  const int64_t tend = min(blk.total, tbeg + per);
  int p = -1;
  for (int64_t t = tbeg; t < tend; ++t) {
    const int64_t tl = t - blk.t_begin;
    if (p < 0) {
      if (lane == 0) p = find_bra(blk.offsets, nbra, t);
      p = __shfl_sync(0xffffffffu, p, 0);
    } else {
      while (t >= __ldg(blk.offsets + p + 1)) ++p;
    }
    const int q = (blk.qbegin ? __ldg(blk.qbegin + p) : 0) + (int)(t - __ldg(blk.offsets + p));
    const double AB[3] = {__ldg(blk.bra.AB + p), __ldg(blk.bra.AB + nbra + p),
                          __ldg(blk.bra.AB + 2 * nbra + p)};
    const double CD[3] = {__ldg(blk.ket.AB + q), __ldg(blk.ket.AB + nket + q),
                          __ldg(blk.ket.AB + 2 * nket + q)};
    const int fa = __ldg(blk.bra.func_a + p), fb = __ldg(blk.bra.func_b + p);
    const int fc = __ldg(blk.ket.func_a + q), fd = __ldg(blk.ket.func_b + q);

    // transfer coefficients of this quartet
    for (int i = lane; i < g.nb * kMaxTerms; i += 32) {
      const int e = bexp[i];
      bcoef[i] = e < 0 ? 0.0 : double(e >> 12) * pow_small(AB[0], e & 15) *
                                   pow_small(AB[1], (e >> 4) & 15) * pow_small(AB[2], (e >> 8) & 15);
    }
    for (int i = lane; i < g.nd * kMaxTerms; i += 32) {
      const int e = kexp[i];
      kcoef[i] = e < 0 ? 0.0 : double(e >> 12) * pow_small(CD[0], e & 15) *
                                   pow_small(CD[1], (e >> 4) & 15) * pow_small(CD[2], (e >> 8) & 15);
    }
    for (int i = lane; i < g.NEF; i += 32) G[i] = 0.0;
    __syncwarp();

    // ---- (e0|f0) accumulation ----
    unsigned int nprim_done = 0;
    for (int it0 = 0; it0 < nitems; it0 += g.nbt) {
      const int it = it0 + lane;
      if (lane < g.nbt && it < nitems) {
        const int pq = it / g.n, r = it - pq * g.n;
        const int ib = pq / Kcd, ik = pq - ib * Kcd;
        const double* pb = blk.bra.prim + (size_t)ib * nbra + p;
        const double* pk = blk.ket.prim + (size_t)ik * nket + q;
        const double zeta = __ldg(pb + PF_ZETA * sb), eta = __ldg(pk + PF_ZETA * sk);
        const double hz = __ldg(pb + PF_HZ * sb), he = __ldg(pk + PF_HZ * sk);
        const double PQ[3] = {__ldg(pb + PF_PX * sb) - __ldg(pk + PF_PX * sk),
                              __ldg(pb + PF_PY * sb) - __ldg(pk + PF_PY * sk),
                              __ldg(pb + PF_PZ * sb) - __ldg(pk + PF_PZ * sk)};
        const double PA[3] = {__ldg(pb + PF_PAX * sb), __ldg(pb + PF_PAY * sb), __ldg(pb + PF_PAZ * sb)};
        const double QC[3] = {__ldg(pk + PF_PAX * sk), __ldg(pk + PF_PAY * sk), __ldg(pk + PF_PAZ * sk)};
        const double skip =
            (__ldg(pb + PF_Q * sb) * __ldg(pk + PF_Q * sk) < args.prim_eps) ? 0.0 : 1.0;
        const double cab = __ldg(pb + PF_C * sb) * skip, ccd = __ldg(pk + PF_C * sk);
        const double s = zeta + eta;
        const double rs = rsqrt(s);
        const double inv = rs * rs;
        const double rz = eta * inv, re = zeta * inv;
        const double T = zeta * rz * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
        double u, w;
        rys_root_one<double>(g.n, r, T, tab, u, w);
        vrr_item(g, tabs + lane * 3 * g.tsz, u, w * cab * ccd * rs, PA, QC, PQ, rz, re, hz, he,
                 0.5 * inv);
        if (r == 0 && skip != 0.0) ++nprim_done;
      }
      __syncwarp();
      const int nb_now = min(g.nbt, nitems - it0);
      for (int base = 0; base < g.NEF; base += 32 * kR) {
        double acc[kR];
        int off[kR];
#pragma unroll
        for (int m = 0; m < kR; ++m) {
          const int idx = base + lane + 32 * m;
          acc[m] = 0.0;
          off[m] = -1;
          if (idx < g.NEF) {
            const int ie = idx / g.NF, jf = idx - ie * g.NF;
            const int ce = ecomp[ie], cf = fcomp[jf];
            off[m] = (comp_x(ce) * W + comp_x(cf)) | ((comp_y(ce) * W + comp_y(cf)) << 10) |
                     ((comp_z(ce) * W + comp_z(cf)) << 20);
          }
        }
        for (int sidx = 0; sidx < nb_now; ++sidx) {
          const double* T3 = tabs + sidx * 3 * g.tsz;
#pragma unroll
          for (int m = 0; m < kR; ++m) {
            const int o = off[m];
            if (o >= 0)
              acc[m] += T3[o & 1023] * T3[g.tsz + ((o >> 10) & 1023)] * T3[2 * g.tsz + (o >> 20)];
          }
        }
#pragma unroll
        for (int m = 0; m < kR; ++m) {
          const int idx = base + lane + 32 * m;
          if (idx < g.NEF) G[idx] += acc[m];
        }
      }
      __syncwarp();
    }

    count_prims(args.prim_count, nprim_done);

    // ---- digestion setup ----
    const double sym = quartet_weight(blk, p, q);
    const SysMats mats = sys_mats(args, blk, p);
    if (args.mode == MODE_JK) {
      const int nbf = mats.nbf;
      for (int i = lane; i < g.na * g.nb; i += 32) {
        const int a = i / g.nb, b = i - a * g.nb;
        Dij[i] = __ldg(mats.D + (size_t)(fa + a) * nbf + fb + b);
      }
      for (int i = lane; i < ncd; i += 32) {
        const int c = i / g.nd, d = i - c * g.nd;
        Dkl[i] = __ldg(mats.D + (size_t)(fc + c) * nbf + fd + d);
        Akl[i] = 0.0;
      }
      for (int i = lane; i < g.na * g.nc; i += 32) {
        const int a = i / g.nc, c = i - a * g.nc;
        Dik[i] = __ldg(mats.D + (size_t)(fa + a) * nbf + fc + c);
      }
      for (int i = lane; i < g.na * g.nd; i += 32) {
        const int a = i / g.nd, d = i - a * g.nd;
        Dil[i] = __ldg(mats.D + (size_t)(fa + a) * nbf + fd + d);
      }
      for (int i = lane; i < g.nb * g.nc; i += 32) {
        const int b = i / g.nc, c = i - b * g.nc;
        Djk[i] = __ldg(mats.D + (size_t)(fb + b) * nbf + fc + c);
        Ajk[i] = 0.0;
      }
      for (int i = lane; i < g.nb * g.nd; i += 32) {
        const int b = i / g.nd, d = i - b * g.nd;
        Djl[i] = __ldg(mats.D + (size_t)(fb + b) * nbf + fd + d);
        Ajl[i] = 0.0;
      }
    }
    double smax = 0.0;
    __syncwarp();

    for (int a = 0; a < g.na; ++a) {
      // bra transfer: tmp[b][f] = sum_m bcoef[b][m] G[brow[a][b][m]][f]
      for (int i = lane; i < g.nb * g.NF; i += 32) {
        const int b = i / g.NF, f = i - b * g.NF;
        const int* rows = brow + (a * g.nb + b) * kMaxTerms;
        const double* cf = bcoef + b * kMaxTerms;
        double v = 0.0;
        for (int m = 0; m < kMaxTerms; ++m) {
          const int row = rows[m];
          if (row < 0) break;
          v += cf[m] * G[row * g.NF + f];
        }
        tmp[i] = v;
      }
      __syncwarp();
      const double na_f = comp_norm(cart_comp(g.la, a));
      for (int i = lane; i < g.nb * ncd; i += 32) {
        const int b = i / ncd, cdi = i - b * ncd;
        const int c = cdi / g.nd, d = cdi - c * g.nd;
        const int* cols = krow + cdi * kMaxTerms;
        const double* cf = kcoef + d * kMaxTerms;
        double v = 0.0;
        for (int m = 0; m < kMaxTerms; ++m) {
          const int col = cols[m];
          if (col < 0) break;
          v += cf[m] * tmp[b * g.NF + col];
        }
        v *= na_f * comp_norm(cart_comp(g.lb, b)) * comp_norm(cart_comp(g.lc, c)) *
             comp_norm(cart_comp(g.ld, d));
        O[i] = v;
        if (args.mode == MODE_RAW) {
          args.raw_out[(size_t)tl * g.na * g.nb * ncd + (size_t)a * g.nb * ncd + i] = v;
        } else if (args.mode == MODE_SCHWARZ) {
          if (c == a && d == b) smax = fmax(smax, fabs(v));
        }
      }
      __syncwarp();
      if (args.mode == MODE_JK) {
        const int nbf = mats.nbf;
        for (int i = lane; i < g.nb + g.nc + g.nd; i += 32) {
          if (i < g.nb) {  // J_ij[a][b] += 2 s sum_cd O[b][c][d] D_kl[c][d]
            const int b = i;
            double v = 0.0;
            for (int x = 0; x < ncd; ++x) v += O[b * ncd + x] * Dkl[x];
            atomicAdd(mats.J + (size_t)(fa + a) * nbf + fb + b, 2.0 * sym * v);
          } else if (i < g.nb + g.nc) {  // K_ik[a][c] += s sum_bd O[b][c][d] D_jl[b][d]
            const int c = i - g.nb;
            double v = 0.0;
            for (int b = 0; b < g.nb; ++b)
              for (int d = 0; d < g.nd; ++d) v += O[b * ncd + c * g.nd + d] * Djl[b * g.nd + d];
            atomicAdd(mats.K + (size_t)(fa + a) * nbf + fc + c, sym * v);
          } else {  // K_il[a][d] += s sum_bc O[b][c][d] D_jk[b][c]
            const int d = i - g.nb - g.nc;
            double v = 0.0;
            for (int b = 0; b < g.nb; ++b)
              for (int c = 0; c < g.nc; ++c) v += O[b * ncd + c * g.nd + d] * Djk[b * g.nc + c];
            atomicAdd(mats.K + (size_t)(fa + a) * nbf + fd + d, sym * v);
          }
        }
        for (int i = lane; i < ncd; i += 32) {  // J_kl[c][d] partial: sum_b O D_ij[a][b]
          double v = 0.0;
          for (int b = 0; b < g.nb; ++b) v += O[b * ncd + i] * Dij[a * g.nb + b];
          Akl[i] += v;
        }
        for (int i = lane; i < g.nb * g.nc; i += 32) {  // K_jk[b][c] partial: sum_d O D_il[a][d]
          const int b = i / g.nc, c = i - b * g.nc;
          double v = 0.0;
          for (int d = 0; d < g.nd; ++d) v += O[b * ncd + c * g.nd + d] * Dil[a * g.nd + d];
          Ajk[i] += v;
        }
        for (int i = lane; i < g.nb * g.nd; i += 32) {  // K_jl[b][d] partial: sum_c O D_ik[a][c]
          const int b = i / g.nd, d = i - b * g.nd;
          double v = 0.0;
          for (int c = 0; c < g.nc; ++c) v += O[b * ncd + c * g.nd + d] * Dik[a * g.nc + c];
          Ajl[i] += v;
        }
      }
      __syncwarp();
    }
    if (args.mode == MODE_JK) {
      const int nbf = mats.nbf;
      for (int i = lane; i < ncd; i += 32) {
        const int c = i / g.nd, d = i - c * g.nd;
        atomicAdd(mats.J + (size_t)(fc + c) * nbf + fd + d, 2.0 * sym * Akl[i]);
      }
      for (int i = lane; i < g.nb * g.nc; i += 32) {
        const int b = i / g.nc, c = i - b * g.nc;
        atomicAdd(mats.K + (size_t)(fb + b) * nbf + fc + c, sym * Ajk[i]);
      }
      for (int i = lane; i < g.nb * g.nd; i += 32) {
        const int b = i / g.nd, d = i - b * g.nd;
        atomicAdd(mats.K + (size_t)(fb + b) * nbf + fd + d, sym * Ajl[i]);
      }
    } else if (args.mode == MODE_RAW) {
      if (lane == 0) {
        int* m = args.raw_meta + 4 * tl;
        m[0] = fa; m[1] = fb; m[2] = fc; m[3] = fd;
      }
    } else if (args.mode == MODE_SCHWARZ) {
      for (int o = 16; o > 0; o >>= 1) smax = fmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
      if (lane == 0) args.schwarz_out[p] = sqrt(smax);
    }
    __syncwarp();
  }
}

}  // namespace

int launch_generic(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab,
                   cudaStream_t stream, double* gscratch, size_t gscratch_doubles, int num_sms) {
  if (blk.total - blk.t_begin <= 0) return 0;
  const int la = blk.bra.la, lb = blk.bra.lb, lc = blk.ket.la, ld = blk.ket.lb;
  int warps = 4;
  const size_t smem_max = 227 * 1024;
  GenericGeom g = make_geom(la, lb, lc, ld, smem_max, warps);
  if (g.per_warp < 0) { warps = 1; g = make_geom(la, lb, lc, ld, smem_max, warps); }
  if (g.per_warp < 0) return -1;
  const size_t smem = g.smem_bytes(warps);
  const int64_t want = (blk.total - blk.t_begin + warps - 1) / warps;
  const int64_t cap = (int64_t)num_sms * 8;
  int grid = (int)(want < cap ? want : cap);
  if (g.G_in_global) {
    const size_t need = (size_t)grid * warps * g.NEF;
    if (need > gscratch_doubles) {
      grid = (int)(gscratch_doubles / ((size_t)warps * g.NEF));
      if (grid < 1) return -2;
    }
  }
  static bool attr_set = false;
  if (!attr_set) {
    if (cudaFuncSetAttribute(eri_generic_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem_max) != cudaSuccess)
      return -3;
    attr_set = true;
  }
  eri_generic_kernel<<<grid, warps * 32, smem, stream>>>(blk, args, tab, g, gscratch);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

size_t generic_global_scratch_doubles(int la, int lb, int lc, int ld, int num_sms) {
  int warps = 4;
  GenericGeom g = make_geom(la, lb, lc, ld, 227 * 1024, warps);
  if (g.per_warp < 0) { warps = 1; g = make_geom(la, lb, lc, ld, 227 * 1024, warps); }
  if (g.per_warp < 0 || !g.G_in_global) return 0;
  return (size_t)num_sms * 8 * warps * g.NEF;
}

}  // namespace lai
