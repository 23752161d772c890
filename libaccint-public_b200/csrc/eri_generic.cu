// Generic warp-per-quartet Rys ERI kernel (any la..ld <= 4, runtime angular
// momenta), fused with J/K digestion.  It is the path for the larger classes,
// whose per-quartet state does not fit one thread's registers; the small classes
// run in the thread-per-quartet kernels of eri_small.cu.
//
// One warp owns one canonical quartet at a time (grid-stride over the block's
// flat quartet range):
//   * lanes split the (primitive quartet x root) items: each lane evaluates one
//     root and builds that root's three 2D tables into shared memory;
//   * lanes then split the (e0|f0) accumulator G: each lane owns up to kRmax
//     entries in registers and sums Ix*Iy*Iz over the staged items;
//   * G goes to shared memory; for each Cartesian component a of the bra's first
//     shell the warp does the bra then ket transfer into an output tile
//     O[b][c][d] and digests it: J_ij[a][:], K_ik[a][:], K_il[a][:] are complete
//     per tile, J_kl, K_jk, K_jl accumulate in shared memory across tiles.
// The reference's counterparts are eri_kernel<La,Lb,Lc,Ld> (thread per quartet,
// src/device/cuda/kernels/eri_kernel.cu:227-461) followed by a separate
// fock_accumulate_batch_kernel (src/device/cuda/consumers/fock_builder_gpu.cu:116-180)
// that re-reads every integral from HBM; here no integral is written to HBM.
#include <cuda_runtime.h>

#include "eri_device.cuh"
#include "eri_kernels.h"

namespace lai {

namespace {

constexpr int kRmax = 32;  // G entries per lane per pass

struct GenericGeom {
  int la, lb, lc, ld;
  int LAB, LCD;            // la+lb, lc+ld
  int na, nb, nc, nd;
  int NE, NF, NEF;         // (e0| and |f0) component counts
  int n;                   // roots
  int nbt;                 // items staged per batch
  int tsz;                 // (LAB+1)*(LCD+1)
  // per-warp shared-memory layout (in doubles)
  int off_tab, off_G, off_tmp, off_O, off_D, off_acc, per_warp;
  int G_in_global;
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
  const int nD = g.na * g.nb + g.nc * g.nd + g.na * g.nc + g.na * g.nd + g.nb * g.nc + g.nb * g.nd;
  const int nacc = g.nc * g.nd + g.nb * g.nc + g.nb * g.nd;
  const int nO = g.nb * g.nc * g.nd;
  const int ntmp = g.nb * g.NF;
  for (int nbt = 32; nbt >= 1; nbt >>= 1) {
    for (int gglob = 0; gglob <= 1; ++gglob) {
      g.nbt = nbt;
      g.G_in_global = gglob;
      int o = 0;
      g.off_tab = o; o += nbt * 3 * g.tsz;
      g.off_G = o; o += gglob ? 0 : g.NEF;
      g.off_tmp = o; o += ntmp;
      g.off_O = o; o += nO;
      g.off_D = o; o += nD;
      g.off_acc = o; o += nacc;
      g.per_warp = (o + 1) & ~1;  // keep 16-byte alignment between warps
      if ((size_t)g.per_warp * 8 * warps <= smem_limit) return g;
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
  // rz = eta/(zeta+eta), re = zeta/(zeta+eta), hz = 0.5/zeta, he = 0.5/eta, hinv = 0.5/(zeta+eta)
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

__global__ void __launch_bounds__(128) eri_generic_kernel(QuartetBlock blk, JKArgs args,
                                                          RysTablesView tab, GenericGeom g,
                                                          double* __restrict__ gscratch) {
  extern __shared__ double smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwarps_blk = blockDim.x >> 5;
  double* ws = smem + (size_t)warp * g.per_warp;
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

  const int Kab = blk.bra.Ka * blk.bra.Kb;
  const int Kcd = blk.ket.Ka * blk.ket.Kb;
  const int nitems = Kab * Kcd * g.n;
  const int nbra = blk.bra.npairs, nket = blk.ket.npairs;
  const int W = g.LCD + 1;

  // each warp owns a contiguous run of quartets: one search, then p advances
  const int64_t nq_all = blk.total - blk.t_begin;
  const int64_t per = (nq_all + nwarps - 1) / nwarps;
  const int64_t tbeg = blk.t_begin + gwarp * per;
  const int64_t tend = min(blk.total, tbeg + per);
  int p = -1;
  for (int64_t t = tbeg; t < tend; ++t) {
    const int64_t tl = t - blk.t_begin;
    // ---- locate the quartet ----
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

    // ---- (e0|f0) accumulation, in passes of 32*kRmax entries ----
    for (int pass0 = 0; pass0 < g.NEF; pass0 += 32 * kRmax) {
      double acc[kRmax];
      int offs[kRmax];
#pragma unroll
      for (int m = 0; m < kRmax; ++m) {
        acc[m] = 0.0;
        const int idx = pass0 + lane + 32 * m;
        int packed = -1;
        if (idx < g.NEF) {
          const int ie = idx / g.NF, jf = idx - ie * g.NF;
          // component of entry ie within shells la..la+lb, jf within lc..lc+ld
          int le = g.la, r = ie;
          while (r >= ncart(le)) { r -= ncart(le); ++le; }
          int lf = g.lc, s = jf;
          while (s >= ncart(lf)) { s -= ncart(lf); ++lf; }
          const int ce = cart_comp(le, r), cf = cart_comp(lf, s);
          const int ox = comp_x(ce) * W + comp_x(cf);
          const int oy = comp_y(ce) * W + comp_y(cf);
          const int oz = comp_z(ce) * W + comp_z(cf);
          packed = ox | (oy << 10) | (oz << 20);
        }
        offs[m] = packed;
      }
      for (int it0 = 0; it0 < nitems; it0 += g.nbt) {
        const int it = it0 + lane;
        if (lane < g.nbt && it < nitems) {
          const int pq = it / g.n, r = it - pq * g.n;
          const int ib = pq / Kcd, ik = pq - ib * Kcd;
          const size_t sb = (size_t)Kab * nbra, sk = (size_t)Kcd * nket;
          const double* pb = blk.bra.prim + (size_t)ib * nbra + p;
          const double* pk = blk.ket.prim + (size_t)ik * nket + q;
          const double zeta = __ldg(pb + PF_ZETA * sb), eta = __ldg(pk + PF_ZETA * sk);
          const double hz = __ldg(pb + PF_HZ * sb), he = __ldg(pk + PF_HZ * sk);
          const double P[3] = {__ldg(pb + PF_PX * sb), __ldg(pb + PF_PY * sb), __ldg(pb + PF_PZ * sb)};
          const double Qc[3] = {__ldg(pk + PF_PX * sk), __ldg(pk + PF_PY * sk), __ldg(pk + PF_PZ * sk)};
          const double PA[3] = {__ldg(pb + PF_PAX * sb), __ldg(pb + PF_PAY * sb), __ldg(pb + PF_PAZ * sb)};
          const double QC[3] = {__ldg(pk + PF_PAX * sk), __ldg(pk + PF_PAY * sk), __ldg(pk + PF_PAZ * sk)};
          const double cab = __ldg(pb + PF_C * sb), ccd = __ldg(pk + PF_C * sk);
          const double s = zeta + eta;
          const double rs = rsqrt(s);
          const double inv = rs * rs;
          const double rz = eta * inv, re = zeta * inv;
          const double PQ[3] = {P[0] - Qc[0], P[1] - Qc[1], P[2] - Qc[2]};
          const double T = zeta * rz * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
          double u, w;
          rys_root_one<double>(g.n, r, T, tab, u, w);
          vrr_item(g, tabs + lane * 3 * g.tsz, u, w * cab * ccd * rs, PA, QC, PQ, rz, re, hz, he,
                   0.5 * inv);
        }
        __syncwarp();
        const int nb_now = min(g.nbt, nitems - it0);
#pragma unroll
        for (int m = 0; m < kRmax; ++m) {
          const int pk = offs[m];
          if (pk >= 0) {
            const int ox = pk & 1023, oy = (pk >> 10) & 1023, oz = pk >> 20;
            double a = acc[m];
            for (int sidx = 0; sidx < nb_now; ++sidx) {
              const double* T3 = tabs + sidx * 3 * g.tsz;
              a += T3[ox] * T3[g.tsz + oy] * T3[2 * g.tsz + oz];
            }
            acc[m] = a;
          }
        }
        __syncwarp();
      }
#pragma unroll
      for (int m = 0; m < kRmax; ++m) {
        const int idx = pass0 + lane + 32 * m;
        if (idx < g.NEF) G[idx] = acc[m];
      }
    }

    // ---- digestion setup ----
    const double sym = quartet_weight(blk, p, q);
    if (args.mode == MODE_JK) {
      const int nbf = args.nbf;
      for (int i = lane; i < g.na * g.nb; i += 32) {
        const int a = i / g.nb, b = i - a * g.nb;
        Dij[i] = __ldg(args.D + (size_t)(fa + a) * nbf + fb + b);
      }
      for (int i = lane; i < g.nc * g.nd; i += 32) {
        const int c = i / g.nd, d = i - c * g.nd;
        Dkl[i] = __ldg(args.D + (size_t)(fc + c) * nbf + fd + d);
        Akl[i] = 0.0;
      }
      for (int i = lane; i < g.na * g.nc; i += 32) {
        const int a = i / g.nc, c = i - a * g.nc;
        Dik[i] = __ldg(args.D + (size_t)(fa + a) * nbf + fc + c);
      }
      for (int i = lane; i < g.na * g.nd; i += 32) {
        const int a = i / g.nd, d = i - a * g.nd;
        Dil[i] = __ldg(args.D + (size_t)(fa + a) * nbf + fd + d);
      }
      for (int i = lane; i < g.nb * g.nc; i += 32) {
        const int b = i / g.nc, c = i - b * g.nc;
        Djk[i] = __ldg(args.D + (size_t)(fb + b) * nbf + fc + c);
        Ajk[i] = 0.0;
      }
      for (int i = lane; i < g.nb * g.nd; i += 32) {
        const int b = i / g.nd, d = i - b * g.nd;
        Djl[i] = __ldg(args.D + (size_t)(fb + b) * nbf + fd + d);
        Ajl[i] = 0.0;
      }
    }
    double smax = 0.0;
    __syncwarp();

    // ---- per bra component a: HRR into O[b][c][d], then digest ----
    const int ncd = g.nc * g.nd;
    for (int a = 0; a < g.na; ++a) {
      const int ca = cart_comp(g.la, a);
      // bra transfer: tmp[b][f] = sum_k C(b,k) AB^(b-k) G[a+k][f]
      for (int i = lane; i < g.nb * g.NF; i += 32) {
        const int b = i / g.NF, f = i - b * g.NF;
        const int cb = cart_comp(g.lb, b);
        const int bx = comp_x(cb), by = comp_y(cb), bz = comp_z(cb);
        double v = 0.0;
        for (int kx = 0; kx <= bx; ++kx)
          for (int ky = 0; ky <= by; ++ky)
            for (int kz = 0; kz <= bz; ++kz) {
              const int ex = comp_x(ca) + kx, ey = comp_y(ca) + ky, ez = comp_z(ca) + kz;
              const int le = ex + ey + ez;
              const int row = ncart_before(g.la, le) + cart_index(ex, ey, ez);
              const double cf = binom(bx, kx) * binom(by, ky) * binom(bz, kz) *
                                ipow(AB[0], bx - kx) * ipow(AB[1], by - ky) * ipow(AB[2], bz - kz);
              v += cf * G[row * g.NF + f];
            }
        tmp[i] = v;
      }
      __syncwarp();
      // ket transfer + normalization: O[b][c][d]
      const double na_f = norm_factor(g.la, a);
      for (int i = lane; i < g.nb * ncd; i += 32) {
        const int b = i / ncd, cdi = i - b * ncd;
        const int c = cdi / g.nd, d = cdi - c * g.nd;
        const int cc = cart_comp(g.lc, c), cdd = cart_comp(g.ld, d);
        const int dx = comp_x(cdd), dy = comp_y(cdd), dz = comp_z(cdd);
        double v = 0.0;
        for (int kx = 0; kx <= dx; ++kx)
          for (int ky = 0; ky <= dy; ++ky)
            for (int kz = 0; kz <= dz; ++kz) {
              const int fx = comp_x(cc) + kx, fy = comp_y(cc) + ky, fz = comp_z(cc) + kz;
              const int lf = fx + fy + fz;
              const int col = ncart_before(g.lc, lf) + cart_index(fx, fy, fz);
              const double cf = binom(dx, kx) * binom(dy, ky) * binom(dz, kz) *
                                ipow(CD[0], dx - kx) * ipow(CD[1], dy - ky) * ipow(CD[2], dz - kz);
              v += cf * tmp[b * g.NF + col];
            }
        v *= na_f * norm_factor(g.lb, b) * norm_factor(g.lc, c) * norm_factor(g.ld, d);
        O[i] = v;
        if (args.mode == MODE_RAW) {
          args.raw_out[(size_t)tl * g.na * g.nb * ncd + (size_t)a * g.nb * ncd + i] = v;
        } else if (args.mode == MODE_SCHWARZ) {
          if (c == a && d == b) smax = fmax(smax, fabs(v));
        }
      }
      __syncwarp();
      if (args.mode == MODE_JK) {
        const int nbf = args.nbf;
        // targets of this tile
        for (int i = lane; i < g.nb + g.nc + g.nd; i += 32) {
          if (i < g.nb) {  // J_ij[a][b] += 2 s sum_cd O[b][c][d] D_kl[c][d]
            const int b = i;
            double v = 0.0;
            for (int x = 0; x < ncd; ++x) v += O[b * ncd + x] * Dkl[x];
            atomicAdd(args.J + (size_t)(fa + a) * nbf + fb + b, 2.0 * sym * v);
          } else if (i < g.nb + g.nc) {  // K_ik[a][c] += s sum_bd O[b][c][d] D_jl[b][d]
            const int c = i - g.nb;
            double v = 0.0;
            for (int b = 0; b < g.nb; ++b)
              for (int d = 0; d < g.nd; ++d) v += O[b * ncd + c * g.nd + d] * Djl[b * g.nd + d];
            atomicAdd(args.K + (size_t)(fa + a) * nbf + fc + c, sym * v);
          } else {  // K_il[a][d] += s sum_bc O[b][c][d] D_jk[b][c]
            const int d = i - g.nb - g.nc;
            double v = 0.0;
            for (int b = 0; b < g.nb; ++b)
              for (int c = 0; c < g.nc; ++c) v += O[b * ncd + c * g.nd + d] * Djk[b * g.nc + c];
            atomicAdd(args.K + (size_t)(fa + a) * nbf + fd + d, sym * v);
          }
        }
        // accumulators across tiles
        for (int i = lane; i < ncd; i += 32) {  // J_kl[c][d] += 2 s sum_b O[b][c][d] D_ij[a][b]
          double v = 0.0;
          for (int b = 0; b < g.nb; ++b) v += O[b * ncd + i] * Dij[a * g.nb + b];
          Akl[i] += v;
        }
        for (int i = lane; i < g.nb * g.nc; i += 32) {  // K_jk[b][c] += s sum_d O D_il[a][d]
          const int b = i / g.nc, c = i - b * g.nc;
          double v = 0.0;
          for (int d = 0; d < g.nd; ++d) v += O[b * ncd + c * g.nd + d] * Dil[a * g.nd + d];
          Ajk[i] += v;
        }
        for (int i = lane; i < g.nb * g.nd; i += 32) {  // K_jl[b][d] += s sum_c O D_ik[a][c]
          const int b = i / g.nd, d = i - b * g.nd;
          double v = 0.0;
          for (int c = 0; c < g.nc; ++c) v += O[b * ncd + c * g.nd + d] * Dik[a * g.nc + c];
          Ajl[i] += v;
        }
      }
      __syncwarp();
    }
    if (args.mode == MODE_JK) {
      const int nbf = args.nbf;
      for (int i = lane; i < ncd; i += 32) {
        const int c = i / g.nd, d = i - c * g.nd;
        atomicAdd(args.J + (size_t)(fc + c) * nbf + fd + d, 2.0 * sym * Akl[i]);
      }
      for (int i = lane; i < g.nb * g.nc; i += 32) {
        const int b = i / g.nc, c = i - b * g.nc;
        atomicAdd(args.K + (size_t)(fb + b) * nbf + fc + c, sym * Ajk[i]);
      }
      for (int i = lane; i < g.nb * g.nd; i += 32) {
        const int b = i / g.nd, d = i - b * g.nd;
        atomicAdd(args.K + (size_t)(fb + b) * nbf + fd + d, sym * Ajl[i]);
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
  const size_t smem = (size_t)g.per_warp * 8 * warps;
  // enough warps to cover the SMs several times; grid-stride inside
  int64_t want = (blk.total - blk.t_begin + warps - 1) / warps;
  int64_t cap = (int64_t)num_sms * 16;
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
    cudaFuncSetAttribute(eri_generic_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem_max);
    attr_set = true;
  }
  eri_generic_kernel<<<grid, warps * 32, smem, stream>>>(blk, args, tab, g, gscratch);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

size_t generic_global_scratch_doubles(int la, int lb, int lc, int ld, int num_sms) {
  GenericGeom g = make_geom(la, lb, lc, ld, 227 * 1024, 4);
  int warps = 4;
  if (g.per_warp < 0) { warps = 1; g = make_geom(la, lb, lc, ld, 227 * 1024, 1); }
  if (g.per_warp < 0 || !g.G_in_global) return 0;
  return (size_t)num_sms * 16 * warps * g.NEF;
}

}  // namespace lai
