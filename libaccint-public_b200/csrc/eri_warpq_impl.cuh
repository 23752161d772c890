// Warp-per-quartet Rys ERI kernel, compile-time specialised per class, for the
// mid-size classes: (dd|pp), (dd|dp), (dd|dd), the d/f classes of triple-zeta
// bases -- every class whose contracted (e0|f0) block has at most kWarpqMaxG
// integrals.  J/K digestion only (the raw-integral and Schwarz modes stay on the
// tiled kernel).
//
// Per quartet (one warp), for every primitive quartet:
//   1. lanes t < 3n (n Rys roots) own (root r = t/3, direction x = t%3): the root,
//      then the 2D table I_x(e, f), e <= la+lb, f <= lc+ld, by the vertical
//      recurrence of eri_device.cuh in registers (compile-time indices), stored to
//      shared memory; the z table carries w_r * prefactor;
//   2. every lane owns the (e0|f0) integrals j = lane + 32 m of the contracted block
//      G[e][f] (e over the Cartesian components of shells la..la+lb, f of lc..lc+ld)
//      and adds sum_r Ix Iy Iz to them in registers.
// After the last primitive quartet, once per contracted quartet: G goes to shared
// memory, the horizontal transfer in closed form (binomial sums, the same transfer
// as eri_device.cuh; the terms of every component, their integer coefficients and
// target indices are tabulated per class in shared memory when the block starts,
// and the quartet's AB/CD powers once per quartet) gives first (ab|f0] and then
// (ab|cd), which is normalized and
// digested by the lanes into the six Fock blocks (lane-owned sums, no shared-memory
// atomics).  J'_ab accumulates in shared memory while consecutive quartets of the
// warp keep their bra pair and goes to global memory once per bra pair; the other
// five blocks take one global atomic per element and quartet.
//
// Compared with the tiled kernel, the transfer runs once per contracted quartet
// instead of once per primitive quartet and root, the per-primitive work is
// compile-time unrolled, and the contraction needs three shared-memory loads per
// (e0|f0) integral and root.  The reference counterparts are the same as the tiled
// kernel's (src/device/cuda/kernels/eri_kernel_warp.cu:140-344 plus the separate
// fock_accumulate_batch_kernel).
#pragma once

#include <cuda_runtime.h>

#include "eri_device.cuh"
#include "eri_kernels.h"

namespace lai {

constexpr int kWarpqMaxG = 1152;    // (e0|f0) integrals per quartet: 36 per lane
constexpr int kWarpqWarps = 4;      // warps per block

__host__ __device__ constexpr int warpq_max(int a, int b) { return a > b ? a : b; }
// most terms prod_x (b_x + 1) of a component of shell l
__host__ __device__ constexpr int warpq_max_terms(int l) {
  int m = 1;
  for (int x = l; x >= 0; --x)
    for (int y = l - x; y >= 0; --y) {
      const int t = (x + 1) * (y + 1) * (l - x - y + 1);
      m = t > m ? t : m;
    }
  return m;
}

template <int LA, int LB, int LC, int LD>
struct WarpqClass {
  static constexpr int LAB = LA + LB, LCD = LC + LD;
  static constexpr int NR = (LAB + LCD) / 2 + 1;
  static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  static constexpr int NE = ncart_range(LA, LAB), NF = ncart_range(LC, LCD);
  static constexpr int NG = NE * NF, MG = (NG + 31) / 32;
  static constexpr int W = LCD + 1, VS = (LAB + 1) * W;
  static constexpr int NAB = NA * NB, NCD = NC * ND;
  static constexpr int NX = NAB * NF, NO = NAB * NCD;
  static constexpr int NACC = NAB + NCD + NA * NC + NA * ND + NB * NC + NB * ND;
  // per-warp shared memory (doubles): root tables, two block buffers, density
  // sub-blocks, the running J'_ab of the current bra pair
  static constexpr int S_V = NR * 3 * VS;
  static constexpr int S_BUF = warpq_max(NG, warpq_max(NX, NO));
  static constexpr int OFF_B0 = S_V, OFF_B1 = OFF_B0 + S_BUF, OFF_D = OFF_B1 + S_BUF;
  static constexpr int OFF_JAB = OFF_D + NACC;
  // transfer terms: a shell-b component takes prod_x (b_x + 1) terms k <= b
  static constexpr int MTB = warpq_max_terms(LB), MTD = warpq_max_terms(LD);
  static constexpr int OFF_CB = OFF_JAB + NAB, OFF_CD = OFF_CB + NB * MTB;
  static constexpr int PER_WARP = ((OFF_CD + ND * MTD) + 1) & ~1;
  // blocks per SM the register allocation targets: the warp's latency (dependent
  // global loads, warp syncs) is hidden by other warps, so the small classes are
  // held to few registers (estimate: G, its offsets, one lane's 2D table, ~40 more)
  static constexpr int REG_EST = 3 * MG + 2 * VS + 40;
  static constexpr int MIN_BLOCKS = REG_EST <= 64 ? 8 : REG_EST <= 80 ? 6 : REG_EST <= 96 ? 5
                                    : REG_EST <= 128 ? 4 : REG_EST <= 168 ? 3 : 2;
};

// The CUDA error of the last failed launch (cudaGetLastError clears it).
inline cudaError_t& warpq_last_error() {
  static thread_local cudaError_t e = cudaSuccess;
  return e;
}

__device__ __forceinline__ int warpq_binom(int n, int k) {
  int r = 1;
  for (int i = 0; i < k; ++i) r = r * (n - i) / (i + 1);
  return r;
}

__device__ __forceinline__ double warpq_pow(double x, int m) {
  double r = 1.0;
  for (int i = 0; i < m; ++i) r *= x;
  return r;
}

// R = double: the whole quartet in FP64.  R = float (the FP32 part of a mixed
// build, d and f classes): roots, 2D tables and the (e0|f0) accumulation in FP32
// (the tables take half the shared memory and its bandwidth); the primitive-pair
// quantities up to T and the prefactor, the transfer, normalization and digestion
// stay FP64.
template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(kWarpqWarps * 32, (WarpqClass<LA, LB, LC, LD>::MIN_BLOCKS)) eri_warpq_kernel(QuartetBlock blk, JKArgs args,
                                                                     RysTablesView tab) {
  using C = WarpqClass<LA, LB, LC, LD>;
  constexpr int NR = C::NR, W = C::W, VS = C::VS, MG = C::MG, NF = C::NF;
  constexpr int NA = C::NA, NB = C::NB, NC = C::NC, ND = C::ND, NCD = C::NCD, NAB = C::NAB;
  constexpr int LAB = C::LAB, LCD = C::LCD;
  extern __shared__ __align__(16) double smem_q[];
  // Cartesian components (packed lx | ly << 4 | lz << 8) and normalization factors
  // of the four shells
  __shared__ int s_comp[4][kNCartMax];
  __shared__ double s_norm[4][kNCartMax];
  for (int i = threadIdx.x; i < 4 * kNCartMax; i += blockDim.x) {
    const int sh = i / kNCartMax, k = i - sh * kNCartMax;
    const int l = sh == 0 ? LA : sh == 1 ? LB : sh == 2 ? LC : LD;
    if (k < ncart(l)) {
      s_comp[sh][k] = cart_comp(l, k);
      s_norm[sh][k] = norm_factor(l, k);
    }
  }
  // transfer tables of the class: for bra component b, term t < s_bn[b] is the
  // shift k <= b with integer coefficient prod_x C(b_x, k_x) (s_bc) and powers
  // b - k of AB (s_bp, 4 bits each); s_be[a][b][t] is the (e0| index of a + k.
  // The same for the ket (d, c, CD).
  constexpr int MTB = C::MTB, MTD = C::MTD;
  __shared__ int s_bn[NB], s_bc[NB * MTB], s_bp[NB * MTB], s_be[NAB * MTB];
  __shared__ int s_dn[ND], s_dc[ND * MTD], s_dp[ND * MTD], s_df[NC * ND * MTD];
  for (int i = threadIdx.x; i < NAB + NC * ND; i += blockDim.x) {
    const bool bra = i < NAB;
    const int u = bra ? i / NB : (i - NAB) / ND;      // a (or c)
    const int v = bra ? i % NB : (i - NAB) % ND;      // b (or d)
    const int lu = bra ? LA : LC, lv = bra ? LB : LD;
    const int cu = cart_comp(lu, u), cv = cart_comp(lv, v);
    const int vx = comp_x(cv), vy = comp_y(cv), vz = comp_z(cv);
    int t = 0;
    for (int kx = 0; kx <= vx; ++kx)
      for (int ky = 0; ky <= vy; ++ky)
        for (int kz = 0; kz <= vz; ++kz, ++t) {
          const int l = lu + kx + ky + kz;
          const int e = ncart_before(lu, l) + cart_index(comp_x(cu) + kx, comp_y(cu) + ky, comp_z(cu) + kz);
          if (bra) {
            s_be[i * MTB + t] = e;
            if (u == 0) {
              s_bc[v * MTB + t] = warpq_binom(vx, kx) * warpq_binom(vy, ky) * warpq_binom(vz, kz);
              s_bp[v * MTB + t] = (vx - kx) | ((vy - ky) << 4) | ((vz - kz) << 8);
            }
          } else {
            s_df[(i - NAB) * MTD + t] = e;
            if (u == 0) {
              s_dc[v * MTD + t] = warpq_binom(vx, kx) * warpq_binom(vy, ky) * warpq_binom(vz, kz);
              s_dp[v * MTD + t] = (vx - kx) | ((vy - ky) << 4) | ((vz - kz) << 8);
            }
          }
        }
    if (u == 0) {
      // unused terms: coefficient 0, no powers (every entry of the tables is read
      // when a quartet's coefficients are formed)
      for (int r = t; r < (bra ? MTB : MTD); ++r) {
        if (bra) {
          s_bc[v * MTB + r] = 0;
          s_bp[v * MTB + r] = 0;
        } else {
          s_dc[v * MTD + r] = 0;
          s_dp[v * MTD + r] = 0;
        }
      }
      if (bra) s_bn[v] = t;
      else s_dn[v] = t;
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  double* const Vs = smem_q + (size_t)warp * C::PER_WARP;
  double* const CoB = Vs + C::OFF_CB;   // per quartet: coefficient of bra term (b, t)
  double* const CoD = Vs + C::OFF_CD;   // per quartet: coefficient of ket term (d, t)
  double* const B0 = Vs + C::OFF_B0;
  double* const B1 = Vs + C::OFF_B1;
  double* const Ds = Vs + C::OFF_D;
  double* const Jab = Vs + C::OFF_JAB;
  constexpr int oDab = 0, oDcd = NAB, oDac = oDcd + NCD, oDad = oDac + NA * NC, oDbc = oDad + NA * ND,
                oDbd = oDbc + NB * NC;

  // this lane's (e0|f0) integrals: packed byte offsets of Ix, Iy, Iz inside one
  // direction's table (10 bits each); entries past the block read I(0,0) and are
  // never written out
  int goff[MG];
#pragma unroll
  for (int m = 0; m < MG; ++m) {
    const int j = lane + 32 * m;
    int o = 0;
    if (j < C::NG) {
      const int e = j / NF, f = j - e * NF;
      int le = LA, re = e;
      while (re >= ncart(le)) re -= ncart(le++);
      int lf = LC, rf = f;
      while (rf >= ncart(lf)) rf -= ncart(lf++);
      const int ce = cart_comp(le, re), cf = cart_comp(lf, rf);
      const int ox = comp_x(ce) * W + comp_x(cf), oy = comp_y(ce) * W + comp_y(cf),
                oz = comp_z(ce) * W + comp_z(cf);
      constexpr int sz = sizeof(R);
      o = (ox * sz) | ((oy * sz) << 10) | ((oz * sz) << 20);
    }
    goff[m] = o;
  }

  const int nbra = blk.bra.npairs, nket = blk.ket.npairs;
  const int Kab = blk.bra.Ka * blk.bra.Kb, Kcd = blk.ket.Ka * blk.ket.Kb;
  (void)nbra; (void)nket;

  const int64_t gw = (int64_t)blockIdx.x * kWarpqWarps + warp;
  const int64_t nw = (int64_t)gridDim.x * kWarpqWarps;
  const int64_t nq_all = blk.total - blk.t_begin;
  const int64_t per = (nq_all + nw - 1) / nw;
  const int64_t tbeg = blk.t_begin + gw * per;
  const int64_t tend = min(blk.total, tbeg + per);
  int p = -1;
  int jab_p = -1;             // bra pair whose J'_ab is accumulating in Jab
  int jab_fa = 0, jab_fb = 0;
  double* jab_J = nullptr;
  size_t jab_n = 0;
  unsigned int nprim_done = 0;
  for (int i = lane; i < NAB; i += 32) Jab[i] = 0.0;

  for (int64_t t = tbeg; t < tend; ++t) {
    if (p < 0) {
      if (lane == 0) p = find_bra(blk.offsets, nbra, t);
      p = __shfl_sync(0xffffffffu, p, 0);
    } else {
      while (t >= __ldg(blk.offsets + p + 1)) ++p;
    }
    const int q = (blk.qbegin ? __ldg(blk.qbegin + p) : 0) + (int)(t - __ldg(blk.offsets + p));
    const int fa = __ldg(blk.bra.func_a + p), fb = __ldg(blk.bra.func_b + p);
    const int fc = __ldg(blk.ket.func_a + q), fd = __ldg(blk.ket.func_b + q);
    const double sym = quartet_weight(blk, p, q);
    const SysMats mats = sys_mats(args, blk, p);
    const size_t n = (size_t)mats.nbf;
    if (p != jab_p) {  // flush the finished bra pair's J'_ab
      __syncwarp();
      if (jab_p >= 0)
        for (int i = lane; i < NAB; i += 32) {
          const double v = Jab[i];
          if (v != 0.0) atomicAdd(jab_J + (size_t)(jab_fa + i / NB) * jab_n + jab_fb + i % NB, v);
          Jab[i] = 0.0;
        }
      jab_p = p;
      jab_fa = fa;
      jab_fb = fb;
      jab_J = mats.J;
      jab_n = n;
    }
    // density sub-blocks of the six scatter targets
    for (int i = lane; i < C::NACC; i += 32) {
      int r0, c0, c1, k;
      if (i < oDcd) { k = i; r0 = fa; c0 = fb; c1 = NB; }
      else if (i < oDac) { k = i - oDcd; r0 = fc; c0 = fd; c1 = ND; }
      else if (i < oDad) { k = i - oDac; r0 = fa; c0 = fc; c1 = NC; }
      else if (i < oDbc) { k = i - oDad; r0 = fa; c0 = fd; c1 = ND; }
      else if (i < oDbd) { k = i - oDbc; r0 = fb; c0 = fc; c1 = NC; }
      else { k = i - oDbd; r0 = fb; c0 = fd; c1 = ND; }
      Ds[i] = __ldg(mats.D + (size_t)(r0 + k / c1) * n + c0 + k % c1);
    }

    R G[MG];
#pragma unroll
    for (int m = 0; m < MG; ++m) G[m] = R(0);

    // the whole warp works on one quartet: bra and ket primitives come from their
    // per-pair records (a few contiguous lines per pair, 16-byte loads)
    const double2* rbp = reinterpret_cast<const double2*>(blk.bra.primb + (size_t)p * Kab * kBraRec);
    const double2* rkp = reinterpret_cast<const double2*>(blk.ket.primb + (size_t)q * Kcd * kBraRec);
    for (int ib = 0; ib < Kab; ++ib) {
      const double2* rb = rbp + ib * (kBraRec / 2);
      const double2 b0 = __ldg(rb), b1 = __ldg(rb + 1);
      const double qab = b0.x;
      if (qab * blk.ket.qprim_max < args.prim_eps) break;
      const double2 b2 = __ldg(rb + 2), b3 = __ldg(rb + 3), b4 = __ldg(rb + 4), b5 = __ldg(rb + 5);
      const double zeta = b0.y, hz = b1.x, cab = b1.y;
      const double Px = b2.x, Py = b2.y, Pz = b3.x;
      const double PAx = b4.x, PAy = b4.y, PAz = b5.x;
      for (int ik = 0; ik < Kcd; ++ik) {
        const double2* rk = rkp + ik * (kBraRec / 2);
        const double2 k0 = __ldg(rk);
        const double qcd = k0.x;
        if (qab * qcd < args.prim_eps) break;
        ++nprim_done;
        const double2 k1 = __ldg(rk + 1), k2 = __ldg(rk + 2), k3 = __ldg(rk + 3);
        const double eta = k0.y, he = k1.x, ccd = k1.y;
        const double PQx = Px - k2.x, PQy = Py - k2.y, PQz = Pz - k3.x;
        const double* pkr = reinterpret_cast<const double*>(rk);
        const double rs = rsqrt(zeta + eta);
        const double inv = rs * rs;
        const double rz = eta * inv, re = zeta * inv;
        const double T = zeta * rz * (PQx * PQx + PQy * PQy + PQz * PQz);
        const double pref = cab * ccd * rs;
        if (lane < 3 * NR) {
          const int r = lane / 3, x = lane - 3 * r;
          R u, w;
          rys_root_one<R>(NR, r, R(T), tab, u, w);
          const R pqx = R(x == 0 ? PQx : x == 1 ? PQy : PQz);
          const R pax = R(x == 0 ? PAx : x == 1 ? PAy : PAz);
          const R qcx = R(__ldg(pkr + BR_PAX + x));
          const R rzr = R(rz), rer = R(re);
          const R pa = pax - rzr * u * pqx;
          const R qc = qcx + rer * u * pqx;
          const R b00 = R(0.5) * R(inv) * u, b10 = R(hz) - R(hz) * rzr * u, b01 = R(he) - R(he) * rer * u;
          R V[LAB + 1][W];
          V[0][0] = (x == 2) ? w * R(pref) : R(1);
#pragma unroll
          for (int e = 0; e < LAB; ++e)
            V[e + 1][0] = pa * V[e][0] + (e ? R(e) * b10 * V[e > 0 ? e - 1 : 0][0] : R(0));
#pragma unroll
          for (int f = 0; f < LCD; ++f)
#pragma unroll
            for (int e = 0; e <= LAB; ++e)
              V[e][f + 1] = qc * V[e][f] + (f ? R(f) * b01 * V[e][f > 0 ? f - 1 : 0] : R(0)) +
                            (e ? R(e) * b00 * V[e > 0 ? e - 1 : 0][f] : R(0));
          R* dst = reinterpret_cast<R*>(Vs) + (r * 3 + x) * VS;
#pragma unroll
          for (int e = 0; e <= LAB; ++e)
#pragma unroll
            for (int f = 0; f < W; ++f) dst[e * W + f] = V[e][f];
        }
        __syncwarp();
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const char* vx = reinterpret_cast<const char*>(reinterpret_cast<const R*>(Vs) + (r * 3) * VS);
          const char* vy = vx + VS * sizeof(R);
          const char* vz = vy + VS * sizeof(R);
#pragma unroll
          for (int m = 0; m < MG; ++m) {
            const int o = goff[m];
            G[m] += *reinterpret_cast<const R*>(vx + (o & 1023)) *
                    *reinterpret_cast<const R*>(vy + ((o >> 10) & 1023)) *
                    *reinterpret_cast<const R*>(vz + (o >> 20));
          }
        }
        __syncwarp();
      }
    }

    // ---- once per contracted quartet: transfer, normalization, digestion ----
#pragma unroll
    for (int m = 0; m < MG; ++m) {
      const int j = lane + 32 * m;
      if (j < C::NG) B0[j] = double(G[m]);
    }
    const double ABx = __ldg(blk.bra.AB + p), ABy = __ldg(blk.bra.AB + nbra + p),
                 ABz = __ldg(blk.bra.AB + 2 * nbra + p);
    const double CDx = __ldg(blk.ket.AB + q), CDy = __ldg(blk.ket.AB + nket + q),
                 CDz = __ldg(blk.ket.AB + 2 * nket + q);
    __syncwarp();
    // this quartet's transfer coefficients C(b, k) AB^(b-k) and C(d, k) CD^(d-k)
    for (int i = lane; i < NB * MTB + ND * MTD; i += 32) {
      const bool bra = i < NB * MTB;
      const int k = bra ? i : i - NB * MTB;
      const int pk = bra ? s_bp[k] : s_dp[k];
      const double cx = bra ? ABx : CDx, cy = bra ? ABy : CDy, cz = bra ? ABz : CDz;
      double v = bra ? (double)s_bc[k] : (double)s_dc[k];
      v *= warpq_pow(cx, pk & 15) * warpq_pow(cy, (pk >> 4) & 15) * warpq_pow(cz, (pk >> 8) & 15);
      (bra ? CoB : CoD)[k] = v;
    }
    __syncwarp();
    // bra transfer: (ab|f0] = sum_k prod_x C(b_x, k_x) AB_x^(b_x - k_x) (a+k 0|f0]
    for (int j = lane; j < C::NX; j += 32) {
      const int ab = j / NF, f = j - ab * NF;
      const int b = ab % NB;
      const int nt = s_bn[b];
      const int* ei = s_be + ab * MTB;
      const double* co = CoB + b * MTB;
      double s = 0.0;
#pragma unroll
      for (int t = 0; t < MTB; ++t)
        if (t < nt) s += co[t] * B0[ei[t] * NF + f];
      B1[j] = s;
    }
    __syncwarp();
    // ket transfer and normalization: (ab|cd) into B0[ab][c][d]
    for (int j = lane; j < C::NO; j += 32) {
      const int ab = j / NCD, cd = j - ab * NCD;
      const int d = cd % ND;
      const int nt = s_dn[d];
      const int* fi = s_df + cd * MTD;
      const double* co = CoD + d * MTD;
      const double* row = B1 + ab * NF;
      double s = 0.0;
#pragma unroll
      for (int t = 0; t < MTD; ++t)
        if (t < nt) s += co[t] * row[fi[t]];
      const int a = ab / NB, b = ab - a * NB, c = cd / ND;
      B0[j] = s * s_norm[0][a] * s_norm[1][b] * s_norm[2][c] * s_norm[3][d];
    }
    __syncwarp();
    // digestion: every lane owns whole Fock elements; J'_ab = 2s sum_cd V D_cd,
    // J'_cd = 2s sum_ab V D_ab, K'_ac = s sum_bd V D_bd, K'_ad = s sum_bc V D_bc,
    // K'_bc = s sum_ad V D_ad, K'_bd = s sum_ac V D_ac
    const double* O = B0;
    for (int i = lane; i < C::NACC; i += 32) {
      double acc = 0.0;
      if (i < oDcd) {
        const double* row = O + i * NCD;
#pragma unroll 4
        for (int cd = 0; cd < NCD; ++cd) acc += row[cd] * Ds[oDcd + cd];
        Jab[i] += 2.0 * sym * acc;
        continue;
      }
      int r0, c0, c1, k;
      double* M;
      if (i < oDac) {
        k = i - oDcd;
#pragma unroll 4
        for (int ab = 0; ab < NAB; ++ab) acc += O[ab * NCD + k] * Ds[oDab + ab];
        acc *= 2.0 * sym;
        r0 = fc; c0 = fd; c1 = ND; M = mats.J;
      } else if (i < oDad) {
        k = i - oDac;
        const int a = k / NC, c = k - a * NC;
        for (int b = 0; b < NB; ++b)
          for (int d = 0; d < ND; ++d) acc += O[((a * NB + b) * NC + c) * ND + d] * Ds[oDbd + b * ND + d];
        acc *= sym;
        r0 = fa; c0 = fc; c1 = NC; M = mats.K;
      } else if (i < oDbc) {
        k = i - oDad;
        const int a = k / ND, d = k - a * ND;
        for (int b = 0; b < NB; ++b)
          for (int c = 0; c < NC; ++c) acc += O[((a * NB + b) * NC + c) * ND + d] * Ds[oDbc + b * NC + c];
        acc *= sym;
        r0 = fa; c0 = fd; c1 = ND; M = mats.K;
      } else if (i < oDbd) {
        k = i - oDbc;
        const int b = k / NC, c = k - b * NC;
        for (int a = 0; a < NA; ++a)
          for (int d = 0; d < ND; ++d) acc += O[((a * NB + b) * NC + c) * ND + d] * Ds[oDad + a * ND + d];
        acc *= sym;
        r0 = fb; c0 = fc; c1 = NC; M = mats.K;
      } else {
        k = i - oDbd;
        const int b = k / ND, d = k - b * ND;
        for (int a = 0; a < NA; ++a)
          for (int c = 0; c < NC; ++c) acc += O[((a * NB + b) * NC + c) * ND + d] * Ds[oDac + a * NC + c];
        acc *= sym;
        r0 = fb; c0 = fd; c1 = ND; M = mats.K;
      }
      if (acc != 0.0) atomicAdd(M + (size_t)(r0 + k / c1) * n + c0 + k % c1, acc);
    }
    __syncwarp();
  }
  // the last bra pair's J'_ab
  __syncwarp();
  if (jab_p >= 0)
    for (int i = lane; i < NAB; i += 32) {
      const double v = Jab[i];
      if (v != 0.0) atomicAdd(jab_J + (size_t)(jab_fa + i / NB) * jab_n + jab_fb + i % NB, v);
    }
  count_prims(args.prim_count, lane == 0 ? nprim_done : 0u);
}

// Host side: per-warp shared memory of class (la, lb, lc, ld), or -1 when the
// class is not instantiated.
template <int LA, int LB, int LC, int LD, typename R>
int launch_warpq_typed(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab,
                       cudaStream_t stream, int num_sms) {
  using C = WarpqClass<LA, LB, LC, LD>;
  const size_t smem = (size_t)C::PER_WARP * 8 * kWarpqWarps;
  static int per_sm = -1;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(eri_warpq_kernel<LA, LB, LC, LD, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return -3;
  if (per_sm < 0) {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, eri_warpq_kernel<LA, LB, LC, LD, R>, kWarpqWarps * 32,
                                                      smem) != cudaSuccess)
      return -3;
    if (b <= 0) return -1;  // does not fit: the tiled kernel takes the class
    per_sm = b;
  }
  const int64_t want = (blk.total - blk.t_begin + kWarpqWarps - 1) / kWarpqWarps;
  const int64_t cap = (int64_t)num_sms * per_sm;
  const int grid = (int)std::min<int64_t>(want, cap);
  eri_warpq_kernel<LA, LB, LC, LD, R><<<grid, kWarpqWarps * 32, smem, stream>>>(blk, args, tab);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    warpq_last_error() = e;
    return -3;
  }
  return 0;
}

// FP32 = the units instantiating an FP32 variant (d and f classes); fp32 asks for
// it (returns 1 when the FP32 kernel ran, 0 for FP64, <0 as launch_warpq).
template <int LA, int LB, int LC, int LD, bool FP32>
int launch_warpq_cls(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab,
                     cudaStream_t stream, int num_sms, bool fp32) {
  if constexpr (FP32) {
    if (fp32) {
      const int rc = launch_warpq_typed<LA, LB, LC, LD, float>(blk, args, tab, stream, num_sms);
      return rc == 0 ? 1 : rc;
    }
  }
  return launch_warpq_typed<LA, LB, LC, LD, double>(blk, args, tab, stream, num_sms);
}

}  // namespace lai
