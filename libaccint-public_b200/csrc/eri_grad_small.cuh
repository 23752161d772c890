// Nuclear gradient of E = 1/2 tr(D J[D]) - 1/4 tr(D K[D]) for the low angular
// momentum classes: one thread per canonical quartet, everything in registers,
// compile-time specialised on (la,lb|lc,ld) and on the derivative centre.
//
// Same mathematics as eri_grad.cu (d/dA_x phi_a = 2 alpha phi_{a+1x} - a_x
// phi_{a-1x}, the D centre by translational invariance), arranged like the J/K
// kernels: the primitive loop only accumulates contracted (e0|f0)-type blocks,
//   W[e][f] = sum_prim 2 kappa sum_r w_r pref Ix Iy Iz  over the raised shells,
//   U[e][f] = sum_prim       sum_r w_r pref Ix Iy Iz    over the lowered shells,
// (kappa = alpha, beta or gamma, the exponent on the derivative centre), and the
// horizontal transfer (closed binomial form, the exact A-B and C-D) and the
// contraction with G_abcd = s n_a n_b n_c n_d (4 D_ab D_cd - D_ac D_bd - D_ad D_bc)
// run once per contracted quartet.  Each pass adds its centres' derivatives and
// subtracts them from the D centre; how many passes a class takes depends on how
// many accumulators fit in registers: all three centres in one pass (the
// smallest classes), A and B in one pass and C in a second, or one per centre.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "eri_device.cuh"
#include "eri_kernels.h"
#include "eri_tables_smem.cuh"

namespace lai {
namespace grad_small {

enum { DA = 0, DB = 1, DC = 2, DAB = 3, DABC = 4, DB_LO = 5, DB_HI = 6 };
// DAB: A and B in one pass; DABC: all three.  DB_LO / DB_HI: the B pass in two halves
// that accumulate the raised and lowered blocks only for the ket's lowest shell
// (f = lc) / the ones above it; the gradient is linear in those blocks, so the two
// halves add up to the B pass while each holds about half its accumulators.

template <int B, int E, typename F>
__device__ __forceinline__ void gfor(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    gfor<B + 1, E>(f);
  }
}

// Index of Cartesian component (x, y, z) inside the component list of shells
// lo..(x+y+z) (the (e0|f0) block layout of the J/K kernels).
__host__ __device__ constexpr int eidx(int lo, int x, int y, int z) {
  return ncart_before(lo, x + y + z) + cart_index(x, y, z);
}

struct GradSmallArgs {
  const double* D;
  int nbf;
  const int* shell_atom;
  double* grad;
  double prim_eps;
};

// Sum over the horizontal-transfer terms of one side: (a b| = sum_{k <= b}
// prod_x C(b_x, k_x) AB_x^(b_x - k_x) (a+k 0|, with a, b packed components.
// f(e_index, coefficient) is called for every term (the index as an integral
// constant, so that the accumulator blocks stay in registers).
template <int CA, int CB, int E0, typename P, typename F>
__device__ __forceinline__ void hrr_terms(const P& abp, F&& f) {
  gfor<0, comp_x(CB) + 1>([&](auto KX) {
    constexpr int kx = decltype(KX)::value;
    gfor<0, comp_y(CB) + 1>([&](auto KY) {
      constexpr int ky = decltype(KY)::value;
      gfor<0, comp_z(CB) + 1>([&](auto KZ) {
        constexpr int kz = decltype(KZ)::value;
        constexpr int e = eidx(E0, comp_x(CA) + kx, comp_y(CA) + ky, comp_z(CA) + kz);
        constexpr double bc = binom(comp_x(CB), kx) * binom(comp_y(CB), ky) * binom(comp_z(CB), kz);
        f(std::integral_constant<int, e>{},
          bc * abp[0][comp_x(CB) - kx] * abp[1][comp_y(CB) - ky] * abp[2][comp_z(CB) - kz]);
      });
    });
  });
}

constexpr int pack(int x, int y, int z) { return x | (y << 4) | (z << 8); }
constexpr int shift(int c, int x, int d) {  // component c with d added in direction x
  return pack(comp_x(c) + (x == 0 ? d : 0), comp_y(c) + (x == 1 ? d : 0), comp_z(c) + (x == 2 ? d : 0));
}
constexpr int comp_n(int c, int x) { return x == 0 ? comp_x(c) : x == 1 ? comp_y(c) : comp_z(c); }

// whether a pass accumulates the raised / lowered block entries of ket shell lf
template <int PASS, int LC>
__host__ __device__ constexpr bool f_in_pass(int lf) {
  return PASS == DB_LO ? lf == LC : PASS == DB_HI ? lf > LC : true;
}

template <int LA, int LB, int LC, int LD, int PASS>
__global__ void __launch_bounds__(128) grad_small_kernel(QuartetBlock blk, GradSmallArgs ga, RysTablesView tab) {
  constexpr int DER = (PASS == DB_LO || PASS == DB_HI) ? DB : PASS;
  constexpr int LAB = LA + LB, LCD = LC + LD;
  constexpr int NR = (LAB + LCD + 1) / 2 + 1;
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  // raised block W (W2: the B block of a merged A+B pass) and lowered block U, as
  // shell ranges [E0, E1] x [F0, F1]
  // ABC_: all three centres in one pass (W: A, W2: B, W3: C); AB_: A and B
  constexpr bool ABC_ = DER == DABC;
  constexpr bool AB_ = DER == DAB || ABC_;
  constexpr int WE0 = (DER == DA || AB_) ? LA + 1 : LA, WE1 = DER == DC ? LAB : LAB + 1;
  constexpr int WF0 = DER == DC ? LC + 1 : LC, WF1 = DER == DC ? LCD + 1 : LCD;
  constexpr bool HAS_U = DER == DA ? LA >= 1 : DER == DB ? LB >= 1 : DER == DC ? LC >= 1
                         : DER == DAB ? (LA >= 1 || LB >= 1) : (LA >= 1 || LB >= 1 || LC >= 1);
  // the lowered block: one rectangle covering the lowered ranges of the pass's centres
  constexpr int UE0 = (DER == DA || AB_) ? (LA >= 1 ? LA - 1 : 0) : LA;
  constexpr int UE1 = (DER == DC || (ABC_ && LC >= 1)) ? LAB : LAB - 1;
  constexpr int UF0 = (DER == DC || ABC_) ? (LC >= 1 ? LC - 1 : 0) : LC;
  constexpr int UF1 = DER == DC ? LCD - 1 : LCD;
  constexpr int NWE = ncart_range(WE0, WE1), NWF = ncart_range(WF0, WF1);
  constexpr int NW2E = AB_ ? ncart_range(LA, LAB + 1) : 1;  // W2: e in [LA, LAB+1], f as W
  constexpr int NW3E = ABC_ ? ncart_range(LA, LAB) : 1;     // W3: e in [LA, LAB], f in [LC+1, LCD+1]
  constexpr int NW3F = ABC_ ? ncart_range(LC + 1, LCD + 1) : 1;
  constexpr int NUE = HAS_U ? ncart_range(UE0, UE1) : 1, NUF = HAS_U ? ncart_range(UF0, UF1) : 1;
  constexpr int EM = DER == DC ? LAB : LAB + 1;  // vertical recurrence extents
  constexpr int FM = (DER == DC || ABC_) ? LCD + 1 : LCD;

  // the Boys grid / the Rys fit table of NR roots, staged once per block (per-lane
  // gathers from global memory would touch up to 32 lines per load)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* stab = reinterpret_cast<double*>(smem_raw);
  stage_table<NR, double>(stab, tab);
  __syncthreads();
  const int nbra = blk.bra.npairs, nket = blk.ket.npairs;
  const int Kab = blk.bra.Ka * blk.bra.Kb, Kcd = blk.ket.Ka * blk.ket.Kb;
  const size_t sb = (size_t)Kab * nbra;
  // warps take chunks of 32 consecutive quartets (grid-stride); one bra search per
  // chunk, then each lane steps forward to its own bra pair (usually the same)
  const int lane = threadIdx.x & 31;
  const int64_t nq = blk.total - blk.t_begin;
  const int64_t nchunks = (nq + 31) / 32;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t ch = wid; ch < nchunks; ch += nw) {
    const int64_t t0 = blk.t_begin + ch * 32;
    const int64_t t = t0 + lane;
    int pw = 0;
    if (lane == 0) pw = find_bra(blk.offsets, nbra, t0);
    pw = __shfl_sync(0xffffffffu, pw, 0);
    if (t >= blk.total) continue;
    int p = pw;
    while (t >= __ldg(blk.offsets + p + 1)) ++p;
    const int q = (blk.qbegin ? __ldg(blk.qbegin + p) : 0) + (int)(t - __ldg(blk.offsets + p));
    const double* __restrict__ pkt = ket_tile_ptr(blk.ket.primk, q, Kcd);
    double W[NWE * NWF], W2[AB_ ? NW2E * NWF : 1], W3[NW3E * NW3F], U[NUE * NUF];
#pragma unroll
    for (int i = 0; i < NW3E * NW3F; ++i) W3[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NWE * NWF; ++i) W[i] = 0.0;
#pragma unroll
    for (int i = 0; i < (AB_ ? NW2E * NWF : 1); ++i) W2[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NUE * NUF; ++i) U[i] = 0.0;

    for (int ib = 0; ib < Kab; ++ib) {
      // bra primitive: its per-pair record (the warp usually shares the bra pair);
      // the exponent on A from the SoA table
      const double2* rb = reinterpret_cast<const double2*>(blk.bra.primb + ((size_t)p * Kab + ib) * kBraRec);
      const double2 b0 = __ldg(rb), b1 = __ldg(rb + 1);
      const double qab = b0.x;
      if (qab * blk.ket.qprim_max < ga.prim_eps) break;
      const double2 b2 = __ldg(rb + 2), b3 = __ldg(rb + 3), b4 = __ldg(rb + 4), b5 = __ldg(rb + 5);
      const double zeta = b0.y, hz = b1.x, cab = b1.y;
      const double alpha = DER != DC ? __ldg(blk.bra.prim + (size_t)ib * nbra + p + PF_ALPHA * sb) : 0.0;
      const double P[3] = {b2.x, b2.y, b3.x};
      const double PA[3] = {b4.x, b4.y, b5.x};
      for (int ik = 0; ik < Kcd; ++ik) {
        // ket primitive ik of pair q in the ket tiles (fields at fixed offsets)
        const double* pk = pkt + (size_t)ik * kKetPrimStride;
        const double qcd = __ldg(pk + KR_Q * kKetTile);
        if (qab * qcd < ga.prim_eps) break;
        const double eta = __ldg(pk + KR_ETA * kKetTile), he = __ldg(pk + KR_HE * kKetTile);
        const double gamma = (DER == DC || ABC_) ? __ldg(pk + KR_ALPHA * kKetTile) : 0.0;
        const double PQ[3] = {P[0] - __ldg(pk + KR_PX * kKetTile), P[1] - __ldg(pk + KR_PY * kKetTile),
                              P[2] - __ldg(pk + KR_PZ * kKetTile)};
        const double QC[3] = {__ldg(pk + KR_QCX * kKetTile), __ldg(pk + KR_QCY * kKetTile),
                              __ldg(pk + KR_QCZ * kKetTile)};
        const double ccd = __ldg(pk + KR_C * kKetTile);
        const double rs = rsqrt(zeta + eta);
        const double inv = rs * rs;
        const double rz = eta * inv, re = zeta * inv;
        const double T = zeta * rz * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
        const double pref = cab * ccd * rs;
        const double kap2 = 2.0 * ((DER == DA || AB_) ? alpha : DER == DB ? zeta - alpha : gamma);
        const double kapb2 = 2.0 * (zeta - alpha);  // the B block of a merged pass
        const double kapc2 = 2.0 * gamma;           // the C block of an all-centre pass
        double u[NR], w[NR];
        rys_smem<NR, double>(T, stab, tab, u, w);
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const double ur = u[r];
          const double b00 = 0.5 * inv * ur, b10 = hz - hz * rz * ur, b01 = he - he * re * ur;
          double I[3][EM + 1][FM + 1];
#pragma unroll
          for (int x = 0; x < 3; ++x) {
            const double pa = PA[x] - rz * ur * PQ[x];
            const double qc = QC[x] + re * ur * PQ[x];
            I[x][0][0] = (x == 2) ? w[r] * pref : 1.0;
#pragma unroll
            for (int e = 0; e < EM; ++e)
              I[x][e + 1][0] = pa * I[x][e][0] + (e ? e * b10 * I[x][e > 0 ? e - 1 : 0][0] : 0.0);
#pragma unroll
            for (int f = 0; f < FM; ++f)
#pragma unroll
              for (int e = 0; e <= EM; ++e)
                I[x][e][f + 1] = qc * I[x][e][f] + (f ? f * b01 * I[x][e][f > 0 ? f - 1 : 0] : 0.0) +
                                 (e ? e * b00 * I[x][e > 0 ? e - 1 : 0][f] : 0.0);
          }
          if constexpr (ABC_) {
            gfor<0, NW3E>([&](auto IE) {
              constexpr int ie = decltype(IE)::value;
              constexpr int le = [] { int l = LA, r = ie; while (r >= ncart(l)) { r -= ncart(l); ++l; } return l; }();
              constexpr int ce = cart_comp(le, ie - ncart_before(LA, le));
              gfor<0, NW3F>([&](auto JF) {
                constexpr int jf = decltype(JF)::value;
                constexpr int lf = [] { int l = LC + 1, r = jf; while (r >= ncart(l)) { r -= ncart(l); ++l; } return l; }();
                constexpr int cf = cart_comp(lf, jf - ncart_before(LC + 1, lf));
                W3[ie * NW3F + jf] += kapc2 * I[0][comp_x(ce)][comp_x(cf)] * I[1][comp_y(ce)][comp_y(cf)] *
                                      I[2][comp_z(ce)][comp_z(cf)];
              });
            });
          }
          if constexpr (AB_) {
            // merged A+B pass: the products over e in [LA, LAB+1] once, into the B
            // block (2 beta) and, for e >= LA+1, the A block (2 alpha)
            gfor<0, NW2E>([&](auto IE) {
              constexpr int ie = decltype(IE)::value;
              constexpr int le = [] { int l = LA, r = ie; while (r >= ncart(l)) { r -= ncart(l); ++l; } return l; }();
              constexpr int ce = cart_comp(le, ie - ncart_before(LA, le));
              gfor<0, NWF>([&](auto JF) {
                constexpr int jf = decltype(JF)::value;
                constexpr int lf = [] { int l = WF0, r = jf; while (r >= ncart(l)) { r -= ncart(l); ++l; } return l; }();
                constexpr int cf = cart_comp(lf, jf - ncart_before(WF0, lf));
                const double X = I[0][comp_x(ce)][comp_x(cf)] * I[1][comp_y(ce)][comp_y(cf)] *
                                 I[2][comp_z(ce)][comp_z(cf)];
                W2[ie * NWF + jf] += kapb2 * X;
                if constexpr (ie >= ncart(LA)) W[(ie - ncart(LA)) * NWF + jf] += kap2 * X;
              });
            });
          } else
          // raised block
          gfor<0, NWE>([&](auto IE) {
            constexpr int ie = decltype(IE)::value;
            constexpr int le = [] { int l = WE0, r = ie; while (r >= ncart(l)) { r -= ncart(l); ++l; } return l; }();
            constexpr int ce = cart_comp(le, ie - ncart_before(WE0, le));
            gfor<0, NWF>([&](auto JF) {
              constexpr int jf = decltype(JF)::value;
              constexpr int lf = [] { int l = WF0, r = jf; while (r >= ncart(l)) { r -= ncart(l); ++l; } return l; }();
              constexpr int cf = cart_comp(lf, jf - ncart_before(WF0, lf));
              if constexpr (f_in_pass<PASS, LC>(lf))
                W[ie * NWF + jf] += kap2 * I[0][comp_x(ce)][comp_x(cf)] * I[1][comp_y(ce)][comp_y(cf)] *
                                    I[2][comp_z(ce)][comp_z(cf)];
            });
          });
          if constexpr (HAS_U) {
            gfor<0, NUE>([&](auto IE) {
              constexpr int ie = decltype(IE)::value;
              constexpr int le = [] { int l = UE0, r = ie; while (r >= ncart(l)) { r -= ncart(l); ++l; } return l; }();
              constexpr int ce = cart_comp(le, ie - ncart_before(UE0, le));
              gfor<0, NUF>([&](auto JF) {
                constexpr int jf = decltype(JF)::value;
                constexpr int lf = [] { int l = UF0, r = jf; while (r >= ncart(l)) { r -= ncart(l); ++l; } return l; }();
                constexpr int cf = cart_comp(lf, jf - ncart_before(UF0, lf));
                if constexpr (f_in_pass<PASS, LC>(lf))
                  U[ie * NUF + jf] += I[0][comp_x(ce)][comp_x(cf)] * I[1][comp_y(ce)][comp_y(cf)] *
                                      I[2][comp_z(ce)][comp_z(cf)];
              });
            });
          }
        }
      }
    }

    // ---- transfer + contraction with G, once per quartet ----
    const double ABx = __ldg(blk.bra.AB + p), ABy = __ldg(blk.bra.AB + nbra + p),
                 ABz = __ldg(blk.bra.AB + 2 * nbra + p);
    const double CDx = __ldg(blk.ket.AB + q), CDy = __ldg(blk.ket.AB + nket + q),
                 CDz = __ldg(blk.ket.AB + 2 * nket + q);
    constexpr int PB = LB + ((DER == DB || AB_) ? 1 : 0), PD = LD;
    double abp[3][PB + 1], cdp[3][PD + 1];
    abp[0][0] = abp[1][0] = abp[2][0] = 1.0;
    cdp[0][0] = cdp[1][0] = cdp[2][0] = 1.0;
#pragma unroll
    for (int k = 1; k <= PB; ++k) {
      abp[0][k] = abp[0][k - 1] * ABx; abp[1][k] = abp[1][k - 1] * ABy; abp[2][k] = abp[2][k - 1] * ABz;
    }
#pragma unroll
    for (int k = 1; k <= PD; ++k) {
      cdp[0][k] = cdp[0][k - 1] * CDx; cdp[1][k] = cdp[1][k - 1] * CDy; cdp[2][k] = cdp[2][k - 1] * CDz;
    }
    const int fa = __ldg(blk.bra.func_a + p), fb = __ldg(blk.bra.func_b + p);
    const int fc = __ldg(blk.ket.func_a + q), fd = __ldg(blk.ket.func_b + q);
    const double s = quartet_weight(blk, p, q);
    const double* __restrict__ D = ga.D;
    const size_t nbf = (size_t)ga.nbf;
    double g[3] = {0.0, 0.0, 0.0}, g2[3] = {0.0, 0.0, 0.0};  // g2: the B centre of a merged pass
    double g3[3] = {0.0, 0.0, 0.0};                         // g3: the C centre of an all-centre pass
    constexpr int D1 = AB_ ? DA : DER;  // the centre g belongs to
    gfor<0, NA>([&](auto IA) {
      constexpr int a = decltype(IA)::value;
      constexpr int ca = cart_comp(LA, a);
      gfor<0, NB>([&](auto IB) {
        constexpr int b = decltype(IB)::value;
        constexpr int cb = cart_comp(LB, b);
        const double Dab = __ldg(D + (fa + a) * nbf + fb + b);
        gfor<0, NC>([&](auto IC) {
          constexpr int c = decltype(IC)::value;
          constexpr int cc = cart_comp(LC, c);
          const double Dac = __ldg(D + (fa + a) * nbf + fc + c), Dbc = __ldg(D + (fb + b) * nbf + fc + c);
          gfor<0, ND>([&](auto ID) {
            constexpr int d = decltype(ID)::value;
            constexpr int cd = cart_comp(LD, d);
            constexpr double den = dfact_odd(comp_x(ca)) * dfact_odd(comp_y(ca)) * dfact_odd(comp_z(ca)) *
                                   dfact_odd(comp_x(cb)) * dfact_odd(comp_y(cb)) * dfact_odd(comp_z(cb)) *
                                   dfact_odd(comp_x(cc)) * dfact_odd(comp_y(cc)) * dfact_odd(comp_z(cc)) *
                                   dfact_odd(comp_x(cd)) * dfact_odd(comp_y(cd)) * dfact_odd(comp_z(cd));
            const double Dcd = __ldg(D + (fc + c) * nbf + fd + d), Dbd = __ldg(D + (fb + b) * nbf + fd + d),
                         Dad = __ldg(D + (fa + a) * nbf + fd + d);
            double G = s * (4.0 * Dab * Dcd - Dac * Dbd - Dad * Dbc);
            if constexpr (den != 1.0) G *= rsqrt(den);
            gfor<0, 3>([&](auto X) {
              constexpr int x = decltype(X)::value;
              // raised term: component shifted by +1 in x on the derivative centre
              constexpr int ra = D1 == DA ? shift(ca, x, 1) : ca;
              constexpr int rb = D1 == DB ? shift(cb, x, 1) : cb;
              constexpr int rc = D1 == DC ? shift(cc, x, 1) : cc;
              double acc = 0.0;
              hrr_terms<ra, rb, WE0>(abp, [&](auto E, double hb) {
                hrr_terms<rc, cd, WF0>(cdp, [&](auto F, double hd) {
                  acc += hb * hd * W[decltype(E)::value * NWF + decltype(F)::value];
                });
              });
              // lowered term: - n_x times the component shifted by -1
              constexpr int nx = comp_n(D1 == DA ? ca : D1 == DB ? cb : cc, x);
              if constexpr (HAS_U && nx > 0) {
                constexpr int la_ = D1 == DA ? shift(ca, x, -1) : ca;
                constexpr int lb_ = D1 == DB ? shift(cb, x, -1) : cb;
                constexpr int lc_ = D1 == DC ? shift(cc, x, -1) : cc;
                double low = 0.0;
                hrr_terms<la_, lb_, UE0>(abp, [&](auto E, double hb) {
                  hrr_terms<lc_, cd, UF0>(cdp, [&](auto F, double hd) {
                    low += hb * hd * U[decltype(E)::value * NUF + decltype(F)::value];
                  });
                });
                acc -= nx * low;
              }
              g[x] += G * acc;
              if constexpr (AB_) {  // the B centre: W2 over e in [LA, LAB+1], U for b - 1x
                double accb = 0.0;
                hrr_terms<ca, shift(cb, x, 1), LA>(abp, [&](auto E, double hb) {
                  hrr_terms<cc, cd, WF0>(cdp, [&](auto F, double hd) {
                    accb += hb * hd * W2[decltype(E)::value * NWF + decltype(F)::value];
                  });
                });
                constexpr int nbx = comp_n(cb, x);
                if constexpr (HAS_U && nbx > 0) {
                  double low = 0.0;
                  hrr_terms<ca, shift(cb, x, -1), UE0>(abp, [&](auto E, double hb) {
                    hrr_terms<cc, cd, UF0>(cdp, [&](auto F, double hd) {
                      low += hb * hd * U[decltype(E)::value * NUF + decltype(F)::value];
                    });
                  });
                  accb -= nbx * low;
                }
                g2[x] += G * accb;
              }
              if constexpr (ABC_) {  // the C centre: W3 over f in [LC+1, LCD+1], U for c - 1x
                double accc = 0.0;
                hrr_terms<ca, cb, LA>(abp, [&](auto E, double hb) {
                  hrr_terms<shift(cc, x, 1), cd, LC + 1>(cdp, [&](auto F, double hd) {
                    accc += hb * hd * W3[decltype(E)::value * NW3F + decltype(F)::value];
                  });
                });
                constexpr int ncx = comp_n(cc, x);
                if constexpr (HAS_U && ncx > 0) {
                  double low = 0.0;
                  hrr_terms<ca, cb, UE0>(abp, [&](auto E, double hb) {
                    hrr_terms<shift(cc, x, -1), cd, UF0>(cdp, [&](auto F, double hd) {
                      low += hb * hd * U[decltype(E)::value * NUF + decltype(F)::value];
                    });
                  });
                  accc -= ncx * low;
                }
                g3[x] += G * accc;
              }
            });
          });
        });
      });
    });
    const int sh = D1 == DA ? __ldg(blk.bra.shell_a + p) : D1 == DB ? __ldg(blk.bra.shell_b + p)
                                                                    : __ldg(blk.ket.shell_a + q);
    const int at = __ldg(ga.shell_atom + sh);
    const int atD = __ldg(ga.shell_atom + __ldg(blk.ket.shell_b + q));
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      atomicAdd(ga.grad + 3 * at + x, g[x]);
      atomicAdd(ga.grad + 3 * atD + x, -(g[x] + g2[x] + g3[x]));
    }
    if constexpr (AB_) {
      const int atB = __ldg(ga.shell_atom + __ldg(blk.bra.shell_b + p));
#pragma unroll
      for (int x = 0; x < 3; ++x) atomicAdd(ga.grad + 3 * atB + x, g2[x]);
    }
    if constexpr (ABC_) {
      const int atC = __ldg(ga.shell_atom + __ldg(blk.ket.shell_a + q));
#pragma unroll
      for (int x = 0; x < 3; ++x) atomicAdd(ga.grad + 3 * atC + x, g3[x]);
    }
  }
}

template <int LA, int LB, int LC, int LD>
int launch(const QuartetBlock& blk, const GradSmallArgs& ga, const RysTablesView& tab, cudaStream_t stream,
           int num_sms) {
  const int64_t nq = blk.total - blk.t_begin;
  if (nq <= 0) return 0;
  constexpr int NR = (LA + LB + LC + LD + 1) / 2 + 1;
  // the A and B centres in one pass when its three accumulator blocks stay small
  constexpr int LAB = LA + LB, LCD = LC + LD;
  constexpr int nf = ncart_range(LC, LCD);
  constexpr int merged_size = (ncart_range(LA + 1, LAB + 1) + ncart_range(LA, LAB + 1) +
                               ((LA >= 1 || LB >= 1) ? ncart_range(LA >= 1 ? LA - 1 : 0, LAB - 1) : 0)) * nf;
  constexpr bool kMerge = merged_size <= 48;
  // all three centres in one pass when that pass's blocks stay small too
  constexpr int all_size = merged_size + ncart_range(LA, LAB) * ncart_range(LC + 1, LCD + 1) +
                           ((LC >= 1) ? ncart_range(LA, LAB) * ncart(LC - 1) : 0);
  constexpr bool kAll = all_size <= 72;
  // a separate B pass in two halves when its raised block alone exceeds 128 doubles
  // ((ds|pp): 144, which ptxas could only place in local memory; the halves hold 48
  // and 96 and run about ten times faster than the whole pass).  Halving the other
  // passes that spill a little ((ds|pp) A and C, (dp|ps), (ds|ds), (dd|ss): 0.5-2.3 KB
  // per thread) measured 9-43 % slower per class: the second primitive loop costs
  // more than those spills.
  constexpr bool kSplitB = ncart_range(LA, LAB + 1) * nf > 128 && LCD > LC;
  const size_t smem = table_bytes<NR, double>();
  // only the kernels this class launches are instantiated (and given their shared memory)
  auto allow = [&](auto kern) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess;
  };
  static bool attr = false;
  if (!attr) {
    bool ok;
    if constexpr (kAll) {
      ok = allow(grad_small_kernel<LA, LB, LC, LD, DABC>);
    } else if constexpr (kMerge) {
      ok = allow(grad_small_kernel<LA, LB, LC, LD, DAB>) && allow(grad_small_kernel<LA, LB, LC, LD, DC>);
    } else if constexpr (kSplitB) {
      ok = allow(grad_small_kernel<LA, LB, LC, LD, DA>) && allow(grad_small_kernel<LA, LB, LC, LD, DB_LO>) &&
           allow(grad_small_kernel<LA, LB, LC, LD, DB_HI>) && allow(grad_small_kernel<LA, LB, LC, LD, DC>);
    } else {
      ok = allow(grad_small_kernel<LA, LB, LC, LD, DA>) && allow(grad_small_kernel<LA, LB, LC, LD, DB>) &&
           allow(grad_small_kernel<LA, LB, LC, LD, DC>);
    }
    if (!ok) return -3;
    attr = true;
  }
  const int threads = 128;
  const int64_t want = (nq + threads - 1) / threads;
  const int grid = (int)(want < (int64_t)num_sms * 8 ? want : (int64_t)num_sms * 8);
  if constexpr (kAll) {
    grad_small_kernel<LA, LB, LC, LD, DABC><<<grid, threads, smem, stream>>>(blk, ga, tab);
  } else {
    if constexpr (kMerge) {
      grad_small_kernel<LA, LB, LC, LD, DAB><<<grid, threads, smem, stream>>>(blk, ga, tab);
    } else if constexpr (kSplitB) {
      grad_small_kernel<LA, LB, LC, LD, DA><<<grid, threads, smem, stream>>>(blk, ga, tab);
      grad_small_kernel<LA, LB, LC, LD, DB_LO><<<grid, threads, smem, stream>>>(blk, ga, tab);
      grad_small_kernel<LA, LB, LC, LD, DB_HI><<<grid, threads, smem, stream>>>(blk, ga, tab);
    } else {
      grad_small_kernel<LA, LB, LC, LD, DA><<<grid, threads, smem, stream>>>(blk, ga, tab);
      grad_small_kernel<LA, LB, LC, LD, DB><<<grid, threads, smem, stream>>>(blk, ga, tab);
    }
    grad_small_kernel<LA, LB, LC, LD, DC><<<grid, threads, smem, stream>>>(blk, ga, tab);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

}  // namespace grad_small
}  // namespace lai
