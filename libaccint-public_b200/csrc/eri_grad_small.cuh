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
// run once per contracted quartet.  One launch per centre (DER = A, B or C) keeps
// the live accumulators to one W and one U block; each launch adds its centre's
// derivative and subtracts it from the D centre.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "eri_device.cuh"
#include "eri_kernels.h"

namespace lai {
namespace grad_small {

enum { DA = 0, DB = 1, DC = 2 };

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

template <int LA, int LB, int LC, int LD, int DER>
__global__ void __launch_bounds__(128) grad_small_kernel(QuartetBlock blk, GradSmallArgs ga, RysTablesView tab) {
  constexpr int LAB = LA + LB, LCD = LC + LD;
  constexpr int NR = (LAB + LCD + 1) / 2 + 1;
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  // raised block W and lowered block U, as shell ranges [E0, E1] x [F0, F1]
  constexpr int WE0 = DER == DA ? LA + 1 : LA, WE1 = DER == DC ? LAB : LAB + 1;
  constexpr int WF0 = DER == DC ? LC + 1 : LC, WF1 = DER == DC ? LCD + 1 : LCD;
  constexpr bool HAS_U = DER == DA ? LA >= 1 : DER == DB ? LB >= 1 : LC >= 1;
  constexpr int UE0 = DER == DA ? (LA >= 1 ? LA - 1 : 0) : LA;
  constexpr int UE1 = DER == DA ? LAB - 1 : DER == DB ? LAB - 1 : LAB;
  constexpr int UF0 = DER == DC ? (LC >= 1 ? LC - 1 : 0) : LC;
  constexpr int UF1 = DER == DC ? LCD - 1 : LCD;
  constexpr int NWE = ncart_range(WE0, WE1), NWF = ncart_range(WF0, WF1);
  constexpr int NUE = HAS_U ? ncart_range(UE0, UE1) : 1, NUF = HAS_U ? ncart_range(UF0, UF1) : 1;
  constexpr int EM = DER == DC ? LAB : LAB + 1;  // vertical recurrence extents
  constexpr int FM = DER == DC ? LCD + 1 : LCD;

  const int nbra = blk.bra.npairs, nket = blk.ket.npairs;
  const int Kab = blk.bra.Ka * blk.bra.Kb, Kcd = blk.ket.Ka * blk.ket.Kb;
  const size_t sb = (size_t)Kab * nbra, sk = (size_t)Kcd * nket;
  const int64_t nthreads = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = blk.t_begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < blk.total; t += nthreads) {
    const int p = find_bra(blk.offsets, nbra, t);
    const int q = (blk.qbegin ? __ldg(blk.qbegin + p) : 0) + (int)(t - __ldg(blk.offsets + p));
    double W[NWE * NWF], U[NUE * NUF];
#pragma unroll
    for (int i = 0; i < NWE * NWF; ++i) W[i] = 0.0;
#pragma unroll
    for (int i = 0; i < NUE * NUF; ++i) U[i] = 0.0;

    for (int ib = 0; ib < Kab; ++ib) {
      const double* pb = blk.bra.prim + (size_t)ib * nbra + p;
      const double qab = __ldg(pb + PF_Q * sb);
      if (qab * blk.ket.qprim_max < ga.prim_eps) break;
      const double zeta = __ldg(pb + PF_ZETA * sb), hz = __ldg(pb + PF_HZ * sb);
      const double alpha = __ldg(pb + PF_ALPHA * sb);
      const double P[3] = {__ldg(pb + PF_PX * sb), __ldg(pb + PF_PY * sb), __ldg(pb + PF_PZ * sb)};
      const double PA[3] = {__ldg(pb + PF_PAX * sb), __ldg(pb + PF_PAY * sb), __ldg(pb + PF_PAZ * sb)};
      const double cab = __ldg(pb + PF_C * sb);
      for (int ik = 0; ik < Kcd; ++ik) {
        const double* pk = blk.ket.prim + (size_t)ik * nket + q;
        const double qcd = __ldg(pk + PF_Q * sk);
        if (qab * qcd < ga.prim_eps) break;
        const double eta = __ldg(pk + PF_ZETA * sk), he = __ldg(pk + PF_HZ * sk);
        const double gamma = __ldg(pk + PF_ALPHA * sk);
        const double PQ[3] = {P[0] - __ldg(pk + PF_PX * sk), P[1] - __ldg(pk + PF_PY * sk),
                              P[2] - __ldg(pk + PF_PZ * sk)};
        const double QC[3] = {__ldg(pk + PF_PAX * sk), __ldg(pk + PF_PAY * sk), __ldg(pk + PF_PAZ * sk)};
        const double ccd = __ldg(pk + PF_C * sk);
        const double rs = rsqrt(zeta + eta);
        const double inv = rs * rs;
        const double rz = eta * inv, re = zeta * inv;
        const double T = zeta * rz * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
        const double pref = cab * ccd * rs;
        const double kap2 = 2.0 * (DER == DA ? alpha : DER == DB ? zeta - alpha : gamma);
        double u[NR], w[NR];
        rys_roots_table<double>(NR, T, tab, u, w);
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
          // raised block
          gfor<0, NWE>([&](auto IE) {
            constexpr int ie = decltype(IE)::value;
            constexpr int le = [] { int l = WE0, r = ie; while (r >= ncart(l)) { r -= ncart(l); ++l; } return l; }();
            constexpr int ce = cart_comp(le, ie - ncart_before(WE0, le));
            gfor<0, NWF>([&](auto JF) {
              constexpr int jf = decltype(JF)::value;
              constexpr int lf = [] { int l = WF0, r = jf; while (r >= ncart(l)) { r -= ncart(l); ++l; } return l; }();
              constexpr int cf = cart_comp(lf, jf - ncart_before(WF0, lf));
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
    constexpr int PB = LB + (DER == DB ? 1 : 0), PD = LD;
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
    double g[3] = {0.0, 0.0, 0.0};
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
              constexpr int ra = DER == DA ? shift(ca, x, 1) : ca;
              constexpr int rb = DER == DB ? shift(cb, x, 1) : cb;
              constexpr int rc = DER == DC ? shift(cc, x, 1) : cc;
              double acc = 0.0;
              hrr_terms<ra, rb, WE0>(abp, [&](auto E, double hb) {
                hrr_terms<rc, cd, WF0>(cdp, [&](auto F, double hd) {
                  acc += hb * hd * W[decltype(E)::value * NWF + decltype(F)::value];
                });
              });
              // lowered term: - n_x times the component shifted by -1
              constexpr int nx = comp_n(DER == DA ? ca : DER == DB ? cb : cc, x);
              if constexpr (HAS_U && nx > 0) {
                constexpr int la_ = DER == DA ? shift(ca, x, -1) : ca;
                constexpr int lb_ = DER == DB ? shift(cb, x, -1) : cb;
                constexpr int lc_ = DER == DC ? shift(cc, x, -1) : cc;
                double low = 0.0;
                hrr_terms<la_, lb_, UE0>(abp, [&](auto E, double hb) {
                  hrr_terms<lc_, cd, UF0>(cdp, [&](auto F, double hd) {
                    low += hb * hd * U[decltype(E)::value * NUF + decltype(F)::value];
                  });
                });
                acc -= nx * low;
              }
              g[x] += G * acc;
            });
          });
        });
      });
    });
    const int sh = DER == DA ? __ldg(blk.bra.shell_a + p) : DER == DB ? __ldg(blk.bra.shell_b + p)
                                                                      : __ldg(blk.ket.shell_a + q);
    const int at = __ldg(ga.shell_atom + sh);
    const int atD = __ldg(ga.shell_atom + __ldg(blk.ket.shell_b + q));
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      atomicAdd(ga.grad + 3 * at + x, g[x]);
      atomicAdd(ga.grad + 3 * atD + x, -g[x]);
    }
  }
}

template <int LA, int LB, int LC, int LD>
int launch(const QuartetBlock& blk, const GradSmallArgs& ga, const RysTablesView& tab, cudaStream_t stream,
           int num_sms) {
  const int64_t nq = blk.total - blk.t_begin;
  if (nq <= 0) return 0;
  const int threads = 128;
  const int64_t want = (nq + threads - 1) / threads;
  const int grid = (int)(want < (int64_t)num_sms * 8 ? want : (int64_t)num_sms * 8);
  grad_small_kernel<LA, LB, LC, LD, DA><<<grid, threads, 0, stream>>>(blk, ga, tab);
  grad_small_kernel<LA, LB, LC, LD, DB><<<grid, threads, 0, stream>>>(blk, ga, tab);
  grad_small_kernel<LA, LB, LC, LD, DC><<<grid, threads, 0, stream>>>(blk, ga, tab);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

}  // namespace grad_small
}  // namespace lai
