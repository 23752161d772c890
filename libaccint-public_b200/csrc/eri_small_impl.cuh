// Thread-per-quartet Rys ERI kernels with fused J/K digestion for the small
// angular-momentum classes, fully specialised at compile time on (la,lb|lc,ld):
// the 2D tables, the (e0|f0) accumulator G, the output block and the density /
// Fock blocks all live in registers.  The same algorithm as eri_generic.cu (see
// eri_device.cuh), unrolled.
//
// Persistent launch (a few blocks per SM, grid-stride over chunks of 32
// consecutive canonical quartets, one per lane).  Consecutive quartets usually
// share the bra pair, so bra primitive data are warp-uniform loads, ket primitive
// data are coalesced (SoA by pair index), and the bra-pair Coulomb block J_ij is
// summed across the warp before its atomic update.  Each block stages the lookup
// table its root count needs in shared memory once (Boys grid for one root, the
// class's Rys table otherwise), with row strides padded so that lanes reading
// different rows hit different banks -- from global memory those per-lane
// gathers would touch up to 32 cache lines per load instruction.
//
// Templated on the compute type R: double for the FP64 path, float for the FP32
// part of a mixed-precision build (roots, recurrences and contraction in FP32;
// the contracted quartet is digested in FP64).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "eri_device.cuh"
#include "eri_kernels.h"
#include "eri_tables_smem.cuh"
#include "fp32_tables.h"

namespace lai {

namespace {

template <int B, int E, typename F>
__device__ __forceinline__ void sfor(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    sfor<B + 1, E>(f);
  }
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Compensated sum s + c (two-sum of Knuth: s' = s + x, z = s' - s,
// c += (s - (s' - z)) + (x - z)).
template <typename R>
struct CompSum {
  R s, c;
};
template <typename R>
__device__ __forceinline__ void comp_add(CompSum<R>& a, R x) {
  const R s1 = a.s + x;
  const R z = s1 - a.s;
  const R e = (a.s - (s1 - z)) + (x - z);
  a.s = s1;
  a.c += e;
}

template <int LA, int LB, int LC, int LD, typename GV>
__device__ __forceinline__ void small_finish(GV&& gval, const QuartetBlock& blk, const JKArgs& args,
                                             int64_t t, int p, int q, bool active, bool uniform_bra);

template <int LA, int LB, int LC, int LD, typename R, bool SPLIT>
__device__ __forceinline__ void small_quartet(const QuartetBlock& blk, const JKArgs& args,
                                              const RysTablesView& tab,
                                              const R* __restrict__ stab, int64_t t, int p,
                                              bool active, bool uniform_bra, int ps, int sub) {
  // ps lanes (a power of two, aligned) share this quartet: lane `sub` of the group
  // runs bra primitive pairs sub, sub+ps, ...; the group then sums its partial
  // (e0|f0) blocks and lane 0 of the group alone transfers and digests.
  constexpr int LAB = LA + LB, LCD = LC + LD;
  constexpr int NR = (LAB + LCD) / 2 + 1;
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int NE = ncart_range(LA, LAB), NF = ncart_range(LC, LCD);
  constexpr int W = LCD + 1;
  const int nbra = blk.bra.npairs, nket = blk.ket.npairs;
  const int q = (blk.qbegin ? __ldg(blk.qbegin + p) : 0) + (int)(t - __ldg(blk.offsets + p));

  const int Kab = blk.bra.Ka * blk.bra.Kb;
  const int Kcd = blk.ket.Ka * blk.ket.Kb;
  const size_t sb = (size_t)Kab * nbra;

  constexpr bool F32 = sizeof(R) == 4;
  // FP32: the primitive terms of one inner loop are summed in G, which is then
  // added to the running total Gc with a compensated (two-sum) step (registers
  // permitting: up to 18 (e0|f0) values); FP64: G is the total.
  constexpr bool COMP = F32 && NE * NF <= 18;
  R G[NE * NF];
  CompSum<R> Gc[COMP ? NE * NF : 1];
#pragma unroll
  for (int i = 0; i < NE * NF; ++i) G[i] = R(0);
#pragma unroll
  for (int i = 0; i < (COMP ? NE * NF : 1); ++i) Gc[i].s = Gc[i].c = R(0);
  auto merge = [&]() {
    if constexpr (COMP) {
#pragma unroll
      for (int i = 0; i < NE * NF; ++i) {
        comp_add(Gc[i], G[i]);
        G[i] = R(0);
      }
    }
  };
  // FP32: P - Q = (A - C) + (P - A) - (Q - C) with A - C, the difference of the
  // bra and ket pairs' first centres, formed in FP64, so that the error of P - Q
  // scales with |P - A| rather than with the absolute coordinates.  FP64: P - Q
  // from the stored centres P and Q (no extra registers held across the loop).
  R AC[3] = {R(0), R(0), R(0)};
  if constexpr (F32) {
#pragma unroll
    for (int x = 0; x < 3; ++x)
      AC[x] = R(__ldg(blk.bra.Acen + x * nbra + p) - __ldg(blk.ket.Acen + x * nket + q));
  }

  const double peps = args.prim_eps;
  unsigned int nprim_done = 0;
  // unsplit: compile-time stride 1 keeps the bra loop warp-uniform
  const int ib0 = SPLIT ? sub : 0, ibs = SPLIT ? ps : 1;
  // One primitive quartet: bra primitive pair (zeta, hz, PA, cab), ket
  // primitive pair `cur`; accumulates into G.  The FP32 kernels read an FP32 copy
  // of the pair tables (half the bytes and registers, no conversions).
  const R* __restrict__ bprim = prim_table<R>(blk.bra);
  struct BraVals {
    R zeta, hz, Px, Py, Pz, PAx, PAy, PAz, cab;
  };
  const R* __restrict__ bprimb = bra_records<R>(blk.bra);
  auto load_bra = [&](int ib, R& qab, BraVals& v) {
    if (uniform_bra || SPLIT) {
      // the warp (or the lane group) reads one pair's primitives: its contiguous
      // per-pair records, 16-byte vector loads
      const R* rb = bprimb + ((size_t)p * Kab + ib) * kBraRec;
      if constexpr (F32) {
        const float4* r4 = reinterpret_cast<const float4*>(rb);
        const float4 a = __ldg(r4), c = __ldg(r4 + 2);
        qab = a.x; v.zeta = a.y; v.hz = a.z; v.cab = a.w;
        v.PAx = c.x; v.PAy = c.y; v.PAz = c.z;
      } else {
        const double2* r2 = reinterpret_cast<const double2*>(rb);
        const double2 a = __ldg(r2), b = __ldg(r2 + 1), c = __ldg(r2 + 2), d = __ldg(r2 + 3),
                      e = __ldg(r2 + 4), f = __ldg(r2 + 5);
        qab = a.x; v.zeta = a.y; v.hz = b.x; v.cab = b.y;
        v.Px = c.x; v.Py = c.y; v.Pz = d.x;
        v.PAx = e.x; v.PAy = e.y; v.PAz = f.x;
      }
      return;
    }
    const R* pb = bprim + (size_t)ib * nbra + p;
    qab = __ldg(pb + PF_Q * sb);
    v.zeta = __ldg(pb + PF_ZETA * sb);
    v.hz = __ldg(pb + PF_HZ * sb);
    if constexpr (!F32) {
      v.Px = __ldg(pb + PF_PX * sb);
      v.Py = __ldg(pb + PF_PY * sb);
      v.Pz = __ldg(pb + PF_PZ * sb);
    }
    v.PAx = __ldg(pb + PF_PAX * sb);
    v.PAy = __ldg(pb + PF_PAY * sb);
    v.PAz = __ldg(pb + PF_PAZ * sb);
    v.cab = __ldg(pb + PF_C * sb);
  };
  // One-root classes accumulate per row of the inner primitive loop: the factor
  // constant along the row (the outer pair's contraction coefficient; for (ps|ss)
  // also PA) multiplies the row sums once, when the row ends (fold_row):
  //   (ss|ss): S0 = sum c' rs F_0;  (ps|ss): S0 as above, S1_i = sum PQ_i c' rs rz F_1,
  //   G_i += c (PA_i S0 - S1_i),
  // with c' the inner pair's coefficient.
  constexpr bool kKetOuter = (LAB == LCD);
  constexpr bool kFold = NR == 1 && (LAB == 0 || !kKetOuter);
  R S0 = R(0), S1[3] = {R(0), R(0), R(0)};
  auto fold_row = [&](R rowc, const BraVals& bv) {
    if constexpr (kFold) {
      if constexpr (LAB == 0) {
        G[0] += rowc * S0;
      } else {
        const R PA[3] = {bv.PAx, bv.PAy, bv.PAz};
        sfor<0, NE>([&](auto IE) {
          constexpr int ie = decltype(IE)::value;
          constexpr int ce = cart_comp(LA, ie);
          constexpr int d = comp_x(ce) ? 0 : comp_y(ce) ? 1 : 2;
          G[ie] += rowc * (PA[d] * S0 - S1[d]);
        });
        S1[0] = S1[1] = S1[2] = R(0);
      }
      S0 = R(0);
    }
  };
  auto prim = [&](const BraVals& bv, const KetPrimT<R>& cur) {
    const R zeta = bv.zeta, hz = bv.hz, cab = bv.cab;
    const R PAx = bv.PAx, PAy = bv.PAy, PAz = bv.PAz;
    const R eta = R(cur.eta);
    const R he = R(cur.he);
    const R QCx = R(cur.qcx), QCy = R(cur.qcy), QCz = R(cur.qcz);
    const R PQx = F32 ? AC[0] + (PAx - QCx) : bv.Px - R(cur.px);
    const R PQy = F32 ? AC[1] + (PAy - QCy) : bv.Py - R(cur.py);
    const R PQz = F32 ? AC[2] + (PAz - QCz) : bv.Pz - R(cur.pz);
    const R ccd = R(cur.c);
    const R s = zeta + eta;
    const R rs = fast_rsqrt(s);
    const R inv = rs * rs;
    const R rz = eta * inv, re = zeta * inv;
    const R T = zeta * rz * (PQx * PQx + PQy * PQy + PQz * PQz);
    if constexpr (NR == 1) {
      // One root: (ss|ss) = pref F_0 and (p_i s|ss) = pref (PA_i F_0 - rz PQ_i F_1)
      // -- the one-point Rys rule (w = F_0, u = F_1/F_0) written without its
      // quotient -- summed per row (fold_row) without the row's constant factor.
      R F0, F1;
      if constexpr (F32) boys01_f32(T, stab, F0, F1); else boys01_smem<R>(T, stab, F0, F1);
      static_assert(LAB == 0 || (LA == 1 && LB == 0 && LCD == 0), "one-root classes: (ss|ss), (ps|ss)");
      if constexpr (kFold) {
        const R pv = (kKetOuter ? cab : ccd) * rs;
        S0 += pv * F0;
        if constexpr (LAB == 1) {
          const R pw1 = pv * rz * F1;
          S1[0] += PQx * pw1;
          S1[1] += PQy * pw1;
          S1[2] += PQz * pw1;
        }
      } else {
        // (ps|ss) with the ket loop outside: PA changes along the inner loop
        const R pref = cab * ccd * rs;
        const R pw0 = pref * F0, pw1 = pref * rz * F1;
        G[0] += PAx * pw0 - PQx * pw1;
        G[1] += PAy * pw0 - PQy * pw1;
        G[2] += PAz * pw0 - PQz * pw1;
      }
      return;
    }
    const R pref = cab * ccd * rs;
    R u[NR], w[NR];
    if constexpr (F32) rys_f32(NR, T, stab, tab.herm_x2, tab.herm_w, u, w);
    else rys_smem<NR, R>(T, stab, tab, u, w);
#pragma unroll
    for (int r = 0; r < NR; ++r) {
      const R ur = u[r];
      const R b00 = R(0.5) * inv * ur;
      const R b10 = hz - hz * rz * ur;
      const R b01 = he - he * re * ur;
      R I[3][LAB + 1][W];
      const R pa[3] = {PAx - rz * ur * PQx, PAy - rz * ur * PQy, PAz - rz * ur * PQz};
      const R qc[3] = {QCx + re * ur * PQx, QCy + re * ur * PQy, QCz + re * ur * PQz};
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        I[x][0][0] = (x == 2) ? w[r] * pref : R(1);
#pragma unroll
        for (int e = 0; e < LAB; ++e)
          I[x][e + 1][0] = pa[x] * I[x][e][0] + (e ? R(e) * b10 * I[x][e > 0 ? e - 1 : 0][0] : R(0));
#pragma unroll
        for (int f = 0; f < LCD; ++f)
#pragma unroll
          for (int e = 0; e <= LAB; ++e)
            I[x][e][f + 1] = qc[x] * I[x][e][f] +
                             (f ? R(f) * b01 * I[x][e][f > 0 ? f - 1 : 0] : R(0)) +
                             (e ? R(e) * b00 * I[x][e > 0 ? e - 1 : 0][f] : R(0));
      }
      sfor<0, NE>([&](auto IE) {
        constexpr int ie = decltype(IE)::value;
        // component ie of shells LA..LAB
        constexpr int le = [] { int l = LA, r = ie; while (r >= ncart(l)) { r -= ncart(l); ++l; } return l; }();
        constexpr int ce = cart_comp(le, ie - ncart_before(LA, le));
        sfor<0, NF>([&](auto JF) {
          constexpr int jf = decltype(JF)::value;
          constexpr int lf = [] { int l = LC, r = jf; while (r >= ncart(l)) { r -= ncart(l); ++l; } return l; }();
          constexpr int cf = cart_comp(lf, jf - ncart_before(LC, lf));
          G[ie * NF + jf] += I[0][comp_x(ce)][comp_x(cf)] * I[1][comp_y(ce)][comp_y(cf)] *
                             I[2][comp_z(ce)][comp_z(cf)];
        });
      });
    }
  };

  // Loop order.  Primitive pairs are sorted by their Schwarz bound, so a loop
  // stops once q_ab q_cd drops below the cut.  Ket data differ per lane (coalesced
  // loads); bra data are the same for the whole warp (broadcast loads that stay in
  // L1).  When bra and ket have the same angular momenta (typically similar
  // primitive counts), kets go outside: each ket primitive pair is then read once
  // per quartet instead of once per bra primitive pair (the re-reads of a warp's
  // 32 ket rows no longer fit in L1).  Otherwise the ket side usually has more
  // primitives (s pairs against p/d pairs) and goes inside, with its next primitive
  // pair loaded one iteration ahead.
  // this lane's ket pair in the ket tiles: primitive ik at pkt + ik * kKetPrimStride
  const R* __restrict__ pkt = ket_tile_ptr(ket_tiles<R>(blk.ket), q, Kcd);
  // FP32 quartets (fp32_prim_rel > 0): primitive quartets below that fraction of the
  // quartet's own Schwarz bound are skipped as well
  const R peps_r = R((F32 && args.prim_rel32 > 0.0)
                         ? fmax(peps, args.prim_rel32 * __ldg(blk.bra.Q + p) * __ldg(blk.ket.Q + q))
                         : peps);
  if constexpr (kKetOuter) {
    const R qab_max = ib0 < Kab ? __ldg(bprim + (size_t)ib0 * nbra + p + PF_Q * sb) : R(0);
    KetPrimT<R> nxt;
    load_ket_rec(pkt, nxt);
    for (int ik = 0; ik < Kcd; ++ik) {
      const KetPrimT<R> cur = nxt;
      if (qab_max * cur.q < peps_r || ib0 >= Kab) break;
      if (ik + 1 < Kcd) load_ket_rec(pkt + (size_t)(ik + 1) * kKetPrimStride, nxt);
      BraVals bv{};
      for (int ib = ib0; ib < Kab; ib += ibs) {
        R qab;
        load_bra(ib, qab, bv);
        if (qab * cur.q < peps_r) break;
        ++nprim_done;
        prim(bv, cur);
      }
      fold_row(R(cur.c), bv);
      merge();
    }
  } else {
    const R qket_max = R(blk.ket.qprim_max);
    // the first ket primitive opens every row: loaded once per quartet
    KetPrimT<R> k0;
    load_ket_rec(pkt, k0);
    for (int ib = ib0; ib < Kab; ib += ibs) {
      R qab;
      BraVals bv;
      load_bra(ib, qab, bv);
      if (qab * qket_max < peps_r) break;
      KetPrimT<R> nxt = k0;
      for (int ik = 0; ik < Kcd; ++ik) {
        const KetPrimT<R> cur = nxt;
        if (qab * cur.q < peps_r) break;
        if (ik + 1 < Kcd) load_ket_rec(pkt + (size_t)(ik + 1) * kKetPrimStride, nxt);
        ++nprim_done;
        prim(bv, cur);
      }
      fold_row(bv.cab, bv);
      merge();
    }
  }

  count_prims(args.prim_count, active ? nprim_done : 0u);
  // contracted (e0|f0) values in FP64 (FP32: the compensated sum s + c)
  double Gd[NE * NF];
#pragma unroll
  for (int i = 0; i < NE * NF; ++i) {
    if constexpr (COMP) Gd[i] = double(Gc[i].s) + double(Gc[i].c);
    else Gd[i] = double(G[i]);
  }
  if (SPLIT) {
#pragma unroll
    for (int i = 0; i < NE * NF; ++i)
      for (int o = ps >> 1; o > 0; o >>= 1) Gd[i] += __shfl_xor_sync(0xffffffffu, Gd[i], o);
    active = active && sub == 0;
  }
  small_finish<LA, LB, LC, LD>([&](int i) { return Gd[i]; }, blk, args, t, p, q, active, uniform_bra);
}

// Horizontal transfer (closed form), normalization and the 8-fold symmetric
// digestion of one contracted quartet (p, q), in double.  gval(i) returns the
// contracted (e0|f0) integral i = e * NF + f.  Every lane of the warp must call
// this together (the bra-pair Coulomb block is summed across the warp when
// uniform_bra holds).
template <int LA, int LB, int LC, int LD, typename GV>
__device__ __forceinline__ void small_finish(GV&& gval, const QuartetBlock& blk, const JKArgs& args,
                                             int64_t t, int p, int q, bool active, bool uniform_bra) {
  constexpr int LAB = LA + LB, LCD = LC + LD;
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int NF = ncart_range(LC, LCD);
  const int nbra = blk.bra.npairs, nket = blk.ket.npairs;
  (void)LAB;
  // ---- horizontal transfer (closed form) + normalization, in double ----
  const double ABx = __ldg(blk.bra.AB + p), ABy = __ldg(blk.bra.AB + nbra + p),
               ABz = __ldg(blk.bra.AB + 2 * nbra + p);
  const double CDx = __ldg(blk.ket.AB + q), CDy = __ldg(blk.ket.AB + nket + q),
               CDz = __ldg(blk.ket.AB + 2 * nket + q);
  double abp[3][LB + 1], cdp[3][LD + 1];
  abp[0][0] = abp[1][0] = abp[2][0] = 1.0;
  cdp[0][0] = cdp[1][0] = cdp[2][0] = 1.0;
#pragma unroll
  for (int k = 1; k <= LB; ++k) {
    abp[0][k] = abp[0][k - 1] * ABx; abp[1][k] = abp[1][k - 1] * ABy; abp[2][k] = abp[2][k - 1] * ABz;
  }
#pragma unroll
  for (int k = 1; k <= LD; ++k) {
    cdp[0][k] = cdp[0][k - 1] * CDx; cdp[1][k] = cdp[1][k - 1] * CDy; cdp[2][k] = cdp[2][k - 1] * CDz;
  }
  // bra transfer: H[a][b][f]
  double H[NA * NB * NF];
  sfor<0, NA>([&](auto IA) {
    constexpr int a = decltype(IA)::value;
    constexpr int ca = cart_comp(LA, a);
    sfor<0, NB>([&](auto IB) {
      constexpr int b = decltype(IB)::value;
      constexpr int cb = cart_comp(LB, b);
#pragma unroll
      for (int f = 0; f < NF; ++f) H[(a * NB + b) * NF + f] = 0.0;
      sfor<0, comp_x(cb) + 1>([&](auto KX) {
        constexpr int kx = decltype(KX)::value;
        sfor<0, comp_y(cb) + 1>([&](auto KY) {
          constexpr int ky = decltype(KY)::value;
          sfor<0, comp_z(cb) + 1>([&](auto KZ) {
            constexpr int kz = decltype(KZ)::value;
            constexpr int ex = comp_x(ca) + kx, ey = comp_y(ca) + ky, ez = comp_z(ca) + kz;
            constexpr int row = ncart_before(LA, ex + ey + ez) + cart_index(ex, ey, ez);
            constexpr double bc = binom(comp_x(cb), kx) * binom(comp_y(cb), ky) * binom(comp_z(cb), kz);
            const double cf = bc * abp[0][comp_x(cb) - kx] * abp[1][comp_y(cb) - ky] *
                              abp[2][comp_z(cb) - kz];
#pragma unroll
            for (int f = 0; f < NF; ++f) H[(a * NB + b) * NF + f] += cf * gval(row * NF + f);
          });
        });
      });
    });
  });
  // ket transfer: V[a][b][c][d]
  double V[NA * NB * NC * ND];
  sfor<0, NC>([&](auto IC) {
    constexpr int c = decltype(IC)::value;
    constexpr int cc = cart_comp(LC, c);
    sfor<0, ND>([&](auto ID) {
      constexpr int d = decltype(ID)::value;
      constexpr int cd = cart_comp(LD, d);
#pragma unroll
      for (int ab = 0; ab < NA * NB; ++ab) V[(ab * NC + c) * ND + d] = 0.0;
      sfor<0, comp_x(cd) + 1>([&](auto KX) {
        constexpr int kx = decltype(KX)::value;
        sfor<0, comp_y(cd) + 1>([&](auto KY) {
          constexpr int ky = decltype(KY)::value;
          sfor<0, comp_z(cd) + 1>([&](auto KZ) {
            constexpr int kz = decltype(KZ)::value;
            constexpr int fx = comp_x(cc) + kx, fy = comp_y(cc) + ky, fz = comp_z(cc) + kz;
            constexpr int col = ncart_before(LC, fx + fy + fz) + cart_index(fx, fy, fz);
            constexpr double bc = binom(comp_x(cd), kx) * binom(comp_y(cd), ky) * binom(comp_z(cd), kz);
            const double cf = bc * cdp[0][comp_x(cd) - kx] * cdp[1][comp_y(cd) - ky] *
                              cdp[2][comp_z(cd) - kz];
#pragma unroll
            for (int ab = 0; ab < NA * NB; ++ab) V[(ab * NC + c) * ND + d] += cf * H[ab * NF + col];
          });
        });
      });
    });
  });
  // normalization
  sfor<0, NA>([&](auto IA) {
    constexpr int a = decltype(IA)::value;
    constexpr int ca = cart_comp(LA, a);
    sfor<0, NB>([&](auto IB) {
      constexpr int b = decltype(IB)::value;
      constexpr int cb = cart_comp(LB, b);
      sfor<0, NC>([&](auto IC) {
        constexpr int c = decltype(IC)::value;
        constexpr int cc = cart_comp(LC, c);
        sfor<0, ND>([&](auto ID) {
          constexpr int d = decltype(ID)::value;
          constexpr int cd = cart_comp(LD, d);
          constexpr double den = dfact_odd(comp_x(ca)) * dfact_odd(comp_y(ca)) * dfact_odd(comp_z(ca)) *
                                 dfact_odd(comp_x(cb)) * dfact_odd(comp_y(cb)) * dfact_odd(comp_z(cb)) *
                                 dfact_odd(comp_x(cc)) * dfact_odd(comp_y(cc)) * dfact_odd(comp_z(cc)) *
                                 dfact_odd(comp_x(cd)) * dfact_odd(comp_y(cd)) * dfact_odd(comp_z(cd));
          if constexpr (den != 1.0) V[((a * NB + b) * NC + c) * ND + d] *= rsqrt(den);
        });
      });
    });
  });

  const int fa = __ldg(blk.bra.func_a + p), fb = __ldg(blk.bra.func_b + p);
  const int fc = __ldg(blk.ket.func_a + q), fd = __ldg(blk.ket.func_b + q);
  if (args.mode == MODE_RAW) {
    if (!active) return;
    const int64_t tl = t - blk.t_begin;
    double* o = args.raw_out + (size_t)tl * (NA * NB * NC * ND);
#pragma unroll
    for (int i = 0; i < NA * NB * NC * ND; ++i) o[i] = V[i];
    int* m = args.raw_meta + 4 * tl;
    m[0] = fa; m[1] = fb; m[2] = fc; m[3] = fd;
    return;
  }
  if (args.mode == MODE_SCHWARZ) {
    if (!active) return;
    double mx = 0.0;
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int b = 0; b < NB; ++b)
        if constexpr (NA == NC && NB == ND) mx = fmax(mx, fabs(V[((a * NB + b) * NC + a) * ND + b]));
    args.schwarz_out[p] = sqrt(mx);
    return;
  }

  // ---- 8-fold symmetric digestion: J' += 2 s g D, K' += s g D ----
  const double sym = active ? quartet_weight(blk, p, q) : 0.0;
  const SysMats mats = sys_mats(args, blk, p);
  const double* __restrict__ D = mats.D;
  const int nbf = mats.nbf;
  double* __restrict__ J = mats.J;
  double* __restrict__ K = mats.K;
  {  // J_ij[a][b] = sum_cd V D_kl
    double Dk[NC * ND];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int d = 0; d < ND; ++d) Dk[c * ND + d] = __ldg(D + (size_t)(fc + c) * nbf + fd + d);
#pragma unroll
    for (int ab = 0; ab < NA * NB; ++ab) {
      double v = 0.0;
#pragma unroll
      for (int cd = 0; cd < NC * ND; ++cd) v += V[ab * NC * ND + cd] * Dk[cd];
      v *= 2.0 * sym;
      if (uniform_bra) {  // every lane has the same bra pair: one atomic per warp
        v = warp_sum(v);
        if ((threadIdx.x & 31) == 0) atomicAdd(J + (size_t)(fa + ab / NB) * nbf + fb + ab % NB, v);
      } else if (active) {
        atomicAdd(J + (size_t)(fa + ab / NB) * nbf + fb + ab % NB, v);
      }
    }
  }
  {  // J_kl[c][d] = sum_ab V D_ij
    double Di[NA * NB];
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int b = 0; b < NB; ++b) Di[a * NB + b] = __ldg(D + (size_t)(fa + a) * nbf + fb + b);
#pragma unroll
    for (int cd = 0; cd < NC * ND; ++cd) {
      double v = 0.0;
#pragma unroll
      for (int ab = 0; ab < NA * NB; ++ab) v += V[ab * NC * ND + cd] * Di[ab];
      if (active) atomicAdd(J + (size_t)(fc + cd / ND) * nbf + fd + cd % ND, 2.0 * sym * v);
    }
  }
  {  // K_ik[a][c] = sum_bd V D_jl
    double Dx[NB * ND];
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
      for (int d = 0; d < ND; ++d) Dx[b * ND + d] = __ldg(D + (size_t)(fb + b) * nbf + fd + d);
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        double v = 0.0;
#pragma unroll
        for (int b = 0; b < NB; ++b)
#pragma unroll
          for (int d = 0; d < ND; ++d) v += V[((a * NB + b) * NC + c) * ND + d] * Dx[b * ND + d];
        if (active) atomicAdd(K + (size_t)(fa + a) * nbf + fc + c, sym * v);
      }
  }
  {  // K_il[a][d] = sum_bc V D_jk
    double Dx[NB * NC];
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
      for (int c = 0; c < NC; ++c) Dx[b * NC + c] = __ldg(D + (size_t)(fb + b) * nbf + fc + c);
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        double v = 0.0;
#pragma unroll
        for (int b = 0; b < NB; ++b)
#pragma unroll
          for (int c = 0; c < NC; ++c) v += V[((a * NB + b) * NC + c) * ND + d] * Dx[b * NC + c];
        if (active) atomicAdd(K + (size_t)(fa + a) * nbf + fd + d, sym * v);
      }
  }
  {  // K_jk[b][c] = sum_ad V D_il
    double Dx[NA * ND];
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int d = 0; d < ND; ++d) Dx[a * ND + d] = __ldg(D + (size_t)(fa + a) * nbf + fd + d);
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        double v = 0.0;
#pragma unroll
        for (int a = 0; a < NA; ++a)
#pragma unroll
          for (int d = 0; d < ND; ++d) v += V[((a * NB + b) * NC + c) * ND + d] * Dx[a * ND + d];
        if (active) atomicAdd(K + (size_t)(fb + b) * nbf + fc + c, sym * v);
      }
  }
  {  // K_jl[b][d] = sum_ac V D_ik
    double Dx[NA * NC];
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
      for (int c = 0; c < NC; ++c) Dx[a * NC + c] = __ldg(D + (size_t)(fa + a) * nbf + fc + c);
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        double v = 0.0;
#pragma unroll
        for (int a = 0; a < NA; ++a)
#pragma unroll
          for (int c = 0; c < NC; ++c) v += V[((a * NB + b) * NC + c) * ND + d] * Dx[a * NC + c];
        if (active) atomicAdd(K + (size_t)(fb + b) * nbf + fd + d, sym * v);
      }
  }
}

// Blocks per SM the register allocation must allow (ptxas caps registers at
// 65536 / (256 * blocks)).  The light classes are latency bound with short
// dependent chains and need the warps: in FP64 (ss|ss) fits 64 registers (4
// blocks, 32 warps; at 3 blocks it takes 72 without spilling and runs 1-2 % slower);
// (ps|ss), with the first ket primitive held across its bra
// rows, takes up to 128 without spilling (2 blocks; measured faster than 80
// registers with spills at 3 blocks); in FP32 the one-root classes fit 64 and the
// L = 2 ones, with their compensated accumulators, 128 (2 blocks).  FP64 (dp|ss)
// and (fs|ss) fit 128 without spilling (left free, ptxas takes 178 for (dp|ss) and
// the class runs 19 % slower on one block).  The other classes keep ptxas's own
// choice (0 = no bound; an explicit 1 would let it take up to 255 registers):
// capping the other L = 3 and 4 classes at 128 registers (2 blocks) measured
// slower in both precisions, (pp|ps) FP64 127 -> 154 ms.
template <int LA, int LB, int LC, int LD, typename R>
__host__ __device__ constexpr int small_min_blocks() {
  constexpr int L = LA + LB + LC + LD;
  return sizeof(R) == 8 ? (L == 0 ? 4 : L == 1 ? 2 : (LA + LB == 3 && LC + LD == 0) ? 2 : 0)
                        : (L <= 1 ? 4 : L == 2 ? 2 : 0);
}

template <int LA, int LB, int LC, int LD, typename R, bool SPLIT>
__global__ void __launch_bounds__(256, (small_min_blocks<LA, LB, LC, LD, R>()))
    eri_small_kernel(QuartetBlock blk, JKArgs args, RysTablesView tab, int kSuper, int ps) {
  constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* stab = reinterpret_cast<R*>(smem_raw);
  if constexpr (sizeof(R) == 4) stage_table_f32<NR>(reinterpret_cast<float*>(smem_raw), tab);
  else stage_table<NR, R>(stab, tab);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  if (!SPLIT) ps = 1;
  const int qpw = 32 / ps;  // quartets per warp chunk
  const int slot = lane / ps, sub = lane & (ps - 1);
  const int64_t nq = blk.total - blk.t_begin;
  const int64_t nchunks = (nq + qpw - 1) / qpw;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int nbra = blk.bra.npairs;
  // grid-stride over super-chunks of kSuper chunks (load balance), one bra search
  // per super-chunk, then the bra index only moves forward
  const int64_t nsuper = (nchunks + kSuper - 1) / kSuper;
  for (int64_t sc = wid; sc < nsuper; sc += nw) {
    const int64_t c1 = min(nchunks, (sc + 1) * kSuper);
    int pw = -1;  // bra pair of the current chunk's first quartet
    for (int64_t c = sc * kSuper; c < c1; ++c) {
      const int64_t t0 = blk.t_begin + c * qpw;
      const int64_t t = t0 + slot;
      const bool active = t < blk.total;
      const int64_t te = active ? t : blk.total - 1;
      if (pw < 0) {
        if (lane == 0) pw = find_bra(blk.offsets, nbra, t0);
        pw = __shfl_sync(0xffffffffu, pw, 0);
      } else {
        while (t0 >= __ldg(blk.offsets + pw + 1)) ++pw;
      }
      int p = pw;
      while (te >= __ldg(blk.offsets + p + 1)) ++p;
      const bool uniform = __all_sync(0xffffffffu, p == pw);
      small_quartet<LA, LB, LC, LD, R, SPLIT>(blk, args, tab, stab, te, p, active, uniform,
                                              SPLIT ? ps : 1, SPLIT ? sub : 0);
    }
  }
}

}  // namespace

namespace small_detail {

template <int LA, int LB, int LC, int LD>
int launch_one(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab,
               cudaStream_t stream, bool fp32, int num_sms, LaunchTune tune) {
  constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
  const int threads = 256;
  const size_t smem = fp32 ? f32_table_bytes<NR>() : table_bytes<NR, double>();
  const int64_t nq = blk.total - blk.t_begin;
  if (nq <= 0) return 1;
  // lanes per quartet: split the bra primitive loop when the launch has too few
  // quartets to fill the device (primitive-heavy classes such as (s9 s9|s9 s9))
  const int Kab = blk.bra.Ka * blk.bra.Kb;
  int ps = 1;
  while (ps < 32 && ps < Kab && nq * ps < (int64_t)num_sms * 1024) ps <<= 1;
  if (tune.ps > 0) ps = tune.ps;
  const int64_t nchunks = (nq + 32 / ps - 1) / (32 / ps);
  // separate instantiations keep the unsplit kernel's register allocation
  // independent of the split one
  const int v = (fp32 ? 2 : 0) + (ps > 1 ? 1 : 0);
  void (*const kerns[4])(QuartetBlock, JKArgs, RysTablesView, int, int) = {
      eri_small_kernel<LA, LB, LC, LD, double, false>, eri_small_kernel<LA, LB, LC, LD, double, true>,
      eri_small_kernel<LA, LB, LC, LD, float, false>, eri_small_kernel<LA, LB, LC, LD, float, true>};
  auto kern = kerns[v];
  static bool attr[4] = {false, false, false, false};
  static int per_sm_cache[4] = {0, 0, 0, 0};
  if (!attr[v]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return -3;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_cache[v], kern, threads, smem) != cudaSuccess)
      return -3;
    attr[v] = true;
  }
  const int per_sm = per_sm_cache[v] > 0 ? per_sm_cache[v] : 1;
  const int64_t want = (nchunks + (threads / 32) - 1) / (threads / 32);
  const int64_t cap = (int64_t)num_sms * per_sm;
  const int grid = (int)(want < cap ? want : cap);
  // chunks per super-chunk (consecutive chunks a warp takes, one bra search per
  // super-chunk; the warp stays on neighbouring bra pairs and ket rows).  On the
  // large launches of (H2O)64/cc-pVDZ the autotuner chose 16 where a quartet has
  // at most 9 primitive quartets and 4 above; a launch keeps at least 8
  // super-chunks per warp for load balance, so small launches stay at 1.
  int ksuper = tune.ksuper;
  if (ksuper <= 0) {
    const int64_t warps = (int64_t)grid * (threads / 32);
    const int64_t kmax = (int64_t)Kab * blk.ket.Ka * blk.ket.Kb <= 9 ? 16 : 4;
    ksuper = (int)std::max<int64_t>(1, std::min<int64_t>(kmax, nchunks / (warps * 8)));
  }
  kern<<<grid, threads, smem, stream>>>(blk, args, tab, ksuper, ps);
  return cudaGetLastError() == cudaSuccess ? 1 : -3;
}

}  // namespace small_detail

}  // namespace lai
