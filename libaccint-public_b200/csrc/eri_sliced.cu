// Bra-sliced Rys ERI kernels with fused J/K digestion for the medium classes
// (the (e0|f0) block of one quartet is too large for one thread's registers,
// e.g. (dp|pp), (dp|dp), (dd|ps), (dd|ds)).
//
// A group of TW = na lanes works on one quartet (32 / na groups per warp, the
// remaining 32 mod na lanes idle); lane a of the group
// owns Cartesian component a of the bra's first shell.  Every lane evaluates the
// roots and the full 2D tables of each primitive quartet (cheap next to the
// assembly for these classes), then accumulates only the rows of (e0|f0) its
// component needs, e = a + k for |k| <= lb, so no data moves between lanes
// until digestion.  Lane a then forms its outputs (a b|c d) for all b, c, d by
// the closed-form transfer (eri_device.cuh) and digests them:
//   J_ij[a][b], K_ik[a][c], K_il[a][d]   complete in the lane -> atomics;
//   J_kl, K_jk, K_jl                      partial over a -> shuffle sum over
//                                         the group, then one atomic per entry.
// The lane-dependent row offset a is applied by selecting rows of the 2D tables
// (compile-time-indexed registers) instead of indexing them at run time.
#include <cuda_runtime.h>

#include <algorithm>
#include <type_traits>

#include "eri_device.cuh"
#include "eri_kernels.h"
#include "eri_tables_smem.cuh"

namespace lai {

namespace {

template <int B, int E, typename F>
__device__ __forceinline__ void sfor(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    sfor<B + 1, E>(f);
  }
}

__host__ __device__ constexpr int next_pow2(int x) {
  int p = 1;
  while (p < x) p <<= 1;
  return p;
}

// Reduction over the TW lanes g*TW .. g*TW+TW-1 of a group (TW need not be a power of
// two) into the group's lane a == 0 (the other lanes' results are partial): the lanes
// past the largest power of two P < TW fold onto the first ones, then a halving tree.
template <int TW, typename T, typename Op>
__device__ __forceinline__ T group_reduce(T v, int a, Op op) {
  constexpr int P = next_pow2(TW) == TW ? TW / 2 : next_pow2(TW) / 2;
  if constexpr (P * 2 > TW) {
    const T u = __shfl_down_sync(0xffffffffu, v, P);
    if (a + P < TW) v = op(v, u);
  } else {
    v = op(v, __shfl_down_sync(0xffffffffu, v, P));
  }
#pragma unroll
  for (int o = P / 2; o > 0; o >>= 1) v = op(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void sliced_quartet(const QuartetBlock& blk, const JKArgs& args,
                                               const RysTablesView& tab,
                                               const R* __restrict__ stab, int64_t t, int p,
                                               bool active, int a) {
  constexpr int LAB = LA + LB, LCD = LC + LD;
  constexpr int NR = (LAB + LCD) / 2 + 1;
  constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
  constexpr int NF = ncart_range(LC, LCD);
  constexpr int NK = ncart_range(0, LB);  // shifts k with |k| <= lb
  constexpr int TW = NA;
  constexpr int W = LCD + 1;
  const int nbra = blk.bra.npairs, nket = blk.ket.npairs;
  const int q = (blk.qbegin ? __ldg(blk.qbegin + p) : 0) + (int)(t - __ldg(blk.offsets + p));
  const bool own = active && a < NA;
  const int ac = cart_comp(LA, a < NA ? a : 0);
  const int ax = comp_x(ac), ay = comp_y(ac), az = comp_z(ac);

  const int Kab = blk.bra.Ka * blk.bra.Kb;
  const int Kcd = blk.ket.Ka * blk.ket.Kb;
  (void)nbra;

  R G[NK * NF];
#pragma unroll
  for (int i = 0; i < NK * NF; ++i) G[i] = R(0);

  // FP32 quartets (fp32_prim_rel > 0): primitive quartets below that fraction of the
  // quartet's own Schwarz bound are skipped as well
  const double peps = (sizeof(R) == 4 && args.prim_rel32 > 0.0)
                          ? fmax(args.prim_eps, args.prim_rel32 * __ldg(blk.bra.Q + p) * __ldg(blk.ket.Q + q))
                          : args.prim_eps;
  unsigned int nprim_done = 0;
  for (int ib = 0; ib < Kab; ++ib) {
    // the bra pair's primitive record (BraRecField): the lanes of a quartet group
    // (and usually the whole warp) read the same contiguous record
    const double2* rb = reinterpret_cast<const double2*>(blk.bra.primb + ((size_t)p * Kab + ib) * kBraRec);
    const double2 b0 = __ldg(rb), b1 = __ldg(rb + 1);
    // primitive pairs are sorted by their Schwarz bound: once the bra bound times
    // the largest ket bound of the class drops below the cut, the rest do too
    const double qab = b0.x;
    if (qab * blk.ket.qprim_max < peps) break;
    const double2 b2 = __ldg(rb + 2), b3 = __ldg(rb + 3), b4 = __ldg(rb + 4), b5 = __ldg(rb + 5);
    const R zeta = R(b0.y);
    const R hz = R(b1.x);
    // P - Q in FP64 on both paths (centres are O(10) bohr)
    const double Px = b2.x, Py = b2.y, Pz = b3.x;
    const R PAx = R(b4.x), PAy = R(b4.y), PAz = R(b5.x);
    const R cab = R(b1.y);
    const double* pkt = ket_tile_ptr(blk.ket.primk, q, Kcd);
    KetPrim nxt;
    load_ket_rec(pkt, nxt);
    for (int ik = 0; ik < Kcd; ++ik) {
      const KetPrim cur = nxt;
      if (qab * cur.q < peps) break;  // sorted: the rest are smaller
      if (ik + 1 < Kcd) load_ket_rec(pkt + (size_t)(ik + 1) * kKetPrimStride, nxt);
      ++nprim_done;
      const R eta = R(cur.eta);
      const R he = R(cur.he);
      const R PQx = R(Px - cur.px);
      const R PQy = R(Py - cur.py);
      const R PQz = R(Pz - cur.pz);
      const R QCx = R(cur.qcx), QCy = R(cur.qcy), QCz = R(cur.qcz);
      const R ccd = R(cur.c);
      const R s = zeta + eta;
      const R rs = fast_rsqrt(s);
      const R inv = rs * rs;
      const R rz = eta * inv, re = zeta * inv;
      const R T = zeta * rz * (PQx * PQx + PQy * PQy + PQz * PQz);
      const R pref = cab * ccd * rs;
      R u[NR], w[NR];
      rys_smem<NR, R>(T, stab, tab, u, w);
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const R ur = u[r];
        const R b00 = R(0.5) * inv * ur;
        const R b10 = hz - hz * rz * ur;
        const R b01 = he - he * re * ur;
        const R pa[3] = {PAx - rz * ur * PQx, PAy - rz * ur * PQy, PAz - rz * ur * PQz};
        const R qc[3] = {QCx + re * ur * PQx, QCy + re * ur * PQy, QCz + re * ur * PQz};
        const int sh[3] = {ax, ay, az};
        R S[3][LB + 1][W];  // rows a_x + j of the 2D table, j <= lb
#pragma unroll
        for (int x = 0; x < 3; ++x) {
          R I[LAB + 1][W];
          I[0][0] = (x == 2) ? w[r] * pref : R(1);
#pragma unroll
          for (int e = 0; e < LAB; ++e)
            I[e + 1][0] = pa[x] * I[e][0] + (e ? R(e) * b10 * I[e > 0 ? e - 1 : 0][0] : R(0));
#pragma unroll
          for (int f = 0; f < LCD; ++f)
#pragma unroll
            for (int e = 0; e <= LAB; ++e)
              I[e][f + 1] = qc[x] * I[e][f] + (f ? R(f) * b01 * I[e][f > 0 ? f - 1 : 0] : R(0)) +
                            (e ? R(e) * b00 * I[e > 0 ? e - 1 : 0][f] : R(0));
          // select rows sh[x] + j (sh[x] in [0, LA]) without run-time indexing
#pragma unroll
          for (int j = 0; j <= LB; ++j)
#pragma unroll
            for (int f = 0; f <= LCD; ++f) {
              R v = I[j][f];
#pragma unroll
              for (int o = 1; o <= LA; ++o)
                if (sh[x] == o) v = I[o + j][f];
              S[x][j][f] = v;
            }
        }
        sfor<0, NK>([&](auto IK) {
          constexpr int k = decltype(IK)::value;
          constexpr int lk = [] { int l = 0, r = k; while (r >= ncart(l)) { r -= ncart(l); ++l; } return l; }();
          constexpr int ck = cart_comp(lk, k - ncart_before(0, lk));
          sfor<0, NF>([&](auto JF) {
            constexpr int jf = decltype(JF)::value;
            constexpr int lf = [] { int l = LC, r = jf; while (r >= ncart(l)) { r -= ncart(l); ++l; } return l; }();
            constexpr int cf = cart_comp(lf, jf - ncart_before(LC, lf));
            G[k * NF + jf] += S[0][comp_x(ck)][comp_x(cf)] * S[1][comp_y(ck)][comp_y(cf)] *
                              S[2][comp_z(ck)][comp_z(cf)];
          });
        });
      }
    }
  }

  count_prims(args.prim_count, (active && a == 0) ? nprim_done : 0u);

  // ---- transfer: H[b][f] = sum_{k<=b} C(b,k) AB^(b-k) G[k][f]; V[b][c][d] ----
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
  double H[NB * NF];
  sfor<0, NB>([&](auto IB) {
    constexpr int b = decltype(IB)::value;
    constexpr int cb = cart_comp(LB, b);
#pragma unroll
    for (int f = 0; f < NF; ++f) H[b * NF + f] = 0.0;
    sfor<0, comp_x(cb) + 1>([&](auto KX) {
      constexpr int kx = decltype(KX)::value;
      sfor<0, comp_y(cb) + 1>([&](auto KY) {
        constexpr int ky = decltype(KY)::value;
        sfor<0, comp_z(cb) + 1>([&](auto KZ) {
          constexpr int kz = decltype(KZ)::value;
          constexpr int row = ncart_before(0, kx + ky + kz) + cart_index(kx, ky, kz);
          constexpr double bc = binom(comp_x(cb), kx) * binom(comp_y(cb), ky) * binom(comp_z(cb), kz);
          const double cf = bc * abp[0][comp_x(cb) - kx] * abp[1][comp_y(cb) - ky] * abp[2][comp_z(cb) - kz];
#pragma unroll
          for (int f = 0; f < NF; ++f) H[b * NF + f] += cf * double(G[row * NF + f]);
        });
      });
    });
  });
  double V[NB * NC * ND];
  sfor<0, NC>([&](auto IC) {
    constexpr int c = decltype(IC)::value;
    constexpr int cc = cart_comp(LC, c);
    sfor<0, ND>([&](auto ID) {
      constexpr int d = decltype(ID)::value;
      constexpr int cd = cart_comp(LD, d);
#pragma unroll
      for (int b = 0; b < NB; ++b) V[(b * NC + c) * ND + d] = 0.0;
      sfor<0, comp_x(cd) + 1>([&](auto KX) {
        constexpr int kx = decltype(KX)::value;
        sfor<0, comp_y(cd) + 1>([&](auto KY) {
          constexpr int ky = decltype(KY)::value;
          sfor<0, comp_z(cd) + 1>([&](auto KZ) {
            constexpr int kz = decltype(KZ)::value;
            constexpr int fx = comp_x(cc) + kx, fy = comp_y(cc) + ky, fz = comp_z(cc) + kz;
            constexpr int col = ncart_before(LC, fx + fy + fz) + cart_index(fx, fy, fz);
            constexpr double bc = binom(comp_x(cd), kx) * binom(comp_y(cd), ky) * binom(comp_z(cd), kz);
            const double cf = bc * cdp[0][comp_x(cd) - kx] * cdp[1][comp_y(cd) - ky] * cdp[2][comp_z(cd) - kz];
#pragma unroll
            for (int b = 0; b < NB; ++b) V[(b * NC + c) * ND + d] += cf * H[b * NF + col];
          });
        });
      });
      // normalization of b, c, d (a is applied below)
      constexpr double den_cd = dfact_odd(comp_x(cc)) * dfact_odd(comp_y(cc)) * dfact_odd(comp_z(cc)) *
                                dfact_odd(comp_x(cd)) * dfact_odd(comp_y(cd)) * dfact_odd(comp_z(cd));
      sfor<0, NB>([&](auto IB) {
        constexpr int b = decltype(IB)::value;
        constexpr int cb = cart_comp(LB, b);
        constexpr double den = den_cd * dfact_odd(comp_x(cb)) * dfact_odd(comp_y(cb)) * dfact_odd(comp_z(cb));
        if constexpr (den != 1.0) V[(b * NC + c) * ND + d] *= rsqrt(den);
      });
    });
  });
  {
    const double na = rsqrt(dfact_odd(ax) * dfact_odd(ay) * dfact_odd(az));
#pragma unroll
    for (int i = 0; i < NB * NC * ND; ++i) V[i] *= na;
  }

  const int fa = __ldg(blk.bra.func_a + p), fb = __ldg(blk.bra.func_b + p);
  const int fc = __ldg(blk.ket.func_a + q), fd = __ldg(blk.ket.func_b + q);
  if (args.mode == MODE_RAW) {
    if (!own) return;
    const int64_t tl = t - blk.t_begin;
    double* o = args.raw_out + (size_t)tl * (NA * NB * NC * ND) + (size_t)a * (NB * NC * ND);
#pragma unroll
    for (int i = 0; i < NB * NC * ND; ++i) o[i] = V[i];
    if (a == 0) {
      int* m = args.raw_meta + 4 * tl;
      m[0] = fa; m[1] = fb; m[2] = fc; m[3] = fd;
    }
    return;
  }
  if (args.mode == MODE_SCHWARZ) {
    double mx = 0.0;
    if constexpr (NA == NC && NB == ND) {
      // (ab|ab): c == a
#pragma unroll
      for (int c = 0; c < NC; ++c)
        if (c == a)
#pragma unroll
          for (int b = 0; b < NB; ++b) mx = fmax(mx, fabs(V[(b * NC + c) * ND + b]));
    }
    mx = group_reduce<TW>(mx, a, [](double x, double y) { return fmax(x, y); });
    if (active && a == 0) args.schwarz_out[p] = sqrt(mx);
    return;
  }

  const double sym = own ? quartet_weight(blk, p, q) : 0.0;
  const SysMats mats = sys_mats(args, blk, p);
  const double* __restrict__ D = mats.D;
  const int nbf = mats.nbf;
  double* __restrict__ J = mats.J;
  double* __restrict__ K = mats.K;
  const int arow = fa + (a < NA ? a : 0);
  // lane-complete targets
  {
    double Dk[NC * ND];
#pragma unroll
    for (int c = 0; c < NC; ++c)
#pragma unroll
      for (int d = 0; d < ND; ++d) Dk[c * ND + d] = __ldg(D + (size_t)(fc + c) * nbf + fd + d);
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      double v = 0.0;
#pragma unroll
      for (int cd = 0; cd < NC * ND; ++cd) v += V[b * NC * ND + cd] * Dk[cd];
      if (own) atomicAdd(J + (size_t)arow * nbf + fb + b, 2.0 * sym * v);
    }
  }
  {
    double Dx[NB * ND];
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
      for (int d = 0; d < ND; ++d) Dx[b * ND + d] = __ldg(D + (size_t)(fb + b) * nbf + fd + d);
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      double v = 0.0;
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int d = 0; d < ND; ++d) v += V[(b * NC + c) * ND + d] * Dx[b * ND + d];
      if (own) atomicAdd(K + (size_t)arow * nbf + fc + c, sym * v);
    }
  }
  {
    double Dx[NB * NC];
#pragma unroll
    for (int b = 0; b < NB; ++b)
#pragma unroll
      for (int c = 0; c < NC; ++c) Dx[b * NC + c] = __ldg(D + (size_t)(fb + b) * nbf + fc + c);
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      double v = 0.0;
#pragma unroll
      for (int b = 0; b < NB; ++b)
#pragma unroll
        for (int c = 0; c < NC; ++c) v += V[(b * NC + c) * ND + d] * Dx[b * NC + c];
      if (own) atomicAdd(K + (size_t)arow * nbf + fd + d, sym * v);
    }
  }
  // partial-over-a targets: group sum into lane a == 0, which does the atomics
  {  // J_kl[c][d] = 2 s sum_a sum_b V D_ij[a][b]
    double Di[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) Di[b] = __ldg(D + (size_t)arow * nbf + fb + b);
#pragma unroll
    for (int cd = 0; cd < NC * ND; ++cd) {
      double v = 0.0;
#pragma unroll
      for (int b = 0; b < NB; ++b) v += V[b * NC * ND + cd] * Di[b];
      v *= 2.0 * sym;
      v = group_reduce<TW>(v, a, [](double x, double y) { return x + y; });
      if (active && a == 0)
        atomicAdd(J + (size_t)(fc + cd / ND) * nbf + fd + cd % ND, v);
    }
  }
  {  // K_jk[b][c] = s sum_a sum_d V D_il[a][d]
    double Dl[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) Dl[d] = __ldg(D + (size_t)arow * nbf + fd + d);
#pragma unroll
    for (int bc = 0; bc < NB * NC; ++bc) {
      double v = 0.0;
#pragma unroll
      for (int d = 0; d < ND; ++d) v += V[bc * ND + d] * Dl[d];
      v *= sym;
      v = group_reduce<TW>(v, a, [](double x, double y) { return x + y; });
      if (active && a == 0)
        atomicAdd(K + (size_t)(fb + bc / NC) * nbf + fc + bc % NC, v);
    }
  }
  {  // K_jl[b][d] = s sum_a sum_c V D_ik[a][c]
    double Dc[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) Dc[c] = __ldg(D + (size_t)arow * nbf + fc + c);
#pragma unroll
    for (int bd = 0; bd < NB * ND; ++bd) {
      const int b = bd / ND, d = bd % ND;
      double v = 0.0;
#pragma unroll
      for (int c = 0; c < NC; ++c) v += V[(b * NC + c) * ND + d] * Dc[c];
      v *= sym;
      v = group_reduce<TW>(v, a, [](double x, double y) { return x + y; });
      if (active && a == 0)
        atomicAdd(K + (size_t)(fb + b) * nbf + fd + d, v);
    }
  }
}

template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(128) eri_sliced_kernel(QuartetBlock blk, JKArgs args,
                                                         RysTablesView tab, int kSuper) {
  constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
  constexpr int TW = ncart(LA);
  constexpr int QPW = 32 / TW;  // quartets per warp (lanes QPW * TW .. 31 idle)
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* stab = reinterpret_cast<R*>(smem_raw);
  stage_table<NR, R>(stab, tab);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int slot = lane / TW, a = lane % TW;
  const int64_t nq = blk.total - blk.t_begin;
  const int64_t nchunks = (nq + QPW - 1) / QPW;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int nbra = blk.bra.npairs;
  const int64_t nsuper = (nchunks + kSuper - 1) / kSuper;
  for (int64_t sc = wid; sc < nsuper; sc += nw) {
    const int64_t c1 = min(nchunks, (sc + 1) * kSuper);
    int pw = -1;
    for (int64_t c = sc * kSuper; c < c1; ++c) {
      const int64_t t0 = blk.t_begin + c * QPW;
      const int64_t t = t0 + slot;
      const bool active = slot < QPW && t < blk.total;
      // idle lanes take the chunk's first quartet (t0 < total), whose bra pair the
      // warp already holds
      const int64_t te = active ? t : t0;
      if (pw < 0) {
        if (lane == 0) pw = find_bra(blk.offsets, nbra, t0);
        pw = __shfl_sync(0xffffffffu, pw, 0);
      } else {
        while (t0 >= __ldg(blk.offsets + pw + 1)) ++pw;
      }
      int p = pw;
      while (te >= __ldg(blk.offsets + p + 1)) ++p;
      sliced_quartet<LA, LB, LC, LD, R>(blk, args, tab, stab, te, p, active, a);
    }
  }
}

template <int LA, int LB, int LC, int LD>
int launch_one(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab,
               cudaStream_t stream, bool fp32, int num_sms) {
  constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
  constexpr int QPW = 32 / ncart(LA);
  const int threads = 128;
  const size_t smem = fp32 ? table_bytes<NR, float>() : table_bytes<NR, double>();
  const int64_t nchunks = (blk.total - blk.t_begin + QPW - 1) / QPW;
  if (nchunks <= 0) return 1;
  auto kern = fp32 ? eri_sliced_kernel<LA, LB, LC, LD, float> : eri_sliced_kernel<LA, LB, LC, LD, double>;
  static bool attr[2] = {false, false};
  static int per_sm_cache[2] = {0, 0};
  if (!attr[fp32]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return -3;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_cache[fp32], kern, threads, smem) != cudaSuccess)
      return -3;
    attr[fp32] = true;
  }
  const int per_sm = per_sm_cache[fp32] > 0 ? per_sm_cache[fp32] : 1;
  const int64_t want = (nchunks + (threads / 32) - 1) / (threads / 32);
  const int64_t cap = (int64_t)num_sms * per_sm;
  const int grid = (int)(want < cap ? want : cap);
  // chunks per super-chunk: long runs (one bra search each) when the launch has
  // plenty of work, short ones when it would otherwise leave warps idle
  const int64_t warps_total = (int64_t)grid * (threads / 32);
  const int ksuper = (int)std::max<int64_t>(1, std::min<int64_t>(16, nchunks / (8 * warps_total)));
  kern<<<grid, threads, smem, stream>>>(blk, args, tab, ksuper);
  return cudaGetLastError() == cudaSuccess ? 1 : -3;
}

}  // namespace

#define LAI_SLICED_CLASSES(X) X(2, 1, 1, 1) X(2, 1, 2, 1) X(2, 2, 2, 0)

bool sliced_class_supported(int la, int lb, int lc, int ld) {
#define X(a, b, c, d) if (la == a && lb == b && lc == c && ld == d) return true;
  LAI_SLICED_CLASSES(X)
#undef X
  return false;
}

int launch_sliced(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab,
                  cudaStream_t stream, bool fp32, int num_sms) {
  const int la = blk.bra.la, lb = blk.bra.lb, lc = blk.ket.la, ld = blk.ket.lb;
#define X(a, b, c, d) \
  if (la == a && lb == b && lc == c && ld == d) return launch_one<a, b, c, d>(blk, args, tab, stream, fp32, num_sms);
  LAI_SLICED_CLASSES(X)
#undef X
  return 0;
}

}  // namespace lai
