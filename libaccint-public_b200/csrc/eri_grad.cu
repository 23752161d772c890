// Nuclear gradient of the two-electron energy at fixed density,
//   E = 1/2 tr(D J[D]) - 1/4 tr(D K[D]),
//   dE/dR = sum over canonical quartets of s * sum_abcd d(ab|cd)/dR * G_abcd,
//   G_abcd = 4 D_ab D_cd - D_ac D_bd - D_ad D_bc,
// with s the degeneracy weight of the quartet (1/2 per i==j, k==l, ij==kl) -- the
// same canonical quartet list and weights as the J/K build, so the gradient is
// that of exactly the energy the build defines.  No derivative integral is stored:
// they are contracted with G as they are formed.  The reference has no derivative
// integrals (MAX_DERIVATIVE_ORDER = 0, config.hpp.in:49).
//
// Derivatives (Rys quadrature, per primitive quartet and root, per direction x):
//   d/dA_x phi_a = 2 alpha phi_{a+1x} - a_x phi_{a-1x}   (alpha: exponent on A)
// and likewise for B and C; D follows from translational invariance,
//   dE/dD = -(dE/dA + dE/dB + dE/dC).
// The 2D integrals I(a, b, c, d) with a <= la+1, b <= lb+1, c <= lc+1, d <= ld+1
// (a+b <= la+lb+1, c+d <= lc+ld+1) come from the vertical recurrence up to
// e = la+lb+1, f = lc+ld+1 (the same recurrence as eri_device.cuh) and the
// horizontal transfer I(a, b+1) = I(a+1, b) + AB_x I(a, b) on both sides; the
// root count is that of total angular momentum L+1.
//
// One warp per quartet: lanes 3 r + x build the tables of root r and direction x in
// shared memory (all roots at once where shared memory allows), then all lanes
// sweep the quartet's Cartesian components over those roots, each keeping nine
// partial derivatives (A, B, C x xyz), reduced over the warp at the end.  (The low
// classes run on the thread-per-quartet kernels of eri_grad_small.cuh.)
#include <cuda_runtime.h>

#include <algorithm>

#include "eri_device.cuh"
#include "eri_kernels.h"

namespace lai {

namespace {

struct GradGeom {
  int la, lb, lc, ld;
  int na, nb, nc, nd, nel;
  int LABp, LCDp;          // la+lb+1, lc+ld+1
  int EA, EB, EC, ED;      // la+2, lb+2, lc+2, ld+1 (d is never raised)
  int n;                   // roots
  int vsz, xsz, hsz;       // (LABp+1)(LCDp+1), EA*EB*(LCDp+1), EA*EB*EC*ED
  int off_v, off_x, off_h, off_g, per_warp;  // shared memory per warp (doubles)
  int gamma_global;        // G_abcd kept in global scratch instead of shared memory
  int rb;                  // roots whose tables are built at once (lanes 3 r + x, r < rb)
};

GradGeom make_grad_geom(int la, int lb, int lc, int ld, int warps, size_t smem_max) {
  GradGeom g{};
  g.la = la; g.lb = lb; g.lc = lc; g.ld = ld;
  g.na = ncart(la); g.nb = ncart(lb); g.nc = ncart(lc); g.nd = ncart(ld);
  g.nel = g.na * g.nb * g.nc * g.nd;
  g.LABp = la + lb + 1; g.LCDp = lc + ld + 1;
  g.EA = la + 2; g.EB = lb + 2; g.EC = lc + 2; g.ED = ld + 1;
  g.n = (la + lb + lc + ld + 1) / 2 + 1;
  g.vsz = (g.LABp + 1) * (g.LCDp + 1);
  g.xsz = g.EA * g.EB * (g.LCDp + 1);
  g.hsz = g.EA * g.EB * g.EC * g.ED;
  // as many roots at once as shared memory allows (all of them for l <= 2), G in
  // shared memory if it fits beside them
  for (int rb = std::min(g.n, 10); rb >= 1; --rb)
    for (int glob = 0; glob <= 1; ++glob) {
      int o = 0;
      g.off_v = o; o += 3 * rb * g.vsz;
      g.off_x = o; o += 3 * rb * g.xsz;
      g.off_h = o; o += 3 * rb * g.hsz;
      g.off_g = o; o += glob ? 0 : g.nel;
      g.per_warp = (o + 1) & ~1;
      g.gamma_global = glob;
      g.rb = rb;
      if ((size_t)g.per_warp * 8 * warps <= smem_max) return g;
    }
  g.per_warp = -1;
  return g;
}

__device__ __forceinline__ int hidx(const GradGeom& g, int a, int b, int c, int d) {
  return ((a * g.EB + b) * g.EC + c) * g.ED + d;
}

struct GradArgs {
  const double* D;
  int nbf;
  const int* shell_atom;  // [nshell]
  double* grad;           // [natom][3], accumulated
  double prim_eps;
};

__global__ void __launch_bounds__(128) eri_grad_kernel(QuartetBlock blk, GradArgs ga, RysTablesView tab,
                                                       GradGeom g, double* gscratch) {
  extern __shared__ __align__(16) double smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int wpb = blockDim.x >> 5;
  double* ws = smem + (size_t)warp * g.per_warp;
  double* V = ws + g.off_v;  // [3][LABp+1][LCDp+1]
  double* X = ws + g.off_x;  // [3][EA][EB][LCDp+1]
  double* H = ws + g.off_h;  // [3][EA][EB][EC][ED]
  const int64_t gw = (int64_t)blockIdx.x * wpb + warp;
  double* Gam = g.gamma_global ? gscratch + (size_t)gw * g.nel : ws + g.off_g;
  const int64_t nwarps = (int64_t)gridDim.x * wpb;
  const int nbra = blk.bra.npairs, nket = blk.ket.npairs;
  const int Kab = blk.bra.Ka * blk.bra.Kb, Kcd = blk.ket.Ka * blk.ket.Kb;
  const size_t sb = (size_t)Kab * nbra, sk = (size_t)Kcd * nket;
  const int W = g.LCDp + 1;

  for (int64_t t = blk.t_begin + gw; t < blk.total; t += nwarps) {
    const int p = find_bra(blk.offsets, nbra, t);
    const int q = (blk.qbegin ? __ldg(blk.qbegin + p) : 0) + (int)(t - __ldg(blk.offsets + p));
    const int fa = __ldg(blk.bra.func_a + p), fb = __ldg(blk.bra.func_b + p);
    const int fc = __ldg(blk.ket.func_a + q), fd = __ldg(blk.ket.func_b + q);
    const double s = quartet_weight(blk, p, q);
    const double* __restrict__ D = ga.D;
    const size_t nbf = (size_t)ga.nbf;
    // G_abcd with the per-component normalization and the degeneracy weight
    for (int e = lane; e < g.nel; e += 32) {
      const int d = e % g.nd, c = (e / g.nd) % g.nc, b = (e / (g.nd * g.nc)) % g.nb,
                a = e / (g.nd * g.nc * g.nb);
      const double Dab = D[(fa + a) * nbf + fb + b], Dcd = D[(fc + c) * nbf + fd + d];
      const double Dac = D[(fa + a) * nbf + fc + c], Dbd = D[(fb + b) * nbf + fd + d];
      const double Dad = D[(fa + a) * nbf + fd + d], Dbc = D[(fb + b) * nbf + fc + c];
      const double nrm = norm_factor(g.la, a) * norm_factor(g.lb, b) * norm_factor(g.lc, c) *
                         norm_factor(g.ld, d);
      Gam[e] = s * nrm * (4.0 * Dab * Dcd - Dac * Dbd - Dad * Dbc);
    }
    const double ABx[3] = {__ldg(blk.bra.AB + p), __ldg(blk.bra.AB + nbra + p), __ldg(blk.bra.AB + 2 * nbra + p)};
    const double CDx[3] = {__ldg(blk.ket.AB + q), __ldg(blk.ket.AB + nket + q), __ldg(blk.ket.AB + 2 * nket + q)};
    double acc[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) acc[i] = 0.0;
    __syncwarp();

    for (int ib = 0; ib < Kab; ++ib) {
      const double* pb = blk.bra.prim + (size_t)ib * nbra + p;
      const double qab = __ldg(pb + PF_Q * sb);
      if (qab * blk.ket.qprim_max < ga.prim_eps) break;
      const double zeta = __ldg(pb + PF_ZETA * sb), hz = __ldg(pb + PF_HZ * sb);
      const double alpha = __ldg(pb + PF_ALPHA * sb), beta = zeta - alpha;
      const double P[3] = {__ldg(pb + PF_PX * sb), __ldg(pb + PF_PY * sb), __ldg(pb + PF_PZ * sb)};
      const double PA[3] = {__ldg(pb + PF_PAX * sb), __ldg(pb + PF_PAY * sb), __ldg(pb + PF_PAZ * sb)};
      const double cab = __ldg(pb + PF_C * sb);
      for (int ik = 0; ik < Kcd; ++ik) {
        const double* pk = blk.ket.prim + (size_t)ik * nket + q;
        const double qcd = __ldg(pk + PF_Q * sk);
        if (qab * qcd < ga.prim_eps) break;
        const double eta = __ldg(pk + PF_ZETA * sk), he = __ldg(pk + PF_HZ * sk);
        const double gamma = __ldg(pk + PF_ALPHA * sk);
        const double Q[3] = {__ldg(pk + PF_PX * sk), __ldg(pk + PF_PY * sk), __ldg(pk + PF_PZ * sk)};
        const double QC[3] = {__ldg(pk + PF_PAX * sk), __ldg(pk + PF_PAY * sk), __ldg(pk + PF_PAZ * sk)};
        const double ccd = __ldg(pk + PF_C * sk);
        const double PQ[3] = {P[0] - Q[0], P[1] - Q[1], P[2] - Q[2]};
        const double rs = rsqrt(zeta + eta);
        const double inv = rs * rs;
        const double rz = eta * inv, re = zeta * inv;
        const double T = zeta * rz * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
        const double pref = cab * ccd * rs;
        double u[kMaxRoots + 1], w[kMaxRoots + 1];
        rys_roots_table<double>(g.n, T, tab, u, w);
        for (int r0 = 0; r0 < g.n; r0 += g.rb) {
          const int nr = min(g.rb, g.n - r0);
          if (lane < 3 * nr) {  // vertical recurrence and transfers of root r0 + lane / 3, direction lane % 3
            const int rr = lane / 3, x = lane - 3 * rr;
            const double ur = u[r0 + rr];
            double* I = V + (rr * 3 + x) * g.vsz;
            const double b00 = 0.5 * inv * ur, b10 = hz - hz * rz * ur, b01 = he - he * re * ur;
            const double pa = PA[x] - rz * ur * PQ[x];
            const double qc = QC[x] + re * ur * PQ[x];
            I[0] = (x == 2) ? w[r0 + rr] * pref : 1.0;
            if (g.LABp > 0) I[W] = pa * I[0];
            for (int e = 1; e < g.LABp; ++e) I[(e + 1) * W] = pa * I[e * W] + e * b10 * I[(e - 1) * W];
            for (int f = 0; f < g.LCDp; ++f)
              for (int e = 0; e <= g.LABp; ++e) {
                double v = qc * I[e * W + f];
                if (f) v += f * b01 * I[e * W + f - 1];
                if (e) v += e * b00 * I[(e - 1) * W + f];
                I[e * W + f + 1] = v;
              }
            // horizontal transfer, bra then ket: X[a][b][f] (a < EA, b < EB), then
            // H[a][b][c][d] (c < EC, d < ED); I(a, b+1) = I(a+1, b) + AB I(a, b)
            double* Xx = X + (rr * 3 + x) * g.xsz;
            const int F = g.LCDp + 1;
            for (int f = 0; f <= g.LCDp; ++f) {
              double row[12];
              for (int a = 0; a <= g.LABp; ++a) row[a] = I[a * W + f];
              for (int a = 0; a < g.EA; ++a) Xx[(a * g.EB) * F + f] = row[a];
              for (int b = 1; b < g.EB; ++b) {
                for (int a = 0; a + b <= g.LABp; ++a) row[a] = row[a + 1] + ABx[x] * row[a];
                for (int a = 0; a < g.EA && a + b <= g.LABp; ++a) Xx[(a * g.EB + b) * F + f] = row[a];
              }
            }
            double* Hx = H + (rr * 3 + x) * g.hsz;
            for (int a = 0; a < g.EA; ++a)
              for (int b = 0; b < g.EB && a + b <= g.LABp; ++b) {
                double col[12];
                for (int c = 0; c <= g.LCDp; ++c) col[c] = Xx[(a * g.EB + b) * F + c];
                for (int c = 0; c < g.EC; ++c) Hx[hidx(g, a, b, c, 0)] = col[c];
                for (int d = 1; d < g.ED; ++d) {
                  for (int c = 0; c + d <= g.LCDp; ++c) col[c] = col[c + 1] + CDx[x] * col[c];
                  for (int c = 0; c < g.EC && c + d <= g.LCDp; ++c) Hx[hidx(g, a, b, c, d)] = col[c];
                }
              }
          }
          __syncwarp();
          const double al2 = 2.0 * alpha, be2 = 2.0 * beta, ga2 = 2.0 * gamma;
          for (int e = lane; e < g.nel; e += 32) {
            const int d = e % g.nd, c = (e / g.nd) % g.nc, b = (e / (g.nd * g.nc)) % g.nb,
                      a = e / (g.nd * g.nc * g.nb);
            const int ca = cart_comp(g.la, a), cb = cart_comp(g.lb, b), cc = cart_comp(g.lc, c),
                      cd = cart_comp(g.ld, d);
            const int A[3] = {comp_x(ca), comp_y(ca), comp_z(ca)};
            const int B[3] = {comp_x(cb), comp_y(cb), comp_z(cb)};
            const int C[3] = {comp_x(cc), comp_y(cc), comp_z(cc)};
            const int Dd[3] = {comp_x(cd), comp_y(cd), comp_z(cd)};
            const double gm = Gam[e];
            for (int rr = 0; rr < nr; ++rr) {
              double base[3], dA[3], dB[3], dC[3];
#pragma unroll
              for (int x = 0; x < 3; ++x) {
                const double* h = H + (rr * 3 + x) * g.hsz;
                const int ax = A[x], bx = B[x], cx = C[x], dx = Dd[x];
                base[x] = h[hidx(g, ax, bx, cx, dx)];
                dA[x] = al2 * h[hidx(g, ax + 1, bx, cx, dx)] - (ax ? ax * h[hidx(g, ax - 1, bx, cx, dx)] : 0.0);
                dB[x] = be2 * h[hidx(g, ax, bx + 1, cx, dx)] - (bx ? bx * h[hidx(g, ax, bx - 1, cx, dx)] : 0.0);
                dC[x] = ga2 * h[hidx(g, ax, bx, cx + 1, dx)] - (cx ? cx * h[hidx(g, ax, bx, cx - 1, dx)] : 0.0);
              }
              const double pyz = base[1] * base[2], pxz = base[0] * base[2], pxy = base[0] * base[1];
              acc[0] += gm * dA[0] * pyz; acc[1] += gm * dA[1] * pxz; acc[2] += gm * dA[2] * pxy;
              acc[3] += gm * dB[0] * pyz; acc[4] += gm * dB[1] * pxz; acc[5] += gm * dB[2] * pxy;
              acc[6] += gm * dC[0] * pyz; acc[7] += gm * dC[1] * pxz; acc[8] += gm * dC[2] * pxy;
            }
          }
          __syncwarp();
        }
      }
    }
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
    if (lane == 0) {
      const int atA = __ldg(ga.shell_atom + __ldg(blk.bra.shell_a + p));
      const int atB = __ldg(ga.shell_atom + __ldg(blk.bra.shell_b + p));
      const int atC = __ldg(ga.shell_atom + __ldg(blk.ket.shell_a + q));
      const int atD = __ldg(ga.shell_atom + __ldg(blk.ket.shell_b + q));
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        atomicAdd(ga.grad + 3 * atA + x, acc[x]);
        atomicAdd(ga.grad + 3 * atB + x, acc[3 + x]);
        atomicAdd(ga.grad + 3 * atC + x, acc[6 + x]);
        atomicAdd(ga.grad + 3 * atD + x, -(acc[x] + acc[3 + x] + acc[6 + x]));
      }
    }
    __syncwarp();
  }
}

}  // namespace

size_t grad_global_scratch_doubles(int la, int lb, int lc, int ld, int num_sms) {
  constexpr int warps = 4;
  const GradGeom g = make_grad_geom(la, lb, lc, ld, warps, 227 * 1024);
  if (g.per_warp < 0 || !g.gamma_global) return 0;
  return (size_t)num_sms * 4 * warps * g.nel;
}

int launch_grad(const QuartetBlock& blk, const double* D, int nbf, const int* shell_atom, double* grad,
                double prim_eps, const RysTablesView& tab, cudaStream_t stream, double* gscratch,
                size_t gscratch_doubles, int num_sms) {
  if (blk.total - blk.t_begin <= 0) return 0;
  constexpr int warps = 4;
  const size_t smem_max = 227 * 1024;
  const GradGeom g = make_grad_geom(blk.bra.la, blk.bra.lb, blk.ket.la, blk.ket.lb, warps, smem_max);
  if (g.per_warp < 0) return -1;
  const size_t smem = (size_t)g.per_warp * 8 * warps;
  const int64_t want = (blk.total - blk.t_begin + warps - 1) / warps;
  int grid = (int)std::min<int64_t>(want, (int64_t)num_sms * 4);
  if (g.gamma_global) {
    const size_t per_block = (size_t)warps * g.nel;
    if ((size_t)grid * per_block > gscratch_doubles) grid = (int)(gscratch_doubles / per_block);
    if (grid < 1) return -2;
  }
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(eri_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max) !=
        cudaSuccess)
      return -3;
    attr = true;
  }
  GradArgs ga{D, nbf, shell_atom, grad, prim_eps};
  eri_grad_kernel<<<grid, warps * 32, smem, stream>>>(blk, ga, tab, g, gscratch);
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

}  // namespace lai
