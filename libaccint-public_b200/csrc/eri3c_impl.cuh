// Three-centre (ab|P) and two-centre (P|Q) Coulomb integrals for density
// fitting, by Rys quadrature with the third centre as a "pair" of the auxiliary
// shell and a unit s function (exponent 0, coefficient 1): eta = gamma_P, Q = C,
// QC = 0, K_CD = 1, so the vertical recurrence and the prefactor are those of the
// four-centre kernels (eri_device.cuh).  Two-centre integrals are the same with
// the bra "pair" (P, unit).  Reference counterparts: compute_three_center_eri
// (src/host/kernels/three_center_eri_kernel.cpp:38-230) and
// compute_two_center_coulomb (src/host/kernels/two_center_coulomb_kernel.cpp:45-180).
//
// One thread per (bra pair, auxiliary shell P, Cartesian component c of P): the
// thread's 1D tables need the ket index f only at f = c_x (c_y, c_z), so per root
// and direction it runs the vertical recurrence to e <= la+lb, f <= lP, keeps the
// column f = c_x, transfers it to (a, b) and adds the products to its block
// (ab|c) in registers.  Consecutive threads take consecutive components and
// auxiliary shells, so the writes of T[ab][P] are contiguous in P.
#pragma once

#include <cuda_runtime.h>

#include "eri_device.cuh"

namespace lai {

struct Eri3cShell {
  double x, y, z;
  int l, np, poff, func;
};

struct Eri3cArgs {
  const Eri3cShell* shells;
  const double* exps;
  const double* coefs;   // normalized
  const int2* pairs;     // bra pairs (a, b) of the launch's class
  int npairs;
  const int* aux;        // auxiliary shells of the launch's l_P class
  int naux_shells;
  double* out;           // three-centre: T[(mu*nbf + nu)*naux + P]; two-centre: V[P*naux + Q]
  long nbf;              // rows of the bra functions (nbf, or naux for two-centre)
  long naux;
  int two_center;        // 1: bra pairs are (P, unit), out = V
  RysTablesView tab;
};

template <int LA, int LB, int LP>
__global__ void __launch_bounds__(128) eri3c_kernel(Eri3cArgs g) {
  constexpr int NA = ncart(LA), NB = ncart(LB), NP = ncart(LP);
  constexpr int LAB = LA + LB;
  constexpr int NR = (LAB + LP) / 2 + 1;
  constexpr int UC = NA * NB <= 36 ? 16 : 1;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t total = (int64_t)g.npairs * g.naux_shells * NP;
  if (tid >= total) return;
  const int c = (int)(tid % NP);
  const int64_t rest = tid / NP;
  const int ps = (int)(rest % g.naux_shells);
  const int pr = (int)(rest / g.naux_shells);
  const int2 ab = g.pairs[pr];
  const Eri3cShell A = g.shells[ab.x], B = g.shells[ab.y], P = g.shells[__ldg(g.aux + ps)];
  const int cc = cart_comp(LP, c);
  const int cxyz[3] = {comp_x(cc), comp_y(cc), comp_z(cc)};
  const double ABv[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
  const double r2 = ABv[0] * ABv[0] + ABv[1] * ABv[1] + ABv[2] * ABv[2];
  double acc[NA * NB];
#pragma unroll UC
  for (int m = 0; m < NA * NB; ++m) acc[m] = 0.0;

  for (int ia = 0; ia < A.np; ++ia) {
    const double al = __ldg(g.exps + A.poff + ia), ca = __ldg(g.coefs + A.poff + ia);
    for (int ib = 0; ib < B.np; ++ib) {
      const double be = __ldg(g.exps + B.poff + ib), cb = __ldg(g.coefs + B.poff + ib);
      const double p = al + be, ip = 1.0 / p;
      const double cab = ca * cb * exp(-al * be * ip * r2);
      const double Pv[3] = {(al * A.x + be * B.x) * ip, (al * A.y + be * B.y) * ip, (al * A.z + be * B.z) * ip};
      const double PA[3] = {Pv[0] - A.x, Pv[1] - A.y, Pv[2] - A.z};
      const double PC[3] = {Pv[0] - P.x, Pv[1] - P.y, Pv[2] - P.z};
      const double pc2 = PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2];
      for (int ic = 0; ic < P.np; ++ic) {
        const double ga = __ldg(g.exps + P.poff + ic), cp = __ldg(g.coefs + P.poff + ic);
        const double s = p + ga;
        const double rs = rsqrt(s);
        const double is = rs * rs;
        const double rz = ga * is, re = p * is;
        const double T = p * rz * pc2;
        // 2 pi^{5/2} / (p gamma sqrt(p + gamma)) c_a c_b c_P K_AB
        const double pref = 34.986836655249725693 * rs / (p * ga) * cab * cp;
        double u[NR], w[NR];
        rys_roots_table<double>(NR, T, g.tab, u, w);
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const double b10 = (1.0 - rz * u[r]) * 0.5 * ip;
          const double b01 = (1.0 - re * u[r]) * 0.5 / ga;
          const double b00 = 0.5 * u[r] * is;
          double h[3][LA + 1][LB + 1];
#pragma unroll
          for (int x = 0; x < 3; ++x) {
            const double pa = PA[x] - rz * u[r] * PC[x];
            const double qc = re * u[r] * PC[x];
            double V[LAB + 1][LP + 1];
            V[0][0] = 1.0;
#pragma unroll
            for (int e = 0; e < LAB; ++e)
              V[e + 1][0] = pa * V[e][0] + (e ? double(e) * b10 * V[e > 0 ? e - 1 : 0][0] : 0.0);
#pragma unroll
            for (int f = 0; f < LP; ++f)
#pragma unroll
              for (int e = 0; e <= LAB; ++e)
                V[e][f + 1] = qc * V[e][f] + (f ? double(f) * b01 * V[e][f > 0 ? f - 1 : 0] : 0.0) +
                              (e ? double(e) * b00 * V[e > 0 ? e - 1 : 0][f] : 0.0);
            // column f = c_x, then the bra transfer I(i, j+1) = I(i+1, j) + AB I(i, j)
            double col[LAB + 1];
#pragma unroll
            for (int e = 0; e <= LAB; ++e) {
              double v = V[e][0];
#pragma unroll
              for (int f = 1; f <= LP; ++f) v = cxyz[x] == f ? V[e][f] : v;
              col[e] = v;
            }
#pragma unroll
            for (int i = 0; i <= LA; ++i) h[x][i][0] = col[i];
#pragma unroll
            for (int j = 1; j <= LB; ++j) {
#pragma unroll
              for (int i = 0; i + j <= LAB; ++i) col[i] = col[i + 1] + ABv[x] * col[i];
#pragma unroll
              for (int i = 0; i <= LA; ++i) h[x][i][j] = col[i];
            }
          }
          const double f = pref * w[r];
#pragma unroll UC
          for (int a = 0; a < NA; ++a) {
            const int qa = cart_comp(LA, a);
#pragma unroll UC
            for (int b = 0; b < NB; ++b) {
              const int qb = cart_comp(LB, b);
              acc[a * NB + b] += f * h[0][comp_x(qa)][comp_x(qb)] * h[1][comp_y(qa)][comp_y(qb)] *
                                 h[2][comp_z(qa)][comp_z(qb)];
            }
          }
        }
      }
    }
  }
  const double nc = norm_factor(LP, c);
  const long col = P.func + c;
#pragma unroll UC
  for (int a = 0; a < NA; ++a) {
    const double na = norm_factor(LA, a) * nc;
#pragma unroll UC
    for (int b = 0; b < NB; ++b) {
      const double v = acc[a * NB + b] * na * norm_factor(LB, b);
      if (g.two_center) {
        // bra pair (P1, unit): V[P1 + a][P + c]; every ordered pair has its thread
        g.out[(A.func + a) * g.naux + col] = v;
      } else {
        g.out[((A.func + a) * g.nbf + B.func + b) * g.naux + col] = v;
        g.out[((B.func + b) * g.nbf + A.func + a) * g.naux + col] = v;
      }
    }
  }
}

// Launches class (la, lb, lP); defined for la <= 4, lb <= min(la, 3), lP <= 4 in
// eri3c_l*.cu.  Returns 0, or -1 for a class that is not instantiated.
int launch_eri3c_l01(int la, int lb, int lp, const Eri3cArgs& g, cudaStream_t s);
int launch_eri3c_l2(int la, int lb, int lp, const Eri3cArgs& g, cudaStream_t s);
int launch_eri3c_l3(int la, int lb, int lp, const Eri3cArgs& g, cudaStream_t s);
int launch_eri3c_l4(int la, int lb, int lp, const Eri3cArgs& g, cudaStream_t s);

template <int LA, int LB, int LP>
int launch_eri3c_cls(const Eri3cArgs& g, cudaStream_t s) {
  const int64_t total = (int64_t)g.npairs * g.naux_shells * ncart(LP);
  if (total <= 0) return 0;
  eri3c_kernel<LA, LB, LP><<<(unsigned)((total + 127) / 128), 128, 0, s>>>(g);
  return 0;
}

}  // namespace lai
