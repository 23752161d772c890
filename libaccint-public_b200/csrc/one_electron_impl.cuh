// Kernel template of the one-electron integrals (overlap, kinetic, point-charge
// attraction); the algorithm is described in one_electron.cu.  Instantiated per
// angular-momentum group in one_electron_l*.cu so the build runs in parallel.
#pragma once

#include <cuda_runtime.h>

#include "../../include/libaccint_b200.h"
#include "eri_device.cuh"

namespace lai {

struct OneEShell {
  double x, y, z;
  int l, np, poff, func;
};

struct OneEArgs {
  const OneEShell* shells;
  const double* exps;
  const double* coefs;
  const double* charges;  // [n][4]: x, y, z, q
  int ncharge;
  long nbf;
  double* out;
  int add;                // 1: out += integrals (second operator of T + V)
  RysTablesView tab;
};

// Overlap-type 1D table s(i, j), i <= LA, j <= JM, from s(k, 0), k <= LA + JM.
template <int LA, int JM>
__device__ __forceinline__ void overlap_1d(double pa, double ab, double hp, double (&s)[LA + 1][JM + 1]) {
  constexpr int KM = LA + JM;
  double h[JM + 1][KM + 1];
  h[0][0] = 1.0;
  if (KM > 0) h[0][1] = pa;
#pragma unroll
  for (int k = 1; k < KM; ++k) h[0][k + 1] = pa * h[0][k] + double(k) * hp * h[0][k - 1];
#pragma unroll
  for (int j = 0; j < JM; ++j)
#pragma unroll
    for (int i = 0; i <= KM - j - 1; ++i) h[j + 1][i] = h[j][i + 1] + ab * h[j][i];
#pragma unroll
  for (int i = 0; i <= LA; ++i)
#pragma unroll
    for (int j = 0; j <= JM; ++j) s[i][j] = h[j][i];
}

// Kinetic 1D table t(i, j) = -1/2 <i| d^2/dx^2 |j> from the overlap table with
// j up to LB + 2: d^2/dx^2 x_B^j e^{-beta x_B^2} = j(j-1) x_B^{j-2}
// - 2 beta (2j+1) x_B^j + 4 beta^2 x_B^{j+2}.
template <int LA, int LB>
__device__ __forceinline__ void kinetic_1d(const double (&s)[LA + 1][LB + 3], double be,
                                           double (&t)[LA + 1][LB + 1]) {
#pragma unroll
  for (int i = 0; i <= LA; ++i)
#pragma unroll
    for (int j = 0; j <= LB; ++j) {
      double v = 4.0 * be * be * s[i][j + 2] - 2.0 * be * double(2 * j + 1) * s[i][j];
      if (j >= 2) v += double(j * (j - 1)) * s[i][j >= 2 ? j - 2 : 0];
      t[i][j] = -0.5 * v;
    }
}

template <int LA, int LB, int OP>
__global__ void __launch_bounds__(128) one_e_kernel(OneEArgs g, const int2* __restrict__ pairs, int npair) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npair) return;
  constexpr int NA = ncart(LA), NB = ncart(LB);
  constexpr bool kOv = OP == LAI_OP_OVERLAP;
  constexpr bool kKin = OP == LAI_OP_KINETIC;
  constexpr bool kNuc = OP == LAI_OP_NUCLEAR;
  constexpr int JM = kKin ? LB + 2 : LB;
  constexpr int NR = (LA + LB) / 2 + 1;
  // blocks up to (dd) are unrolled into registers; larger ones (f, g: rare) keep
  // runtime loops so the build stays small
  constexpr int UC = NA * NB <= 36 ? 16 : 1;
  const int2 pr = pairs[t];
  const OneEShell A = g.shells[pr.x], B = g.shells[pr.y];
  const double ABx = A.x - B.x, ABy = A.y - B.y, ABz = A.z - B.z;
  const double r2 = ABx * ABx + ABy * ABy + ABz * ABz;
  double acc[NA * NB];
#pragma unroll UC
  for (int m = 0; m < NA * NB; ++m) acc[m] = 0.0;

  for (int ia = 0; ia < A.np; ++ia) {
    const double al = __ldg(g.exps + A.poff + ia), ca = __ldg(g.coefs + A.poff + ia);
    for (int ib = 0; ib < B.np; ++ib) {
      const double be = __ldg(g.exps + B.poff + ib), cb = __ldg(g.coefs + B.poff + ib);
      const double p = al + be, ip = 1.0 / p, hp = 0.5 * ip;
      const double c = ca * cb * exp(-al * be * ip * r2);
      const double Px = (al * A.x + be * B.x) * ip, Py = (al * A.y + be * B.y) * ip,
                   Pz = (al * A.z + be * B.z) * ip;
      const double PAx = Px - A.x, PAy = Py - A.y, PAz = Pz - A.z;
      if (kOv || kKin) {
        double sx[LA + 1][JM + 1], sy[LA + 1][JM + 1], sz[LA + 1][JM + 1];
        overlap_1d<LA, JM>(PAx, ABx, hp, sx);
        overlap_1d<LA, JM>(PAy, ABy, hp, sy);
        overlap_1d<LA, JM>(PAz, ABz, hp, sz);
        const double pip = 3.14159265358979323846 * ip;
        const double pref = c * pip * sqrt(pip);
        double tx[LA + 1][LB + 1], ty[LA + 1][LB + 1], tz[LA + 1][LB + 1];
        if constexpr (kKin) {
          kinetic_1d<LA, LB>(sx, be, tx);
          kinetic_1d<LA, LB>(sy, be, ty);
          kinetic_1d<LA, LB>(sz, be, tz);
        }
#pragma unroll UC
        for (int a = 0; a < NA; ++a) {
          const int qa = cart_comp(LA, a);
          const int ax = comp_x(qa), ay = comp_y(qa), az = comp_z(qa);
#pragma unroll UC
          for (int b = 0; b < NB; ++b) {
            const int qb = cart_comp(LB, b);
            const int bx = comp_x(qb), by = comp_y(qb), bz = comp_z(qb);
            if constexpr (kKin)
              acc[a * NB + b] += pref * (tx[ax][bx] * sy[ay][by] * sz[az][bz] +
                                         sx[ax][bx] * ty[ay][by] * sz[az][bz] +
                                         sx[ax][bx] * sy[ay][by] * tz[az][bz]);
            else
              acc[a * NB + b] += pref * sx[ax][bx] * sy[ay][by] * sz[az][bz];
          }
        }
      }
      if (kNuc) {
        const double pv = -2.0 * 3.14159265358979323846 * ip * c;
        for (int ic = 0; ic < g.ncharge; ++ic) {
          const double Cx = __ldg(g.charges + 4 * ic), Cy = __ldg(g.charges + 4 * ic + 1),
                       Cz = __ldg(g.charges + 4 * ic + 2), q = __ldg(g.charges + 4 * ic + 3);
          const double PCx = Px - Cx, PCy = Py - Cy, PCz = Pz - Cz;
          const double T = p * (PCx * PCx + PCy * PCy + PCz * PCz);
          double u[NR], w[NR];
          rys_roots_table<double>(NR, T, g.tab, u, w);
#pragma unroll UC
          for (int r = 0; r < NR; ++r) {
            const double hb = (1.0 - u[r]) * hp;
            double ix[LA + 1][LB + 1], iy[LA + 1][LB + 1], iz[LA + 1][LB + 1];
            overlap_1d<LA, LB>(PAx - u[r] * PCx, ABx, hb, ix);
            overlap_1d<LA, LB>(PAy - u[r] * PCy, ABy, hb, iy);
            overlap_1d<LA, LB>(PAz - u[r] * PCz, ABz, hb, iz);
            const double f = pv * q * w[r];
#pragma unroll UC
            for (int a = 0; a < NA; ++a) {
              const int qa = cart_comp(LA, a);
              const int ax = comp_x(qa), ay = comp_y(qa), az = comp_z(qa);
#pragma unroll UC
              for (int b = 0; b < NB; ++b) {
                const int qb = cart_comp(LB, b);
                acc[a * NB + b] += f * ix[ax][comp_x(qb)] * iy[ay][comp_y(qb)] * iz[az][comp_z(qb)];
              }
            }
          }
        }
      }
    }
  }
  const long nbf = g.nbf;
#pragma unroll UC
  for (int a = 0; a < NA; ++a) {
    const double na = norm_factor(LA, a);
#pragma unroll UC
    for (int b = 0; b < NB; ++b) {
      const double v = acc[a * NB + b] * na * norm_factor(LB, b);
      double* o1 = g.out + (A.func + a) * nbf + B.func + b;
      double* o2 = g.out + (B.func + b) * nbf + A.func + a;
      if (g.add) {
        // the first operator left the matrix bitwise symmetric; a diagonal shell
        // pair adds its lower triangle only, writing each sum to both positions
        if (A.func == B.func && b > a) continue;
        const double v1 = *o1 + v;
        *o1 = v1;
        *o2 = v1;
      } else {
        *o1 = v;
        *o2 = v;
      }
    }
  }
}

template <int LA, int LB, int OP>
void launch_cls(const OneEArgs& g, const int2* pairs, int n, cudaStream_t s) {
  one_e_kernel<LA, LB, OP><<<(n + 127) / 128, 128, 0, s>>>(g, pairs, n);
}

template <int LA, int LB>
int launch_op(int op, const OneEArgs& g, const int2* pairs, int n, cudaStream_t s) {
  switch (op) {
    case LAI_OP_OVERLAP: launch_cls<LA, LB, LAI_OP_OVERLAP>(g, pairs, n, s); break;
    case LAI_OP_KINETIC: launch_cls<LA, LB, LAI_OP_KINETIC>(g, pairs, n, s); break;
    default: launch_cls<LA, LB, LAI_OP_NUCLEAR>(g, pairs, n, s); break;
  }
  return 0;
}

// One launch of class (la, lb), la >= lb, for op OVERLAP, KINETIC or NUCLEAR;
// defined for la <= 2, la == 3 and la == 4 in one_electron_l012/l3/l4.cu.
// Returns -1 for a class outside the group.
int launch_one_e_l012(int la, int lb, int op, const OneEArgs& g, const int2* pairs, int n, cudaStream_t s);
int launch_one_e_l3(int la, int lb, int op, const OneEArgs& g, const int2* pairs, int n, cudaStream_t s);
int launch_one_e_l4(int la, int lb, int op, const OneEArgs& g, const int2* pairs, int n, cudaStream_t s);

}  // namespace lai
