// Lookup tables staged in shared memory by the persistent ERI kernels: the Boys
// grid (one-root classes) or the class's Rys root table, with row strides padded
// so that lanes reading different rows fall into different banks (a warp's
// per-lane gathers from global memory would touch up to 32 cache lines per load
// instruction).  Same arithmetic as rys_eval.h.
#pragma once

#include <cuda_runtime.h>

#include "eri_device.cuh"
#include "rys_eval.h"

namespace lai {

// Shared-memory table layouts (in doubles).
constexpr int kBoysRow = 14;  // F_0..F_11 per grid point + 2 pad: 16-byte rows, stride/2 odd
template <int NR>
__host__ __device__ constexpr int rys_row() { return 24 * NR + 2; }  // 12 degrees x NR x (u,w) + pad
template <int NR>
__host__ __device__ constexpr int table_doubles() {
  return NR == 1 ? kBoysNGrid * kBoysRow : rys_tmax_c(NR) * rys_row<NR>();
}

template <int NR>
__device__ __forceinline__ void stage_table(double* __restrict__ st, const RysTablesView& tab) {
  if constexpr (NR == 1) {
    for (int i = threadIdx.x; i < kBoysNGrid * 12; i += blockDim.x) {
      const int k = i / 12, j = i - k * 12;
      st[k * kBoysRow + j] = __ldg(tab.boys + k * kBoysNM + j);
    }
  } else {
    constexpr int W = 24 * NR;
    const double* src = tab.coef + rys_off(NR);
    for (int i = threadIdx.x; i < rys_tmax_c(NR) * W; i += blockDim.x) {
      const int k = i / W, j = i - k * W;
      st[k * rys_row<NR>() + j] = __ldg(src + i);
    }
  }
}

// Roots/weights of the NR-point Rys rule from the staged table (same arithmetic
// as rys_roots_table in rys_eval.h).
template <int NR, typename R>
__device__ __forceinline__ void rys_smem(R T, const double* __restrict__ st, const RysTablesView& tab,
                                         R* __restrict__ u, R* __restrict__ w) {
  if constexpr (NR == 1) {
    R F0, F1;
    if (T < R(kBoysTmax)) {
      const int k = __double2int_rn(double(T) * 10.0);
      const R x = R(k) * R(0.1) - T;
      const double2* f = reinterpret_cast<const double2*>(st + k * kBoysRow);
      double g[12];
#pragma unroll
      for (int j = 0; j < 6; ++j) {
        const double2 v = f[j];
        g[2 * j] = v.x;
        g[2 * j + 1] = v.y;
      }
      R tpow[10];
      tpow[0] = R(1);
#pragma unroll
      for (int j = 1; j < 10; ++j) tpow[j] = tpow[j - 1] * x * R(1.0 / j);
      R a = 0, b = 0;
#pragma unroll
      for (int j = 9; j >= 0; --j) {
        a += R(g[j]) * tpow[j];
        b += R(g[j + 1]) * tpow[j];
      }
      F0 = a;
      F1 = b;
    } else {
      const R rt = R(1) / sqrt(T);
      F0 = R(0.88622692545275801365) * rt;
      F1 = F0 * R(0.5) / T;
    }
    u[0] = F1 / F0;
    w[0] = F0;
  } else {
    if (T < R(rys_tmax_c(NR))) {
      const int k = (int)T;
      const R x = R(2) * (T - R(k)) - R(1);
      const double2* c = reinterpret_cast<const double2*>(st + k * rys_row<NR>());
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const double2 v = c[kRysDeg * NR + r];
        u[r] = R(v.x);
        w[r] = R(v.y);
      }
#pragma unroll
      for (int j = kRysDeg - 1; j >= 0; --j)
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const double2 v = c[j * NR + r];
          u[r] = u[r] * x + R(v.x);
          w[r] = w[r] * x + R(v.y);
        }
    } else {
      const R it = R(1) / T;
      const R rt = sqrt(it);
      const int h = rys_hoff(NR);
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        u[r] = R(__ldg(tab.herm_x2 + h + r)) * it;
        w[r] = R(__ldg(tab.herm_w + h + r)) * rt;
      }
    }
  }
}

}  // namespace lai
