// Lookup tables staged in shared memory by the persistent ERI kernels: the Boys
// grid (one-root classes) or the class's Rys root table, with row strides padded
// so that lanes reading different rows fall into different banks (a warp's
// per-lane gathers from global memory would touch up to 32 cache lines per load
// instruction).  Same arithmetic as rys_eval.h.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "eri_device.cuh"
#include "rys_eval.h"

namespace lai {

// Shared-memory table layouts, in elements of the compute type R (the FP32 kernels
// stage FP32 copies: half the shared memory, and single-width loads).
//
// (A layout with the Taylor coefficients pre-divided by j!, which saves the x/j
// products, was measured slower: its 18-double rows take more shared memory, and
// the carve-out shrinks L1, which these kernels lean on.)
// FP64 rows: F_0..F_9 at T0 = k / 10 (five 16-byte units, odd, so lanes on
// different rows spread over the banks).
constexpr int kBoysRowsS = kBoysNGrid;
constexpr double kBoysTmaxS = kBoysTmax;
constexpr int kBoysRowS = 10;
constexpr int kBoysRowF = 12;     // FP32: F_0..F_11, three 16-byte units (odd)
template <typename R>
__host__ __device__ constexpr int boys_row() { return sizeof(R) == 8 ? kBoysRowS : kBoysRowF; }
template <typename R>
__host__ __device__ constexpr int boys_rows() { return sizeof(R) == 8 ? kBoysRowsS : kBoysNGrid; }
template <int NR>
__host__ __device__ constexpr int rys_row() { return 24 * NR + 2; }  // 12 degrees x NR x (u,w) + pad
template <int NR, typename R>
__host__ __device__ constexpr int table_elems() {
  return NR == 1 ? boys_rows<R>() * boys_row<R>() : rys_tmax_c(NR) * rys_row<NR>();
}
// 1.5 * 2^52: adding it to a double y with 0 <= |y| < 2^31 leaves rint(y) in the
// low word of the sum (round to nearest even), with no conversion instruction.
constexpr double kRoundMagicD = 6755399441055744.0;
template <int NR, typename R>
__host__ __device__ constexpr size_t table_bytes() {
  return (sizeof(R) * table_elems<NR, R>() + 15) & ~size_t(15);  // what follows stays 16-byte aligned
}

template <int NR, typename R>
__device__ __forceinline__ void stage_table(R* __restrict__ st, const RysTablesView& tab) {
  if constexpr (NR == 1 && sizeof(R) == 8) {
    constexpr int NV = kBoysRowS;
    for (int i = threadIdx.x; i < kBoysRowsS * NV; i += blockDim.x) {
      const int k = i / NV, j = i - k * NV;
      st[k * NV + j] = __ldg(tab.boys + k * kBoysNM + j);
    }
  } else if constexpr (NR == 1) {
    constexpr int NV = boys_row<R>();  // values per row (the row holds no padding)
    for (int i = threadIdx.x; i < kBoysNGrid * NV; i += blockDim.x) {
      const int k = i / NV, j = i - k * NV;
      st[k * NV + j] = R(__ldg(tab.boys + k * kBoysNM + j));
    }
  } else {
    constexpr int W = 24 * NR;
    const double* src = tab.coef + rys_off(NR);
    for (int i = threadIdx.x; i < rys_tmax_c(NR) * W; i += blockDim.x) {
      const int k = i / W, j = i - k * W;
      st[k * rys_row<NR>() + j] = R(__ldg(src + i));
    }
  }
}

// F_0(T) and F_1(T) from the staged Boys grid (the Taylor series of boys01 in
// rys_eval.h; FP64 from the pre-divided rows).
template <typename R>
__device__ __forceinline__ void boys01_smem(R T, const R* __restrict__ st, R& F0, R& F1) {
  constexpr bool F64 = sizeof(R) == 8;
  if constexpr (F64) {
    // FP64: nearest grid point by the rounding constant (no conversion
    // instructions), 8-term Taylor series (first omitted term below 6e-17 relative)
    if (T < kBoysTmaxS) {
      const double km = fma(double(T), 10.0, kRoundMagicD);
      const int k = min(__double2loint(km), kBoysRowsS - 1);
      const double x = fma(km - kRoundMagicD, 0.1, -double(T));
      const double2* f = reinterpret_cast<const double2*>(st + k * kBoysRowS);
      double g[10];
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        const double2 v = f[j];
        g[2 * j] = v.x;
        g[2 * j + 1] = v.y;
      }
      double a, b;
      boys_taylor<double>(x, g, a, b);
      F0 = R(a);
      F1 = R(b);
    } else {
      const R rt = fast_rsqrt(T);
      F0 = R(0.88622692545275801365) * rt;  // sqrt(pi)/2
      F1 = R(0.5) * F0 * rt * rt;
    }
  } else {
    // FP32: nearest grid point; T just below kBoysTmax can round up to the row past
    // the end, hence the clamp
    if (T < R(kBoysTmax)) {
      const int k = min(__float2int_rn(float(T) * 10.0f), kBoysNGrid - 1);
      const R x = R(k) * R(0.1) - T;
      constexpr int NG = boys_terms<R>() + 1;  // grid values used: F_0..F_N
      R g[12];
      const float4* f = reinterpret_cast<const float4*>(st + k * kBoysRowF);
#pragma unroll
      for (int j = 0; j < (NG + 3) / 4; ++j) {
        const float4 v = f[j];
        g[4 * j] = v.x;
        g[4 * j + 1] = v.y;
        g[4 * j + 2] = v.z;
        g[4 * j + 3] = v.w;
      }
      boys_taylor<R>(x, g, F0, F1);
    } else {
      const R rt = fast_rsqrt(T);
      F0 = R(0.88622692545275801365) * rt;  // sqrt(pi)/2
      F1 = R(0.5) * F0 * rt * rt;
    }
  }
}

// Roots/weights of the NR-point Rys rule from the staged table (same arithmetic
// as rys_roots_table in rys_eval.h).
template <int NR, typename R>
__device__ __forceinline__ void rys_smem(R T, const R* __restrict__ st, const RysTablesView& tab,
                                         R* __restrict__ u, R* __restrict__ w) {
  constexpr bool F64 = sizeof(R) == 8;
  if constexpr (NR == 1) {
    if (T < R(kBoysTmax)) {
      R F0, F1;
      boys01_smem<R>(T, st, F0, F1);
      u[0] = fast_div(F1, F0);
      w[0] = F0;
    } else {
      rys1_asymptotic<R>(T, u[0], w[0]);
    }
  } else {
    if (T < R(rys_tmax_c(NR))) {
      int k;
      R x;
      if constexpr (F64) {
        // unit interval by the rounding constant: rint(T - 1/2) (an integer T may
        // land on the interval below, at its end x = 1)
        const double km = (double(T) - 0.5) + kRoundMagicD;
        k = __double2loint(km);
        x = fma(2.0, double(T) - (km - kRoundMagicD), -1.0);
      } else {
        k = (int)T;
        x = R(2) * (T - R(k)) - R(1);
      }
      using V2 = typename std::conditional<F64, double2, float2>::type;
      const V2* c = reinterpret_cast<const V2*>(st + k * rys_row<NR>());
#pragma unroll
      for (int r = 0; r < NR; ++r) {
        const V2 v = c[kRysDeg * NR + r];
        u[r] = v.x;
        w[r] = v.y;
      }
#pragma unroll
      for (int j = kRysDeg - 1; j >= 0; --j)
#pragma unroll
        for (int r = 0; r < NR; ++r) {
          const V2 v = c[j * NR + r];
          u[r] = u[r] * x + v.x;
          w[r] = w[r] * x + v.y;
        }
    } else {
      const R rt = fast_rsqrt(T);
      const R it = rt * rt;
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
