// Lookup tables of the packed FP32 kernels (eri_small_x2.cuh): a Boys grid with
// a finer step and fewer Taylor terms, and Rys root/weight fits of lower degree,
// both derived on the host from the FP64 tables of rys_tables.inc at engine
// creation and rounded to float.  Accuracy (checked by tests/test_tables.py on the
// host copy of the same arithmetic):
//   * Boys F_0, F_1 below kBoysF32Tmax: F_m(T) = sum_{j<4} F_{m+j}(T0) (T0-T)^j/j!
//     about T0 = k/16, |T - T0| <= 1/32; the first omitted term is below
//     (1/32)^4/4! = 4.0e-8 times F_{m+4}(T0), and F_{m+4}/F_m <= F_{m+4}(0)/F_m(0)
//     <= 3/11 for m <= 1, so < 1.1e-8 relative.  At and above kBoysF32Tmax the
//     asymptotic forms F_0 = sqrt(pi/T)/2, F_1 = F_0/(2T) are within 3e-10 relative.
//   * Rys u_r, w_r: the degree-11 Chebyshev interpolants of rys_tables.inc
//     truncated to degree 6 on every unit interval: <= 2.4e-8 relative for
//     n = 2..9 (the truncated Chebyshev coefficients), then converted to the
//     monomial basis in x = 2(T-k)-1.
#pragma once

#include "rys_eval.h"

namespace lai {

constexpr int kBoysF32Rows = 384;          // grid points T0 = k/16, k < 384
constexpr int kBoysF32Stride = 6;          // F_0..F_5 per point (three 8-byte units)
constexpr float kBoysF32Tmax = 23.9375f;   // T < this: table (nearest point k <= 383)
constexpr int kRysF32Deg = 6;
// float2 (u, w) coefficients per unit interval of the n-root table: 7 degrees x n
// roots, padded to an odd count so lanes on different intervals spread over banks.
__host__ __device__ constexpr int rys_f32_row(int n) { return (7 * n) | 1; }
__host__ __device__ constexpr int rys_f32_off(int n) {  // in float2 units
  int o = 0;
  for (int m = 2; m < n; ++m) o += rys_tmax_c(m) * rys_f32_row(m);
  return o;
}
constexpr int kRysF32Len = rys_f32_off(kMaxRoots + 1);  // float2 units, n = 2..9

}  // namespace lai

// ---------------------------------------------------------------------------
// Host-side construction (engine creation) and a scalar host/device mirror of
// the packed kernels' evaluation, per quartet (used by the table tests).
// ---------------------------------------------------------------------------
#include <cmath>

namespace lai {

// out[k * kBoysF32Stride + m] = F_m(k/16), m < 6, k < kBoysF32Rows, from the FP64
// grid (step 0.1, F_0..F_15) by its 10-term Taylor series (|x| <= 0.05).
inline void build_boys_f32(const double* grid, float* out) {
  for (int k = 0; k < kBoysF32Rows; ++k) {
    const double T0 = k / 16.0;
    const int g = (int)std::lround(T0 * 10.0);
    const double x = g * 0.1 - T0;
    for (int m = 0; m < kBoysF32Stride; ++m) {
      double f = 0.0;
      for (int j = 9; j >= 0; --j) f = f * x / (j + 1) + grid[g * kBoysNM + m + j];
      out[k * kBoysF32Stride + m] = (float)f;
    }
  }
}

// Degree-6 truncation of the degree-11 interpolants: monomial -> Chebyshev on
// [-1, 1], drop T_7..T_11, back to monomials.  out holds float2 (u, w) pairs:
// out[2 * (rys_f32_off(n) + k * rys_f32_row(n) + j * n + r) + {0, 1}].
inline void build_rys_f32(const double* coef, float* out) {
  constexpr int D = kRysDeg, d = kRysF32Deg;
  // X[j][i]: Chebyshev coefficients of x^j; Tm[k][i]: monomial coefficients of T_k
  double X[D + 1][D + 1] = {}, Tm[d + 1][d + 1] = {};
  X[0][0] = 1.0;
  for (int j = 0; j < D; ++j)
    for (int i = 0; i <= j; ++i) {
      if (i == 0) X[j + 1][1] += X[j][0];
      else {
        X[j + 1][i - 1] += 0.5 * X[j][i];
        X[j + 1][i + 1] += 0.5 * X[j][i];
      }
    }
  Tm[0][0] = 1.0;
  Tm[1][1] = 1.0;
  for (int k = 1; k < d; ++k)
    for (int i = 0; i <= d; ++i) Tm[k + 1][i] = (i ? 2.0 * Tm[k][i - 1] : 0.0) - Tm[k - 1][i];
  for (int i = 0; i < 2 * kRysF32Len; ++i) out[i] = 0.f;
  for (int n = 2; n <= kMaxRoots; ++n)
    for (int k = 0; k < rys_tmax_c(n); ++k) {
      const double* c = coef + rys_off(n) + k * (D + 1) * 2 * n;
      for (int r = 0; r < n; ++r)
        for (int which = 0; which < 2; ++which) {
          double ch[D + 1] = {};
          for (int j = 0; j <= D; ++j)
            for (int i = 0; i <= D; ++i) ch[i] += c[(j * n + r) * 2 + which] * X[j][i];
          double mono[d + 1] = {};
          for (int kk = 0; kk <= d; ++kk)
            for (int i = 0; i <= d; ++i) mono[i] += ch[kk] * Tm[kk][i];
          for (int j = 0; j <= d; ++j)
            out[2 * (rys_f32_off(n) + k * rys_f32_row(n) + j * n + r) + which] = (float)mono[j];
        }
    }
}

// Round-to-nearest integer of a non-negative float below 2^22 without the
// conversion pipe: adding 1.5 * 2^23 leaves the integer in the low mantissa bits.
constexpr float kRoundMagic = 12582912.0f;

__host__ __device__ inline int f32_bits(float x) {
#ifdef __CUDA_ARCH__
  return __float_as_int(x);
#else
  int i;
  __builtin_memcpy(&i, &x, 4);
  return i;
#endif
}
__host__ __device__ inline float f32_rsqrt(float x) {
#ifdef __CUDA_ARCH__
  return rsqrtf(x);
#else
  return 1.0f / std::sqrt(x);
#endif
}

// Scalar mirror of boys01_x2 (eri_small_x2.cuh) for one quartet.
__host__ __device__ inline void boys01_f32(float T, const float* st, float& F0, float& F1) {
  const float Tc = fminf(T, kBoysF32Tmax);
  const float km = fmaf(Tc, 16.f, kRoundMagic);
  const int k = f32_bits(km) - f32_bits(kRoundMagic);
  const float kf = km - kRoundMagic;
  const float y = fmaf(kf, 1.f / 16.f, -Tc);
  const float* g = st + k * kBoysF32Stride;
  const float y2 = y * 0.5f, y3 = y * (1.f / 3.f);
  F0 = fmaf(fmaf(fmaf(g[3], y3, g[2]), y2, g[1]), y, g[0]);
  F1 = fmaf(fmaf(fmaf(g[4], y3, g[3]), y2, g[2]), y, g[1]);
  if (!(T < kBoysF32Tmax)) {
    const float rt = f32_rsqrt(fmaxf(T, 1.f));
    F0 = rt * 0.88622692545275801365f;
    F1 = F0 * (rt * rt) * 0.5f;
  }
}

// Scalar mirror of rys_x2 for one quartet; st = the n-root block of the FP32 fits.
__host__ __device__ inline void rys_f32(int n, float T, const float* st, const double* herm_x2,
                                        const double* herm_w, float* u, float* w) {
  const float tmax = float(rys_tmax_c(n));
  const float Tc = fminf(T, tmax - 1.f / 131072.f);  // the float below tmax (tmax in [32, 128))
  const float km = (Tc - 0.5f) + kRoundMagic;  // rint(Tc - 1/2)
  const int k = f32_bits(km) - f32_bits(kRoundMagic);
  const float kf = km - kRoundMagic;
  const float x = fmaf(Tc - kf, 2.f, -1.f);
  const float* c = st + 2 * k * rys_f32_row(n);
  for (int r = 0; r < n; ++r) {
    u[r] = c[2 * (kRysF32Deg * n + r)];
    w[r] = c[2 * (kRysF32Deg * n + r) + 1];
  }
  for (int j = kRysF32Deg - 1; j >= 0; --j)
    for (int r = 0; r < n; ++r) {
      u[r] = fmaf(u[r], x, c[2 * (j * n + r)]);
      w[r] = fmaf(w[r], x, c[2 * (j * n + r) + 1]);
    }
  if (!(T < tmax)) {
    const float rt = f32_rsqrt(fmaxf(T, 1.f));
    const float it = rt * rt;
    const int h = rys_hoff(n);
    for (int r = 0; r < n; ++r) {
      u[r] = it * (float)herm_x2[h + r];
      w[r] = rt * (float)herm_w[h + r];
    }
  }
}

}  // namespace lai

#ifdef __CUDACC__
namespace lai {

// Shared-memory copies of the FP32 tables: the Boys grid (one root) or the
// n-root block of the degree-6 Rys fits, as laid out by build_boys_f32 /
// build_rys_f32 (the evaluators above read them with the same indexing).
template <int NR>
__host__ __device__ constexpr int f32_table_floats() {
  return NR == 1 ? kBoysF32Rows * kBoysF32Stride : 2 * rys_tmax_c(NR) * rys_f32_row(NR);
}
template <int NR>
__host__ __device__ constexpr size_t f32_table_bytes() {
  return (sizeof(float) * f32_table_floats<NR>() + 15) & ~size_t(15);
}
template <int NR>
__device__ __forceinline__ void stage_table_f32(float* __restrict__ st, const RysTablesView& tab) {
  const float* src = NR == 1 ? tab.boys_f32 : tab.rys_f32 + 2 * rys_f32_off(NR);
  for (int i = threadIdx.x; i < f32_table_floats<NR>(); i += blockDim.x) st[i] = __ldg(src + i);
}

}  // namespace lai
#endif
