// Device-side building blocks shared by the ERI/J-K kernels.
//
// Algorithm (per contracted shell quartet (ab|cd), la>=lb, lc>=ld):
//   1. For each primitive quartet and each Rys root u_r (weight w_r), build the
//      2D tables I_x(e, f), I_y, I_z for e <= la+lb, f <= lc+ld by the vertical
//      recurrence of the reference's build_2d_rys (src/host/kernels/eri_kernel.cpp:
//      119-141):
//        I(e+1,0) = PA' I(e,0) + e B10 I(e-1,0)
//        I(e,f+1) = QC' I(e,f) + f B01 I(e,f-1) + e B00 I(e-1,f)
//      with PA' = PA - (eta/(zeta+eta)) u PQ, QC' = QC + (zeta/(zeta+eta)) u PQ,
//      B10 = (1 - eta u/(zeta+eta))/(2 zeta), B01 = (1 - zeta u/(zeta+eta))/(2 eta),
//      B00 = u/(2(zeta+eta)) (eri_kernel.cpp:302-317).
//   2. Accumulate G[e][f] = sum_{prim,r} w_r pref I_x I_y I_z over the Cartesian
//      components e of shells la..la+lb and f of lc..lc+ld -- the "(e0|f0)"
//      integrals, contracted over primitives BEFORE the horizontal transfer.
//   3. Horizontal transfer once per contracted quartet, in closed (binomial) form:
//      (a b| = sum_{k<=b} prod_x C(b_x,k_x) (A-B)_x^{b_x-k_x} (a+k 0|, same for |c d),
//      which equals the reference's HRR I(a,b+1) = I(a+1,b) + AB I(a,b)
//      (eri_kernel.cpp:143-163) applied in each direction.
//   4. Per-component normalization 1/sqrt((2lx-1)!!(2ly-1)!!(2lz-1)!!)
//      (include/libaccint/kernels/norm_correction.hpp:28-34).
#pragma once

#include <cuda_runtime.h>

#include "lai_common.h"
#include "rys_eval.h"

namespace lai {

constexpr int kMaxCartL = 9;                  // components tabulated up to l = 9
constexpr int kNCartMax = 55;                 // (9+1)(9+2)/2

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
// Number of components of shells lo..hi.
__host__ __device__ constexpr int ncart_range(int lo, int hi) {
  return ((hi + 1) * (hi + 2) * (hi + 3) - lo * (lo + 1) * (lo + 2)) / 6;
}
// Index of (lx, ly, lz) inside its shell: lx descending, then ly descending.
__host__ __device__ constexpr int cart_index(int lx, int ly, int lz) {
  return ((ly + lz) * (ly + lz + 1)) / 2 + lz;
}
// Offset of shell l inside a component list that starts at shell lo.
__host__ __device__ constexpr int ncart_before(int lo, int l) { return ncart_range(lo, l) - ncart(l); }

// Packed component (lx | ly << 4 | lz << 8) of the i-th Cartesian function of shell l.
__host__ __device__ constexpr int cart_comp(int l, int i) {
  int k = 0;
  for (int x = l; x >= 0; --x)
    for (int y = l - x; y >= 0; --y) {
      if (k == i) return x | (y << 4) | ((l - x - y) << 8);
      ++k;
    }
  return 0;
}
__host__ __device__ constexpr int comp_x(int c) { return c & 15; }
__host__ __device__ constexpr int comp_y(int c) { return (c >> 4) & 15; }
__host__ __device__ constexpr int comp_z(int c) { return (c >> 8) & 15; }

__host__ __device__ constexpr double dfact_odd(int l) {  // (2l-1)!!
  double r = 1;
  for (int k = 2 * l - 1; k > 1; k -= 2) r *= k;
  return r;
}
__host__ __device__ constexpr double binom(int n, int k) {
  double r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

// Per-component normalization factor of component i of shell l.
__device__ __forceinline__ double norm_factor(int l, int i) {
  const int c = cart_comp(l, i);
  return rsqrt(dfact_odd(comp_x(c)) * dfact_odd(comp_y(c)) * dfact_odd(comp_z(c)));
}

// x^m for small non-negative m.
template <typename R>
__device__ __forceinline__ R ipow(R x, int m) {
  R r = R(1);
  for (int i = 0; i < m; ++i) r *= x;
  return r;
}

// Arguments of one J/K (or raw-integral) launch.
struct JKArgs {
  const double* D;       // nbf x nbf density, row-major (symmetric)
  double* J;             // nbf x nbf, receives the un-symmetrized J' (J = J' + J'^T)
  double* K;             // nbf x nbf, receives the un-symmetrized K' (K = K' + K'^T)
  int nbf;
  int mode;              // MODE_JK, MODE_RAW, MODE_SCHWARZ
  double* raw_out;       // MODE_RAW: [quartet][a][b][c][d]
  int* raw_meta;         // MODE_RAW: [quartet][4] first function index of a, b, c, d
  double* schwarz_out;   // MODE_SCHWARZ: [bra pair] sqrt(max |(ab|ab)|)
  unsigned int* status;  // device status word (0 = ok)
  double prim_eps;       // skip primitive quartets with q_ab * q_cd < prim_eps (0 = none)
  double prim_rel32;     // FP32 kernels: also skip q_ab * q_cd < prim_rel32 * Q_ij * Q_kl
  unsigned long long* prim_count;  // optional: += primitive quartets executed by the launch
  // batched engines (many independent systems): D, J and K hold one nbf_s x nbf_s
  // block per system, block s at element offset sys_off[s]; function indices are
  // local to the system.  nullptr for a single system.
  const int64_t* sys_off;
  const int* sys_nbf;
};

// The density and Fock-matrix blocks of the system quartet (p, .) belongs to.
struct SysMats {
  const double* D;
  double* J;
  double* K;
  int nbf;
};
__device__ __forceinline__ SysMats sys_mats(const JKArgs& args, const QuartetBlock& blk, int p) {
  SysMats m{args.D, args.J, args.K, args.nbf};
  if (blk.bra.sys) {
    const int s = __ldg(blk.bra.sys + p);
    const int64_t o = __ldg(args.sys_off + s);
    m.D += o;
    m.J += o;
    m.K += o;
    m.nbf = __ldg(args.sys_nbf + s);
  }
  return m;
}

// One ket primitive pair's data, loaded a loop iteration ahead of its use so the
// global-memory latency overlaps the previous primitive's arithmetic (fields a
// class never reads are removed by the compiler).
template <typename T>
struct KetPrimT {
  T q, eta, he, px, py, pz, qcx, qcy, qcz, c;
};
using KetPrim = KetPrimT<double>;
template <typename T>
__device__ __forceinline__ void load_ket_prim(const T* __restrict__ pk, size_t sk, KetPrimT<T>& k) {
  k.q = __ldg(pk + PF_Q * sk);
  k.eta = __ldg(pk + PF_ZETA * sk);
  k.he = __ldg(pk + PF_HZ * sk);
  k.px = __ldg(pk + PF_PX * sk);
  k.py = __ldg(pk + PF_PY * sk);
  k.pz = __ldg(pk + PF_PZ * sk);
  k.qcx = __ldg(pk + PF_PAX * sk);
  k.qcy = __ldg(pk + PF_PAY * sk);
  k.qcz = __ldg(pk + PF_PAZ * sk);
  k.c = __ldg(pk + PF_C * sk);
}

// Ket tiles (KetRecField): the address of primitive 0 of pair q, the distance
// between consecutive primitives of one pair, and one primitive's fields, all at
// compile-time offsets from that address.
constexpr int kKetPrimStride = kKetRec * kKetTile;
template <typename T>
__device__ __forceinline__ const T* ket_tile_ptr(const T* __restrict__ tiles, int q, int Kcd) {
  return tiles + (size_t)(q / kKetTile) * Kcd * kKetPrimStride + (q % kKetTile);
}
template <typename T>
__device__ __forceinline__ void load_ket_rec(const T* __restrict__ pk, KetPrimT<T>& k) {
  k.q = __ldg(pk + KR_Q * kKetTile);
  k.eta = __ldg(pk + KR_ETA * kKetTile);
  k.he = __ldg(pk + KR_HE * kKetTile);
  k.px = __ldg(pk + KR_PX * kKetTile);
  k.py = __ldg(pk + KR_PY * kKetTile);
  k.pz = __ldg(pk + KR_PZ * kKetTile);
  k.qcx = __ldg(pk + KR_QCX * kKetTile);
  k.qcy = __ldg(pk + KR_QCY * kKetTile);
  k.qcz = __ldg(pk + KR_QCZ * kKetTile);
  k.c = __ldg(pk + KR_C * kKetTile);
}
template <typename R>
__device__ __forceinline__ const R* ket_tiles(const PairClassDev& c);
template <>
__device__ __forceinline__ const double* ket_tiles<double>(const PairClassDev& c) { return c.primk; }
template <>
__device__ __forceinline__ const float* ket_tiles<float>(const PairClassDev& c) { return c.primkf; }

// Primitive-pair table of a class in the kernel's compute type: the FP64 table,
// or its FP32 copy for the FP32 kernels.
template <typename R>
__device__ __forceinline__ const R* prim_table(const PairClassDev& c);
template <>
__device__ __forceinline__ const double* prim_table<double>(const PairClassDev& c) { return c.prim; }
template <>
__device__ __forceinline__ const float* prim_table<float>(const PairClassDev& c) { return c.primf; }

// Per-pair primitive records (BraRecField) in the kernel's compute type.
template <typename R>
__device__ __forceinline__ const R* bra_records(const PairClassDev& c);
template <>
__device__ __forceinline__ const double* bra_records<double>(const PairClassDev& c) { return c.primb; }
template <>
__device__ __forceinline__ const float* bra_records<float>(const PairClassDev& c) { return c.primbf; }

// Bra primitive-pair data of one pair (same fields, bra side).
struct BraPrim {
  double q, zeta, hz, px, py, pz, pax, pay, paz, c;
};
__device__ __forceinline__ void load_bra_prim(const double* __restrict__ pb, size_t sb, BraPrim& b) {
  b.q = __ldg(pb + PF_Q * sb);
  b.zeta = __ldg(pb + PF_ZETA * sb);
  b.hz = __ldg(pb + PF_HZ * sb);
  b.px = __ldg(pb + PF_PX * sb);
  b.py = __ldg(pb + PF_PY * sb);
  b.pz = __ldg(pb + PF_PZ * sb);
  b.pax = __ldg(pb + PF_PAX * sb);
  b.pay = __ldg(pb + PF_PAY * sb);
  b.paz = __ldg(pb + PF_PAZ * sb);
  b.c = __ldg(pb + PF_C * sb);
}

// Requests the cache lines of one primitive pair's fields into L1 without
// waiting (PTX prefetch.global.L1): the loads that follow later hit L1.
__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}
__device__ __forceinline__ void prefetch_prim_l1(const double* __restrict__ pp, size_t s) {
#pragma unroll
  for (int f = 0; f < PF_COUNT; ++f) prefetch_l1(pp + f * s);
}

// Add a per-lane count to a launch counter (one atomic per warp).
__device__ __forceinline__ void count_prims(unsigned long long* ctr, unsigned int n) {
  if (!ctr) return;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(ctr, (unsigned long long)n);
}
enum { MODE_JK = 0, MODE_RAW = 1, MODE_SCHWARZ = 2 };

// Locate the bra pair p of flat quartet index t: largest p with offsets[p] <= t.
__device__ __forceinline__ int find_bra(const int64_t* __restrict__ offsets, int npairs, int64_t t) {
  int lo = 0, hi = npairs;  // offsets[lo] <= t < offsets[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(offsets + mid) <= t) lo = mid; else hi = mid;
  }
  return lo;
}

// Degeneracy weight of a canonical quartet for the 8-fold symmetric scatter:
// 1/2 for each of i==j, k==l, (ij)==(kl) (the permutation flags of the reference's
// accumulate_symmetric, src/shared/consumers/fock_builder.cpp:123-222).
__device__ __forceinline__ double quartet_weight(const QuartetBlock& blk, int p, int q) {
  const int a = __ldg(blk.bra.shell_a + p), b = __ldg(blk.bra.shell_b + p);
  const int c = __ldg(blk.ket.shell_a + q), d = __ldg(blk.ket.shell_b + q);
  double s = 1.0;
  if (a == b) s *= 0.5;
  if (c == d) s *= 0.5;
  if (a == c && b == d) s *= 0.5;  // same (oriented) shell pair on both sides
  return s;
}

}  // namespace lai
