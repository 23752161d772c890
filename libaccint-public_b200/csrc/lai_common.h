// Shared host/device definitions for the libaccint-b200 J/K engine.
//
// Work units follow the reference's shell-quartet model
// (include/libaccint/basis/shell_set_quartet.hpp): a canonical contracted shell
// quartet (ij|kl) is one unit.  Shells are grouped into SHELL PAIRS; pairs with the
// same (la, lb, Ka, Kb) form a PAIR CLASS (the reference keys ShellSets by (l, K),
// src/shared/basis/basis_set.cpp:191-211; here K counts NONZERO primitives only).
// Inside a class the pairs are sorted by their Schwarz bound Q (descending), so the
// ket partners of a bra pair that pass Q_bra*Q_ket >= thr form a prefix of the
// ket class list -- quartet lists are never materialized.
#pragma once

#include <cstdint>

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#define __device__
#define __forceinline__ inline
#endif
#endif

namespace lai {

constexpr int kMaxL = 4;          // shells up to g (the reference's LIBACCINT_MAX_AM)
constexpr int kMaxLDeriv = 5;     // l+1 shells needed by the derivative integrals
constexpr int kMaxRoots = 9;      // n = (la+lb+lc+ld)/2 + 1 <= 9 for l <= 4 (+1 derivative)

// Fields of one primitive pair, stored SoA as prim[f * (Kab * npairs) + t * npairs + p]
// (t = primitive-pair index, p = pair index in the class), so that lanes working on
// consecutive pairs load consecutive addresses.
enum PrimField : int {
  PF_ZETA = 0,   // zeta = alpha_a + alpha_b
  PF_HZ,         // 0.5 / zeta
  PF_PX, PF_PY, PF_PZ,     // Gaussian product centre P
  PF_PAX, PF_PAY, PF_PAZ,  // P - A
  PF_C,          // sqrt(2) pi^{5/4} c_a c_b exp(-alpha_a alpha_b |AB|^2 / zeta) / zeta
  PF_Q,          // primitive Schwarz bound sqrt(max |(a_p b_q|a_p b_q)|); primitive pairs
                 // of each shell pair are stored in descending PF_Q order
  PF_ALPHA,      // alpha_a, the exponent on the first shell (nuclear derivatives)
  PF_COUNT
};

// The same primitive-pair data per pair (AoS), for the kernels whose whole warp
// reads one pair's primitives (the bra of the thread-per-quartet kernels): record
// [p][t][kBraRec] with the fields below, so that one pair's primitives are a few
// contiguous cache lines (SoA by pair index spreads them over one line per field
// and primitive) and each record is read with 16-byte vector loads.
enum BraRecField : int {
  BR_Q = 0, BR_ZETA, BR_HZ, BR_C,   // first 16 bytes (FP32) / first two double2 (FP64)
  BR_PX, BR_PY, BR_PZ, BR_PAD0,
  BR_PAX, BR_PAY, BR_PAZ, BR_PAD1,
  kBraRec
};

// The same data tiled for the ket side of the thread-per-quartet kernels, whose
// lanes read consecutive pairs: [npairs / 32 tiles][Ka*Kb][kKetRec][32], field f
// of primitive t of pair q at ((q / 32 * Kab + t) * kKetRec + f) * 32 + q % 32.
// A field's 32 lanes stay contiguous (coalesced, as in the SoA table), and the
// fields and primitives of one pair are at fixed offsets from one address (no
// per-field address arithmetic in the primitive loop).
enum KetRecField : int {
  KR_Q = 0, KR_ETA, KR_HE, KR_PX, KR_PY, KR_PZ, KR_QCX, KR_QCY, KR_QCZ, KR_C,
  KR_ALPHA,  // exponent on the pair's first shell (the gradient kernels)
  kKetRec
};
constexpr int kKetTile = 32;

struct PairClassDev {
  int la, lb;          // la >= lb (pairs are oriented so the bra-side HRR moves to the smaller l)
  int Ka, Kb;          // nonzero primitive counts
  int npairs;
  const int* shell_a;  // [npairs] shell index of the first (higher-l) shell
  const int* shell_b;  // [npairs]
  const int* func_a;   // [npairs] first basis-function index of shell a
  const int* func_b;   // [npairs]
  const double* Q;     // [npairs] Schwarz bound, descending
  const double* AB;    // [3 * npairs] A - B, SoA
  const double* Acen;  // [3 * npairs] centre A of the first shell, SoA
  const double* prim;  // [PF_COUNT * Ka*Kb * npairs]
  double qprim_max;    // largest PF_Q of the class
  const int* sys;      // [npairs] system of each pair in a batched engine, else nullptr
  const float* primf;  // FP32 copy of prim (the FP32 kernels of mixed precision)
  const double* primb;  // [npairs][Ka*Kb][kBraRec] per-pair records (BraRecField)
  const float* primbf;  // FP32 copy of primb
  const double* primk;  // ket tiles (KetRecField), ceil(npairs / 32) * Ka*Kb * kKetRec * 32
  const float* primkf;  // FP32 copy of primk
};

// One launch: the canonical quartets (p, q) with p a pair of class `bra` and q a
// pair of class `ket` in the ket range [qbegin(p), qbegin(p) + count(p)), where
// offsets[p] = sum_{p' < p} count(p') and qbegin(p) = qbegin ? qbegin[p] : 0.
// For the FP64 part of a block qbegin is null; the FP32 part of a mixed-precision
// build starts where the FP64 prefix of each bra row ends.  When bra and ket are
// the same class, q <= p (canonical bra >= ket).
struct QuartetBlock {
  PairClassDev bra, ket;
  const int64_t* offsets;   // [bra.npairs + 1]
  const int* qbegin;        // [bra.npairs] or nullptr
  int64_t t_begin;          // a launch covers flat quartet indices [t_begin, total)
  int64_t total;
  int same_class;
};

}  // namespace lai
