// Host orchestration of the J/K engine and the C ABI (include/libaccint_b200.h).
//
// Pipeline of one engine (built once per basis, reused for every density):
//   1. lai_basis_create: normalize contraction coefficients like the reference
//      Shell constructor (src/shared/basis/shell.cpp:32-113); drop primitives whose
//      normalized coefficient is exactly zero (general-contraction padding kept by
//      the reference's BSE reader, src/shared/data/bse_json_parser.cpp:43-57 --
//      their contribution is exactly zero).
//   2. Shell pairs (i >= j) oriented so la >= lb, grouped into pair classes
//      (la, lb, Ka, Kb); primitive-pair data (zeta, P, P-A, prefactor) in SoA.
//   3. Schwarz bounds from the diagonal quartets (ab|ab) on the device
//      (src/shared/screening/schwarz_bounds.cpp:20-59 computes the same on the host).
//   4. Pairs sorted by Q (descending) within their class; pairs with
//      Q * Q_max < threshold dropped; for every ordered class pair (bra >= ket) the
//      number of passing kets of each bra pair is a prefix length (binary search),
//      prefix-summed into the launch's flat quartet range.
//   5. lai_jk_build: one launch per class pair (thread-per-quartet kernels for the
//      small classes, warp-per-quartet otherwise), then J = J' + J'^T, K = K' + K'^T.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/libaccint_b200.h"
#include "engine_internal.h"
#include "eri_kernels.h"
#include "rys_tables.inc"
#include "fp32_tables.h"

namespace lai {
void spherical_forget_basis(const lai_basis* basis);  // spherical.cu
}  // namespace lai

using namespace lai::host;

static_assert(RYS_DEG == lai::kRysDeg, "table degree mismatch");
static_assert(BOYS_NM == lai::kBoysNM, "Boys table width mismatch");
static_assert(BOYS_NGRID == lai::kBoysNGrid, "Boys grid mismatch");

namespace lai {
namespace host {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

double dfact_odd(int l) {
  double r = 1;
  for (int k = 2 * l - 1; k > 1; k -= 2) r *= k;
  return r;
}

}  // namespace host
}  // namespace lai

// ---------------------------------------------------------------------------
// Basis
// ---------------------------------------------------------------------------

extern "C" {

const char* lai_last_error(void) { return g_last_error.c_str(); }
int lai_abi_version(void) { return LAI_ABI_VERSION; }

int lai_basis_create(int nshell, const int* l, const int* nprim, const double* centers,
                     const double* exps, const double* coefs, const int* atom_index, int flags,
                     lai_basis** out) {
  if (!out) return fail(LAI_EINVAL, "lai_basis_create: out is NULL");
  *out = nullptr;
  if (nshell < 0 || (nshell > 0 && (!l || !nprim || !centers || !exps || !coefs)))
    return fail(LAI_EINVAL, "lai_basis_create: null array");
  auto b = std::make_unique<lai_basis>();
  long off = 0;
  for (int s = 0; s < nshell; ++s) {
    if (l[s] < 0 || l[s] > lai::kMaxL)
      return fail(LAI_EINVAL, "lai_basis_create: shell " + std::to_string(s) +
                                  " angular momentum outside [0, 4]");
    if (nprim[s] < 1) return fail(LAI_EINVAL, "lai_basis_create: shell with no primitive");
    HostShell sh;
    sh.l = l[s];
    for (int x = 0; x < 3; ++x) sh.center[x] = centers[3 * s + x];
    sh.atom = atom_index ? atom_index[s] : -1;
    sh.exps_all.assign(exps + off, exps + off + nprim[s]);
    sh.coefs_all.assign(coefs + off, coefs + off + nprim[s]);
    off += nprim[s];
    for (double e : sh.exps_all)
      if (!(e > 0.0)) return fail(LAI_EINVAL, "lai_basis_create: non-positive exponent");
    if (!(flags & LAI_BASIS_PRENORMALIZED)) {
      // Reference Shell normalization (shell.cpp:32-113): primitive factor
      // (2a/pi)^{3/4} (4a)^{l/2} / sqrt((2l-1)!!), then unit (l,0,0) self-overlap.
      const int L = sh.l;
      const int n = (int)sh.exps_all.size();
      for (int p = 0; p < n; ++p) {
        const double a = sh.exps_all[p];
        sh.coefs_all[p] *= std::pow(2.0 * a / M_PI, 0.75) * std::pow(4.0 * a, 0.5 * L) /
                           std::sqrt(dfact_odd(L));
      }
      double ov = 0.0;
      for (int p = 0; p < n; ++p)
        for (int q = 0; q < n; ++q) {
          const double z = sh.exps_all[p] + sh.exps_all[q];
          double o = std::pow(M_PI / z, 1.5);
          for (int k = 0; k < L; ++k) o *= 0.5 / z;
          ov += sh.coefs_all[p] * sh.coefs_all[q] * o;
        }
      if (!(ov > 0.0)) return fail(LAI_EINVAL, "lai_basis_create: zero contraction");
      const double sc = 1.0 / std::sqrt(ov);
      for (auto& c : sh.coefs_all) c *= sc;
    }
    for (size_t p = 0; p < sh.exps_all.size(); ++p)
      if (sh.coefs_all[p] != 0.0) {
        sh.exps.push_back(sh.exps_all[p]);
        sh.coefs.push_back(sh.coefs_all[p]);
      }
    if (sh.exps.empty()) return fail(LAI_EINVAL, "lai_basis_create: all coefficients zero");
    sh.func = b->nbf;
    b->nbf += lai::ncart(sh.l);
    b->shells.push_back(std::move(sh));
  }
  *out = b.release();
  return LAI_OK;
}

void lai_basis_destroy(lai_basis* basis) {
  if (!basis) return;
  lai::spherical_forget_basis(basis);
  delete basis;
}
long lai_basis_nbf(const lai_basis* basis) { return basis ? basis->nbf : 0; }
int lai_basis_nshell(const lai_basis* basis) { return basis ? (int)basis->shells.size() : 0; }

int lai_basis_shell(const lai_basis* basis, int s, int* l, int* nprim, double* center,
                    double* exps, double* coefs, long* func_index) {
  if (!basis || s < 0 || s >= (int)basis->shells.size())
    return fail(LAI_EINVAL, "lai_basis_shell: bad shell index");
  const HostShell& sh = basis->shells[s];
  if (l) *l = sh.l;
  if (nprim) *nprim = (int)sh.exps_all.size();
  if (center) for (int x = 0; x < 3; ++x) center[x] = sh.center[x];
  if (exps) std::copy(sh.exps_all.begin(), sh.exps_all.end(), exps);
  if (coefs) std::copy(sh.coefs_all.begin(), sh.coefs_all.end(), coefs);
  if (func_index) *func_index = sh.func;
  return LAI_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
namespace lai {
namespace host {


// Algorithmic FP work of one canonical quartet (one unit), the single accounting
// used for roofline fractions:  P (40 + 64 n + n (20 + T2D + 4 Ncart)) + 25 Ncart
// with P the product of nonzero primitive counts, n the root count and
// T2D = 3 [5 (La+Lb+1)(Lc+Ld+1) + 2 Lb (La+Lb+1)(Lc+Ld+1)(Ld+1) + 2 Ld (La+1)(Lb+1)(Lc+Ld+1)].
double alg_per_prim(int la, int lb, int lc, int ld) {
  const int n = (la + lb + lc + ld) / 2 + 1;
  const double nc = (double)lai::ncart(la) * lai::ncart(lb) * lai::ncart(lc) * lai::ncart(ld);
  const double t2d = 3.0 * (5.0 * (la + lb + 1) * (lc + ld + 1) +
                            2.0 * lb * (la + lb + 1) * (lc + ld + 1) * (ld + 1) +
                            2.0 * ld * (la + 1) * (lb + 1) * (lc + ld + 1));
  return 40.0 + 64.0 * n + n * (20.0 + t2d + 4.0 * nc);
}
double alg_per_quartet(int la, int lb, int lc, int ld) {
  return 25.0 * lai::ncart(la) * lai::ncart(lb) * lai::ncart(lc) * lai::ncart(ld);
}
double alg_work(int la, int lb, int lc, int ld, int Ka, int Kb, int Kc, int Kd) {
  const double P = (double)Ka * Kb * Kc * Kd;
  return P * alg_per_prim(la, lb, lc, ld) + alg_per_quartet(la, lb, lc, ld);
}

__global__ void symmetrize_kernel(const double* __restrict__ Jp, const double* __restrict__ Kp,
                                  double* __restrict__ J, double* __restrict__ K, int n) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * n) return;
  const int i = (int)(idx / n), j = (int)(idx - (int64_t)i * n);
  const int64_t tr = (int64_t)j * n + i;
  J[idx] = Jp[idx] + Jp[tr];
  K[idx] = Kp[idx] + Kp[tr];
}

}  // namespace host
}  // namespace lai


namespace lai {
namespace host {

int build_classes(lai_engine* E) {
  const auto& sh = E->basis->shells;
  const int ns = (int)sh.size();
  // class key -> index
  std::vector<std::array<int, 4>> keys;
  auto class_of = [&](int la, int lb, int Ka, int Kb) {
    std::array<int, 4> k{la, lb, Ka, Kb};
    for (size_t i = 0; i < keys.size(); ++i)
      if (keys[i] == k) return (int)i;
    keys.push_back(k);
    E->classes.push_back(std::make_unique<PairClassHost>());
    auto& c = *E->classes.back();
    c.la = la; c.lb = lb; c.Ka = Ka; c.Kb = Kb;
    return (int)keys.size() - 1;
  };
  // pairs within one system only (shells of a system are contiguous)
  int sys_first = 0;
  for (int i = 0; i < ns; ++i) {
    if (i > 0 && sh[i].sys != sh[i - 1].sys) sys_first = i;
    for (int j = sys_first; j <= i; ++j) {
      int a = i, b = j;
      const int Ki = (int)sh[i].exps.size(), Kj = (int)sh[j].exps.size();
      // orient: higher l first, then more primitives first
      if (sh[j].l > sh[i].l || (sh[j].l == sh[i].l && Kj > Ki)) std::swap(a, b);
      const HostShell& A = sh[a];
      const HostShell& B = sh[b];
      const int ci = class_of(A.l, B.l, (int)A.exps.size(), (int)B.exps.size());
      auto& c = *E->classes[ci];
      c.sa.push_back(a); c.sb.push_back(b);
      c.fa.push_back((int)A.func); c.fb.push_back((int)B.func);
      c.sys.push_back(A.sys);
    }
  }
  // sort classes by key so that bra >= ket implies (la,lb) >= (lc,ld)
  std::vector<int> order(keys.size());
  std::iota(order.begin(), order.end(), 0);
  std::sort(order.begin(), order.end(), [&](int x, int y) { return keys[x] < keys[y]; });
  std::vector<std::unique_ptr<PairClassHost>> sorted;
  for (int o : order) sorted.push_back(std::move(E->classes[o]));
  E->classes = std::move(sorted);
  return LAI_OK;
}

void fill_pair_data(const lai_basis* basis, PairClassHost& c) {
  const auto& sh = basis->shells;
  const int n = c.n();
  const int Kab = c.Ka * c.Kb;
  c.AB.assign(3 * (size_t)n, 0.0);
  c.Acen.assign(3 * (size_t)n, 0.0);
  c.prim.assign((size_t)lai::PF_COUNT * Kab * n, 0.0);
  const double pi54s2 = std::sqrt(2.0) * std::pow(M_PI, 1.25);
  for (int p = 0; p < n; ++p) {
    const HostShell& A = sh[c.sa[p]];
    const HostShell& B = sh[c.sb[p]];
    double AB[3], ab2 = 0;
    for (int x = 0; x < 3; ++x) {
      AB[x] = A.center[x] - B.center[x];
      ab2 += AB[x] * AB[x];
      c.AB[(size_t)x * n + p] = AB[x];
      c.Acen[(size_t)x * n + p] = A.center[x];
    }
    for (int ia = 0; ia < c.Ka; ++ia)
      for (int ib = 0; ib < c.Kb; ++ib) {
        const int t = ia * c.Kb + ib;
        const double al = A.exps[ia], be = B.exps[ib];
        const double z = al + be;
        auto at = [&](int f) -> double& { return c.prim[((size_t)f * Kab + t) * n + p]; };
        at(lai::PF_ZETA) = z;
        at(lai::PF_ALPHA) = al;
        at(lai::PF_HZ) = 0.5 / z;
        for (int x = 0; x < 3; ++x) {
          const double P = (al * A.center[x] + be * B.center[x]) / z;
          at(lai::PF_PX + x) = P;
          at(lai::PF_PAX + x) = P - A.center[x];
        }
        at(lai::PF_C) = pi54s2 * A.coefs[ia] * B.coefs[ib] * std::exp(-al * be / z * ab2) / z;
      }
  }
}

int upload_class(PairClassHost& c) {
  LAI_CUDA_TRY(upload(c.d_sa, c.sa));
  LAI_CUDA_TRY(upload(c.d_sb, c.sb));
  LAI_CUDA_TRY(upload(c.d_fa, c.fa));
  LAI_CUDA_TRY(upload(c.d_fb, c.fb));
  LAI_CUDA_TRY(upload(c.d_AB, c.AB));
  LAI_CUDA_TRY(upload(c.d_Acen, c.Acen));
  LAI_CUDA_TRY(upload(c.d_prim, c.prim));
  if (c.Q.empty()) c.Q.assign(c.n(), 0.0);
  LAI_CUDA_TRY(upload(c.d_Q, c.Q));
  {  // per-pair primitive records (lai::BraRecField), FP64 and FP32
    const int n = c.n(), Kab = c.Ka * c.Kb;
    std::vector<double> rb((size_t)n * Kab * lai::kBraRec, 0.0);
    static const int from[lai::kBraRec] = {lai::PF_Q,  lai::PF_ZETA, lai::PF_HZ,  lai::PF_C,
                                           lai::PF_PX, lai::PF_PY,   lai::PF_PZ,  -1,
                                           lai::PF_PAX, lai::PF_PAY, lai::PF_PAZ, -1};
    for (int p = 0; p < n; ++p)
      for (int t = 0; t < Kab; ++t)
        for (int f = 0; f < lai::kBraRec; ++f)
          if (from[f] >= 0)
            rb[((size_t)p * Kab + t) * lai::kBraRec + f] = c.prim[((size_t)from[f] * Kab + t) * n + p];
    std::vector<float> rbf(rb.size());
    for (size_t i = 0; i < rb.size(); ++i) rbf[i] = (float)rb[i];
    LAI_CUDA_TRY(upload(c.d_primb, rb));
    LAI_CUDA_TRY(upload(c.d_primbf, rbf));
  }
  {  // ket tiles of 32 pairs (lai::KetRecField), FP64 and FP32; pad lanes stay 0
    const int n = c.n(), Kab = c.Ka * c.Kb;
    const size_t ntile = ((size_t)n + lai::kKetTile - 1) / lai::kKetTile;
    std::vector<double> rk(ntile * Kab * lai::kKetRec * lai::kKetTile, 0.0);
    static const int from[lai::kKetRec] = {lai::PF_Q,   lai::PF_ZETA, lai::PF_HZ,  lai::PF_PX,
                                           lai::PF_PY,  lai::PF_PZ,   lai::PF_PAX, lai::PF_PAY,
                                           lai::PF_PAZ, lai::PF_C,    lai::PF_ALPHA};
    for (int p = 0; p < n; ++p)
      for (int t = 0; t < Kab; ++t)
        for (int f = 0; f < lai::kKetRec; ++f)
          rk[(((size_t)(p / lai::kKetTile) * Kab + t) * lai::kKetRec + f) * lai::kKetTile + p % lai::kKetTile] =
              c.prim[((size_t)from[f] * Kab + t) * n + p];
    std::vector<float> rkf(rk.size());
    for (size_t i = 0; i < rk.size(); ++i) rkf[i] = (float)rk[i];
    LAI_CUDA_TRY(upload(c.d_primk, rk));
    LAI_CUDA_TRY(upload(c.d_primkf, rkf));
  }
  return LAI_OK;
}

int ensure_scratch(lai_engine* E, size_t doubles) {
  if (doubles <= E->scratch_doubles) return LAI_OK;
  E->release_graph();
  LAI_CUDA_TRY(E->d_scratch.alloc(doubles * sizeof(double)));
  E->scratch_doubles = doubles;
  return LAI_OK;
}

// Launches the kernel of the block's class.  fp32 asks for the FP32 variant; the
// classes without one (generic kernel) run in FP64, and *ran_fp32 says which ran.
int launch_block(lai_engine* E, const lai::QuartetBlock& blk, const lai::JKArgs& args,
                 bool fp32, bool* ran_fp32, lai::LaunchTune tune) {
  const int la = blk.bra.la, lb = blk.bra.lb, lc = blk.ket.la, ld = blk.ket.lb;
  if (ran_fp32) *ran_fp32 = false;
  if (lai::small_class_supported(la, lb, lc, ld)) {
    const int rc = lai::launch_small(blk, args, E->tab, E->stream, fp32, E->num_sms, tune);
    if (ran_fp32) *ran_fp32 = fp32;
    if (rc < 0) return fail(LAI_ECUDA, std::string("small-class launch failed: ") +
                                           cudaGetErrorString(cudaGetLastError()));
    return LAI_OK;
  }
  // the other classes: warp-per-quartet, bra-sliced or tiled kernel, as tuned for
  // this block (lai_engine_autotune) or by the measured per-class default; FP32
  // requests go to the sliced kernel where it exists, else to the warp-per-quartet
  // kernel's FP32 variant (d and f classes; the tiled and generic kernels are FP64
  // only)
  int kern = tune.kernel != lai::KERNEL_DEFAULT ? tune.kernel : lai::default_kernel(la, lb, lc, ld);
  if (fp32 && lai::sliced_class_supported(la, lb, lc, ld)) kern = lai::KERNEL_SLICED;
  else if (fp32 && lai::warpq_class_supported(la, lb, lc, ld)) kern = lai::KERNEL_WARPQ;
  if (kern == lai::KERNEL_WARPQ) {
    const int rc = lai::launch_warpq(blk, args, E->tab, E->stream, E->num_sms, fp32);
    if (rc == 1) {
      if (ran_fp32) *ran_fp32 = true;
      return LAI_OK;
    }
    if (rc == 0) return LAI_OK;
    if (rc < -1) return fail(LAI_ECUDA, std::string("warp-per-quartet launch failed: ") +
                                            cudaGetErrorString(lai::warpq_launch_error()));
  }
  if (kern != lai::KERNEL_TILED && lai::sliced_class_supported(la, lb, lc, ld)) {
    const int rc = lai::launch_sliced(blk, args, E->tab, E->stream, fp32, E->num_sms);
    if (ran_fp32) *ran_fp32 = fp32;
    if (rc < 0) return fail(LAI_ECUDA, std::string("sliced launch failed: ") +
                                           cudaGetErrorString(cudaGetLastError()));
    return LAI_OK;
  }
  {
    const int rc = lai::launch_tiled(blk, args, E->tab, E->stream, E->num_sms);
    if (rc == 0) return LAI_OK;
    if (rc < -1) return fail(LAI_ECUDA, std::string("tiled launch failed: ") +
                                            cudaGetErrorString(cudaGetLastError()));
  }
  const size_t need = lai::generic_global_scratch_doubles(la, lb, lc, ld, E->num_sms);
  if (int rc = ensure_scratch(E, need)) return rc;
  const int rc = lai::launch_generic(blk, args, E->tab, E->stream, E->d_scratch.as<double>(),
                                     E->scratch_doubles, E->num_sms);
  if (rc < 0) return fail(LAI_ECUDA, std::string("generic launch failed: ") +
                                         cudaGetErrorString(cudaGetLastError()));
  return LAI_OK;
}

int compute_schwarz(lai_engine* E) {
  // Diagonal quartets (ab|ab) of every pair: offsets[p] = p, qbegin[p] = p.
  for (auto& cp : E->classes) {
    auto& c = *cp;
    const int n = c.n();
    std::vector<int64_t> off(n + 1);
    std::vector<int> qb(n);
    for (int p = 0; p <= n; ++p) off[p] = p;
    for (int p = 0; p < n; ++p) qb[p] = p;
    DevBuf d_off, d_qb, d_out;
    LAI_CUDA_TRY(upload(d_off, off));
    LAI_CUDA_TRY(upload(d_qb, qb));
    LAI_CUDA_TRY(d_out.alloc(sizeof(double) * n));
    lai::QuartetBlock blk{};
    blk.bra = blk.ket = c.view();
    blk.offsets = d_off.as<int64_t>();
    blk.qbegin = d_qb.as<int>();
    blk.total = n;
    blk.same_class = 1;
    lai::JKArgs args{};
    args.mode = lai::MODE_SCHWARZ;
    args.schwarz_out = d_out.as<double>();
    if (int rc = launch_block(E, blk, args)) return rc;
    c.Q.resize(n);
    LAI_CUDA_TRY(cudaMemcpyAsync(c.Q.data(), d_out.p, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                 E->stream));
    LAI_CUDA_TRY(cudaStreamSynchronize(E->stream));
  }
  return LAI_OK;
}

// Primitive Schwarz bounds: every primitive pair of every shell pair is run as a
// one-primitive pair through the diagonal kernel, q = sqrt(max |(a_p b_q|a_p b_q)|)
// (contraction coefficients included).  By the Schwarz inequality a primitive
// quartet contributes at most q_ab q_cd to any integral of its quartet.
int compute_prim_schwarz(lai_engine* E) {
  for (auto& cp : E->classes) {
    auto& c = *cp;
    const int n = c.n();
    const int Kab = c.Ka * c.Kb;
    const int ne = n * Kab;
    if (ne == 0) continue;
    PairClassHost pc;
    pc.la = c.la; pc.lb = c.lb; pc.Ka = 1; pc.Kb = 1;
    pc.sa.resize(ne); pc.sb.resize(ne); pc.fa.resize(ne); pc.fb.resize(ne);
    pc.AB.resize(3 * (size_t)ne);
    pc.Acen.resize(3 * (size_t)ne);
    pc.prim.assign((size_t)lai::PF_COUNT * ne, 0.0);
    for (int p = 0; p < n; ++p)
      for (int t = 0; t < Kab; ++t) {
        const int e = p * Kab + t;
        pc.sa[e] = c.sa[p]; pc.sb[e] = c.sb[p]; pc.fa[e] = c.fa[p]; pc.fb[e] = c.fb[p];
        for (int x = 0; x < 3; ++x) {
          pc.AB[(size_t)x * ne + e] = c.AB[(size_t)x * n + p];
          pc.Acen[(size_t)x * ne + e] = c.Acen[(size_t)x * n + p];
        }
        for (int f = 0; f < lai::PF_COUNT; ++f)
          pc.prim[(size_t)f * ne + e] = c.prim[((size_t)f * Kab + t) * n + p];
      }
    if (int rc = upload_class(pc)) return rc;
    std::vector<int64_t> off(ne + 1);
    std::vector<int> qb(ne);
    for (int e = 0; e <= ne; ++e) off[e] = e;
    for (int e = 0; e < ne; ++e) qb[e] = e;
    DevBuf d_off, d_qb, d_out;
    LAI_CUDA_TRY(upload(d_off, off));
    LAI_CUDA_TRY(upload(d_qb, qb));
    LAI_CUDA_TRY(d_out.alloc(sizeof(double) * ne));
    lai::QuartetBlock blk{};
    blk.bra = blk.ket = pc.view();
    blk.offsets = d_off.as<int64_t>();
    blk.qbegin = d_qb.as<int>();
    blk.total = ne;
    blk.same_class = 1;
    lai::JKArgs args{};
    args.mode = lai::MODE_SCHWARZ;
    args.schwarz_out = d_out.as<double>();
    if (int rc = launch_block(E, blk, args)) return rc;
    std::vector<double> q(ne);
    LAI_CUDA_TRY(cudaMemcpyAsync(q.data(), d_out.p, sizeof(double) * ne, cudaMemcpyDeviceToHost,
                                 E->stream));
    LAI_CUDA_TRY(cudaStreamSynchronize(E->stream));
    for (int p = 0; p < n; ++p)
      for (int t = 0; t < Kab; ++t)
        c.prim[((size_t)lai::PF_Q * Kab + t) * n + p] = q[(size_t)p * Kab + t];
  }
  return LAI_OK;
}

int sort_and_screen(lai_engine* E) {
  const int ns = (int)E->basis->shells.size();
  const bool batched = E->nsys > 1;
  if (!batched) E->Q_all.assign((size_t)ns * ns, 0.0);  // (a full matrix only for one system)
  double qmax = 0.0;
  for (auto& cp : E->classes)
    for (int p = 0; p < cp->n(); ++p) {
      qmax = std::max(qmax, cp->Q[p]);
      if (!batched) {
        E->Q_all[(size_t)cp->sa[p] * ns + cp->sb[p]] = cp->Q[p];
        E->Q_all[(size_t)cp->sb[p] * ns + cp->sa[p]] = cp->Q[p];
      }
    }
  for (auto& cp : E->classes) {
    auto& c = *cp;
    const int n = c.n();
    // pairs ordered by system, then by Schwarz bound (descending); pairs that pass
    // with no partner dropped -- each system's kept pairs are a prefix of its segment
    std::vector<int> idx;
    idx.reserve(n);
    for (int i = 0; i < n; ++i)
      if (c.Q[i] * qmax >= E->thr) idx.push_back(i);
    std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
      return c.sys[x] != c.sys[y] ? c.sys[x] < c.sys[y] : c.Q[x] > c.Q[y];
    });
    const int keep = (int)idx.size();
    const int Kab = c.Ka * c.Kb;
    auto perm = [&](const std::vector<int>& v) {
      std::vector<int> o(keep);
      for (int i = 0; i < keep; ++i) o[i] = v[idx[i]];
      return o;
    };
    std::vector<double> Q(keep), AB(3 * (size_t)keep), Acen(3 * (size_t)keep),
        prim((size_t)lai::PF_COUNT * Kab * keep);
    for (int i = 0; i < keep; ++i) {
      Q[i] = c.Q[idx[i]];
      for (int x = 0; x < 3; ++x) {
        AB[(size_t)x * keep + i] = c.AB[(size_t)x * n + idx[i]];
        Acen[(size_t)x * keep + i] = c.Acen[(size_t)x * n + idx[i]];
      }
      for (int f = 0; f < lai::PF_COUNT * Kab; ++f)
        prim[(size_t)f * keep + i] = c.prim[(size_t)f * n + idx[i]];
    }
    // primitive pairs of each shell pair in descending primitive-Schwarz order
    c.qprim_max = 0.0;
    std::vector<int> tix(Kab);
    std::vector<double> tmp(Kab);
    for (int i = 0; i < keep; ++i) {
      auto qat = [&](int t) { return prim[((size_t)lai::PF_Q * Kab + t) * keep + i]; };
      std::iota(tix.begin(), tix.end(), 0);
      std::stable_sort(tix.begin(), tix.end(), [&](int x, int y) { return qat(x) > qat(y); });
      for (int f = 0; f < lai::PF_COUNT; ++f) {
        for (int t = 0; t < Kab; ++t) tmp[t] = prim[((size_t)f * Kab + tix[t]) * keep + i];
        for (int t = 0; t < Kab; ++t) prim[((size_t)f * Kab + t) * keep + i] = tmp[t];
      }
      c.qprim_max = std::max(c.qprim_max, qat(0));
    }
    c.sa = perm(c.sa); c.sb = perm(c.sb); c.fa = perm(c.fa); c.fb = perm(c.fb);
    c.sys = perm(c.sys);
    c.Q = std::move(Q); c.AB = std::move(AB); c.Acen = std::move(Acen); c.prim = std::move(prim);
    c.seg.assign(E->nsys + 1, 0);
    for (int i = 0, s = 0; s <= E->nsys; ++s) {
      while (i < keep && c.sys[i] < s) ++i;
      c.seg[s] = i;
    }
    c.batched = batched;
    if (int rc = upload_class(c)) return rc;
    if (batched) LAI_CUDA_TRY(upload(c.d_sys, c.sys));
    {  // FP32 copy of the primitive-pair table for the FP32 kernels
      std::vector<float> pf(c.prim.size());
      for (size_t i = 0; i < pf.size(); ++i) pf[i] = (float)c.prim[i];
      LAI_CUDA_TRY(upload(c.d_primf, pf));
    }
  }
  // quartet blocks
  const int nc = (int)E->classes.size();
  for (int A = 0; A < nc; ++A)
    for (int B = 0; B <= A; ++B) {
      const auto& ca = *E->classes[A];
      const auto& cb = *E->classes[B];
      if (ca.n() == 0 || cb.n() == 0) continue;
      auto blk = std::make_unique<ClassPairBlock>();
      blk->bra = A;
      blk->ket = B;
      blk->offsets.resize(ca.n() + 1);
      blk->offsets[0] = 0;
      if (batched) blk->qbegin.resize(ca.n());
      for (int p = 0; p < ca.n(); ++p) {
        // largest prefix of the bra pair's system segment of the ket list with
        // Q_p * Q_q >= thr (the whole list for a single system)
        const int s0 = cb.seg[ca.sys[p]], s1 = cb.seg[ca.sys[p] + 1];
        int lo = s0, hi = s1;
        while (lo < hi) {
          const int mid = (lo + hi) / 2;
          if (ca.Q[p] * cb.Q[mid] >= E->thr) lo = mid + 1; else hi = mid;
        }
        int cnt = lo - s0;
        if (A == B) cnt = std::min(cnt, p - s0 + 1);  // canonical q <= p (same segment)
        blk->offsets[p + 1] = blk->offsets[p] + cnt;
        if (batched) blk->qbegin[p] = s0;
      }
      blk->total = blk->offsets[ca.n()];
      if (blk->total == 0) continue;
      if (batched) LAI_CUDA_TRY(upload(blk->d_qbegin, blk->qbegin));
      blk->alg_flops = alg_work(ca.la, ca.lb, cb.la, cb.lb, ca.Ka, ca.Kb, cb.Ka, cb.Kb);
      blk->flops_per_prim = alg_per_prim(ca.la, ca.lb, cb.la, cb.lb);
      blk->flops_per_quartet = alg_per_quartet(ca.la, ca.lb, cb.la, cb.lb);
      LAI_CUDA_TRY(upload(blk->d_offsets, blk->offsets));
      E->blocks.push_back(std::move(blk));
    }
  return LAI_OK;
}

lai::QuartetBlock make_block(const lai_engine* E, const ClassPairBlock& b) {
  lai::QuartetBlock q{};
  q.bra = E->classes[b.bra]->view();
  q.ket = E->classes[b.ket]->view();
  q.offsets = b.d_offsets.as<int64_t>();
  q.qbegin = b.qbegin.empty() ? nullptr : b.d_qbegin.as<int>();
  q.total = b.total;
  q.same_class = (b.bra == b.ket);
  return q;
}

__global__ void absmax_kernel(const double* __restrict__ x, size_t n, unsigned long long* out) {
  double m = 0.0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    m = fmax(m, fabs(x[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  // non-negative doubles order like their bit patterns
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// max |x_i| of a device array (one stream synchronisation).
int device_absmax(lai_engine* E, const double* x, size_t n, cudaStream_t stream, double* out) {
  if (E->d_absmax.bytes < sizeof(unsigned long long)) LAI_CUDA_TRY(E->d_absmax.alloc(sizeof(unsigned long long)));
  LAI_CUDA_TRY(cudaMemsetAsync(E->d_absmax.p, 0, sizeof(unsigned long long), stream));
  if (n > 0) {
    const size_t want = (n + 255) / 256;
    const unsigned grid = (unsigned)std::min<size_t>(want, (size_t)E->num_sms * 8);
    absmax_kernel<<<grid, 256, 0, stream>>>(x, n, E->d_absmax.as<unsigned long long>());
    LAI_CUDA_TRY(cudaGetLastError());
  }
  unsigned long long bits = 0;
  LAI_CUDA_TRY(cudaMemcpyAsync(&bits, E->d_absmax.p, sizeof(bits), cudaMemcpyDeviceToHost, stream));
  LAI_CUDA_TRY(cudaStreamSynchronize(stream));
  std::memcpy(out, &bits, sizeof(double));
  return LAI_OK;
}

// Elements of the engine's D/J/K arrays: nbf^2, or the packed blocks of a batched engine.
size_t engine_mat_elems(const lai_engine* E) {
  if (E->nsys > 1) return (size_t)E->sys_off[E->nsys];
  return (size_t)E->basis->nbf * (size_t)E->basis->nbf;
}

// Builds (once per cut value) the FP64/FP32 split of every block.
int build_split(lai_engine* E, double cut) {
  if (E->split_cut == cut) return LAI_OK;
  E->release_graph();  // a captured graph points into the buffers rebuilt here
  E->split_cut = -1.0;
  for (auto& bp : E->blocks) {
    auto& b = *bp;
    const auto& ca = *E->classes[b.bra];
    const auto& cb = *E->classes[b.ket];
    const int n = ca.n();
    std::vector<int64_t> o64(n + 1), o32(n + 1);
    std::vector<int> qb32(n);
    o64[0] = o32[0] = 0;
    for (int p = 0; p < n; ++p) {
      const int64_t cnt = b.offsets[p + 1] - b.offsets[p];
      const int base = b.qbegin.empty() ? 0 : b.qbegin[p];  // first ket of the bra's range
      int lo = 0, hi = (int)cnt;  // first ket with Q_p Q_q < cut
      while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (ca.Q[p] * cb.Q[base + mid] >= cut) lo = mid + 1; else hi = mid;
      }
      o64[p + 1] = o64[p] + lo;
      o32[p + 1] = o32[p] + (cnt - lo);
      qb32[p] = base + lo;
    }
    b.total64 = o64[n];
    b.total32 = o32[n];
    LAI_CUDA_TRY(upload(b.d_off64, o64));
    LAI_CUDA_TRY(upload(b.d_off32, o32));
    LAI_CUDA_TRY(upload(b.d_qb32, qb32));
  }
  E->split_cut = cut;
  return LAI_OK;
}

// J = J' + J'^T, K = K' + K'^T on every system block of a batched engine's packed
// matrices (block s = nbf_s x nbf_s at element offset off[s]).
__global__ void symmetrize_batched_kernel(const double* __restrict__ Jp, const double* __restrict__ Kp,
                                          double* __restrict__ J, double* __restrict__ K,
                                          const int64_t* __restrict__ off, const int* __restrict__ nbfs,
                                          int nsys) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= off[nsys]) return;
  int lo = 0, hi = nsys;  // off[lo] <= idx < off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= idx) lo = mid; else hi = mid;
  }
  const int n = nbfs[lo];
  const int64_t l = idx - off[lo];
  const int i = (int)(l / n), j = (int)(l - (int64_t)i * n);
  const int64_t tr = off[lo] + (int64_t)j * n + i;
  J[idx] = Jp[idx] + Jp[tr];
  K[idx] = Kp[idx] + Kp[tr];
}

// forced_cut >= 0: use this Schwarz cut for the FP32 split instead of deriving it
// from max|D| (which synchronizes the stream; not allowed while capturing a graph).
int run_jk(lai_engine* E, const double* dD, double* dJ, double* dK, cudaStream_t stream,
           const lai_jk_opts& o, lai_jk_report* rep, bool timed, double forced_cut = -1.0) {
  const int nbf = (int)E->basis->nbf;
  const bool batched = E->nsys > 1;
  const size_t elems = engine_mat_elems(E);
  const size_t bytes = sizeof(double) * elems;
  if (o.shard_count < 1 || o.shard_index < 0 || o.shard_index >= o.shard_count)
    return fail(LAI_EINVAL, "lai_jk: bad shard_index/shard_count");
  if (E->d_Jp.bytes < bytes) {
    E->release_graph();
    LAI_CUDA_TRY(E->d_Jp.alloc(bytes));
    LAI_CUDA_TRY(E->d_Kp.alloc(bytes));
  }
  cudaStream_t saved = E->stream;
  E->stream = stream;
  LAI_CUDA_TRY(cudaMemsetAsync(E->d_Jp.p, 0, bytes, stream));
  LAI_CUDA_TRY(cudaMemsetAsync(E->d_Kp.p, 0, bytes, stream));
  if (timed) LAI_CUDA_TRY(cudaEventRecord(E->ev0, stream));
  lai::JKArgs args{};
  args.D = dD;
  args.J = E->d_Jp.as<double>();
  args.K = E->d_Kp.as<double>();
  args.nbf = nbf;
  args.mode = lai::MODE_JK;
  args.prim_eps = E->prim_eps;
  args.prim_rel32 = o.fp32_prim_rel;
  if (batched) {
    args.sys_off = E->d_sys_off.as<int64_t>();
    args.sys_nbf = E->d_sys_nbf.as<int>();
  }
  int launches = 0;
  int64_t nq = 0, nq32 = 0;
  double flops = 0;
  // Mixed precision: a quartet runs in FP32 when Q_ij Q_kl max|D| < fp32_cut.  The
  // Schwarz cut fp32_cut / max|D| is rounded down to a power of two (conservative:
  // fewer FP32 quartets), so that the split, built on the host, is rebuilt only
  // when max|D| moves past a power of two.
  double cut = forced_cut >= 0.0 ? forced_cut : 0.0;
  if (o.fp32_cut > 0.0 && forced_cut < 0.0) {
    double maxd = 0.0;
    if (int rc = device_absmax(E, dD, elems, stream, &maxd)) { E->stream = saved; return rc; }
    if (maxd > 0.0 && std::isfinite(maxd)) cut = std::exp2(std::floor(std::log2(o.fp32_cut / maxd)));
  }
  const bool mixed = cut > 0.0;
  if (mixed) {
    if (int rc = build_split(E, cut)) { E->stream = saved; return rc; }
  }
  const int nparts = mixed ? 2 : 1;
  if (o.profile) {
    const size_t need = 2 * nparts * E->blocks.size();
    while (E->prof_ev.size() < need) {
      cudaEvent_t ev;
      LAI_CUDA_TRY(cudaEventCreate(&ev));
      E->prof_ev.push_back(ev);
    }
    E->prof_block.clear();
    E->prof_quartets.clear();
    if (E->d_prof_prims.bytes < sizeof(unsigned long long) * nparts * E->blocks.size())
      LAI_CUDA_TRY(E->d_prof_prims.alloc(sizeof(unsigned long long) *
                                         std::max<size_t>(1, nparts * E->blocks.size())));
    LAI_CUDA_TRY(cudaMemsetAsync(E->d_prof_prims.p, 0, E->d_prof_prims.bytes, stream));
  }
  E->prof_n = 0;
  for (size_t b = 0; b < E->blocks.size(); ++b) {
    const auto& bp = *E->blocks[b];
    for (int part = 0; part < nparts; ++part) {
      // part 0: the whole block (FP64), or its FP64 prefix when mixed; part 1: the
      // FP32 suffix
      lai::QuartetBlock q = make_block(E, bp);
      int64_t total = bp.total;
      if (mixed) {
        total = part == 0 ? bp.total64 : bp.total32;
        q.offsets = (part == 0 ? bp.d_off64 : bp.d_off32).as<int64_t>();
        if (part == 1) q.qbegin = bp.d_qb32.as<int>();  // the FP64 part keeps the block's ket starts
      }
      // this shard's contiguous slice of the part
      int64_t lo = 0, hi = 0;
      lai_shard_range(total, o.shard_index, o.shard_count, &lo, &hi);
      if (hi <= lo) continue;
      q.t_begin = lo;
      q.total = hi;
      args.prim_count = o.profile ? E->d_prof_prims.as<unsigned long long>() + E->prof_n : nullptr;
      if (o.profile) LAI_CUDA_TRY(cudaEventRecord(E->prof_ev[2 * E->prof_n], stream));
      bool ran32 = false;
      if (int rc = launch_block(E, q, args, part == 1, &ran32, bp.tune)) { E->stream = saved; return rc; }
      if (o.profile) {
        LAI_CUDA_TRY(cudaEventRecord(E->prof_ev[2 * E->prof_n + 1], stream));
        E->prof_block.push_back((int)b);
        E->prof_quartets.push_back(hi - lo);
        ++E->prof_n;
      }
      ++launches;
      nq += hi - lo;
      if (ran32) nq32 += hi - lo;
      flops += bp.alg_flops * (double)(hi - lo);
    }
  }
  const int64_t nn = (int64_t)elems;
  if (nn > 0) {
    if (batched)
      symmetrize_batched_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, stream>>>(
          E->d_Jp.as<double>(), E->d_Kp.as<double>(), dJ, dK, E->d_sys_off.as<int64_t>(),
          E->d_sys_nbf.as<int>(), E->nsys);
    else
      symmetrize_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, stream>>>(
          E->d_Jp.as<double>(), E->d_Kp.as<double>(), dJ, dK, nbf);
    ++launches;
  }
  LAI_CUDA_TRY(cudaGetLastError());
  if (timed) LAI_CUDA_TRY(cudaEventRecord(E->ev1, stream));
  E->stream = saved;
  if (rep) {
    rep->quartets_fp64 = nq - nq32;
    rep->quartets_fp32 = nq32;
    rep->fp32_schwarz_cut = cut;
    rep->alg_flops = flops;
    rep->kernel_launches = launches;
    rep->seconds_device = 0;
  }
  return LAI_OK;
}

// splitmix64
inline uint64_t mix64(uint64_t& x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void fp64_fma_probe(double* out, int iters) {
  double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-10, a2 = a0 + 2e-10, a3 = a0 + 3e-10;
  double a4 = a0 + 4e-10, a5 = a0 + 5e-10, a6 = a0 + 6e-10, a7 = a0 + 7e-10;
  const double m = 0.999999, c = 1e-7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
      a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
    }
  }
  const double r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (r == 12345.678) out[0] = r;  // keep the chain alive
}

}  // namespace host
}  // namespace lai

extern "C" {

int lai_shard_range(int64_t total, int index, int count, int64_t* lo, int64_t* hi) {
  if (count < 1 || index < 0 || index >= count || total < 0 || !lo || !hi)
    return fail(LAI_EINVAL, "lai_shard_range: bad arguments");
  // 128-bit products: total * count may exceed 63 bits for huge blocks
  *lo = (int64_t)((__int128)total * index / count);
  *hi = (int64_t)((__int128)total * (index + 1) / count);
  return LAI_OK;
}

void lai_engine_opts_default(lai_engine_opts* opts) {
  if (!opts) return;
  opts->schwarz_threshold = 1e-12;
  opts->device = 0;
  opts->prim_threshold = -1.0;
}

void lai_jk_opts_default(lai_jk_opts* opts) {
  if (!opts) return;
  opts->fp32_cut = 0.0;
  opts->check_symmetric = 0;
  opts->shard_index = 0;
  opts->shard_count = 1;
  opts->profile = 0;
  opts->graph = 0;
  opts->fp32_prim_rel = 0.0;
}

}  // extern "C"

namespace lai {
namespace host {

// Engine over `basis`; for a batched engine, `merged` is the concatenation of the
// systems' shells (each tagged with its system) and sys_nbf their function counts.
int create_engine(const lai_basis* basis, std::unique_ptr<lai_basis> merged, const std::vector<int>& sys_nbf,
                  const lai_engine_opts* opts, lai_engine** out) {
  lai_engine_opts o;
  lai_engine_opts_default(&o);
  if (opts) o = *opts;
  if (!(o.schwarz_threshold >= 0.0)) return fail(LAI_EINVAL, "negative Schwarz threshold");
  int ndev = 0;
  LAI_CUDA_TRY(cudaGetDeviceCount(&ndev));
  if (o.device < 0 || o.device >= ndev) return fail(LAI_EINVAL, "lai_engine_create: bad device");
  // The kernel launchers set their launch attributes (dynamic shared-memory
  // limits) and cache occupancies once per process, and CUDA keeps those per
  // device: every engine of a process therefore uses the first engine's device.
  static std::atomic<int> process_device{-1};
  int first = -1;
  if (!process_device.compare_exchange_strong(first, o.device) && first != o.device)
    return fail(LAI_ENOTSUP, "lai_engine_create: this process already runs engines on another CUDA device "
                             "(one device per process: run one process per GPU)");
  LAI_CUDA_TRY(cudaSetDevice(o.device));
  auto E = std::make_unique<lai_engine>();
  if (merged) {
    E->merged = std::move(merged);
    E->basis = E->merged.get();
    E->nsys = (int)sys_nbf.size();
    E->sys_nbf = sys_nbf;
    E->sys_off.assign(E->nsys + 1, 0);
    for (int i = 0; i < E->nsys; ++i) E->sys_off[i + 1] = E->sys_off[i] + (int64_t)sys_nbf[i] * sys_nbf[i];
    LAI_CUDA_TRY(upload(E->d_sys_nbf, E->sys_nbf));
    LAI_CUDA_TRY(upload(E->d_sys_off, E->sys_off));
  } else {
    E->basis = basis;
  }
  basis = E->basis;
  E->device = o.device;
  E->thr = o.schwarz_threshold;
  E->prim_eps = o.prim_threshold < 0.0 ? 1e-3 * o.schwarz_threshold : o.prim_threshold;
  LAI_CUDA_TRY(cudaDeviceGetAttribute(&E->num_sms, cudaDevAttrMultiProcessorCount, o.device));
  LAI_CUDA_TRY(cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking));
  LAI_CUDA_TRY(cudaEventCreate(&E->ev0));
  LAI_CUDA_TRY(cudaEventCreate(&E->ev1));
  {
    std::vector<double> coef(RYS_COEF_H, RYS_COEF_H + RYS_COEF_LEN);
    std::vector<double> hx(RYS_HERM_X2_H, RYS_HERM_X2_H + RYS_HERM_LEN);
    std::vector<double> hw(RYS_HERM_W_H, RYS_HERM_W_H + RYS_HERM_LEN);
    std::vector<double> bg(BOYS_GRID_H, BOYS_GRID_H + BOYS_NGRID * BOYS_NM);
    LAI_CUDA_TRY(upload(E->d_coef, coef));
    LAI_CUDA_TRY(upload(E->d_hx2, hx));
    LAI_CUDA_TRY(upload(E->d_hw, hw));
    LAI_CUDA_TRY(upload(E->d_boys, bg));
    // FP32 tables of the packed FP32 kernels, derived from the FP64 ones
    std::vector<float> bf((size_t)lai::kBoysF32Rows * lai::kBoysF32Stride), rf(2 * (size_t)lai::kRysF32Len);
    lai::build_boys_f32(BOYS_GRID_H, bf.data());
    lai::build_rys_f32(RYS_COEF_H, rf.data());
    LAI_CUDA_TRY(upload(E->d_boys_f32, bf));
    LAI_CUDA_TRY(upload(E->d_rys_f32, rf));
    E->tab = {E->d_coef.as<double>(), E->d_hx2.as<double>(), E->d_hw.as<double>(),
              E->d_boys.as<double>(), E->d_boys_f32.as<float>(), E->d_rys_f32.as<float>()};
  }
  if (int rc = build_classes(E.get())) return rc;
  for (auto& c : E->classes) {
    fill_pair_data(basis, *c);
    if (int rc = upload_class(*c)) return rc;
  }
  if (int rc = compute_schwarz(E.get())) return rc;
  if (int rc = compute_prim_schwarz(E.get())) return rc;
  if (int rc = sort_and_screen(E.get())) return rc;
  *out = E.release();
  return LAI_OK;
}

}  // namespace host
}  // namespace lai

extern "C" {

int lai_engine_create(const lai_basis* basis, const lai_engine_opts* opts, lai_engine** out) {
  if (!out || !basis) return fail(LAI_EINVAL, "lai_engine_create: null argument");
  *out = nullptr;
  return create_engine(basis, nullptr, {}, opts, out);
}

int lai_engine_create_batched(int nsys, const lai_basis* const* bases, const lai_engine_opts* opts,
                              lai_engine** out) {
  if (!out || nsys < 1 || !bases) return fail(LAI_EINVAL, "lai_engine_create_batched: null argument");
  *out = nullptr;
  auto merged = std::make_unique<lai_basis>();
  std::vector<int> nbf(nsys);
  for (int s = 0; s < nsys; ++s) {
    if (!bases[s]) return fail(LAI_EINVAL, "lai_engine_create_batched: null basis");
    for (const HostShell& sh : bases[s]->shells) {
      merged->shells.push_back(sh);
      merged->shells.back().sys = s;  // func stays local to the system
    }
    nbf[s] = (int)bases[s]->nbf;
  }
  merged->nbf = 0;  // no single matrix size: D/J/K are packed per system
  return create_engine(nullptr, std::move(merged), nbf, opts, out);
}

int lai_engine_batch_layout(lai_engine* engine, int* nsys, int64_t* offsets, int* nbf) {
  if (!engine) return fail(LAI_EINVAL, "lai_engine_batch_layout: null engine");
  if (nsys) *nsys = engine->nsys;
  if (engine->nsys == 1) {
    if (offsets) { offsets[0] = 0; offsets[1] = (int64_t)engine->basis->nbf * engine->basis->nbf; }
    if (nbf) nbf[0] = (int)engine->basis->nbf;
    return LAI_OK;
  }
  if (offsets) std::copy(engine->sys_off.begin(), engine->sys_off.end(), offsets);
  if (nbf) std::copy(engine->sys_nbf.begin(), engine->sys_nbf.end(), nbf);
  return LAI_OK;
}

void lai_engine_destroy(lai_engine* engine) {
  if (engine) {
    cudaSetDevice(engine->device);
    delete engine;
  }
}

int lai_engine_schwarz(lai_engine* engine, double* Q) {
  if (engine && engine->nsys > 1) return fail(LAI_ENOTSUP, "lai_engine_schwarz: not available for a batched engine");
  if (!engine || !Q) return fail(LAI_EINVAL, "lai_engine_schwarz: null argument");
  std::copy(engine->Q_all.begin(), engine->Q_all.end(), Q);
  return LAI_OK;
}

int lai_jk_build_device(lai_engine* engine, const double* d_D, double* d_J, double* d_K,
                        void* stream, const lai_jk_opts* opts, lai_jk_report* report) {
  if (!engine || !d_D || !d_J || !d_K) return fail(LAI_EINVAL, "lai_jk_build_device: null argument");
  lai_jk_opts o;
  lai_jk_opts_default(&o);
  if (opts) o = *opts;
  if (!(o.fp32_cut >= 0.0)) return fail(LAI_EINVAL, "lai_jk_build_device: fp32_cut must be >= 0");
  if (!(o.fp32_prim_rel >= 0.0 && o.fp32_prim_rel < 1.0))
    return fail(LAI_EINVAL, "lai_jk_build_device: fp32_prim_rel must be in [0, 1)");
  LAI_CUDA_TRY(cudaSetDevice(engine->device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!o.graph) return run_jk(engine, d_D, d_J, d_K, s, o, report, false);
  if (!s || o.profile) return fail(LAI_EINVAL, "lai_jk_build_device: graph mode needs a stream and profile = 0");
  lai_engine::GraphKey key{d_D, d_J, d_K, s, o.fp32_cut, o.shard_index, o.shard_count, o.fp32_prim_rel};
  if (engine->graph_exec && engine->graph_key == key) {
    LAI_CUDA_TRY(cudaGraphLaunch(engine->graph_exec, s));
    if (report) *report = engine->graph_report;
    return LAI_OK;
  }
  // First call: an ordinary build (allocations, the FP32 split and its cut), whose
  // result is this call's; then the same launch sequence captured for the replays.
  lai_jk_report rep{};
  if (int rc = run_jk(engine, d_D, d_J, d_K, s, o, &rep, false)) return rc;
  engine->release_graph();
  cudaGraph_t graph = nullptr;
  LAI_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  lai_jk_report rep2{};
  const int rc = run_jk(engine, d_D, d_J, d_K, s, o, &rep2, false, rep.fp32_schwarz_cut);
  const cudaError_t ce = cudaStreamEndCapture(s, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  LAI_CUDA_TRY(ce);
  const cudaError_t ie = cudaGraphInstantiate(&engine->graph_exec, graph, 0);
  cudaGraphDestroy(graph);
  LAI_CUDA_TRY(ie);
  engine->graph_key = key;
  engine->graph_report = rep;
  if (report) *report = rep;
  return LAI_OK;
}

int lai_jk_build(lai_engine* engine, const double* D, size_t nbf, double* J, double* K,
                 const lai_jk_opts* opts, lai_jk_report* report) {
  auto t0 = std::chrono::steady_clock::now();
  if (!engine || !D || !J || !K) return fail(LAI_EINVAL, "lai_jk_build: null argument");
  if (engine->nsys > 1) return fail(LAI_EINVAL, "lai_jk_build: batched engine (use lai_jk_build_batched)");
  if ((long)nbf != engine->basis->nbf)
    return fail(LAI_EINVAL, "lai_jk_build: nbf mismatch (expected " +
                                std::to_string(engine->basis->nbf) + ", got " +
                                std::to_string(nbf) + ")");
  lai_jk_opts o;
  lai_jk_opts_default(&o);
  if (opts) o = *opts;
  if (!(o.fp32_cut >= 0.0)) return fail(LAI_EINVAL, "lai_jk_build: fp32_cut must be >= 0");
  if (!(o.fp32_prim_rel >= 0.0 && o.fp32_prim_rel < 1.0))
    return fail(LAI_EINVAL, "lai_jk_build: fp32_prim_rel must be in [0, 1)");
  if (o.check_symmetric) {
    for (size_t i = 0; i < nbf; ++i)
      for (size_t j = 0; j < i; ++j)
        if (std::fabs(D[i * nbf + j] - D[j * nbf + i]) > 1e-12 * (1.0 + std::fabs(D[i * nbf + j])))
          return fail(LAI_EINVAL, "lai_jk_build: density matrix is not symmetric");
  }
  LAI_CUDA_TRY(cudaSetDevice(engine->device));
  const size_t bytes = sizeof(double) * nbf * nbf;
  if (engine->d_D.bytes < bytes) {
    LAI_CUDA_TRY(engine->d_D.alloc(bytes));
    LAI_CUDA_TRY(engine->d_J.alloc(bytes));
    LAI_CUDA_TRY(engine->d_K.alloc(bytes));
  }
  cudaStream_t s = engine->stream;
  LAI_CUDA_TRY(cudaMemcpyAsync(engine->d_D.p, D, bytes, cudaMemcpyHostToDevice, s));
  if (int rc = run_jk(engine, engine->d_D.as<double>(), engine->d_J.as<double>(),
                      engine->d_K.as<double>(), s, o, report, true))
    return rc;
  LAI_CUDA_TRY(cudaMemcpyAsync(J, engine->d_J.p, bytes, cudaMemcpyDeviceToHost, s));
  LAI_CUDA_TRY(cudaMemcpyAsync(K, engine->d_K.p, bytes, cudaMemcpyDeviceToHost, s));
  LAI_CUDA_TRY(cudaStreamSynchronize(s));
  if (report) {
    float ms = 0;
    cudaEventElapsedTime(&ms, engine->ev0, engine->ev1);
    report->seconds_device = ms * 1e-3;
    report->seconds_total =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  return LAI_OK;
}

int lai_jk_build_batched(lai_engine* engine, const double* D, double* J, double* K, const lai_jk_opts* opts,
                         lai_jk_report* report) {
  auto t0 = std::chrono::steady_clock::now();
  if (!engine || !D || !J || !K) return fail(LAI_EINVAL, "lai_jk_build_batched: null argument");
  lai_jk_opts o;
  lai_jk_opts_default(&o);
  if (opts) o = *opts;
  if (!(o.fp32_cut >= 0.0)) return fail(LAI_EINVAL, "lai_jk_build_batched: fp32_cut must be >= 0");
  if (!(o.fp32_prim_rel >= 0.0 && o.fp32_prim_rel < 1.0))
    return fail(LAI_EINVAL, "lai_jk_build_batched: fp32_prim_rel must be in [0, 1)");
  LAI_CUDA_TRY(cudaSetDevice(engine->device));
  const size_t bytes = sizeof(double) * engine_mat_elems(engine);
  if (engine->d_D.bytes < bytes) {
    LAI_CUDA_TRY(engine->d_D.alloc(bytes));
    LAI_CUDA_TRY(engine->d_J.alloc(bytes));
    LAI_CUDA_TRY(engine->d_K.alloc(bytes));
  }
  cudaStream_t s = engine->stream;
  LAI_CUDA_TRY(cudaMemcpyAsync(engine->d_D.p, D, bytes, cudaMemcpyHostToDevice, s));
  if (int rc = run_jk(engine, engine->d_D.as<double>(), engine->d_J.as<double>(), engine->d_K.as<double>(), s, o,
                      report, true))
    return rc;
  LAI_CUDA_TRY(cudaMemcpyAsync(J, engine->d_J.p, bytes, cudaMemcpyDeviceToHost, s));
  LAI_CUDA_TRY(cudaMemcpyAsync(K, engine->d_K.p, bytes, cudaMemcpyDeviceToHost, s));
  LAI_CUDA_TRY(cudaStreamSynchronize(s));
  if (report) {
    float ms = 0;
    cudaEventElapsedTime(&ms, engine->ev0, engine->ev1);
    report->seconds_device = ms * 1e-3;
    report->seconds_total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  return LAI_OK;
}

int lai_eri_batch_screened(lai_engine* engine, double* out, size_t out_capacity,
                           lai_quartet_meta* meta, size_t meta_capacity, int64_t* n_quartets,
                           int64_t* n_values) {
  if (engine && engine->nsys > 1) return fail(LAI_ENOTSUP, "lai_eri_batch_screened: not available for a batched engine");
  if (!engine) return fail(LAI_EINVAL, "lai_eri_batch_screened: null engine");
  int64_t nq = 0, nv = 0;
  std::vector<int64_t> vals_per(engine->blocks.size());
  for (size_t b = 0; b < engine->blocks.size(); ++b) {
    const auto& bp = *engine->blocks[b];
    const auto& ca = *engine->classes[bp.bra];
    const auto& cb = *engine->classes[bp.ket];
    vals_per[b] = (int64_t)lai::ncart(ca.la) * lai::ncart(ca.lb) * lai::ncart(cb.la) * lai::ncart(cb.lb);
    nq += bp.total;
    nv += bp.total * vals_per[b];
  }
  if (n_quartets) *n_quartets = nq;
  if (n_values) *n_values = nv;
  if (!out || !meta) return LAI_OK;
  if ((int64_t)out_capacity < nv || (int64_t)meta_capacity < nq)
    return fail(LAI_EINVAL, "lai_eri_batch_screened: output capacity too small");
  LAI_CUDA_TRY(cudaSetDevice(engine->device));
  DevBuf d_out, d_meta;
  LAI_CUDA_TRY(d_out.alloc(sizeof(double) * (size_t)std::max<int64_t>(nv, 1)));
  LAI_CUDA_TRY(d_meta.alloc(sizeof(int) * 4 * (size_t)std::max<int64_t>(nq, 1)));
  int64_t qo = 0, vo = 0;
  for (size_t b = 0; b < engine->blocks.size(); ++b) {
    const auto& bp = *engine->blocks[b];
    lai::JKArgs args{};
    args.mode = lai::MODE_RAW;
    args.raw_out = d_out.as<double>() + vo;
    args.raw_meta = d_meta.as<int>() + 4 * qo;
    if (int rc = launch_block(engine, make_block(engine, bp), args)) return rc;
    qo += bp.total;
    vo += bp.total * vals_per[b];
  }
  std::vector<int> hmeta(4 * (size_t)nq);
  LAI_CUDA_TRY(cudaMemcpyAsync(out, d_out.p, sizeof(double) * nv, cudaMemcpyDeviceToHost, engine->stream));
  LAI_CUDA_TRY(cudaMemcpyAsync(hmeta.data(), d_meta.p, sizeof(int) * 4 * nq, cudaMemcpyDeviceToHost,
                               engine->stream));
  LAI_CUDA_TRY(cudaStreamSynchronize(engine->stream));
  qo = 0;
  vo = 0;
  for (size_t b = 0; b < engine->blocks.size(); ++b) {
    const auto& bp = *engine->blocks[b];
    const auto& ca = *engine->classes[bp.bra];
    const auto& cb = *engine->classes[bp.ket];
    for (int64_t t = 0; t < bp.total; ++t) {
      lai_quartet_meta& m = meta[qo + t];
      m.offset = vo + t * vals_per[b];
      m.fa = hmeta[4 * (qo + t)]; m.fb = hmeta[4 * (qo + t) + 1];
      m.fc = hmeta[4 * (qo + t) + 2]; m.fd = hmeta[4 * (qo + t) + 3];
      m.na = lai::ncart(ca.la); m.nb = lai::ncart(ca.lb);
      m.nc = lai::ncart(cb.la); m.nd = lai::ncart(cb.lb);
    }
    qo += bp.total;
    vo += bp.total * vals_per[b];
  }
  return LAI_OK;
}

int lai_jk_last_profile(lai_engine* engine, int capacity, double* ms, double* alg_flops,
                        double* alg_flops_executed, int64_t* quartets, int64_t* prim_quartets,
                        int* lclass) {
  if (!engine) return fail(LAI_EINVAL, "lai_jk_last_profile: null engine");
  const int n = engine->prof_n;
  if (capacity < n || !ms) return n;
  std::vector<unsigned long long> prims(n, 0);
  if (n > 0) {
    LAI_CUDA_TRY(cudaEventSynchronize(engine->prof_ev[2 * n - 1]));
    LAI_CUDA_TRY(cudaMemcpy(prims.data(), engine->d_prof_prims.p, sizeof(unsigned long long) * n,
                            cudaMemcpyDeviceToHost));
  }
  for (int i = 0; i < n; ++i) {
    float t = 0;
    LAI_CUDA_TRY(cudaEventElapsedTime(&t, engine->prof_ev[2 * i], engine->prof_ev[2 * i + 1]));
    ms[i] = t;
    const auto& b = *engine->blocks[engine->prof_block[i]];
    const auto& ca = *engine->classes[b.bra];
    const auto& cb = *engine->classes[b.ket];
    const double nq = (double)engine->prof_quartets[i];
    if (alg_flops) alg_flops[i] = b.alg_flops * nq;
    if (alg_flops_executed)
      alg_flops_executed[i] = b.flops_per_prim * (double)prims[i] + b.flops_per_quartet * nq;
    if (quartets) quartets[i] = engine->prof_quartets[i];
    if (prim_quartets) prim_quartets[i] = (int64_t)prims[i];
    if (lclass) {
      lclass[4 * i] = ca.la; lclass[4 * i + 1] = ca.lb;
      lclass[4 * i + 2] = cb.la; lclass[4 * i + 3] = cb.lb;
    }
  }
  return n;
}

int64_t lai_engine_quartet_count(lai_engine* engine) {
  if (!engine) return -1;
  int64_t n = 0;
  for (auto& b : engine->blocks) n += b->total;
  return n;
}

int lai_engine_sample_quartets(lai_engine* engine, int64_t n, uint64_t seed, int32_t* quartets) {
  if (engine && engine->nsys > 1) return fail(LAI_ENOTSUP, "lai_engine_sample_quartets: not available for a batched engine");
  if (!engine || n < 0 || (n > 0 && !quartets)) return fail(LAI_EINVAL, "lai_engine_sample_quartets");
  std::vector<int64_t> pref(engine->blocks.size() + 1, 0);
  for (size_t b = 0; b < engine->blocks.size(); ++b) pref[b + 1] = pref[b] + engine->blocks[b]->total;
  const int64_t total = pref.back();
  if (total == 0) return n == 0 ? LAI_OK : fail(LAI_ESTATE, "engine has no quartets");
  uint64_t st = seed;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t t = (int64_t)(mix64(st) % (uint64_t)total);
    const size_t b = std::upper_bound(pref.begin(), pref.end(), t) - pref.begin() - 1;
    const auto& bp = *engine->blocks[b];
    const int64_t tl = t - pref[b];
    const int p = (int)(std::upper_bound(bp.offsets.begin(), bp.offsets.end(), tl) - bp.offsets.begin() - 1);
    const int q = (int)(tl - bp.offsets[p]);
    const auto& ca = *engine->classes[bp.bra];
    const auto& cb = *engine->classes[bp.ket];
    quartets[4 * i] = ca.sa[p];
    quartets[4 * i + 1] = ca.sb[p];
    quartets[4 * i + 2] = cb.sa[q];
    quartets[4 * i + 3] = cb.sb[q];
  }
  return LAI_OK;
}

int lai_engine_autotune(lai_engine* engine, const double* d_D, void* stream, double* ms_before,
                        double* ms_after) {
  if (!engine || !d_D) return fail(LAI_EINVAL, "lai_engine_autotune: null argument");
  LAI_CUDA_TRY(cudaSetDevice(engine->device));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // one ordinary build first: allocations and accumulators
  lai_jk_opts o;
  lai_jk_opts_default(&o);
  const size_t elems = engine_mat_elems(engine);
  DevBuf dJ, dK;
  LAI_CUDA_TRY(dJ.alloc(sizeof(double) * elems));
  LAI_CUDA_TRY(dK.alloc(sizeof(double) * elems));
  if (int rc = run_jk(engine, d_D, dJ.as<double>(), dK.as<double>(), s, o, nullptr, false)) return rc;
  engine->release_graph();
  cudaEvent_t e0, e1;
  LAI_CUDA_TRY(cudaEventCreate(&e0));
  LAI_CUDA_TRY(cudaEventCreate(&e1));
  lai::JKArgs args{};
  args.D = d_D;
  args.J = engine->d_Jp.as<double>();
  args.K = engine->d_Kp.as<double>();
  args.nbf = (int)engine->basis->nbf;
  args.mode = lai::MODE_JK;
  args.prim_eps = engine->prim_eps;
  if (engine->nsys > 1) {
    args.sys_off = engine->d_sys_off.as<int64_t>();
    args.sys_nbf = engine->d_sys_nbf.as<int>();
  }
  cudaStream_t saved = engine->stream;
  engine->stream = s;
  double before = 0.0, after = 0.0;
  int rc = LAI_OK;
  auto time_launch = [&](const lai::QuartetBlock& q, lai::LaunchTune t, float* ms) -> int {
    float best = 1e30f;
    for (int rep = 0; rep < 2; ++rep) {  // the first run warms caches, the minimum counts
      if (cudaEventRecord(e0, s) != cudaSuccess) return LAI_ECUDA;
      if (int r = launch_block(engine, q, args, false, nullptr, t)) return r;
      if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) return LAI_ECUDA;
      float m = 0;
      cudaEventElapsedTime(&m, e0, e1);
      best = std::min(best, m);
    }
    *ms = best;
    return LAI_OK;
  };
  for (auto& bp : engine->blocks) {
    const lai::QuartetBlock q = make_block(engine, *bp);
    bp->tune = lai::LaunchTune{};
    float base = 0;
    if ((rc = time_launch(q, bp->tune, &base))) break;
    before += base;
    if (!lai::small_class_supported(q.bra.la, q.bra.lb, q.ket.la, q.ket.lb)) {
      // kernel family: warp-per-quartet, bra-sliced, tiled
      lai::LaunchTune best = bp->tune;
      float best_ms = base;
      for (int k : {lai::KERNEL_WARPQ, lai::KERNEL_SLICED, lai::KERNEL_TILED}) {
        if (k == lai::KERNEL_WARPQ && !lai::warpq_class_supported(q.bra.la, q.bra.lb, q.ket.la, q.ket.lb))
          continue;
        if (k == lai::KERNEL_SLICED && !lai::sliced_class_supported(q.bra.la, q.bra.lb, q.ket.la, q.ket.lb))
          continue;
        lai::LaunchTune t;
        t.kernel = k;
        float m = 0;
        if ((rc = time_launch(q, t, &m))) break;
        if (m < 0.98f * best_ms) { best_ms = m; best = t; }
      }
      if (rc) break;
      bp->tune = best;
      after += best_ms;
      continue;
    }
    const int Kab = q.bra.Ka * q.bra.Kb;
    lai::LaunchTune best = bp->tune;
    float best_ms = base;
    for (int ps = 1; ps <= 8 && ps < 2 * Kab; ps <<= 1)
      for (int ks : {1, 4, 16}) {
        float m = 0;
        if ((rc = time_launch(q, lai::LaunchTune{ps, ks}, &m))) break;
        if (m < 0.98f * best_ms) { best_ms = m; best = lai::LaunchTune{ps, ks}; }
      }
    if (rc) break;
    bp->tune = best;
    after += best_ms;
  }
  engine->stream = saved;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return fail(rc, "lai_engine_autotune: a timing launch failed");
  if (ms_before) *ms_before = before;
  if (ms_after) *ms_after = after;
  return LAI_OK;
}

int lai_engine_tune_table(lai_engine* engine, int capacity, int* rows) {
  if (!engine) return fail(LAI_EINVAL, "lai_engine_tune_table: null engine");
  const int n = (int)engine->blocks.size();
  if (!rows || capacity < n) return n;
  for (int b = 0; b < n; ++b) {
    const auto& bp = *engine->blocks[b];
    const auto& ca = *engine->classes[bp.bra];
    const auto& cb = *engine->classes[bp.ket];
    int* r = rows + 10 * b;
    r[0] = ca.la; r[1] = ca.lb; r[2] = cb.la; r[3] = cb.lb;
    r[4] = ca.Ka * ca.Kb; r[5] = cb.Ka * cb.Kb;
    r[6] = (int)std::min<int64_t>(bp.total, INT32_MAX);
    r[7] = bp.tune.kernel ? -bp.tune.kernel : bp.tune.ps; r[8] = bp.tune.ksuper;
    r[9] = (int)std::min<int64_t>(bp.total / 1000, INT32_MAX);
  }
  return n;
}

int lai_probe_fp64_peak(int device, double* tflops) {
  if (!tflops) return fail(LAI_EINVAL, "lai_probe_fp64_peak: null output");
  LAI_CUDA_TRY(cudaSetDevice(device));
  int sms = 0;
  LAI_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  DevBuf out;
  LAI_CUDA_TRY(out.alloc(8));
  cudaEvent_t a, b;
  LAI_CUDA_TRY(cudaEventCreate(&a));
  LAI_CUDA_TRY(cudaEventCreate(&b));
  const int threads = 256, blocks = sms * 8, iters = 4096;
  fp64_fma_probe<<<blocks, threads>>>(out.as<double>(), 64);  // warm-up
  double best = 0;
  for (int rep = 0; rep < 3; ++rep) {
    LAI_CUDA_TRY(cudaEventRecord(a));
    fp64_fma_probe<<<blocks, threads>>>(out.as<double>(), iters);
    LAI_CUDA_TRY(cudaEventRecord(b));
    LAI_CUDA_TRY(cudaEventSynchronize(b));
    float ms = 0;
    LAI_CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
    const double fl = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    best = std::max(best, fl / (ms * 1e-3) / 1e12);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *tflops = best;
  return LAI_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Read-only accessors for other translation units of the library (not C ABI).
// ---------------------------------------------------------------------------
namespace lai {

int engine_device(const lai_engine* E) { return E->device; }
int engine_num_sms(const lai_engine* E) { return E->num_sms; }
int engine_nbf(const lai_engine* E) { return (int)E->basis->nbf; }
double engine_prim_eps(const lai_engine* E) { return E->prim_eps; }
RysTablesView engine_tables(const lai_engine* E) { return E->tab; }
const lai_basis* engine_basis(const lai_engine* E) { return E->basis; }
int engine_nsys(const lai_engine* E) { return E->nsys; }
int engine_block_count(const lai_engine* E) { return (int)E->blocks.size(); }
QuartetBlock engine_block(const lai_engine* E, int i) { return make_block(E, *E->blocks[i]); }
void engine_set_error(const char* msg) { g_last_error = msg; }

}  // namespace lai
