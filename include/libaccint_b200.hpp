/* C++ adaptors with the reference's consumer shapes over the C ABI of
 * libaccint_b200.h (header-only; link libaccint_b200.so).
 *
 *   lai::BasisSet     ~ libaccint::BasisSet (src/shared/basis/basis_set.cpp:21-29)
 *   lai::Engine       ~ libaccint::Engine: compute(Operator::coulomb(), consumer)
 *                       (include/libaccint/engine/engine.hpp:435-499, 727-731)
 *   lai::FockBuilder  ~ consumers::FockBuilder: set_density / get_coulomb_matrix /
 *                       get_exchange_matrix / get_fock_matrix / reset
 *                       (include/libaccint/consumers/fock_builder.hpp:41-170)
 *   lai::GpuFockBuilder ~ consumers::GpuFockBuilder: device J/K, D uploaded by
 *                       set_density, results copied back by get_*
 *                       (include/libaccint/consumers/fock_builder_gpu.hpp:46-159)
 *   lai::Operator / PointChargeParams and Engine::compute_1e, compute_overlap_matrix,
 *                       compute_kinetic_matrix, compute_nuclear_matrix
 *                       (include/libaccint/engine/engine.hpp:166-201, 831-900;
 *                       include/libaccint/operators/operator_types.hpp:50-60)
 *   lai::BasisSet::from_bse_json ~ data::BseJsonParser::parse
 *                       (src/shared/data/bse_json_parser.cpp:27-140)
 *   lai::ShellSet / ShellSetPair / ShellSetQuartet, BasisSet::shell_set_quartets,
 *   Engine::compute_shell_set_quartet, compute_batch, compute_batch_screened,
 *   IntegralBuffer / ShellQuartetMeta, ScreeningOptions,
 *   GpuFockBuilder::accumulate_device_eri_batch ~ the reference's work-unit and
 *                       raw-integral API (include/libaccint/basis/shell_set_quartet.hpp,
 *                       include/libaccint/engine/{engine.hpp:1008-1187,
 *                       cuda_engine.hpp:462-466, integral_buffer.hpp},
 *                       include/libaccint/consumers/fock_builder_gpu.hpp)
 *
 * Errors become exceptions here (std::invalid_argument for LAI_EINVAL,
 * std::runtime_error otherwise), as in the reference; the C ABI itself never
 * throws.  The per-quartet accumulate() of the reference's consumers has no
 * counterpart: the integrals are digested inside the device kernels.
 */
#ifndef LIBACCINT_B200_HPP
#define LIBACCINT_B200_HPP

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "libaccint_b200.h"

#define LAI_STR_(x) #x
#define LAI_STR(x) LAI_STR_(x)

namespace lai {

inline void check(int rc, const char* what) {
  if (rc == LAI_OK) return;
  const std::string msg = std::string(what) + ": " + lai_last_error();
  if (rc == LAI_EINVAL) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

// The reference's scalar and size types (include/libaccint/core/types.hpp).
using Real = double;
using Size = std::size_t;

struct Point3D {
  double x = 0.0, y = 0.0, z = 0.0;
};

// Library identity: this build has one backend, the B200 one.
inline const char* version() { return "libaccint-b200 (C ABI " LAI_STR(LAI_ABI_VERSION) ")"; }
inline bool has_cuda_backend() { return true; }

struct Shell {
  int l = 0;
  double center[3] = {0.0, 0.0, 0.0};
  std::vector<double> exps, coefs;  // raw contraction coefficients
  int atom = -1;
  Shell() = default;
  // Shell(am, center, exps, coefs) (src/shared/basis/shell.cpp:163-187); the
  // library normalizes the raw coefficients when the BasisSet is built.
  Shell(int am, Point3D c, std::vector<double> e, std::vector<double> k)
      : l(am), center{c.x, c.y, c.z}, exps(std::move(e)), coefs(std::move(k)) {}
};

// Shells of one angular momentum and primitive count, by their index in the
// BasisSet (the reference's ShellSet, include/libaccint/basis/shell_set.hpp:117-183,
// holds the shells themselves).
class ShellSet {
 public:
  ShellSet(int am, int n_primitives) : am_(am), nprim_(n_primitives) {}
  void add_shell(int shell_index) { shells_.push_back(shell_index); }
  int angular_momentum() const { return am_; }
  int n_primitives() const { return nprim_; }
  int n_functions_per_shell() const { return (am_ + 1) * (am_ + 2) / 2; }
  std::size_t n_shells() const { return shells_.size(); }
  int shell_index(std::size_t i) const { return shells_[i]; }
  const std::vector<int>& shell_indices() const { return shells_; }

 private:
  int am_, nprim_;
  std::vector<int> shells_;
};

// (set_a, set_b): every shell pair of the product (include/libaccint/basis/shell_set_pair.hpp:24-70).
class ShellSetPair {
 public:
  ShellSetPair(const ShellSet& set_a, const ShellSet& set_b) : a_(&set_a), b_(&set_b) {}
  const ShellSet& shell_set_a() const { return *a_; }
  const ShellSet& shell_set_b() const { return *b_; }
  int La() const { return a_->angular_momentum(); }
  int Lb() const { return b_->angular_momentum(); }
  std::size_t n_pairs() const { return a_->n_shells() * b_->n_shells(); }

 private:
  const ShellSet* a_;
  const ShellSet* b_;
};

// (bra | ket) over two set pairs: the work unit of compute_shell_set_quartet and
// compute_batch (include/libaccint/basis/shell_set_quartet.hpp:20-80).
class ShellSetQuartet {
 public:
  ShellSetQuartet(const ShellSetPair& bra, const ShellSetPair& ket) : bra_(&bra), ket_(&ket) {}
  const ShellSetPair& bra_pair() const { return *bra_; }
  const ShellSetPair& ket_pair() const { return *ket_; }
  int La() const { return bra_->La(); }
  int Lb() const { return bra_->Lb(); }
  int Lc() const { return ket_->La(); }
  int Ld() const { return ket_->Lb(); }
  int L_total() const { return La() + Lb() + Lc() + Ld(); }
  std::size_t n_quartets() const { return bra_->n_pairs() * ket_->n_pairs(); }

  // Shell-index quartets (i, j, k, l), 4 per quartet, of the full product
  // (canonical = false), or only of one representative of every permutation
  // orbit inside it (canonical = true): where both bra sets are the same set the
  // bra pairs with a >= b, likewise on the ket, and where bra and ket are the
  // same set pair the quartets with bra rank >= ket rank.  Over all of
  // BasisSet::shell_set_quartets() the canonical lists hold every orbit of the
  // basis exactly once (sets are compared by identity, like the ij_same /
  // kl_same / braket_same flags of cuda_engine.hpp:808-816).
  std::vector<int32_t> shell_quartets(bool canonical) const {
    const ShellSet &A = bra_->shell_set_a(), &B = bra_->shell_set_b();
    const ShellSet &C = ket_->shell_set_a(), &D = ket_->shell_set_b();
    const bool ij_same = &A == &B, kl_same = &C == &D;
    const bool braket_same = &A == &C && &B == &D;
    std::vector<int32_t> q;
    q.reserve(4 * n_quartets());
    for (std::size_t a = 0; a < A.n_shells(); ++a)
      for (std::size_t b = 0; b < B.n_shells(); ++b) {
        if (canonical && ij_same && b > a) continue;
        for (std::size_t c = 0; c < C.n_shells(); ++c)
          for (std::size_t d = 0; d < D.n_shells(); ++d) {
            if (canonical && kl_same && d > c) continue;
            if (canonical && braket_same && c * D.n_shells() + d > a * B.n_shells() + b) continue;
            q.insert(q.end(), {A.shell_index(a), B.shell_index(b), C.shell_index(c), D.shell_index(d)});
          }
      }
    return q;
  }

 private:
  const ShellSetPair* bra_;
  const ShellSetPair* ket_;
};

class BasisSet {
 public:
  explicit BasisSet(const std::vector<Shell>& shells) {
    std::vector<int> l, np, atom;
    std::vector<double> c, e, k;
    for (const Shell& s : shells) {
      l.push_back(s.l);
      np.push_back((int)s.exps.size());
      atom.push_back(s.atom);
      c.insert(c.end(), s.center, s.center + 3);
      e.insert(e.end(), s.exps.begin(), s.exps.end());
      k.insert(k.end(), s.coefs.begin(), s.coefs.end());
    }
    check(lai_basis_create((int)shells.size(), l.data(), np.data(), c.data(), e.data(), k.data(),
                           atom.data(), 0, &h_),
          "BasisSet");
  }
  // Basis Set Exchange JSON text on atoms (atomic numbers Z, positions xyz[3*i], Bohr).
  static BasisSet from_bse_json(const std::string& json, const std::vector<int>& Z,
                                const std::vector<double>& xyz) {
    if (xyz.size() != 3 * Z.size()) throw std::invalid_argument("BasisSet::from_bse_json: xyz size");
    lai_basis* h = nullptr;
    check(lai_basis_from_bse_json(json.data(), json.size(), (int)Z.size(), Z.data(), xyz.data(), &h),
          "BasisSet::from_bse_json");
    return BasisSet(h);
  }
  BasisSet(BasisSet&& o) noexcept
      : h_(o.h_), sets_(std::move(o.sets_)), pairs_(std::move(o.pairs_)), quartets_(std::move(o.quartets_)) {
    o.h_ = nullptr;
  }
  ~BasisSet() { lai_basis_destroy(h_); }
  BasisSet(const BasisSet&) = delete;
  BasisSet& operator=(const BasisSet&) = delete;
  std::size_t n_basis_functions() const { return (std::size_t)lai_basis_nbf(h_); }
  std::size_t n_shells() const { return (std::size_t)lai_basis_nshell(h_); }
  const lai_basis* handle() const { return h_; }

  // Shells grouped by (angular momentum, primitive count) in order of first
  // appearance; the set pairs (i <= j) and set quartets (pair i <= pair j) over
  // them, as BasisSet::shell_sets / shell_set_pairs / shell_set_quartets
  // (src/shared/basis/basis_set.cpp:48-140, 191-210).  Built on first use; the
  // references stay valid for the lifetime of the basis.
  std::vector<const ShellSet*> shell_sets() const;
  const std::vector<ShellSetPair>& shell_set_pairs() const;
  const std::vector<ShellSetQuartet>& shell_set_quartets() const;

 private:
  explicit BasisSet(lai_basis* h) : h_(h) {}
  lai_basis* h_ = nullptr;
  mutable std::vector<std::unique_ptr<ShellSet>> sets_;
  mutable std::vector<ShellSetPair> pairs_;
  mutable std::vector<ShellSetQuartet> quartets_;
};

inline std::vector<const ShellSet*> BasisSet::shell_sets() const {
  if (sets_.empty()) {
    const int ns = lai_basis_nshell(h_);
    for (int s = 0; s < ns; ++s) {
      int l = 0, np = 0;
      check(lai_basis_shell(h_, s, &l, &np, nullptr, nullptr, nullptr, nullptr), "BasisSet::shell_sets");
      auto it = std::find_if(sets_.begin(), sets_.end(), [&](const std::unique_ptr<ShellSet>& x) {
        return x->angular_momentum() == l && x->n_primitives() == np;
      });
      if (it == sets_.end()) {
        sets_.push_back(std::make_unique<ShellSet>(l, np));
        it = sets_.end() - 1;
      }
      (*it)->add_shell(s);
    }
  }
  std::vector<const ShellSet*> r;
  for (const auto& p : sets_) r.push_back(p.get());
  return r;
}

inline const std::vector<ShellSetPair>& BasisSet::shell_set_pairs() const {
  if (pairs_.empty()) {
    const std::vector<const ShellSet*> s = shell_sets();
    pairs_.reserve(s.size() * (s.size() + 1) / 2);
    for (std::size_t i = 0; i < s.size(); ++i)
      for (std::size_t j = i; j < s.size(); ++j) pairs_.emplace_back(*s[i], *s[j]);
  }
  return pairs_;
}

inline const std::vector<ShellSetQuartet>& BasisSet::shell_set_quartets() const {
  if (quartets_.empty()) {
    const std::vector<ShellSetPair>& p = shell_set_pairs();  // never grows after this
    quartets_.reserve(p.size() * (p.size() + 1) / 2);
    for (std::size_t i = 0; i < p.size(); ++i)
      for (std::size_t j = i; j < p.size(); ++j) quartets_.emplace_back(p[i], p[j]);
  }
  return quartets_;
}

// Where one shell quartet's block sits in an IntegralBuffer, [a][b][c][d]
// row-major over the functions fi.., fj.., fk.., fl.. (integral_buffer.hpp:27-35).
struct ShellQuartetMeta {
  std::size_t offset = 0;
  long fi = 0, fj = 0, fk = 0, fl = 0;
  int na = 0, nb = 0, nc = 0, nd = 0;
};

// Owning buffer of norm-corrected Cartesian integrals plus per-quartet metadata
// (the reference's IntegralBuffer, include/libaccint/engine/integral_buffer.hpp:65-165;
// C++17, so blocks come back as pointer + size instead of std::span).
class IntegralBuffer {
 public:
  std::size_t n_quartets() const { return meta_.size(); }
  const ShellQuartetMeta& quartet_meta(std::size_t i) const { return meta_[i]; }
  const double* quartet_data(std::size_t i) const { return data_.data() + meta_[i].offset; }
  std::size_t quartet_size(std::size_t i) const {
    const ShellQuartetMeta& m = meta_[i];
    return (std::size_t)m.na * m.nb * m.nc * m.nd;
  }
  const std::vector<double>& data() const { return data_; }
  const std::vector<ShellQuartetMeta>& metas() const { return meta_; }
  std::size_t n_integrals() const { return data_.size(); }
  bool empty() const { return data_.empty(); }

 private:
  friend class Engine;
  std::vector<double> data_;
  std::vector<ShellQuartetMeta> meta_;
};

// Screening of compute_batch_screened (include/libaccint/screening/screening_options.hpp:20-110):
// a quartet is kept iff Q_ij Q_kl >= threshold (every quartet when !enabled).
// density_weighted screening is not offered by this build (compute_batch_screened
// throws std::invalid_argument); use_permutation_symmetry is accepted and has no
// effect: the screened batch always holds one quartet per permutation orbit.
struct ScreeningOptions {
  double threshold = 1e-12;
  bool enabled = true;
  bool density_weighted = false;
  bool use_permutation_symmetry = false;
  static ScreeningOptions none() { return with(0.0, false); }
  static ScreeningOptions loose() { return with(1e-10, true); }
  static ScreeningOptions normal() { return with(1e-12, true); }
  static ScreeningOptions tight() { return with(1e-14, true); }

 private:
  static ScreeningOptions with(double t, bool on) {
    ScreeningOptions o;
    o.threshold = t;
    o.enabled = on;
    return o;
  }
};

// Structure-of-arrays point charges (nuclei: charge = atomic number).
struct PointChargeParams {
  std::vector<double> x, y, z, charge;
  std::size_t n_centers() const { return charge.size(); }
};

struct Operator {
  enum class Kind { Coulomb, Overlap, Kinetic, Nuclear };
  Kind kind = Kind::Coulomb;
  PointChargeParams charges;
  static Operator coulomb() { return Operator{}; }
  static Operator overlap() { return Operator{Kind::Overlap, {}}; }
  static Operator kinetic() { return Operator{Kind::Kinetic, {}}; }
  static Operator nuclear(const PointChargeParams& c) { return Operator{Kind::Nuclear, c}; }
};

class Engine;

class FockBuilder {
 public:
  explicit FockBuilder(std::size_t nbf) : n_(nbf), J_(nbf * nbf, 0.0), K_(nbf * nbf, 0.0) {}
  void set_density(const double* D, std::size_t nbf) {
    if (nbf != n_) throw std::invalid_argument("FockBuilder::set_density: nbf mismatch");
    D_ = D;
  }
  const double* density() const { return D_; }
  std::size_t nbf() const { return n_; }
  const std::vector<double>& get_coulomb_matrix() const { return J_; }
  const std::vector<double>& get_exchange_matrix() const { return K_; }
  std::vector<double> get_fock_matrix(const std::vector<double>& H, double exchange_fraction = 0.5) const {
    std::vector<double> F(H);
    for (std::size_t i = 0; i < F.size(); ++i) F[i] += J_[i] - exchange_fraction * K_[i];
    return F;
  }
  void reset() {
    std::fill(J_.begin(), J_.end(), 0.0);
    std::fill(K_.begin(), K_.end(), 0.0);
  }
  // Adds one build's J/K (used by Engine::compute).
  void add(const std::vector<double>& J, const std::vector<double>& K) {
    for (std::size_t i = 0; i < J_.size(); ++i) {
      J_[i] += J[i];
      K_[i] += K[i];
    }
  }

 private:
  friend class Engine;  // work units add into J_/K_ in place
  std::size_t n_;
  const double* D_ = nullptr;
  std::vector<double> J_, K_;
};

class GpuFockBuilder {
 public:
  explicit GpuFockBuilder(std::size_t nbf, cudaStream_t stream = nullptr) : n_(nbf), stream_(stream) {
    const std::size_t bytes = sizeof(double) * nbf * nbf;
    if (cudaMalloc(&d_D_, bytes) != cudaSuccess || cudaMalloc(&d_J_, bytes) != cudaSuccess ||
        cudaMalloc(&d_K_, bytes) != cudaSuccess)
      throw std::runtime_error("GpuFockBuilder: device allocation failed");
    reset();
  }
  ~GpuFockBuilder() {
    cudaFree(d_D_);
    cudaFree(d_J_);
    cudaFree(d_K_);
  }
  GpuFockBuilder(const GpuFockBuilder&) = delete;
  GpuFockBuilder& operator=(const GpuFockBuilder&) = delete;
  // Asynchronous on the builder's stream: keep host_D alive until synchronize().
  void set_density(const double* host_D, std::size_t nbf) {
    if (nbf != n_) throw std::invalid_argument("GpuFockBuilder::set_density: nbf mismatch");
    if (cudaMemcpyAsync(d_D_, host_D, sizeof(double) * n_ * n_, cudaMemcpyHostToDevice, stream_) != cudaSuccess)
      throw std::runtime_error("GpuFockBuilder::set_density: copy failed");
  }
  // J/K contributions of an integral batch already on the device, added in
  // place (plain accumulation, J_ij += (ij|kl) D_kl, K_ik += (ij|kl) D_jl): block t
  // is d_eri + meta[t].offset, [a][b][c][d] over the functions of meta[t], as an
  // IntegralBuffer lays it out.  GpuFockBuilder::accumulate_device_eri_batch
  // (src/device/cuda/consumers/fock_builder_gpu.cu:600-621); the engine supplies
  // the device context.  Asynchronous on the builder's stream.
  void accumulate_device_eri_batch(Engine& engine, const double* d_eri,
                                   const std::vector<ShellQuartetMeta>& meta);
  std::vector<double> get_coulomb_matrix() const { return download(d_J_); }
  std::vector<double> get_exchange_matrix() const { return download(d_K_); }
  void reset() {
    cudaMemsetAsync(d_J_, 0, sizeof(double) * n_ * n_, stream_);
    cudaMemsetAsync(d_K_, 0, sizeof(double) * n_ * n_, stream_);
  }
  void synchronize() const { cudaStreamSynchronize(stream_); }
  double* d_J() const { return d_J_; }
  double* d_K() const { return d_K_; }
  double* d_D() const { return d_D_; }
  cudaStream_t stream() const { return stream_; }
  std::size_t nbf() const { return n_; }

 private:
  std::vector<double> download(const double* d) const {
    std::vector<double> h(n_ * n_);
    if (cudaMemcpyAsync(h.data(), d, sizeof(double) * n_ * n_, cudaMemcpyDeviceToHost, stream_) != cudaSuccess ||
        cudaStreamSynchronize(stream_) != cudaSuccess)
      throw std::runtime_error("GpuFockBuilder: copy failed");
    return h;
  }
  std::size_t n_;
  cudaStream_t stream_;
  double *d_D_ = nullptr, *d_J_ = nullptr, *d_K_ = nullptr;
};

class Engine {
 public:
  // The caller keeps the basis alive while the engine lives (engine.hpp:86-89).
  explicit Engine(const BasisSet& basis, double threshold = 1e-12)
      : basis_(&basis), threshold_(threshold), nbf_(basis.n_basis_functions()) {
    lai_engine_opts o;
    lai_engine_opts_default(&o);
    o.schwarz_threshold = threshold;
    check(lai_engine_create(basis.handle(), &o, &h_), "Engine");
  }
  ~Engine() { lai_engine_destroy(h_); }
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  // The reference's backend hint (include/libaccint/engine/dispatch_policy.hpp:41-47):
  // every hint that allows the GPU runs the B200 path; ForceCPU throws
  // std::invalid_argument, since this build has no CPU path.
  enum class BackendHint { Auto, ForceCPU, ForceGPU, PreferCPU, PreferGPU };
  template <class Builder>
  void compute(const Operator& op, Builder& fb, BackendHint hint) {
    if (hint == BackendHint::ForceCPU)
      throw std::invalid_argument("Engine::compute: BackendHint::ForceCPU -- this build has no CPU backend");
    compute(op, fb);
  }
  bool gpu_available() const { return true; }  // an Engine exists only on a usable device

  // Engine::compute(Operator::coulomb(), FockBuilder&): J/K added to the builder's.
  void compute(const Operator& op, FockBuilder& fb) {
    if (op.kind != Operator::Kind::Coulomb) throw std::invalid_argument("Engine::compute: not a two-electron operator");
    if (!fb.density()) throw std::logic_error("FockBuilder: density matrix not set");
    if (fb.nbf() != nbf_) throw std::invalid_argument("Engine::compute: nbf mismatch");
    std::vector<double> J(nbf_ * nbf_), K(nbf_ * nbf_);
    check(lai_jk_build(h_, fb.density(), nbf_, J.data(), K.data(), nullptr, nullptr), "Engine::compute");
    fb.add(J, K);
  }
  // Engine::compute(Operator::coulomb(), GpuFockBuilder&): device J/K on the
  // builder's stream (overwritten, as after reset()).
  void compute(const Operator& op, GpuFockBuilder& fb) {
    if (op.kind != Operator::Kind::Coulomb) throw std::invalid_argument("Engine::compute: not a two-electron operator");
    if (fb.nbf() != nbf_) throw std::invalid_argument("Engine::compute: nbf mismatch");
    check(lai_jk_build_device(h_, fb.d_D(), fb.d_J(), fb.d_K(), fb.stream(), nullptr, nullptr),
          "Engine::compute");
  }
  // One-electron matrices (nbf x nbf, row-major) of Operator::overlap(), kinetic()
  // or nuclear(charges); Engine::compute_1e(op, result) of the reference.
  void compute_1e(const Operator& op, std::vector<double>& result) {
    result.assign(nbf_ * nbf_, 0.0);
    int code = LAI_OP_OVERLAP;
    std::vector<double> xyz, q;
    switch (op.kind) {
      case Operator::Kind::Overlap: code = LAI_OP_OVERLAP; break;
      case Operator::Kind::Kinetic: code = LAI_OP_KINETIC; break;
      case Operator::Kind::Nuclear: {
        code = LAI_OP_NUCLEAR;
        const auto& c = op.charges;
        const std::size_t n = c.n_centers();
        if (c.x.size() != n || c.y.size() != n || c.z.size() != n)
          throw std::invalid_argument("compute_1e: PointChargeParams sizes differ");
        for (std::size_t i = 0; i < n; ++i) {
          xyz.insert(xyz.end(), {c.x[i], c.y[i], c.z[i]});
          q.push_back(c.charge[i]);
        }
        break;
      }
      default: throw std::invalid_argument("compute_1e: not a one-electron operator");
    }
    check(lai_one_electron(h_, code, (int)q.size(), xyz.empty() ? nullptr : xyz.data(),
                           q.empty() ? nullptr : q.data(), result.data()),
          "Engine::compute_1e");
  }
  void compute_overlap_matrix(std::vector<double>& result) { compute_1e(Operator::overlap(), result); }
  void compute_kinetic_matrix(std::vector<double>& result) { compute_1e(Operator::kinetic(), result); }
  void compute_nuclear_matrix(const PointChargeParams& charges, std::vector<double>& result) {
    compute_1e(Operator::nuclear(charges), result);
  }
  // H_core = T + V in one pass (Engine::compute_core_hamiltonian, engine.hpp:831-900).
  void compute_core_hamiltonian(const PointChargeParams& charges, std::vector<double>& result) {
    const std::size_t n = charges.n_centers();
    if (charges.x.size() != n || charges.y.size() != n || charges.z.size() != n)
      throw std::invalid_argument("compute_core_hamiltonian: PointChargeParams sizes differ");
    std::vector<double> xyz, q(charges.charge);
    for (std::size_t i = 0; i < n; ++i) xyz.insert(xyz.end(), {charges.x[i], charges.y[i], charges.z[i]});
    result.assign(nbf_ * nbf_, 0.0);
    check(lai_one_electron(h_, LAI_OP_HCORE, (int)n, xyz.empty() ? nullptr : xyz.data(),
                           q.empty() ? nullptr : q.data(), result.data()),
          "Engine::compute_core_hamiltonian");
  }

  // ---- work units (no Schwarz or primitive screening inside a unit) ----

  // Integrals of every quartet of the set quartet's full product, in product
  // order (a, b, c, d of the four sets), each block [a][b][c][d]: Engine::compute_batch
  // (include/libaccint/engine/engine.hpp:1008-1122).
  IntegralBuffer compute_batch(const Operator& op, const ShellSetQuartet& quartet) {
    require_coulomb(op, "Engine::compute_batch");
    return listed_integrals(quartet.shell_quartets(false));
  }

  // Every quartet that passes the screening, one representative per permutation
  // orbit, grouped into one IntegralBuffer per run of quartets of the same
  // (la, lb, lc, ld) class: Engine::compute_batch_screened (engine.hpp:1181-1187).
  // A threshold other than the engine's is served by a temporary engine.
  std::vector<IntegralBuffer> compute_batch_screened(const Operator& op, const ScreeningOptions& screening) {
    require_coulomb(op, "Engine::compute_batch_screened");
    if (screening.density_weighted)
      throw std::invalid_argument("Engine::compute_batch_screened: density-weighted screening is not supported");
    const double thr = screening.enabled ? screening.threshold : 0.0;
    if (thr == threshold_) return screened_batch(h_);
    Engine tmp(*basis_, thr);
    return tmp.screened_batch(tmp.h_);
  }

  // J/K contributions of one work unit added to the builder's J and K:
  // CudaEngine::compute_shell_set_quartet(op, quartet, consumer, canonical_symmetry)
  // (include/libaccint/engine/cuda_engine.hpp:462-466, 792-980).  canonical_symmetry
  // = false: plain accumulation of every quartet of the full product
  // (FockBuilder::accumulate); = true: the canonical quartets of the unit
  // (ShellSetQuartet::shell_quartets(true)), each scattered over its permutation
  // orbit (accumulate_symmetric), so that the units of BasisSet::shell_set_quartets()
  // together give the full J and K.
  void compute_shell_set_quartet(const Operator& op, const ShellSetQuartet& quartet, FockBuilder& fb,
                                 bool canonical_symmetry = false) {
    require_coulomb(op, "Engine::compute_shell_set_quartet");
    if (!fb.density()) throw std::logic_error("FockBuilder: density matrix not set");
    if (fb.nbf() != nbf_) throw std::invalid_argument("Engine::compute_shell_set_quartet: nbf mismatch");
    const std::vector<int32_t> q = quartet.shell_quartets(canonical_symmetry);
    check(lai_jk_accumulate_quartets(h_, q.data(), (int64_t)(q.size() / 4), fb.density(), fb.J_.data(),
                                     fb.K_.data(), canonical_symmetry ? 1 : 0),
          "Engine::compute_shell_set_quartet");
  }
  // The same into a GpuFockBuilder's device J/K; returns once the unit's kernels
  // have finished on the builder's stream.
  void compute_shell_set_quartet(const Operator& op, const ShellSetQuartet& quartet, GpuFockBuilder& fb,
                                 bool canonical_symmetry = false) {
    require_coulomb(op, "Engine::compute_shell_set_quartet");
    if (fb.nbf() != nbf_) throw std::invalid_argument("Engine::compute_shell_set_quartet: nbf mismatch");
    const std::vector<int32_t> q = quartet.shell_quartets(canonical_symmetry);
    check(lai_jk_accumulate_quartets_device(h_, q.data(), (int64_t)(q.size() / 4), fb.d_D(), fb.d_J(),
                                            fb.d_K(), fb.stream(), canonical_symmetry ? 1 : 0),
          "Engine::compute_shell_set_quartet");
  }

  lai_engine* handle() const { return h_; }
  std::size_t nbf() const { return nbf_; }

 private:
  static void require_coulomb(const Operator& op, const char* what) {
    if (op.kind != Operator::Kind::Coulomb)
      throw std::invalid_argument(std::string(what) + ": not a two-electron operator");
  }
  static ShellQuartetMeta to_meta(const lai_quartet_meta& m) {
    ShellQuartetMeta r;
    r.offset = (std::size_t)m.offset;
    r.fi = m.fa; r.fj = m.fb; r.fk = m.fc; r.fl = m.fd;
    r.na = m.na; r.nb = m.nb; r.nc = m.nc; r.nd = m.nd;
    return r;
  }
  IntegralBuffer listed_integrals(const std::vector<int32_t>& q) {
    const int64_t n = (int64_t)(q.size() / 4);
    std::size_t nv = 0;
    for (int64_t t = 0; t < n; ++t) {
      std::size_t v = 1;
      for (int x = 0; x < 4; ++x) {
        int l = 0;
        check(lai_basis_shell(basis_->handle(), q[4 * t + x], &l, nullptr, nullptr, nullptr, nullptr, nullptr),
              "Engine::compute_batch");
        v *= (std::size_t)(l + 1) * (l + 2) / 2;
      }
      nv += v;
    }
    IntegralBuffer buf;
    if (n == 0) return buf;
    buf.data_.resize(nv);
    std::vector<lai_quartet_meta> m((std::size_t)n);
    check(lai_eri_quartets(h_, q.data(), n, buf.data_.data(), nv, m.data()), "Engine::compute_batch");
    for (const lai_quartet_meta& x : m) buf.meta_.push_back(to_meta(x));
    return buf;
  }
  std::vector<IntegralBuffer> screened_batch(lai_engine* h) {
    int64_t nq = 0, nv = 0;
    check(lai_eri_batch_screened(h, nullptr, 0, nullptr, 0, &nq, &nv), "Engine::compute_batch_screened");
    std::vector<double> vals((std::size_t)nv);
    std::vector<lai_quartet_meta> m((std::size_t)nq);
    check(lai_eri_batch_screened(h, vals.data(), vals.size(), m.data(), m.size(), &nq, &nv),
          "Engine::compute_batch_screened");
    std::vector<IntegralBuffer> out;
    for (int64_t t = 0; t < nq; ++t) {
      const lai_quartet_meta& x = m[(std::size_t)t];
      const bool same = t > 0 && x.na == m[t - 1].na && x.nb == m[t - 1].nb && x.nc == m[t - 1].nc &&
                        x.nd == m[t - 1].nd;
      if (!same) out.emplace_back();
      IntegralBuffer& b = out.back();
      ShellQuartetMeta r = to_meta(x);
      r.offset = b.data_.size();
      const std::size_t sz = (std::size_t)x.na * x.nb * x.nc * x.nd;
      b.data_.insert(b.data_.end(), vals.begin() + x.offset, vals.begin() + x.offset + sz);
      b.meta_.push_back(r);
    }
    return out;
  }

  const BasisSet* basis_;
  double threshold_;
  std::size_t nbf_;
  lai_engine* h_ = nullptr;
};

inline void GpuFockBuilder::accumulate_device_eri_batch(Engine& engine, const double* d_eri,
                                                        const std::vector<ShellQuartetMeta>& meta) {
  if (engine.nbf() != n_) throw std::invalid_argument("GpuFockBuilder::accumulate_device_eri_batch: nbf mismatch");
  std::vector<lai_quartet_meta> m(meta.size());
  for (std::size_t t = 0; t < meta.size(); ++t) {
    const ShellQuartetMeta& x = meta[t];
    m[t].offset = (int64_t)x.offset;
    m[t].fa = (int32_t)x.fi; m[t].fb = (int32_t)x.fj; m[t].fc = (int32_t)x.fk; m[t].fd = (int32_t)x.fl;
    m[t].na = x.na; m[t].nb = x.nb; m[t].nc = x.nc; m[t].nd = x.nd;
  }
  check(lai_jk_accumulate_eri_batch_device(engine.handle(), d_eri, m.data(), (int64_t)m.size(), d_D_, d_J_,
                                           d_K_, stream_),
        "GpuFockBuilder::accumulate_device_eri_batch");
}

// The reference's namespace for its consumers (include/libaccint/consumers/).
namespace consumers {
using lai::FockBuilder;
using lai::GpuFockBuilder;
}  // namespace consumers

using BackendHint = Engine::BackendHint;

}  // namespace lai

#endif /* LIBACCINT_B200_HPP */
