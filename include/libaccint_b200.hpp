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
#include <stdexcept>
#include <string>
#include <vector>

#include "libaccint_b200.h"

namespace lai {

inline void check(int rc, const char* what) {
  if (rc == LAI_OK) return;
  const std::string msg = std::string(what) + ": " + lai_last_error();
  if (rc == LAI_EINVAL) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

struct Shell {
  int l;
  double center[3];
  std::vector<double> exps, coefs;  // raw contraction coefficients
  int atom = -1;
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
  BasisSet(BasisSet&& o) noexcept : h_(o.h_) { o.h_ = nullptr; }
  ~BasisSet() { lai_basis_destroy(h_); }
  BasisSet(const BasisSet&) = delete;
  BasisSet& operator=(const BasisSet&) = delete;
  std::size_t n_basis_functions() const { return (std::size_t)lai_basis_nbf(h_); }
  const lai_basis* handle() const { return h_; }

 private:
  explicit BasisSet(lai_basis* h) : h_(h) {}
  lai_basis* h_ = nullptr;
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
  explicit Engine(const BasisSet& basis, double threshold = 1e-12) : nbf_(basis.n_basis_functions()) {
    lai_engine_opts o;
    lai_engine_opts_default(&o);
    o.schwarz_threshold = threshold;
    check(lai_engine_create(basis.handle(), &o, &h_), "Engine");
  }
  ~Engine() { lai_engine_destroy(h_); }
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

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
  lai_engine* handle() const { return h_; }

 private:
  std::size_t nbf_;
  lai_engine* h_ = nullptr;
};

}  // namespace lai

#endif /* LIBACCINT_B200_HPP */
