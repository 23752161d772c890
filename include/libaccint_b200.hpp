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
  ~BasisSet() { lai_basis_destroy(h_); }
  BasisSet(const BasisSet&) = delete;
  BasisSet& operator=(const BasisSet&) = delete;
  std::size_t n_basis_functions() const { return (std::size_t)lai_basis_nbf(h_); }
  const lai_basis* handle() const { return h_; }

 private:
  lai_basis* h_ = nullptr;
};

struct Operator {
  static Operator coulomb() { return Operator{}; }
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
  void compute(const Operator&, FockBuilder& fb) {
    if (!fb.density()) throw std::logic_error("FockBuilder: density matrix not set");
    if (fb.nbf() != nbf_) throw std::invalid_argument("Engine::compute: nbf mismatch");
    std::vector<double> J(nbf_ * nbf_), K(nbf_ * nbf_);
    check(lai_jk_build(h_, fb.density(), nbf_, J.data(), K.data(), nullptr, nullptr), "Engine::compute");
    fb.add(J, K);
  }
  // Engine::compute(Operator::coulomb(), GpuFockBuilder&): device J/K on the
  // builder's stream (overwritten, as after reset()).
  void compute(const Operator&, GpuFockBuilder& fb) {
    if (fb.nbf() != nbf_) throw std::invalid_argument("Engine::compute: nbf mismatch");
    check(lai_jk_build_device(h_, fb.d_D(), fb.d_J(), fb.d_K(), fb.stream(), nullptr, nullptr),
          "Engine::compute");
  }
  lai_engine* handle() const { return h_; }

 private:
  std::size_t nbf_;
  lai_engine* h_ = nullptr;
};

}  // namespace lai

#endif /* LIBACCINT_B200_HPP */
