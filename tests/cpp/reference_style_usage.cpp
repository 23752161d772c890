// Compile-and-link check: code written with the reference's names and shapes
// (Shell(am, Point3D, exps, coefs), BasisSet({...}), Engine, consumers::FockBuilder,
// BackendHint, PointChargeParams, compute_core_hamiltonian, Real / Size) builds
// against include/libaccint_b200.hpp with only the namespace changed.
//   usage: reference_style_usage   (needs a CUDA device to run; the CPU tests only link it)
#include <cmath>
#include <cstdio>
#include <vector>

#include "libaccint_b200.hpp"

using namespace lai;

int main() {
  std::printf("%s, CUDA backend %s\n", version(), has_cuda_backend() ? "on" : "off");
  // two s shells of a stretched H2 (STO-3G exponents and raw coefficients)
  const std::vector<Real> e = {3.42525091, 0.62391373, 0.16885540};
  const std::vector<Real> c = {0.15432897, 0.53532814, 0.44463454};
  Shell a(0, Point3D{0.0, 0.0, 0.0}, e, c);
  Shell b(0, Point3D{0.0, 0.0, 1.4}, e, c);
  BasisSet basis({a, b});
  Engine engine(basis);
  const Size nbf = basis.n_basis_functions();
  if (!engine.gpu_available()) return 2;

  PointChargeParams nuclei;
  for (double z : {0.0, 1.4}) {
    nuclei.x.push_back(0.0);
    nuclei.y.push_back(0.0);
    nuclei.z.push_back(z);
    nuclei.charge.push_back(1.0);
  }
  std::vector<Real> S, H;
  engine.compute_overlap_matrix(S);
  engine.compute_core_hamiltonian(nuclei, H);

  std::vector<Real> D(nbf * nbf, 0.0);
  for (Size i = 0; i < nbf; ++i) D[i * nbf + i] = 1.0;
  consumers::FockBuilder fock(nbf);
  fock.set_density(D.data(), nbf);
  engine.compute(Operator::coulomb(), fock, BackendHint::PreferGPU);
  const std::vector<Real> F = fock.get_fock_matrix(H);
  bool threw = false;
  try {
    engine.compute(Operator::coulomb(), fock, BackendHint::ForceCPU);
  } catch (const std::invalid_argument&) {
    threw = true;
  }
  std::printf("S01 %.10f  F00 %.10f  ForceCPU refused: %s\n", S[1], F[0], threw ? "yes" : "no");
  return threw && std::isfinite(F[0]) ? 0 : 1;
}
