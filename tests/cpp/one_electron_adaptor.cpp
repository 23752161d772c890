// Compile-and-link check of the one-electron and BSE parts of the C++ adaptors
// (include/libaccint_b200.hpp): builds S, T and V of a basis read from Basis Set
// Exchange JSON, as a reference user would call Engine::compute_overlap_matrix /
// compute_kinetic_matrix / compute_nuclear_matrix.
//   usage: one_electron_adaptor basis.json out_prefix
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "libaccint_b200.hpp"

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  std::ifstream f(argv[1]);
  std::stringstream ss;
  ss << f.rdbuf();
  const std::vector<int> Z = {8, 1, 1};
  const std::vector<double> xyz = {0.0, 0.0, 0.0, 0.0, 1.43233673, -1.10866041, 0.0, -1.43233673, -1.10866041};
  lai::BasisSet basis = lai::BasisSet::from_bse_json(ss.str(), Z, xyz);
  lai::Engine engine(basis);
  lai::PointChargeParams nuclei;
  for (std::size_t a = 0; a < Z.size(); ++a) {
    nuclei.x.push_back(xyz[3 * a]);
    nuclei.y.push_back(xyz[3 * a + 1]);
    nuclei.z.push_back(xyz[3 * a + 2]);
    nuclei.charge.push_back(Z[a]);
  }
  std::vector<double> S, T, V;
  engine.compute_overlap_matrix(S);
  engine.compute_kinetic_matrix(T);
  engine.compute_nuclear_matrix(nuclei, V);
  const std::string prefix = argv[2];
  for (auto& [tag, M] : {std::pair<const char*, std::vector<double>*>{"S", &S}, {"T", &T}, {"V", &V}}) {
    std::ofstream o(prefix + "_" + tag + ".txt");
    o.precision(17);
    for (double x : *M) o << x << "\n";
  }
  return 0;
}
