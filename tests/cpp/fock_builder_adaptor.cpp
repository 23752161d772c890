// Drives the C++ adaptors of include/libaccint_b200.hpp the way a reference user
// drives Engine/FockBuilder/GpuFockBuilder: reads shells and a density from text
// files, writes J and K from both builders.
//   usage: fock_builder_adaptor basis.txt density.txt out_prefix
//   basis.txt: one shell per line: l atom x y z nprim exp... coef...
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "libaccint_b200.hpp"

static void write(const std::string& path, const std::vector<double>& v) {
  std::ofstream f(path);
  f.precision(17);
  for (double x : v) f << x << "\n";
}

int main(int argc, char** argv) {
  if (argc < 4) return 2;
  std::vector<lai::Shell> shells;
  std::ifstream bf(argv[1]);
  std::string line;
  while (std::getline(bf, line)) {
    std::istringstream in(line);
    lai::Shell s;
    int np = 0;
    if (!(in >> s.l >> s.atom >> s.center[0] >> s.center[1] >> s.center[2] >> np)) continue;
    s.exps.resize(np);
    s.coefs.resize(np);
    for (double& e : s.exps) in >> e;
    for (double& c : s.coefs) in >> c;
    shells.push_back(s);
  }
  std::vector<double> D;
  std::ifstream df(argv[2]);
  for (double x; df >> x;) D.push_back(x);
  try {
    lai::BasisSet basis(shells);
    const std::size_t n = basis.n_basis_functions();
    if (D.size() != n * n) return 3;
    lai::Engine engine(basis);
    lai::FockBuilder fb(n);
    fb.set_density(D.data(), n);
    engine.compute(lai::Operator::coulomb(), fb);
    write(std::string(argv[3]) + "_J.txt", fb.get_coulomb_matrix());
    write(std::string(argv[3]) + "_K.txt", fb.get_exchange_matrix());
    lai::GpuFockBuilder gfb(n);
    gfb.set_density(D.data(), n);
    engine.compute(lai::Operator::coulomb(), gfb);
    gfb.synchronize();
    write(std::string(argv[3]) + "_Jgpu.txt", gfb.get_coulomb_matrix());
    write(std::string(argv[3]) + "_Kgpu.txt", gfb.get_exchange_matrix());
    // errors surface as exceptions, as in the reference
    try {
      lai::FockBuilder wrong(n + 1);
      std::vector<double> Dw((n + 1) * (n + 1), 0.0);
      wrong.set_density(Dw.data(), n + 1);
      engine.compute(lai::Operator::coulomb(), wrong);
      return 4;
    } catch (const std::invalid_argument&) {
    }
  } catch (const std::exception& ex) {
    std::fprintf(stderr, "%s\n", ex.what());
    return 1;
  }
  return 0;
}
