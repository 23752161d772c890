// Drives the work-unit and raw-integral adaptors of include/libaccint_b200.hpp
// the way a reference user drives ShellSetQuartet work units,
// compute_batch / compute_batch_screened and GpuFockBuilder's external-batch
// digestion.
//
//   work_unit_adaptor cpu basis.txt
//       host-only checks, no device needed: the shell sets, the canonical
//       enumeration over BasisSet::shell_set_quartets() (every permutation orbit
//       exactly once), the full-product enumeration over all ordered set
//       quartets (every ordered quartet exactly once), and the orbit scatter of
//       an integral batch, on a synthetic integral with the 8-fold symmetry of
//       (mn|ls) against the direct sum J_mn = sum_ls v D_ls, K_ml = sum_ns v D_ns.
//   work_unit_adaptor gpu basis.txt density.txt out_prefix
//       writes J and K (out_prefix_<route>_{J,K}.txt) of five routes:
//         sym      compute_shell_set_quartet(canonical_symmetry) over
//                  shell_set_quartets(), FockBuilder
//         gsym     the same into a GpuFockBuilder
//         plain    compute_shell_set_quartet (plain) over every ordered set quartet
//         screened compute_batch_screened(none()) + the orbit scatter on the host
//         devbatch compute_batch over every ordered set quartet, uploaded, and
//                  GpuFockBuilder::accumulate_device_eri_batch
//   basis.txt: one shell per line: l atom x y z nprim exp... coef...
#include <cmath>
#include <cstdio>
#include <fstream>
#include <set>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "libaccint_b200.hpp"

namespace {

std::vector<lai::Shell> read_shells(const char* path) {
  std::vector<lai::Shell> shells;
  std::ifstream bf(path);
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
  return shells;
}

void write(const std::string& path, const std::vector<double>& v) {
  std::ofstream f(path);
  f.precision(17);
  for (double x : v) f << x << "\n";
}

// The ordered (bra | ket) set quartets over all ordered set pairs: their full
// products hold every ordered shell quartet of the basis exactly once.
struct OrderedUnits {
  std::vector<lai::ShellSetPair> pairs;
  std::vector<lai::ShellSetQuartet> units;
  explicit OrderedUnits(const lai::BasisSet& basis) {
    const std::vector<const lai::ShellSet*> s = basis.shell_sets();
    pairs.reserve(s.size() * s.size());
    for (const lai::ShellSet* a : s)
      for (const lai::ShellSet* b : s) pairs.emplace_back(*a, *b);
    for (const auto& p : pairs)
      for (const auto& q : pairs) units.emplace_back(p, q);
  }
};

// Adds one quartet block (one representative of its permutation orbit) to J and
// K over every distinct ordered shell quartet of the orbit, as the reference's
// FockBuilder::accumulate_symmetric does with its degeneracy flags
// (src/shared/consumers/fock_builder.cpp:123-222).
void scatter_orbit(const lai::ShellQuartetMeta& m, const double* v, const std::vector<double>& D,
                   std::size_t nbf, std::vector<double>& J, std::vector<double>& K) {
  static const int perms[8][4] = {{0, 1, 2, 3}, {1, 0, 2, 3}, {0, 1, 3, 2}, {1, 0, 3, 2},
                                  {2, 3, 0, 1}, {3, 2, 0, 1}, {2, 3, 1, 0}, {3, 2, 1, 0}};
  const long f[4] = {m.fi, m.fj, m.fk, m.fl};
  const int n[4] = {m.na, m.nb, m.nc, m.nd};
  std::set<std::tuple<long, long, long, long>> seen;
  for (const auto& P : perms) {
    if (!seen.insert({f[P[0]], f[P[1]], f[P[2]], f[P[3]]}).second) continue;
    int x[4];
    std::size_t e = 0;
    for (x[0] = 0; x[0] < n[0]; ++x[0])
      for (x[1] = 0; x[1] < n[1]; ++x[1])
        for (x[2] = 0; x[2] < n[2]; ++x[2])
          for (x[3] = 0; x[3] < n[3]; ++x[3], ++e) {
            const std::size_t mu = f[P[0]] + x[P[0]], nu = f[P[1]] + x[P[1]];
            const std::size_t la = f[P[2]] + x[P[2]], si = f[P[3]] + x[P[3]];
            J[mu * nbf + nu] += v[e] * D[la * nbf + si];
            K[mu * nbf + la] += v[e] * D[nu * nbf + si];
          }
  }
}

// Plain accumulation of an ordered quartet block (FockBuilder::accumulate).
void accumulate_plain(const lai::ShellQuartetMeta& m, const double* v, const std::vector<double>& D,
                      std::size_t nbf, std::vector<double>& J, std::vector<double>& K) {
  std::size_t e = 0;
  for (int a = 0; a < m.na; ++a)
    for (int b = 0; b < m.nb; ++b)
      for (int c = 0; c < m.nc; ++c)
        for (int d = 0; d < m.nd; ++d, ++e) {
          const std::size_t mu = m.fi + a, nu = m.fj + b, la = m.fk + c, si = m.fl + d;
          J[mu * nbf + nu] += v[e] * D[la * nbf + si];
          K[mu * nbf + la] += v[e] * D[nu * nbf + si];
        }
}

double sym_s(std::size_t m, std::size_t n) { return 1.0 / (1.0 + m + n) + 0.01 * (double)((m * n) % 7); }
// A synthetic "integral" with the 8-fold symmetry of (mn|ls).
double synth(std::size_t m, std::size_t n, std::size_t l, std::size_t s) {
  return sym_s(m, n) * sym_s(l, s) + 0.5 * (sym_s(m, n) + sym_s(l, s));
}

struct ShellInfo {
  long func;
  int ncart;
};

lai::ShellQuartetMeta meta_of(const std::vector<ShellInfo>& sh, const int32_t* q) {
  lai::ShellQuartetMeta m;
  m.fi = sh[q[0]].func; m.fj = sh[q[1]].func; m.fk = sh[q[2]].func; m.fl = sh[q[3]].func;
  m.na = sh[q[0]].ncart; m.nb = sh[q[1]].ncart; m.nc = sh[q[2]].ncart; m.nd = sh[q[3]].ncart;
  return m;
}

std::vector<double> synth_block(const lai::ShellQuartetMeta& m) {
  std::vector<double> v;
  for (int a = 0; a < m.na; ++a)
    for (int b = 0; b < m.nb; ++b)
      for (int c = 0; c < m.nc; ++c)
        for (int d = 0; d < m.nd; ++d) v.push_back(synth(m.fi + a, m.fj + b, m.fk + c, m.fl + d));
  return v;
}

double max_diff(const std::vector<double>& a, const std::vector<double>& b) {
  double r = 0.0;
  for (std::size_t i = 0; i < a.size(); ++i) r = std::fmax(r, std::fabs(a[i] - b[i]));
  return r;
}

int run_cpu(const lai::BasisSet& basis) {
  const std::size_t nbf = basis.n_basis_functions(), ns = basis.n_shells();
  std::vector<ShellInfo> sh(ns);
  for (std::size_t s = 0; s < ns; ++s) {
    int l = 0;
    long f = 0;
    lai::check(lai_basis_shell(basis.handle(), (int)s, &l, nullptr, nullptr, nullptr, nullptr, &f), "shell");
    sh[s] = {f, (l + 1) * (l + 2) / 2};
  }
  int bad = 0;
  // shell sets: every shell once, one (l, nprim) per set, in first-appearance order
  std::size_t nin = 0;
  for (const lai::ShellSet* s : basis.shell_sets()) nin += s->n_shells();
  if (nin != ns) { std::fprintf(stderr, "shell sets hold %zu of %zu shells\n", nin, ns); ++bad; }
  // canonical enumeration: every orbit exactly once
  std::set<std::tuple<int, int, int, int>> orbits;
  std::size_t listed = 0;
  auto key = [](int a, int b, int c, int d) {
    if (a < b) std::swap(a, b);
    if (c < d) std::swap(c, d);
    if (std::make_pair(a, b) < std::make_pair(c, d)) { std::swap(a, c); std::swap(b, d); }
    return std::make_tuple(a, b, c, d);
  };
  std::vector<double> D(nbf * nbf), J0(nbf * nbf, 0.0), K0(nbf * nbf, 0.0);
  for (std::size_t i = 0; i < nbf; ++i)
    for (std::size_t j = 0; j <= i; ++j) D[i * nbf + j] = D[j * nbf + i] = std::cos(0.37 * i + 0.11 * j * j);
  for (std::size_t m = 0; m < nbf; ++m)
    for (std::size_t n = 0; n < nbf; ++n)
      for (std::size_t l = 0; l < nbf; ++l)
        for (std::size_t s = 0; s < nbf; ++s) {
          const double v = synth(m, n, l, s);
          J0[m * nbf + n] += v * D[l * nbf + s];
          K0[m * nbf + l] += v * D[n * nbf + s];
        }
  std::vector<double> J(nbf * nbf, 0.0), K(nbf * nbf, 0.0);
  for (const lai::ShellSetQuartet& u : basis.shell_set_quartets()) {
    const std::vector<int32_t> q = u.shell_quartets(true);
    for (std::size_t t = 0; t < q.size(); t += 4) {
      ++listed;
      orbits.insert(key(q[t], q[t + 1], q[t + 2], q[t + 3]));
      const lai::ShellQuartetMeta m = meta_of(sh, &q[t]);
      const std::vector<double> v = synth_block(m);
      scatter_orbit(m, v.data(), D, nbf, J, K);
    }
  }
  const std::size_t npair = ns * (ns + 1) / 2, norbit = npair * (npair + 1) / 2;
  if (listed != norbit || orbits.size() != norbit) {
    std::fprintf(stderr, "canonical units list %zu quartets, %zu distinct orbits, expected %zu\n", listed,
                 orbits.size(), norbit);
    ++bad;
  }
  const double scale = std::fmax(1.0, max_diff(J0, std::vector<double>(J0.size(), 0.0)));
  if (max_diff(J, J0) > 1e-12 * scale || max_diff(K, K0) > 1e-12 * scale) {
    std::fprintf(stderr, "orbit scatter: max|dJ| %.3e max|dK| %.3e\n", max_diff(J, J0), max_diff(K, K0));
    ++bad;
  }
  // full products of the ordered units: every ordered quartet exactly once
  OrderedUnits ou(basis);
  std::set<std::tuple<int, int, int, int>> ordered;
  std::size_t nord = 0;
  std::fill(J.begin(), J.end(), 0.0);
  std::fill(K.begin(), K.end(), 0.0);
  for (const lai::ShellSetQuartet& u : ou.units) {
    const std::vector<int32_t> q = u.shell_quartets(false);
    if (q.size() != 4 * u.n_quartets()) ++bad;
    for (std::size_t t = 0; t < q.size(); t += 4) {
      ++nord;
      ordered.insert({q[t], q[t + 1], q[t + 2], q[t + 3]});
      const lai::ShellQuartetMeta m = meta_of(sh, &q[t]);
      const std::vector<double> v = synth_block(m);
      accumulate_plain(m, v.data(), D, nbf, J, K);
    }
  }
  if (nord != ns * ns * ns * ns || ordered.size() != nord) {
    std::fprintf(stderr, "ordered units list %zu quartets (%zu distinct), expected %zu\n", nord, ordered.size(),
                 ns * ns * ns * ns);
    ++bad;
  }
  if (max_diff(J, J0) > 1e-12 * scale || max_diff(K, K0) > 1e-12 * scale) {
    std::fprintf(stderr, "plain accumulation: max|dJ| %.3e max|dK| %.3e\n", max_diff(J, J0), max_diff(K, K0));
    ++bad;
  }
  std::printf("cpu checks: %zu shells, %zu sets, %zu orbits, %zu ordered quartets, %d failures\n", ns,
              basis.shell_sets().size(), orbits.size(), nord, bad);
  return bad ? 1 : 0;
}

int run_gpu(const lai::BasisSet& basis, const std::vector<double>& D, const std::string& prefix) {
  const std::size_t n = basis.n_basis_functions();
  if (D.size() != n * n) return 3;
  lai::Engine engine(basis, 0.0);
  const lai::Operator op = lai::Operator::coulomb();
  auto out = [&](const char* route, const std::vector<double>& J, const std::vector<double>& K) {
    write(prefix + "_" + route + "_J.txt", J);
    write(prefix + "_" + route + "_K.txt", K);
  };
  {  // canonical units, host builder
    lai::FockBuilder fb(n);
    fb.set_density(D.data(), n);
    for (const lai::ShellSetQuartet& u : basis.shell_set_quartets()) engine.compute_shell_set_quartet(op, u, fb, true);
    out("sym", fb.get_coulomb_matrix(), fb.get_exchange_matrix());
  }
  {  // canonical units, device builder
    lai::GpuFockBuilder gfb(n);
    gfb.set_density(D.data(), n);
    for (const lai::ShellSetQuartet& u : basis.shell_set_quartets()) engine.compute_shell_set_quartet(op, u, gfb, true);
    gfb.synchronize();
    out("gsym", gfb.get_coulomb_matrix(), gfb.get_exchange_matrix());
  }
  OrderedUnits ou(basis);
  {  // ordered units, plain accumulation
    lai::FockBuilder fb(n);
    fb.set_density(D.data(), n);
    for (const lai::ShellSetQuartet& u : ou.units) engine.compute_shell_set_quartet(op, u, fb, false);
    out("plain", fb.get_coulomb_matrix(), fb.get_exchange_matrix());
  }
  {  // screened batch (no screening) scattered on the host
    std::vector<double> J(n * n, 0.0), K(n * n, 0.0);
    const std::vector<lai::IntegralBuffer> bufs = engine.compute_batch_screened(op, lai::ScreeningOptions::none());
    std::size_t nq = 0;
    for (const lai::IntegralBuffer& b : bufs)
      for (std::size_t i = 0; i < b.n_quartets(); ++i, ++nq) {
        const lai::ShellQuartetMeta& m = b.quartet_meta(i);
        if (b.quartet_size(i) != (std::size_t)m.na * m.nb * m.nc * m.nd) return 4;
        scatter_orbit(m, b.quartet_data(i), D, n, J, K);
      }
    const std::size_t ns = basis.n_shells(), npair = ns * (ns + 1) / 2;
    if (nq != npair * (npair + 1) / 2) {
      std::fprintf(stderr, "screened batch: %zu quartets, expected %zu\n", nq, npair * (npair + 1) / 2);
      return 5;
    }
    out("screened", J, K);
  }
  {  // compute_batch per ordered unit, digested on the device
    lai::GpuFockBuilder gfb(n);
    gfb.set_density(D.data(), n);
    double* d_eri = nullptr;
    std::size_t cap = 0;
    for (const lai::ShellSetQuartet& u : ou.units) {
      const lai::IntegralBuffer b = engine.compute_batch(op, u);
      if (b.n_quartets() != u.n_quartets()) return 6;
      if (b.empty()) continue;
      if (b.n_integrals() > cap) {
        gfb.synchronize();
        cudaFree(d_eri);
        cap = b.n_integrals();
        if (cudaMalloc(&d_eri, sizeof(double) * cap) != cudaSuccess) return 7;
      }
      gfb.synchronize();  // the previous batch's digestion reads d_eri
      if (cudaMemcpy(d_eri, b.data().data(), sizeof(double) * b.n_integrals(), cudaMemcpyHostToDevice) !=
          cudaSuccess)
        return 7;
      gfb.accumulate_device_eri_batch(engine, d_eri, b.metas());
    }
    gfb.synchronize();
    cudaFree(d_eri);
    out("devbatch", gfb.get_coulomb_matrix(), gfb.get_exchange_matrix());
  }
  // errors surface as exceptions, as in the reference
  try {
    (void)engine.compute_batch_screened(lai::Operator::overlap(), lai::ScreeningOptions::normal());
    return 8;
  } catch (const std::invalid_argument&) {
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  try {
    lai::BasisSet basis(read_shells(argv[2]));
    if (std::string(argv[1]) == "cpu") return run_cpu(basis);
    if (argc < 5) return 2;
    std::vector<double> D;
    std::ifstream df(argv[3]);
    for (double x; df >> x;) D.push_back(x);
    return run_gpu(basis, D, argv[4]);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "exception: %s\n", e.what());
    return 10;
  }
}
