// One-electron integrals (overlap, kinetic energy, point-charge attraction) over
// the engine's contracted Cartesian shells, written as full symmetric nbf x nbf
// matrices, and the C ABI around them.  They complete the core Hamiltonian of an
// SCF iteration whose two-electron part is the J/K build.
//
// One thread per shell pair (a, b) with la >= lb, one launch per (la, lb) class,
// compile-time specialised so the 1D tables and the output block live in
// registers.  Per primitive pair (alpha, beta), p = alpha + beta,
// P = (alpha A + beta B)/p, K_AB = exp(-alpha beta |AB|^2 / p):
//   overlap   s(i+1, 0) = PA s(i, 0) + i/(2p) s(i-1, 0), s(0, 0) = 1, then the
//             transfer s(i, j+1) = s(i+1, j) + AB s(i, j); S = c (pi/p)^{3/2}
//             sx sy sz (Obara-Saika, src/host/kernels/overlap_kernel.cpp:23-74);
//   kinetic   t(i, j) = -1/2 [ j(j-1) s(i, j-2) - 2 beta (2j+1) s(i, j)
//             + 4 beta^2 s(i, j+2) ] (the second derivative taken on the ket
//             Gaussian), T = c (pi/p)^{3/2} (tx sy sz + sx ty sz + sx sy tz)
//             (src/host/kernels/kinetic_kernel.cpp:27-108 writes the same
//             integrals through overlap differences);
//   nuclear   per charge C and root t^2 = u of the n = (la+lb)/2 + 1 point Rys rule
//             at T = p |PC|^2: I(i+1, 0) = (PA - u PC) I(i, 0) + i (1-u)/(2p) I(i-1, 0),
//             the same transfer, V = -q_C c (2 pi/p) sum_r w_r Ix Iy Iz
//             (src/host/kernels/nuclear_kernel.cpp:28-86, 124-230).
// Every shell pair is written once into both triangles, so the matrix needs no
// zeroing and no atomics; T + V is a kinetic pass followed by a nuclear pass that
// adds to it.  Per-component normalization as in the J/K kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "engine_internal.h"
#include "one_electron_impl.cuh"

using namespace lai::host;

namespace lai {
namespace {

int launch_class(int la, int lb, int op, const OneEArgs& g, const int2* pairs, int n, cudaStream_t s) {
  if (la <= 2) return launch_one_e_l012(la, lb, op, g, pairs, n, s);
  if (la == 3) return launch_one_e_l3(la, lb, op, g, pairs, n, s);
  return launch_one_e_l4(la, lb, op, g, pairs, n, s);
}

// Shell table, primitives and class-grouped shell pairs of the engine's basis.
int ensure_tables(lai_engine* E) {
  if (!E->one_e_class.empty()) return LAI_OK;
  const auto& sh = E->basis->shells;
  const int n = (int)sh.size();
  std::vector<OneEShell> tab(n);
  std::vector<double> ex, co;
  for (int s = 0; s < n; ++s) {
    if (sh[s].l > 4) return fail(LAI_ENOTSUP, "one-electron integrals: shells up to l = 4");
    tab[s] = {sh[s].center[0], sh[s].center[1], sh[s].center[2], sh[s].l, (int)sh[s].exps.size(),
              (int)ex.size(), (int)sh[s].func};
    ex.insert(ex.end(), sh[s].exps.begin(), sh[s].exps.end());
    co.insert(co.end(), sh[s].coefs.begin(), sh[s].coefs.end());
  }
  std::vector<std::vector<int2>> cls(25);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      int a = i, b = j;
      if (sh[a].l < sh[b].l) std::swap(a, b);
      cls[sh[a].l * 5 + sh[b].l].push_back(make_int2(a, b));
    }
  std::vector<int2> all;
  std::vector<int> meta;
  for (int k = 0; k < 25; ++k) {
    if (cls[k].empty()) continue;
    meta.insert(meta.end(), {k / 5, k % 5, (int)all.size(), (int)cls[k].size()});
    all.insert(all.end(), cls[k].begin(), cls[k].end());
  }
  LAI_CUDA_TRY(upload(E->d_1e_shell, tab));
  LAI_CUDA_TRY(upload(E->d_1e_exp, ex));
  LAI_CUDA_TRY(upload(E->d_1e_coef, co));
  LAI_CUDA_TRY(upload(E->d_1e_pairs, all));
  E->one_e_class = meta;
  return LAI_OK;
}

}  // namespace
}  // namespace lai

extern "C" {

int lai_one_electron_device(lai_engine* engine, int op, int ncharge, const double* charge_xyz,
                            const double* charge_q, double* d_out, void* stream) {
  if (!engine || !d_out) return fail(LAI_EINVAL, "lai_one_electron_device: null argument");
  if (engine->nsys > 1) return fail(LAI_ENOTSUP, "lai_one_electron: not available for a batched engine");
  if (op < LAI_OP_OVERLAP || op > LAI_OP_HCORE) return fail(LAI_EINVAL, "lai_one_electron: unknown operator");
  const bool nuc = op == LAI_OP_NUCLEAR || op == LAI_OP_HCORE;
  if (nuc && (ncharge < 0 || (ncharge > 0 && (!charge_xyz || !charge_q))))
    return fail(LAI_EINVAL, "lai_one_electron: charges missing");
  LAI_CUDA_TRY(cudaSetDevice(engine->device));
  if (int rc = lai::ensure_tables(engine)) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nc = nuc ? ncharge : 0;
  if (nc > 0) {
    std::vector<double> ch(4 * (size_t)nc);
    for (int c = 0; c < nc; ++c) {
      ch[4 * c] = charge_xyz[3 * c];
      ch[4 * c + 1] = charge_xyz[3 * c + 1];
      ch[4 * c + 2] = charge_xyz[3 * c + 2];
      ch[4 * c + 3] = charge_q[c];
    }
    if ((size_t)nc > engine->charges_cap) {
      LAI_CUDA_TRY(cudaStreamSynchronize(s));
      LAI_CUDA_TRY(engine->d_1e_charges.alloc(sizeof(double) * ch.size()));
      engine->charges_cap = nc;
    }
    LAI_CUDA_TRY(cudaMemcpyAsync(engine->d_1e_charges.p, ch.data(), sizeof(double) * ch.size(),
                                 cudaMemcpyHostToDevice, s));
    // the host staging vector dies here: make sure the copy has consumed it
    LAI_CUDA_TRY(cudaStreamSynchronize(s));
  }
  lai::OneEArgs g;
  g.shells = engine->d_1e_shell.as<lai::OneEShell>();
  g.exps = engine->d_1e_exp.as<double>();
  g.coefs = engine->d_1e_coef.as<double>();
  g.charges = engine->d_1e_charges.as<double>();
  g.ncharge = nc;
  g.nbf = engine->basis->nbf;
  g.out = d_out;
  g.tab = engine->tab;
  const int2* pairs = engine->d_1e_pairs.as<int2>();
  const auto& m = engine->one_e_class;
  // T + V: the kinetic pass writes every element, the nuclear pass adds to it
  const int ops[2] = {op == LAI_OP_HCORE ? LAI_OP_KINETIC : op, LAI_OP_NUCLEAR};
  for (int pass = 0; pass < (op == LAI_OP_HCORE ? 2 : 1); ++pass) {
    g.add = pass;
    for (size_t k = 0; k < m.size(); k += 4) {
      if (lai::launch_class(m[k], m[k + 1], ops[pass], g, pairs + m[k + 2], m[k + 3], s) < 0)
        return fail(LAI_ENOTSUP, "lai_one_electron: class not supported");
    }
  }
  LAI_CUDA_TRY(cudaGetLastError());
  return LAI_OK;
}

int lai_one_electron(lai_engine* engine, int op, int ncharge, const double* charge_xyz,
                     const double* charge_q, double* out) {
  if (!engine || !out) return fail(LAI_EINVAL, "lai_one_electron: null argument");
  LAI_CUDA_TRY(cudaSetDevice(engine->device));
  const size_t bytes = sizeof(double) * engine->basis->nbf * engine->basis->nbf;
  DevBuf d;
  LAI_CUDA_TRY(d.alloc(bytes));
  cudaStream_t s = engine->stream;
  if (int rc = lai_one_electron_device(engine, op, ncharge, charge_xyz, charge_q, d.as<double>(), s)) return rc;
  LAI_CUDA_TRY(cudaMemcpyAsync(out, d.p, bytes, cudaMemcpyDeviceToHost, s));
  LAI_CUDA_TRY(cudaStreamSynchronize(s));
  return LAI_OK;
}

}  // extern "C"
