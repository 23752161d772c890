// C ABI of the density-fitting integrals: three-centre (mu nu|P) over the
// engine's orbital basis and an auxiliary basis, two-centre (P|Q) over the
// auxiliary basis (kernels in eri3c_impl.cuh).  Shell tables and pair lists are
// staged in stream-ordered device memory (cudaMallocAsync / cudaFreeAsync), so the
// device variants stay asynchronous.
#include <cuda_runtime.h>

#include <vector>

#include "engine_internal.h"
#include "eri3c_impl.cuh"

using namespace lai::host;

namespace {

int launch_class(int la, int lb, int lp, const lai::Eri3cArgs& g, cudaStream_t s) {
  if (la <= 1) return lai::launch_eri3c_l01(la, lb, lp, g, s);
  if (la == 2) return lai::launch_eri3c_l2(la, lb, lp, g, s);
  if (la == 3) return lai::launch_eri3c_l3(la, lb, lp, g, s);
  return lai::launch_eri3c_l4(la, lb, lp, g, s);
}

template <typename T>
cudaError_t stage(const std::vector<T>& h, T** d, cudaStream_t s) {
  *d = nullptr;
  if (h.empty()) return cudaSuccess;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(d), sizeof(T) * h.size(), s);
  if (e != cudaSuccess) return e;
  return cudaMemcpyAsync(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s);
}

// Orbital shells [0, norb), auxiliary shells [norb, norb + naux), the unit shell last.
int run(lai_engine* E, const lai_basis* aux, double* d_out, cudaStream_t s, bool two_center) {
  if (!E || !aux || !d_out) return fail(LAI_EINVAL, "density-fitting integrals: null argument");
  if (E->nsys > 1) return fail(LAI_ENOTSUP, "density-fitting integrals: not available for a batched engine");
  LAI_CUDA_TRY(cudaSetDevice(E->device));
  const auto& orb = E->basis->shells;
  const auto& ax = aux->shells;
  std::vector<lai::Eri3cShell> tab;
  std::vector<double> ex, co;
  auto add = [&](const HostShell& sh) {
    tab.push_back({sh.center[0], sh.center[1], sh.center[2], sh.l, (int)sh.exps.size(), (int)ex.size(),
                   (int)sh.func});
    ex.insert(ex.end(), sh.exps.begin(), sh.exps.end());
    co.insert(co.end(), sh.coefs.begin(), sh.coefs.end());
  };
  const int norb = (int)orb.size(), naux = (int)ax.size();
  for (const auto& sh : orb) add(sh);
  for (const auto& sh : ax) {
    if (sh.l > 4) return fail(LAI_ENOTSUP, "density-fitting integrals: auxiliary shells up to l = 4");
    add(sh);
  }
  const int unit = (int)tab.size();
  tab.push_back({0.0, 0.0, 0.0, 0, 1, (int)ex.size(), 0});
  ex.push_back(0.0);
  co.push_back(1.0);
  // bra pairs by (la, lb) class, la >= lb
  std::vector<std::vector<int2>> cls(25);
  if (two_center) {
    for (int p = 0; p < naux; ++p) cls[ax[p].l * 5].push_back(make_int2(norb + p, unit));
  } else {
    for (int i = 0; i < norb; ++i)
      for (int j = 0; j <= i; ++j) {
        int a = i, b = j;
        if (orb[a].l < orb[b].l) std::swap(a, b);
        const int la = orb[a].l, lb = orb[b].l;
        if (la > 4 || lb > 3 || (la == 4 && lb > 0))
          return fail(LAI_ENOTSUP, "density-fitting integrals: orbital shell pair class not supported "
                                   "(orbital shells up to f, g only with s)");
        cls[la * 5 + lb].push_back(make_int2(a, b));
      }
  }
  std::vector<std::vector<int>> auxl(5);
  for (int p = 0; p < naux; ++p) auxl[ax[p].l].push_back(norb + p);
  std::vector<int2> pairs;
  std::vector<int> pmeta;  // per class: la, lb, first, count
  for (int k = 0; k < 25; ++k)
    if (!cls[k].empty()) {
      pmeta.insert(pmeta.end(), {k / 5, k % 5, (int)pairs.size(), (int)cls[k].size()});
      pairs.insert(pairs.end(), cls[k].begin(), cls[k].end());
    }
  std::vector<int> auxs;
  int aoff[6] = {0};
  for (int l = 0; l < 5; ++l) {
    aoff[l] = (int)auxs.size();
    auxs.insert(auxs.end(), auxl[l].begin(), auxl[l].end());
  }
  aoff[5] = (int)auxs.size();

  lai::Eri3cShell* d_tab = nullptr;
  double *d_ex = nullptr, *d_co = nullptr;
  int2* d_pairs = nullptr;
  int* d_aux = nullptr;
  int rc = LAI_OK;
  cudaError_t e = stage(tab, &d_tab, s);
  if (e == cudaSuccess) e = stage(ex, &d_ex, s);
  if (e == cudaSuccess) e = stage(co, &d_co, s);
  if (e == cudaSuccess) e = stage(pairs, &d_pairs, s);
  if (e == cudaSuccess) e = stage(auxs, &d_aux, s);
  if (e == cudaSuccess) {
    lai::Eri3cArgs g{};
    g.shells = d_tab;
    g.exps = d_ex;
    g.coefs = d_co;
    g.out = d_out;
    g.nbf = two_center ? aux->nbf : E->basis->nbf;
    g.naux = aux->nbf;
    g.two_center = two_center ? 1 : 0;
    g.tab = E->tab;
    for (size_t k = 0; k < pmeta.size() && rc == LAI_OK; k += 4)
      for (int lp = 0; lp < 5 && rc == LAI_OK; ++lp) {
        if (aoff[lp + 1] == aoff[lp]) continue;
        g.pairs = d_pairs + pmeta[k + 2];
        g.npairs = pmeta[k + 3];
        g.aux = d_aux + aoff[lp];
        g.naux_shells = aoff[lp + 1] - aoff[lp];
        if (launch_class(pmeta[k], pmeta[k + 1], lp, g, s) < 0)
          rc = fail(LAI_ENOTSUP, "density-fitting integrals: class not instantiated");
      }
    e = cudaGetLastError();
  }
  // stream-ordered frees: the staged tables live until the kernels are done
  cudaFreeAsync(d_tab, s);
  cudaFreeAsync(d_ex, s);
  cudaFreeAsync(d_co, s);
  cudaFreeAsync(d_pairs, s);
  cudaFreeAsync(d_aux, s);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(LAI_ECUDA, std::string("density-fitting integrals: ") + cudaGetErrorString(e));
  return LAI_OK;
}

int run_host(lai_engine* E, const lai_basis* aux, double* out, bool two_center) {
  if (!E || !aux || !out) return fail(LAI_EINVAL, "density-fitting integrals: null argument");
  LAI_CUDA_TRY(cudaSetDevice(E->device));
  const size_t n = two_center ? (size_t)aux->nbf * aux->nbf
                              : (size_t)E->basis->nbf * E->basis->nbf * aux->nbf;
  DevBuf d;
  LAI_CUDA_TRY(d.alloc(sizeof(double) * n));
  cudaStream_t s = E->stream;
  if (int rc = run(E, aux, d.as<double>(), s, two_center)) return rc;
  LAI_CUDA_TRY(cudaMemcpyAsync(out, d.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  LAI_CUDA_TRY(cudaStreamSynchronize(s));
  return LAI_OK;
}

}  // namespace

extern "C" {

int lai_eri3c_device(lai_engine* engine, const lai_basis* aux, double* d_T, void* stream) {
  return run(engine, aux, d_T, static_cast<cudaStream_t>(stream), false);
}

int lai_eri2c_device(lai_engine* engine, const lai_basis* aux, double* d_V, void* stream) {
  return run(engine, aux, d_V, static_cast<cudaStream_t>(stream), true);
}

int lai_eri3c(lai_engine* engine, const lai_basis* aux, double* T) { return run_host(engine, aux, T, false); }

int lai_eri2c(lai_engine* engine, const lai_basis* aux, double* V) { return run_host(engine, aux, V, true); }

}  // extern "C"
