// Nuclear gradient of the two-electron energy E = 1/2 tr(D J) - 1/4 tr(D K) at
// fixed density over the engine's screened canonical quartets (the quartets the
// J/K build computes), and the C ABI around it.  dE/dD = J - K/2 comes from the
// J/K build itself.  No counterpart in the reference (MAX_DERIVATIVE_ORDER = 0,
// config.hpp.in:49).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "engine_internal.h"
#include "eri_kernels.h"

using namespace lai::host;

namespace {

int ensure_atoms(lai_engine* E) {
  if (E->natom >= 0) return LAI_OK;
  const auto& sh = E->basis->shells;
  std::vector<int> at(sh.size());
  int natom = 0;
  for (size_t s = 0; s < sh.size(); ++s) {
    if (sh[s].atom < 0) return fail(LAI_EINVAL, "gradient: the basis was created without atom indices");
    at[s] = sh[s].atom;
    natom = std::max(natom, sh[s].atom + 1);
  }
  LAI_CUDA_TRY(upload(E->d_shell_atom, at));
  E->natom = natom;
  return LAI_OK;
}

}  // namespace

extern "C" {

int lai_engine_natom(lai_engine* engine) {
  if (!engine) return fail(LAI_EINVAL, "lai_engine_natom: null engine");
  LAI_CUDA_TRY(cudaSetDevice(engine->device));
  if (int rc = ensure_atoms(engine)) return rc;
  return engine->natom;
}

int lai_jk_gradient_device(lai_engine* engine, const double* d_D, double* d_grad, void* stream) {
  if (engine && engine->nsys > 1) return fail(LAI_ENOTSUP, "lai_jk_gradient: not available for a batched engine");
  if (!engine || !d_D || !d_grad) return fail(LAI_EINVAL, "lai_jk_gradient_device: null argument");
  LAI_CUDA_TRY(cudaSetDevice(engine->device));
  if (int rc = ensure_atoms(engine)) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  LAI_CUDA_TRY(cudaMemsetAsync(d_grad, 0, sizeof(double) * 3 * engine->natom, s));
  const int nbf = (int)engine->basis->nbf;
  for (const auto& bp : engine->blocks) {
    const lai::QuartetBlock q = make_block(engine, *bp);
    const int rs = lai::launch_grad_small(q, d_D, nbf, engine->d_shell_atom.as<int>(), d_grad, engine->prim_eps,
                                          engine->tab, s, engine->num_sms);
    if (rs == 0) continue;
    if (rs != -1)
      return fail(LAI_ECUDA, std::string("gradient launch failed: ") + cudaGetErrorString(cudaGetLastError()));
    const size_t need = lai::grad_global_scratch_doubles(q.bra.la, q.bra.lb, q.ket.la, q.ket.lb,
                                                         engine->num_sms);
    if (int rc = ensure_scratch(engine, need)) return rc;
    const int rc = lai::launch_grad(q, d_D, nbf, engine->d_shell_atom.as<int>(), d_grad, engine->prim_eps,
                                    engine->tab, s, engine->d_scratch.as<double>(), engine->scratch_doubles,
                                    engine->num_sms);
    if (rc < 0)
      return fail(LAI_ECUDA, std::string("gradient launch failed: ") + cudaGetErrorString(cudaGetLastError()));
  }
  return LAI_OK;
}

int lai_jk_gradient(lai_engine* engine, const double* D, size_t nbf, double* grad) {
  if (!engine || !D || !grad) return fail(LAI_EINVAL, "lai_jk_gradient: null argument");
  if ((long)nbf != engine->basis->nbf) return fail(LAI_EINVAL, "lai_jk_gradient: nbf mismatch");
  LAI_CUDA_TRY(cudaSetDevice(engine->device));
  if (int rc = ensure_atoms(engine)) return rc;
  const size_t bytes = sizeof(double) * nbf * nbf;
  DevBuf dD, dG;
  LAI_CUDA_TRY(dD.alloc(bytes));
  LAI_CUDA_TRY(dG.alloc(sizeof(double) * 3 * engine->natom));
  cudaStream_t s = engine->stream;
  LAI_CUDA_TRY(cudaMemcpyAsync(dD.p, D, bytes, cudaMemcpyHostToDevice, s));
  if (int rc = lai_jk_gradient_device(engine, dD.as<double>(), dG.as<double>(), s)) return rc;
  LAI_CUDA_TRY(cudaMemcpyAsync(grad, dG.p, sizeof(double) * 3 * engine->natom, cudaMemcpyDeviceToHost, s));
  LAI_CUDA_TRY(cudaStreamSynchronize(s));
  return LAI_OK;
}

}  // extern "C"
