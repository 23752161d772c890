// J/K build that performs no device allocation at call time.
//
// Who needs it: hosts that cannot call cudaMalloc when they ask for J and K --
// plugins living in an application that reserves the whole device up front for
// its own pool allocator (a cudaMalloc there fails or steals the pool's memory),
// and real-time drivers that forbid allocation once initialised (an allocation
// can synchronize the device and take unbounded time).  lai_jk_build_device() allocates its two nbf x nbf
// accumulators on first use; this variant keeps them instead in a fixed array in
// the library's device image, so the call itself allocates nothing.  The caller
// still owns D, J and K, and the engine (created earlier with lai_engine_create,
// which does allocate).
//
// Limits and rules (also in include/libaccint_b200.h):
//   * nbf <= LAI_NOALLOC_MAX_NBF (512): the array holds 2 x 512 x 512 doubles
//     (4 MiB), resident on every GPU that loads the library until the process ends;
//   * all calls share the array: calls whose device work overlaps (different
//     streams, or different engines on one device) race; serialize them;
//   * the first call on a device looks up the array's device address (host code
//     only sees a host-side stand-in for it); make that first call before any
//     stream capture.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/libaccint_b200.h"
#include "eri_kernels.h"

namespace lai {
int engine_device(const lai_engine* E);
int engine_num_sms(const lai_engine* E);
int engine_nbf(const lai_engine* E);
int engine_nsys(const lai_engine* E);
double engine_prim_eps(const lai_engine* E);
RysTablesView engine_tables(const lai_engine* E);
int engine_block_count(const lai_engine* E);
QuartetBlock engine_block(const lai_engine* E, int i);
void engine_set_error(const char* msg);
}  // namespace lai

namespace {

constexpr int kMaxNbf = LAI_NOALLOC_MAX_NBF;

// J' and K' accumulators: [0, nbf^2) and [nbf^2, 2 nbf^2).
static __device__ __align__(256) double g_noalloc_scratch[2 * (size_t)kMaxNbf * kMaxNbf];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mutex;
double* g_addr[kMaxDevices] = {nullptr};

__global__ void noalloc_symmetrize(const double* __restrict__ Jp, const double* __restrict__ Kp,
                                   double* __restrict__ J, double* __restrict__ K, int n) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * n) return;
  const int i = (int)(idx / n), j = (int)(idx - (int64_t)i * n);
  const int64_t tr = (int64_t)j * n + i;
  J[idx] = Jp[idx] + Jp[tr];
  K[idx] = Kp[idx] + Kp[tr];
}

int err(int code, const char* msg) {
  lai::engine_set_error(msg);
  return code;
}

}  // namespace

extern "C" int lai_jk_build_noalloc(lai_engine* engine, const double* d_D, double* d_J,
                                    double* d_K, void* stream) {
  if (!engine || !d_D || !d_J || !d_K) return err(LAI_EINVAL, "lai_jk_build_noalloc: null argument");
  if (lai::engine_nsys(engine) > 1)
    return err(LAI_ENOTSUP, "lai_jk_build_noalloc: not available for a batched engine");
  const int nbf = lai::engine_nbf(engine);
  if (nbf > kMaxNbf)
    return err(LAI_EINVAL, "lai_jk_build_noalloc: nbf exceeds LAI_NOALLOC_MAX_NBF (512); "
                           "use lai_jk_build_device");
  const int dev = lai::engine_device(engine);
  if (dev < 0 || dev >= kMaxDevices) return err(LAI_EINVAL, "lai_jk_build_noalloc: device ordinal");
  if (cudaSetDevice(dev) != cudaSuccess) return err(LAI_ECUDA, "lai_jk_build_noalloc: cudaSetDevice");
  const int nb = lai::engine_block_count(engine);
  const int sms = lai::engine_num_sms(engine);
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
        return err(LAI_ECUDA, "lai_jk_build_noalloc: cudaGetSymbolAddress failed");
      g_addr[dev] = static_cast<double*>(p);
    }
    scratch = g_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t nn = (size_t)nbf * nbf;
  if (cudaMemsetAsync(scratch, 0, 2 * nn * sizeof(double), s) != cudaSuccess)
    return err(LAI_ECUDA, "lai_jk_build_noalloc: clearing the accumulators failed");
  lai::JKArgs args{};
  args.D = d_D;
  args.J = scratch;
  args.K = scratch + nn;
  args.nbf = nbf;
  args.mode = lai::MODE_JK;
  args.prim_eps = lai::engine_prim_eps(engine);
  const lai::RysTablesView tab = lai::engine_tables(engine);
  for (int b = 0; b < nb; ++b) {
    const lai::QuartetBlock q = lai::engine_block(engine, b);
    const int la = q.bra.la, lb = q.bra.lb, lc = q.ket.la, ld = q.ket.lb;
    int rc;
    if (lai::small_class_supported(la, lb, lc, ld))
      rc = lai::launch_small(q, args, tab, s, false, sms) == 1 ? 0 : -3;
    else if (lai::sliced_class_supported(la, lb, lc, ld))
      rc = lai::launch_sliced(q, args, tab, s, false, sms) == 1 ? 0 : -3;
    else
      rc = lai::launch_tiled(q, args, tab, s, sms);
    if (rc == -1) {  // launch_tiled only
      // the tiled kernel's shared-memory tables do not fit this class; the
      // allocating entry point would fall back to the generic kernel, which needs
      // global scratch memory
      char msg[160];
      snprintf(msg, sizeof msg,
               "lai_jk_build_noalloc: class (%c%c|%c%c) does not fit the tiled kernel's shared "
               "memory; use lai_jk_build_device", "spdfghik"[la], "spdfghik"[lb], "spdfghik"[lc],
               "spdfghik"[ld]);
      return err(LAI_ENOTSUP, msg);
    }
    if (rc < 0) return err(LAI_ECUDA, "lai_jk_build_noalloc: kernel launch failed");
  }
  if (nn > 0)
    noalloc_symmetrize<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(scratch, scratch + nn, d_J, d_K, nbf);
  if (cudaGetLastError() != cudaSuccess) return err(LAI_ECUDA, "lai_jk_build_noalloc: launch failed");
  return LAI_OK;
}
