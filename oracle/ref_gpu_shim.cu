// Test infrastructure only: a C-ABI driver for the UNMODIFIED reference (LibAccInt)
// GPU route, compiled from the reference's own CUDA sources by `make -C oracle
// refgpu` into oracle/_ref/libref_gpu.so.  It measures the reference kernel on the
// same device as the product; nothing in the product links it.
//
// The route is the reference's correct GPU J/K: the four-set product of every
// ordered ShellSet 4-tuple, each through
//   - basis::upload_shell_set                  src/device/cuda/basis/device_data.cu:21-80
//   - device::math::boys_device_init           src/device/cuda/math/boys_device.cu:44-89
//   - kernels::cuda::launch_eri_kernel         src/device/cuda/kernels/eri_kernel.cu:635-689
//     (thread per shell quartet, integrals written to a device buffer)
//   - consumers::detail::launch_fock_accumulate_batch_kernel
//                                              src/device/cuda/consumers/fock_builder_gpu.cu:116-180
//     (plain J_mn += (mn|ls) D_ls, K_ml += (mn|ls) D_ns with FP64 atomics),
// so that the units together give the full J and K with no screening and no
// permutational symmetry.  Shells and sets come from the reference's own
// Shell / BasisSet constructors (src/shared/basis/shell.cpp:163-187,
// src/shared/basis/basis_set.cpp:21-29, 191-210).
#include <libaccint/basis/basis_set.hpp>
#include <libaccint/basis/device_data.hpp>
#include <libaccint/basis/shell.hpp>
#include <libaccint/basis/shell_set.hpp>
#include <libaccint/consumers/fock_builder_gpu.hpp>
#include <libaccint/kernels/eri_kernel_cuda.hpp>

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

namespace libaccint::device::math {
double* boys_device_init(cudaStream_t stream);  // src/device/cuda/math/boys_device.cuh:282
}

using namespace libaccint;

namespace {

thread_local char g_err[512] = {0};

void set_err(const std::string& msg) {
  std::strncpy(g_err, msg.c_str(), sizeof(g_err) - 1);
  g_err[sizeof(g_err) - 1] = 0;
}

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

struct GpuRefBasis {
  std::unique_ptr<BasisSet> basis;
};

// Device copies of every ShellSet of a basis, freed on scope exit.
struct UploadedSets {
  std::vector<basis::ShellSetDeviceData> sets;
  ~UploadedSets() {
    for (auto& s : sets) basis::free_shell_set_device_data(s);
  }
};

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  double* alloc(size_t n, const char* what) {
    check(cudaMalloc(&p, sizeof(double) * (n ? n : 1)), what);
    return static_cast<double*>(p);
  }
};

}  // namespace

extern "C" {

const char* refgpu_last_error() { return g_err; }

// Raw (un-normalized) contraction coefficients; the reference Shell constructor
// normalizes them.  Shells with l > 2 are rejected: this library is compiled with
// LIBACCINT_MAX_AM = 2 (the (H2O)n / STO-3G and cc-pVDZ workloads).
void* refgpu_basis_create(int nshell, const int* am, const int* nprim, const double* centers,
                          const double* exps, const double* coefs) {
  try {
    std::vector<Shell> shells;
    shells.reserve(nshell);
    long off = 0;
    for (int s = 0; s < nshell; ++s) {
      if (am[s] > 2) throw std::invalid_argument("refgpu: shells up to d only (built with LIBACCINT_MAX_AM = 2)");
      std::vector<Real> e(exps + off, exps + off + nprim[s]);
      std::vector<Real> c(coefs + off, coefs + off + nprim[s]);
      off += nprim[s];
      shells.emplace_back(am[s], Point3D(centers[3 * s], centers[3 * s + 1], centers[3 * s + 2]), std::move(e),
                          std::move(c));
    }
    auto* rb = new GpuRefBasis();
    rb->basis = std::make_unique<BasisSet>(std::move(shells));
    return rb;
  } catch (const std::exception& ex) {
    set_err(ex.what());
    return nullptr;
  }
}

void refgpu_basis_free(void* h) { delete static_cast<GpuRefBasis*>(h); }

long refgpu_nbf(void* h) { return (long)static_cast<GpuRefBasis*>(h)->basis->n_basis_functions(); }

// Number of ShellSets; the units are the nsets^4 ordered set 4-tuples, unit u =
// ((ia * nsets + ib) * nsets + ic) * nsets + id.
long refgpu_nsets(void* h) { return (long)static_cast<GpuRefBasis*>(h)->basis->shell_sets().size(); }

// Shell quartets and output doubles of unit u (host arithmetic, no device).
int refgpu_unit_size(void* h, long u, long* quartets, long* values) {
  const auto sets = static_cast<GpuRefBasis*>(h)->basis->shell_sets();
  const long n = (long)sets.size();
  if (u < 0 || u >= n * n * n * n) return -1;
  const long idx[4] = {u / (n * n * n), (u / (n * n)) % n, (u / n) % n, u % n};
  long q = 1, v = 1;
  for (long x : idx) {
    const ShellSet& s = *sets[x];
    q *= (long)s.n_shells();
    v *= (long)s.n_functions_per_shell();
  }
  *quartets = q;
  *values = q * v;
  return 0;
}

// Runs units [u_begin, u_end) on the current device: J and K (host, nbf x nbf)
// receive the plain accumulation of exactly those units (all units = the full J
// and K).  device_ms = CUDA-event time of the launches of the units (integral
// kernel + digestion), quartets = shell quartets computed.  Returns 0 or -1
// (refgpu_last_error()).
int refgpu_jk(void* h, const double* D, double* J, double* K, long u_begin, long u_end, double* device_ms,
              long* quartets) {
  try {
    BasisSet& B = *static_cast<GpuRefBasis*>(h)->basis;
    const auto sets = B.shell_sets();
    const long n = (long)sets.size();
    const long nbf = (long)B.n_basis_functions();
    if (u_begin < 0 || u_end > n * n * n * n || u_begin > u_end) throw std::invalid_argument("refgpu_jk: bad unit range");
    cudaStream_t stream = nullptr;
    check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "stream");
    struct StreamGuard {
      cudaStream_t s;
      ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{stream};
    UploadedSets up;
    for (const ShellSet* s : sets) up.sets.push_back(basis::upload_shell_set(*s, stream));
    const double* d_boys = device::math::boys_device_init(stream);
    long max_vals = 0;
    for (long u = u_begin; u < u_end; ++u) {
      long q = 0, v = 0;
      refgpu_unit_size(h, u, &q, &v);
      max_vals = std::max(max_vals, v);
    }
    DevBuf bD, bJ, bK, bE;
    double* d_D = bD.alloc((size_t)nbf * nbf, "D");
    double* d_J = bJ.alloc((size_t)nbf * nbf, "J");
    double* d_K = bK.alloc((size_t)nbf * nbf, "K");
    double* d_eri = bE.alloc((size_t)max_vals, "integral buffer");
    const size_t bytes = sizeof(double) * (size_t)nbf * nbf;
    check(cudaMemcpyAsync(d_D, D, bytes, cudaMemcpyHostToDevice, stream), "D upload");
    check(cudaMemsetAsync(d_J, 0, bytes, stream), "J clear");
    check(cudaMemsetAsync(d_K, 0, bytes, stream), "K clear");
    cudaEvent_t e0, e1;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    long nq = 0;
    check(cudaEventRecord(e0, stream), "event record");
    for (long u = u_begin; u < u_end; ++u) {
      const long idx[4] = {u / (n * n * n), (u / (n * n)) % n, (u / n) % n, u % n};
      basis::ShellSetQuartetDeviceData q{up.sets[idx[0]], up.sets[idx[1]], up.sets[idx[2]], up.sets[idx[3]]};
      kernels::cuda::launch_eri_kernel(q, d_boys, d_eri, stream);
      check(cudaGetLastError(), "launch_eri_kernel");
      consumers::detail::launch_fock_accumulate_batch_kernel(d_eri, q, d_D, d_J, d_K, (int)nbf, stream);
      check(cudaGetLastError(), "launch_fock_accumulate_batch_kernel");
      nq += (long)q.n_quartets();
    }
    check(cudaEventRecord(e1, stream), "event record");
    check(cudaMemcpyAsync(J, d_J, bytes, cudaMemcpyDeviceToHost, stream), "J download");
    check(cudaMemcpyAsync(K, d_K, bytes, cudaMemcpyDeviceToHost, stream), "K download");
    check(cudaStreamSynchronize(stream), "synchronize");
    float ms = 0.f;
    check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (device_ms) *device_ms = ms;
    if (quartets) *quartets = nq;
    return 0;
  } catch (const std::exception& ex) {
    set_err(ex.what());
    return -1;
  }
}

}  // extern "C"
