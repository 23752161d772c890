// Launch entry points of the ERI/J-K kernels (host side).
#pragma once

#include <cuda_runtime.h>

#include "eri_device.cuh"

namespace lai {

// Thread-per-quartet kernels for the small classes (eri_small.cu).  Returns 1 if
// the class (la,lb|lc,ld) has a specialised kernel and it was launched, 0 if the
// class is not covered (use the generic kernel), <0 on a launch error.
// Launch parameters of the thread-per-quartet kernels chosen by the autotuner
// (lai_engine_autotune); 0 = the built-in heuristic.  ps = lanes per quartet
// (primitive split, power of two), ksuper = chunks per super-chunk.
struct LaunchTune {
  int ps = 0;
  int ksuper = 0;
  int kernel = 0;  // classes outside the thread-per-quartet set: 0 = default choice,
                   // KERNEL_WARPQ, KERNEL_TILED or KERNEL_SLICED
};
enum { KERNEL_DEFAULT = 0, KERNEL_WARPQ = 1, KERNEL_TILED = 2, KERNEL_SLICED = 3 };
int launch_small(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab,
                 cudaStream_t stream, bool fp32, int num_sms, LaunchTune tune = LaunchTune{});
bool small_class_supported(int la, int lb, int lc, int ld);

// Bra-sliced kernels for the medium classes (eri_sliced.cu); same return codes.
int launch_sliced(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab,
                  cudaStream_t stream, bool fp32, int num_sms);
bool sliced_class_supported(int la, int lb, int lc, int ld);

// Warp-per-quartet kernel with lanes over the output integrals (eri_tiled.cu),
// any class with l <= 4; 0 on success, -1 if the class does not fit shared memory.
// Warp-per-quartet kernel compile-time specialised per class (J/K mode only).
// Returns 0 when launched in FP64, 1 when fp32 asked for and got the FP32 variant
// (d and f classes), -1 when the class is not instantiated (or the mode is not
// J/K), < -1 on a CUDA error.
int launch_warpq(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab, cudaStream_t stream,
                 int num_sms, bool fp32 = false);
cudaError_t warpq_launch_error();  // CUDA error of the last failed launch_warpq
bool warpq_class_supported(int la, int lb, int lc, int ld);
// Kernel family of a class outside the thread-per-quartet set when no tuned choice
// exists (measured per class on B200: eri_warpq.cu).
int default_kernel(int la, int lb, int lc, int ld);
int launch_tiled(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab, cudaStream_t stream,
                 int num_sms);

// Warp-per-quartet generic kernel (eri_generic.cu), any class with l <= 4.
int launch_generic(const QuartetBlock& blk, const JKArgs& args, const RysTablesView& tab,
                   cudaStream_t stream, double* gscratch, size_t gscratch_doubles, int num_sms);
// Global scratch (doubles) the generic kernel needs for class (la,lb|lc,ld) when
// its (e0|f0) block does not fit in shared memory; 0 if it fits.
size_t generic_global_scratch_doubles(int la, int lb, int lc, int ld, int num_sms);

// Nuclear-gradient kernel (eri_grad.cu): adds dE/dR of the block's quartets to
// grad[natom][3] (E = 1/2 tr DJ - 1/4 tr DK at fixed D).  0 on success.
int launch_grad(const QuartetBlock& blk, const double* D, int nbf, const int* shell_atom, double* grad,
                double prim_eps, const RysTablesView& tab, cudaStream_t stream, double* gscratch,
                size_t gscratch_doubles, int num_sms);
size_t grad_global_scratch_doubles(int la, int lb, int lc, int ld, int num_sms);
// Thread-per-quartet gradient kernels for the low classes (eri_grad_small.cu): 0 when
// launched, -1 when the class is not covered (use launch_grad), -3 on a CUDA error.
int launch_grad_small(const QuartetBlock& blk, const double* D, int nbf, const int* shell_atom, double* grad,
                      double prim_eps, const RysTablesView& tab, cudaStream_t stream, int num_sms);
bool grad_small_supported(int la, int lb, int lc, int ld);

}  // namespace lai
