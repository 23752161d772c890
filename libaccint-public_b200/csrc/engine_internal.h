// Host-side types shared by the translation units of the engine: device buffers,
// shells and bases, pair classes, quartet blocks and the engine object behind the
// opaque C handles of include/libaccint_b200.h.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../../include/libaccint_b200.h"
#include "eri_device.cuh"
#include "eri_kernels.h"

namespace lai {
namespace host {

// Records msg as the thread's last error (lai_last_error) and returns code.
int fail(int code, const std::string& msg);

#define LAI_CUDA_TRY(expr)                                                              \
  do {                                                                                  \
    cudaError_t e_ = (expr);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail(e_ == cudaErrorMemoryAllocation ? LAI_ENOMEM : LAI_ECUDA,             \
                  std::string(#expr) + ": " + cudaGetErrorString(e_));                  \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { if (p) cudaFree(p); }
  cudaError_t alloc(size_t n) {
    if (p) { cudaFree(p); p = nullptr; }
    bytes = n;
    if (n == 0) return cudaSuccess;
    return cudaMalloc(&p, n);
  }
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

template <typename T>
cudaError_t upload(DevBuf& b, const std::vector<T>& v) {
  cudaError_t e = b.alloc(v.size() * sizeof(T));
  if (e != cudaSuccess || v.empty()) return e;
  return cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

}  // namespace host
}  // namespace lai

// ---------------------------------------------------------------------------
// Basis
// ---------------------------------------------------------------------------
struct HostShell {
  int l;
  double center[3];
  std::vector<double> exps_all, coefs_all;  // normalized, all primitives as given
  std::vector<double> exps, coefs;          // nonzero-coefficient primitives only
  int atom;
  long func;     // first function of the shell within its system
  int sys = 0;   // system index (batched engines merge independent systems)
};

struct lai_basis {
  std::vector<HostShell> shells;
  long nbf = 0;
};

namespace lai {
namespace host {

struct PairClassHost {
  int la, lb, Ka, Kb;
  double qprim_max = 0.0;
  std::vector<int> sa, sb, fa, fb;  // shell and function indices (oriented)
  std::vector<int> sys;             // system of each pair (batched engines)
  std::vector<int> seg;             // [nsys + 1] first pair of each system (pairs sorted by system)
  std::vector<double> Q;
  std::vector<double> AB;          // SoA [3][n]
  std::vector<double> Acen;        // SoA [3][n] centre of the first shell (a)
  std::vector<double> prim;        // SoA [PF_COUNT][Kab][n]
  int n() const { return (int)sa.size(); }
  // device copies
  DevBuf d_sa, d_sb, d_fa, d_fb, d_Q, d_AB, d_Acen, d_prim, d_sys, d_primf, d_primb, d_primbf, d_primk,
      d_primkf;
  bool batched = false;             // d_sys is set (more than one system)
  lai::PairClassDev view() const {
    lai::PairClassDev v;
    v.la = la; v.lb = lb; v.Ka = Ka; v.Kb = Kb; v.npairs = n();
    v.shell_a = d_sa.as<int>(); v.shell_b = d_sb.as<int>();
    v.func_a = d_fa.as<int>(); v.func_b = d_fb.as<int>();
    v.Q = d_Q.as<double>(); v.AB = d_AB.as<double>(); v.Acen = d_Acen.as<double>();
    v.prim = d_prim.as<double>();
    v.qprim_max = qprim_max;
    v.sys = batched ? d_sys.as<int>() : nullptr;
    v.primf = d_primf.as<float>();
    v.primb = d_primb.as<double>();
    v.primbf = d_primbf.as<float>();
    v.primk = d_primk.as<double>();
    v.primkf = d_primkf.as<float>();
    return v;
  }
};

struct ClassPairBlock {
  int bra, ket;                 // class indices, bra >= ket
  std::vector<int64_t> offsets; // host copy
  DevBuf d_offsets;
  std::vector<int> qbegin;      // first ket of each bra pair (batched engines: its system's segment)
  DevBuf d_qbegin;              // empty for a single system (every ket range starts at 0)
  int64_t total = 0;
  double alg_flops = 0;         // per quartet of this block (all nonzero primitives)
  double flops_per_prim = 0;    // per primitive quartet
  double flops_per_quartet = 0; // per contracted quartet (normalization + digestion)
  // Mixed-precision split of this block for one FP32 cut: the kets of bra pair p
  // are sorted by Schwarz bound, so those with Q_p Q_q >= cut form a prefix (the
  // FP64 part, offsets64) and the rest a suffix (the FP32 part: offsets32, with
  // qbegin32[p] its first ket).
  int64_t total64 = 0, total32 = 0;
  DevBuf d_off64, d_off32, d_qb32;

  lai::LaunchTune tune;         // launch parameters chosen by lai_engine_autotune (0 = heuristic)
};

}  // namespace host
}  // namespace lai

struct lai_engine {
  const lai_basis* basis = nullptr;
  // batched engines: the merged basis (owned) and the per-system layout of the
  // packed D/J/K arrays (block s = nbf_s x nbf_s at element offset sys_off[s])
  std::unique_ptr<lai_basis> merged;
  int nsys = 1;
  std::vector<int> sys_nbf;
  std::vector<int64_t> sys_off;   // [nsys + 1]
  lai::host::DevBuf d_sys_nbf, d_sys_off;
  int device = 0;
  int num_sms = 148;
  double thr = 1e-12;
  double prim_eps = 1e-15;
  cudaStream_t stream = nullptr;
  lai::host::DevBuf d_coef, d_hx2, d_hw, d_boys, d_boys_f32, d_rys_f32;
  lai::RysTablesView tab{};
  std::vector<std::unique_ptr<lai::host::PairClassHost>> classes;
  std::vector<std::unique_ptr<lai::host::ClassPairBlock>> blocks;
  std::vector<double> Q_all;     // nshell x nshell Schwarz matrix
  lai::host::DevBuf d_Jp, d_Kp, d_D, d_J, d_K;
  lai::host::DevBuf d_scratch;
  size_t scratch_doubles = 0;
  lai::host::DevBuf d_status;
  double split_cut = -1.0;       // FP32 cut the blocks' mixed-precision split was built for
  lai::host::DevBuf d_absmax;
  lai::host::DevBuf d_shell_atom;  // [nshell] atom of each shell (gradients)
  int natom = -1;
  // one-electron integrals: shell table, primitives and shell pairs grouped by
  // (la, lb) class (built on first use; one_electron.cu)
  lai::host::DevBuf d_1e_shell, d_1e_exp, d_1e_coef, d_1e_pairs, d_1e_charges;
  std::vector<int> one_e_class;    // per class: la, lb, first pair, pair count
  size_t charges_cap = 0;
  // CUDA graph of one device build (lai_jk_opts.graph) and what it was captured for
  struct GraphKey {
    const double* D;
    double* J;
    double* K;
    cudaStream_t stream;
    double fp32_cut;
    int shard_index, shard_count;
    double fp32_prim_rel;
    bool operator==(const GraphKey& o) const {
      return D == o.D && J == o.J && K == o.K && stream == o.stream && fp32_cut == o.fp32_cut &&
             shard_index == o.shard_index && shard_count == o.shard_count && fp32_prim_rel == o.fp32_prim_rel;
    }
  };
  cudaGraphExec_t graph_exec = nullptr;
  GraphKey graph_key{};
  lai_jk_report graph_report{};
  void release_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    graph_exec = nullptr;
  }
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // per-launch profile of the last build with opts.profile
  std::vector<cudaEvent_t> prof_ev;
  std::vector<int> prof_block;
  std::vector<int64_t> prof_quartets;
  lai::host::DevBuf d_prof_prims;
  int prof_n = 0;
  ~lai_engine() {
    release_graph();
    for (auto e : prof_ev) cudaEventDestroy(e);
    classes.clear();
    blocks.clear();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace lai {
namespace host {

// Implemented in engine.cu.
void fill_pair_data(const lai_basis* basis, PairClassHost& c);
int upload_class(PairClassHost& c);
int launch_block(lai_engine* E, const lai::QuartetBlock& blk, const lai::JKArgs& args,
                 bool fp32 = false, bool* ran_fp32 = nullptr, lai::LaunchTune tune = lai::LaunchTune{});
lai::QuartetBlock make_block(const lai_engine* E, const ClassPairBlock& b);
int ensure_scratch(lai_engine* E, size_t doubles);
double alg_work(int la, int lb, int lc, int ld, int Ka, int Kb, int Kc, int Kd);

}  // namespace host
}  // namespace lai
