// Work-unit API: integrals and J/K contributions of a caller-supplied list of
// shell quartets, and digestion of an external integral batch.
//
// Reference counterparts:
//   * CudaEngine/CpuEngine::compute_shell_set_quartet(op, quartet, consumer,
//     canonical_symmetry) (include/libaccint/engine/cuda_engine.hpp:462-466,792-980;
//     cpu_engine.hpp:436-549): J/K from a given set of quartets, either plain
//     accumulation of exactly those (FockBuilder::accumulate,
//     src/shared/consumers/fock_builder.cpp:64-121) or, with canonical_symmetry,
//     each as the representative of its 8-fold permutation orbit
//     (accumulate_symmetric, fock_builder.cpp:123-222);
//   * Engine::compute_batch (include/libaccint/engine/engine.hpp:1008-1122): raw
//     norm-corrected Cartesian integrals of given quartets, [a][b][c][d];
//   * GpuFockBuilder::accumulate_device_eri_batch
//     (src/device/cuda/consumers/fock_builder_gpu.cu:600-621): plain J/K
//     accumulation of an integral batch already on the device.
//
// The listed quartets run through the same class-specialised kernels as the full
// build.  Each quartet is oriented like the engine's pairs (higher l first, then
// more primitives, then the higher shell index) and grouped by (bra class, ket
// class); a group is one launch over ad-hoc pair tables holding the group's bra
// pairs and ket pairs side by side (quartet t = bra pair t with ket pair t).
// Primitive screening is off (every primitive quartet is computed).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <map>
#include <memory>
#include <vector>

#include "engine_internal.h"
#include "eri_kernels.h"

using namespace lai::host;

namespace {

struct Oriented {
  int a, b, c, d;  // canonical shells: (ab| bra, |cd) ket
  int role[4];     // role[r] = canonical slot (0..3 for a,b,c,d) holding listed shell r (i,j,k,l)
};

std::array<int, 4> pair_key(const lai_basis* B, int a, int b) {
  const auto& A = B->shells[a];
  const auto& C = B->shells[b];
  return {A.l, C.l, (int)A.exps.size(), (int)C.exps.size()};
}

// Orientation of the engine's pair classes (engine.cu build_classes): a = the
// shell with higher l, then more nonzero primitives, then the higher index.
void orient_pair(const lai_basis* B, int x, int y, int& a, int& b, bool& swapped) {
  int hi = std::max(x, y), lo = std::min(x, y);
  const auto& H = B->shells[hi];
  const auto& L = B->shells[lo];
  if (L.l > H.l || (L.l == H.l && L.exps.size() > H.exps.size())) std::swap(hi, lo);
  a = hi;
  b = lo;
  swapped = (a != x);
}

Oriented orient(const lai_basis* B, const int32_t* q) {
  Oriented o;
  bool s1, s2;
  int a, b, c, d;
  orient_pair(B, q[0], q[1], a, b, s1);
  orient_pair(B, q[2], q[3], c, d, s2);
  // listed slots -> canonical slots before a bra/ket swap
  int ri = s1 ? 1 : 0, rj = s1 ? 0 : 1, rk = s2 ? 3 : 2, rl = s2 ? 2 : 3;
  if (pair_key(B, a, b) < pair_key(B, c, d)) {  // kernels take bra class >= ket class
    std::swap(a, c);
    std::swap(b, d);
    ri ^= 2; rj ^= 2; rk ^= 2; rl ^= 2;
  }
  o.a = a; o.b = b; o.c = c; o.d = d;
  o.role[0] = ri; o.role[1] = rj; o.role[2] = rk; o.role[3] = rl;
  return o;
}

struct Group {
  std::vector<int64_t> members;  // indices into the listed quartets
  std::unique_ptr<PairClassHost> bra, ket;
  DevBuf d_off, d_qb;
  int64_t out_offset = 0;  // first double of the group's canonical blocks
  int nval = 0;            // values per quartet
};

int build_groups(lai_engine* E, const int32_t* quartets, int64_t n, std::vector<Oriented>& ori,
                 std::vector<std::unique_ptr<Group>>& groups) {
  const lai_basis* B = E->basis;
  const int ns = (int)B->shells.size();
  ori.resize(n);
  std::map<std::array<int, 8>, size_t> gidx;
  for (int64_t t = 0; t < n; ++t) {
    const int32_t* q = quartets + 4 * t;
    for (int r = 0; r < 4; ++r)
      if (q[r] < 0 || q[r] >= ns) return fail(LAI_EINVAL, "quartet list: shell index out of range");
    ori[t] = orient(B, q);
    const auto kb = pair_key(B, ori[t].a, ori[t].b), kk = pair_key(B, ori[t].c, ori[t].d);
    const std::array<int, 8> key{kb[0], kb[1], kb[2], kb[3], kk[0], kk[1], kk[2], kk[3]};
    auto it = gidx.find(key);
    if (it == gidx.end()) {
      it = gidx.emplace(key, groups.size()).first;
      groups.push_back(std::make_unique<Group>());
    }
    groups[it->second]->members.push_back(t);
  }
  int64_t off = 0;
  for (auto& gp : groups) {
    Group& g = *gp;
    const int64_t m = (int64_t)g.members.size();
    g.bra = std::make_unique<PairClassHost>();
    g.ket = std::make_unique<PairClassHost>();
    const Oriented& o0 = ori[g.members[0]];
    const auto kb = pair_key(B, o0.a, o0.b), kk = pair_key(B, o0.c, o0.d);
    g.bra->la = kb[0]; g.bra->lb = kb[1]; g.bra->Ka = kb[2]; g.bra->Kb = kb[3];
    g.ket->la = kk[0]; g.ket->lb = kk[1]; g.ket->Ka = kk[2]; g.ket->Kb = kk[3];
    for (int64_t t : g.members) {
      const Oriented& o = ori[t];
      g.bra->sa.push_back(o.a); g.bra->sb.push_back(o.b);
      g.bra->fa.push_back((int)B->shells[o.a].func); g.bra->fb.push_back((int)B->shells[o.b].func);
      g.ket->sa.push_back(o.c); g.ket->sb.push_back(o.d);
      g.ket->fa.push_back((int)B->shells[o.c].func); g.ket->fb.push_back((int)B->shells[o.d].func);
    }
    for (PairClassHost* c : {g.bra.get(), g.ket.get()}) {
      fill_pair_data(B, *c);
      c->qprim_max = 0.0;  // with primitive screening off, the bounds are never read
      if (int rc = upload_class(*c)) return rc;
    }
    std::vector<int64_t> offs(m + 1);
    std::vector<int> qb(m);
    for (int64_t p = 0; p <= m; ++p) offs[p] = p;
    for (int64_t p = 0; p < m; ++p) qb[p] = (int)p;
    LAI_CUDA_TRY(upload(g.d_off, offs));
    LAI_CUDA_TRY(upload(g.d_qb, qb));
    g.nval = lai::ncart(kb[0]) * lai::ncart(kb[1]) * lai::ncart(kk[0]) * lai::ncart(kk[1]);
    g.out_offset = off;
    off += m * g.nval;
  }
  return LAI_OK;
}

lai::QuartetBlock group_block(const Group& g) {
  lai::QuartetBlock q{};
  q.bra = g.bra->view();
  q.ket = g.ket->view();
  q.offsets = g.d_off.as<int64_t>();
  q.qbegin = g.d_qb.as<int>();
  q.t_begin = 0;
  q.total = (int64_t)g.members.size();
  q.same_class = 0;
  return q;
}

// Canonical blocks of every group into d_out (group after group), on E->stream.
int run_raw(lai_engine* E, std::vector<std::unique_ptr<Group>>& groups, double* d_out, int* d_meta) {
  int64_t qoff = 0;
  for (auto& gp : groups) {
    lai::JKArgs args{};
    args.mode = lai::MODE_RAW;
    args.raw_out = d_out + gp->out_offset;
    args.raw_meta = d_meta + 4 * qoff;
    args.prim_eps = 0.0;
    if (int rc = launch_block(E, group_block(*gp), args)) return rc;
    qoff += (int64_t)gp->members.size();
  }
  return LAI_OK;
}

// Plain digestion: J[i][j] += (ij|kl) D[k][l], K[i][k] += (ij|kl) D[j][l] for every
// element of every block.  A warp per quartet; desc = {offset, f[4], n[4], role[4]}
// with the block stored [n0][n1][n2][n3] over functions f0.., and role[r] the slot
// holding listed index r (i, j, k, l).
struct DigestDesc {
  int64_t offset;
  int f[4], n[4], role[4];
};

__global__ void plain_digest_kernel(const double* __restrict__ eri, const DigestDesc* __restrict__ desc,
                                    int64_t nq, const double* __restrict__ D, double* __restrict__ J,
                                    double* __restrict__ K, int nbf) {
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= nq) return;
  const DigestDesc d = desc[w];
  const int n3 = d.n[3], n23 = d.n[2] * n3, n123 = d.n[1] * n23;
  const int total = d.n[0] * n123;
  for (int e = lane; e < total; e += 32) {
    const int x0 = e / n123, r1 = e - x0 * n123;
    const int x1 = r1 / n23, r2 = r1 - x1 * n23;
    const int x2 = r2 / n3, x3 = r2 - x2 * n3;
    const int idx[4] = {d.f[0] + x0, d.f[1] + x1, d.f[2] + x2, d.f[3] + x3};
    const int i = idx[d.role[0]], j = idx[d.role[1]], k = idx[d.role[2]], l = idx[d.role[3]];
    const double v = eri[d.offset + e];
    atomicAdd(J + (size_t)i * nbf + j, v * __ldg(D + (size_t)k * nbf + l));
    atomicAdd(K + (size_t)i * nbf + k, v * __ldg(D + (size_t)j * nbf + l));
  }
}

__global__ void add_symmetrized_kernel(const double* __restrict__ Jp, const double* __restrict__ Kp,
                                       double* __restrict__ J, double* __restrict__ K, int n) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)n * n) return;
  const int i = (int)(idx / n), j = (int)(idx - (int64_t)i * n);
  const int64_t tr = (int64_t)j * n + i;
  J[idx] += Jp[idx] + Jp[tr];
  K[idx] += Kp[idx] + Kp[tr];
}

int launch_plain_digest(const double* d_eri, const std::vector<DigestDesc>& desc, const double* d_D,
                        double* d_J, double* d_K, int nbf, cudaStream_t stream, DevBuf& d_desc) {
  if (desc.empty()) return LAI_OK;
  LAI_CUDA_TRY(d_desc.alloc(sizeof(DigestDesc) * desc.size()));
  LAI_CUDA_TRY(cudaMemcpyAsync(d_desc.p, desc.data(), sizeof(DigestDesc) * desc.size(),
                               cudaMemcpyHostToDevice, stream));
  const int64_t threads = 32 * (int64_t)desc.size();
  plain_digest_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, stream>>>(
      d_eri, d_desc.as<DigestDesc>(), (int64_t)desc.size(), d_D, d_J, d_K, nbf);
  LAI_CUDA_TRY(cudaGetLastError());
  // the descriptor buffer must outlive the kernel
  LAI_CUDA_TRY(cudaStreamSynchronize(stream));
  return LAI_OK;
}

struct StreamSwap {  // launch_block launches on E->stream
  lai_engine* E;
  cudaStream_t saved;
  StreamSwap(lai_engine* e, cudaStream_t s) : E(e), saved(e->stream) { E->stream = s; }
  ~StreamSwap() { E->stream = saved; }
};

// Values per listed quartet, its canonical-group position, and the total count.
int64_t listed_layout(const std::vector<std::unique_ptr<Group>>& groups, int64_t n,
                      std::vector<int64_t>& canon_off, std::vector<int>& nval) {
  canon_off.assign(n, 0);
  nval.assign(n, 0);
  int64_t tot = 0;
  for (auto& gp : groups)
    for (size_t r = 0; r < gp->members.size(); ++r) {
      const int64_t t = gp->members[r];
      canon_off[t] = gp->out_offset + (int64_t)r * gp->nval;
      nval[t] = gp->nval;
      tot += gp->nval;
    }
  return tot;
}

}  // namespace

extern "C" {

int lai_eri_quartets(lai_engine* engine, const int32_t* quartets, int64_t n, double* out,
                     size_t out_capacity, lai_quartet_meta* meta) {
  if (engine && engine->nsys > 1) return fail(LAI_ENOTSUP, "lai_eri_quartets: not available for a batched engine");
  if (!engine || n < 0 || (n > 0 && (!quartets || !out || !meta)))
    return fail(LAI_EINVAL, "lai_eri_quartets: null argument");
  if (n == 0) return LAI_OK;
  LAI_CUDA_TRY(cudaSetDevice(engine->device));
  std::vector<Oriented> ori;
  std::vector<std::unique_ptr<Group>> groups;
  if (int rc = build_groups(engine, quartets, n, ori, groups)) return rc;
  std::vector<int64_t> canon_off;
  std::vector<int> nval;
  const int64_t nv = listed_layout(groups, n, canon_off, nval);
  if ((int64_t)out_capacity < nv) return fail(LAI_EINVAL, "lai_eri_quartets: output capacity too small");
  DevBuf d_out, d_meta;
  LAI_CUDA_TRY(d_out.alloc(sizeof(double) * (size_t)nv));
  LAI_CUDA_TRY(d_meta.alloc(sizeof(int) * 4 * (size_t)n));
  std::vector<double> canon((size_t)nv);
  {
    StreamSwap sw(engine, engine->stream);
    if (int rc = run_raw(engine, groups, d_out.as<double>(), d_meta.as<int>())) return rc;
    LAI_CUDA_TRY(cudaMemcpyAsync(canon.data(), d_out.p, sizeof(double) * nv, cudaMemcpyDeviceToHost,
                                 engine->stream));
    LAI_CUDA_TRY(cudaStreamSynchronize(engine->stream));
  }
  // canonical [a][b][c][d] -> listed [i][j][k][l]
  const lai_basis* B = engine->basis;
  int64_t o = 0;
  for (int64_t t = 0; t < n; ++t) {
    const Oriented& r = ori[t];
    const int shells[4] = {r.a, r.b, r.c, r.d};
    int nc[4];
    for (int s = 0; s < 4; ++s) nc[s] = lai::ncart(B->shells[shells[s]].l);
    int nl[4];  // listed sizes
    for (int x = 0; x < 4; ++x) nl[x] = nc[r.role[x]];
    lai_quartet_meta& m = meta[t];
    m.offset = o;
    const int32_t* q = quartets + 4 * t;
    m.fa = (int32_t)B->shells[q[0]].func; m.fb = (int32_t)B->shells[q[1]].func;
    m.fc = (int32_t)B->shells[q[2]].func; m.fd = (int32_t)B->shells[q[3]].func;
    m.na = nl[0]; m.nb = nl[1]; m.nc = nl[2]; m.nd = nl[3];
    const double* src = canon.data() + canon_off[t];
    int x[4];
    for (x[0] = 0; x[0] < nl[0]; ++x[0])
      for (x[1] = 0; x[1] < nl[1]; ++x[1])
        for (x[2] = 0; x[2] < nl[2]; ++x[2])
          for (x[3] = 0; x[3] < nl[3]; ++x[3]) {
            int c[4];
            for (int s = 0; s < 4; ++s) c[r.role[s]] = x[s];
            out[o++] = src[((c[0] * nc[1] + c[1]) * nc[2] + c[2]) * nc[3] + c[3]];
          }
  }
  return LAI_OK;
}

int lai_jk_accumulate_quartets_device(lai_engine* engine, const int32_t* quartets, int64_t n,
                                      const double* d_D, double* d_J, double* d_K, void* stream,
                                      int canonical_symmetry) {
  if (engine && engine->nsys > 1) return fail(LAI_ENOTSUP, "lai_jk_accumulate_quartets: not available for a batched engine");
  if (!engine || n < 0 || (n > 0 && !quartets) || !d_D || !d_J || !d_K)
    return fail(LAI_EINVAL, "lai_jk_accumulate_quartets: null argument");
  if (n == 0) return LAI_OK;
  LAI_CUDA_TRY(cudaSetDevice(engine->device));
  std::vector<Oriented> ori;
  std::vector<std::unique_ptr<Group>> groups;
  if (int rc = build_groups(engine, quartets, n, ori, groups)) return rc;
  const int nbf = (int)engine->basis->nbf;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  StreamSwap sw(engine, s);
  if (canonical_symmetry) {
    const size_t bytes = sizeof(double) * (size_t)nbf * nbf;
    if (engine->d_Jp.bytes < bytes) {
      engine->release_graph();
      LAI_CUDA_TRY(engine->d_Jp.alloc(bytes));
      LAI_CUDA_TRY(engine->d_Kp.alloc(bytes));
    }
    LAI_CUDA_TRY(cudaMemsetAsync(engine->d_Jp.p, 0, bytes, s));
    LAI_CUDA_TRY(cudaMemsetAsync(engine->d_Kp.p, 0, bytes, s));
    lai::JKArgs args{};
    args.mode = lai::MODE_JK;
    args.D = d_D;
    args.J = engine->d_Jp.as<double>();
    args.K = engine->d_Kp.as<double>();
    args.nbf = nbf;
    args.prim_eps = 0.0;
    for (auto& gp : groups)
      if (int rc = launch_block(engine, group_block(*gp), args)) return rc;
    const int64_t nn = (int64_t)nbf * nbf;
    add_symmetrized_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, s>>>(
        engine->d_Jp.as<double>(), engine->d_Kp.as<double>(), d_J, d_K, nbf);
    LAI_CUDA_TRY(cudaGetLastError());
    // the ad-hoc pair tables are freed on return: wait for the kernels
    LAI_CUDA_TRY(cudaStreamSynchronize(s));
    return LAI_OK;
  }
  std::vector<int64_t> canon_off;
  std::vector<int> nval;
  const int64_t nv = listed_layout(groups, n, canon_off, nval);
  DevBuf d_out, d_meta, d_desc;
  LAI_CUDA_TRY(d_out.alloc(sizeof(double) * (size_t)nv));
  LAI_CUDA_TRY(d_meta.alloc(sizeof(int) * 4 * (size_t)n));
  if (int rc = run_raw(engine, groups, d_out.as<double>(), d_meta.as<int>())) return rc;
  std::vector<DigestDesc> desc(n);
  const lai_basis* B = engine->basis;
  for (int64_t t = 0; t < n; ++t) {
    const Oriented& r = ori[t];
    const int shells[4] = {r.a, r.b, r.c, r.d};
    DigestDesc& d = desc[t];
    d.offset = canon_off[t];
    for (int x = 0; x < 4; ++x) {
      d.f[x] = (int)B->shells[shells[x]].func;
      d.n[x] = lai::ncart(B->shells[shells[x]].l);
      d.role[x] = r.role[x];
    }
  }
  return launch_plain_digest(d_out.as<double>(), desc, d_D, d_J, d_K, nbf, s, d_desc);
}

int lai_jk_accumulate_quartets(lai_engine* engine, const int32_t* quartets, int64_t n, const double* D,
                               double* J, double* K, int canonical_symmetry) {
  if (!engine || !D || !J || !K) return fail(LAI_EINVAL, "lai_jk_accumulate_quartets: null argument");
  LAI_CUDA_TRY(cudaSetDevice(engine->device));
  const size_t nbf = (size_t)engine->basis->nbf;
  const size_t bytes = sizeof(double) * nbf * nbf;
  DevBuf dD, dJ, dK;
  LAI_CUDA_TRY(dD.alloc(bytes));
  LAI_CUDA_TRY(dJ.alloc(bytes));
  LAI_CUDA_TRY(dK.alloc(bytes));
  cudaStream_t s = engine->stream;
  LAI_CUDA_TRY(cudaMemcpyAsync(dD.p, D, bytes, cudaMemcpyHostToDevice, s));
  LAI_CUDA_TRY(cudaMemcpyAsync(dJ.p, J, bytes, cudaMemcpyHostToDevice, s));
  LAI_CUDA_TRY(cudaMemcpyAsync(dK.p, K, bytes, cudaMemcpyHostToDevice, s));
  if (int rc = lai_jk_accumulate_quartets_device(engine, quartets, n, dD.as<double>(), dJ.as<double>(),
                                                 dK.as<double>(), s, canonical_symmetry))
    return rc;
  LAI_CUDA_TRY(cudaMemcpyAsync(J, dJ.p, bytes, cudaMemcpyDeviceToHost, s));
  LAI_CUDA_TRY(cudaMemcpyAsync(K, dK.p, bytes, cudaMemcpyDeviceToHost, s));
  LAI_CUDA_TRY(cudaStreamSynchronize(s));
  return LAI_OK;
}

int lai_jk_accumulate_eri_batch_device(lai_engine* engine, const double* d_eri, const lai_quartet_meta* meta,
                                       int64_t n, const double* d_D, double* d_J, double* d_K,
                                       void* stream) {
  if (engine && engine->nsys > 1) return fail(LAI_ENOTSUP, "lai_jk_accumulate_eri_batch_device: not available for a batched engine");
  if (!engine || n < 0 || (n > 0 && (!d_eri || !meta)) || !d_D || !d_J || !d_K)
    return fail(LAI_EINVAL, "lai_jk_accumulate_eri_batch_device: null argument");
  if (n == 0) return LAI_OK;
  LAI_CUDA_TRY(cudaSetDevice(engine->device));
  const int nbf = (int)engine->basis->nbf;
  std::vector<DigestDesc> desc(n);
  for (int64_t t = 0; t < n; ++t) {
    const lai_quartet_meta& m = meta[t];
    const int f[4] = {m.fa, m.fb, m.fc, m.fd}, nn[4] = {m.na, m.nb, m.nc, m.nd};
    for (int x = 0; x < 4; ++x) {
      if (nn[x] < 1 || f[x] < 0 || f[x] + nn[x] > nbf)
        return fail(LAI_EINVAL, "lai_jk_accumulate_eri_batch_device: quartet meta out of range");
      desc[t].f[x] = f[x];
      desc[t].n[x] = nn[x];
      desc[t].role[x] = x;
    }
    desc[t].offset = m.offset;
  }
  DevBuf d_desc;
  return launch_plain_digest(d_eri, desc, d_D, d_J, d_K, nbf, static_cast<cudaStream_t>(stream), d_desc);
}

}  // extern "C"
