// Cartesian -> real-spherical (pure) transformation of the J/K path: the per-shell
// matrices C_l [2l+1 x (l+1)(l+2)/2] and their block-diagonal application to
// two-index quantities (J, K: T M T^T) and to the density (T^T D T), on the host
// and on the device.
//
// Reference counterparts: math::get_cart_to_sph_matrix and transform_2d
// (include/libaccint/math/spherical_transform.hpp:20-70,
// src/shared/math/spherical_transform.cpp), whose matrices are tabulated for
// l <= 4.  Here they are generated from the closed form of the real solid
// harmonics (Helgaker, Jorgensen, Olsen, Molecular Electronic-Structure Theory,
// eqs. 6.4.47-6.4.52):
//   S_lm = N_lm sum_{t,u,v} C^{lm}_{tuv} x^{2t+|m|-2(u+v)} y^{2(u+v)} z^{l-2t-|m|}
//   C^{lm}_{tuv} = (-1)^{t+v-v_m} (1/4)^t binom(l,t) binom(l-t,|m|+t) binom(t,u) binom(|m|,2v)
//   N_lm = sqrt(2 (l+|m|)! (l-|m|)! / 2^{delta_m0}) / (2^|m| l!)
// with v_m = 0 (m >= 0) or 1/2 (m < 0), in the reference's orders: spherical
// m = 0, 1, -1, 2, -2, ...; Cartesian lx descending, then ly descending.  The
// coefficients act on Cartesian functions that share the x^l normalization, the
// convention of the reference's tables (checked against them by the tests).
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/libaccint_b200.h"
#include "eri_device.cuh"

namespace lai {
int engine_device(const lai_engine* E);
const lai_basis* engine_basis(const lai_engine* E);
int engine_nsys(const lai_engine* E);
void engine_set_error(const char* msg);
}  // namespace lai

namespace {

constexpr int kMaxL = 4;

double binom_d(int n, int k) {
  if (k < 0 || k > n) return 0.0;
  double r = 1.0;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}
double fact_d(int n) {
  double r = 1.0;
  for (int i = 2; i <= n; ++i) r *= i;
  return r;
}

// Coefficient of x^lx y^ly z^lz in S_lm.
double solid_harmonic_coef(int l, int m, int lx, int ly, int lz) {
  const int am = std::abs(m);
  const int vm2 = m < 0 ? 1 : 0;  // 2 v_m
  const int tt = l - am - lz;     // 2t
  if (tt < 0 || (tt & 1)) return 0.0;
  const int t = tt / 2;
  if (2 * t + am - ly != lx) return 0.0;
  double s = 0.0;
  for (int u = 0; u <= t; ++u) {
    const int vv = ly - 2 * u;  // 2v
    if (vv < 0 || vv > am || ((vv - vm2) & 1)) continue;
    const int sgn = t + (vv - vm2) / 2;
    s += ((sgn & 1) ? -1.0 : 1.0) * std::pow(0.25, t) * binom_d(l, t) * binom_d(l - t, am + t) *
         binom_d(t, u) * binom_d(am, vv);
  }
  const double n = std::sqrt(2.0 * fact_d(l + am) * fact_d(l - am) / (m == 0 ? 2.0 : 1.0)) /
                   (std::pow(2.0, am) * fact_d(l));
  return n * s;
}

// m of the i-th spherical function: 0, 1, -1, 2, -2, ...
int sph_m(int i) { return i == 0 ? 0 : ((i & 1) ? (i + 1) / 2 : -(i / 2)); }

void fill_matrix(int l, double* C) {
  const int nc = lai::ncart(l);
  for (int i = 0; i < 2 * l + 1; ++i)
    for (int j = 0; j < nc; ++j) {
      const int c = lai::cart_comp(l, j);
      C[i * nc + j] = solid_harmonic_coef(l, sph_m(i), lai::comp_x(c), lai::comp_y(c), lai::comp_z(c));
    }
}

// Offsets of the matrices of l = 0..kMaxL in one concatenated array.
int mat_offset(int l) {
  int o = 0;
  for (int k = 0; k < l; ++k) o += (2 * k + 1) * lai::ncart(k);
  return o;
}
const std::vector<double>& all_matrices() {
  static std::vector<double> m = [] {
    std::vector<double> v(mat_offset(kMaxL + 1));
    for (int l = 0; l <= kMaxL; ++l) fill_matrix(l, v.data() + mat_offset(l));
    return v;
  }();
  return m;
}

int err(int code, const std::string& msg) {
  lai::engine_set_error(msg.c_str());
  return code;
}

// Per-function map of a basis: shell angular momentum, the shell's first
// Cartesian and spherical function, and the function's index inside its shell.
struct FuncMap {
  long ncart = 0, nsph = 0;
  std::vector<int> cart_l, cart_first_sph, cart_first_cart, cart_local;  // per Cartesian function
  std::vector<int> sph_l, sph_first_sph, sph_first_cart, sph_local;      // per spherical function
};

int build_map(const lai_basis* basis, FuncMap& f) {
  const int ns = lai_basis_nshell(basis);
  if (ns < 0) return err(LAI_EINVAL, "spherical transform: bad basis");
  long cc = 0, sc = 0;
  for (int s = 0; s < ns; ++s) {
    int l = 0, np = 0;
    double ctr[3];
    long func = 0;
    if (lai_basis_shell(basis, s, &l, &np, ctr, nullptr, nullptr, &func) != LAI_OK)
      return err(LAI_EINVAL, "spherical transform: bad shell");
    if (l > kMaxL) return err(LAI_ENOTSUP, "spherical transform: l > 4");
    if (func != cc) return err(LAI_EINVAL, "spherical transform: shells must be in function order");
    for (int j = 0; j < lai::ncart(l); ++j) {
      f.cart_l.push_back(l); f.cart_first_sph.push_back((int)sc);
      f.cart_first_cart.push_back((int)cc); f.cart_local.push_back(j);
    }
    for (int i = 0; i < 2 * l + 1; ++i) {
      f.sph_l.push_back(l); f.sph_first_sph.push_back((int)sc);
      f.sph_first_cart.push_back((int)cc); f.sph_local.push_back(i);
    }
    cc += lai::ncart(l);
    sc += 2 * l + 1;
  }
  f.ncart = cc;
  f.nsph = sc;
  return LAI_OK;
}

// ---- device ----------------------------------------------------------------
struct DevMap {
  int* sph = nullptr;   // [4][nsph]: l, first sph, first cart, local
  int* cart = nullptr;  // [4][ncart]
  double* mats = nullptr;
  long nsph = 0, ncart = 0;
};

__device__ __forceinline__ const double* dmat(const double* mats, int l) {
  int o = 0;
  for (int k = 0; k < l; ++k) o += (2 * k + 1) * ((k + 1) * (k + 2) / 2);
  return mats + o;
}

// M_sph[mu][nu] = sum_{a,b} C[mu][a] M_cart[a][b] C[nu][b] (a, b in the shells of mu, nu)
__global__ void cart_to_sph_2d_kernel(const double* __restrict__ M, double* __restrict__ S,
                                      const int* __restrict__ sph, const double* __restrict__ mats,
                                      long nsph, long ncart) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nsph * nsph) return;
  const long mu = idx / nsph, nu = idx - mu * nsph;
  const int la = sph[mu], ca0 = sph[2 * nsph + mu], ia = sph[3 * nsph + mu];
  const int lb = sph[nu], cb0 = sph[2 * nsph + nu], ib = sph[3 * nsph + nu];
  const int nca = (la + 1) * (la + 2) / 2, ncb = (lb + 1) * (lb + 2) / 2;
  const double* Ca = dmat(mats, la) + ia * nca;
  const double* Cb = dmat(mats, lb) + ib * ncb;
  double s = 0.0;
  for (int a = 0; a < nca; ++a) {
    const double ca = Ca[a];
    if (ca == 0.0) continue;
    const double* row = M + (size_t)(ca0 + a) * ncart + cb0;
    double t = 0.0;
    for (int b = 0; b < ncb; ++b) t += row[b] * Cb[b];
    s += ca * t;
  }
  S[idx] = s;
}

// D_cart[a][b] = sum_{mu,nu} C[mu][a] D_sph[mu][nu] C[nu][b]
__global__ void sph_to_cart_density_kernel(const double* __restrict__ Ds, double* __restrict__ Dc,
                                           const int* __restrict__ cart, const double* __restrict__ mats,
                                           long nsph, long ncart) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= ncart * ncart) return;
  const long a = idx / ncart, b = idx - a * ncart;
  const int la = cart[a], sa0 = cart[ncart + a], ja = cart[3 * ncart + a];
  const int lb = cart[b], sb0 = cart[ncart + b], jb = cart[3 * ncart + b];
  const int nca = (la + 1) * (la + 2) / 2, ncb = (lb + 1) * (lb + 2) / 2;
  const double* Ca = dmat(mats, la);
  const double* Cb = dmat(mats, lb);
  double s = 0.0;
  for (int mu = 0; mu < 2 * la + 1; ++mu) {
    const double ca = Ca[mu * nca + ja];
    if (ca == 0.0) continue;
    const double* row = Ds + (size_t)(sa0 + mu) * nsph + sb0;
    double t = 0.0;
    for (int nu = 0; nu < 2 * lb + 1; ++nu) t += row[nu] * Cb[nu * ncb + jb];
    s += ca * t;
  }
  Dc[idx] = s;
}

std::mutex g_map_mutex;
struct CachedMap {
  const lai_basis* basis;
  int device;
  DevMap m;
};
std::vector<CachedMap> g_maps;

// Device copy of the map of (basis, device), built once.
int device_map(const lai_basis* basis, int device, DevMap* out) {
  std::lock_guard<std::mutex> lock(g_map_mutex);
  for (auto& c : g_maps)
    if (c.basis == basis && c.device == device) { *out = c.m; return LAI_OK; }
  FuncMap f;
  if (int rc = build_map(basis, f)) return rc;
  std::vector<int> sph(4 * f.nsph), cart(4 * f.ncart);
  for (long i = 0; i < f.nsph; ++i) {
    sph[i] = f.sph_l[i]; sph[f.nsph + i] = f.sph_first_sph[i];
    sph[2 * f.nsph + i] = f.sph_first_cart[i]; sph[3 * f.nsph + i] = f.sph_local[i];
  }
  for (long i = 0; i < f.ncart; ++i) {
    cart[i] = f.cart_l[i]; cart[f.ncart + i] = f.cart_first_sph[i];
    cart[2 * f.ncart + i] = f.cart_first_cart[i]; cart[3 * f.ncart + i] = f.cart_local[i];
  }
  const auto& mats = all_matrices();
  DevMap m;
  m.nsph = f.nsph;
  m.ncart = f.ncart;
  if (cudaMalloc(&m.sph, sizeof(int) * std::max<size_t>(1, sph.size())) != cudaSuccess ||
      cudaMalloc(&m.cart, sizeof(int) * std::max<size_t>(1, cart.size())) != cudaSuccess ||
      cudaMalloc(&m.mats, sizeof(double) * mats.size()) != cudaSuccess)
    return err(LAI_ENOMEM, "spherical transform: device allocation failed");
  if (cudaMemcpy(m.sph, sph.data(), sizeof(int) * sph.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(m.cart, cart.data(), sizeof(int) * cart.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(m.mats, mats.data(), sizeof(double) * mats.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return err(LAI_ECUDA, "spherical transform: upload failed");
  g_maps.push_back({basis, device, m});
  *out = m;
  return LAI_OK;
}

}  // namespace

namespace lai {
// Forget the device maps of a basis that is being destroyed.
void spherical_forget_basis(const lai_basis* basis) {
  std::lock_guard<std::mutex> lock(g_map_mutex);
  for (size_t i = 0; i < g_maps.size();) {
    if (g_maps[i].basis == basis) {
      int cur = 0;
      cudaGetDevice(&cur);
      cudaSetDevice(g_maps[i].device);
      cudaFree(g_maps[i].m.sph);
      cudaFree(g_maps[i].m.cart);
      cudaFree(g_maps[i].m.mats);
      cudaSetDevice(cur);
      g_maps.erase(g_maps.begin() + i);
    } else {
      ++i;
    }
  }
}
}  // namespace lai

extern "C" {

int lai_cart_to_sph_matrix(int l, double* C) {
  if (l < 0 || l > kMaxL) return err(LAI_EINVAL, "lai_cart_to_sph_matrix: l must be 0..4");
  if (!C) return err(LAI_EINVAL, "lai_cart_to_sph_matrix: null output");
  fill_matrix(l, C);
  return LAI_OK;
}

long lai_basis_nbf_spherical(const lai_basis* basis) {
  if (!basis) return -1;
  FuncMap f;
  if (build_map(basis, f) != LAI_OK) return -1;
  return f.nsph;
}

int lai_cart_to_sph_2d(const lai_basis* basis, const double* M_cart, double* M_sph) {
  if (!basis || !M_cart || !M_sph) return err(LAI_EINVAL, "lai_cart_to_sph_2d: null argument");
  FuncMap f;
  if (int rc = build_map(basis, f)) return rc;
  const auto& mats = all_matrices();
  const long nc = f.ncart, ns = f.nsph;
  for (long mu = 0; mu < ns; ++mu)
    for (long nu = 0; nu < ns; ++nu) {
      const int la = f.sph_l[mu], lb = f.sph_l[nu];
      const int nca = lai::ncart(la), ncb = lai::ncart(lb);
      const double* Ca = mats.data() + mat_offset(la) + f.sph_local[mu] * nca;
      const double* Cb = mats.data() + mat_offset(lb) + f.sph_local[nu] * ncb;
      double s = 0.0;
      for (int a = 0; a < nca; ++a) {
        if (Ca[a] == 0.0) continue;
        const double* row = M_cart + (size_t)(f.sph_first_cart[mu] + a) * nc + f.sph_first_cart[nu];
        double t = 0.0;
        for (int b = 0; b < ncb; ++b) t += row[b] * Cb[b];
        s += Ca[a] * t;
      }
      M_sph[mu * ns + nu] = s;
    }
  return LAI_OK;
}

int lai_sph_to_cart_density(const lai_basis* basis, const double* D_sph, double* D_cart) {
  if (!basis || !D_sph || !D_cart) return err(LAI_EINVAL, "lai_sph_to_cart_density: null argument");
  FuncMap f;
  if (int rc = build_map(basis, f)) return rc;
  const auto& mats = all_matrices();
  const long nc = f.ncart, ns = f.nsph;
  for (long a = 0; a < nc; ++a)
    for (long b = 0; b < nc; ++b) {
      const int la = f.cart_l[a], lb = f.cart_l[b];
      const double* Ca = mats.data() + mat_offset(la);
      const double* Cb = mats.data() + mat_offset(lb);
      const int nca = lai::ncart(la), ncb = lai::ncart(lb);
      double s = 0.0;
      for (int mu = 0; mu < 2 * la + 1; ++mu) {
        const double ca = Ca[mu * nca + f.cart_local[a]];
        if (ca == 0.0) continue;
        const double* row = D_sph + (size_t)(f.cart_first_sph[a] + mu) * ns + f.cart_first_sph[b];
        double t = 0.0;
        for (int nu = 0; nu < 2 * lb + 1; ++nu) t += row[nu] * Cb[nu * ncb + f.cart_local[b]];
        s += ca * t;
      }
      D_cart[a * nc + b] = s;
    }
  return LAI_OK;
}

int lai_cart_to_sph_2d_device(lai_engine* engine, const double* d_M_cart, double* d_M_sph, void* stream) {
  if (!engine || !d_M_cart || !d_M_sph) return err(LAI_EINVAL, "lai_cart_to_sph_2d_device: null argument");
  if (lai::engine_nsys(engine) > 1) return err(LAI_ENOTSUP, "lai_cart_to_sph_2d_device: not available for a batched engine");
  const int dev = lai::engine_device(engine);
  if (cudaSetDevice(dev) != cudaSuccess) return err(LAI_ECUDA, "lai_cart_to_sph_2d_device: cudaSetDevice");
  DevMap m;
  if (int rc = device_map(lai::engine_basis(engine), dev, &m)) return rc;
  const long n = m.nsph * m.nsph;
  if (n > 0)
    cart_to_sph_2d_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        d_M_cart, d_M_sph, m.sph, m.mats, m.nsph, m.ncart);
  if (cudaGetLastError() != cudaSuccess) return err(LAI_ECUDA, "lai_cart_to_sph_2d_device: launch failed");
  return LAI_OK;
}

int lai_sph_to_cart_density_device(lai_engine* engine, const double* d_D_sph, double* d_D_cart,
                                   void* stream) {
  if (!engine || !d_D_sph || !d_D_cart) return err(LAI_EINVAL, "lai_sph_to_cart_density_device: null argument");
  if (lai::engine_nsys(engine) > 1) return err(LAI_ENOTSUP, "lai_sph_to_cart_density_device: not available for a batched engine");
  const int dev = lai::engine_device(engine);
  if (cudaSetDevice(dev) != cudaSuccess) return err(LAI_ECUDA, "lai_sph_to_cart_density_device: cudaSetDevice");
  DevMap m;
  if (int rc = device_map(lai::engine_basis(engine), dev, &m)) return rc;
  const long n = m.ncart * m.ncart;
  if (n > 0)
    sph_to_cart_density_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        d_D_sph, d_D_cart, m.cart, m.mats, m.nsph, m.ncart);
  if (cudaGetLastError() != cudaSuccess)
    return err(LAI_ECUDA, "lai_sph_to_cart_density_device: launch failed");
  return LAI_OK;
}

}  // extern "C"
