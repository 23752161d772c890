// Test infrastructure only: a C-ABI shim over the UNMODIFIED reference
// (LibAccInt) CPU implementation, compiled from the reference's own sources
// by oracle/Makefile into oracle/_ref/libref_oracle.so.  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline/reference arm load it;
// nothing in the product links it.
//
// Every entry point calls the reference's public C++ API:
//   - Shell(am, center, exps, coefs)          src/shared/basis/shell.cpp:163-187
//   - BasisSet(shells)                        src/shared/basis/basis_set.cpp:21-29
//   - data::create_builtin_basis("sto-3g")    src/shared/data/builtin_basis.cpp
//   - Engine::compute(Operator::coulomb(), FockBuilder)
//                                             include/libaccint/engine/engine.hpp:435-499,727-731
//   - Engine::compute_and_consume(op, fb, ScreeningOptions{use_permutation_symmetry})
//                                             include/libaccint/engine/engine.hpp:1635-1666,1806-1861
//   - kernels::compute_eri                    src/host/kernels/eri_kernel.cpp:168-381
//   - screening::SchwarzBounds                src/shared/screening/schwarz_bounds.cpp:16-59
//   - math::rys_compute / boys_evaluate_array src/shared/math/rys_quadrature.cpp:455-513,
//                                             src/shared/math/boys_function.cpp:253-303
//   - FockBuilder::accumulate_symmetric       src/shared/consumers/fock_builder.cpp:123-222
//   - math::get_cart_to_sph_matrix            include/libaccint/math/spherical_transform.hpp:20-40
//   - Engine::compute_overlap_matrix / compute_kinetic_matrix / compute_nuclear_matrix
//                                             include/libaccint/engine/engine.hpp:831-900
//   - data::create_builtin_auxiliary_basis    src/shared/data/auxiliary_basis_data.cpp:735-776
//   - kernels::compute_three_center_tensor (abP) / compute_two_center_metric
//                                             src/host/kernels/three_center_eri_kernel.cpp:273-362,
//                                             src/host/kernels/two_center_coulomb_kernel.cpp:212-251
//   - consumers::DFFockBuilder                src/shared/consumers/df_fock_builder.cpp:102-450
#include <libaccint/libaccint.hpp>
#include <libaccint/engine/engine.hpp>
#include <libaccint/consumers/fock_builder.hpp>
#include <libaccint/data/builtin_basis.hpp>
#include <libaccint/kernels/eri_kernel.hpp>
#include <libaccint/math/rys_quadrature.hpp>
#include <libaccint/math/boys_function.hpp>
#include <libaccint/math/spherical_transform.hpp>
#include <libaccint/screening/schwarz_bounds.hpp>
#include <libaccint/screening/screening_options.hpp>
#include <libaccint/basis/auxiliary_basis_set.hpp>
#include <libaccint/data/auxiliary_basis_data.hpp>
#include <libaccint/consumers/df_fock_builder.hpp>
#include <libaccint/kernels/three_center_eri_kernel.hpp>
#include <libaccint/kernels/two_center_coulomb_kernel.hpp>

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <exception>
#include <memory>
#include <vector>

using namespace libaccint;

namespace {

struct RefBasis {
    std::unique_ptr<BasisSet> basis;
};

thread_local char g_err[512] = {0};

void set_err(const char* msg) {
    std::strncpy(g_err, msg, sizeof(g_err) - 1);
    g_err[sizeof(g_err) - 1] = 0;
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err; }

// Build a basis from raw (un-normalized) contraction coefficients; the
// reference Shell constructor applies its own normalization.
void* ref_basis_create(int nshell, const int* am, const int* nprim,
                       const double* centers, const double* exps,
                       const double* coefs, const int* atom_index) {
    try {
        std::vector<Shell> shells;
        shells.reserve(nshell);
        long off = 0;
        for (int s = 0; s < nshell; ++s) {
            std::vector<Real> e(exps + off, exps + off + nprim[s]);
            std::vector<Real> c(coefs + off, coefs + off + nprim[s]);
            off += nprim[s];
            Point3D ctr(centers[3 * s], centers[3 * s + 1], centers[3 * s + 2]);
            shells.emplace_back(am[s], ctr, std::move(e), std::move(c));
            if (atom_index) shells.back().set_atom_index(atom_index[s]);
        }
        auto* rb = new RefBasis();
        rb->basis = std::make_unique<BasisSet>(std::move(shells));
        return rb;
    } catch (const std::exception& ex) {
        set_err(ex.what());
        return nullptr;
    }
}

void* ref_basis_builtin_sto3g(int natom, const int* Z, const double* xyz) {
    try {
        std::vector<data::Atom> atoms;
        for (int a = 0; a < natom; ++a)
            atoms.push_back({Z[a], Point3D(xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2])});
        auto* rb = new RefBasis();
        rb->basis = std::make_unique<BasisSet>(data::create_builtin_basis("sto-3g", atoms));
        return rb;
    } catch (const std::exception& ex) {
        set_err(ex.what());
        return nullptr;
    }
}

void ref_basis_free(void* h) { delete static_cast<RefBasis*>(h); }

long ref_basis_nbf(void* h) { return (long)static_cast<RefBasis*>(h)->basis->n_basis_functions(); }
long ref_basis_nshell(void* h) { return (long)static_cast<RefBasis*>(h)->basis->n_shells(); }

// Export one shell: am, nprim, center, exponents and NORMALIZED coefficients.
int ref_basis_shell(void* h, long i, int* am, int* nprim, double* center,
                    double* exps, double* coefs, long* func_index) {
    const auto& sh = static_cast<RefBasis*>(h)->basis->shell((Size)i);
    *am = sh.angular_momentum();
    *nprim = (int)sh.n_primitives();
    center[0] = sh.center().x;
    center[1] = sh.center().y;
    center[2] = sh.center().z;
    if (exps) for (Size p = 0; p < sh.n_primitives(); ++p) exps[p] = sh.exponents()[p];
    if (coefs) for (Size p = 0; p < sh.n_primitives(); ++p) coefs[p] = sh.coefficients()[p];
    *func_index = (long)sh.function_index();
    return 0;
}

// Full N^4 race-free OpenMP path: Engine::compute(coulomb, FockBuilder).
// Returns wall seconds of the compute call, or -1 on error.
double ref_jk_full(void* h, const double* D, double* J, double* K, int nthreads) {
    try {
        auto& basis = *static_cast<RefBasis*>(h)->basis;
        const Size n = basis.n_basis_functions();
        if (nthreads > 0) omp_set_num_threads(nthreads);
        Engine engine(basis);
        consumers::FockBuilder fb(n);
        fb.set_density(D, n);
        auto t0 = std::chrono::steady_clock::now();
        engine.compute(Operator::coulomb(), fb);
        auto t1 = std::chrono::steady_clock::now();
        auto Jm = fb.get_coulomb_matrix();
        auto Km = fb.get_exchange_matrix();
        std::memcpy(J, Jm.data(), sizeof(double) * n * n);
        std::memcpy(K, Km.data(), sizeof(double) * n * n);
        return std::chrono::duration<double>(t1 - t0).count();
    } catch (const std::exception& ex) {
        set_err(ex.what());
        return -1.0;
    }
}

// Serial Schwarz-screened canonical path with 8-fold symmetric scatter.
double ref_jk_screened_sym(void* h, const double* D, double* J, double* K, double thr) {
    try {
        auto& basis = *static_cast<RefBasis*>(h)->basis;
        const Size n = basis.n_basis_functions();
        Engine engine(basis);
        consumers::FockBuilder fb(n);
        fb.set_density(D, n);
        screening::ScreeningOptions opt;
        opt.threshold = thr;
        opt.enabled = true;
        opt.use_permutation_symmetry = true;
        auto t0 = std::chrono::steady_clock::now();
        engine.compute_and_consume(Operator::coulomb(), fb, opt);
        auto t1 = std::chrono::steady_clock::now();
        auto Jm = fb.get_coulomb_matrix();
        auto Km = fb.get_exchange_matrix();
        std::memcpy(J, Jm.data(), sizeof(double) * n * n);
        std::memcpy(K, Km.data(), sizeof(double) * n * n);
        return std::chrono::duration<double>(t1 - t0).count();
    } catch (const std::exception& ex) {
        set_err(ex.what());
        return -1.0;
    }
}

// One contracted shell quartet, [a][b][c][d] row-major, norm-corrected Cartesian.
int ref_eri_quartet(void* h, long i, long j, long k, long l, double* out) {
    try {
        auto& basis = *static_cast<RefBasis*>(h)->basis;
        TwoElectronBuffer<0> buf;
        kernels::compute_eri(basis.shell(i), basis.shell(j), basis.shell(k), basis.shell(l), buf);
        const int na = basis.shell(i).n_functions(), nb = basis.shell(j).n_functions();
        const int nc = basis.shell(k).n_functions(), nd = basis.shell(l).n_functions();
        long o = 0;
        for (int a = 0; a < na; ++a)
            for (int b = 0; b < nb; ++b)
                for (int c = 0; c < nc; ++c)
                    for (int d = 0; d < nd; ++d) out[o++] = buf(a, b, c, d);
        return 0;
    } catch (const std::exception& ex) {
        set_err(ex.what());
        return -1;
    }
}

// Schwarz bounds Q_ij (packed upper triangle as the reference stores them).
int ref_schwarz(void* h, double* Q) {
    try {
        auto& basis = *static_cast<RefBasis*>(h)->basis;
        screening::SchwarzBounds sb(basis);
        const Size n = basis.n_shells();
        for (Size i = 0; i < n; ++i)
            for (Size j = i; j < n; ++j) Q[i * n + j] = Q[j * n + i] = sb(i, j);
        return 0;
    } catch (const std::exception& ex) {
        set_err(ex.what());
        return -1;
    }
}

// Same bounds as SchwarzBounds(basis) (schwarz_bounds.cpp:20-59: Q_ij =
// sqrt(max_ab |(ab|ab)|) from kernels::compute_eri), with the pair loop spread
// over OpenMP threads.  Q is the full nshell x nshell matrix.
int ref_schwarz_parallel(void* h, double* Q, int nthreads) {
    try {
        auto& basis = *static_cast<RefBasis*>(h)->basis;
        const long n = (long)basis.n_shells();
        if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
        {
            TwoElectronBuffer<0> buf;
#pragma omp for schedule(dynamic, 16)
            for (long ij = 0; ij < n * n; ++ij) {
                const long i = ij / n, j = ij % n;
                if (j < i) continue;
                const auto& si = basis.shell(i);
                const auto& sj = basis.shell(j);
                kernels::compute_eri(si, sj, si, sj, buf);
                double mx = 0.0;
                for (int a = 0; a < si.n_functions(); ++a)
                    for (int b = 0; b < sj.n_functions(); ++b)
                        mx = std::max(mx, std::abs(buf(a, b, a, b)));
                Q[i * n + j] = Q[j * n + i] = std::sqrt(mx);
            }
        }
        return 0;
    } catch (const std::exception& ex) {
        set_err(ex.what());
        return -1;
    }
}

void ref_rys(int n, double T, double* roots, double* weights) {
    math::rys_compute(n, T, roots, weights);
}

void ref_boys(int mmax, double T, double* out) { math::boys_evaluate_array(mmax, T, out); }

// Time a caller-supplied list of canonical shell quartets through the
// reference's compute_2e_shell_quartet + FockBuilder::accumulate_symmetric,
// on nthreads OpenMP threads with one FockBuilder per thread (race-free),
// reduced into J/K at the end.  Returns wall seconds of the parallel region.
double ref_time_quartets(void* h, const double* D, const long* quartets, long nq,
                         int nthreads, double* J, double* K) {
    try {
        auto& basis = *static_cast<RefBasis*>(h)->basis;
        const Size n = basis.n_basis_functions();
        if (nthreads <= 0) nthreads = omp_get_max_threads();
        std::vector<std::unique_ptr<consumers::FockBuilder>> fbs(nthreads);
        for (int t = 0; t < nthreads; ++t) {
            fbs[t] = std::make_unique<consumers::FockBuilder>(n);
            fbs[t]->set_density(D, n);
        }
        Engine engine(basis);
        auto& cpu = engine.cpu_engine();
        const Operator op = Operator::coulomb();
        auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel num_threads(nthreads)
        {
            TwoElectronBuffer<0> buf;
            auto& fb = *fbs[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 8)
            for (long q = 0; q < nq; ++q) {
                const long i = quartets[4 * q], j = quartets[4 * q + 1];
                const long k = quartets[4 * q + 2], l = quartets[4 * q + 3];
                const auto& a = basis.shell(i);
                const auto& b = basis.shell(j);
                const auto& c = basis.shell(k);
                const auto& d = basis.shell(l);
                cpu.compute_2e_shell_quartet(op, a, b, c, d, buf);
                fb.accumulate_symmetric(buf, a.function_index(), b.function_index(),
                                        c.function_index(), d.function_index(),
                                        a.n_functions(), b.n_functions(), c.n_functions(),
                                        d.n_functions(), i == j, k == l, (i == k && j == l));
            }
        }
        auto t1 = std::chrono::steady_clock::now();
        if (J && K) {
            std::memset(J, 0, sizeof(double) * n * n);
            std::memset(K, 0, sizeof(double) * n * n);
            for (int t = 0; t < nthreads; ++t) {
                auto Jm = fbs[t]->get_coulomb_matrix();
                auto Km = fbs[t]->get_exchange_matrix();
                for (Size x = 0; x < n * n; ++x) {
                    J[x] += Jm[x];
                    K[x] += Km[x];
                }
            }
        }
        return std::chrono::duration<double>(t1 - t0).count();
    } catch (const std::exception& ex) {
        set_err(ex.what());
        return -1.0;
    }
}

int ref_max_threads() { return omp_get_max_threads(); }

// C_l [n_sph x n_cart] row-major of the reference (l <= 4); returns n_sph*n_cart or -1.
int ref_cart_to_sph(int l, double* out) {
    try {
        const double* C = libaccint::math::get_cart_to_sph_matrix(l);
        const int n = (2 * l + 1) * (l + 1) * (l + 2) / 2;
        std::memcpy(out, C, sizeof(double) * n);
        return n;
    } catch (const std::exception& ex) {
        set_err(ex.what());
        return -1;
    }
}

// One-electron matrix of the reference CPU engine: kind 0 overlap, 1 kinetic,
// 2 nuclear attraction of the point charges (xyz [n][3], q [n]).  Returns 0 or -1.
int ref_one_electron(void* h, int kind, int ncharge, const double* xyz, const double* q, double* out) {
    try {
        auto& basis = *static_cast<RefBasis*>(h)->basis;
        const Size n = basis.n_basis_functions();
        Engine engine(basis);
        std::vector<Real> r;
        if (kind == 0) {
            engine.compute_overlap_matrix(r, BackendHint::ForceCPU);
        } else if (kind == 1) {
            engine.compute_kinetic_matrix(r, BackendHint::ForceCPU);
        } else {
            PointChargeParams c;
            for (int i = 0; i < ncharge; ++i) {
                c.x.push_back(xyz[3 * i]);
                c.y.push_back(xyz[3 * i + 1]);
                c.z.push_back(xyz[3 * i + 2]);
                c.charge.push_back(q[i]);
            }
            engine.compute_nuclear_matrix(c, r, BackendHint::ForceCPU);
        }
        if (r.size() != n * n) { set_err("ref_one_electron: unexpected result size"); return -1; }
        std::memcpy(out, r.data(), sizeof(double) * n * n);
        return 0;
    } catch (const std::exception& ex) {
        set_err(ex.what());
        return -1;
    }
}

// Built-in auxiliary basis (e.g. "cc-pVDZ-RI") on the atoms; NULL on error.
void* ref_aux_builtin(const char* name, int natom, const int* Z, const double* xyz) {
    try {
        std::vector<data::Atom> atoms;
        for (int a = 0; a < natom; ++a)
            atoms.push_back({Z[a], Point3D(xyz[3 * a], xyz[3 * a + 1], xyz[3 * a + 2])});
        return new AuxiliaryBasisSet(data::create_builtin_auxiliary_basis(name, atoms));
    } catch (const std::exception& ex) {
        set_err(ex.what());
        return nullptr;
    }
}

void ref_aux_free(void* h) { delete static_cast<AuxiliaryBasisSet*>(h); }
long ref_aux_nbf(void* h) { return (long)static_cast<AuxiliaryBasisSet*>(h)->n_functions(); }
long ref_aux_nshell(void* h) { return (long)static_cast<AuxiliaryBasisSet*>(h)->shells().size(); }

// One auxiliary shell: am, nprim, center, exponents, NORMALIZED coefficients.
int ref_aux_shell(void* h, long i, int* am, int* nprim, double* center, double* exps, double* coefs) {
    const auto& sh = static_cast<AuxiliaryBasisSet*>(h)->shells()[(Size)i];
    *am = sh.angular_momentum();
    *nprim = (int)sh.n_primitives();
    center[0] = sh.center().x;
    center[1] = sh.center().y;
    center[2] = sh.center().z;
    if (exps) for (Size p = 0; p < sh.n_primitives(); ++p) exps[p] = sh.exponents()[p];
    if (coefs) for (Size p = 0; p < sh.n_primitives(); ++p) coefs[p] = sh.coefficients()[p];
    return 0;
}

// T[(a*n + b)*naux + P] = (ab|P) and V[P*naux + Q] = (P|Q) of the reference kernels.
int ref_eri3c(void* hb, void* ha, double* T) {
    try {
        auto& basis = *static_cast<RefBasis*>(hb)->basis;
        auto& aux = *static_cast<AuxiliaryBasisSet*>(ha);
        kernels::compute_three_center_tensor(basis.shells(), aux.shells(), T, basis.n_basis_functions(),
                                             aux.n_functions(), kernels::ThreeCenterStorageFormat::abP);
        return 0;
    } catch (const std::exception& ex) {
        set_err(ex.what());
        return -1;
    }
}

int ref_eri2c(void* ha, double* V) {
    try {
        auto& aux = *static_cast<AuxiliaryBasisSet*>(ha);
        kernels::compute_two_center_metric(aux.shells(), V, aux.n_functions());
        return 0;
    } catch (const std::exception& ex) {
        set_err(ex.what());
        return -1;
    }
}

// DFFockBuilder(orbital, aux): set_density(D), compute_coulomb(), compute_exchange().
int ref_df_jk(void* hb, void* ha, const double* D, double* J, double* K) {
    try {
        auto& basis = *static_cast<RefBasis*>(hb)->basis;
        auto& aux = *static_cast<AuxiliaryBasisSet*>(ha);
        const Size n = basis.n_basis_functions();
        consumers::DFFockBuilder df(basis, aux);
        df.set_density(std::span<const Real>(D, n * n));
        const auto j = df.compute_coulomb();
        const auto k = df.compute_exchange();
        std::memcpy(J, j.data(), sizeof(double) * n * n);
        std::memcpy(K, k.data(), sizeof(double) * n * n);
        return 0;
    } catch (const std::exception& ex) {
        set_err(ex.what());
        return -1;
    }
}

}  // extern "C"
