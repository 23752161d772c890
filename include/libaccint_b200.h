/*
 * libaccint-b200: C ABI of the B200-native two-electron J/K engine.
 *
 * Rys-quadrature electron-repulsion integrals over contracted Cartesian
 * Gaussians (l <= 4), Schwarz-screened, digested straight into Coulomb (J) and
 * exchange (K) matrices on one NVIDIA B200 (sm_100a).  Plain C types only: every
 * matrix is a row-major nbf x nbf array of doubles, every pointer is owned by the
 * caller, and every function returns 0 (LAI_OK) or a negative error code; no C++
 * exception crosses this boundary.  lai_last_error() gives a message for the
 * calling thread.  An engine is not thread-safe: serialize calls per engine
 * (the reference's FockBuilder has the same contract,
 * include/libaccint/consumers/fock_builder.hpp).
 *
 * Basis conventions are the reference's (LibAccInt v0.1.0-alpha.2):
 *   - Cartesian components ordered lx descending, then ly descending
 *     (include/libaccint/math/cartesian_indices.hpp:26-36);
 *   - contraction coefficients normalized so the (l,0,0) component has unit
 *     self-overlap, each component scaled by 1/sqrt((2lx-1)!!(2ly-1)!!(2lz-1)!!)
 *     (src/shared/basis/shell.cpp:32-113, include/libaccint/kernels/norm_correction.hpp:28-34);
 *   - basis functions numbered shell by shell in input order
 *     (src/shared/basis/basis_set.cpp:161-185);
 *   - J_mn = sum_ls (mn|ls) D_ls, K_ml = sum_ns (mn|ls) D_ns
 *     (include/libaccint/consumers/fock_builder.hpp:41-43).
 */
#ifndef LIBACCINT_B200_H
#define LIBACCINT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LAI_ABI_VERSION 2

#if defined(__GNUC__)
#define LAI_API __attribute__((visibility("default")))
#else
#define LAI_API
#endif

enum lai_status {
  LAI_OK = 0,
  LAI_EINVAL = -1,   /* bad argument (sizes, null pointers, l > 4, ...)      */
  LAI_ENOMEM = -2,   /* device or host allocation failed                      */
  LAI_ECUDA = -3,    /* CUDA runtime error (no device, launch failure, ...)   */
  LAI_ETIMEOUT = -4, /* a bounded device wait gave up                         */
  LAI_ESTATE = -5,   /* call out of order (e.g. no density set)               */
  LAI_ENOTSUP = -6   /* feature not available in this build                   */
};

typedef struct lai_basis lai_basis;
typedef struct lai_engine lai_engine;

/* Last error message of the calling thread (never NULL). */
LAI_API const char* lai_last_error(void);
LAI_API int lai_abi_version(void);

/* ---------------------------------------------------------------------------
 * Basis.  Replaces Shell(am, center, exps, coefs) + BasisSet(shells)
 * (src/shared/basis/shell.cpp:163-187, src/shared/basis/basis_set.cpp:21-29).
 * l[s], nprim[s]: angular momentum (0..4) and primitive count of shell s;
 * centers[3*s..]: Bohr; exps/coefs: primitives of all shells concatenated.
 * Coefficients are RAW contraction coefficients and are normalized here exactly
 * like the reference Shell constructor, unless flags has LAI_BASIS_PRENORMALIZED.
 * atom_index may be NULL (then every shell gets its own atom id = -1).
 * ------------------------------------------------------------------------- */
#define LAI_BASIS_PRENORMALIZED 1
LAI_API int lai_basis_create(int nshell, const int* l, const int* nprim, const double* centers,
                     const double* exps, const double* coefs, const int* atom_index, int flags,
                     lai_basis** out);
/* A basis from Basis Set Exchange JSON text (the format of the reference's
 * share/basis_sets/<name>.json, "complete" or "minimal" schema) on natom atoms with
 * atomic numbers Z and positions xyz [natom][3] (Bohr); shells per atom in the
 * file's order, general contractions split into one shell per coefficient column,
 * SP shells into one shell per l, all-zero columns skipped, raw coefficients
 * normalized as by lai_basis_create.  Replaces data::BseJsonParser::parse
 * (src/shared/data/bse_json_parser.cpp:27-140). */
LAI_API int lai_basis_from_bse_json(const char* json_text, size_t length, int natom, const int* Z,
                                    const double* xyz, lai_basis** out);
LAI_API void lai_basis_destroy(lai_basis* basis);
LAI_API long lai_basis_nbf(const lai_basis* basis);
LAI_API int lai_basis_nshell(const lai_basis* basis);
/* Shell s after normalization: exps/coefs get nprim entries (input order, zero
 * coefficients kept); func_index = first basis function of the shell. */
LAI_API int lai_basis_shell(const lai_basis* basis, int s, int* l, int* nprim, double* center,
                    double* exps, double* coefs, long* func_index);

/* ---------------------------------------------------------------------------
 * Engine: device-resident pair data for one basis, Schwarz bounds and the
 * sorted pair lists.  Replaces Engine(basis) + precompute_schwarz_bounds()
 * (include/libaccint/engine/engine.hpp:86-107,1578-1583).
 * ------------------------------------------------------------------------- */
typedef struct {
  double schwarz_threshold; /* pass iff Q_ij*Q_kl >= threshold (default 1e-12) */
  int device;               /* CUDA device ordinal (default 0)                  */
  double prim_threshold;    /* skip primitive quartets whose primitive Schwarz
                               bound q_ab*q_cd is below this (no counterpart in
                               the reference); < 0 = 1e-3 * schwarz_threshold
                               (default), 0 = keep every primitive quartet       */
} lai_engine_opts;
LAI_API void lai_engine_opts_default(lai_engine_opts* opts);
/* All engines of one process use one device: creating an engine on another
 * device than the process's first engine returns LAI_ENOTSUP (run one process
 * per GPU, as the multi-GPU build does). */
LAI_API int lai_engine_create(const lai_basis* basis, const lai_engine_opts* opts, lai_engine** out);
LAI_API void lai_engine_destroy(lai_engine* engine);
/* Schwarz bounds Q[i*nshell+j] = sqrt(max |(ij|ij)|) of all shell pairs
 * (src/shared/screening/schwarz_bounds.cpp:20-59). */
LAI_API int lai_engine_schwarz(lai_engine* engine, double* Q);

/* ---------------------------------------------------------------------------
 * J/K build.  Replaces Engine::compute(Operator::coulomb(), FockBuilder&) and
 * Engine::compute_and_consume(op, FockBuilder&, ScreeningOptions)
 * (include/libaccint/engine/engine.hpp:435-499,727-731,1635-1666) followed by
 * FockBuilder::get_coulomb_matrix()/get_exchange_matrix()
 * (include/libaccint/consumers/fock_builder.hpp:111-119).
 * D must be symmetric (the reference's symmetric scatter assumes it too,
 * src/shared/consumers/fock_builder.cpp:163-171).
 * ------------------------------------------------------------------------- */
typedef struct {
  double fp32_cut;   /* mixed precision: quartets with Q_ij*Q_kl*max|D| < fp32_cut
                        run roots, recurrences and primitive contraction in FP32
                        (transfer, normalization and J/K digestion stay FP64);
                        0 = all FP64.  The Schwarz cut fp32_cut/max|D| is rounded
                        down to a power of two; reading max|D| costs one stream
                        synchronisation.  No counterpart in the reference, whose
                        float path computes in FP64 and casts
                        (include/libaccint/engine/precision_dispatch.hpp:200-259). */
  int check_symmetric; /* 1 = reject a D that is not symmetric to 1e-12 (host)  */
  int shard_index;     /* multi-GPU: this rank computes shard shard_index of     */
  int shard_count;     /* shard_count equal slices of every quartet block (1 = all);
                          J/K then hold this rank's partial sums -- add them over
                          ranks (one all-reduce) to get the full J/K            */
  int profile;         /* 1 = time every kernel launch (lai_jk_last_profile)    */
  int graph;           /* lai_jk_build_device only: 1 = run the build as a CUDA
                          graph, captured on the first call for these (D, J, K,
                          stream, fp32_cut, shard) and replayed afterwards (one
                          launch instead of one per shell-quartet class).  Needs
                          a non-NULL stream and profile = 0; the replays keep
                          the FP32 cut derived from max|D| at capture time.     */
  double fp32_prim_rel; /* mixed precision, FP32 quartets only: also skip their
                          primitive quartets whose bound q_ab*q_cd is below
                          fp32_prim_rel * Q_ij*Q_kl (the quartet's own Schwarz
                          bound), so that each skipped term is below that
                          fraction of the quartet -- primitive accuracy matched
                          to the FP32 arithmetic.  0 = off (the engine's
                          absolute primitive cut only).  No counterpart in the
                          reference.                                            */
} lai_jk_opts;
LAI_API void lai_jk_opts_default(lai_jk_opts* opts);
/* The slice [lo, hi) of a block of `total` quartets that shard `index` of `count`
 * computes (contiguous, sizes differ by at most one; the shards tile [0, total)).
 * Host-only arithmetic, no device needed.  The multi-GPU driver calls the build
 * with shard_index = rank, shard_count = world size and sums J and K over ranks. */
LAI_API int lai_shard_range(int64_t total, int index, int count, int64_t* lo, int64_t* hi);

typedef struct {
  int64_t quartets_fp64;   /* canonical shell quartets computed in FP64       */
  int64_t quartets_fp32;   /* ... and in FP32                                 */
  double alg_flops;        /* algorithmic FP work of those quartets (FLOP)    */
  double seconds_device;   /* device time of the integral + digestion kernels */
  double seconds_total;    /* wall time of the call                           */
  int kernel_launches;     /* kernels launched by the call                    */
  double fp32_schwarz_cut; /* Q_ij*Q_kl below which quartets ran in FP32 (0 = none) */
} lai_jk_report;

/* Host buffers (nbf*nbf doubles each). report may be NULL. */
LAI_API int lai_jk_build(lai_engine* engine, const double* D, size_t nbf, double* J, double* K,
                 const lai_jk_opts* opts, lai_jk_report* report);
/* Device buffers on the engine's device; stream is a cudaStream_t (NULL = legacy
 * default stream).  Asynchronous: returns after enqueueing (report times are
 * then not filled), except that opts->fp32_cut > 0 first synchronises the stream
 * once to read max|D|. */
LAI_API int lai_jk_build_device(lai_engine* engine, const double* d_D, double* d_J, double* d_K,
                        void* stream, const lai_jk_opts* opts, lai_jk_report* report);

/* J/K build that allocates nothing when called (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc at this point: plugins
 * whose host application owns the whole device through its own allocator, and
 * real-time drivers that forbid allocation after start-up (an allocation can
 * synchronize the device).  Same result as lai_jk_build_device(); the two nbf x nbf
 * accumulators live in a fixed 4 MiB array of the library's device image
 * (held on every GPU that loads the library until exit), hence
 * nbf <= LAI_NOALLOC_MAX_NBF, else LAI_EINVAL.  All calls share the
 * array: calls whose device work overlaps race.  The first call on a device
 * looks up the array's address -- make it before any stream capture.
 * Asynchronous on `stream` (a cudaStream_t, NULL = legacy default stream). */
#define LAI_NOALLOC_MAX_NBF 512
LAI_API int lai_jk_build_noalloc(lai_engine* engine, const double* d_D, double* d_J, double* d_K,
                                 void* stream);

/* ---------------------------------------------------------------------------
 * Raw integrals of every canonical shell quartet that passes the engine's
 * Schwarz threshold.  Replaces Engine::compute_batch_screened(op, screening)
 * (include/libaccint/engine/engine.hpp:1181-1187) returning IntegralBuffers with
 * quartet_meta {offset, fi..fl, na..nd} (include/libaccint/engine/integral_buffer.hpp:27-35).
 * Each quartet's block is [a][b][c][d] row-major starting at meta.offset, in the
 * shell order given by the function offsets fa..fd (one representative of the
 * 8-fold permutation orbit; all quartets are distinct orbits).
 * Call with out == NULL / meta == NULL to get the counts only.
 * ------------------------------------------------------------------------- */
typedef struct {
  int64_t offset;
  int32_t fa, fb, fc, fd;
  int32_t na, nb, nc, nd;
} lai_quartet_meta;
LAI_API int lai_eri_batch_screened(lai_engine* engine, double* out, size_t out_capacity,
                                   lai_quartet_meta* meta, size_t meta_capacity,
                                   int64_t* n_quartets, int64_t* n_values);

/* ---------------------------------------------------------------------------
 * Batched engine: many independent systems (molecules, clusters) in one engine,
 * so that every shell-quartet class of all of them runs as one persistent launch.
 * Quartets never mix systems.  D, J and K are packed: system s's nbf_s x nbf_s
 * block (row-major) starts at element offsets[s] (lai_engine_batch_layout).
 * lai_jk_build_device takes packed device arrays for a batched engine; the host
 * variant is lai_jk_build_batched.  No counterpart in the reference (one basis
 * per Engine).  Entry points that address one basis-wide matrix (lai_jk_build,
 * lai_engine_schwarz, lai_eri_batch_screened, work units, gradients, spherical
 * transforms, lai_jk_build_noalloc) return LAI_ENOTSUP for a batched engine.
 * ------------------------------------------------------------------------- */
LAI_API int lai_engine_create_batched(int nsys, const lai_basis* const* bases, const lai_engine_opts* opts,
                                      lai_engine** out);
/* nsys; offsets[nsys + 1] (elements); nbf[nsys].  Any output may be NULL. */
LAI_API int lai_engine_batch_layout(lai_engine* engine, int* nsys, int64_t* offsets, int* nbf);
LAI_API int lai_jk_build_batched(lai_engine* engine, const double* D, double* J, double* K,
                                 const lai_jk_opts* opts, lai_jk_report* report);

/* ---------------------------------------------------------------------------
 * Work units: a caller-supplied list of shell quartets, quartets[4t..4t+3] =
 * shell indices (i, j, k, l) of quartet t, in any order and orientation.
 * Replaces CudaEngine/CpuEngine::compute_shell_set_quartet(op, quartet, consumer,
 * canonical_symmetry) (include/libaccint/engine/cuda_engine.hpp:462-466,792-980;
 * include/libaccint/engine/cpu_engine.hpp:436-549) and Engine::compute_batch
 * (include/libaccint/engine/engine.hpp:1008-1122).  No Schwarz or primitive
 * screening is applied to a listed quartet.
 * ------------------------------------------------------------------------- */
/* Raw norm-corrected Cartesian integrals of each listed quartet, block t =
 * [i][j][k][l] in the listed shell order at out + meta[t].offset (meta also gives
 * the first functions and sizes).  out_capacity in doubles. */
LAI_API int lai_eri_quartets(lai_engine* engine, const int32_t* quartets, int64_t n, double* out,
                             size_t out_capacity, lai_quartet_meta* meta);
/* J/K contributions ADDED to J and K (nbf x nbf).  canonical_symmetry = 0: plain
 * accumulation of exactly the listed ordered quartets, J_ij += (ij|kl) D_kl,
 * K_ik += (ij|kl) D_jl (FockBuilder::accumulate, src/shared/consumers/fock_builder.cpp:64-121);
 * = 1: each listed quartet stands for its whole 8-fold permutation orbit, with the
 * degeneracy of equal shells (accumulate_symmetric, fock_builder.cpp:123-222).
 * Host buffers; the device variant takes device D/J/K and returns after the
 * kernels finished (the per-call pair tables are freed on return). */
LAI_API int lai_jk_accumulate_quartets(lai_engine* engine, const int32_t* quartets, int64_t n,
                                       const double* D, double* J, double* K, int canonical_symmetry);
LAI_API int lai_jk_accumulate_quartets_device(lai_engine* engine, const int32_t* quartets, int64_t n,
                                              const double* d_D, double* d_J, double* d_K, void* stream,
                                              int canonical_symmetry);
/* Plain J/K accumulation of an integral batch already on the device: block t is
 * d_eri[meta[t].offset ...], [a][b][c][d] over functions fa.., sizes na.. (meta on
 * the host).  Replaces GpuFockBuilder::accumulate_device_eri_batch
 * (src/device/cuda/consumers/fock_builder_gpu.cu:600-621). */
LAI_API int lai_jk_accumulate_eri_batch_device(lai_engine* engine, const double* d_eri,
                                               const lai_quartet_meta* meta, int64_t n, const double* d_D,
                                               double* d_J, double* d_K, void* stream);

/* ---------------------------------------------------------------------------
 * Nuclear gradient of E = 1/2 tr(D J[D]) - 1/4 tr(D K[D]) at fixed D, over the
 * engine's screened canonical quartets (those the J/K build computes):
 * dE/dR_A = sum_q s_q sum_abcd d(ab|cd)/dR_A (4 D_ab D_cd - D_ac D_bd - D_ad D_bc),
 * with derivative integrals formed and contracted on the fly.  dE/dD = J - K/2
 * comes from the J/K build.  No counterpart in the reference, which has no
 * derivative integrals (config.hpp.in:49, MAX_DERIVATIVE_ORDER = 0).  Needs the
 * basis created with atom indices; grad is [natom][3] (Hartree/Bohr), natom =
 * 1 + the largest atom index (lai_engine_natom).
 * ------------------------------------------------------------------------- */
LAI_API int lai_engine_natom(lai_engine* engine);
LAI_API int lai_jk_gradient(lai_engine* engine, const double* D, size_t nbf, double* grad);
/* Device D and grad; asynchronous on stream. */
LAI_API int lai_jk_gradient_device(lai_engine* engine, const double* d_D, double* d_grad, void* stream);

/* ---------------------------------------------------------------------------
 * Cartesian -> spherical (real solid harmonics, l <= 4).  The J/K path is
 * Cartesian, as in the reference; these move D in and J/K out of a spherical
 * basis: D_cart = T^T D_sph T, M_sph = T M_cart T^T, T = block-diag(C_l).
 * Replaces math::get_cart_to_sph_matrix / transform_2d
 * (include/libaccint/math/spherical_transform.hpp:20-70): same orders
 * (spherical m = 0, 1, -1, 2, -2, ...; Cartesian lx, then ly descending).
 * ------------------------------------------------------------------------- */
/* C_l, (2l+1) x (l+1)(l+2)/2 row-major. */
LAI_API int lai_cart_to_sph_matrix(int l, double* C);
/* Number of spherical functions of the basis (sum of 2l+1), or -1. */
LAI_API long lai_basis_nbf_spherical(const lai_basis* basis);
/* Host: M_sph (nsph x nsph) = T M_cart T^T;  D_cart (ncart x ncart) = T^T D_sph T. */
LAI_API int lai_cart_to_sph_2d(const lai_basis* basis, const double* M_cart, double* M_sph);
LAI_API int lai_sph_to_cart_density(const lai_basis* basis, const double* D_sph, double* D_cart);
/* The same on the engine's device (device pointers; asynchronous on stream). */
LAI_API int lai_cart_to_sph_2d_device(lai_engine* engine, const double* d_M_cart, double* d_M_sph,
                                      void* stream);
LAI_API int lai_sph_to_cart_density_device(lai_engine* engine, const double* d_D_sph, double* d_D_cart,
                                           void* stream);

/* ---------------------------------------------------------------------------
 * One-electron integrals over the engine's basis, full nbf x nbf row-major
 * (symmetric), same normalization and Cartesian order as J/K:
 *   LAI_OP_OVERLAP  S_ab = <a|b>
 *   LAI_OP_KINETIC  T_ab = <a|-1/2 nabla^2|b>
 *   LAI_OP_NUCLEAR  V_ab = -sum_C q_C <a|1/|r-C||b>   (point charges; atomic
 *                   numbers for the nuclei)
 *   LAI_OP_HCORE    T + V in one pass
 * Replaces Engine::compute_1e(OneElectronOperator, result) / compute_overlap_matrix /
 * compute_kinetic_matrix / compute_nuclear_matrix (include/libaccint/engine/
 * engine.hpp:166-201, 831-900; kernels src/host/kernels/{overlap,kinetic,nuclear}
 * _kernel.cpp).  charge_xyz [ncharge][3] (Bohr) and charge_q [ncharge] are host
 * arrays (NULL with ncharge = 0 for S and T).  Not available for batched engines.
 * ------------------------------------------------------------------------- */
/* ---------------------------------------------------------------------------
 * Density-fitting integrals.  aux: an auxiliary basis (any lai_basis, e.g. the
 * reference's built-in cc-pVDZ-RI shells), normalized like an orbital basis.
 *   lai_eri3c: T[(mu*nbf + nu)*naux + P] = (mu nu|P), both mu nu orders
 *              (the reference's ThreeCenterStorageFormat::abP,
 *              src/host/kernels/three_center_eri_kernel.cpp:273-362);
 *   lai_eri2c: V[P*naux + Q] = (P|Q) (compute_two_center_metric,
 *              src/host/kernels/two_center_coulomb_kernel.cpp:212-251).
 * Orbital shells up to f (g only paired with s), auxiliary shells up to g.  The
 * _device variants write device buffers asynchronously on stream.
 * ------------------------------------------------------------------------- */
LAI_API int lai_eri3c(lai_engine* engine, const lai_basis* aux, double* T);
LAI_API int lai_eri2c(lai_engine* engine, const lai_basis* aux, double* V);
LAI_API int lai_eri3c_device(lai_engine* engine, const lai_basis* aux, double* d_T, void* stream);
LAI_API int lai_eri2c_device(lai_engine* engine, const lai_basis* aux, double* d_V, void* stream);

#define LAI_OP_OVERLAP 0
#define LAI_OP_KINETIC 1
#define LAI_OP_NUCLEAR 2
#define LAI_OP_HCORE 3
LAI_API int lai_one_electron(lai_engine* engine, int op, int ncharge, const double* charge_xyz,
                             const double* charge_q, double* out);
/* Device output (nbf x nbf), asynchronous on stream (charges are staged through
 * the engine before the call returns). */
LAI_API int lai_one_electron_device(lai_engine* engine, int op, int ncharge, const double* charge_xyz,
                                    const double* charge_q, double* d_out, void* stream);

/* ---------------------------------------------------------------------------
 * Measurement helpers (no counterpart in the reference, which has no device
 * profiling of this path).
 * ------------------------------------------------------------------------- */
/* Per-launch device times of the last build made with opts.profile = 1.  For
 * launch i: ms[i]; algorithmic FLOP with every nonzero primitive quartet counted
 * (alg_flops) and with only the primitive quartets that passed the primitive
 * cut and were executed (alg_flops_executed); quartets[i]; primitive quartets
 * executed (prim_quartets[i]); class (la,lb,lc,ld) in lclass[4*i..4*i+3].
 * Any output may be NULL except ms.  Returns the launch count, or < 0. */
LAI_API int lai_jk_last_profile(lai_engine* engine, int capacity, double* ms, double* alg_flops,
                                double* alg_flops_executed, int64_t* quartets,
                                int64_t* prim_quartets, int* lclass);
/* n canonical screened quartets drawn uniformly (seeded) from all of the
 * engine's quartets, as shell indices [n][4] in the order the engine computes
 * them.  Used to time the reference CPU path on a bounded sample. */
LAI_API int lai_engine_sample_quartets(lai_engine* engine, int64_t n, uint64_t seed,
                                       int32_t* quartets);
/* Total canonical screened quartets of the engine. */
LAI_API int64_t lai_engine_quartet_count(lai_engine* engine);
/* Autotuner: times every thread-per-quartet class launch of the engine under a
 * few launch configurations (lanes per quartet 1..8, chunks per super-chunk 1, 4,
 * 16), and every other class launch under each kernel family that covers it
 * (warp-per-quartet, bra-sliced, tiled), on the device density d_D, and keeps the
 * fastest for later builds.
 * ms_before/ms_after (may be NULL): summed launch times with the built-in
 * heuristic and with the chosen configurations.  Synchronizes `stream`. */
LAI_API int lai_engine_autotune(lai_engine* engine, const double* d_D, void* stream, double* ms_before,
                                double* ms_after);
/* The launch table: per class-pair block, 10 ints: la, lb, lc, ld, bra and ket
 * primitive pairs per shell pair, quartets (capped at INT32_MAX), tuned lanes per
 * quartet (or -1 warp-per-quartet, -2 tiled, -3 bra-sliced kernel for the classes
 * outside the thread-per-quartet set) and chunks per super-chunk (0 = heuristic),
 * quartets / 1000.  Returns
 * the block count; rows may be NULL to query it. */
LAI_API int lai_engine_tune_table(lai_engine* engine, int capacity, int* rows);
/* FP64 FMA throughput of the device measured by a register-resident FMA loop
 * (TFLOP/s, 2 FLOP per FMA): the speed-of-light denominator of the FP64 path. */
LAI_API int lai_probe_fp64_peak(int device, double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* LIBACCINT_B200_H */
