/*
 * Test infrastructure only -- the CPU ORACLE for the J/K hot path.
 *
 * A plain-C restatement of the reference (LibAccInt v0.1.0-alpha.2) algorithm
 * for Rys-quadrature ERIs over contracted Cartesian Gaussians and their 8-fold
 * symmetric digestion into J and K.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load this library; the product never does.
 *
 * Precision: Boys moments and Rys roots/weights are computed in IEEE binary128
 * (__float128, libquadmath) and rounded to double; everything downstream runs in
 * double like the reference.  That makes the roots independent of (and more
 * accurate than) both the reference's FP64 Chebyshev+QL+Newton path and the
 * CUDA path's fitted tables, so the oracle can arbitrate between them.
 *
 * Functions and the reference code each one restates:
 *   orc_boys           src/shared/math/boys_function.cpp:253-303 (F_0..F_m(T));
 *                      here: positive series for T<=50, erf + upward recursion above.
 *   orc_rys            src/shared/math/rys_quadrature.cpp:455-513 (rys_compute):
 *                      moments F_k(T) -> recurrence coefficients (Chebyshev
 *                      algorithm on ordinary moments, in binary128 instead of the
 *                      reference's modified moments in double, :24-66) -> roots as
 *                      eigenvalues of the Jacobi matrix (Sturm bisection in x87
 *                      extended precision, then binary128 Newton on the
 *                      characteristic polynomial, instead of implicit QL, :75-157)
 *                      -> Christoffel weights.
 *                      Roots clamped to [1e-14, 1-1e-14] as at :497-500.
 *   orc_normalize      src/shared/basis/shell.cpp:32-113 (primitive normalization
 *                      and (l,0,0) self-overlap rescaling).
 *   orc_eri_quartet    src/host/kernels/eri_kernel.cpp:104-164 (build_2d_rys: VRR on
 *                      a then c, HRR to b then d) and :168-381 (primitive loops,
 *                      prefactor 2 pi^{5/2}/(zeta eta sqrt(zeta+eta)) K_AB K_CD,
 *                      assembly, norm_correction of
 *                      include/libaccint/kernels/norm_correction.hpp:28-34).
 *   orc_schwarz        src/shared/screening/schwarz_bounds.cpp:20-59.
 *   orc_jk_sym         include/libaccint/engine/engine.hpp:1806-1861 (canonical
 *                      i<=j, k>=i, l>=(k==i?j:k) loop with Schwarz test) and
 *                      src/shared/consumers/fock_builder.cpp:123-222
 *                      (accumulate_symmetric: 8 permutations with degeneracy flags).
 *
 * Cartesian order inside a shell: lx descending, then ly descending
 * (include/libaccint/math/cartesian_indices.hpp:26-36).
 */
#include <math.h>
#include <quadmath.h>
#include <stdlib.h>
#include <string.h>

typedef __float128 q_t;

#define ORC_MAX_L 6           /* shells up to l=6 (gradient tests shift l by +1) */
#define ORC_MAX_ROOTS 13
#define ORC_MAX_MOM (2 * ORC_MAX_ROOTS)

/* ------------------------------------------------------------------------- */
/* Boys function F_m(T) = int_0^1 t^{2m} exp(-T t^2) dt, binary128.           */
/* ------------------------------------------------------------------------- */
static void boys_q(int mmax, q_t T, q_t *F) {
    if (T <= 50) {
        /* F_m(T) = exp(-T) sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)); all terms
           positive, so no cancellation.  Evaluate at mmax, recurse downward. */
        q_t term = 1.0Q / (2 * mmax + 1), sum = term;
        for (int k = 1; k < 2000; ++k) {
            term *= 2 * T / (2 * mmax + 2 * k + 1);
            sum += term;
            if (term < 1e-38Q * sum) break;
        }
        q_t e = expq(-T);
        F[mmax] = e * sum;
        for (int m = mmax; m >= 1; --m) F[m - 1] = (2 * T * F[m] + e) / (2 * m - 1);
    } else {
        /* upward recursion is stable while (2m+1)/(2T) < 1, true for m <= 2*13 */
        q_t e = expq(-T);
        F[0] = 0.5Q * sqrtq(M_PIq / T) * erfq(sqrtq(T));
        for (int m = 0; m < mmax; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) / (2 * T);
    }
}

void orc_boys(int mmax, double T, double *out) {
    q_t F[64];
    if (mmax > 63) mmax = 63;
    boys_q(mmax, (q_t)T, F);
    for (int m = 0; m <= mmax; ++m) out[m] = (double)F[m];
}

/* ------------------------------------------------------------------------- */
/* Rys roots and weights in binary128.                                        */
/* Measure: d mu(u) on [0,1] with moments mu_k = F_k(T) (u = t^2).            */
/* ------------------------------------------------------------------------- */
static void chebyshev_recurrence(int n, const q_t *mu, q_t *alpha, q_t *beta) {
    /* Chebyshev algorithm on ordinary moments (Gautschi's sigma table). */
    q_t sig_prev[ORC_MAX_MOM + 2], sig[ORC_MAX_MOM + 2], sig_new[ORC_MAX_MOM + 2];
    const int nm = 2 * n;
    for (int l = 0; l < nm; ++l) { sig_prev[l] = 0; sig[l] = mu[l]; }
    alpha[0] = mu[1] / mu[0];
    beta[0] = mu[0];
    for (int k = 1; k < n; ++k) {
        for (int l = k; l < nm - k; ++l)
            sig_new[l] = sig[l + 1] - alpha[k - 1] * sig[l] - beta[k - 1] * sig_prev[l];
        alpha[k] = sig_new[k + 1] / sig_new[k] - sig[k] / sig[k - 1];
        beta[k] = sig_new[k] / sig[k - 1];
        for (int l = 0; l < nm; ++l) { sig_prev[l] = sig[l]; sig[l] = sig_new[l]; }
    }
}

/* Monic orthogonal polynomial p_n(x) and derivative via the recurrence. */
static void charpoly(int n, const q_t *a, const q_t *b, q_t x, q_t *p, q_t *dp) {
    q_t pm1 = 0, p0 = 1, dpm1 = 0, dp0 = 0;
    for (int k = 0; k < n; ++k) {
        q_t p1 = (x - a[k]) * p0 - (k ? b[k] * pm1 : 0);
        q_t dp1 = p0 + (x - a[k]) * dp0 - (k ? b[k] * dpm1 : 0);
        pm1 = p0; p0 = p1; dpm1 = dp0; dp0 = dp1;
    }
    *p = p0;
    *dp = dp0;
}

static int sturm_count_ld(int n, const long double *a, const long double *b, long double x) {
    int cnt = 0;
    long double d = a[0] - x;
    if (d < 0) cnt++;
    for (int k = 1; k < n; ++k) {
        if (d == 0) d = 1e-4000L;
        d = a[k] - x - b[k] / d;
        if (d < 0) cnt++;
    }
    return cnt;
}

static void rys_q(int n, q_t T, q_t *roots, q_t *weights) {
    q_t mu[ORC_MAX_MOM + 2], a[ORC_MAX_ROOTS], b[ORC_MAX_ROOTS];
    long double al[ORC_MAX_ROOTS], bl[ORC_MAX_ROOTS];
    boys_q(2 * n - 1, T, mu);
    chebyshev_recurrence(n, mu, a, b);
    for (int k = 0; k < n; ++k) { al[k] = (long double)a[k]; bl[k] = (long double)b[k]; }
    for (int r = 0; r < n; ++r) {
        /* r-th smallest eigenvalue: Sturm bisection in extended precision to
           bracket it, then Newton on the binary128 characteristic polynomial. */
        long double lo = 0, hi = 1;
        for (int it = 0; it < 64; ++it) {
            long double mid = 0.5L * (lo + hi);
            if (sturm_count_ld(n, al, bl, mid) > r) hi = mid; else lo = mid;
        }
        q_t x = 0.5Q * ((q_t)lo + (q_t)hi);
        for (int it = 0; it < 4; ++it) {
            q_t p, dp;
            charpoly(n, a, b, x, &p, &dp);
            if (dp == 0) break;
            x = x - p / dp;
        }
        roots[r] = x;
        /* Christoffel number: w = 1 / sum_k P_k(x)^2 with orthonormal P_k. */
        q_t pm1 = 0, p0 = 1 / sqrtq(b[0]), s = p0 * p0;
        for (int k = 0; k + 1 < n; ++k) {
            q_t p1 = ((x - a[k]) * p0 - (k ? sqrtq(b[k]) * pm1 : 0)) / sqrtq(b[k + 1]);
            s += p1 * p1;
            pm1 = p0; p0 = p1;
        }
        weights[r] = 1 / s;
    }
}

void orc_rys(int n, double T, double *roots, double *weights) {
    q_t r[ORC_MAX_ROOTS], w[ORC_MAX_ROOTS];
    rys_q(n, (q_t)T, r, w);
    for (int i = 0; i < n; ++i) {
        double u = (double)r[i];
        if (u < 1e-14) u = 1e-14;
        if (u > 1.0 - 1e-14) u = 1.0 - 1e-14;
        roots[i] = u;
        weights[i] = (double)w[i];
    }
}

/* ------------------------------------------------------------------------- */
/* Shell normalization (PySCF cart convention, unit (l,0,0) self-overlap).   */
/* ------------------------------------------------------------------------- */
static double dfact_odd(int l) { /* (2l-1)!! */
    double r = 1;
    for (int k = 2 * l - 1; k > 1; k -= 2) r *= k;
    return r;
}

void orc_normalize(int l, int nprim, const double *exps, const double *coefs, double *out) {
    for (int p = 0; p < nprim; ++p)
        out[p] = coefs[p] * pow(2 * exps[p] / M_PI, 0.75) * pow(4 * exps[p], 0.5 * l) /
                 sqrt(dfact_odd(l));
    double s = 0;
    for (int p = 0; p < nprim; ++p)
        for (int q = 0; q < nprim; ++q) {
            double z = exps[p] + exps[q];
            double ov = pow(M_PI / z, 1.5);
            for (int k = 0; k < l; ++k) ov *= 0.5 / z;
            s += out[p] * out[q] * ov;
        }
    double sc = 1 / sqrt(s);
    for (int p = 0; p < nprim; ++p) out[p] *= sc;
}

/* ------------------------------------------------------------------------- */
/* One contracted shell quartet (ab|cd), out[a][b][c][d] row-major.           */
/* ------------------------------------------------------------------------- */
static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

static void cart_list(int l, int (*c)[3]) {
    int k = 0;
    for (int x = l; x >= 0; --x)
        for (int y = l - x; y >= 0; --y) { c[k][0] = x; c[k][1] = y; c[k][2] = l - x - y; ++k; }
}

/* 2D table I[a][b][c][d] for one direction and one root. */
static void table2d(int la, int lb, int lc, int ld, double pa, double qc, double ab, double cd,
                    double b10, double b01, double b00, double *I) {
    const int da = la + lb + 1, db = lb + 1, dc = lc + ld + 1, dd = ld + 1;
#define IX(a, b, c, d) I[(((a) * db + (b)) * dc + (c)) * dd + (d)]
    memset(I, 0, sizeof(double) * da * db * dc * dd);
    IX(0, 0, 0, 0) = 1.0;
    for (int a = 0; a < la + lb; ++a)
        IX(a + 1, 0, 0, 0) = pa * IX(a, 0, 0, 0) + (a ? a * b10 * IX(a - 1, 0, 0, 0) : 0.0);
    for (int c = 0; c < lc + ld; ++c)
        for (int a = 0; a <= la + lb; ++a)
            IX(a, 0, c + 1, 0) = qc * IX(a, 0, c, 0) + (c ? c * b01 * IX(a, 0, c - 1, 0) : 0.0) +
                                 (a ? a * b00 * IX(a - 1, 0, c, 0) : 0.0);
    for (int b = 0; b < lb; ++b)
        for (int a = 0; a <= la + lb - b - 1; ++a)
            for (int c = 0; c <= lc + ld; ++c)
                IX(a, b + 1, c, 0) = IX(a + 1, b, c, 0) + ab * IX(a, b, c, 0);
    for (int d = 0; d < ld; ++d)
        for (int a = 0; a <= la; ++a)
            for (int b = 0; b <= lb; ++b)
                for (int c = 0; c <= lc + ld - d - 1; ++c)
                    IX(a, b, c, d + 1) = IX(a, b, c + 1, d) + cd * IX(a, b, c, d);
#undef IX
}

/* Shell descriptors: l[4], centers[4][3], nprim[4], exps/coefs (normalized). */
int orc_eri_quartet(const int *l, const double *ctr, const int *nprim, const double *const *exps,
                    const double *const *coefs, double *out) {
    const int la = l[0], lb = l[1], lc = l[2], ld = l[3];
    if (la > ORC_MAX_L || lb > ORC_MAX_L || lc > ORC_MAX_L || ld > ORC_MAX_L) return -1;
    const double *A = ctr, *B = ctr + 3, *C = ctr + 6, *D = ctr + 9;
    const int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
    int ca[28][3], cb[28][3], cc[28][3], cdl[28][3];
    cart_list(la, ca); cart_list(lb, cb); cart_list(lc, cc); cart_list(ld, cdl);
    const int nroots = (la + lb + lc + ld) / 2 + 1;
    const int da = la + lb + 1, db = lb + 1, dc = lc + ld + 1, dd = ld + 1;
    const int tsz = da * db * dc * dd;
    double *Ix = malloc(sizeof(double) * tsz * 3), *Iy = Ix + tsz, *Iz = Iy + tsz;
    const long nout = (long)na * nb * nc * nd;
    memset(out, 0, sizeof(double) * nout);
    const double pi52 = M_PI * M_PI * sqrt(M_PI);
    double AB[3], CD[3];
    for (int x = 0; x < 3; ++x) { AB[x] = A[x] - B[x]; CD[x] = C[x] - D[x]; }
    double roots[ORC_MAX_ROOTS], wts[ORC_MAX_ROOTS];
#define TI(T, a, b, c, d) T[(((a) * db + (b)) * dc + (c)) * dd + (d)]
    for (int p = 0; p < nprim[0]; ++p)
        for (int q = 0; q < nprim[1]; ++q) {
            const double al = exps[0][p], be = exps[1][q];
            const double zeta = al + be;
            double P[3], ab2 = 0;
            for (int x = 0; x < 3; ++x) { P[x] = (al * A[x] + be * B[x]) / zeta; ab2 += AB[x] * AB[x]; }
            const double Kab = exp(-al * be / zeta * ab2);
            for (int r = 0; r < nprim[2]; ++r)
                for (int s = 0; s < nprim[3]; ++s) {
                    const double ga = exps[2][r], de = exps[3][s];
                    const double eta = ga + de;
                    double Q[3], cd2 = 0, PQ[3], pq2 = 0;
                    for (int x = 0; x < 3; ++x) {
                        Q[x] = (ga * C[x] + de * D[x]) / eta;
                        cd2 += CD[x] * CD[x];
                        PQ[x] = P[x] - Q[x];
                        pq2 += PQ[x] * PQ[x];
                    }
                    const double Kcd = exp(-ga * de / eta * cd2);
                    const double rho = zeta * eta / (zeta + eta);
                    const double T = rho * pq2;
                    const double pref = 2.0 * pi52 / (zeta * eta * sqrt(zeta + eta)) * Kab * Kcd;
                    const double coef = coefs[0][p] * coefs[1][q] * coefs[2][r] * coefs[3][s] * pref;
                    orc_rys(nroots, T, roots, wts);
                    for (int k = 0; k < nroots; ++k) {
                        const double u = roots[k];
                        const double b10 = 0.5 / zeta * (1.0 - rho / zeta * u);
                        const double b01 = 0.5 / eta * (1.0 - rho / eta * u);
                        const double b00 = 0.5 / (zeta + eta) * u;
                        double *T3[3] = {Ix, Iy, Iz};
                        for (int x = 0; x < 3; ++x) {
                            const double pa = (P[x] - A[x]) - rho / zeta * u * PQ[x];
                            const double qc = (Q[x] - C[x]) + rho / eta * u * PQ[x];
                            table2d(la, lb, lc, ld, pa, qc, AB[x], CD[x], b10, b01, b00, T3[x]);
                        }
                        const double wc = coef * wts[k];
                        long o = 0;
                        for (int ia = 0; ia < na; ++ia)
                            for (int ib = 0; ib < nb; ++ib)
                                for (int ic = 0; ic < nc; ++ic)
                                    for (int id = 0; id < nd; ++id, ++o)
                                        out[o] += wc *
                                            TI(Ix, ca[ia][0], cb[ib][0], cc[ic][0], cdl[id][0]) *
                                            TI(Iy, ca[ia][1], cb[ib][1], cc[ic][1], cdl[id][1]) *
                                            TI(Iz, ca[ia][2], cb[ib][2], cc[ic][2], cdl[id][2]);
                    }
                }
        }
#undef TI
    long o = 0;
    for (int ia = 0; ia < na; ++ia)
        for (int ib = 0; ib < nb; ++ib)
            for (int ic = 0; ic < nc; ++ic)
                for (int id = 0; id < nd; ++id, ++o) {
                    double den = dfact_odd(ca[ia][0]) * dfact_odd(ca[ia][1]) * dfact_odd(ca[ia][2]) *
                                 dfact_odd(cb[ib][0]) * dfact_odd(cb[ib][1]) * dfact_odd(cb[ib][2]) *
                                 dfact_odd(cc[ic][0]) * dfact_odd(cc[ic][1]) * dfact_odd(cc[ic][2]) *
                                 dfact_odd(cdl[id][0]) * dfact_odd(cdl[id][1]) * dfact_odd(cdl[id][2]);
                    out[o] /= sqrt(den);
                }
    free(Ix);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Basis-level helpers: shells given as flat arrays, coefficients normalized. */
/* ------------------------------------------------------------------------- */
typedef struct {
    int n;
    const int *l, *nprim;
    const double *ctr, *exps, *coefs;
    long *poff, *foff;
} basis_t;

static void basis_init(basis_t *b, int n, const int *l, const int *nprim, const double *ctr,
                       const double *exps, const double *coefs) {
    b->n = n; b->l = l; b->nprim = nprim; b->ctr = ctr; b->exps = exps; b->coefs = coefs;
    b->poff = malloc(sizeof(long) * (n + 1));
    b->foff = malloc(sizeof(long) * (n + 1));
    b->poff[0] = b->foff[0] = 0;
    for (int s = 0; s < n; ++s) {
        b->poff[s + 1] = b->poff[s] + nprim[s];
        b->foff[s + 1] = b->foff[s] + ncart(l[s]);
    }
}

static void basis_free(basis_t *b) { free(b->poff); free(b->foff); }

static int quartet(const basis_t *b, int i, int j, int k, int m, double *out) {
    int l[4] = {b->l[i], b->l[j], b->l[k], b->l[m]};
    int np[4] = {b->nprim[i], b->nprim[j], b->nprim[k], b->nprim[m]};
    double ctr[12];
    memcpy(ctr, b->ctr + 3 * i, 24); memcpy(ctr + 3, b->ctr + 3 * j, 24);
    memcpy(ctr + 6, b->ctr + 3 * k, 24); memcpy(ctr + 9, b->ctr + 3 * m, 24);
    const double *e[4] = {b->exps + b->poff[i], b->exps + b->poff[j], b->exps + b->poff[k],
                          b->exps + b->poff[m]};
    const double *c[4] = {b->coefs + b->poff[i], b->coefs + b->poff[j], b->coefs + b->poff[k],
                          b->coefs + b->poff[m]};
    return orc_eri_quartet(l, ctr, np, e, c, out);
}

/* One contracted quartet of a basis by shell indices. */
int orc_basis_quartet(int n, const int *l, const int *nprim, const double *ctr, const double *exps,
                      const double *coefs, int i, int j, int k, int m, double *out) {
    basis_t b;
    basis_init(&b, n, l, nprim, ctr, exps, coefs);
    int rc = quartet(&b, i, j, k, m, out);
    basis_free(&b);
    return rc;
}

static void scatter_sym(const basis_t *b, const int *l, long nbf, int i, int j, int k, int m,
                        const double *g, const double *D, double *J, double *K);

/* J/K contributions of listed canonical quartets (shell indices q[4t..4t+3],
   i >= j, k >= l, ij >= kl in the canonical loop's sense), ADDED to J and K. */
void orc_jk_list(int n, const int *l, const int *nprim, const double *ctr, const double *exps,
                 const double *coefs, const double *D, long nq, const int *q, double *J, double *K) {
    basis_t b;
    basis_init(&b, n, l, nprim, ctr, exps, coefs);
    const long nbf = b.foff[n];
    double *g = malloc(sizeof(double) * 28 * 28 * 28 * 28);
    for (long t = 0; t < nq; ++t) {
        const int *x = q + 4 * t;
        quartet(&b, x[0], x[1], x[2], x[3], g);
        scatter_sym(&b, l, nbf, x[0], x[1], x[2], x[3], g, D, J, K);
    }
    free(g);
    basis_free(&b);
}

/* Many contracted quartets (shell indices q[4t..4t+3]), blocks concatenated in
   order into out (each [a][b][c][d]); OpenMP over quartets.  Returns 0. */
int orc_basis_quartets(int n, const int *l, const int *nprim, const double *ctr, const double *exps,
                       const double *coefs, long nq, const int *q, double *out) {
    basis_t b;
    basis_init(&b, n, l, nprim, ctr, exps, coefs);
    long *off = malloc(sizeof(long) * (nq + 1));
    off[0] = 0;
    for (long t = 0; t < nq; ++t)
        off[t + 1] = off[t] + (long)ncart(l[q[4 * t]]) * ncart(l[q[4 * t + 1]]) *
                                  ncart(l[q[4 * t + 2]]) * ncart(l[q[4 * t + 3]]);
    int rc = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(| : rc)
    for (long t = 0; t < nq; ++t)
        rc |= quartet(&b, q[4 * t], q[4 * t + 1], q[4 * t + 2], q[4 * t + 3], out + off[t]);
    free(off);
    basis_free(&b);
    return rc;
}

/* Schwarz bounds Q[i*n+j] = sqrt(max_ab |(ab|ab)|). */
int orc_schwarz(int n, const int *l, const int *nprim, const double *ctr, const double *exps,
                const double *coefs, double *Q) {
    basis_t b;
    basis_init(&b, n, l, nprim, ctr, exps, coefs);
    double *buf = malloc(sizeof(double) * 28 * 28 * 28 * 28);
    for (int i = 0; i < n; ++i)
        for (int j = i; j < n; ++j) {
            quartet(&b, i, j, i, j, buf);
            const int ni = ncart(l[i]), nj = ncart(l[j]);
            double mx = 0;
            for (int a = 0; a < ni; ++a)
                for (int c = 0; c < nj; ++c) {
                    double v = fabs(buf[((long)(a * nj + c) * ni + a) * nj + c]);
                    if (v > mx) mx = v;
                }
            Q[i * n + j] = Q[j * n + i] = sqrt(mx);
        }
    free(buf);
    basis_free(&b);
    return 0;
}

/* 8-fold symmetric scatter of one canonical quartet's block g into J, K
   (fock_builder.cpp:123-222 accumulate_symmetric). */
static void scatter_sym(const basis_t *b, const int *l, long nbf, int i, int j, int k, int m,
                        const double *g, const double *D, double *J, double *K) {
    const int ij = (i == j), kl = (k == m), bk = (i == k && j == m);
    const int na = ncart(l[i]), nb = ncart(l[j]), nc = ncart(l[k]), nd = ncart(l[m]);
    long o = 0;
    for (int a = 0; a < na; ++a)
        for (int bb = 0; bb < nb; ++bb)
            for (int c = 0; c < nc; ++c)
                for (int d = 0; d < nd; ++d, ++o) {
                    const long mu = b->foff[i] + a, nu = b->foff[j] + bb;
                    const long la = b->foff[k] + c, si = b->foff[m] + d;
                    const double v = g[o];
                    J[mu * nbf + nu] += v * D[la * nbf + si];
                    K[mu * nbf + la] += v * D[nu * nbf + si];
                    if (!kl) {
                        J[mu * nbf + nu] += v * D[si * nbf + la];
                        K[mu * nbf + si] += v * D[nu * nbf + la];
                    }
                    if (!ij) {
                        J[nu * nbf + mu] += v * D[la * nbf + si];
                        K[nu * nbf + la] += v * D[mu * nbf + si];
                    }
                    if (!ij && !kl) {
                        J[nu * nbf + mu] += v * D[si * nbf + la];
                        K[nu * nbf + si] += v * D[mu * nbf + la];
                    }
                    if (!bk) {
                        J[la * nbf + si] += v * D[mu * nbf + nu];
                        K[la * nbf + mu] += v * D[nu * nbf + si];
                        if (!ij) {
                            J[la * nbf + si] += v * D[nu * nbf + mu];
                            K[la * nbf + nu] += v * D[mu * nbf + si];
                        }
                        if (!kl) {
                            J[si * nbf + la] += v * D[mu * nbf + nu];
                            K[si * nbf + mu] += v * D[nu * nbf + la];
                        }
                        if (!ij && !kl) {
                            J[si * nbf + la] += v * D[nu * nbf + mu];
                            K[si * nbf + nu] += v * D[mu * nbf + la];
                        }
                    }
                }
}

/* Canonical screened loop + 8-fold symmetric scatter (serial).  D symmetric,
   row-major nbf x nbf; J and K are overwritten.  Returns the number of
   canonical quartets computed. */
long orc_jk_sym(int n, const int *l, const int *nprim, const double *ctr, const double *exps,
                const double *coefs, const double *D, double *J, double *K, double thr) {
    basis_t b;
    basis_init(&b, n, l, nprim, ctr, exps, coefs);
    const long nbf = b.foff[n];
    double *Q = malloc(sizeof(double) * n * n);
    orc_schwarz(n, l, nprim, ctr, exps, coefs, Q);
    double *g = malloc(sizeof(double) * 28 * 28 * 28 * 28);
    memset(J, 0, sizeof(double) * nbf * nbf);
    memset(K, 0, sizeof(double) * nbf * nbf);
    long count = 0;
    for (int i = 0; i < n; ++i)
        for (int j = i; j < n; ++j)
            for (int k = i; k < n; ++k)
                for (int m = (k == i ? j : k); m < n; ++m) {
                    if (Q[i * n + j] * Q[k * n + m] < thr) continue;
                    quartet(&b, i, j, k, m, g);
                    ++count;
                    scatter_sym(&b, l, nbf, i, j, k, m, g, D, J, K);
                }
    free(g);
    free(Q);
    basis_free(&b);
    return count;
}

/* ------------------------------------------------------------------------- */
/* One-electron integrals by McMurchie-Davidson Hermite expansion: a method   */
/* independent of the Obara-Saika/Rys recurrences of both the reference       */
/* (src/host/kernels/{overlap,kinetic,nuclear}_kernel.cpp) and the CUDA path, */
/* with the Boys function F_n(T) in binary128 (boys_q).                       */
/*   E^{i+1,j}_t = E^{ij}_{t-1}/(2p) + PA E^{ij}_t + (t+1) E^{ij}_{t+1}        */
/*   E^{i,j+1}_t = E^{ij}_{t-1}/(2p) + PB E^{ij}_t + (t+1) E^{ij}_{t+1}        */
/*   s_ij = E^{ij}_0 sqrt(pi/p) exp(-mu X_AB^2)                               */
/*   t_ij = 1/2 [ i j s_{i-1,j-1} - 2 a j s_{i+1,j-1} - 2 b i s_{i-1,j+1}     */
/*               + 4 a b s_{i+1,j+1} ]   (symmetric derivative form)          */
/*   V_ab = -q (2 pi/p) K_AB sum_tuv E_t E_u E_v R_tuv,                       */
/*   R^n_000 = (-2p)^n F_n(p PC^2), R^n_{t+1,u,v} = t R^{n+1}_{t-1,u,v}       */
/*             + PC_x R^{n+1}_{t,u,v} (same for u, v).                        */
/* ------------------------------------------------------------------------- */
#define MD_L (2 * ORC_MAX_L + 3)
static void md_e(int imax, int jmax, double pa, double pb, double p, double E[MD_L][MD_L][2 * MD_L]) {
    memset(E, 0, sizeof(double) * MD_L * MD_L * 2 * MD_L);
    E[0][0][0] = 1.0;
    const double h = 0.5 / p;
    for (int i = 0; i <= imax; ++i)
        for (int j = 0; j <= jmax; ++j) {
            if (i == 0 && j == 0) continue;
            for (int t = 0; t <= i + j; ++t) {
                double v;
                if (i > 0) {
                    const double (*e)[2 * MD_L] = E[i - 1];
                    v = pa * e[j][t] + (t + 1) * e[j][t + 1] + (t > 0 ? h * e[j][t - 1] : 0.0);
                } else {
                    const double *e = E[i][j - 1];
                    v = pb * e[t] + (t + 1) * e[t + 1] + (t > 0 ? h * e[t - 1] : 0.0);
                }
                E[i][j][t] = v;
            }
        }
}

/* Hermite Coulomb integrals R_{tuv} (n = 0) for t+u+v <= L. */
static void md_r(int L, double p, double x, double y, double z, double *R /* [L+1]^3 */) {
    const int d = L + 1;
    double *W = calloc((size_t)(L + 1) * d * d * d, sizeof(double));
#define RW(n, t, u, v) W[(((n) * d + (t)) * d + (u)) * d + (v)]
    q_t F[ORC_MAX_MOM + 8];
    boys_q(L, (q_t)(p * (x * x + y * y + z * z)), F);
    double m = 1.0;
    for (int n = 0; n <= L; ++n) { RW(n, 0, 0, 0) = m * (double)F[n]; m *= -2.0 * p; }
    for (int n = L - 1; n >= 0; --n)
        for (int s = 1; s <= L - n; ++s)
            for (int t = 0; t <= s; ++t)
                for (int u = 0; u <= s - t; ++u) {
                    const int v = s - t - u;
                    double r;
                    if (t > 0) r = x * RW(n + 1, t - 1, u, v) + (t > 1 ? (t - 1) * RW(n + 1, t - 2, u, v) : 0.0);
                    else if (u > 0) r = y * RW(n + 1, t, u - 1, v) + (u > 1 ? (u - 1) * RW(n + 1, t, u - 2, v) : 0.0);
                    else r = z * RW(n + 1, t, u, v - 1) + (v > 1 ? (v - 1) * RW(n + 1, t, u, v - 2) : 0.0);
                    RW(n, t, u, v) = r;
                }
    for (int t = 0; t <= L; ++t)
        for (int u = 0; u <= L; ++u)
            for (int v = 0; v <= L; ++v) R[(t * d + u) * d + v] = (t + u + v <= L) ? RW(0, t, u, v) : 0.0;
#undef RW
    free(W);
}

/* kind 0 overlap, 1 kinetic, 2 nuclear (charges xyz [nc][3], q [nc]); out nbf x nbf. */
int orc_one_electron(int n, const int *l, const int *nprim, const double *ctr, const double *exps,
                     const double *coefs, int kind, int nc, const double *xyz, const double *q,
                     double *out) {
    basis_t b;
    basis_init(&b, n, l, nprim, ctr, exps, coefs);
    const long nbf = b.foff[n];
    static double E[3][MD_L][MD_L][2 * MD_L];
    for (int s1 = 0; s1 < n; ++s1)
        for (int s2 = 0; s2 < n; ++s2) {
            const int la = l[s1], lb = l[s2], na = ncart(la), nb = ncart(lb);
            if (la > ORC_MAX_L || lb > ORC_MAX_L) { basis_free(&b); return -1; }
            int ca[28][3], cb[28][3];
            cart_list(la, ca);
            cart_list(lb, cb);
            const double *A = ctr + 3 * s1, *B = ctr + 3 * s2;
            double *blk = calloc((size_t)na * nb, sizeof(double));
            for (int i1 = 0; i1 < nprim[s1]; ++i1)
                for (int i2 = 0; i2 < nprim[s2]; ++i2) {
                    const double al = exps[b.poff[s1] + i1], be = exps[b.poff[s2] + i2];
                    const double c = coefs[b.poff[s1] + i1] * coefs[b.poff[s2] + i2];
                    const double p = al + be, mu = al * be / p;
                    double P[3], K = 1.0;
                    for (int x = 0; x < 3; ++x) {
                        P[x] = (al * A[x] + be * B[x]) / p;
                        K *= exp(-mu * (A[x] - B[x]) * (A[x] - B[x]));
                        md_e(la + 1, lb + 1, P[x] - A[x], P[x] - B[x], p, E[x]);
                    }
                    const double sp = sqrt(M_PI / p);
                    if (kind == 0 || kind == 1) {
                        for (int ia = 0; ia < na; ++ia)
                            for (int ib = 0; ib < nb; ++ib) {
                                double s[3], t[3];
                                for (int x = 0; x < 3; ++x) {
                                    const int i = ca[ia][x], j = cb[ib][x];
                                    s[x] = E[x][i][j][0] * sp;
                                    if (kind == 1) {
                                        double v = 4 * al * be * E[x][i + 1][j + 1][0];
                                        if (j > 0) v -= 2 * al * j * E[x][i + 1][j - 1][0];
                                        if (i > 0) v -= 2 * be * i * E[x][i - 1][j + 1][0];
                                        if (i > 0 && j > 0) v += i * j * E[x][i - 1][j - 1][0];
                                        t[x] = 0.5 * v * sp;
                                    }
                                }
                                double v = kind == 0 ? s[0] * s[1] * s[2]
                                                     : t[0] * s[1] * s[2] + s[0] * t[1] * s[2] + s[0] * s[1] * t[2];
                                blk[ia * nb + ib] += c * K * v;
                            }
                    } else {
                        const int L = la + lb, d = L + 1;
                        double *R = malloc(sizeof(double) * d * d * d);
                        for (int ic = 0; ic < nc; ++ic) {
                            md_r(L, p, P[0] - xyz[3 * ic], P[1] - xyz[3 * ic + 1], P[2] - xyz[3 * ic + 2], R);
                            const double f = -q[ic] * 2 * M_PI / p * c * K;
                            for (int ia = 0; ia < na; ++ia)
                                for (int ib = 0; ib < nb; ++ib) {
                                    const int ix = ca[ia][0], jx = cb[ib][0], iy = ca[ia][1], jy = cb[ib][1],
                                              iz = ca[ia][2], jz = cb[ib][2];
                                    double v = 0.0;
                                    for (int t = 0; t <= ix + jx; ++t)
                                        for (int u = 0; u <= iy + jy; ++u)
                                            for (int w = 0; w <= iz + jz; ++w)
                                                v += E[0][ix][jx][t] * E[1][iy][jy][u] * E[2][iz][jz][w] *
                                                     R[(t * d + u) * d + w];
                                    blk[ia * nb + ib] += f * v;
                                }
                        }
                        free(R);
                    }
                }
            for (int ia = 0; ia < na; ++ia)
                for (int ib = 0; ib < nb; ++ib) {
                    const double nrm = 1.0 / sqrt(dfact_odd(ca[ia][0]) * dfact_odd(ca[ia][1]) * dfact_odd(ca[ia][2]) *
                                                  dfact_odd(cb[ib][0]) * dfact_odd(cb[ib][1]) * dfact_odd(cb[ib][2]));
                    out[(b.foff[s1] + ia) * nbf + b.foff[s2] + ib] = blk[ia * nb + ib] * nrm;
                }
            free(blk);
        }
    basis_free(&b);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Density-fitting integrals through orc_eri_quartet with a unit s function   */
/* (exponent 0, coefficient 1) as the fourth shell: (ab|P) = (ab|P u),        */
/* (P|Q) = (P u|Q u).  Orbital shells (no, lo, npo, co_, eo, cfo) and         */
/* auxiliary shells (nx, ...) with normalized coefficients.                    */
/*   T[(a*nbf + b)*naux + P] (both a b orders), V[P*naux + Q].                */
/* Reference: compute_three_center_tensor (abP) and compute_two_center_metric */
/* (src/host/kernels/three_center_eri_kernel.cpp:273-362,                      */
/*  src/host/kernels/two_center_coulomb_kernel.cpp:212-251).                  */
/* ------------------------------------------------------------------------- */
static const double ORC_ZERO = 0.0, ORC_ONE = 1.0;

int orc_eri3c(int no, const int *lo, const int *npo, const double *co, const double *eo, const double *cfo,
              int nx, const int *lx, const int *npx, const double *cx, const double *ex, const double *cfx,
              double *T) {
    basis_t bo, bx;
    basis_init(&bo, no, lo, npo, co, eo, cfo);
    basis_init(&bx, nx, lx, npx, cx, ex, cfx);
    const long nbf = bo.foff[no], naux = bx.foff[nx];
    double *blk = malloc(sizeof(double) * 28 * 28 * 28);
    int rc = 0;
    for (int a = 0; a < no && !rc; ++a)
        for (int b = a; b < no && !rc; ++b)
            for (int p = 0; p < nx && !rc; ++p) {
                const int l[4] = {lo[a], lo[b], lx[p], 0};
                const int np[4] = {npo[a], npo[b], npx[p], 1};
                double ctr[12];
                memcpy(ctr, co + 3 * a, 24); memcpy(ctr + 3, co + 3 * b, 24);
                memcpy(ctr + 6, cx + 3 * p, 24); memcpy(ctr + 9, cx + 3 * p, 24);
                const double *e[4] = {eo + bo.poff[a], eo + bo.poff[b], ex + bx.poff[p], &ORC_ZERO};
                const double *c[4] = {cfo + bo.poff[a], cfo + bo.poff[b], cfx + bx.poff[p], &ORC_ONE};
                rc = orc_eri_quartet(l, ctr, np, e, c, blk);
                const int na = ncart(l[0]), nb = ncart(l[1]), nq = ncart(l[2]);
                for (int i = 0; i < na; ++i)
                    for (int j = 0; j < nb; ++j)
                        for (int k = 0; k < nq; ++k) {
                            const double v = blk[(i * nb + j) * nq + k];
                            const long ia = bo.foff[a] + i, jb = bo.foff[b] + j, kp = bx.foff[p] + k;
                            T[(ia * nbf + jb) * naux + kp] = v;
                            T[(jb * nbf + ia) * naux + kp] = v;
                        }
            }
    free(blk);
    basis_free(&bo);
    basis_free(&bx);
    return rc;
}

int orc_eri2c(int nx, const int *lx, const int *npx, const double *cx, const double *ex, const double *cfx,
              double *V) {
    basis_t bx;
    basis_init(&bx, nx, lx, npx, cx, ex, cfx);
    const long naux = bx.foff[nx];
    double *blk = malloc(sizeof(double) * 28 * 28);
    int rc = 0;
    for (int p = 0; p < nx && !rc; ++p)
        for (int q = p; q < nx && !rc; ++q) {
            const int l[4] = {lx[p], 0, lx[q], 0};
            const int np[4] = {npx[p], 1, npx[q], 1};
            double ctr[12];
            memcpy(ctr, cx + 3 * p, 24); memcpy(ctr + 3, cx + 3 * p, 24);
            memcpy(ctr + 6, cx + 3 * q, 24); memcpy(ctr + 9, cx + 3 * q, 24);
            const double *e[4] = {ex + bx.poff[p], &ORC_ZERO, ex + bx.poff[q], &ORC_ZERO};
            const double *c[4] = {cfx + bx.poff[p], &ORC_ONE, cfx + bx.poff[q], &ORC_ONE};
            rc = orc_eri_quartet(l, ctr, np, e, c, blk);
            const int na = ncart(l[0]), nq = ncart(l[2]);
            for (int i = 0; i < na; ++i)
                for (int k = 0; k < nq; ++k) {
                    const double v = blk[i * nq + k];
                    V[(bx.foff[p] + i) * naux + bx.foff[q] + k] = v;
                    V[(bx.foff[q] + k) * naux + bx.foff[p] + i] = v;
                }
        }
    free(blk);
    basis_free(&bx);
    return rc;
}
