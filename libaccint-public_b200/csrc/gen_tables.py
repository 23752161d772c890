"""Generate the device lookup tables for the Boys function and the Rys roots.

Run once offline (``python gen_tables.py``); writes ``rys_tables.inc`` next to this
file.  The output is committed so the CUDA build needs neither mpmath nor time.

Everything is computed at 40 significant digits with mpmath from the definitions:

* Boys function  F_m(T) = int_0^1 t^{2m} exp(-T t^2) dt
  = gamma(m+1/2, T) / (2 T^{m+1/2})  (lower incomplete gamma), F_m(0) = 1/(2m+1).
* Rys quadrature for n roots: the n-point Gauss rule of the measure
  exp(-T t^2) dt on t in [0,1] in the variable u = t^2, i.e. sum_r w_r p(u_r) =
  int_0^1 p(t^2) exp(-T t^2) dt for deg p < 2n.  Computed here from the exact
  moments F_k(T) by the Chebyshev algorithm (recurrence coefficients), then the
  eigen-decomposition of the Jacobi matrix (Golub-Welsch).  At 40 digits the
  conditioning of the moment map (about 1e13 for n = 9) is harmless.

Tables written:

* ``BOYS_GRID`` : F_m(k*0.1) for k = 0..BOYS_NGRID-1 and m = 0..BOYS_NM-1.  The device
  evaluates F_m(T) by a Taylor series about the nearest grid point,
  F_m(T) = sum_j F_{m+j}(T0) (T0-T)^j / j!, |T-T0| <= 0.05, 10 terms (truncation
  below 1e-17 relative).  Above BOYS_TMAX the asymptotic form is exact to 1e-17.
* ``RYS_COEF`` : for each n in [2, RYS_NMAX], unit intervals [k, k+1) of T up to
  RYS_TMAX[n]; on each interval each root u_r(T) and weight w_r(T) is a degree-11
  polynomial in x = 2(T-k)-1 in [-1,1], obtained as the Chebyshev interpolant on
  12 Chebyshev points and converted to the monomial basis (Horner on the device;
  the coefficients decay geometrically, so Horner is stable).  Layout per
  interval: [j][r] -> (a_j of u_r, a_j of w_r) as interleaved double pairs,
  j = degree 0..11 -- one 16-byte load per (root, degree).
  Beyond RYS_TMAX[n] the half-range Gauss-Hermite limit is used:
  u_r = x_r^2 / T, w_r = W_r / sqrt(T) with (x_r, W_r) the positive nodes and
  weights of the 2n-point Gauss-Hermite rule (``RYS_HERM``).  RYS_TMAX[n] is the
  smallest integer beyond which that limit is within 4e-16 relative for all roots
  and weights (checked on a grid of T).
"""
import os
import sys
from multiprocessing import Pool

import mpmath as mp

mp.mp.dps = 40

RYS_NMAX = 9
DEG = 11
BOYS_NGRID = 400
BOYS_DT = mp.mpf(1) / 10
BOYS_NM = 16          # F_0..F_15 stored per grid point (orders used <= 2n-1+10)


def boys(kmax, T):
    T = mp.mpf(T)
    if T == 0:
        return [mp.mpf(1) / (2 * k + 1) for k in range(kmax + 1)]
    return [mp.gammainc(k + mp.mpf(1) / 2, 0, T) / (2 * T ** (k + mp.mpf(1) / 2))
            for k in range(kmax + 1)]


def rys(n, T):
    mu = boys(2 * n - 1, T)
    nm = 2 * n
    sp = [mp.mpf(0)] * nm
    s = list(mu)
    a = [mu[1] / mu[0]]
    b = [mu[0]]
    for k in range(1, n):
        sn = [mp.mpf(0)] * nm
        for l in range(k, nm - k):
            sn[l] = s[l + 1] - a[k - 1] * s[l] - b[k - 1] * sp[l]
        a.append(sn[k + 1] / sn[k] - s[k] / s[k - 1])
        b.append(sn[k] / s[k - 1])
        sp, s = s, sn
    J = mp.zeros(n, n)
    for i in range(n):
        J[i, i] = a[i]
        if i + 1 < n:
            J[i, i + 1] = J[i + 1, i] = mp.sqrt(b[i + 1])
    E, Q = mp.eigsy(J)
    order = sorted(range(n), key=lambda i: E[i])
    return [E[i] for i in order], [b[0] * Q[0, i] ** 2 for i in order]


def hermite_half(n):
    """Positive nodes x_r and weights W_r of the 2n-point Gauss-Hermite rule."""
    m = 2 * n
    J = mp.zeros(m, m)
    for k in range(1, m):
        J[k - 1, k] = J[k, k - 1] = mp.sqrt(mp.mpf(k) / 2)
    E, Q = mp.eigsy(J)
    pairs = sorted([(E[i], mp.sqrt(mp.pi) * Q[0, i] ** 2) for i in range(m) if E[i] > 0])
    return [p[0] for p in pairs], [p[1] for p in pairs]


def asym_ok(n, T, herm):
    x, W = herm
    r, w = rys(n, T)
    err = 0
    for i in range(n):
        ua = x[i] ** 2 / T
        wa = W[i] / mp.sqrt(T)
        err = max(err, abs(r[i] - ua) / ua, abs(w[i] - wa) / wa)
    return err


def find_tmax(n):
    herm = hermite_half(n)
    T = 30
    while True:
        # require the limit to hold at T and on a few points beyond
        if all(asym_ok(n, mp.mpf(T) + d, herm) < mp.mpf('4e-16') for d in (0, 0.5, 3, 10)):
            return T
        T += 1


def cheb_to_monomial(c):
    """Chebyshev series coefficients -> monomial coefficients (exact in mp)."""
    D = len(c) - 1
    Tk = [[mp.mpf(1)], [mp.mpf(0), mp.mpf(1)]]
    for k in range(2, D + 1):
        prev, prev2 = Tk[k - 1], Tk[k - 2]
        nxt = [mp.mpf(0)] * (k + 1)
        for i, v in enumerate(prev):
            nxt[i + 1] += 2 * v
        for i, v in enumerate(prev2):
            nxt[i] -= v
        Tk.append(nxt)
    a = [mp.mpf(0)] * (D + 1)
    for k in range(D + 1):
        for i, v in enumerate(Tk[k]):
            a[i] += c[k] * v
    return a


def fit_interval(args):
    n, k = args
    N = DEG + 1
    xs = [mp.cos(mp.pi * (j + mp.mpf(1) / 2) / N) for j in range(N)]
    vals = [rys(n, k + (x + 1) / 2) for x in xs]
    out = []   # out[j][r] = (a_j(u_r), a_j(w_r))
    funcs = []
    for r in range(n):
        for which in (0, 1):
            y = [v[which][r] for v in vals]
            c = []
            for m in range(N):
                s = sum(y[j] * mp.cos(m * mp.pi * (j + mp.mpf(1) / 2) / N) for j in range(N))
                c.append(s * (1 if m == 0 else 2) / N)
            funcs.append(cheb_to_monomial(c))
    for j in range(N):
        row = []
        for r in range(n):
            row.append((funcs[2 * r][j], funcs[2 * r + 1][j]))
        out.append(row)
    return n, k, out


def boys_row(k):
    return k, boys(BOYS_NM - 1, k * BOYS_DT)


def fmt(v):
    return mp.nstr(v, 20, min_fixed=0, max_fixed=0, strip_zeros=False)


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    with Pool(os.cpu_count()) as pool:
        tmax = dict(zip(range(2, RYS_NMAX + 1), pool.map(find_tmax, range(2, RYS_NMAX + 1))))
        print("RYS_TMAX", tmax, file=sys.stderr)
        jobs = [(n, k) for n in range(2, RYS_NMAX + 1) for k in range(tmax[n])]
        fits = pool.map(fit_interval, jobs, chunksize=4)
        brows = pool.map(boys_row, range(BOYS_NGRID))
    fits.sort(key=lambda t: (t[0], t[1]))
    lines = ["// Generated by gen_tables.py -- do not edit.", "#pragma once", ""]
    lines.append(f"#define RYS_NMAX {RYS_NMAX}")
    lines.append(f"#define RYS_DEG {DEG}")
    lines.append(f"#define BOYS_NGRID {BOYS_NGRID}")
    lines.append(f"#define BOYS_NM {BOYS_NM}")
    lines.append("#define BOYS_DT 0.1")
    lines.append(f"#define BOYS_TMAX {float(BOYS_NGRID * BOYS_DT) - 0.05}")
    tm = [0, 0] + [tmax[n] for n in range(2, RYS_NMAX + 1)]
    lines.append("static const int RYS_TMAX_H[RYS_NMAX + 1] = {" + ", ".join(map(str, tm)) + "};")
    off = [0, 0]
    acc = 0
    for n in range(2, RYS_NMAX + 1):
        off.append(acc)
        acc += tmax[n] * (DEG + 1) * n * 2
    lines.append("static const int RYS_OFF_H[RYS_NMAX + 1] = {" + ", ".join(map(str, off)) + "};")
    lines.append(f"#define RYS_COEF_LEN {acc}")
    lines.append("static const double RYS_COEF_H[RYS_COEF_LEN] = {")
    for n, k, out in fits:
        vals = []
        for j in range(DEG + 1):
            for r in range(n):
                vals += [out[j][r][0], out[j][r][1]]
        lines.append("  " + ", ".join(fmt(v) for v in vals) + ",  // n=%d T in [%d,%d)" % (n, k, k + 1))
    lines.append("};")
    # Gauss-Hermite half-range limit, flattened by n: x_r^2 and W_r for r < n.
    hx, hw, hoff = [], [], [0, 0]
    for n in range(2, RYS_NMAX + 1):
        hoff.append(len(hx))
        x, W = hermite_half(n)
        hx += [xi ** 2 for xi in x]
        hw += W
    lines.append("static const int RYS_HOFF_H[RYS_NMAX + 1] = {" + ", ".join(map(str, hoff)) + "};")
    lines.append(f"#define RYS_HERM_LEN {len(hx)}")
    lines.append("static const double RYS_HERM_X2_H[RYS_HERM_LEN] = {" + ", ".join(fmt(v) for v in hx) + "};")
    lines.append("static const double RYS_HERM_W_H[RYS_HERM_LEN] = {" + ", ".join(fmt(v) for v in hw) + "};")
    lines.append("static const double BOYS_GRID_H[BOYS_NGRID * BOYS_NM] = {")
    brows.sort()
    for k, row in brows:
        lines.append("  " + ", ".join(fmt(v) for v in row) + ",")
    lines.append("};")
    with open(os.path.join(here, "rys_tables.inc"), "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
