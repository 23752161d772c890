"""Seeded synthetic molecules and densities of the benchmark workloads.

The reference measures on no public data set; these generators define the inputs
(all coordinates in Bohr, seeds through numpy.random.default_rng):

* water: O at the site, H at O + r (0, +-sin(t/2), -cos(t/2)) with r = 1.809,
  t = 104.52 deg, rotated about O by a uniform random rotation (QR of a 3x3
  N(0,1) matrix, signs fixed so R has positive diagonal, det +1), then moved to
  the grid site 5.5 (i, j, k) plus a U(-0.5, 0.5)^3 jitter.  Sites are visited in
  (i, j, k) order with k fastest; per site the rotation is drawn before the jitter.
* density: D = C C^T with C an nbf x nocc matrix of N(0, 1/nbf) entries (drawn
  after the geometry from the same generator unless a seed is given).
* alkane: all-trans CnH2n+2, C-C 2.91, C-H 2.06, tetrahedral angles, backbone in
  the xy plane.
"""
import itertools
import math

import numpy as np

R_OH = 1.809
THETA_HOH = math.radians(104.52)
GRID = 5.5
JITTER = 0.5


def random_rotation(rng):
    A = rng.standard_normal((3, 3))
    Q, R = np.linalg.qr(A)
    Q = Q * np.sign(np.diag(R))
    if np.linalg.det(Q) < 0:
        Q[:, 0] = -Q[:, 0]
    return Q


def water_cluster(dims, rng):
    """Z (int32) and xyz (n,3) of waters on a dims[0] x dims[1] x dims[2] grid."""
    h = np.array([[0.0, math.sin(THETA_HOH / 2), -math.cos(THETA_HOH / 2)],
                  [0.0, -math.sin(THETA_HOH / 2), -math.cos(THETA_HOH / 2)]]) * R_OH
    Z, xyz = [], []
    for site in itertools.product(range(dims[0]), range(dims[1]), range(dims[2])):
        Rm = random_rotation(rng)
        o = GRID * np.array(site, dtype=np.float64) + rng.uniform(-JITTER, JITTER, 3)
        Z += [8, 1, 1]
        xyz += [o, o + Rm @ h[0], o + Rm @ h[1]]
    return np.array(Z, dtype=np.int32), np.array(xyz)


def water_cluster_n(n, rng):
    """n waters on the smallest near-cubic grid that holds them (first n sites)."""
    nx = math.ceil(round(n ** (1.0 / 3.0), 9))
    ny = max(1, math.ceil(round(math.sqrt(n / nx), 9)))
    nz = math.ceil(n / (nx * ny))
    Z, xyz = water_cluster((nx, ny, nz), rng)
    return Z[: 3 * n], xyz[: 3 * n]


def alkane(n_carbon=12, r_cc=2.91, r_ch=2.06):
    """All-trans CnH2n+2 (carbons first, then hydrogens carbon by carbon)."""
    tet = math.acos(-1.0 / 3.0)
    dx = r_cc * math.sin(tet / 2)
    dy = r_cc * math.cos(tet / 2)
    C = [np.array([k * dx, (k % 2) * dy, 0.0]) for k in range(-1, n_carbon + 1)]
    carbons = C[1:-1]
    Hs = []
    half = tet / 2
    for k in range(1, n_carbon + 1):
        c, a, b = C[k], C[k - 1], C[k + 1]
        ua = (a - c) / np.linalg.norm(a - c)
        ub = (b - c) / np.linalg.norm(b - c)
        bis = -(ua + ub)
        bis /= np.linalg.norm(bis)
        nz = np.array([0.0, 0.0, 1.0])
        for sgn in (1.0, -1.0):
            d = bis * math.cos(half) + sgn * nz * math.sin(half)
            Hs.append(c + r_ch * d)
        if k == 1:
            Hs.append(c + r_ch * ua)
        if k == n_carbon:
            Hs.append(c + r_ch * ub)
    Z = [6] * n_carbon + [1] * len(Hs)
    return np.array(Z, dtype=np.int32), np.array(carbons + Hs)


def random_density(nbf, nocc, rng):
    Cm = rng.normal(0.0, 1.0 / math.sqrt(nbf), size=(nbf, nocc))
    return Cm @ Cm.T


def energy(D, J, K):
    """E = tr(DJ)/2 - tr(DK)/4."""
    return 0.5 * float(np.sum(D * J)) - 0.25 * float(np.sum(D * K))
