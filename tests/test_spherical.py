"""Cartesian -> spherical transformation (host side; no GPU): the generated C_l
against the reference's tables, against the defining properties of real solid
harmonics, and the block-diagonal transforms against a dense numpy T."""
import numpy as np
import pytest


def _dfact(n):  # (n)!! for odd n >= -1
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def _cart_list(l):
    return [(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)]


@pytest.mark.parametrize("l", range(5))
def test_matrix_matches_reference(lai, oracle, l):
    if oracle.reference() is None:
        pytest.skip("oracle/_ref not built")
    C = lai.cart_to_sph_matrix(l)
    assert np.max(np.abs(C - oracle.ref_cart_to_sph(l))) < 1e-14


@pytest.mark.parametrize("l", range(5))
def test_matrix_is_orthonormal_solid_harmonics(lai, l):
    """Rows are orthonormal under the overlap of Cartesian components normalized like
    x^l (angular integrals (a+a'-1)!!(b+b'-1)!!(c+c'-1)!!/(2l-1)!!), and each row is
    a harmonic polynomial (zero Laplacian)."""
    C = lai.cart_to_sph_matrix(l)
    comps = _cart_list(l)
    S = np.zeros((len(comps), len(comps)))
    for i, a in enumerate(comps):
        for j, b in enumerate(comps):
            s = [a[k] + b[k] for k in range(3)]
            if all(v % 2 == 0 for v in s):
                S[i, j] = np.prod([_dfact(v - 1) for v in s]) / _dfact(2 * l - 1)
    assert np.max(np.abs(C @ S @ C.T - np.eye(2 * l + 1))) < 1e-13
    # Laplacian of sum_c C[m,c] x^a y^b z^c, as coefficients on degree l-2 monomials
    if l >= 2:
        low = {c: i for i, c in enumerate(_cart_list(l - 2))}
        for m in range(2 * l + 1):
            lap = np.zeros(len(low))
            for j, (a, b, c) in enumerate(comps):
                for k, e in enumerate((a, b, c)):
                    if e >= 2:
                        t = [a, b, c]
                        t[k] -= 2
                        lap[low[tuple(t)]] += C[m, j] * e * (e - 1)
            assert np.max(np.abs(lap)) < 1e-12


def _dense_T(lai, basis):
    n, ns = basis.nbf, basis.nbf_spherical
    T = np.zeros((ns, n))
    r = c = 0
    for s in basis.shells:
        C = lai.cart_to_sph_matrix(s.l)
        T[r:r + C.shape[0], c:c + C.shape[1]] = C
        r += C.shape[0]
        c += C.shape[1]
    return T


def test_transforms_match_dense(lai):
    Z = np.array([6, 1, 8], dtype=np.int32)
    xyz = np.array([[0.0, 0.0, 0.0], [1.1, 0.7, -0.9], [-2.1, 0.4, 0.3]])
    b = lai.BasisSet.from_atoms(Z, xyz, "cc-pvqz")  # s..g
    assert max(s.l for s in b.shells) == 4
    T = _dense_T(lai, b)
    rng = np.random.default_rng(1)
    M = rng.standard_normal((b.nbf, b.nbf))
    assert np.max(np.abs(b.cart_to_sph(M) - T @ M @ T.T)) < 1e-11
    Ds = rng.standard_normal((b.nbf_spherical, b.nbf_spherical))
    assert np.max(np.abs(b.sph_to_cart_density(Ds) - T.T @ Ds @ T)) < 1e-11
    assert lai.lib().lai_basis_nbf_spherical(b.handle()) == b.nbf_spherical


def test_bad_l_is_an_error(lai):
    with pytest.raises(lai.LibAccIntError):
        lai.cart_to_sph_matrix(5)
