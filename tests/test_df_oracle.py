"""CPU pins of the density-fitting checker (no GPU): the three- and two-centre
restatement (orc_eri_quartet with a unit s shell) in its point-charge limits
against the McMurchie-Davidson nuclear attraction and Coulomb's law, the fitted
J/K against the exact four-centre J/K they approximate, and the finding that the
reference's own DF path is unusable (its metric is not positive definite)."""
import numpy as np
import pytest

WATER = (np.array([8, 1, 1]), np.array([[0.0, 0.0, 0.0], [0.0, 1.43233673, -1.10866041],
                                        [0.0, -1.43233673, -1.10866041]]))


def _point_aux(lai, centers, gamma=1e12):
    return lai.BasisSet([lai.Shell(0, c, [gamma], [1.0]) for c in centers])


def test_three_center_point_charge_limit(lai, oracle):
    """(ab|P) of a very tight normalized s function P at C = q * (a|1/|r-C||b),
    q = (2 gamma/pi)^{3/4} (pi/gamma)^{3/2}: the MD nuclear attraction restatement."""
    Z, xyz = WATER
    b = lai.BasisSet.from_atoms(Z, xyz, "cc-pvdz")
    C = np.array([[0.3, -0.4, 1.1]])
    gamma = 1e12
    T = oracle.orc_eri3c(b, _point_aux(lai, C, gamma))[:, :, 0]
    q = (2 * gamma / np.pi) ** 0.75 * (np.pi / gamma) ** 1.5
    V = -oracle.orc_one_electron(b, 2, C, np.array([1.0]))
    assert np.max(np.abs(T / q - V)) < 1e-6 * np.max(np.abs(V))


def test_two_center_coulomb_law(lai, oracle):
    C = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 2.5], [1.0, 1.5, -0.5]])
    gamma = 1e12
    V = oracle.orc_eri2c(_point_aux(lai, C, gamma))
    q = (2 * gamma / np.pi) ** 0.75 * (np.pi / gamma) ** 1.5
    for i in range(3):
        for j in range(3):
            if i != j:
                assert abs(V[i, j] / q ** 2 - 1.0 / np.linalg.norm(C[i] - C[j])) < 1e-9


def test_fitted_jk_approximate_four_center(lai, oracle):
    """Exact DF (B = T L^-T) on the restatement's integrals against the four-centre
    J/K of the same density: the fitting error of the built-in cc-pVDZ-RI set."""
    Z, xyz = WATER
    b = lai.BasisSet.from_atoms(Z, xyz, "cc-pvdz")
    aux = lai.BasisSet.from_atoms(Z, xyz, "cc-pvdz-ri")
    T, V = oracle.orc_eri3c(b, aux), oracle.orc_eri2c(aux)
    assert np.min(np.linalg.eigvalsh(V)) > 0
    D = lai.molecules.random_density(b.nbf, 5, np.random.default_rng(0))
    J4, K4, _ = oracle.orc_jk(b, D, 0.0)
    J, K = oracle.df_jk_from_integrals(T, V, D)
    E4, E = lai.molecules.energy(D, J4, K4), lai.molecules.energy(D, J, K)
    assert abs(E - E4) < 5e-3 * abs(E4)
    assert np.max(np.abs(J - J4)) < 2e-2 and np.max(np.abs(K - K4)) < 5e-2


def test_reference_df_metric_is_not_positive_definite(lai, oracle):
    """Finding: the reference's two-centre metric (compute_two_center_metric) for
    water / cc-pVDZ-RI has negative eigenvalues and differs from (P|Q), so its
    DFFockBuilder raises in the Cholesky step (its DF tests skip on it)."""
    if oracle.reference() is None:
        pytest.skip("oracle/_ref not built")
    Z, xyz = WATER
    A = oracle.RefAux("cc-pVDZ-RI", Z, xyz)
    aux = lai.BasisSet.from_atoms(Z, xyz, "cc-pvdz-ri")
    shells = A.shells()
    assert [s[0] for s in shells] == [s.l for s in aux.shells]
    for s, c in zip(shells, aux.normalized_coefs()):   # same shells, same normalization
        assert np.allclose(s[3], c, rtol=1e-13)
    Vr = A.eri2c()
    assert np.min(np.linalg.eigvalsh(Vr)) < 0
    assert np.min(np.linalg.eigvalsh(oracle.orc_eri2c(aux))) > 0
    b = oracle.RefBasis(lai.BasisSet.from_atoms(Z, xyz, "cc-pvdz"))
    with pytest.raises(RuntimeError, match="not positive definite"):
        A.df_jk(b, np.eye(b.nbf))
