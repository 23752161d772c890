"""CPU checks of the one-electron / RHF checkers against the reference's golden
data (no GPU): the McMurchie-Davidson restatement of S, T, V and the compiled
reference against the PySCF matrices of tests/integration/test_one_electron.cpp,
the two against each other up to g shells, and the numpy RHF driver against the
PySCF energies of tests/integration/test_hf_energy.cpp."""
import numpy as np
import pytest

from conftest import golden


def _basis(lai, d, name):
    l, ctr, npr = d[name + "_l"], d[name + "_center"], d[name + "_nprim"]
    ex, co = d[name + "_exps"], d[name + "_coefs"]
    shells, off = [], 0
    for s in range(len(l)):
        k = int(npr[s])
        shells.append(lai.Shell(int(l[s]), ctr[s], ex[off:off + k], co[off:off + k]))
        off += k
    return lai.BasisSet(shells)


@pytest.mark.parametrize("name", ["h2", "h2o"])
def test_restatement_matches_pyscf_matrices(lai, oracle, name):
    d = golden("one_electron_sto3g.npz")
    b = _basis(lai, d, name)
    xyz, q = d[name + "_charge_xyz"], d[name + "_charge_q"]
    up = name.upper()
    assert np.max(np.abs(oracle.orc_one_electron(b, 0) - d[up + "_S_REF"])) < 1e-12
    assert np.max(np.abs(oracle.orc_one_electron(b, 1) - d[up + "_T_REF"])) < 1e-12
    assert np.max(np.abs(oracle.orc_one_electron(b, 2, xyz, q) - d[up + "_V_REF"])) < 1e-12


@pytest.mark.parametrize("name", ["h2", "h2o"])
def test_reference_matches_pyscf_matrices(lai, oracle, name):
    if oracle.reference() is None:
        pytest.skip("oracle/_ref not built")
    d = golden("one_electron_sto3g.npz")
    b = _basis(lai, d, name)
    R = oracle.RefBasis(b)
    xyz, q = d[name + "_charge_xyz"], d[name + "_charge_q"]
    up = name.upper()
    assert np.max(np.abs(R.one_electron(0) - d[up + "_S_REF"])) < 1e-12
    assert np.max(np.abs(R.one_electron(1) - d[up + "_T_REF"])) < 1e-12
    assert np.max(np.abs(R.one_electron(2, xyz, q) - d[up + "_V_REF"])) < 1e-12


@pytest.mark.parametrize("basis_name", ["cc-pvdz", "cc-pvqz"])
def test_restatement_matches_reference_high_l(lai, oracle, basis_name):
    """Up to g shells (cc-pVQZ oxygen): the two checkers agree element by element."""
    if oracle.reference() is None:
        pytest.skip("oracle/_ref not built")
    Z = np.array([8, 1])
    xyz = np.array([[0.0, 0.0, 0.0], [0.3, 1.2, -1.4]])
    b = lai.BasisSet.from_atoms(Z, xyz, basis_name)
    R = oracle.RefBasis(b)
    q = Z.astype(float)
    for kind in (0, 1, 2):
        a = oracle.orc_one_electron(b, kind, xyz, q)
        r = R.one_electron(kind, xyz, q)
        scale = max(1.0, np.max(np.abs(r)))
        assert np.max(np.abs(a - r)) < 1e-12 * scale, kind
        assert np.max(np.abs(a - a.T)) < 1e-12 * scale


@pytest.mark.parametrize("key", ["hf_h2", "hf_h2o", "hf_ch4"])
def test_oracle_rhf_matches_pyscf_energy(lai, oracle, key):
    d = golden("one_electron_sto3g.npz")
    Z, xyz = d[key + "_Z"], d[key + "_xyz"]
    b = lai.BasisSet.from_atoms(Z, xyz, "sto-3g")
    q = Z.astype(float)
    S = oracle.orc_one_electron(b, 0)
    H = oracle.orc_one_electron(b, 1) + oracle.orc_one_electron(b, 2, xyz, q)
    enuc = oracle.nuclear_repulsion(Z, xyz)
    E, it, conv = oracle.orc_rhf(S, H, lambda D: oracle.orc_jk(b, D, 0.0)[:2], int(d[key + "_nelec"]) // 2, enuc)
    assert conv and it < 50
    assert abs(E - float(d[key + "_energy"])) < 1e-10


def test_nuclear_repulsion_matches_pyscf(lai, oracle):
    d = golden("one_electron_sto3g.npz")
    assert abs(oracle.nuclear_repulsion(d["hf_h2o_Z"], d["hf_h2o_xyz"]) - float(d["h2o_enuc"])) < 1e-12
    atoms = [lai.Atom(z, r) for z, r in zip(d["hf_h2o_Z"], d["hf_h2o_xyz"])]
    assert abs(lai.scf.nuclear_repulsion(atoms) - float(d["h2o_enuc"])) < 1e-12


def test_point_charges_accepts_reference_forms(lai):
    class PCP:
        x, y, z, charge = [0.0, 1.0], [0.0, 2.0], [0.5, 3.0], [8.0, 1.0]
    xyz, q = lai.point_charges(PCP())
    assert xyz.shape == (2, 3) and list(q) == [8.0, 1.0] and list(xyz[1]) == [1.0, 2.0, 3.0]
    xyz2, q2 = lai.point_charges([(8, (0.0, 0.0, 0.5)), lai.Atom(1, [1.0, 2.0, 3.0])])
    assert np.array_equal(xyz, xyz2) and np.array_equal(q, q2)
