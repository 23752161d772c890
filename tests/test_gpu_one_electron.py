"""One-electron kernels and the device RHF driver (GPU): S, T, V against the
PySCF matrices of the reference's tests/integration/test_one_electron.cpp and
against the oracle up to g shells; RHF energies against the PySCF values of
tests/integration/test_hf_energy.cpp and against the oracle's RHF."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


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
def test_matrices_match_pyscf(lai, name):
    d = golden("one_electron_sto3g.npz")
    b = _basis(lai, d, name)
    e = lai.Engine(b)
    atoms = list(zip(d[name + "_charge_q"], d[name + "_charge_xyz"]))
    up = name.upper()
    S, T, V = e.compute_overlap_matrix(), e.compute_kinetic_matrix(), e.compute_nuclear_matrix(atoms)
    assert np.max(np.abs(S - d[up + "_S_REF"])) < 1e-12
    assert np.max(np.abs(T - d[up + "_T_REF"])) < 1e-12
    assert np.max(np.abs(V - d[up + "_V_REF"])) < 1e-12
    assert np.max(np.abs(np.diag(S) - 1.0)) < 1e-12
    H = e.compute_core_hamiltonian(atoms)
    assert np.max(np.abs(H - (T + V))) < 1e-12
    assert np.array_equal(H, H.T) and np.array_equal(S, S.T)


@pytest.mark.parametrize("basis_name,Z", [("cc-pvdz", [8, 1, 1]), ("cc-pvtz", [6, 1, 8]),
                                          ("cc-pvqz", [8, 1]), ("aug-cc-pvdz", [8, 1, 1])])
def test_matrices_match_oracle_all_classes(lai, oracle, basis_name, Z):
    """Every (la, lb) class up to (g|g) against the McMurchie-Davidson restatement."""
    Z = np.array(Z)
    rng = np.random.default_rng(len(Z) + len(basis_name))
    xyz = rng.uniform(-1.6, 1.6, size=(len(Z), 3))
    b = lai.BasisSet.from_atoms(Z, xyz, basis_name)
    e = lai.Engine(b)
    q = Z.astype(float)
    got = [e.compute_overlap_matrix(), e.compute_kinetic_matrix(), e.compute_nuclear_matrix()]
    for kind, g in enumerate(got):
        ref = oracle.orc_one_electron(b, kind, xyz, q)
        scale = max(1.0, np.max(np.abs(ref)))
        assert np.max(np.abs(g - ref)) < 1e-12 * scale, (basis_name, kind, np.max(np.abs(g - ref)))
    H = e.compute_core_hamiltonian()
    assert np.max(np.abs(H - got[1] - got[2])) < 1e-12 * max(1.0, np.max(np.abs(H)))


def test_point_charges_are_additive(lai):
    """V of two charge sets equals the sum of their separate V (linearity)."""
    Z = np.array([8, 1, 1])
    xyz = np.array([[0.0, 0.0, 0.0], [0.0, 1.43, -1.1], [0.0, -1.43, -1.1]])
    b = lai.BasisSet.from_atoms(Z, xyz, "cc-pvdz")
    e = lai.Engine(b)
    c1 = [(0.7, (3.0, 0.5, -1.0)), (-0.4, (-2.0, 1.5, 2.0))]
    c2 = [(1.3, (0.1, -3.0, 0.7))]
    V12 = e.compute_nuclear_matrix(c1 + c2)
    V1, V2 = e.compute_nuclear_matrix(c1), e.compute_nuclear_matrix(c2)
    assert np.max(np.abs(V12 - V1 - V2)) < 1e-13
    assert np.max(np.abs(e.compute_nuclear_matrix([]))) == 0.0


def test_device_variant_and_errors(lai):
    import torch
    Z = np.array([8, 1, 1])
    xyz = np.array([[0.0, 0.0, 0.0], [0.0, 1.43, -1.1], [0.0, -1.43, -1.1]])
    b = lai.BasisSet.from_atoms(Z, xyz, "cc-pvdz")
    e = lai.Engine(b)
    n = b.nbf
    d = torch.full((n, n), np.nan, dtype=torch.float64, device="cuda")
    e.one_electron_device("kinetic", d.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy(), e.compute_kinetic_matrix())
    with pytest.raises(lai.LibAccIntError):
        lai._lib.check(lai.lib().lai_one_electron(e._h, 7, 0, None, None, d.data_ptr()))
    with pytest.raises(lai.LibAccIntError):
        lai._lib.check(lai.lib().lai_one_electron(e._h, 2, 3, None, None, d.data_ptr()))


@pytest.mark.parametrize("key", ["hf_h2", "hf_h2o", "hf_ch4"])
def test_rhf_matches_pyscf_energy(lai, key):
    """The reference's HF quality gate: RHF/STO-3G energies within 1e-10 of PySCF."""
    d = golden("one_electron_sto3g.npz")
    Z, xyz = d[key + "_Z"], d[key + "_xyz"]
    atoms = [lai.Atom(z, r) for z, r in zip(Z, xyz)]
    b = lai.BasisSet.from_atoms(Z, xyz, "sto-3g")
    res = lai.scf.run_rhf(atoms, b, int(d[key + "_nelec"]))
    assert res.converged and res.iterations < 50
    assert abs(res.total_energy - float(d[key + "_energy"])) < 1e-10
    if key == "hf_h2":
        assert res.iterations < 20


def test_rhf_water_dimer_ccpvdz_matches_oracle(lai, oracle):
    """(H2O)2/cc-pVDZ (d shells): the device RHF against the numpy RHF on the
    oracle's S, T, V and J/K (compiled reference J/K when present)."""
    w = lai.workloads.make("h2o2_ccpvdz")
    b = w.basis
    q = np.asarray(w.Z, dtype=float)
    res = lai.scf.run_rhf(b.atoms, b, int(q.sum()))
    assert res.converged
    S = oracle.orc_one_electron(b, 0)
    H = oracle.orc_one_electron(b, 1) + oracle.orc_one_electron(b, 2, w.xyz, q)
    if oracle.reference() is not None:
        R = oracle.RefBasis(b)
        jk = lambda D: R.jk_full(D)[:2]  # noqa: E731
    else:
        jk = lambda D: oracle.orc_jk(b, D, 0.0)[:2]  # noqa: E731
    E, it, conv = oracle.orc_rhf(S, H, jk, int(q.sum()) // 2, oracle.nuclear_repulsion(w.Z, w.xyz))
    assert conv
    assert abs(res.total_energy - E) < 1e-9, (res.total_energy, E)


def test_rhf_mixed_precision_energy(lai):
    """The mixed-precision J/K build (FP32 below a 1e-7 cut) inside the SCF: the
    converged energy stays within 1e-8 of the FP64 one."""
    w = lai.workloads.make("h2o4_ccpvdz")
    b = w.basis
    r64 = lai.scf.RHF(b).run(energy_threshold=1e-10, density_threshold=1e-7)
    r32 = lai.scf.RHF(b, fp32_cut=1e-7).run(energy_threshold=1e-10, density_threshold=1e-7)
    assert r64.converged and r32.converged
    assert abs(r64.total_energy - r32.total_energy) < 1e-8
