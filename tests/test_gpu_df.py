"""Density fitting on the GPU: three- and two-centre kernels against the
restatement for every class up to (ff|g) and (g|g), the device DF J/K against
numpy fitting of the restatement's integrals, and DF-RHF against four-centre RHF."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev_ints(lai, eng, aux):
    import torch
    n, na = eng.basis.nbf, aux.nbf
    T = torch.empty((n, n, na), dtype=torch.float64, device="cuda")
    V = torch.empty((na, na), dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    lai._lib.check(lai.lib().lai_eri3c_device(eng._h, aux.handle(), ctypes.c_void_p(T.data_ptr()),
                                              ctypes.c_void_p(s)))
    lai._lib.check(lai.lib().lai_eri2c_device(eng._h, aux.handle(), ctypes.c_void_p(V.data_ptr()),
                                              ctypes.c_void_p(s)))
    torch.cuda.synchronize()
    return T.cpu().numpy(), V.cpu().numpy()


@pytest.mark.parametrize("orb,auxname,Z", [("cc-pvdz", "cc-pvdz-ri", [8, 1, 1]),
                                           ("cc-pvtz", "def2-tzvp-jkfit", [6, 8, 1]),
                                           ("6-31g", "def2-svp-jkfit", [7, 1])])
def test_integrals_match_restatement(lai, oracle, orb, auxname, Z):
    Z = np.array(Z)
    xyz = np.random.default_rng(len(Z)).uniform(-1.5, 1.5, size=(len(Z), 3))
    b = lai.BasisSet.from_atoms(Z, xyz, orb)
    aux = lai.BasisSet.from_atoms(Z, xyz, auxname)
    eng = lai.Engine(b)
    T, V = _dev_ints(lai, eng, aux)
    To, Vo = oracle.orc_eri3c(b, aux), oracle.orc_eri2c(aux)
    assert np.max(np.abs(T - To)) < 1e-12 * max(1.0, np.max(np.abs(To)))
    assert np.max(np.abs(V - Vo)) < 1e-12 * max(1.0, np.max(np.abs(Vo)))
    # host variants give the same numbers
    Th = np.zeros_like(T)
    lai._lib.check(lai.lib().lai_eri3c(eng._h, aux.handle(), Th.ctypes.data))
    assert np.array_equal(Th, T)


def test_df_jk_matches_numpy_fitting(lai, oracle):
    import torch
    w = lai.workloads.make("h2o2_ccpvdz")
    aux = lai.BasisSet.from_atoms(w.Z, w.xyz, "cc-pvdz-ri")
    eng = lai.Engine(w.basis)
    df = lai.df.DFFockBuilder(eng, aux)
    df.set_density(w.D)
    J = df.compute_coulomb().cpu().numpy()
    K = df.compute_exchange().cpu().numpy()
    Jo, Ko = oracle.df_jk_from_integrals(oracle.orc_eri3c(w.basis, aux), oracle.orc_eri2c(aux), w.D)
    assert np.max(np.abs(J - Jo)) < 1e-10 and np.max(np.abs(K - Ko)) < 1e-10
    F = df.compute().cpu().numpy()
    assert np.max(np.abs(F - (J - 0.5 * K))) < 1e-12
    # an indefinite density (K from both signs of its spectrum)
    D2 = w.D - 0.3 * np.eye(w.nbf)
    df.set_density(D2)
    K2 = df.compute_exchange().cpu().numpy()
    _, Ko2 = oracle.df_jk_from_integrals(oracle.orc_eri3c(w.basis, aux), oracle.orc_eri2c(aux), D2)
    assert np.max(np.abs(K2 - Ko2)) < 1e-10
    assert torch.is_tensor(df.get_coulomb_matrix())



def test_df_exchange_from_orbitals(lai):
    """set_orbitals(C, w): D = w C C^T and K built from C directly (no factoring of
    D) equal the set_density build of the same D; a second exchange build at the
    same density reuses its factors and gives the same K."""
    import torch
    w = lai.workloads.make("h2o2_ccpvdz")
    aux = lai.BasisSet.from_atoms(w.Z, w.xyz, "cc-pvdz-ri")
    eng = lai.Engine(w.basis)
    rng = np.random.default_rng(5)
    C = rng.standard_normal((w.nbf, 10)) / np.sqrt(w.nbf)
    df = lai.df.DFFockBuilder(eng, aux)
    df.set_orbitals(C, 2.0)
    Jo, Ko = df.compute_coulomb().cpu().numpy(), df.compute_exchange().cpu().numpy()
    df.set_density(2.0 * C @ C.T)
    Jd, Kd = df.compute_coulomb().cpu().numpy(), df.compute_exchange().cpu().numpy()
    assert np.max(np.abs(Jo - Jd)) < 1e-12
    assert np.max(np.abs(Ko - Kd)) < 1e-11
    K2 = df.compute_exchange().cpu().numpy()
    assert np.array_equal(K2, Kd)
    with pytest.raises(ValueError):
        df.set_orbitals(torch.zeros((w.nbf + 1, 3)), 1.0)

def test_df_rhf_close_to_four_center(lai):
    w = lai.workloads.make("h2o2_ccpvdz")
    aux = lai.BasisSet.from_atoms(w.Z, w.xyz, "cc-pvdz-ri")
    r4 = lai.scf.RHF(w.basis).run(energy_threshold=1e-10, density_threshold=1e-8)
    rd = lai.scf.RHF(w.basis, aux=aux).run(energy_threshold=1e-10, density_threshold=1e-8)
    assert r4.converged and rd.converged
    # the fitting error of the built-in cc-pVDZ-RI set: a few mHa at most
    assert abs(rd.total_energy - r4.total_energy) < 1e-2
