"""The CPU oracle pinned against the reference's golden vectors (no GPU)."""
import numpy as np
import pytest

from conftest import golden


def test_boys_vs_mpmath_golden(oracle):
    g = golden("boys_mpmath.npz")
    for T, F in zip(g["T"], g["F"]):
        f = oracle.orc_boys(len(F) - 1, T)
        assert np.max(np.abs(f - F) / np.abs(F)) < 2e-15, T


@pytest.mark.parametrize("n", range(1, 10))
def test_rys_T0_is_gauss_legendre(oracle, n):
    x, w = np.polynomial.legendre.leggauss(2 * n)
    m = x > 0
    o = np.argsort(x[m] ** 2)
    u, wt = oracle.orc_rys(n, 0.0)
    assert np.allclose(u, (x[m] ** 2)[o], rtol=1e-14, atol=0)
    assert np.allclose(wt, w[m][o], rtol=1e-13, atol=0)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 9])
def test_rys_moments(oracle, n):
    for T in [1e-9, 0.3, 2.0, 11.0, 29.0, 47.0, 93.0, 400.0]:
        u, w = oracle.orc_rys(n, T)
        F = oracle.orc_boys(2 * n - 1, T)
        for k in range(2 * n):
            assert abs(np.sum(w * u ** k) - F[k]) <= 1e-14 * F[k] * (k + 1), (n, T, k)


def test_rys_vs_reference_regression(oracle):
    """Agreement with the reference's own rys_compute outputs where those are
    accurate (n <= 4), and the reference's documented drift for many roots."""
    g = golden("rys_refgen.npz")
    for n in range(1, 5):
        for T, r, w in zip(g[f"n{n}_T"], g[f"n{n}_roots"], g[f"n{n}_weights"]):
            u, wt = oracle.orc_rys(n, T)
            assert np.max(np.abs(u - r) / r) < 1e-12 and np.max(np.abs(wt - w) / w) < 1e-12, (n, T)
    # n = 9 at T = 0: Gauss-Legendre is exact; the reference's table is off by ~1e-6
    x, w = np.polynomial.legendre.leggauss(18)
    exact = np.sort(x[x > 0] ** 2)
    ref = g["n9_roots"][0]
    assert g["n9_T"][0] == 0.0
    assert np.max(np.abs(ref - exact) / exact) > 1e-8
    u, _ = oracle.orc_rys(9, 0.0)
    assert np.max(np.abs(u - exact) / exact) < 1e-14


def test_eri_samples_vs_reference_compute_eri(oracle):
    """400 sampled cc-pVQZ quartets (all l-classes up to g): the reference's
    compute_eri values (committed) against the oracle (recomputed here for a subset)."""
    g = golden("eri_ccpvqz_samples.npz")
    assert np.max(np.abs(g["ref"] - g["orc"])) < 1e-11


def test_oracle_jk_vs_reference_golden(lai, oracle):
    g = golden("h2o2_sto3g_ref.npz")
    b = lai.BasisSet.from_atoms(g["Z"], g["xyz"], "sto-3g")
    J, K, nq = oracle.orc_jk(b, g["D"], 0.0)
    assert np.max(np.abs(J - g["J"])) < 1e-12
    assert np.max(np.abs(K - g["K"])) < 1e-12


def test_oracle_normalization_vs_reference(lai, oracle):
    g = golden("norm_ccpvqz_ref.npz")
    b = lai.BasisSet.from_atoms(g["Z"], g["xyz"], "cc-pvqz")
    l, nprim, centers, exps, coefs = oracle.normalized_arrays(b)
    assert np.max(np.abs(coefs - g["coefs"])) < 1e-13 * np.max(np.abs(g["coefs"]))


def test_reference_gpu_route_units_on_host(lai, oracle):
    """Host side of the reference GPU harness (oracle/ref_gpu_shim.cu; built by
    `make -C oracle refgpu`): the reference groups (H2O)8/STO-3G into its two ShellSets,
    and the ordered set 4-tuples cover every ordered shell quartet exactly once.  No
    device call is made here."""
    if oracle.reference_gpu() is None:
        pytest.skip("oracle/_ref/libref_gpu.so not built (make -C oracle refgpu)")
    w = lai.workloads.make("h2o8_sto3g")
    rb = oracle.RefGpuBasis(w.basis)
    assert rb.nbf == w.nbf and rb.nsets == 2 and rb.nunits == 16
    total = sum(rb.unit_size(u)[0] for u in range(rb.nunits))
    assert total == w.basis.n_shells ** 4
    with pytest.raises(ValueError):
        rb.unit_size(rb.nunits)


def test_oracle_jk_vs_reference_h2o_ccpvdz(lai, oracle):
    """The restatement's J/K against the compiled reference's full Engine::compute path
    for H2O / cc-pVDZ (s, p, d shells; up to 5 Rys roots), no screening."""
    if oracle.reference() is None:
        pytest.skip("oracle/_ref/libref_oracle.so not built")
    w = lai.workloads.make("h2o1_ccpvdz")
    J, K, nq = oracle.orc_jk(w.basis, w.D, 0.0)
    Jr, Kr, _ = oracle.RefBasis(w.basis).jk_full(w.D)
    assert nq == 3081  # every canonical quartet of 12 shells
    assert np.max(np.abs(J - Jr)) < 1e-12
    assert np.max(np.abs(K - Kr)) < 1e-12
