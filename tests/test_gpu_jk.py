"""CUDA J/K and integrals against the oracle / reference (GPU).

Bars (stated in the task): FP64 integrals within 1e-11 absolute of the reference's
compute_eri; J/K within 1e-10 max-abs of the reference's FockBuilder; the PySCF
fixture of the reference's own validation test within 1e-7.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

ERI_TOL = 1e-11
JK_TOL = 1e-10


def _engine(lai, basis, thr=1e-12):
    return lai.Engine(basis, threshold=thr)


def _jk_case(lai, name, basis_name):
    g = golden(name)
    b = lai.BasisSet.from_atoms(g["Z"], g["xyz"], basis_name)
    e = _engine(lai, b)
    J, K, rep = e.jk(g["D"])
    return g, J, K, rep


def test_jk_h2o8_sto3g_vs_reference(lai):
    """Config 0 in full: (H2O)8 / built-in STO-3G vs the reference's full N^4 J/K."""
    g, J, K, rep = _jk_case(lai, "h2o8_sto3g_ref.npz", "sto-3g")
    assert np.max(np.abs(J - g["J"])) < JK_TOL
    assert np.max(np.abs(K - g["K"])) < JK_TOL
    assert rep.quartets_fp64 > 0


def test_jk_h2o2_ccpvdz_vs_reference(lai):
    g, J, K, _ = _jk_case(lai, "h2o2_ccpvdz_ref.npz", "cc-pvdz")
    assert np.max(np.abs(J - g["J"])) < JK_TOL
    assert np.max(np.abs(K - g["K"])) < JK_TOL


def test_jk_h2o2_sto3g_vs_reference(lai):
    g, J, K, _ = _jk_case(lai, "h2o2_sto3g_ref.npz", "sto-3g")
    assert np.max(np.abs(J - g["J"])) < JK_TOL
    assert np.max(np.abs(K - g["K"])) < JK_TOL



def test_jk_h2o_ccpvqz_g_shells_vs_reference(lai):
    """H2O / cc-pVQZ (140 Cartesian functions, s..g, every class up to (gg|gg)):
    J and K against the unmodified reference's full N^4 FockBuilder build, Schwarz
    and primitive screening off, at the J/K bar."""
    g = golden("h2o1_ccpvqz_ref.npz")
    b = lai.BasisSet.from_atoms(g["Z"], g["xyz"], "cc-pvqz")
    assert max(s.l for s in b.shells) == 4
    e = lai.Engine(b, threshold=0.0, prim_threshold=0.0)
    J, K, _ = e.jk(g["D"])
    assert np.max(np.abs(J - g["J"])) < JK_TOL, np.max(np.abs(J - g["J"]))
    assert np.max(np.abs(K - g["K"])) < JK_TOL, np.max(np.abs(K - g["K"]))

def test_jk_water_aug_cc_pvtz_vs_pyscf(lai):
    """The reference's own PySCF validation fixture (l <= 3), tolerance 1e-7 as in
    tests/validation/test_water_cluster_validation.cpp:454-495."""
    g = golden("water1_augccpvtz.npz")
    b = lai.BasisSet.from_atoms(g["Z"], g["xyz"], "aug-cc-pvtz")
    assert b.nbf == g["D"].shape[0] == 105
    e = _engine(lai, b, thr=0.0)
    J, K, _ = e.jk(g["D"])
    assert np.max(np.abs(J - g["J"])) < 1e-7
    assert np.max(np.abs(K - g["K"])) < 1e-7


def _eri_lookup(vals, meta, basis):
    """Function (i,j,k,l) -> integral from the canonical batch (8-fold symmetry)."""
    blocks = {}
    for off, fa, fb, fc, fd, na, nb, nc, nd in meta:
        blocks[(int(fa), int(fb), int(fc), int(fd))] = (int(off), (int(na), int(nb), int(nc), int(nd)))
    offs = basis.function_offsets()
    def shell_of(f):
        s = int(np.searchsorted(offs, f, side="right") - 1)
        return int(offs[s]), f - int(offs[s])
    def get(i, j, k, l):
        (a, ia), (b, ib), (c, ic), (d, id_) = map(shell_of, (i, j, k, l))
        for (p, q), (r, t) in (((0, 1), (2, 3)), ((2, 3), (0, 1))):
            for swap1 in (False, True):
                for swap2 in (False, True):
                    F = [(a, ia), (b, ib), (c, ic), (d, id_)]
                    x, y = (F[p], F[q]) if not swap1 else (F[q], F[p])
                    z, w = (F[r], F[t]) if not swap2 else (F[t], F[r])
                    key = (x[0], y[0], z[0], w[0])
                    if key in blocks:
                        off, sh = blocks[key]
                        blk = vals[off:off + int(np.prod(sh))].reshape(sh)
                        return blk[x[1], y[1], z[1], w[1]]
        raise KeyError((i, j, k, l))
    return get


def test_pyscf_sampled_eri(lai):
    g = golden("water1_augccpvtz.npz")
    b = lai.BasisSet.from_atoms(g["Z"], g["xyz"], "aug-cc-pvtz")
    e = _engine(lai, b, thr=0.0)
    vals, meta = e.compute_batch_screened()
    get = _eri_lookup(vals, meta, b)
    for (i, j, k, l), v in zip(g["eri_idx"], g["eri_val"]):
        assert abs(get(i, j, k, l) - v) < 1e-8


def test_eri_all_quartets_h2o_ccpvdz_vs_oracle(lai, oracle):
    """Every canonical quartet of H2O/cc-pVDZ (s, p, d; up to 5 roots), per integral."""
    w = lai.workloads.make("h2o1_ccpvdz")
    b = w.basis
    e = _engine(lai, b, thr=0.0)
    vals, meta = e.compute_batch_screened()
    f2s = {int(x): i for i, x in enumerate(b.function_offsets()[:-1])}
    R = oracle.reference()
    worst = 0.0
    for off, fa, fb, fc, fd, na, nb, nc, nd in meta:
        sh = [f2s[int(x)] for x in (fa, fb, fc, fd)]
        got = vals[off:off + na * nb * nc * nd].reshape(na, nb, nc, nd)
        if R is not None:
            rb = getattr(test_eri_all_quartets_h2o_ccpvdz_vs_oracle, "_rb", None)
            if rb is None:
                rb = oracle.RefBasis(b)
                test_eri_all_quartets_h2o_ccpvdz_vs_oracle._rb = rb
            ref = rb.quartet(*sh, (na, nb, nc, nd))
        else:
            ref = oracle.orc_quartet(b, *sh)
        worst = max(worst, float(np.max(np.abs(got - ref))))
    assert worst < ERI_TOL, worst


def _small_high_l_basis(lai):
    """Seven shells s..g on two centres (cc-pVQZ carbon/hydrogen exponents)."""
    data = lai.basis_data("cc-pvqz")
    C = [s for s in data["C"]]
    H = [s for s in data["H"]]
    pick = [C[0], C[5], C[9], C[12], C[14], H[0], H[4]]  # s(12) p(6) d f g | s(6) p
    ls = [p[0] for p in pick]
    assert sorted(set(ls)) == [0, 1, 2, 3, 4]
    ctr = [np.zeros(3)] * 5 + [np.array([1.1, -0.7, 1.6])] * 2
    shells = [lai.Shell(l, c, e, co) for (l, e, co), c in zip(pick, ctr)]
    return lai.BasisSet(shells)


def test_eri_all_classes_up_to_g_vs_oracle(lai, oracle):
    """All canonical quartets of a 7-shell s..g basis (every class up to (gg|gg),
    up to 9 roots) against the binary128-root oracle."""
    b = _small_high_l_basis(lai)
    e = _engine(lai, b, thr=0.0)
    vals, meta = e.compute_batch_screened()
    f2s = {int(x): i for i, x in enumerate(b.function_offsets()[:-1])}
    worst = 0.0
    for off, fa, fb, fc, fd, na, nb, nc, nd in meta:
        sh = [f2s[int(x)] for x in (fa, fb, fc, fd)]
        got = vals[off:off + na * nb * nc * nd].reshape(na, nb, nc, nd)
        ref = oracle.orc_quartet(b, *sh)
        worst = max(worst, float(np.max(np.abs(got - ref))))
    assert worst < ERI_TOL, worst


def test_schwarz_vs_oracle(lai, oracle):
    w = lai.workloads.make("h2o1_ccpvdz")
    e = _engine(lai, w.basis)
    Q = e.schwarz()
    Qo = oracle.orc_schwarz(w.basis)
    assert np.max(np.abs(Q - Qo)) < 1e-12


def test_jk_properties_h2o64_ccpvdz(lai):
    """Config 1 at full size: size-independent properties (symmetry, energy,
    run-to-run agreement), the quartet count, and J/K linearity in D."""
    w = lai.workloads.make("h2o64_ccpvdz")
    assert w.nbf == 1600 and w.basis.n_shells == 768
    e = _engine(lai, w.basis)
    J, K, rep = e.jk(w.D)
    assert np.max(np.abs(J - J.T)) < 1e-12 * max(1.0, np.max(np.abs(J)))
    assert np.max(np.abs(K - K.T)) < 1e-12 * max(1.0, np.max(np.abs(K)))
    J2, K2, _ = e.jk(w.D)
    assert np.max(np.abs(J - J2)) < 1e-11 and np.max(np.abs(K - K2)) < 1e-11
    J3, K3, _ = e.jk(2.0 * w.D)
    assert np.max(np.abs(J3 - 2 * J)) < 1e-10 and np.max(np.abs(K3 - 2 * K)) < 1e-10
    E = lai.molecules.energy(w.D, J, K)
    assert np.isfinite(E)
    assert rep.quartets_fp64 > 1e9


def test_nbf_mismatch_is_an_error(lai):
    w = lai.workloads.make("h2o1_sto3g")
    e = _engine(lai, w.basis)
    import ctypes
    L = lai.lib()
    D = np.zeros((3, 3))
    J = np.zeros((3, 3))
    rc = L.lai_jk_build(e._h, D.ctypes.data, 3, J.ctypes.data, J.ctypes.data, None, None)
    assert rc == -1
    assert b"nbf mismatch" in L.lai_last_error()


def test_nonsymmetric_density_rejected_when_checked(lai):
    w = lai.workloads.make("h2o1_sto3g")
    e = _engine(lai, w.basis)
    D = w.D.copy()
    D[0, 1] += 1e-3
    with pytest.raises(lai.LibAccIntError):
        e.jk(D, check_symmetric=True)


def test_primitive_screening_is_within_tolerance(lai):
    """Primitive-quartet screening (q_ab q_cd < 1e-3 * threshold) changes J/K by
    far less than the 1e-10 parity bar: compare with the cut switched off."""
    w = lai.workloads.make("h2o8_ccpvdz")
    e_on = lai.Engine(w.basis, threshold=1e-12)
    e_off = lai.Engine(w.basis, threshold=1e-12, prim_threshold=0.0)
    J1, K1, r1 = e_on.jk(w.D)
    J0, K0, r0 = e_off.jk(w.D)
    assert r1.quartets_fp64 == r0.quartets_fp64
    assert np.max(np.abs(J1 - J0)) < 1e-11
    assert np.max(np.abs(K1 - K0)) < 1e-11


MIXED_DE_TOL = 1e-8  # |E(mixed) - E(FP64)| bar for the FP32 Rys path (Hartree)


def test_mixed_precision_energy_within_bar(lai):
    """FP32 Rys path for quartets with Q_ij Q_kl max|D| < 1e-7: the energy moves by
    less than 1e-8 Eh, J/K stay symmetric, and the FP32 path really ran (its
    results differ from FP64 in the last digits, and the report counts it)."""
    w = lai.workloads.make("h2o16_ccpvdz")
    e = _engine(lai, w.basis)
    J0, K0, r0 = e.jk(w.D)
    J1, K1, r1 = e.jk(w.D, fp32_cut=1e-7)
    assert r1.quartets_fp32 > 0.3 * (r1.quartets_fp32 + r1.quartets_fp64)
    assert r1.quartets_fp32 + r1.quartets_fp64 == r0.quartets_fp64
    maxd = np.max(np.abs(w.D))
    assert 0.5 * 1e-7 / maxd < r1.fp32_schwarz_cut <= 1e-7 / maxd
    E0 = lai.molecules.energy(w.D, J0, K0)
    E1 = lai.molecules.energy(w.D, J1, K1)
    assert abs(E1 - E0) < MIXED_DE_TOL
    assert 0.0 < np.max(np.abs(J1 - J0)) < 1e-7
    assert 0.0 < np.max(np.abs(K1 - K0)) < 1e-7
    assert np.max(np.abs(J1 - J1.T)) < 1e-12 and np.max(np.abs(K1 - K1.T)) < 1e-12



def test_mixed_precision_relative_primitive_cut(lai):
    """lai_jk_opts.fp32_prim_rel: FP32 quartets also skip primitive quartets below
    that fraction of their own Schwarz bound.  0 reproduces the plain mixed build
    (to the run-to-run spread of the FP64 atomic digestion); 1e-6 at cut 1e-6 stays
    inside the 1e-8 Eh bar and skips nothing in the FP64 quartets; values outside
    [0, 1) are refused."""
    w = lai.workloads.make("h2o8_ccpvdz")
    e = _engine(lai, w.basis)
    J64, K64, _ = e.jk(w.D)
    Jm, Km, rm = e.jk(w.D, fp32_cut=1e-6)
    J0, K0, r0 = e.jk(w.D, fp32_cut=1e-6, fp32_prim_rel=0.0)
    assert np.max(np.abs(Jm - J0)) < 1e-12 and np.max(np.abs(Km - K0)) < 1e-12
    Jr, Kr, rr = e.jk(w.D, fp32_cut=1e-6, fp32_prim_rel=1e-6)
    assert rr.quartets_fp32 == rm.quartets_fp32 > 0
    dE = 0.5 * np.sum(w.D * (Jr - J64)) - 0.25 * np.sum(w.D * (Kr - K64))
    assert abs(dE) < 1e-8
    assert np.max(np.abs(Jr - J64)) < 1e-8 and np.max(np.abs(Kr - K64)) < 1e-8
    # the FP64 quartets are untouched: with every quartet in FP64 the option is inert
    Jf, Kf, _ = e.jk(w.D, fp32_cut=0.0, fp32_prim_rel=1e-3)
    assert np.max(np.abs(Jf - J64)) < 1e-12 and np.max(np.abs(Kf - K64)) < 1e-12
    with pytest.raises(lai.LibAccIntError):
        e.jk(w.D, fp32_cut=1e-6, fp32_prim_rel=1.5)


def test_mixed_precision_f_classes_run_fp32(lai):
    """(H2O)2 / cc-pVTZ (f on O) at cut 1e-6: quartets of f classes below the FP32
    Schwarz cut run in FP32 (the warp-per-quartet FP32 variant; only classes too
    large for it stay FP64): the FP32 count, checked against the canonical
    quartets in [threshold, cut) worked out on the host from the engine's Schwarz
    matrix, exceeds what the classes up to d hold, and the energy stays inside the
    1e-8 Eh bar."""
    w = lai.workloads.make("h2o2_ccpvtz")
    e = _engine(lai, w.basis)
    Q = e.schwarz()
    ls = np.array([s.l for s in w.basis.shells])
    n = len(ls)
    i, j = np.tril_indices(n)
    q = Q[i, j]
    J64, K64, r64 = e.jk(w.D)
    Jm, Km, rm = e.jk(w.D, fp32_cut=1e-6)
    cut = rm.fp32_schwarz_cut
    assert cut > 0
    prod = np.multiply.outer(q, q)[np.tril_indices(len(q))]  # canonical pairs of pairs
    lmax = np.maximum.outer(np.maximum(ls[i], ls[j]), np.maximum(ls[i], ls[j]))[np.tril_indices(len(q))]
    keep = prod >= 1e-12
    assert int(keep.sum()) == r64.quartets_fp64
    below = keep & (prod < cut)
    assert int((below & (lmax == 3)).sum()) > 0
    assert int((below & (lmax <= 2)).sum()) < rm.quartets_fp32 <= int(below.sum())
    dE = 0.5 * np.sum(w.D * (Jm - J64)) - 0.25 * np.sum(w.D * (Km - K64))
    assert abs(dE) < 1e-8
    assert np.max(np.abs(Jm - J64)) < 1e-8 and np.max(np.abs(Km - K64)) < 1e-8

def test_mixed_precision_cut_zero_is_fp64(lai):
    """fp32_cut = 0 is the plain FP64 build (equal up to the order of the FP64
    atomic additions); a negative cut is an error."""
    w = lai.workloads.make("h2o2_ccpvdz")
    e = _engine(lai, w.basis)
    J0, K0, _ = e.jk(w.D)
    J1, K1, r1 = e.jk(w.D, fp32_cut=0.0)
    assert r1.quartets_fp32 == 0 and r1.fp32_schwarz_cut == 0.0
    assert np.max(np.abs(J0 - J1)) < 1e-13 and np.max(np.abs(K0 - K1)) < 1e-13
    with pytest.raises(lai.LibAccIntError):
        e.jk(w.D, fp32_cut=-1.0)


def test_mixed_precision_all_fp32_close_to_reference(lai):
    """Every quartet in FP32 (a cut above every bound): J/K still agree with the
    reference's FP64 J/K to FP32 accuracy -- a check of the FP32 kernels of every
    class present, including those that fall back to FP64 kernels."""
    g = golden("h2o2_ccpvdz_ref.npz")
    b = lai.BasisSet.from_atoms(g["Z"], g["xyz"], "cc-pvdz")
    e = _engine(lai, b)
    J, K, r = e.jk(g["D"], fp32_cut=1e30)
    assert r.quartets_fp32 > 0.9 * (r.quartets_fp32 + r.quartets_fp64)
    scale = max(np.max(np.abs(g["J"])), 1.0)
    assert np.max(np.abs(J - g["J"])) < 1e-5 * scale
    assert np.max(np.abs(K - g["K"])) < 1e-5 * scale


@pytest.mark.parametrize("name,nshard", [("h2o8_sto3g", 2), ("h2o4_ccpvdz", 2), ("h2o4_ccpvdz", 3)])
def test_quartet_shards_sum_to_full_build(lai, name, nshard):
    """The multi-GPU split on one device: every shard (shard_index of shard_count,
    a contiguous slice of every quartet block) built separately; their J and K
    summed must equal the unsharded build (what the NCCL all-reduce of the ranks
    forms), and the shards' quartet counts must add up to the whole."""
    w = lai.workloads.make(name)
    e = _engine(lai, w.basis)
    J, K, rep = e.jk(w.D)
    Js = np.zeros_like(J)
    Ks = np.zeros_like(K)
    nq = 0
    for s in range(nshard):
        Jp, Kp, rp = e.jk(w.D, shard=(s, nshard))
        Js += Jp
        Ks += Kp
        nq += rp.quartets_fp64
    assert nq == rep.quartets_fp64
    assert np.max(np.abs(Js - J)) < 1e-12
    assert np.max(np.abs(Ks - K)) < 1e-12
