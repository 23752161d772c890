"""Work-unit API on the GPU: raw integrals of listed quartets (any order and
orientation) against the binary128-root oracle on large samples drawn from the
benchmark geometries, and J/K of listed quartets (plain and 8-fold symmetric)
against the full build and the reference."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

ERI_TOL = 1e-11
JK_TOL = 1e-10


def _classes(basis, q):
    ls = np.array([s.l for s in basis.shells])
    return ls[q[:, 0]] * 125 + ls[q[:, 1]] * 25 + ls[q[:, 2]] * 5 + ls[q[:, 3]]


def _stratified(basis, pool, per_class, rng):
    """Up to per_class quartets of every (la,lb,lc,ld) class of the pool."""
    cls = _classes(basis, pool)
    pick = []
    for c in np.unique(cls):
        idx = np.flatnonzero(cls == c)
        pick.append(rng.choice(idx, size=min(per_class, idx.size), replace=False))
    return pool[np.sort(np.concatenate(pick))]


def _scramble(q, rng):
    """Random listed orientation: swap i<->j, k<->l and bra<->ket independently."""
    q = q.copy()
    s1, s2, s3 = (rng.random(len(q)) < 0.5 for _ in range(3))
    q[s1, 0], q[s1, 1] = q[s1, 1].copy(), q[s1, 0].copy()
    q[s2, 2], q[s2, 3] = q[s2, 3].copy(), q[s2, 2].copy()
    q[s3] = q[s3][:, [2, 3, 0, 1]]
    return q


def _check_sample(lai, oracle, w, npool, per_class, seed):
    e = lai.Engine(w.basis, threshold=w.thr)
    rng = np.random.default_rng(seed)
    pool = e.sample_quartets(npool, seed=seed)
    q = _scramble(_stratified(w.basis, pool, per_class, rng), rng)
    vals, meta = e.eri_quartets(q)
    ref = oracle.orc_quartets(w.basis, q)
    assert vals.shape == ref.shape
    err = np.abs(vals - ref)
    worst = int(np.argmax(err))
    assert err[worst] < ERI_TOL, (err[worst], vals[worst], ref[worst])
    return len(q), len(np.unique(_classes(w.basis, q)))


def test_sampled_integrals_h2o64_ccpvdz(lai, oracle):
    """>= 1e5 canonical quartets of the (H2O)64 / cc-pVDZ benchmark geometry, every
    class present, in scrambled orientation, within 1e-11 of the oracle."""
    n, ncls = _check_sample(lai, oracle, lai.workloads.make("h2o64_ccpvdz"), 400000, 12000, 11)
    assert n >= 100000 and ncls >= 15


def test_sampled_integrals_c12h26_ccpvtz(lai, oracle):
    """C12H26 / cc-pVTZ (s..f): every class present, up to 600 quartets each."""
    n, ncls = _check_sample(lai, oracle, lai.workloads.make("c12h26_ccpvtz"), 200000, 600, 12)
    assert ncls >= 30


def _all_canonical(ns):
    q = [(i, j, k, l) for i in range(ns) for j in range(i + 1) for k in range(i + 1)
         for l in range(k + 1 if k < i else j + 1)]
    return np.array(q, dtype=np.int32)


def test_listed_canonical_quartets_symmetric_vs_reference(lai):
    """All canonical quartets of (H2O)2 / cc-pVDZ listed with canonical_symmetry:
    the reference's full J/K."""
    g = golden("h2o2_ccpvdz_ref.npz")
    b = lai.BasisSet.from_atoms(g["Z"], g["xyz"], "cc-pvdz")
    e = lai.Engine(b)
    q = _all_canonical(b.n_shells)
    J = np.zeros_like(g["J"])
    K = np.zeros_like(g["K"])
    e.jk_accumulate_quartets(q, g["D"], J, K, canonical_symmetry=True)
    assert np.max(np.abs(J - g["J"])) < JK_TOL
    assert np.max(np.abs(K - g["K"])) < JK_TOL


def test_listed_full_product_plain_vs_full_build(lai):
    """Every ordered quartet of (H2O)1 / cc-pVDZ listed without symmetry (plain
    accumulation, in two halves added onto each other) equals the full build."""
    w = lai.workloads.make("h2o1_ccpvdz")
    e = lai.Engine(w.basis, threshold=0.0, prim_threshold=0.0)
    ns = w.basis.n_shells
    q = np.array([(i, j, k, l) for i in range(ns) for j in range(ns) for k in range(ns)
                  for l in range(ns)], dtype=np.int32)
    J = np.zeros((w.nbf, w.nbf))
    K = np.zeros((w.nbf, w.nbf))
    h = len(q) // 2
    e.jk_accumulate_quartets(q[:h], w.D, J, K, canonical_symmetry=False)
    e.jk_accumulate_quartets(q[h:], w.D, J, K, canonical_symmetry=False)
    J0, K0, _ = e.jk(w.D)
    assert np.max(np.abs(J - J0)) < JK_TOL
    assert np.max(np.abs(K - K0)) < JK_TOL


def test_external_batch_digestion(lai):
    """accumulate_device_eri_batch: raw integrals of the full product list digested
    on the device equal the full build."""
    import ctypes
    import torch
    w = lai.workloads.make("h2o1_ccpvdz")
    e = lai.Engine(w.basis, threshold=0.0, prim_threshold=0.0)
    ns = w.basis.n_shells
    q = np.array([(i, j, k, l) for i in range(ns) for j in range(ns) for k in range(ns)
                  for l in range(ns)], dtype=np.int32)
    vals, meta = e.eri_quartets(q)
    cmeta = (lai._lib.QuartetMeta * len(meta))()
    for t, m in enumerate(meta):
        cmeta[t].offset = int(m[0])
        cmeta[t].fa, cmeta[t].fb, cmeta[t].fc, cmeta[t].fd = (int(x) for x in m[1:5])
        cmeta[t].na, cmeta[t].nb, cmeta[t].nc, cmeta[t].nd = (int(x) for x in m[5:9])
    dev = torch.device("cuda", 0)
    d_eri = torch.from_numpy(vals).to(dev)
    D = torch.from_numpy(w.D).to(dev)
    J = torch.zeros_like(D)
    K = torch.zeros_like(D)
    lai._lib.check(lai.lib().lai_jk_accumulate_eri_batch_device(
        e._h, ctypes.c_void_p(d_eri.data_ptr()), cmeta, len(meta), ctypes.c_void_p(D.data_ptr()),
        ctypes.c_void_p(J.data_ptr()), ctypes.c_void_p(K.data_ptr()),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    J0, K0, _ = e.jk(w.D)
    assert np.max(np.abs(J.cpu().numpy() - J0)) < JK_TOL
    assert np.max(np.abs(K.cpu().numpy() - K0)) < JK_TOL


def test_bad_shell_index_is_an_error(lai):
    w = lai.workloads.make("h2o1_sto3g")
    e = lai.Engine(w.basis)
    with pytest.raises(lai.LibAccIntError):
        e.eri_quartets(np.array([[0, 0, 0, 99]], dtype=np.int32))
