"""The C-ABI library: loads, exports every declared symbol, host-side logic (no GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden

HEADER = os.path.join(ROOT, "include", "libaccint_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"LAI_API\s+[\w\s\*]*?\b(lai_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol(lai):
    L = lai.lib()
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert sorted(lai._lib.EXPORTED) == names
    assert L.lai_abi_version() == 2


def test_basis_normalization_matches_reference(lai):
    g = golden("norm_ccpvqz_ref.npz")
    b = lai.BasisSet.from_atoms(g["Z"], g["xyz"], "cc-pvqz")
    c = np.concatenate(b.normalized_coefs())
    assert np.max(np.abs(c - g["coefs"])) < 1e-13 * np.max(np.abs(g["coefs"]))


def test_basis_counts(lai):
    w = lai.workloads.make("h2o64_ccpvdz")
    assert w.basis.n_shells == 768
    assert w.nbf == 1600  # Cartesian (1536 spherical)
    assert w.D.shape == (1600, 1600)
    assert np.allclose(w.D, w.D.T)
    w0 = lai.workloads.make("h2o8_sto3g")
    assert w0.nbf == 56 and w0.basis.n_shells == 40
    assert lai.BasisSet.from_atoms(*lai.molecules.alkane(12), "cc-pvtz").nbf == 810


def _create(lai, l, nprim, exps, coefs):
    L = lai.lib()
    l = np.array(l, dtype=np.int32)
    nprim = np.array(nprim, dtype=np.int32)
    centers = np.zeros(3 * len(l))
    exps = np.array(exps, dtype=np.float64)
    coefs = np.array(coefs, dtype=np.float64)
    h = ctypes.c_void_p()
    rc = L.lai_basis_create(len(l), l.ctypes.data, nprim.ctypes.data, centers.ctypes.data,
                            exps.ctypes.data, coefs.ctypes.data, None, 0, ctypes.byref(h))
    if rc == 0:
        L.lai_basis_destroy(h)
    return rc, L.lai_last_error().decode()


def test_basis_rejects_bad_shells(lai):
    assert _create(lai, [5], [1], [1.0], [1.0])[0] == -1        # l > 4
    assert _create(lai, [0], [1], [-1.0], [1.0])[0] == -1       # exponent <= 0
    assert _create(lai, [0], [2], [1.0, 2.0], [0.0, 0.0])[0] == -1  # all-zero contraction
    assert _create(lai, [0], [0], [], [])[0] == -1              # no primitive
    assert _create(lai, [2], [1], [0.8], [1.0])[0] == 0


def test_zero_coefficient_primitives_are_dropped_exactly(lai):
    """A general-contraction column with zero padding equals the single primitive."""
    data = lai.basis_data("cc-pvdz")["O"]
    l, e, c = data[2]  # O 3rd s: 9 exponents, 1 nonzero coefficient
    assert sum(1 for x in c if x != 0.0) == 1
    b1 = lai.BasisSet([lai.Shell(l, np.zeros(3), e, c)])
    k = [i for i, x in enumerate(c) if x != 0.0][0]
    b2 = lai.BasisSet([lai.Shell(l, np.zeros(3), [e[k]], [c[k]])])
    c1 = b1.normalized_coefs()[0]
    c2 = b2.normalized_coefs()[0]
    assert c1[k] == pytest.approx(c2[0], rel=1e-15)


def test_engine_without_gpu_fails_loudly(lai):
    """No silent CPU path: creating an engine with no usable device is an error."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    w = lai.workloads.make("h2o1_sto3g")
    with pytest.raises(lai.LibAccIntError):
        lai.Engine(w.basis)
