"""Native Basis Set Exchange JSON loader (lai_basis_from_bse_json), CPU only:
its shells against the package's bundled basis data (extracted from the same BSE
files by data/make_basis_data.py, the reference's expansion rules), hand-written
BSE text for the expansion rules (general contractions, SP shells, all-zero
columns), and the reference parser's error cases
(src/shared/data/bse_json_parser.cpp:90-140)."""
import json
import os

import numpy as np
import pytest

# the reference checkout ($LIBACCINT_REFERENCE, else the default below), when present
REF_SHARE = os.path.join(os.environ.get("LIBACCINT_REFERENCE", "/root/reference"), "share", "basis_sets")


def _shells(b):
    return [(s.l, tuple(np.round(s.center, 12)), tuple(s.exps)) for s in b.shells]


def _bse(elements, schema="complete"):
    return json.dumps({"molssi_bse_schema": {"schema_type": schema, "schema_version": "0.1"},
                       "elements": elements})


def test_expansion_rules(lai):
    el = {"8": {"electron_shells": [
        {"function_type": "gto", "angular_momentum": [0],
         "exponents": ["1.0E+01", "2.0E+00", "5.0E-01"],
         "coefficients": [["0.1", "0.5", "0.4"], ["0", "0", "0"], ["-0.1", "0.0", "1.0E+00"]]},
        {"function_type": "gto", "angular_momentum": [0, 1],
         "exponents": ["3.0", "0.7"], "coefficients": [["0.2", "0.8"], ["0.3", "0.6"]]},
        {"function_type": "gto", "angular_momentum": [2], "exponents": ["0.9"], "coefficients": [["1.0"]]}]},
        "1": {"electron_shells": [
            {"function_type": "gto", "angular_momentum": [0], "exponents": ["1.5"], "coefficients": [["1.0"]]}]}}
    Z = [8, 1, 8]
    xyz = np.array([[0.0, 0.0, 0.0], [0.0, 1.4, -1.1], [3.0, 0.0, 0.0]])
    b = lai.BasisSet.from_bse_json(_bse(el), Z, xyz)
    # O: 2 s (zero column skipped) + SP (s, p) + d = 5 shells; H: 1; O again: 5
    assert [s.l for s in b.shells] == [0, 0, 0, 1, 2, 0, 0, 0, 0, 1, 2]
    assert b.nbf == 2 * (1 + 1 + 1 + 3 + 6) + 1
    assert len(b.shells[0].exps) == 3 and len(b.shells[1].exps) == 3   # all exponents kept
    assert np.allclose(b.shells[9].center, xyz[2])
    # the same shells written through lai_basis_create give the same normalized coefficients
    ref = lai.BasisSet([lai.Shell(0, xyz[0], [10.0, 2.0, 0.5], [0.1, 0.5, 0.4])])
    h = ref.handle()
    e = np.zeros(3)
    c = np.zeros(3)
    ctr = np.zeros(3)
    import ctypes
    l_, k_, fi = ctypes.c_int(), ctypes.c_int(), ctypes.c_long()
    lai.lib().lai_basis_shell(h, 0, ctypes.byref(l_), ctypes.byref(k_), ctr.ctypes.data, e.ctypes.data,
                              c.ctypes.data, ctypes.byref(fi))
    assert np.array_equal(c, b.shells[0].coefs)


@pytest.mark.parametrize("text,msg", [
    ("{", "Failed to parse BSE JSON"),
    ('{"elements": {}} x', "Failed to parse BSE JSON"),
    ('{"molssi_bse_schema": {"schema_type": "component"}, "elements": {}}', "Unsupported BSE schema type"),
    ('{"name": "x"}', "missing 'elements'"),
    ('{"elements": {"1": {"electron_shells": []}}}', "Z=8 not found"),
])
def test_errors(lai, text, msg):
    with pytest.raises(lai.LibAccIntError, match=msg):
        lai.BasisSet.from_bse_json(text, [8], np.zeros((1, 3)))


def test_string_escapes_and_numbers(lai):
    text = ('{"description": "tab\\t quote\\" \\u00e9 \\ud83d\\ude00", "n": -1.5e-3, "ok": true, "no": null,'
            '"elements": {"1": {"electron_shells": [{"angular_momentum": [0], "exponents": [1.25],'
            '"coefficients": [[1]]}]}}}')
    b = lai.BasisSet.from_bse_json(text, [1, 1], np.array([[0.0, 0, 0], [0, 0, 1.4]]))
    assert b.nbf == 2 and b.shells[0].exps[0] == 1.25


@pytest.mark.skipif(not os.path.isdir(REF_SHARE), reason="reference basis files absent")
@pytest.mark.parametrize("name", ["sto-3g", "6-31g", "cc-pvdz", "cc-pvtz", "cc-pvqz", "aug-cc-pvdz",
                                  "aug-cc-pvtz"])
def test_matches_bundled_data(lai, name):
    """Every bundled basis (H, C, N, O): the native loader on the BSE file gives the
    same shells and normalized coefficients as the package's Python loader."""
    text = open(os.path.join(REF_SHARE, name + ".json")).read()
    Z = [8, 1, 6, 7, 1]
    xyz = np.array([[0.0, 0.0, 0.0], [0.0, 1.4, -1.1], [2.5, 0.3, 0.1], [-2.0, 1.0, 0.5], [0.7, -1.9, 0.2]])
    nat = lai.BasisSet.from_bse_json(text, Z, xyz)
    py = lai.BasisSet.from_atoms(Z, xyz, name if name != "sto-3g" else "sto-3g-bse")
    assert _shells(nat) == _shells(py)
    py_norm = py.normalized_coefs()
    for s, c in zip(nat.shells, py_norm):
        assert np.allclose(s.coefs, c, rtol=1e-14, atol=0)
