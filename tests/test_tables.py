"""The device root/Boys tables, evaluated by the device code compiled for the host
(rys_eval.h is host+device), against the binary128 oracle and mpmath (no GPU)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden

CSRC = os.path.join(ROOT, "libaccint-public_b200", "csrc")
HARNESS = r'''
#include "rys_tables.inc"
#include "rys_eval.h"
extern "C" void tab_rys(int n, double T, double* u, double* w) {
  lai::RysTablesView v{RYS_COEF_H, RYS_HERM_X2_H, RYS_HERM_W_H, BOYS_GRID_H};
  lai::rys_roots_table<double>(n, T, v, u, w);
}
extern "C" void tab_rys_one(int n, int r, double T, double* u, double* w) {
  lai::RysTablesView v{RYS_COEF_H, RYS_HERM_X2_H, RYS_HERM_W_H, BOYS_GRID_H};
  lai::rys_root_one<double>(n, r, T, v, *u, *w);
}
extern "C" void tab_boys01(double T, double* f) { lai::boys01<double>(T, BOYS_GRID_H, f[0], f[1]); }
'''


@pytest.fixture(scope="module")
def tab(tmp_path_factory):
    d = tmp_path_factory.mktemp("tab")
    src = d / "h.cpp"
    src.write_text(HARNESS)
    so = d / "libtab.so"
    subprocess.run(["g++", "-O2", "-ffp-contract=fast", "-shared", "-fPIC", "-I", CSRC, str(src),
                    "-o", str(so)], check=True)
    L = ctypes.CDLL(str(so))
    L.tab_rys.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    L.tab_rys_one.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    L.tab_boys01.argtypes = [ctypes.c_double, ctypes.c_void_p]
    return L


def _T_points():
    rng = np.random.default_rng(5)
    edges = []
    for n in range(2, 10):
        edges += [44.999, 45.001, 51.9999, 52.0, 86.9999, 87.0, 87.0001]
    return np.concatenate([[0.0, 1e-300, 1e-14, 0.05, 0.0499999, 39.95, 39.9499, 1e3, 1e8],
                           edges, rng.uniform(0, 100, 600), 10 ** rng.uniform(-10, 3, 200)])


@pytest.mark.parametrize("n", range(1, 10))
def test_rys_table_vs_oracle(tab, oracle, n):
    worst = 0.0
    for T in _T_points():
        u = np.zeros(n)
        w = np.zeros(n)
        tab.tab_rys(n, T, u.ctypes.data, w.ctypes.data)
        uo, wo = oracle.orc_rys(n, T)
        worst = max(worst, np.max(np.abs(u - uo) / uo), np.max(np.abs(w - wo) / wo))
        r = n - 1
        u1 = ctypes.c_double()
        w1 = ctypes.c_double()
        tab.tab_rys_one(n, r, T, ctypes.byref(u1), ctypes.byref(w1))
        assert u1.value == pytest.approx(u[r], rel=1e-15) and w1.value == pytest.approx(w[r], rel=1e-15)
    assert worst < 1.5e-15, worst


def test_boys01_vs_mpmath(tab):
    g = golden("boys_mpmath.npz")
    for T, F in zip(g["T"], g["F"]):
        f = np.zeros(2)
        tab.tab_boys01(T, f.ctypes.data)
        assert np.max(np.abs(f - F[:2]) / F[:2]) < 1e-15, T
