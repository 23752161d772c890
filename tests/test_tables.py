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
#include "fp32_tables.h"
static float g_boys32[lai::kBoysF32Rows * lai::kBoysF32Stride];
static float g_rys32[2 * lai::kRysF32Len];
extern "C" void tab_f32_build() {
  lai::build_boys_f32(BOYS_GRID_H, g_boys32);
  lai::build_rys_f32(RYS_COEF_H, g_rys32);
}
extern "C" void tab_boys01_f32(double T, double* f) {
  float F0, F1;
  lai::boys01_f32((float)T, g_boys32, F0, F1);
  f[0] = F0; f[1] = F1;
}
extern "C" void tab_rys_f32(int n, double T, double* u, double* w) {
  float uf[lai::kMaxRoots], wf[lai::kMaxRoots];
  lai::rys_f32(n, (float)T, g_rys32 + 2 * lai::rys_f32_off(n), RYS_HERM_X2_H, RYS_HERM_W_H, uf, wf);
  for (int r = 0; r < n; ++r) { u[r] = uf[r]; w[r] = wf[r]; }
}
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
    L.tab_boys01_f32.argtypes = [ctypes.c_double, ctypes.c_void_p]
    L.tab_rys_f32.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
    L.tab_f32_build()
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


def _f32_points():
    """T values exactly representable in float (the FP32 kernels see float T)."""
    T = np.concatenate([_T_points(), np.arange(0, 24, 1 / 64), [23.9375, 23.93749, 23.9376, 44.5, 45.0, 45.5]])
    return np.unique(T.astype(np.float32).astype(np.float64))


def test_boys01_f32_vs_oracle(tab, oracle):
    """FP32 Boys grid (step 1/16, 4 Taylor terms) and its asymptotic branch
    against the binary128 oracle: within 1.5e-7 relative on the grid (FP32
    rounding of a few operations on top of the < 1.1e-8 truncation bound of
    fp32_tables.h) and 5e-7 above it (rounding of 1/sqrt(T) and three products)."""
    worst_grid = worst_asym = 0.0
    for T in _f32_points():
        f = np.zeros(2)
        tab.tab_boys01_f32(T, f.ctypes.data)
        uo, wo = oracle.orc_rys(1, T)  # one-point rule: w = F_0, u = F_1 / F_0
        F0, F1 = wo[0], uo[0] * wo[0]
        e = max(abs(f[0] - F0) / F0, abs(f[1] - F1) / F1)
        if T < 23.9375:
            worst_grid = max(worst_grid, e)
        else:
            worst_asym = max(worst_asym, e)
    assert worst_grid < 1.5e-7, worst_grid
    assert worst_asym < 5e-7, worst_asym


@pytest.mark.parametrize("n", range(2, 10))
def test_rys_f32_vs_oracle(tab, oracle, n):
    """Degree-6 FP32 Rys fits: roots and weights within 3e-7 relative (the
    < 2.4e-8 truncation of the degree-11 fits plus FP32 rounding of the Horner
    steps, or of 1/sqrt(T) and one product in the Gauss-Hermite limit)."""
    worst = 0.0
    for T in _f32_points():
        u = np.zeros(n)
        w = np.zeros(n)
        tab.tab_rys_f32(n, T, u.ctypes.data, w.ctypes.data)
        uo, wo = oracle.orc_rys(n, T)
        worst = max(worst, np.max(np.abs(u - uo) / uo), np.max(np.abs(w - wo) / wo))
    assert worst < 3e-7, worst
