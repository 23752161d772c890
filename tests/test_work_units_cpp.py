"""The C++ work-unit and raw-integral adaptors (include/libaccint_b200.hpp):
ShellSet / ShellSetPair / ShellSetQuartet, Engine::compute_shell_set_quartet,
compute_batch, compute_batch_screened and GpuFockBuilder::accumulate_device_eri_batch,
driven by tests/cpp/work_unit_adaptor.cpp.

CPU: the program compiles and links, and its host-only mode checks the shell
sets, that the canonical lists of BasisSet::shell_set_quartets() hold every
permutation orbit exactly once, that the ordered units hold every ordered quartet
exactly once, and the orbit scatter, on a synthetic 8-fold symmetric integral.
GPU: every route gives the J and K of the full build (threshold 0)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "work_unit_adaptor.cpp")
LIBDIR = os.path.join(ROOT, "libaccint-public_b200")
TOL = 1e-10  # the J/K parity tolerance of the GPU tests


def _build(tmp_path):
    exe = tmp_path / "work_unit_adaptor"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-I",
           "/usr/local/cuda/include", SRC, "-o", str(exe), "-L", LIBDIR, "-laccint_b200", "-L",
           "/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath," + LIBDIR, "-Wl,-rpath,/usr/local/cuda/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _write_basis(path, basis):
    with open(path, "w") as f:
        for s in basis.shells:
            f.write(" ".join(map(str, [s.l, s.atom, *s.center, len(s.exps), *s.exps, *s.coefs])) + "\n")


@pytest.mark.parametrize("name", ["h2o1_ccpvdz", "h2o2_sto3g"])
def test_work_unit_enumeration_and_scatter_on_host(tmp_path, lai, name):
    exe = _build(tmp_path)
    w = lai.workloads.make(name)
    _write_basis(tmp_path / "basis.txt", w.basis)
    r = subprocess.run([str(exe), "cpu", str(tmp_path / "basis.txt")], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "0 failures" in r.stdout


@pytest.mark.gpu
def test_work_unit_routes_match_full_build(tmp_path, lai):
    exe = _build(tmp_path)
    w = lai.workloads.make("h2o1_ccpvdz")  # five shell sets: (s,9) (s,4) (p,4) (p,1) (d,1)
    _write_basis(tmp_path / "basis.txt", w.basis)
    np.savetxt(tmp_path / "D.txt", w.D.reshape(-1))
    r = subprocess.run([str(exe), "gpu", str(tmp_path / "basis.txt"), str(tmp_path / "D.txt"),
                        str(tmp_path / "out")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    J0, K0, _ = lai.Engine(w.basis, threshold=0.0).jk(w.D)
    n = w.nbf
    for route in ("sym", "gsym", "plain", "screened", "devbatch"):
        J = np.loadtxt(tmp_path / f"out_{route}_J.txt").reshape(n, n)
        K = np.loadtxt(tmp_path / f"out_{route}_K.txt").reshape(n, n)
        assert np.max(np.abs(J - J0)) < TOL, route
        assert np.max(np.abs(K - K0)) < TOL, route
