"""The C++ adaptors (include/libaccint_b200.hpp): they compile against the C ABI
and link the library (CPU), and on the GPU the FockBuilder and GpuFockBuilder
routes give the same J/K as the Python engine."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "fock_builder_adaptor.cpp")
LIBDIR = os.path.join(ROOT, "libaccint-public_b200")


def _build(tmp_path):
    exe = tmp_path / "fock_builder_adaptor"
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
           SRC, "-o", str(exe), "-L", LIBDIR, "-laccint_b200", "-L", "/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath," + LIBDIR, "-Wl,-rpath,/usr/local/cuda/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_adaptor_compiles_and_links(tmp_path):
    assert _build(tmp_path).exists()


def test_one_electron_adaptor_compiles_and_links(tmp_path):
    exe = tmp_path / "one_electron_adaptor"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
           os.path.join(ROOT, "tests", "cpp", "one_electron_adaptor.cpp"), "-o", str(exe), "-L", LIBDIR,
           "-laccint_b200", "-L", "/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath," + LIBDIR,
           "-Wl,-rpath,/usr/local/cuda/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert exe.exists()


def test_reference_style_usage_compiles_and_links(tmp_path):
    """Code written with the reference's names (Shell(am, Point3D, ...), BasisSet({...}),
    consumers::FockBuilder, BackendHint, compute_core_hamiltonian, Real/Size) builds."""
    exe = tmp_path / "reference_style_usage"
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), "-I",
           "/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "reference_style_usage.cpp"), "-o",
           str(exe), "-L", LIBDIR, "-laccint_b200", "-L", "/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath," + LIBDIR, "-Wl,-rpath,/usr/local/cuda/lib64"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "warning" not in r.stderr, r.stderr


@pytest.mark.gpu
def test_reference_style_usage_runs(tmp_path):
    """The same program on the device: H2 / STO-3G overlap S01 at 1.4 Bohr (0.6593, the
    textbook value), a finite Fock element, and BackendHint::ForceCPU refused."""
    test_reference_style_usage_compiles_and_links(tmp_path)
    r = subprocess.run([str(tmp_path / "reference_style_usage")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    s01 = float(r.stdout.split("S01")[1].split()[0])
    assert abs(s01 - 0.6593182061) < 1e-9
    assert "ForceCPU refused: yes" in r.stdout


@pytest.mark.gpu
def test_adaptor_jk_matches_engine(tmp_path, lai):
    exe = _build(tmp_path)
    w = lai.workloads.make("h2o2_ccpvdz")
    with open(tmp_path / "basis.txt", "w") as f:
        for s in w.basis.shells:
            f.write(" ".join(map(str, [s.l, s.atom, *s.center, len(s.exps), *s.exps, *s.coefs])) + "\n")
    np.savetxt(tmp_path / "D.txt", w.D.reshape(-1))
    r = subprocess.run([str(exe), str(tmp_path / "basis.txt"), str(tmp_path / "D.txt"), str(tmp_path / "out")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    J0, K0, _ = lai.Engine(w.basis).jk(w.D)
    n = w.nbf
    for tag, ref in (("J", J0), ("K", K0), ("Jgpu", J0), ("Kgpu", K0)):
        M = np.loadtxt(tmp_path / f"out_{tag}.txt").reshape(n, n)
        assert np.max(np.abs(M - ref)) < 1e-12, tag
