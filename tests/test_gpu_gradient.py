"""Nuclear gradient of E = 1/2 tr(DJ) - 1/4 tr(DK) (GPU): central finite
differences (h = 1e-4 Bohr) of our own energy and of the reference's FockBuilder
energy, translational invariance, and the torch.autograd.Function wrapper.
Bar: 1e-7 Eh/Bohr against finite differences."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-7
H = 1e-4


def _energy(lai, Z, xyz, D, basis_name, thr=0.0):
    b = lai.BasisSet.from_atoms(Z, xyz, basis_name)
    e = lai.Engine(b, threshold=thr, prim_threshold=0.0)
    J, K, _ = e.jk(D)
    return lai.molecules.energy(D, J, K)


def _grad(lai, Z, xyz, D, basis_name, thr=0.0):
    b = lai.BasisSet.from_atoms(Z, xyz, basis_name)
    e = lai.Engine(b, threshold=thr, prim_threshold=0.0)
    return e.gradient(D)


def test_gradient_vs_finite_differences_h2o2_ccpvdz(lai):
    """Every coordinate of (H2O)2 / cc-pVDZ (no screening, so the energy is smooth)."""
    w = lai.workloads.make("h2o2_ccpvdz")
    g = _grad(lai, w.Z, w.xyz, w.D, "cc-pvdz")
    assert g.shape == (len(w.Z), 3)
    fd = np.zeros_like(g)
    for a in range(len(w.Z)):
        for x in range(3):
            xp = w.xyz.copy(); xp[a, x] += H
            xm = w.xyz.copy(); xm[a, x] -= H
            fd[a, x] = (_energy(lai, w.Z, xp, w.D, "cc-pvdz") - _energy(lai, w.Z, xm, w.D, "cc-pvdz")) / (2 * H)
    assert np.max(np.abs(g - fd)) < GRAD_TOL, np.max(np.abs(g - fd))
    assert np.max(np.abs(g.sum(axis=0))) < 1e-9  # translational invariance


def test_gradient_vs_reference_finite_differences(lai, oracle):
    """A seeded subset of coordinates of (H2O)2 / cc-pVDZ against central
    differences of the UNMODIFIED reference's energy (Engine::compute with a
    FockBuilder, full N^4)."""
    if oracle.reference() is None:
        pytest.skip("oracle/_ref not built")
    w = lai.workloads.make("h2o2_ccpvdz")
    g = _grad(lai, w.Z, w.xyz, w.D, "cc-pvdz")
    rng = np.random.default_rng(4)
    coords = [(int(a), int(x)) for a, x in zip(rng.integers(0, len(w.Z), 6), rng.integers(0, 3, 6))]

    def eref(xyz):
        R = oracle.RefBasis(lai.BasisSet.from_atoms(w.Z, xyz, "cc-pvdz"))
        J, K, _ = R.jk_full(w.D, 0)
        return lai.molecules.energy(w.D, J, K)

    for a, x in coords:
        xp = w.xyz.copy(); xp[a, x] += H
        xm = w.xyz.copy(); xm[a, x] -= H
        fd = (eref(xp) - eref(xm)) / (2 * H)
        assert abs(g[a, x] - fd) < GRAD_TOL, (a, x, g[a, x], fd)


def test_gradient_h2o16_screened(lai):
    """Config-4 system (H2O)16 / cc-pVDZ with the 1e-12 Schwarz cut: translational
    invariance and a few coordinates against finite differences of the screened
    energy (the displacement is far too small to change the screened list)."""
    w = lai.workloads.make("h2o16_ccpvdz")
    g = _grad(lai, w.Z, w.xyz, w.D, "cc-pvdz", thr=1e-12)
    assert np.max(np.abs(g.sum(axis=0))) < 1e-8
    for a, x in [(0, 0), (17, 1), (40, 2)]:
        xp = w.xyz.copy(); xp[a, x] += H
        xm = w.xyz.copy(); xm[a, x] -= H
        fd = (_energy(lai, w.Z, xp, w.D, "cc-pvdz", 1e-12) - _energy(lai, w.Z, xm, w.D, "cc-pvdz", 1e-12)) / (2 * H)
        assert abs(g[a, x] - fd) < GRAD_TOL, (a, x, g[a, x], fd)


def test_autograd_function(lai):
    import torch
    w = lai.workloads.make("h2o2_ccpvdz")
    R = torch.tensor(w.xyz, dtype=torch.float64, requires_grad=True)
    D = torch.tensor(w.D, dtype=torch.float64, requires_grad=True)
    E = lai.autograd.jk_energy(R, D, w.Z, "cc-pvdz", 0.0, 0.0)
    E.backward()
    b = lai.BasisSet.from_atoms(w.Z, w.xyz, "cc-pvdz")
    e = lai.Engine(b, threshold=0.0, prim_threshold=0.0)
    J, K, _ = e.jk(w.D)
    assert abs(E.item() - lai.molecules.energy(w.D, J, K)) < 1e-10
    assert np.max(np.abs(R.grad.numpy() - e.gradient(w.D))) < 1e-12
    assert np.max(np.abs(D.grad.numpy() - (J - 0.5 * K))) < 1e-12
    # dE/dD against a finite difference along a random symmetric direction
    rng = np.random.default_rng(0)
    X = rng.standard_normal(w.D.shape)
    X = 0.5 * (X + X.T)
    ep = lai.molecules.energy(w.D + 1e-5 * X, *e.jk(w.D + 1e-5 * X)[:2])
    em = lai.molecules.energy(w.D - 1e-5 * X, *e.jk(w.D - 1e-5 * X)[:2])
    assert abs((ep - em) / 2e-5 - np.sum(D.grad.numpy() * X)) < 1e-6



def test_autograd_mixed_forward_vs_finite_differences(lai):
    """Config 4's mixed-precision variant on (H2O)2 / cc-pVDZ: the forward in mixed
    precision (FP32 below Q_ij Q_kl max|D| = 1e-7), the gradient of every
    coordinate against central differences (h = 1e-4) of that same mixed forward,
    and the mixed energy against the FP64 one (bar 1e-8 Eh)."""
    import torch
    w = lai.workloads.make("h2o2_ccpvdz")
    dev = torch.device("cuda", 0)
    D = torch.tensor(w.D, dtype=torch.float64, device=dev)
    cut = 1e-7

    def e_mixed(xyz):
        R = torch.tensor(xyz, dtype=torch.float64)
        return lai.autograd.jk_energy(R, D, w.Z, "cc-pvdz", 0.0, 0.0, cut).item()

    R = torch.tensor(w.xyz, dtype=torch.float64, requires_grad=True)
    E = lai.autograd.jk_energy(R, D, w.Z, "cc-pvdz", 0.0, 0.0, cut)
    E.backward()
    E64 = lai.autograd.jk_energy(torch.tensor(w.xyz, dtype=torch.float64), D, w.Z, "cc-pvdz", 0.0, 0.0)
    assert abs(E.item() - E64.item()) < 1e-8
    g = R.grad.numpy()
    fd = np.zeros_like(g)
    for a in range(len(w.Z)):
        for x in range(3):
            xp = w.xyz.copy(); xp[a, x] += H
            xm = w.xyz.copy(); xm[a, x] -= H
            fd[a, x] = (e_mixed(xp) - e_mixed(xm)) / (2 * H)
    assert np.max(np.abs(g - fd)) < GRAD_TOL, np.max(np.abs(g - fd))


def test_autograd_device_tensors_and_engine_cache(lai):
    """CUDA tensors in, CUDA gradients out; a second density at the same geometry
    reuses the cached engine; a moved geometry rebuilds it."""
    import torch
    w = lai.workloads.make("h2o2_sto3g")
    dev = torch.device("cuda", 0)
    R = torch.tensor(w.xyz, dtype=torch.float64, device=dev, requires_grad=True)
    D = torch.tensor(w.D, dtype=torch.float64, device=dev, requires_grad=True)
    E = lai.autograd.jk_energy(R, D, w.Z, "sto-3g", 0.0, 0.0)
    E.backward()
    assert R.grad.is_cuda and D.grad.is_cuda and E.is_cuda
    eng = lai.autograd._engines.eng
    b = lai.BasisSet.from_atoms(w.Z, w.xyz, "sto-3g")
    e = lai.Engine(b, threshold=0.0, prim_threshold=0.0)
    assert np.max(np.abs(R.grad.cpu().numpy() - e.gradient(w.D))) < 1e-12
    lai.autograd.jk_energy(R.detach(), 2.0 * D.detach(), w.Z, "sto-3g", 0.0, 0.0)
    assert lai.autograd._engines.eng is eng
    lai.autograd.jk_energy(R.detach() + 0.01, D.detach(), w.Z, "sto-3g", 0.0, 0.0)
    assert lai.autograd._engines.eng is not eng


def test_gradient_h2o16_device_time(lai):
    """Config 4 (H2O)16 / cc-pVDZ, Schwarz 1e-12: device time of the J/K build and
    of the gradient kernel (CUDA events, after a warm-up), printed for the record."""
    import torch
    w = lai.workloads.make("h2o16_ccpvdz")
    e = lai.Engine(w.basis, threshold=1e-12)
    dev = torch.device("cuda", 0)
    D = torch.tensor(w.D, dtype=torch.float64, device=dev)
    J = torch.empty_like(D)
    K = torch.empty_like(D)
    G = torch.empty((e.natom(), 3), dtype=torch.float64, device=dev)
    s = torch.cuda.current_stream()
    import ctypes

    def grad():
        lai._lib.check(lai.lib().lai_jk_gradient_device(e._h, ctypes.c_void_p(D.data_ptr()),
                                                         ctypes.c_void_p(G.data_ptr()),
                                                         ctypes.c_void_p(s.cuda_stream)))

    def jk():
        e.jk_device(D.data_ptr(), J.data_ptr(), K.data_ptr(), stream=s.cuda_stream)

    out = {}
    for name, f in (("jk", jk), ("gradient", grad)):
        f()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for _ in range(3):
            f()
        b.record(s)
        torch.cuda.synchronize()
        out[name] = a.elapsed_time(b) / 3
    print(f"(H2O)16/cc-pVDZ: J/K build {out['jk']:.2f} ms, gradient {out['gradient']:.2f} ms")
    assert np.max(np.abs(G.sum(dim=0).cpu().numpy())) < 1e-8


def test_gradient_f_shells_vs_finite_differences(lai):
    """H2O / cc-pVTZ (f on O, d on H): the warp-per-quartet gradient kernel on the
    classes above d, and the thread-per-quartet ones on the rest, against central
    differences of our energy (no screening) on three coordinates."""
    w = lai.workloads.make("h2o1_ccpvtz")
    assert max(s.l for s in w.basis.shells) == 3
    g = _grad(lai, w.Z, w.xyz, w.D, "cc-pvtz")
    assert np.max(np.abs(g.sum(axis=0))) < 1e-9
    for a, x in [(0, 0), (1, 1), (2, 2)]:
        xp = w.xyz.copy(); xp[a, x] += H
        xm = w.xyz.copy(); xm[a, x] -= H
        fd = (_energy(lai, w.Z, xp, w.D, "cc-pvtz") - _energy(lai, w.Z, xm, w.D, "cc-pvtz")) / (2 * H)
        assert abs(g[a, x] - fd) < GRAD_TOL, (a, x, g[a, x], fd)

def test_gradient_requires_atoms(lai):
    w = lai.workloads.make("h2o1_sto3g")
    shells = [lai.Shell(s.l, s.center, s.exps, s.coefs) for s in w.basis.shells]  # atom = -1
    e = lai.Engine(lai.BasisSet(shells))
    with pytest.raises(lai.LibAccIntError):
        e.gradient(w.D)
