"""Device Cartesian <-> spherical transforms against the host ones, and a
spherical J/K build (GPU)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_device_transforms_match_host(lai):
    import torch
    Z = np.array([6, 1, 8], dtype=np.int32)
    xyz = np.array([[0.0, 0.0, 0.0], [1.1, 0.7, -0.9], [-2.1, 0.4, 0.3]])
    b = lai.BasisSet.from_atoms(Z, xyz, "cc-pvqz")
    e = lai.Engine(b)
    rng = np.random.default_rng(2)
    n, ns = b.nbf, b.nbf_spherical
    M = rng.standard_normal((n, n))
    Ds = rng.standard_normal((ns, ns))
    dev = torch.device("cuda", 0)
    dM = torch.from_numpy(M).to(dev)
    dS = torch.empty((ns, ns), dtype=torch.float64, device=dev)
    dDs = torch.from_numpy(Ds).to(dev)
    dDc = torch.empty((n, n), dtype=torch.float64, device=dev)
    L = lai.lib()
    s = torch.cuda.current_stream().cuda_stream
    lai._lib.check(L.lai_cart_to_sph_2d_device(e._h, ctypes.c_void_p(dM.data_ptr()),
                                               ctypes.c_void_p(dS.data_ptr()), ctypes.c_void_p(s)))
    lai._lib.check(L.lai_sph_to_cart_density_device(e._h, ctypes.c_void_p(dDs.data_ptr()),
                                                    ctypes.c_void_p(dDc.data_ptr()), ctypes.c_void_p(s)))
    torch.cuda.synchronize()
    assert np.max(np.abs(dS.cpu().numpy() - b.cart_to_sph(M))) < 1e-12
    assert np.max(np.abs(dDc.cpu().numpy() - b.sph_to_cart_density(Ds))) < 1e-12


def test_spherical_jk_is_consistent(lai):
    """J_sph[D_sph] = T J_cart[T^T D_sph T] T^T, and the spherical energy equals the
    Cartesian energy of the transformed density."""
    w = lai.workloads.make("h2o2_ccpvdz")
    b = w.basis
    e = lai.Engine(b)
    rng = np.random.default_rng(3)
    C = rng.standard_normal((b.nbf_spherical, 10)) / np.sqrt(b.nbf_spherical)
    Ds = C @ C.T
    Js, Ks, _ = e.jk_spherical(Ds)
    Dc = b.sph_to_cart_density(Ds)
    Jc, Kc, _ = e.jk(Dc)
    Es = lai.molecules.energy(Ds, Js, Ks)
    Ec = lai.molecules.energy(Dc, Jc, Kc)
    assert abs(Es - Ec) < 1e-10 * max(1.0, abs(Ec))
    assert np.max(np.abs(Js - Js.T)) < 1e-12 and np.max(np.abs(Ks - Ks.T)) < 1e-12
