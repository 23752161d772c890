"""The allocation-free J/K entry point, lai_jk_build_noalloc (GPU).

It serves callers that cannot allocate device memory when they ask for J and K
(a host application that owns all device memory through its own allocator, or a
real-time loop that forbids allocation after start-up).  Its accumulators live in a fixed
array inside the library's device image, so its results must match
lai_jk_build_device() -- which allocates its accumulators -- call after call,
and it must refuse bases larger than the array.  This file sorts last so that a
failure here does not hide the other tests of a run that stops at the first.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10  # the J/K parity tolerance used across the GPU tests


def _call_noalloc(lai, eng, D, J, K, stream):
    return lai.lib().lai_jk_build_noalloc(eng._h, ctypes.c_void_p(D.data_ptr()),
                                          ctypes.c_void_p(J.data_ptr()),
                                          ctypes.c_void_p(K.data_ptr()), ctypes.c_void_p(stream))


def test_noalloc_matches_allocating_build_twice(lai):
    import torch
    w = lai.workloads.make("h2o2_ccpvdz")
    eng = lai.Engine(w.basis)
    n = w.nbf
    dev = torch.device("cuda", 0)
    D = torch.from_numpy(w.D).to(dev)
    J0 = torch.empty((n, n), dtype=torch.float64, device=dev)
    K0 = torch.empty_like(J0)
    stream = torch.cuda.current_stream().cuda_stream
    eng.jk_device(D.data_ptr(), J0.data_ptr(), K0.data_ptr(), stream=stream)
    for _ in range(2):  # twice in a row: the shared accumulators must be cleared every call
        J1 = torch.full((n, n), np.nan, dtype=torch.float64, device=dev)
        K1 = torch.full((n, n), np.nan, dtype=torch.float64, device=dev)
        rc = _call_noalloc(lai, eng, D, J1, K1, stream)
        assert rc == 0, lai.lib().lai_last_error()
        torch.cuda.synchronize()
        assert torch.max(torch.abs(J1 - J0)).item() < TOL
        assert torch.max(torch.abs(K1 - K0)).item() < TOL


def test_noalloc_rejects_basis_above_limit(lai):
    import torch
    big = lai.workloads.make("h2o64_ccpvdz")  # 1600 functions, above the 512 limit
    eng = lai.Engine(big.basis)
    dev = torch.device("cuda", 0)
    D = torch.zeros((4, 4), dtype=torch.float64, device=dev)
    rc = _call_noalloc(lai, eng, D, D, D, torch.cuda.current_stream().cuda_stream)
    assert rc == -1
    assert b"LAI_NOALLOC_MAX_NBF" in lai.lib().lai_last_error()


def test_noalloc_g_shells_match_allocating_build(lai):
    """(H2O)2/cc-pVQZ (280 functions, classes up to (gg|gg)): every class the
    allocation-free path runs, f and g included, against the allocating build."""
    import torch
    w = lai.workloads.make("h2o2_ccpvqz")
    assert w.nbf <= 512
    eng = lai.Engine(w.basis)
    n = w.nbf
    dev = torch.device("cuda", 0)
    D = torch.from_numpy(w.D).to(dev)
    J0 = torch.empty((n, n), dtype=torch.float64, device=dev)
    K0 = torch.empty_like(J0)
    stream = torch.cuda.current_stream().cuda_stream
    eng.jk_device(D.data_ptr(), J0.data_ptr(), K0.data_ptr(), stream=stream)
    J1 = torch.full((n, n), np.nan, dtype=torch.float64, device=dev)
    K1 = torch.full((n, n), np.nan, dtype=torch.float64, device=dev)
    rc = _call_noalloc(lai, eng, D, J1, K1, stream)
    assert rc == 0, lai.lib().lai_last_error()
    torch.cuda.synchronize()
    assert torch.max(torch.abs(J1 - J0)).item() < TOL
    assert torch.max(torch.abs(K1 - K0)).item() < TOL
