"""Batched engine (many independent systems per launch) on the GPU: per-system
J/K equal the single-system builds, mixed precision stays within the energy bar
for every system, and the device path matches the host path."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _clusters(lai, n=6, seed=3):
    return lai.workloads.clusters(n_clusters=n, seed=seed)


def test_batched_equals_single_engines(lai):
    ws = _clusters(lai)
    be = lai.BatchedEngine([w.basis for w in ws])
    Js, Ks, rep = be.jk([w.D for w in ws])
    nq = 0
    for w, J, K in zip(ws, Js, Ks):
        e = lai.Engine(w.basis)
        J0, K0, r0 = e.jk(w.D)
        nq += r0.quartets_fp64
        assert np.max(np.abs(J - J0)) < 1e-12
        assert np.max(np.abs(K - K0)) < 1e-12
    assert rep.quartets_fp64 == nq


def test_batched_mixed_precision_per_system_energy(lai):
    ws = _clusters(lai, n=8, seed=5)
    be = lai.BatchedEngine([w.basis for w in ws])
    J0, K0, _ = be.jk([w.D for w in ws])
    J1, K1, rep = be.jk([w.D for w in ws], fp32_cut=1e-7)
    assert rep.quartets_fp32 > 0
    for w, a, b, c, d in zip(ws, J0, K0, J1, K1):
        dE = lai.molecules.energy(w.D, c, d) - lai.molecules.energy(w.D, a, b)
        assert abs(dE) < 1e-8


def test_batched_device_path(lai):
    import torch
    ws = _clusters(lai, n=4, seed=9)
    be = lai.BatchedEngine([w.basis for w in ws])
    Jh, Kh, _ = be.jk([w.D for w in ws])
    dev = torch.device("cuda", 0)
    D = torch.from_numpy(be.pack([w.D for w in ws])).to(dev)
    J = torch.empty_like(D)
    K = torch.empty_like(D)
    be.jk_device(D.data_ptr(), J.data_ptr(), K.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    for s, (a, b) in enumerate(zip(be.unpack(J.cpu().numpy()), be.unpack(K.cpu().numpy()))):
        assert np.max(np.abs(a - Jh[s])) < 1e-13 and np.max(np.abs(b - Kh[s])) < 1e-13


def test_batched_rejects_single_matrix_calls(lai):
    ws = _clusters(lai, n=2, seed=1)
    be = lai.BatchedEngine([w.basis for w in ws])
    L = lai.lib()
    D = np.zeros((4, 4))
    assert L.lai_jk_build(be._h, D.ctypes.data, 4, D.ctypes.data, D.ctypes.data, None, None) == -1
    Q = np.zeros(16)
    assert L.lai_engine_schwarz(be._h, Q.ctypes.data) == -6


def test_graph_replay_matches_plain_build(lai):
    """CUDA-graph mode: the capture call and later replays (after the density
    changed in place) give the plain build's J/K."""
    import torch
    ws = _clusters(lai, n=5, seed=11)
    be = lai.BatchedEngine([w.basis for w in ws])
    dev = torch.device("cuda", 0)
    s = torch.cuda.Stream()
    D = torch.from_numpy(be.pack([w.D for w in ws])).to(dev)
    J = torch.empty_like(D)
    K = torch.empty_like(D)
    Jr = torch.empty_like(D)
    Kr = torch.empty_like(D)
    for scale in (1.0, 0.5, 2.0):
        with torch.cuda.stream(s):
            D.copy_(torch.from_numpy(be.pack([scale * w.D for w in ws])).to(dev))
            be.jk_device(D.data_ptr(), J.data_ptr(), K.data_ptr(), stream=s.cuda_stream, graph=True)
            be.jk_device(D.data_ptr(), Jr.data_ptr(), Kr.data_ptr(), stream=s.cuda_stream)
        s.synchronize()
        assert torch.max(torch.abs(J - Jr)).item() < 1e-12
        assert torch.max(torch.abs(K - Kr)).item() < 1e-12
    with pytest.raises(lai.LibAccIntError):
        be.jk_device(D.data_ptr(), J.data_ptr(), K.data_ptr(), stream=s.cuda_stream, graph=True, profile=True)
