"""PyTorch autograd over the J/K energy: E(R, D) = 1/2 tr(D J[D]) - 1/4 tr(D K[D]).

    E = JKEnergy.apply(R, D, Z, basis_name)     # R: (natom, 3) Bohr, D: (nbf, nbf)
    E.backward()                                 # R.grad = dE/dR, D.grad = dE/dD

The forward pass stays on the device: D is used in place when it is a CUDA
float64 tensor (else copied to the engine's device once), J and K are built by
lai_jk_build_device into device tensors on the current torch stream, and E is
reduced there.  The engine (basis on the centres R, Schwarz bounds, screened
quartet list) is cached and rebuilt only when R, Z, the basis or the thresholds
change, so a loop over densities at fixed geometry pays for it once.  Backward
returns dE/dR from the device gradient kernel (lai_jk_gradient_device:
derivative integrals contracted with 4 D_ab D_cd - D_ac D_bd - D_ad D_bc, never
stored) and dE/dD = J - K/2 from the forward's J and K.

``fp32_cut`` > 0 runs the forward in mixed precision (FP32 for quartets with
Q_ij Q_kl max|D| below the cut, FP64 accumulation); the gradient kernel is
FP64 throughout, so dE/dR is the derivative of the FP64 energy, which the mixed
forward matches to well inside 1e-8 Eh at cut 1e-7.

The energy functional is the one of the screened build, so gradients and finite
differences agree as long as the screened quartet list does not change between
the displaced geometries (threshold=0 makes that exact).  No counterpart in the
reference, whose Python bindings expose no derivatives.
"""
import ctypes

import numpy as np

from . import _lib
from .basis import BasisSet
from .engine import Engine


def _torch():
    import torch
    return torch


class _EngineCache:
    """The engine of the last geometry: rebuilt when the key changes."""

    def __init__(self):
        self.key = None
        self.eng = None

    def get(self, Rn, Z, basis_name, threshold, prim_threshold, device):
        key = (Rn.tobytes(), tuple(int(z) for z in np.asarray(Z).ravel()), basis_name, threshold,
               prim_threshold, device)
        if key != self.key:
            basis = BasisSet.from_atoms(np.asarray(Z), Rn, basis_name)
            self.eng = Engine(basis, threshold=threshold, device=device, prim_threshold=prim_threshold)
            self.key = key
        return self.eng


_engines = _EngineCache()


def _device_of(*tensors):
    torch = _torch()
    for t in tensors:
        if t.is_cuda:
            return t.device
    return torch.device("cuda", torch.cuda.current_device())


def _make_function():
    torch = _torch()

    class JKEnergy(torch.autograd.Function):
        @staticmethod
        def forward(ctx, R, D, Z, basis_name="cc-pvdz", threshold=1e-12, prim_threshold=None,
                    fp32_cut=0.0):
            dev = _device_of(R, D)
            Rn = R.detach().to("cpu", torch.float64).numpy()
            eng = _engines.get(Rn, Z, basis_name, threshold, prim_threshold, dev.index)
            n = eng.basis.nbf
            if D.shape != (n, n):
                raise ValueError(f"density must be {n}x{n}")
            Dd = D.detach().to(dev, torch.float64).contiguous()
            J = torch.empty_like(Dd)
            K = torch.empty_like(Dd)
            stream = torch.cuda.current_stream(dev).cuda_stream
            eng.jk_device(Dd.data_ptr(), J.data_ptr(), K.data_ptr(), stream=stream, fp32_cut=fp32_cut)
            E = 0.5 * torch.sum(Dd * J) - 0.25 * torch.sum(Dd * K)
            ctx.eng = eng
            ctx.save_for_backward(Dd, J, K)
            ctx.R_meta = (R.dtype, R.device)
            ctx.D_meta = (D.dtype, D.device)
            return E.to(R.device)

        @staticmethod
        def backward(ctx, gE):
            Dd, J, K = ctx.saved_tensors
            g = gE.to(Dd.device, torch.float64)
            gR = gD = None
            if ctx.needs_input_grad[0]:
                eng = ctx.eng
                G = torch.empty((eng.natom(), 3), dtype=torch.float64, device=Dd.device)
                stream = torch.cuda.current_stream(Dd.device).cuda_stream
                _lib.check(_lib.lib().lai_jk_gradient_device(eng._h, ctypes.c_void_p(Dd.data_ptr()),
                                                             ctypes.c_void_p(G.data_ptr()),
                                                             ctypes.c_void_p(stream)))
                gR = (G * g).to(device=ctx.R_meta[1], dtype=ctx.R_meta[0])
            if ctx.needs_input_grad[1]:
                gD = ((J - 0.5 * K) * g).to(device=ctx.D_meta[1], dtype=ctx.D_meta[0])
            return gR, gD, None, None, None, None, None

    return JKEnergy


_cache = {}


def __getattr__(name):
    if name == "JKEnergy":
        if "JKEnergy" not in _cache:
            _cache["JKEnergy"] = _make_function()
        return _cache["JKEnergy"]
    raise AttributeError(name)


def jk_energy(R, D, Z, basis_name="cc-pvdz", threshold=1e-12, prim_threshold=None, fp32_cut=0.0):
    """E(R, D) with autograd support (see JKEnergy); fp32_cut > 0 = mixed-precision forward."""
    return __getattr__("JKEnergy").apply(R, D, Z, basis_name, threshold, prim_threshold, fp32_cut)
