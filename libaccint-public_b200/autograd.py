"""PyTorch autograd over the J/K energy: E(R, D) = 1/2 tr(D J[D]) - 1/4 tr(D K[D]).

    E = JKEnergy.apply(R, D, Z, basis_name)     # R: (natom, 3) Bohr, D: (nbf, nbf)
    E.backward()                                 # R.grad = dE/dR, D.grad = dE/dD

Forward builds the basis on the centres R, the engine (Schwarz bounds and the
screened quartet list) and J/K; backward returns dE/dR from the device gradient
kernel (derivative integrals contracted with 4 D_ab D_cd - D_ac D_bd - D_ad D_bc)
and dE/dD = J - K/2.  The energy functional is the one of the screened build, so
gradients and finite differences agree as long as the screened quartet list does
not change between the displaced geometries (threshold=0 makes that exact).
No counterpart in the reference, whose Python bindings expose no derivatives.
"""
import numpy as np

from .basis import BasisSet
from .engine import Engine


def _torch():
    import torch
    return torch


def _make_function():
    torch = _torch()

    class JKEnergy(torch.autograd.Function):
        @staticmethod
        def forward(ctx, R, D, Z, basis_name="cc-pvdz", threshold=1e-12, prim_threshold=None):
            Rn = R.detach().to("cpu", torch.float64).numpy()
            Dn = np.ascontiguousarray(D.detach().to("cpu", torch.float64).numpy())
            basis = BasisSet.from_atoms(np.asarray(Z), Rn, basis_name)
            eng = Engine(basis, threshold=threshold, prim_threshold=prim_threshold)
            J, K, _ = eng.jk(Dn)
            E = 0.5 * float(np.sum(Dn * J)) - 0.25 * float(np.sum(Dn * K))
            ctx.eng, ctx.D, ctx.J, ctx.K = eng, Dn, J, K
            ctx.R_meta = (R.dtype, R.device)
            ctx.D_meta = (D.dtype, D.device)
            return torch.tensor(E, dtype=torch.float64, device=R.device)

        @staticmethod
        def backward(ctx, gE):
            g = float(gE)
            gR = gD = None
            if ctx.needs_input_grad[0]:
                gR = torch.from_numpy(ctx.eng.gradient(ctx.D) * g).to(*ctx.R_meta[::-1])
            if ctx.needs_input_grad[1]:
                gD = torch.from_numpy((ctx.J - 0.5 * ctx.K) * g).to(*ctx.D_meta[::-1])
            return gR, gD, None, None, None, None

    return JKEnergy


_cache = {}


def __getattr__(name):
    if name == "JKEnergy":
        if "JKEnergy" not in _cache:
            _cache["JKEnergy"] = _make_function()
        return _cache["JKEnergy"]
    raise AttributeError(name)


def jk_energy(R, D, Z, basis_name="cc-pvdz", threshold=1e-12, prim_threshold=None):
    """E(R, D) with autograd support (see JKEnergy)."""
    return __getattr__("JKEnergy").apply(R, D, Z, basis_name, threshold, prim_threshold)
