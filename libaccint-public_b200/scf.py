"""Restricted Hartree-Fock with every matrix resident on the GPU.

    res = run_rhf(atoms, basis, n_electrons)        # atoms: [Atom] or [(Z, xyz)]
    res.total_energy, res.iterations, res.converged

The loop is the reference's RHF test driver (tests/integration/test_hf_energy.cpp:
64-294, the driver behind its PySCF-checked energies; the Python mini-app
examples/mini-apps/python-hf/hf.py:239-372 runs the same iteration):

* S and H_core = T + V from the one-electron kernels (lai_one_electron_device);
* symmetric orthogonalization X = U s^-1/2 U^T with eigenvalues <= 1e-10 dropped;
* core-Hamiltonian guess, D = 2 C_occ C_occ^T;
* per iteration: J/K from the device build on D, F = H + J - K/2,
  E = 1/2 tr((H + F) D) + E_nuc, DIIS over the last 6 Fock matrices with the
  error e = F D S - S D F, diagonalization of X^T F X;
* converged when |dE| < energy_threshold and max |dD| < density_threshold after
  the first iteration; the final energy comes from a fresh build at the
  converged density.

With ``aux`` (an auxiliary BasisSet) J and K come from density fitting
(df.DFFockBuilder) instead of the four-centre build.

D, F, J, K, S, H and the DIIS history stay in device memory (torch float64
tensors on the engine's device); only the energy, max |dD| and the DIIS
B-matrix cross the bus each iteration.  The symmetric eigensolver is
torch.linalg.eigh on the device.  Per-iteration times of the J/K build and of
the whole iteration are recorded with CUDA events.
"""
import numpy as np

from .basis import Atom, BasisSet, point_charges
from .engine import Engine


def _torch():
    import torch
    return torch


def nuclear_repulsion(atoms):
    xyz, q = point_charges(atoms)
    e = 0.0
    for i in range(len(q)):
        for j in range(i + 1, len(q)):
            e += q[i] * q[j] / float(np.linalg.norm(xyz[i] - xyz[j]))
    return e


class SCFResult:
    def __init__(self, total_energy, iterations, converged, energies, jk_ms, iter_ms, one_e_ms):
        self.total_energy = total_energy
        self.iterations = iterations
        self.converged = converged
        self.energies = energies          # total energy of every iteration
        self.jk_ms = jk_ms                # device time of each J/K build
        self.iter_ms = iter_ms            # device time of each whole iteration
        self.one_e_ms = one_e_ms          # S and H_core
        self.density = None               # converged D (device tensor)
        self.fock = None                  # F at the converged D (device tensor)
        self.orbital_energies = None

    def __repr__(self):
        return (f"SCFResult(total_energy={self.total_energy!r}, iterations={self.iterations}, "
                f"converged={self.converged})")


class RHF:
    """Device-resident RHF over an Engine (J/K and one-electron integrals from
    libaccint_b200.so).  ``fp32_cut`` enables the mixed-precision J/K build."""

    def __init__(self, basis, atoms=None, n_electrons=None, threshold=1e-12, device=0, fp32_cut=0.0,
                 diis_size=6, engine=None, aux=None):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("RHF runs on a CUDA device; none is available")
        self.basis = basis
        self.atoms = atoms if atoms is not None else basis.atoms
        if self.atoms is None:
            raise ValueError("atoms are required (the basis was not built from atoms)")
        _, q = point_charges(self.atoms)
        self.n_electrons = int(round(q.sum())) if n_electrons is None else int(n_electrons)
        if self.n_electrons % 2:
            raise ValueError("RHF needs an even number of electrons")
        self.nocc = self.n_electrons // 2
        self.engine = engine if engine is not None else Engine(basis, threshold=threshold, device=device)
        self.dev = torch.device("cuda", device)
        self.fp32_cut = fp32_cut
        self.diis_size = diis_size
        self.e_nuc = nuclear_repulsion(self.atoms)
        # density fitting: J/K from the auxiliary basis instead of the four-centre build
        self.df = None
        if aux is not None:
            from .df import DFFockBuilder
            self.df = DFFockBuilder(self.engine, aux)

    def _jk(self, D, J, K, stream, Cocc=None):
        if self.df is not None:
            if Cocc is not None:  # D = 2 Cocc Cocc^T: the exchange contracts with Cocc, no factoring
                self.df.set_orbitals(Cocc, 2.0)
            else:
                self.df.set_density(D)
            J.copy_(self.df.compute_coulomb())
            K.copy_(self.df.compute_exchange())
            return
        self.engine.jk_device(D.data_ptr(), J.data_ptr(), K.data_ptr(), stream=stream.cuda_stream,
                              fp32_cut=self.fp32_cut)

    def run(self, energy_threshold=1e-12, density_threshold=1e-10, max_iterations=100):
        torch = _torch()
        n = self.basis.nbf
        dev = self.dev
        with torch.cuda.device(dev):
            stream = torch.cuda.current_stream(dev)
            ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
            e0, e1 = ev(), ev()
            e0.record(stream)
            S = torch.empty((n, n), dtype=torch.float64, device=dev)
            H = torch.empty_like(S)
            self.engine.one_electron_device("overlap", S.data_ptr(), stream=stream.cuda_stream)
            self.engine.one_electron_device("hcore", H.data_ptr(), atoms=self.atoms, stream=stream.cuda_stream)
            e1.record(stream)
            s, U = torch.linalg.eigh(S)
            keep = s > 1e-10
            sinv = torch.where(keep, 1.0 / torch.sqrt(torch.where(keep, s, torch.ones_like(s))),
                               torch.zeros_like(s))
            X = (U * sinv) @ U.T

            def solve(F):
                eps, Cp = torch.linalg.eigh(X.T @ F @ X)
                return eps, X @ Cp

            def density(C):
                Co = C[:, :self.nocc]
                return 2.0 * (Co @ Co.T)

            _, C = solve(H)
            D = density(C)
            Cocc = C[:, :self.nocc]
            J = torch.empty_like(S)
            K = torch.empty_like(S)
            one_e_ms = e0.elapsed_time(e1)
            E_old = 0.0
            fock_hist, err_hist = [], []
            energies, jk_ms, iter_ms = [], [], []
            converged = False
            it = 0
            for it in range(max_iterations):
                a, b, c = ev(), ev(), ev()
                a.record(stream)
                self._jk(D, J, K, stream, Cocc)
                b.record(stream)
                F = H + J - 0.5 * K
                E = 0.5 * float(torch.sum((H + F) * D)) + self.e_nuc
                err = F @ D @ S - S @ D @ F
                fock_hist.append(F)
                err_hist.append(err)
                if len(fock_hist) > self.diis_size:
                    fock_hist.pop(0)
                    err_hist.pop(0)
                m = len(fock_hist)
                if m < 2:
                    Fd = fock_hist[-1]
                else:
                    E_mat = torch.stack([e.reshape(-1) for e in err_hist])
                    Bm = (E_mat @ E_mat.T).cpu().numpy()
                    B = np.zeros((m + 1, m + 1))
                    B[:m, :m] = Bm
                    B[m, :m] = B[:m, m] = -1.0
                    rhs = np.zeros(m + 1)
                    rhs[m] = -1.0
                    coef = np.linalg.lstsq(B, rhs, rcond=None)[0]
                    Fd = sum(float(coef[i]) * fock_hist[i] for i in range(m))
                eps, C = solve(Fd)
                Dn = density(C)
                Cn = C[:, :self.nocc]
                dD = float(torch.max(torch.abs(Dn - D)))
                c.record(stream)
                c.synchronize()
                jk_ms.append(a.elapsed_time(b))
                iter_ms.append(a.elapsed_time(c))
                energies.append(E)
                if abs(E - E_old) < energy_threshold and dD < density_threshold and it > 0:
                    D, Cocc = Dn, Cn
                    converged = True
                    break
                D, Cocc = Dn, Cn
                E_old = E
            if converged:
                a, b = ev(), ev()
                a.record(stream)
                self._jk(D, J, K, stream, Cocc)
                b.record(stream)
                F = H + J - 0.5 * K
                E_final = 0.5 * float(torch.sum((H + F) * D)) + self.e_nuc
                jk_ms.append(a.elapsed_time(b))
                res = SCFResult(E_final, it + 1, True, energies, jk_ms, iter_ms, one_e_ms)
                res.fock = F
                res.orbital_energies = eps
            else:
                res = SCFResult(E_old, max_iterations, False, energies, jk_ms, iter_ms, one_e_ms)
            res.density = D
            return res


def run_rhf(atoms, basis, n_electrons, energy_threshold=1e-12, density_threshold=1e-10, max_iterations=100,
            **opts):
    """run_rhf(atoms, basis, n_electrons, ...) of the reference's HF test driver
    (tests/integration/test_hf_energy.cpp:162-294) on the device."""
    return RHF(basis, atoms=atoms, n_electrons=n_electrons, **opts).run(energy_threshold, density_threshold,
                                                                          max_iterations)


def rhf_from_atoms(Z, xyz, basis_name, **opts):
    """Convenience: basis from the bundled data on atoms (Z, xyz in Bohr)."""
    basis = BasisSet.from_atoms(Z, xyz, basis_name)
    atoms = [Atom(z, r) for z, r in zip(Z, np.asarray(xyz, dtype=np.float64).reshape(-1, 3))]
    return RHF(basis, atoms=atoms, **opts)
