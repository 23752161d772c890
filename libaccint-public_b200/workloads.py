"""Named benchmark workloads (geometry + basis + density), seeded and reproducible.

  h2o8_sto3g      (H2O)8 on a 2x2x2 grid, built-in STO-3G, nocc 20, Schwarz 1e-12
  h2o64_ccpvdz    (H2O)64 on a 4x4x4 grid, cc-pVDZ, nocc 320, Schwarz 1e-12
  c12h26_ccpvtz   all-trans C12H26, cc-pVTZ, nocc 49
  c12h26_ccpvqz   all-trans C12H26, cc-pVQZ, nocc 49
  h2o16_ccpvdz    (H2O)16 on a 2x2x4 grid, cc-pVDZ, nocc 80
  clusters256     256 water clusters of U{1..12} waters, cc-pVDZ, nocc 5 per water
  h2oN_<basis>    small (H2O)N clusters for tests (N = 1, 2, 4, 8)

Densities are generated in the Cartesian basis the J/K build works in (the
reference's J/K path is Cartesian: src/host/kernels/eri_kernel.cpp).
"""
import numpy as np

from . import molecules
from .basis import BasisSet


class Workload:
    def __init__(self, name, Z, xyz, basis_name, nocc, seed, thr=1e-12):
        self.name = name
        self.Z = Z
        self.xyz = xyz
        self.basis_name = basis_name
        self.basis = BasisSet.from_atoms(Z, xyz, basis_name)
        self.nocc = nocc
        self.thr = thr
        rng = np.random.default_rng(seed + 7919)
        self.D = molecules.random_density(self.basis.nbf, nocc, rng)

    @property
    def nbf(self):
        return self.basis.nbf


_GRIDS = {"h2o1": (1, 1, 1), "h2o2": (2, 1, 1), "h2o4": (2, 2, 1), "h2o8": (2, 2, 2),
          "h2o16": (2, 2, 4), "h2o64": (4, 4, 4)}


def make(name, seed=0):
    if name.startswith("h2o") and "_" in name:
        key, bas = name.split("_", 1)
        dims = _GRIDS[key]
        n = dims[0] * dims[1] * dims[2]
        rng = np.random.default_rng(seed)
        Z, xyz = molecules.water_cluster(dims, rng)
        basis = {"sto3g": "sto-3g", "ccpvdz": "cc-pvdz", "ccpvtz": "cc-pvtz", "631g": "6-31g",
                 "ccpvqz": "cc-pvqz", "augccpvdz": "aug-cc-pvdz"}[bas]
        nocc = {"h2o8_sto3g": 20, "h2o64_ccpvdz": 320}.get(name, 5 * n)
        return Workload(name, Z, xyz, basis, nocc, seed)
    if name.startswith("c12h26_"):
        Z, xyz = molecules.alkane(12)
        basis = {"c12h26_ccpvtz": "cc-pvtz", "c12h26_ccpvqz": "cc-pvqz"}[name]
        return Workload(name, Z, xyz, basis, 49, seed)
    raise KeyError(name)


def clusters(n_clusters=256, seed=0, basis="cc-pvdz"):
    """The batched workload: independent clusters of U{1..12} waters."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(1, 13, size=n_clusters)
    out = []
    for i, n in enumerate(sizes):
        Z, xyz = molecules.water_cluster_n(int(n), rng)
        w = Workload(f"cluster{i}", Z, xyz, basis, 5 * int(n), seed * 100003 + i)
        out.append(w)
    return out
