"""Basis sets: shells of contracted Cartesian Gaussians on atoms.

Mirrors the reference's ``Shell`` / ``BasisSet`` (include/libaccint/basis/shell.hpp,
src/shared/basis/basis_set.cpp): shells are emitted per atom in the order of the
basis-set data (the BSE reader's order, src/shared/data/bse_json_parser.cpp:27-87),
functions are numbered shell by shell, and contraction coefficients are given raw
and normalized by the library exactly like the reference Shell constructor.
"""
import ctypes
import json
import os

import numpy as np

from . import _lib

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "basis_sets.json")
_SYMBOL = {1: "H", 6: "C", 7: "N", 8: "O"}
_cache = None


def basis_data(name):
    """Per-element shell lists [(l, exps, coefs), ...] of a bundled basis set."""
    global _cache
    if _cache is None:
        with open(_DATA) as f:
            _cache = json.load(f)["basis_sets"]
    key = name.lower()
    if key in ("sto-3g", "sto3g"):
        key = "sto-3g-builtin"  # the reference's create_builtin_basis("sto-3g") data
    elif key == "sto-3g-bse":
        key = "sto-3g"          # the Basis Set Exchange file of the same name
    if key not in _cache:
        raise KeyError(f"basis set {name!r} not bundled (have {sorted(_cache)})")
    return _cache[key]


def cart_to_sph_matrix(l):
    """C_l [(2l+1) x (l+1)(l+2)/2] of real solid harmonics (spherical m = 0, 1, -1,
    ...; Cartesian lx, then ly descending) -- get_cart_to_sph_matrix of the reference."""
    C = np.zeros((2 * l + 1, (l + 1) * (l + 2) // 2))
    _lib.check(_lib.lib().lai_cart_to_sph_matrix(int(l), C.ctypes.data))
    return C


class Atom:
    """Atomic number and position (Bohr): data::Atom of the reference
    (include/libaccint/data/builtin_basis.hpp:17)."""
    __slots__ = ("atomic_number", "position")

    def __init__(self, atomic_number, position):
        self.atomic_number = int(atomic_number)
        self.position = np.asarray(position, dtype=np.float64).reshape(3)


def point_charges(atoms):
    """(xyz [n][3], q [n]) from a list of Atom or (Z, (x, y, z)) pairs, or from an
    object with x, y, z, charge sequences (PointChargeParams of the reference,
    include/libaccint/operators/operator_types.hpp:50-60)."""
    if hasattr(atoms, "charge"):
        xyz = np.stack([np.asarray(atoms.x, dtype=np.float64), np.asarray(atoms.y, dtype=np.float64),
                        np.asarray(atoms.z, dtype=np.float64)], axis=1)
        return np.ascontiguousarray(xyz), np.ascontiguousarray(atoms.charge, dtype=np.float64)
    xyz, q = [], []
    for a in atoms:
        if isinstance(a, Atom):
            q.append(float(a.atomic_number))
            xyz.append(a.position)
        else:
            z, r = a
            q.append(float(z))
            xyz.append(np.asarray(r, dtype=np.float64).reshape(3))
    return (np.ascontiguousarray(np.array(xyz, dtype=np.float64).reshape(-1, 3)),
            np.ascontiguousarray(q, dtype=np.float64))


class Shell:
    __slots__ = ("l", "center", "exps", "coefs", "atom")

    def __init__(self, l, center, exps, coefs, atom=-1):
        self.l = int(l)
        self.center = np.asarray(center, dtype=np.float64).reshape(3)
        self.exps = np.asarray(exps, dtype=np.float64)
        self.coefs = np.asarray(coefs, dtype=np.float64)
        self.atom = int(atom)

    @property
    def n_functions(self):
        return (self.l + 1) * (self.l + 2) // 2


class BasisSet:
    """A list of shells plus the C-ABI handle (created lazily)."""

    def __init__(self, shells, prenormalized=False):
        self.shells = list(shells)
        self.prenormalized = prenormalized
        self._handle = None
        self.atoms = None   # [Atom] when built by from_atoms

    @classmethod
    def from_atoms(cls, Z, xyz, name):
        data = basis_data(name)
        shells = []
        xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
        for a, (z, r) in enumerate(zip(Z, xyz)):
            sym = _SYMBOL.get(int(z))
            if sym is None or sym not in data:
                raise KeyError(f"element Z={z} not in basis {name}")
            for l, e, c in data[sym]:
                shells.append(Shell(l, r, e, c, a))
        b = cls(shells)
        b.atoms = [Atom(z, r) for z, r in zip(Z, xyz)]
        return b

    @classmethod
    def from_bse_json(cls, text, Z, xyz):
        """A basis from Basis Set Exchange JSON text parsed by the native loader
        (lai_basis_from_bse_json; data::BseJsonParser::parse of the reference).  The
        shells are read back from the library, so the Python side mirrors exactly
        what the C ABI built (coefficients already normalized)."""
        L = _lib.lib()
        raw = text.encode() if isinstance(text, str) else bytes(text)
        Zi = np.ascontiguousarray(Z, dtype=np.int32)
        R = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        h = ctypes.c_void_p()
        _lib.check(L.lai_basis_from_bse_json(raw, len(raw), len(Zi), Zi.ctypes.data, R.ctypes.data,
                                             ctypes.byref(h)))
        try:
            shells = []
            ns = L.lai_basis_nshell(h)
            for s in range(ns):
                l_, k_ = ctypes.c_int(), ctypes.c_int()
                c = np.zeros(3)
                fi = ctypes.c_long()
                L.lai_basis_shell(h, s, ctypes.byref(l_), ctypes.byref(k_), c.ctypes.data, None, None,
                                  ctypes.byref(fi))
                e = np.zeros(k_.value)
                cf = np.zeros(k_.value)
                L.lai_basis_shell(h, s, ctypes.byref(l_), ctypes.byref(k_), c.ctypes.data, e.ctypes.data,
                                  cf.ctypes.data, ctypes.byref(fi))
                atom = int(np.argmin(np.linalg.norm(R - c, axis=1))) if len(R) else -1
                shells.append(Shell(l_.value, c, e, cf, atom))
        finally:
            L.lai_basis_destroy(h)
        b = cls(shells, prenormalized=True)
        b.atoms = [Atom(z, r) for z, r in zip(Zi, R)]
        return b

    # --- flat arrays (the C-ABI layout) ---
    def arrays(self):
        l = np.array([s.l for s in self.shells], dtype=np.int32)
        nprim = np.array([len(s.exps) for s in self.shells], dtype=np.int32)
        centers = np.array([s.center for s in self.shells], dtype=np.float64).reshape(-1)
        exps = np.concatenate([s.exps for s in self.shells]) if self.shells else np.zeros(0)
        coefs = np.concatenate([s.coefs for s in self.shells]) if self.shells else np.zeros(0)
        atom = np.array([s.atom for s in self.shells], dtype=np.int32)
        return l, nprim, centers, np.ascontiguousarray(exps), np.ascontiguousarray(coefs), atom

    @property
    def n_shells(self):
        return len(self.shells)

    @property
    def nbf(self):
        return sum(s.n_functions for s in self.shells)

    @property
    def max_l(self):
        return max(s.l for s in self.shells)

    def function_offsets(self):
        off = np.zeros(len(self.shells) + 1, dtype=np.int64)
        for i, s in enumerate(self.shells):
            off[i + 1] = off[i] + s.n_functions
        return off

    def handle(self):
        if self._handle is None:
            L = _lib.lib()
            l, nprim, centers, exps, coefs, atom = self.arrays()
            self._arrs = (l, nprim, centers, exps, coefs, atom)
            h = ctypes.c_void_p()
            _lib.check(L.lai_basis_create(len(self.shells), l.ctypes.data, nprim.ctypes.data,
                                          centers.ctypes.data, exps.ctypes.data, coefs.ctypes.data,
                                          atom.ctypes.data,
                                          _lib.LAI_BASIS_PRENORMALIZED if self.prenormalized else 0,
                                          ctypes.byref(h)))
            self._handle = h
        return self._handle

    @property
    def nbf_spherical(self):
        return sum(2 * s.l + 1 for s in self.shells)

    def cart_to_sph(self, M_cart):
        """T M_cart T^T: a Cartesian two-index matrix (J, K, F) in the spherical basis."""
        n, ns = self.nbf, self.nbf_spherical
        M = np.ascontiguousarray(M_cart, dtype=np.float64)
        if M.shape != (n, n):
            raise ValueError(f"matrix must be {n}x{n}")
        out = np.empty((ns, ns))
        _lib.check(_lib.lib().lai_cart_to_sph_2d(self.handle(), M.ctypes.data, out.ctypes.data))
        return out

    def sph_to_cart_density(self, D_sph):
        """T^T D_sph T: a spherical density on the Cartesian functions the J/K path uses."""
        n, ns = self.nbf, self.nbf_spherical
        D = np.ascontiguousarray(D_sph, dtype=np.float64)
        if D.shape != (ns, ns):
            raise ValueError(f"density must be {ns}x{ns}")
        out = np.empty((n, n))
        _lib.check(_lib.lib().lai_sph_to_cart_density(self.handle(), D.ctypes.data, out.ctypes.data))
        return out

    def normalized_coefs(self):
        """Normalized coefficients per shell as computed by the library."""
        L = _lib.lib()
        out = []
        for i, s in enumerate(self.shells):
            e = np.zeros(len(s.exps))
            c = np.zeros(len(s.exps))
            li = ctypes.c_int()
            np_ = ctypes.c_int()
            ctr = np.zeros(3)
            fi = ctypes.c_long()
            _lib.check(L.lai_basis_shell(self.handle(), i, ctypes.byref(li), ctypes.byref(np_),
                                         ctr.ctypes.data, e.ctypes.data, c.ctypes.data, ctypes.byref(fi)))
            out.append(c)
        return out

    def __del__(self):
        if getattr(self, "_handle", None) is not None and _lib._lib is not None:
            _lib._lib.lai_basis_destroy(self._handle)
            self._handle = None
