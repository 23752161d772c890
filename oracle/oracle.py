"""Test infrastructure only: Python access to the two CPU checkers.

* ``restatement()`` -- liboracle.so, the plain-C restatement of the reference
  algorithm in rys_oracle.c (binary128 Rys roots, double ERIs, serial 8-fold
  symmetric J/K).  Built by ``make -C oracle restatement`` (no reference tree needed).
* ``reference()``   -- _ref/libref_oracle.so, the UNMODIFIED reference CPU code
  compiled from its own sources by oracle/Makefile, behind ref_shim.cpp.  None when
  it was not built (the reference tree is absent).
* ``reference_gpu()`` -- _ref/libref_gpu.so, the reference's own GPU route (its CUDA
  sources for sm_100a behind ref_gpu_shim.cu, ``make -C oracle refgpu``), used only to
  time the reference kernel on the same device (ref_gpu_bench.py).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
use this module.  The product (libaccint-public_b200) never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT = os.path.join(HERE, "liboracle.so")
REFERENCE = os.path.join(HERE, "_ref", "libref_oracle.so")
REFERENCE_GPU = os.path.join(HERE, "_ref", "libref_gpu.so")

_P, _I, _D, _L = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_long
_orc = None
_ref = None


def build_restatement():
    subprocess.run(["make", "-s", "-C", HERE, "restatement"], check=True)


def restatement():
    global _orc
    if _orc is None:
        if not os.path.exists(RESTATEMENT) or (
                os.path.exists(os.path.join(HERE, "rys_oracle.c")) and
                os.path.getmtime(os.path.join(HERE, "rys_oracle.c")) > os.path.getmtime(RESTATEMENT)):
            build_restatement()
        L = ctypes.CDLL(RESTATEMENT)
        L.orc_boys.argtypes = [_I, _D, _P]
        L.orc_rys.argtypes = [_I, _D, _P, _P]
        L.orc_normalize.argtypes = [_I, _I, _P, _P, _P]
        L.orc_eri_quartet.argtypes = [_P, _P, _P, _P, _P, _P]
        L.orc_basis_quartet.argtypes = [_I, _P, _P, _P, _P, _P, _I, _I, _I, _I, _P]
        L.orc_basis_quartets.argtypes = [_I, _P, _P, _P, _P, _P, _L, _P, _P]
        L.orc_jk_list.argtypes = [_I, _P, _P, _P, _P, _P, _P, _L, _P, _P, _P]
        L.orc_schwarz.argtypes = [_I, _P, _P, _P, _P, _P, _P]
        L.orc_jk_sym.argtypes = [_I, _P, _P, _P, _P, _P, _P, _P, _P, _D]
        L.orc_jk_sym.restype = ctypes.c_long
        L.orc_one_electron.argtypes = [_I, _P, _P, _P, _P, _P, _I, _I, _P, _P, _P]
        L.orc_eri3c.argtypes = [_I, _P, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P, _P]
        L.orc_eri2c.argtypes = [_I, _P, _P, _P, _P, _P, _P]
        _orc = L
    return _orc


def reference():
    """The compiled reference, or None if oracle/_ref was not built."""
    global _ref
    if _ref is None:
        if not os.path.exists(REFERENCE):
            return None
        L = ctypes.CDLL(REFERENCE)
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_basis_create.restype = _P
        L.ref_basis_create.argtypes = [_I, _P, _P, _P, _P, _P, _P]
        L.ref_basis_builtin_sto3g.restype = _P
        L.ref_basis_builtin_sto3g.argtypes = [_I, _P, _P]
        L.ref_basis_free.argtypes = [_P]
        L.ref_basis_nbf.restype = _L
        L.ref_basis_nbf.argtypes = [_P]
        L.ref_basis_nshell.restype = _L
        L.ref_basis_nshell.argtypes = [_P]
        L.ref_basis_shell.argtypes = [_P, _L, _P, _P, _P, _P, _P, _P]
        L.ref_jk_full.restype = _D
        L.ref_jk_full.argtypes = [_P, _P, _P, _P, _I]
        L.ref_jk_screened_sym.restype = _D
        L.ref_jk_screened_sym.argtypes = [_P, _P, _P, _P, _D]
        L.ref_eri_quartet.argtypes = [_P, _L, _L, _L, _L, _P]
        L.ref_schwarz.argtypes = [_P, _P]
        L.ref_schwarz_parallel.argtypes = [_P, _P, _I]
        L.ref_rys.argtypes = [_I, _D, _P, _P]
        L.ref_boys.argtypes = [_I, _D, _P]
        L.ref_time_quartets.restype = _D
        L.ref_time_quartets.argtypes = [_P, _P, _P, _L, _I, _P, _P]
        L.ref_max_threads.restype = _I
        L.ref_cart_to_sph.restype = _I
        L.ref_cart_to_sph.argtypes = [_I, _P]
        L.ref_one_electron.restype = _I
        L.ref_one_electron.argtypes = [_P, _I, _I, _P, _P, _P]
        L.ref_aux_builtin.restype = _P
        L.ref_aux_builtin.argtypes = [ctypes.c_char_p, _I, _P, _P]
        L.ref_aux_free.argtypes = [_P]
        L.ref_aux_nbf.restype = _L
        L.ref_aux_nbf.argtypes = [_P]
        L.ref_aux_nshell.restype = _L
        L.ref_aux_nshell.argtypes = [_P]
        L.ref_aux_shell.argtypes = [_P, _L, _P, _P, _P, _P, _P]
        L.ref_eri3c.argtypes = [_P, _P, _P]
        L.ref_eri2c.argtypes = [_P, _P]
        L.ref_df_jk.argtypes = [_P, _P, _P, _P, _P]
        _ref = L
    return _ref


_ref_gpu = None


def reference_gpu():
    """The reference's own GPU route (make -C oracle refgpu), or None if not built."""
    global _ref_gpu
    if _ref_gpu is None:
        if not os.path.exists(REFERENCE_GPU):
            return None
        L = ctypes.CDLL(REFERENCE_GPU)
        L.refgpu_last_error.restype = ctypes.c_char_p
        L.refgpu_basis_create.restype = _P
        L.refgpu_basis_create.argtypes = [_I, _P, _P, _P, _P, _P]
        L.refgpu_basis_free.argtypes = [_P]
        for f in ("refgpu_nbf", "refgpu_nsets"):
            getattr(L, f).restype = _L
            getattr(L, f).argtypes = [_P]
        L.refgpu_unit_size.argtypes = [_P, _L, _P, _P]
        L.refgpu_jk.argtypes = [_P, _P, _P, _P, _L, _L, _P, _P]
        _ref_gpu = L
    return _ref_gpu


class RefGpuBasis:
    """A basis inside the reference's GPU route (raw coefficients; the reference
    Shell constructor normalizes them).  Units are the ordered ShellSet 4-tuples."""

    def __init__(self, basis):
        L = reference_gpu()
        if L is None:
            raise RuntimeError("oracle/_ref/libref_gpu.so not built (make -C oracle refgpu)")
        self._L = L
        l, nprim, centers, exps, coefs, _ = basis.arrays()
        self._keep = [np.ascontiguousarray(a, dtype=t) for a, t in
                      ((l, np.int32), (nprim, np.int32), (centers, np.float64), (exps, np.float64),
                       (coefs, np.float64))]
        a = self._keep
        self._h = L.refgpu_basis_create(len(a[0]), *(x.ctypes.data for x in a))
        if not self._h:
            raise RuntimeError(L.refgpu_last_error().decode())
        self.nbf = int(L.refgpu_nbf(self._h))
        self.nsets = int(L.refgpu_nsets(self._h))
        self.nunits = self.nsets ** 4

    def unit_size(self, u):
        """(shell quartets, integral doubles) of unit u."""
        q, v = ctypes.c_long(), ctypes.c_long()
        if self._L.refgpu_unit_size(self._h, u, ctypes.byref(q), ctypes.byref(v)) != 0:
            raise ValueError("bad unit")
        return q.value, v.value

    def jk(self, D, u_begin=0, u_end=None):
        """(J, K, device ms, shell quartets) of units [u_begin, u_end) (all = full J/K)."""
        u_end = self.nunits if u_end is None else u_end
        D = np.ascontiguousarray(D, dtype=np.float64)
        J = np.zeros((self.nbf, self.nbf))
        K = np.zeros((self.nbf, self.nbf))
        ms, nq = ctypes.c_double(), ctypes.c_long()
        if self._L.refgpu_jk(self._h, D.ctypes.data, J.ctypes.data, K.ctypes.data, u_begin, u_end,
                             ctypes.byref(ms), ctypes.byref(nq)) != 0:
            raise RuntimeError(self._L.refgpu_last_error().decode())
        return J, K, ms.value, nq.value

    def __del__(self):
        if getattr(self, "_h", None):
            self._L.refgpu_basis_free(self._h)
            self._h = None


def ref_cart_to_sph(l):
    """The reference's math::get_cart_to_sph_matrix(l) (spherical_transform.hpp:20-40)."""
    R = reference()
    C = np.zeros((2 * l + 1, (l + 1) * (l + 2) // 2))
    if R.ref_cart_to_sph(l, C.ctypes.data) < 0:
        raise RuntimeError(R.ref_last_error().decode())
    return C


# ----------------------------------------------------------------------------
# Helpers on a libaccint BasisSet-like object (shells with l, center, exps, coefs)
# ----------------------------------------------------------------------------
def normalized_arrays(basis):
    """Flat arrays with coefficients normalized by the restatement (shell.cpp rule)."""
    O = restatement()
    l, nprim, centers, exps, coefs, atom = basis.arrays()
    out = np.zeros_like(coefs)
    off = 0
    for s in range(len(l)):
        k = int(nprim[s])
        e = np.ascontiguousarray(exps[off:off + k])
        c = np.ascontiguousarray(coefs[off:off + k])
        o = np.zeros(k)
        if basis.prenormalized:
            o[:] = c
        else:
            O.orc_normalize(int(l[s]), k, e.ctypes.data, c.ctypes.data, o.ctypes.data)
        out[off:off + k] = o
        off += k
    return l, nprim, centers, exps, out


def orc_jk(basis, D, thr=1e-12):
    O = restatement()
    l, nprim, centers, exps, coefs = normalized_arrays(basis)
    n = basis.nbf
    D = np.ascontiguousarray(D, dtype=np.float64)
    J = np.zeros((n, n))
    K = np.zeros((n, n))
    nq = O.orc_jk_sym(len(l), l.ctypes.data, nprim.ctypes.data, centers.ctypes.data,
                      exps.ctypes.data, coefs.ctypes.data, D.ctypes.data, J.ctypes.data,
                      K.ctypes.data, float(thr))
    return J, K, nq


def orc_quartet(basis, i, j, k, m):
    O = restatement()
    l, nprim, centers, exps, coefs = normalized_arrays(basis)
    nf = [(int(l[x]) + 1) * (int(l[x]) + 2) // 2 for x in (i, j, k, m)]
    out = np.zeros(int(np.prod(nf)))
    rc = O.orc_basis_quartet(len(l), l.ctypes.data, nprim.ctypes.data, centers.ctypes.data,
                             exps.ctypes.data, coefs.ctypes.data, i, j, k, m, out.ctypes.data)
    assert rc == 0
    return out.reshape(nf)


def orc_jk_list(basis, D, quartets, J, K):
    """Adds the 8-fold symmetric J/K contributions of listed canonical quartets."""
    O = restatement()
    l, nprim, centers, exps, coefs = normalized_arrays(basis)
    q = np.ascontiguousarray(quartets, dtype=np.int32)
    D = np.ascontiguousarray(D, dtype=np.float64)
    O.orc_jk_list(len(l), l.ctypes.data, nprim.ctypes.data, centers.ctypes.data, exps.ctypes.data,
                  coefs.ctypes.data, D.ctypes.data, len(q), q.ctypes.data, J.ctypes.data, K.ctypes.data)


def orc_quartets(basis, quartets):
    """Blocks of many quartets (int array [n][4] of shell indices), concatenated in
    order, each [a][b][c][d]; OpenMP over quartets."""
    O = restatement()
    l, nprim, centers, exps, coefs = normalized_arrays(basis)
    q = np.ascontiguousarray(quartets, dtype=np.int32)
    nc = (l + 1) * (l + 2) // 2
    sizes = nc[q[:, 0]] * nc[q[:, 1]] * nc[q[:, 2]] * nc[q[:, 3]]
    out = np.zeros(int(sizes.sum()))
    rc = O.orc_basis_quartets(len(l), l.ctypes.data, nprim.ctypes.data, centers.ctypes.data,
                              exps.ctypes.data, coefs.ctypes.data, len(q), q.ctypes.data, out.ctypes.data)
    assert rc == 0
    return out


def orc_schwarz(basis):
    O = restatement()
    l, nprim, centers, exps, coefs = normalized_arrays(basis)
    n = len(l)
    Q = np.zeros((n, n))
    O.orc_schwarz(n, l.ctypes.data, nprim.ctypes.data, centers.ctypes.data, exps.ctypes.data,
                  coefs.ctypes.data, Q.ctypes.data)
    return Q


def orc_one_electron(basis, kind, xyz=None, q=None):
    """kind 0 S, 1 T, 2 V (point charges xyz [n][3], q [n]) by the McMurchie-Davidson
    restatement in rys_oracle.c."""
    O = restatement()
    l, nprim, centers, exps, coefs = normalized_arrays(basis)
    n = basis.nbf
    out = np.zeros((n, n))
    nc = 0
    if kind == 2:
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(q, dtype=np.float64)
        nc = len(q)
    rc = O.orc_one_electron(len(l), l.ctypes.data, nprim.ctypes.data, centers.ctypes.data, exps.ctypes.data,
                            coefs.ctypes.data, kind, nc, None if xyz is None else xyz.ctypes.data,
                            None if q is None else q.ctypes.data, out.ctypes.data)
    if rc != 0:
        raise RuntimeError("orc_one_electron failed")
    return out


def orc_eri3c(basis, aux):
    """T[a][b][P] = (ab|P) by the restatement (orc_eri_quartet with a unit s shell)."""
    O = restatement()
    l, nprim, centers, exps, coefs = normalized_arrays(basis)
    lx, npx, cx, ex, cfx = normalized_arrays(aux)
    T = np.zeros((basis.nbf, basis.nbf, aux.nbf))
    rc = O.orc_eri3c(len(l), l.ctypes.data, nprim.ctypes.data, centers.ctypes.data, exps.ctypes.data,
                     coefs.ctypes.data, len(lx), lx.ctypes.data, npx.ctypes.data, cx.ctypes.data,
                     ex.ctypes.data, cfx.ctypes.data, T.ctypes.data)
    assert rc == 0
    return T


def orc_eri2c(aux):
    """V[P][Q] = (P|Q) by the restatement."""
    O = restatement()
    lx, npx, cx, ex, cfx = normalized_arrays(aux)
    V = np.zeros((aux.nbf, aux.nbf))
    assert O.orc_eri2c(len(lx), lx.ctypes.data, npx.ctypes.data, cx.ctypes.data, ex.ctypes.data,
                       cfx.ctypes.data, V.ctypes.data) == 0
    return V


def nuclear_repulsion(Z, xyz):
    xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    e = 0.0
    for i in range(len(Z)):
        for j in range(i + 1, len(Z)):
            e += float(Z[i]) * float(Z[j]) / float(np.linalg.norm(xyz[i] - xyz[j]))
    return e


def orc_rhf(S, H, jk, nocc, enuc, energy_threshold=1e-12, density_threshold=1e-10, max_iterations=100,
            diis_size=6):
    """Restricted Hartree-Fock in numpy, step for step the driver of the reference's
    tests/integration/test_hf_energy.cpp:64-294: symmetric orthogonalization
    X = U s^-1/2 U^T (eigenvalues <= 1e-10 dropped), core-Hamiltonian guess,
    D = 2 C_occ C_occ^T, F = H + J - K/2, E = 1/2 tr((H + F) D) + E_nuc, DIIS on
    e = F D S - S D F (last 6), convergence |dE| < 1e-12 and max |dD| < 1e-10 after
    the first iteration, final energy from a fresh build at the converged D.
    jk(D) -> (J, K).  Returns (E, iterations, converged)."""
    s, U = np.linalg.eigh(S)
    sinv = np.where(s > 1e-10, 1.0 / np.sqrt(np.where(s > 1e-10, s, 1.0)), 0.0)
    X = (U * sinv) @ U.T

    def solve(F):
        e, Cp = np.linalg.eigh(X.T @ F @ X)
        return X @ Cp

    def density(C):
        Co = C[:, :nocc]
        return 2.0 * Co @ Co.T

    D = density(solve(H))
    E_old = 0.0
    fs, es = [], []
    for it in range(max_iterations):
        J, K = jk(D)
        F = H + J - 0.5 * K
        E = 0.5 * float(np.sum((H + F) * D)) + enuc
        err = F @ D @ S - S @ D @ F
        fs.append(F)
        es.append(err)
        if len(fs) > diis_size:
            fs.pop(0)
            es.pop(0)
        if len(fs) < 2:
            Fd = fs[-1]
        else:
            m = len(fs)
            B = np.zeros((m + 1, m + 1))
            for i in range(m):
                for j in range(m):
                    B[i, j] = float(np.sum(es[i] * es[j]))
            B[m, :m] = B[:m, m] = -1.0
            rhs = np.zeros(m + 1)
            rhs[m] = -1.0
            c = np.linalg.lstsq(B, rhs, rcond=None)[0]
            Fd = sum(c[i] * fs[i] for i in range(m))
        Dn = density(solve(Fd))
        dD = float(np.max(np.abs(Dn - D)))
        if abs(E - E_old) < energy_threshold and dD < density_threshold and it > 0:
            D = Dn
            J, K = jk(D)
            F = H + J - 0.5 * K
            return 0.5 * float(np.sum((H + F) * D)) + enuc, it + 1, True
        D = Dn
        E_old = E
    return E_old, max_iterations, False


def orc_rys(n, T):
    O = restatement()
    u = np.zeros(n)
    w = np.zeros(n)
    O.orc_rys(n, float(T), u.ctypes.data, w.ctypes.data)
    return u, w


def orc_boys(mmax, T):
    O = restatement()
    f = np.zeros(mmax + 1)
    O.orc_boys(mmax, float(T), f.ctypes.data)
    return f


class RefBasis:
    """A reference BasisSet built from the same shells (reference normalization)."""

    def __init__(self, basis=None, builtin_sto3g=None):
        R = reference()
        if R is None:
            raise RuntimeError("oracle/_ref/libref_oracle.so not built")
        self.R = R
        if builtin_sto3g is not None:
            Z, xyz = builtin_sto3g
            Z = np.ascontiguousarray(Z, dtype=np.int32)
            xyz = np.ascontiguousarray(xyz, dtype=np.float64)
            self.h = R.ref_basis_builtin_sto3g(len(Z), Z.ctypes.data, xyz.ctypes.data)
        else:
            l, nprim, centers, exps, coefs, atom = basis.arrays()
            self._keep = (l, nprim, centers, exps, coefs, atom)
            self.h = R.ref_basis_create(len(l), l.ctypes.data, nprim.ctypes.data, centers.ctypes.data,
                                        exps.ctypes.data, coefs.ctypes.data, atom.ctypes.data)
        if not self.h:
            raise RuntimeError(R.ref_last_error().decode())
        self.nbf = R.ref_basis_nbf(self.h)
        self.nshell = R.ref_basis_nshell(self.h)

    def jk_full(self, D, nthreads=0):
        n = self.nbf
        D = np.ascontiguousarray(D, dtype=np.float64)
        J = np.zeros((n, n))
        K = np.zeros((n, n))
        t = self.R.ref_jk_full(self.h, D.ctypes.data, J.ctypes.data, K.ctypes.data, nthreads)
        if t < 0:
            raise RuntimeError(self.R.ref_last_error().decode())
        return J, K, t

    def jk_screened(self, D, thr):
        n = self.nbf
        D = np.ascontiguousarray(D, dtype=np.float64)
        J = np.zeros((n, n))
        K = np.zeros((n, n))
        t = self.R.ref_jk_screened_sym(self.h, D.ctypes.data, J.ctypes.data, K.ctypes.data, float(thr))
        if t < 0:
            raise RuntimeError(self.R.ref_last_error().decode())
        return J, K, t

    def quartet(self, i, j, k, m, shape):
        out = np.zeros(int(np.prod(shape)))
        rc = self.R.ref_eri_quartet(self.h, i, j, k, m, out.ctypes.data)
        assert rc == 0, self.R.ref_last_error().decode()
        return out.reshape(shape)

    def schwarz(self):
        Q = np.zeros((self.nshell, self.nshell))
        self.R.ref_schwarz(self.h, Q.ctypes.data)
        return Q

    def schwarz_parallel(self, nthreads=0):
        Q = np.zeros((self.nshell, self.nshell))
        rc = self.R.ref_schwarz_parallel(self.h, Q.ctypes.data, nthreads)
        if rc != 0:
            raise RuntimeError(self.R.ref_last_error().decode())
        return Q

    def time_quartets(self, D, quartets, nthreads=0, want_jk=False):
        n = self.nbf
        D = np.ascontiguousarray(D, dtype=np.float64)
        q = np.ascontiguousarray(quartets, dtype=np.int64).reshape(-1, 4)
        J = np.zeros((n, n)) if want_jk else None
        K = np.zeros((n, n)) if want_jk else None
        t = self.R.ref_time_quartets(self.h, D.ctypes.data, q.ctypes.data, len(q), nthreads,
                                     J.ctypes.data if want_jk else None,
                                     K.ctypes.data if want_jk else None)
        if t < 0:
            raise RuntimeError(self.R.ref_last_error().decode())
        return t, J, K

    def one_electron(self, kind, xyz=None, q=None):
        """kind 0 S, 1 T, 2 V of the point charges: the reference CPU engine's
        compute_overlap_matrix / compute_kinetic_matrix / compute_nuclear_matrix."""
        n = self.nbf
        out = np.zeros((n, n))
        nc = 0
        if kind == 2:
            xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
            q = np.ascontiguousarray(q, dtype=np.float64)
            nc = len(q)
        rc = self.R.ref_one_electron(self.h, kind, nc, None if xyz is None else xyz.ctypes.data,
                                     None if q is None else q.ctypes.data, out.ctypes.data)
        if rc != 0:
            raise RuntimeError(self.R.ref_last_error().decode())
        return out

    def shell_info(self, i):
        l = ctypes.c_int()
        k = ctypes.c_int()
        c = np.zeros(3)
        fi = ctypes.c_long()
        self.R.ref_basis_shell(self.h, i, ctypes.byref(l), ctypes.byref(k), c.ctypes.data, None, None,
                               ctypes.byref(fi))
        e = np.zeros(k.value)
        cf = np.zeros(k.value)
        self.R.ref_basis_shell(self.h, i, ctypes.byref(l), ctypes.byref(k), c.ctypes.data,
                               e.ctypes.data, cf.ctypes.data, ctypes.byref(fi))
        return l.value, c, e, cf, fi.value

    def __del__(self):
        if getattr(self, "h", None):
            self.R.ref_basis_free(self.h)
            self.h = None


class RefAux:
    """The reference's built-in auxiliary basis (data::create_builtin_auxiliary_basis)."""

    def __init__(self, name, Z, xyz):
        R = reference()
        if R is None:
            raise RuntimeError("oracle/_ref/libref_oracle.so not built")
        self.R = R
        Z = np.ascontiguousarray(Z, dtype=np.int32)
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        self.h = R.ref_aux_builtin(name.encode(), len(Z), Z.ctypes.data, xyz.ctypes.data)
        if not self.h:
            raise RuntimeError(R.ref_last_error().decode())
        self.nbf = R.ref_aux_nbf(self.h)
        self.nshell = R.ref_aux_nshell(self.h)

    def shells(self):
        """[(l, center, exps, normalized coefs)]"""
        out = []
        for i in range(self.nshell):
            l, k = ctypes.c_int(), ctypes.c_int()
            c = np.zeros(3)
            self.R.ref_aux_shell(self.h, i, ctypes.byref(l), ctypes.byref(k), c.ctypes.data, None, None)
            e, cf = np.zeros(k.value), np.zeros(k.value)
            self.R.ref_aux_shell(self.h, i, ctypes.byref(l), ctypes.byref(k), c.ctypes.data, e.ctypes.data,
                                 cf.ctypes.data)
            out.append((l.value, c, e, cf))
        return out

    def eri3c(self, ref_basis):
        T = np.zeros((ref_basis.nbf, ref_basis.nbf, self.nbf))
        assert self.R.ref_eri3c(ref_basis.h, self.h, T.ctypes.data) == 0, self.R.ref_last_error().decode()
        return T

    def eri2c(self):
        V = np.zeros((self.nbf, self.nbf))
        assert self.R.ref_eri2c(self.h, V.ctypes.data) == 0, self.R.ref_last_error().decode()
        return V

    def df_jk(self, ref_basis, D):
        n = ref_basis.nbf
        D = np.ascontiguousarray(D, dtype=np.float64)
        J, K = np.zeros((n, n)), np.zeros((n, n))
        rc = self.R.ref_df_jk(ref_basis.h, self.h, D.ctypes.data, J.ctypes.data, K.ctypes.data)
        if rc != 0:
            raise RuntimeError(self.R.ref_last_error().decode())
        return J, K

    def __del__(self):
        if getattr(self, "h", None):
            self.R.ref_aux_free(self.h)
            self.h = None


def df_jk_from_integrals(T, V, D, convention="exact"):
    """J and K of density fitting from three-centre T[a][b][P] and metric V[P][Q]
    (numpy, test infrastructure).  exact: B = T L^-T with V = L L^T, so B B^T =
    T V^-1 T^T.  reference: B = T L^-1, the B tensor of the reference's
    DFFockBuilder::compute_b_tensor (src/host/kernels/three_center_eri_kernel.cpp:
    364-387 with L_inv from math::triangular_inverse)."""
    n, naux = T.shape[0], T.shape[2]
    L = np.linalg.cholesky(V)
    Li = np.linalg.inv(L)
    Tm = T.reshape(n * n, naux)
    B = Tm @ (Li.T if convention == "exact" else Li)
    gamma = B.T @ D.reshape(-1)
    J = (B @ gamma).reshape(n, n)
    Bp = B.reshape(n, n, naux)
    K = np.einsum("abP,bd,cdP->ac", Bp, D, Bp)
    return J, K


class CanonicalQuartets:
    """The canonical Schwarz-screened shell quartets of a basis, from a Schwarz
    matrix Q: unordered pairs {P, Q'} of shell pairs with Q_P * Q_Q' >= thr
    (the reference's canonical loop, include/libaccint/engine/engine.hpp:1815-1858,
    with passes_screening).  Counts them and draws uniform samples, without
    materializing the list."""

    def __init__(self, Q, thr):
        n = Q.shape[0]
        i, j = np.triu_indices(n)
        q = Q[i, j]
        order = np.argsort(-q, kind="stable")
        self.pi, self.pj, self.q = i[order], j[order], q[order]
        # partners of sorted pair p: sorted positions r <= p with q[r] * q[p] >= thr
        neg = -self.q
        with np.errstate(divide="ignore"):
            lim = np.where(self.q > 0, thr / np.where(self.q > 0, self.q, 1.0), np.inf)
        cut = np.searchsorted(neg, -lim, side="right")
        # exact test at the boundary (product form, as the reference compares)
        self.count = np.minimum(cut, np.arange(len(self.q)) + 1).astype(np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.count)])
        self.total = int(self.offsets[-1])

    def sample(self, n, seed=0):
        rng = np.random.default_rng(seed)
        t = rng.integers(0, self.total, size=n)
        p = np.searchsorted(self.offsets, t, side="right") - 1
        r = t - self.offsets[p]
        return np.stack([self.pi[p], self.pj[p], self.pi[r], self.pj[r]], axis=1).astype(np.int64)
