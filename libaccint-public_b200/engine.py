"""Python surface mirroring the reference's operator/consumer API for the J/K path.

    basis = BasisSet.from_atoms(Z, xyz, "cc-pvdz")
    engine = Engine(basis)
    fb = FockBuilder(basis.nbf)
    fb.set_density(D)
    engine.compute(Operator.coulomb(), fb)          # Engine::compute(op, FockBuilder&)
    J, K = fb.get_coulomb_matrix(), fb.get_exchange_matrix()

Reference counterparts: Engine (include/libaccint/engine/engine.hpp:86-107,
435-499, 727-731, 1635-1666), FockBuilder (include/libaccint/consumers/fock_builder.hpp,
src/shared/consumers/fock_builder.cpp), ScreeningOptions
(include/libaccint/screening/screening_options.hpp).  Every call goes through the
C ABI of libaccint_b200.so; there is no CPU path.
"""
import ctypes

import numpy as np

from . import _lib
from .basis import point_charges


class Operator:
    """Only the Coulomb two-electron operator is on this path."""

    def __init__(self, kind):
        self.kind = kind

    @staticmethod
    def coulomb():
        return Operator("coulomb")

    def is_two_electron(self):
        return self.kind == "coulomb"


class ScreeningOptions:
    def __init__(self, threshold=1e-12, enabled=True, use_permutation_symmetry=True):
        self.threshold = threshold
        self.enabled = enabled
        self.use_permutation_symmetry = use_permutation_symmetry

    @staticmethod
    def normal():
        return ScreeningOptions(1e-12)

    @staticmethod
    def tight():
        return ScreeningOptions(1e-14)

    @staticmethod
    def loose():
        return ScreeningOptions(1e-10)

    @staticmethod
    def none():
        """Every quartet (screening_options.hpp: threshold 0, disabled)."""
        return ScreeningOptions(0.0, enabled=False)

    def effective_threshold(self):
        return self.threshold if self.enabled else 0.0


class FockBuilder:
    """J/K accumulator (reference consumers::FockBuilder).  J and K accumulate
    across compute calls until reset(), like the reference's J_/K_ buffers."""

    def __init__(self, nbf):
        self.nbf = int(nbf)
        self.J = np.zeros((self.nbf, self.nbf))
        self.K = np.zeros((self.nbf, self.nbf))
        self.D = None
        self.last_report = None

    def set_density(self, D, nbf=None):
        D = np.ascontiguousarray(D, dtype=np.float64)
        n = D.shape[0] if nbf is None else int(nbf)
        if n != self.nbf or D.shape != (self.nbf, self.nbf):
            raise ValueError(f"FockBuilder::set_density: nbf mismatch (expected {self.nbf}, got {n})")
        self.D = D

    def get_coulomb_matrix(self):
        return self.J

    def get_exchange_matrix(self):
        return self.K

    def get_fock_matrix(self, H_core, exchange_fraction=0.5):
        H = np.asarray(H_core, dtype=np.float64).reshape(self.nbf, self.nbf)
        return H + self.J - exchange_fraction * self.K

    def reset(self):
        self.J[:] = 0.0
        self.K[:] = 0.0


class GpuFockBuilder:
    """Device J/K accumulator (reference consumers::GpuFockBuilder,
    include/libaccint/consumers/fock_builder_gpu.hpp:46-159, and its Python binding,
    python/src/advanced_bindings.cpp:680-749).  D, J and K are float64 torch
    tensors on the device (``d_D``, ``d_J``, ``d_K``); set_density uploads D,
    get_coulomb_matrix / get_exchange_matrix / get_fock_matrix download.  J and K
    accumulate across Engine.compute calls until reset().  As in the reference
    binding, ``nbf()`` is a method and get_fock_matrix defaults to
    exchange_fraction = 1.0."""

    def __init__(self, nbf, device=0):
        import torch
        self._torch = torch
        self._nbf = int(nbf)
        self.device = torch.device("cuda", device)
        self.d_D = torch.zeros((self._nbf, self._nbf), dtype=torch.float64, device=self.device)
        self.d_J = torch.zeros_like(self.d_D)
        self.d_K = torch.zeros_like(self.d_D)
        self.has_density = False
        self.last_report = None

    def nbf(self):
        return self._nbf

    def set_density(self, D):
        D = np.ascontiguousarray(D, dtype=np.float64)
        if D.size != self._nbf * self._nbf:
            raise ValueError("Density matrix must have nbf*nbf elements")
        self.d_D.copy_(self._torch.from_numpy(D.reshape(self._nbf, self._nbf)))
        self.has_density = True

    def get_coulomb_matrix(self):
        return self.d_J.cpu().numpy()

    def get_exchange_matrix(self):
        return self.d_K.cpu().numpy()

    def get_fock_matrix(self, H_core, exchange_fraction=1.0):
        H = np.asarray(H_core, dtype=np.float64)
        if H.size != self._nbf * self._nbf:
            raise ValueError("H_core must have nbf*nbf elements")
        Hd = self._torch.from_numpy(np.ascontiguousarray(H).reshape(self._nbf, self._nbf)).to(self.device)
        return (Hd + self.d_J - exchange_fraction * self.d_K).cpu().numpy()

    def reset(self):
        self.d_J.zero_()
        self.d_K.zero_()

    def synchronize(self):
        self._torch.cuda.synchronize(self.device)

    def __repr__(self):
        return f"GpuFockBuilder(nbf={self._nbf})"


class Engine:
    def __init__(self, basis, threshold=1e-12, device=0, prim_threshold=None):
        """``prim_threshold``: primitive-quartet cut (None = 1e-3 * threshold, 0 = off)."""
        self.basis = basis
        self.threshold = threshold
        self.device = device
        L = _lib.lib()
        opts = _lib.EngineOpts()
        L.lai_engine_opts_default(ctypes.byref(opts))
        opts.schwarz_threshold = threshold
        opts.device = device
        if prim_threshold is not None:
            opts.prim_threshold = prim_threshold
        h = ctypes.c_void_p()
        _lib.check(L.lai_engine_create(basis.handle(), ctypes.byref(opts), ctypes.byref(h)))
        self._h = h

    def schwarz(self):
        n = self.basis.n_shells
        Q = np.zeros((n, n))
        _lib.check(_lib.lib().lai_engine_schwarz(self._h, Q.ctypes.data))
        return Q

    @staticmethod
    def _opts(fp32_cut=0.0, check_symmetric=False, shard=(0, 1), profile=False, graph=False, fp32_prim_rel=0.0):
        opts = _lib.JKOpts()
        _lib.lib().lai_jk_opts_default(ctypes.byref(opts))
        opts.fp32_cut = fp32_cut
        opts.fp32_prim_rel = fp32_prim_rel
        opts.check_symmetric = int(check_symmetric)
        opts.shard_index, opts.shard_count = shard
        opts.profile = int(profile)
        opts.graph = int(graph)
        return opts

    def jk(self, D, fp32_cut=0.0, check_symmetric=False, shard=(0, 1), profile=False, out=None,
           fp32_prim_rel=0.0):
        """(J, K, report) for a host density D.  ``out`` = (J, K) host arrays to
        fill (e.g. pinned memory); ``shard`` = (index, count) computes one
        rank's partial J/K of a multi-GPU build; ``fp32_prim_rel`` skips, in the
        FP32 quartets only, primitive quartets below that fraction of the
        quartet's Schwarz bound (lai_jk_opts.fp32_prim_rel)."""
        L = _lib.lib()
        n = self.basis.nbf
        D = np.ascontiguousarray(D, dtype=np.float64)
        if D.shape != (n, n):
            raise ValueError(f"density must be {n}x{n}")
        if out is None:
            J = np.empty((n, n))
            K = np.empty((n, n))
        else:
            J, K = out
        opts = self._opts(fp32_cut, check_symmetric, shard, profile, fp32_prim_rel=fp32_prim_rel)
        rep = _lib.JKReport()
        _lib.check(L.lai_jk_build(self._h, D.ctypes.data, n, J.ctypes.data, K.ctypes.data,
                                  ctypes.byref(opts), ctypes.byref(rep)))
        return J, K, rep

    def jk_spherical(self, D_sph, fp32_cut=0.0):
        """(J_sph, K_sph, report) for a density in the spherical basis: the Cartesian
        build on T^T D_sph T, then T J T^T and T K T^T."""
        Dc = self.basis.sph_to_cart_density(D_sph)
        J, K, rep = self.jk(Dc, fp32_cut=fp32_cut)
        return self.basis.cart_to_sph(J), self.basis.cart_to_sph(K), rep

    def jk_device(self, d_D, d_J, d_K, stream=0, fp32_cut=0.0, shard=(0, 1), profile=False, graph=False,
                  fp32_prim_rel=0.0):
        """Device-pointer variant (integers from torch.Tensor.data_ptr()).  graph=True
        captures the build as a CUDA graph on the first call and replays it after."""
        L = _lib.lib()
        opts = self._opts(fp32_cut, False, shard, profile, graph, fp32_prim_rel)
        rep = _lib.JKReport()
        _lib.check(L.lai_jk_build_device(self._h, ctypes.c_void_p(d_D), ctypes.c_void_p(d_J),
                                         ctypes.c_void_p(d_K), ctypes.c_void_p(stream),
                                         ctypes.byref(opts), ctypes.byref(rep)))
        return rep

    def last_profile(self):
        """Per-launch profile of the last build made with profile=True: dict of arrays
        ms, alg_flops (all nonzero primitives), alg_flops_executed (primitive
        quartets that passed the primitive cut), quartets, prim_quartets, lclass."""
        L = _lib.lib()
        n = L.lai_jk_last_profile(self._h, 0, None, None, None, None, None, None)
        out = {"ms": np.zeros(n), "alg_flops": np.zeros(n), "alg_flops_executed": np.zeros(n),
               "quartets": np.zeros(n, dtype=np.int64), "prim_quartets": np.zeros(n, dtype=np.int64),
               "lclass": np.zeros(4 * n, dtype=np.int32)}
        got = L.lai_jk_last_profile(self._h, n, *(out[k].ctypes.data for k in
                                                  ("ms", "alg_flops", "alg_flops_executed", "quartets",
                                                   "prim_quartets", "lclass")))
        if got < 0:
            _lib.check(got)
        out["lclass"] = out["lclass"].reshape(-1, 4)
        return out

    def quartet_count(self):
        return int(_lib.lib().lai_engine_quartet_count(self._h))

    def sample_quartets(self, n, seed=0):
        q = np.zeros((n, 4), dtype=np.int32)
        _lib.check(_lib.lib().lai_engine_sample_quartets(self._h, n, seed, q.ctypes.data))
        return q

    def compute_batch_screened(self, op=None):
        """All canonical screened quartets: (values, meta) with meta rows
        (offset, fa, fb, fc, fd, na, nb, nc, nd) -- the IntegralBuffer layout."""
        L = _lib.lib()
        nq = ctypes.c_int64()
        nv = ctypes.c_int64()
        _lib.check(L.lai_eri_batch_screened(self._h, None, 0, None, 0, ctypes.byref(nq), ctypes.byref(nv)))
        out = np.zeros(max(nv.value, 1))
        meta = (_lib.QuartetMeta * max(nq.value, 1))()
        _lib.check(L.lai_eri_batch_screened(self._h, out.ctypes.data, out.size, meta, nq.value,
                                            ctypes.byref(nq), ctypes.byref(nv)))
        m = np.array([(x.offset, x.fa, x.fb, x.fc, x.fd, x.na, x.nb, x.nc, x.nd)
                      for x in meta[:nq.value]], dtype=np.int64).reshape(-1, 9)
        return out[:nv.value], m

    def eri_quartets(self, quartets):
        """Raw integrals of listed shell quartets ([n][4] shell indices, any order):
        (values, meta) as compute_batch_screened, block t = [i][j][k][l]."""
        L = _lib.lib()
        q = np.ascontiguousarray(quartets, dtype=np.int32).reshape(-1, 4)
        n = len(q)
        if n and (q.min() < 0 or q.max() >= self.basis.n_shells):
            raise _lib.LibAccIntError(_lib.LAI_EINVAL, "quartet list: shell index out of range")
        nc = np.array([(s.l + 1) * (s.l + 2) // 2 for s in self.basis.shells])
        nv = int(np.sum(nc[q[:, 0]] * nc[q[:, 1]] * nc[q[:, 2]] * nc[q[:, 3]])) if n else 0
        out = np.zeros(max(nv, 1))
        meta = (_lib.QuartetMeta * max(n, 1))()
        _lib.check(L.lai_eri_quartets(self._h, q.ctypes.data, n, out.ctypes.data, out.size, meta))
        m = np.array([(x.offset, x.fa, x.fb, x.fc, x.fd, x.na, x.nb, x.nc, x.nd)
                      for x in meta[:n]], dtype=np.int64).reshape(-1, 9)
        return out[:nv], m

    def jk_accumulate_quartets(self, quartets, D, J, K, canonical_symmetry=True):
        """Adds the J/K contributions of listed quartets to J and K (host arrays,
        modified in place): plain accumulation of exactly those ordered quartets, or
        with canonical_symmetry each standing for its 8-fold orbit."""
        q = np.ascontiguousarray(quartets, dtype=np.int32).reshape(-1, 4)
        n = self.basis.nbf
        D = np.ascontiguousarray(D, dtype=np.float64)
        for M in (D, J, K):
            if M.shape != (n, n) or (M is not D and not M.flags.c_contiguous):
                raise ValueError(f"D, J, K must be contiguous {n}x{n} arrays")
        _lib.check(_lib.lib().lai_jk_accumulate_quartets(self._h, q.ctypes.data, len(q), D.ctypes.data,
                                                         J.ctypes.data, K.ctypes.data,
                                                         int(bool(canonical_symmetry))))

    def autotune(self, d_D, stream=0):
        """Times each class launch under a few launch configurations on the device
        density d_D and keeps the fastest; returns (ms_before, ms_after)."""
        a = ctypes.c_double()
        b = ctypes.c_double()
        _lib.check(_lib.lib().lai_engine_autotune(self._h, ctypes.c_void_p(d_D), ctypes.c_void_p(stream),
                                                  ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def tune_table(self):
        """Per class-pair block: la, lb, lc, ld, Kab, Kcd, quartets, ps, ksuper, quartets/1000."""
        L = _lib.lib()
        n = L.lai_engine_tune_table(self._h, 0, None)
        rows = np.zeros((max(n, 1), 10), dtype=np.int32)
        L.lai_engine_tune_table(self._h, n, rows.ctypes.data)
        return rows[:n]

    def natom(self):
        n = _lib.lib().lai_engine_natom(self._h)
        if n < 0:
            _lib.check(n)
        return n

    def gradient(self, D):
        """dE/dR [natom][3] of E = 1/2 tr(DJ) - 1/4 tr(DK) at fixed D."""
        n = self.basis.nbf
        D = np.ascontiguousarray(D, dtype=np.float64)
        if D.shape != (n, n):
            raise ValueError(f"density must be {n}x{n}")
        g = np.zeros((self.natom(), 3))
        _lib.check(_lib.lib().lai_jk_gradient(self._h, D.ctypes.data, n, g.ctypes.data))
        return g

    # --- one-electron integrals: Engine::compute_overlap_matrix / compute_kinetic_matrix /
    # compute_nuclear_matrix (include/libaccint/engine/engine.hpp:831-900; Python
    # bindings python/src/engine_bindings.cpp:146-200) ---
    def _charges(self, atoms):
        if atoms is None:
            atoms = self.basis.atoms
            if atoms is None:
                raise ValueError("nuclear attraction needs atoms (the basis was not built from atoms)")
        return point_charges(atoms)

    def _one_electron(self, op, atoms=None):
        n = self.basis.nbf
        out = np.empty((n, n))
        xyz = q = None
        nc = 0
        if op in (_lib.LAI_OP_NUCLEAR, _lib.LAI_OP_HCORE):
            xyz, q = self._charges(atoms)
            nc = len(q)
        _lib.check(_lib.lib().lai_one_electron(self._h, op, nc, None if xyz is None else xyz.ctypes.data,
                                                None if q is None else q.ctypes.data, out.ctypes.data))
        return out

    def compute_overlap_matrix(self):
        """S (nbf x nbf)."""
        return self._one_electron(_lib.LAI_OP_OVERLAP)

    def compute_kinetic_matrix(self):
        """T (nbf x nbf)."""
        return self._one_electron(_lib.LAI_OP_KINETIC)

    def compute_nuclear_matrix(self, atoms=None):
        """V (nbf x nbf) of the nuclei (list of Atom / (Z, xyz) pairs, or
        PointChargeParams-like); default: the atoms the basis was built on."""
        return self._one_electron(_lib.LAI_OP_NUCLEAR, atoms)

    def compute_core_hamiltonian(self, atoms=None):
        """H_core = T + V in one call."""
        return self._one_electron(_lib.LAI_OP_HCORE, atoms)

    def one_electron_device(self, op, d_out, atoms=None, stream=0):
        """op in {"overlap", "kinetic", "nuclear", "hcore"} into the device buffer
        d_out (nbf x nbf doubles), asynchronous on stream."""
        code = {"overlap": _lib.LAI_OP_OVERLAP, "kinetic": _lib.LAI_OP_KINETIC,
                "nuclear": _lib.LAI_OP_NUCLEAR, "hcore": _lib.LAI_OP_HCORE}[op]
        xyz = q = None
        nc = 0
        if code in (_lib.LAI_OP_NUCLEAR, _lib.LAI_OP_HCORE):
            xyz, q = self._charges(atoms)
            nc = len(q)
        _lib.check(_lib.lib().lai_one_electron_device(
            self._h, code, nc, None if xyz is None else xyz.ctypes.data,
            None if q is None else q.ctypes.data, ctypes.c_void_p(d_out), ctypes.c_void_p(stream)))

    def compute_and_consume(self, op, consumer, screening=None):
        if not op.is_two_electron():
            raise ValueError("compute_and_consume requires a two-electron operator")
        if isinstance(consumer, GpuFockBuilder):
            return self._consume_device(consumer, screening)
        if consumer.D is None:
            raise RuntimeError("FockBuilder::accumulate called without density matrix")
        if consumer.nbf != self.basis.nbf:
            raise ValueError("FockBuilder nbf does not match the basis")
        self._check_screening(screening)
        J, K, rep = self.jk(consumer.D)
        consumer.J += J
        consumer.K += K
        consumer.last_report = rep

    def compute(self, op, consumer):
        self.compute_and_consume(op, consumer)

    def _check_screening(self, screening):
        # the Schwarz cut is fixed when the engine is built (its pair lists depend on it)
        if screening is not None and screening.effective_threshold() != self.threshold:
            raise ValueError("screening threshold %g differs from the engine's %g; build an Engine "
                             "with threshold=%g" % (screening.effective_threshold(), self.threshold,
                                                    screening.effective_threshold()))

    def _consume_device(self, fb, screening):
        # device J/K of fb.d_D on torch's current stream of fb's device, added to
        # fb.d_J / fb.d_K (the builder accumulates until reset())
        torch = fb._torch
        if not fb.has_density:
            raise RuntimeError("GpuFockBuilder: density matrix not set")
        if fb.nbf() != self.basis.nbf:
            raise ValueError("GpuFockBuilder nbf does not match the basis")
        if fb.device.index != self.device:
            raise ValueError(f"GpuFockBuilder is on cuda:{fb.device.index}, the engine on cuda:{self.device}")
        self._check_screening(screening)
        J = torch.empty_like(fb.d_J)
        K = torch.empty_like(fb.d_K)
        stream = torch.cuda.current_stream(fb.device)
        fb.last_report = self.jk_device(fb.d_D.data_ptr(), J.data_ptr(), K.data_ptr(), stream=stream.cuda_stream)
        fb.d_J.add_(J)
        fb.d_K.add_(K)

    def close(self):
        if getattr(self, "_h", None) is not None:
            _lib.lib().lai_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchedEngine(Engine):
    """Many independent systems (a list of BasisSet) in one engine: every
    shell-quartet class of all systems runs as one persistent launch.  D, J and K
    are lists of per-system matrices on the host side, packed on the device
    (``layout()`` gives the element offsets)."""

    def __init__(self, bases, threshold=1e-12, device=0, prim_threshold=None):
        self.bases = list(bases)
        self.basis = None
        self.threshold = threshold
        L = _lib.lib()
        opts = _lib.EngineOpts()
        L.lai_engine_opts_default(ctypes.byref(opts))
        opts.schwarz_threshold = threshold
        opts.device = device
        if prim_threshold is not None:
            opts.prim_threshold = prim_threshold
        handles = (ctypes.c_void_p * len(self.bases))(*[b.handle() for b in self.bases])
        h = ctypes.c_void_p()
        _lib.check(L.lai_engine_create_batched(len(self.bases), handles, ctypes.byref(opts), ctypes.byref(h)))
        self._h = h

    def layout(self):
        n = len(self.bases)
        off = np.zeros(n + 1, dtype=np.int64)
        nbf = np.zeros(n, dtype=np.int32)
        _lib.check(_lib.lib().lai_engine_batch_layout(self._h, None, off.ctypes.data, nbf.ctypes.data))
        return off, nbf

    def pack(self, mats):
        off, nbf = self.layout()
        out = np.empty(int(off[-1]))
        for s, M in enumerate(mats):
            out[off[s]:off[s + 1]] = np.ascontiguousarray(M, dtype=np.float64).reshape(-1)
        return out

    def unpack(self, packed):
        off, nbf = self.layout()
        return [packed[off[s]:off[s + 1]].reshape(nbf[s], nbf[s]) for s in range(len(nbf))]

    def jk(self, Ds, fp32_cut=0.0, profile=False):
        """([J_s], [K_s], report) for the per-system densities Ds."""
        D = self.pack(Ds)
        J = np.empty_like(D)
        K = np.empty_like(D)
        opts = self._opts(fp32_cut, False, (0, 1), profile)
        rep = _lib.JKReport()
        _lib.check(_lib.lib().lai_jk_build_batched(self._h, D.ctypes.data, J.ctypes.data, K.ctypes.data,
                                                   ctypes.byref(opts), ctypes.byref(rep)))
        return self.unpack(J), self.unpack(K), rep


def probe_fp64_peak(device=0):
    """FP64 FMA throughput of the device (TFLOP/s) from a register-resident FMA loop."""
    v = ctypes.c_double()
    _lib.check(_lib.lib().lai_probe_fp64_peak(device, ctypes.byref(v)))
    return v.value


def jk(basis, D, threshold=1e-12, fp32_cut=0.0):
    """One-shot J/K for a basis and density."""
    e = Engine(basis, threshold)
    try:
        J, K, _ = e.jk(D, fp32_cut=fp32_cut)
    finally:
        e.close()
    return J, K
