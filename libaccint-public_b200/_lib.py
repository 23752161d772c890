"""ctypes binding of the C ABI declared in include/libaccint_b200.h.

The library is the in-tree ``libaccint_b200.so`` built by ``build.py``.  There is
no fallback: if the library is missing or a CUDA device is absent, calls fail
loudly with ``LibAccIntError``.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaccint_b200.so")

LAI_OK, LAI_EINVAL, LAI_ENOMEM, LAI_ECUDA, LAI_ETIMEOUT, LAI_ESTATE, LAI_ENOTSUP = 0, -1, -2, -3, -4, -5, -6
LAI_BASIS_PRENORMALIZED = 1

# Every symbol include/libaccint_b200.h declares (checked by the CPU test suite).
EXPORTED = [
    "lai_last_error", "lai_abi_version",
    "lai_basis_create", "lai_basis_destroy", "lai_basis_nbf", "lai_basis_nshell", "lai_basis_shell",
    "lai_engine_opts_default", "lai_engine_create", "lai_engine_destroy", "lai_engine_schwarz",
    "lai_jk_opts_default", "lai_jk_build", "lai_jk_build_device", "lai_eri_batch_screened",
    "lai_jk_last_profile", "lai_engine_sample_quartets", "lai_engine_quartet_count",
    "lai_probe_fp64_peak", "lai_jk_build_noalloc",
    "lai_cart_to_sph_matrix", "lai_basis_nbf_spherical", "lai_cart_to_sph_2d", "lai_sph_to_cart_density",
    "lai_cart_to_sph_2d_device", "lai_sph_to_cart_density_device",
    "lai_eri_quartets", "lai_jk_accumulate_quartets", "lai_jk_accumulate_quartets_device",
    "lai_jk_accumulate_eri_batch_device",
    "lai_engine_natom", "lai_jk_gradient", "lai_jk_gradient_device",
    "lai_engine_create_batched", "lai_engine_batch_layout", "lai_jk_build_batched",
    "lai_engine_autotune", "lai_shard_range", "lai_engine_tune_table",
    "lai_one_electron", "lai_one_electron_device", "lai_basis_from_bse_json",
    "lai_eri3c", "lai_eri2c", "lai_eri3c_device", "lai_eri2c_device",
]

LAI_OP_OVERLAP, LAI_OP_KINETIC, LAI_OP_NUCLEAR, LAI_OP_HCORE = 0, 1, 2, 3


class LibAccIntError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libaccint_b200 error {code}: {msg}")
        self.code = code


class EngineOpts(ctypes.Structure):
    _fields_ = [("schwarz_threshold", ctypes.c_double), ("device", ctypes.c_int),
                ("prim_threshold", ctypes.c_double)]


class JKOpts(ctypes.Structure):
    _fields_ = [("fp32_cut", ctypes.c_double), ("check_symmetric", ctypes.c_int),
                ("shard_index", ctypes.c_int), ("shard_count", ctypes.c_int), ("profile", ctypes.c_int),
                ("graph", ctypes.c_int), ("fp32_prim_rel", ctypes.c_double)]


class QuartetMeta(ctypes.Structure):
    _fields_ = [("offset", ctypes.c_int64), ("fa", ctypes.c_int32), ("fb", ctypes.c_int32),
                ("fc", ctypes.c_int32), ("fd", ctypes.c_int32), ("na", ctypes.c_int32),
                ("nb", ctypes.c_int32), ("nc", ctypes.c_int32), ("nd", ctypes.c_int32)]


class JKReport(ctypes.Structure):
    _fields_ = [("quartets_fp64", ctypes.c_int64), ("quartets_fp32", ctypes.c_int64),
                ("alg_flops", ctypes.c_double), ("seconds_device", ctypes.c_double),
                ("seconds_total", ctypes.c_double), ("kernel_launches", ctypes.c_int),
                ("fp32_schwarz_cut", ctypes.c_double)]


_lib = None


def lib():
    """Load the shared library once (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise LibAccIntError(LAI_ENOTSUP, f"{LIB_PATH} not built (run build.py)")
    L = ctypes.CDLL(LIB_PATH)
    P, I, D, V, L64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, None, ctypes.c_long
    sig = {
        "lai_last_error": (ctypes.c_char_p, []),
        "lai_abi_version": (I, []),
        "lai_basis_create": (I, [I, P, P, P, P, P, P, I, ctypes.POINTER(P)]),
        "lai_basis_destroy": (V, [P]),
        "lai_basis_nbf": (L64, [P]),
        "lai_basis_nshell": (I, [P]),
        "lai_basis_shell": (I, [P, I, P, P, P, P, P, P]),
        "lai_engine_opts_default": (V, [ctypes.POINTER(EngineOpts)]),
        "lai_engine_create": (I, [P, ctypes.POINTER(EngineOpts), ctypes.POINTER(P)]),
        "lai_engine_destroy": (V, [P]),
        "lai_engine_schwarz": (I, [P, P]),
        "lai_jk_opts_default": (V, [ctypes.POINTER(JKOpts)]),
        "lai_jk_build": (I, [P, P, ctypes.c_size_t, P, P, ctypes.POINTER(JKOpts), ctypes.POINTER(JKReport)]),
        "lai_jk_build_device": (I, [P, P, P, P, P, ctypes.POINTER(JKOpts), ctypes.POINTER(JKReport)]),
        "lai_eri_batch_screened": (I, [P, P, ctypes.c_size_t, P, ctypes.c_size_t,
                                       ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
        "lai_jk_last_profile": (I, [P, I, P, P, P, P, P, P]),
        "lai_engine_sample_quartets": (I, [P, ctypes.c_int64, ctypes.c_uint64, P]),
        "lai_engine_quartet_count": (ctypes.c_int64, [P]),
        "lai_probe_fp64_peak": (I, [I, ctypes.POINTER(ctypes.c_double)]),
        "lai_jk_build_noalloc": (I, [P, P, P, P, P]),
        "lai_cart_to_sph_matrix": (I, [I, P]),
        "lai_basis_nbf_spherical": (L64, [P]),
        "lai_cart_to_sph_2d": (I, [P, P, P]),
        "lai_sph_to_cart_density": (I, [P, P, P]),
        "lai_cart_to_sph_2d_device": (I, [P, P, P, P]),
        "lai_sph_to_cart_density_device": (I, [P, P, P, P]),
        "lai_eri_quartets": (I, [P, P, ctypes.c_int64, P, ctypes.c_size_t, P]),
        "lai_jk_accumulate_quartets": (I, [P, P, ctypes.c_int64, P, P, P, I]),
        "lai_jk_accumulate_quartets_device": (I, [P, P, ctypes.c_int64, P, P, P, P, I]),
        "lai_jk_accumulate_eri_batch_device": (I, [P, P, P, ctypes.c_int64, P, P, P, P]),
        "lai_engine_natom": (I, [P]),
        "lai_jk_gradient": (I, [P, P, ctypes.c_size_t, P]),
        "lai_jk_gradient_device": (I, [P, P, P, P]),
        "lai_engine_create_batched": (I, [I, P, ctypes.POINTER(EngineOpts), ctypes.POINTER(P)]),
        "lai_engine_batch_layout": (I, [P, P, P, P]),
        "lai_jk_build_batched": (I, [P, P, P, P, ctypes.POINTER(JKOpts), ctypes.POINTER(JKReport)]),
        "lai_engine_autotune": (I, [P, P, P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
        "lai_shard_range": (I, [ctypes.c_int64, I, I, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
        "lai_engine_tune_table": (I, [P, I, P]),
        "lai_one_electron": (I, [P, I, I, P, P, P]),
        "lai_one_electron_device": (I, [P, I, I, P, P, P, P]),
        "lai_basis_from_bse_json": (I, [ctypes.c_char_p, ctypes.c_size_t, I, P, P, ctypes.POINTER(P)]),
        "lai_eri3c": (I, [P, P, P]),
        "lai_eri2c": (I, [P, P, P]),
        "lai_eri3c_device": (I, [P, P, P, P]),
        "lai_eri2c_device": (I, [P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(rc):
    if rc != LAI_OK:
        raise LibAccIntError(rc, lib().lai_last_error().decode())
    return rc
