"""ctypes binding of libaoa_b200.so (include/aoa_ckks.h).

The library is the product: if it is missing or fails to load this module
raises, there is no fallback path.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libaoa_b200.so")

c_int, c_long, c_size_t, c_double = ctypes.c_int, ctypes.c_long, ctypes.c_size_t, ctypes.c_double
c_u64, c_i64, c_void_p, c_char_p = ctypes.c_uint64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_char_p
u64p = ctypes.POINTER(ctypes.c_uint64)
i64p = ctypes.POINTER(ctypes.c_int64)
f64p = ctypes.POINTER(ctypes.c_double)
intp = ctypes.POINTER(ctypes.c_int)
vpp = ctypes.POINTER(ctypes.c_void_p)

AOA_OK = 0
STATUS = {
    1: "AOA_ERR_BAD_PARAM", 2: "AOA_ERR_LEVEL_EXHAUSTED", 3: "AOA_ERR_NO_KEY", 4: "AOA_ERR_OOM",
    5: "AOA_ERR_CUDA", 6: "AOA_ERR_TIMEOUT", 7: "AOA_ERR_SLOT_MISMATCH", 8: "AOA_ERR_NOT_INITIALIZED",
    9: "AOA_ERR_NO_DEVICE",
}
AOA_COEF, AOA_NTT, AOA_DGT = 1, 2, 3


class AoaError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("%s: %s" % (STATUS.get(status, status), msg))
        self.status = status
        self.name = STATUS.get(status, str(status))


class Params(ctypes.Structure):
    _fields_ = [("log_n", c_int), ("k", c_int), ("kl", c_int), ("primes", u64p),
                ("generators", u64p), ("scale_bits", c_int), ("dnum", c_int), ("dgt_roots", u64p)]


# name -> (restype, argtypes); every function returns an aoa_status unless noted
SIGNATURES = {
    "aoa_last_error": (c_char_p, []),
    "aoa_status_string": (c_char_p, [c_int]),
    "aoa_kernel_launches": (c_long, []),
    "aoa_search_primes": (c_int, [c_int, c_u64, c_int, u64p]),
    "aoa_primitive_root": (c_u64, [c_u64]),
    "aoa_engine_create": (c_int, [ctypes.POINTER(Params), vpp]),
    "aoa_engine_destroy": (c_int, [c_void_p]),
    "aoa_engine_info": (c_int, [c_void_p, intp, intp, intp, u64p]),
    "aoa_ctx_create": (c_int, [c_void_p, c_void_p, vpp]),
    "aoa_ctx_destroy": (c_int, [c_void_p]),
    "aoa_ctx_sync": (c_int, [c_void_p]),
    "aoa_ctx_wait_check": (c_int, [c_void_p, c_int]),
    "aoa_ctx_stream": (c_int, [c_void_p, vpp]),
    "aoa_device_alloc": (c_int, [c_void_p, c_size_t, vpp]),
    "aoa_device_free": (c_int, [c_void_p, c_void_p]),
    "aoa_host_alloc": (c_int, [c_size_t, vpp]),
    "aoa_host_free": (c_int, [c_void_p]),
    "aoa_memcpy_h2d": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t]),
    "aoa_memcpy_d2h": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t]),
    "aoa_memcpy_d2d": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t]),
    "aoa_ntt_fwd": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int]),
    "aoa_ntt_inv": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int]),
    "aoa_modup": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "aoa_moddown": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "aoa_rescale_polys": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int]),
    "aoa_ct_create": (c_int, [c_void_p, vpp]),
    "aoa_ct_destroy": (c_int, [c_void_p, c_void_p]),
    "aoa_ct_set": (c_int, [c_void_p, c_int, c_int, c_u64, c_int]),
    "aoa_ct_get": (c_int, [c_void_p, intp, intp, u64p, intp]),
    "aoa_ct_data": (c_int, [c_void_p, vpp]),
    "aoa_ct_upload": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int]),
    "aoa_ct_download": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int]),
    "aoa_ct_download_async": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int]),
    "aoa_swk_create": (c_int, [c_void_p, c_void_p, c_void_p, c_int, vpp]),
    "aoa_swk_destroy": (c_int, [c_void_p, c_void_p]),
    "aoa_hmult": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "aoa_hmult_relin_rescale": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "aoa_hmult_plain": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "aoa_rotate_plain": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "aoa_conjugate_plain": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "aoa_hmult_relin_rescale_noalloc": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "aoa_hmult_batch": (c_int, [c_void_p, c_int, vpp, vpp, vpp, c_void_p, c_int]),
    "aoa_rescale": (c_int, [c_void_p, c_void_p]),
    "aoa_add": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "aoa_sub": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "aoa_rotate": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "aoa_rotate_batch": (c_int, [c_void_p, c_int, vpp, vpp, c_int, c_void_p]),
    "aoa_rotate_batch_steps": (c_int, [c_void_p, c_int, vpp, vpp, ctypes.POINTER(c_int), vpp]),
    "aoa_conjugate_batch": (c_int, [c_void_p, c_int, vpp, vpp, c_void_p]),
    "aoa_conjugate": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "aoa_encode": (c_int, [c_void_p, c_void_p, c_int, c_int, c_u64, c_int, c_int, c_void_p]),
    "aoa_decode": (c_int, [c_void_p, c_void_p, c_int, c_int, c_u64, c_void_p]),
    "aoa_encrypt": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_int,
                            c_u64]),
    "aoa_decrypt": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "aoa_dgt_fwd": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int]),
    "aoa_dgt_inv": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int]),
    "aoa_gi_mul": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int]),
    "aoa_gi_to_planar": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "aoa_gi_from_planar": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "aoa_engine_dgt_roots": (c_int, [c_void_p, c_void_p]),
    "aoa_ctx_set_transform": (c_int, [c_void_p, c_int]),
    "aoa_engine_tune": (c_int, [c_void_p, c_char_p, c_double]),
    "aoa_engine_tune_get": (c_int, [c_void_p, c_char_p, ctypes.POINTER(c_double)]),
    "aoa_engine_autotune": (c_int, [c_void_p, c_int, c_char_p, c_size_t]),
    "aoa_mul_plaintext": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_u64, c_int]),
    "aoa_mul_const": (c_int, [c_void_p, c_void_p, c_void_p, c_double, c_int]),
    "aoa_add_const": (c_int, [c_void_p, c_void_p, c_void_p, c_double]),
    "aoa_sumslots": (c_int, [c_void_p, c_void_p, c_void_p, vpp, c_int]),
    "aoa_power": (c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_uint64, c_void_p]),
    "aoa_sample_uniform": (c_int, [c_void_p, c_void_p, c_int, c_int, ctypes.c_uint64, ctypes.c_uint64]),
    "aoa_sample_gaussian": (c_int, [c_void_p, c_void_p, c_long, c_double, ctypes.c_uint64, ctypes.c_uint64]),
    "aoa_sample_ternary": (c_int, [c_void_p, c_void_p, c_long, c_long, ctypes.c_uint64, ctypes.c_uint64]),
    "aoa_signed_to_residues": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int]),
    "aoa_ct_wire_size": (c_size_t, [c_void_p, c_void_p]),
    "aoa_ct_serialize": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t, ctypes.POINTER(c_size_t)]),
    "aoa_ct_deserialize": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t]),
    "aoa_swk_wire_size": (c_size_t, [c_void_p]),
    "aoa_swk_serialize": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t, ctypes.POINTER(c_size_t)]),
    "aoa_swk_deserialize": (c_int, [c_void_p, c_void_p, c_size_t, vpp]),
    "aoa_eval_polynomial": (c_int, [c_void_p, c_void_p, c_void_p, ctypes.POINTER(c_double), c_int, c_void_p]),
    "aoa_inner_prod": (c_int, [c_void_p, c_void_p, vpp, vpp, c_int, c_void_p]),
    "aoa_inner_prod_const": (c_int, [c_void_p, c_void_p, vpp, ctypes.POINTER(c_double), c_int]),
    "aoa_ctx_capture_begin": (c_int, [c_void_p]),
    "aoa_ctx_capture_end": (c_int, [c_void_p, c_void_p]),
    "aoa_graph_launch": (c_int, [c_void_p, c_void_p]),
    "aoa_graph_nodes": (c_int, [c_void_p, c_void_p]),
    "aoa_graph_destroy": (c_int, [c_void_p]),
    "aoa_swk_data": (c_int, [c_void_p, c_void_p, c_void_p]),
    "aoa_swk_generate": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "aoa_pk_generate": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "aoa_secret_square": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "aoa_secret_galois": (c_int, [c_void_p, c_void_p, c_void_p, c_long, c_int]),
}

_lib = None


def load():
    """Load the CUDA library; raises if it is absent (build it with aoa_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libaoa_b200.so is not built (%s); run python -m aoa_b200.build" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    return list(SIGNATURES)


def check(status):
    if status != AOA_OK:
        msg = load().aoa_last_error().decode()
        raise AoaError(status, msg)


def ptr(a):
    """Host pointer of a C-contiguous numpy array."""
    assert a.flags["C_CONTIGUOUS"]
    return ctypes.c_void_p(a.ctypes.data)
