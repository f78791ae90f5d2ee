"""aoa_b200 — B200-native CKKS evaluation engine (host-side Python mirror).

The compute path is libaoa_b200.so (hand-written sm_100a CUDA behind the C ABI
in include/aoa_ckks.h).  This package wraps that ABI with the objects of the
reference's API (pdroalves/aoa aoa-ntt: CUDAManager/Context/poly_t/cipher_t
and the ckks_* free functions) for Python callers, tests and the benchmark.
"""
import ctypes

import numpy as np

from . import capi
from .capi import AoaError, AOA_COEF, AOA_NTT

__all__ = ["Engine", "Context", "DeviceArray", "AoaError", "AOA_COEF", "AOA_NTT"]


class Engine:
    """One parameter set (ring degree, Q primes, special primes).

    Replaces CUDAManager::init(k, kl, N, scalingfactor) (aoa-ntt
    src/cuda/manager.cu:762-800) with explicit prime lists.
    """

    def __init__(self, log_n, q_primes, b_primes, scale_bits=0, generators=None):
        lib = capi.load()
        self.log_n, self.N = log_n, 1 << log_n
        self.q_primes = [int(q) for q in q_primes]
        self.b_primes = [int(q) for q in b_primes]
        self.k, self.kl = len(self.q_primes), len(self.b_primes)
        self.primes = self.q_primes + self.b_primes
        self._primes_arr = np.array(self.primes, dtype=np.uint64)
        self._gens_arr = None if generators is None else np.array(generators, dtype=np.uint64)
        p = capi.Params()
        p.log_n, p.k, p.kl = log_n, self.k, self.kl
        p.primes = self._primes_arr.ctypes.data_as(capi.u64p)
        p.generators = None if self._gens_arr is None else self._gens_arr.ctypes.data_as(capi.u64p)
        p.scale_bits, p.dnum = scale_bits, 1
        self.scale_bits = scale_bits
        h = ctypes.c_void_p()
        capi.check(lib.aoa_engine_create(ctypes.byref(p), ctypes.byref(h)))
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            capi.load().aoa_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """A CUDA stream bound to an engine (reference Context, tool/context.h:16-49)."""

    def __init__(self, engine, stream=None):
        self.engine = engine
        h = ctypes.c_void_p()
        capi.check(capi.load().aoa_ctx_create(engine.handle, stream, ctypes.byref(h)))
        self.handle = h

    @property
    def stream(self):
        s = ctypes.c_void_p()
        capi.check(capi.load().aoa_ctx_stream(self.handle, ctypes.byref(s)))
        return s.value

    def sync(self):
        capi.check(capi.load().aoa_ctx_sync(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            capi.load().aoa_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- memory ------------------------------------------------------------
    def alloc(self, shape, dtype=np.uint64):
        return DeviceArray(self, shape, dtype)

    def upload(self, host):
        host = np.ascontiguousarray(host)
        d = DeviceArray(self, host.shape, host.dtype)
        d.copy_from(host)
        return d

    # -- transforms ------------------------------------------------------------
    def ntt_fwd(self, d, npolys, first_prime, nlimbs, poly_stride=None):
        capi.check(capi.load().aoa_ntt_fwd(self.handle, d.ptr, npolys, first_prime, nlimbs,
                                           poly_stride or nlimbs))

    def ntt_inv(self, d, npolys, first_prime, nlimbs, poly_stride=None):
        capi.check(capi.load().aoa_ntt_inv(self.handle, d.ptr, npolys, first_prime, nlimbs,
                                           poly_stride or nlimbs))


class DeviceArray:
    """Device allocation on a context's stream (stream-ordered malloc/free)."""

    def __init__(self, ctx, shape, dtype=np.uint64):
        self.ctx, self.shape, self.dtype = ctx, tuple(np.atleast_1d(shape)), np.dtype(dtype)
        self.nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        h = ctypes.c_void_p()
        capi.check(capi.load().aoa_device_alloc(ctx.handle, max(self.nbytes, 8), ctypes.byref(h)))
        self.ptr = h

    def copy_from(self, host):
        host = np.ascontiguousarray(host, dtype=self.dtype)
        assert host.nbytes == self.nbytes
        capi.check(capi.load().aoa_memcpy_h2d(self.ctx.handle, self.ptr, capi.ptr(host), self.nbytes))
        self.ctx.sync()

    def numpy(self):
        out = np.empty(self.shape, dtype=self.dtype)
        capi.check(capi.load().aoa_memcpy_d2h(self.ctx.handle, capi.ptr(out), self.ptr, self.nbytes))
        self.ctx.sync()
        return out

    def offset(self, elements):
        return ctypes.c_void_p(self.ptr.value + elements * self.dtype.itemsize)

    def free(self):
        if getattr(self, "ptr", None) is not None and self.ctx.handle:
            capi.load().aoa_device_free(self.ctx.handle, self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
