"""The CUDA path against outputs of the reference evaluator itself.

The same golden outputs of pdroalves/aoa's own aoa-ntt kernels that pin the
oracle (tests/test_oracle_reference_outputs.py) are compared here with this
library's kernels, through the C ABI, on the reference's primes: forward and
inverse transforms, ModUp, ModDown and rescale, word for word."""
import numpy as np
import pytest

from tests.gpu_util import require_gpu
from tests.test_oracle_reference_outputs import _configs, _load, splitmix_residues

pytestmark = pytest.mark.gpu


def test_cuda_kernels_equal_reference_outputs():
    require_gpu()
    import aoa_b200 as aoa
    g = _load()
    lib = aoa.capi.load()
    checked = 0
    for tag, N, k, kl, prec, primes in _configs(g):
        E = aoa.Engine(N.bit_length() - 1, primes[:k], primes[k:])
        ctx = aoa.Context(E)
        for which, seed, fwd, mx in (("fwd", 1, True, False), ("fwd_max", 1, True, True), ("inv", 2, False, False)):
            x = splitmix_residues(seed, primes, N, max_=mx)
            d = ctx.upload(x)
            (ctx.ntt_fwd if fwd else ctx.ntt_inv)(d, 1, 0, k + kl)
            assert np.array_equal(d.numpy(), g["%s_ntt_%s_l0" % (tag, which)].reshape(k + kl, N)), (tag, which)
            checked += 1
        for key in g.files:
            if not key.startswith(tag + "_") or "ntt" in key or key.endswith(("_params", "_primes")):
                continue
            name, level = key[len(tag) + 1:].rsplit("_l", 1)
            level = int(level)
            want = g[key]
            if name in ("modup", "modup_max"):
                x = splitmix_residues(2 + 1000 * level, primes[:k], N, max_=name == "modup_max")
                out = ctx.alloc((kl, N))
                aoa.capi.check(lib.aoa_modup(ctx.handle, ctx.upload(x).ptr, out.ptr, level))
                assert np.array_equal(out.numpy(), want.reshape(kl, N)), key
            elif name == "moddown":
                x = splitmix_residues(3 + 1000 * level, primes, N)
                out = ctx.alloc((k, N))
                aoa.capi.check(lib.aoa_moddown(ctx.handle, ctx.upload(x).ptr, out.ptr, level))
                assert np.array_equal(out.numpy()[: level + 1], want.reshape(level + 1, N)), key
            elif name == "rescale":
                x = np.stack([splitmix_residues(4 + 1000 * level, primes[:k], N),
                              splitmix_residues(5 + 1000 * level, primes[:k], N)])
                d = ctx.upload(x)
                aoa.capi.check(lib.aoa_rescale_polys(ctx.handle, d.ptr, 2, k, level))
                got = d.numpy()[:, :level]
                assert np.array_equal(got, want.reshape(2, level, N)), key
            checked += 1
    assert checked >= 14
