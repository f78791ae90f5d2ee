"""The CUDA engine's DGT and its RNS kernels on DGT primes against outputs of
the reference's DGT evaluator itself.

The golden outputs of pdroalves/aoa's aoa-dgt that pin the oracle
(tests/test_oracle_reference_dgt.py) are compared here with this library's
kernels through the C ABI, on aoa-dgt's primes and roots: the single-kernel
and hierarchical forward / inverse DGT (planar Gaussian-integer limbs here,
the reference's interleaved layout there), the DGT product, ModUp, ModDown
and rescale, word for word."""
import json
import os

import numpy as np
import pytest

from oracle import dgt_roots, unfold
from tests.gpu_util import require_gpu
from tests.test_oracle_reference_dgt import configs, load
from tests.test_oracle_reference_outputs import splitmix_residues

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def dgt_table():
    with open(os.path.join(HERE, "golden", "dgt_roots.json")) as f:
        return json.load(f)


def _engine(aoa, dgt_table, nphi, k, primes):
    g, r = dgt_roots(dgt_table, primes, nphi // 2)
    E = aoa.Engine(nphi.bit_length() - 1, primes[:k], primes[k:], generators=g, dgt_roots=r)
    return E, aoa.Context(E)


def test_cuda_dgt_equals_reference(dgt_table):
    require_gpu()
    import aoa_b200 as aoa
    g = load()
    checked = 0
    for tag, nphi, k, kl, prec, primes in configs(g):
        E, ctx = _engine(aoa, dgt_table, nphi, k, primes)
        n, nr = nphi // 2, len(primes)
        x = splitmix_residues(1, primes, nphi)                   # coefficients = planar limbs
        d = ctx.upload(x)
        ctx.dgt_fwd(d, 1, 0, nr)
        assert np.array_equal(d.numpy(), unfold(g[tag + "_dgt_fwd_l0"].reshape(nr, n, 2))), tag
        y = splitmix_residues(2, primes, nphi).reshape(nr, n, 2)  # the reference's raw words
        d = ctx.upload(unfold(y))
        ctx.dgt_inv(d, 1, 0, nr)
        assert np.array_equal(d.numpy(), unfold(g[tag + "_dgt_inv_l0"].reshape(nr, n, 2))), tag
        checked += 1
    assert checked == 2


def test_cuda_product_and_rns_kernels_equal_reference(dgt_table):
    require_gpu()
    import aoa_b200 as aoa
    g = load()
    tag = "n1024"
    nphi, k, kl, prec = (int(v) for v in g[tag + "_params"])
    primes = [int(p) for p in g[tag + "_primes"]]
    E, ctx = _engine(aoa, dgt_table, nphi, k, primes)
    lib = aoa.capi.load()
    da = ctx.upload(splitmix_residues(3, primes[:k], nphi))
    db = ctx.upload(splitmix_residues(4, primes[:k], nphi))
    ctx.dgt_fwd(da, 1, 0, k)
    ctx.dgt_fwd(db, 1, 0, k)
    aoa.capi.check(lib.aoa_gi_mul(ctx.handle, da.ptr, da.ptr, db.ptr, 0, k))
    ctx.dgt_inv(da, 1, 0, k)
    assert np.array_equal(da.numpy(), g[tag + "_mul_l0"].reshape(k, nphi))
    for level in (k - 1, 1):
        x = splitmix_residues(10 + level, primes[:k], nphi)
        out = ctx.alloc((kl, nphi))
        aoa.capi.check(lib.aoa_modup(ctx.handle, ctx.upload(x).ptr, out.ptr, level))
        assert np.array_equal(out.numpy(), g["%s_modup_l%d" % (tag, level)].reshape(kl, nphi)), level
        x = splitmix_residues(20 + level, primes, nphi)
        out = ctx.alloc((k, nphi))
        aoa.capi.check(lib.aoa_moddown(ctx.handle, ctx.upload(x).ptr, out.ptr, level))
        assert np.array_equal(out.numpy()[: level + 1],
                              g["%s_moddown_l%d" % (tag, level)].reshape(level + 1, nphi)), level
        x = np.stack([splitmix_residues(30 + level, primes[:k], nphi),
                      splitmix_residues(40 + level, primes[:k], nphi)])
        d = ctx.upload(x)
        aoa.capi.check(lib.aoa_rescale_polys(ctx.handle, d.ptr, 2, k, level))
        assert np.array_equal(d.numpy()[:, :level], g["%s_rescale_l%d" % (tag, level)].reshape(2, level, nphi))
