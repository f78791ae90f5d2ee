"""Device samplers (Sampler, aoa-ntt src/cuda/sampler.cu) on Philox4x32-10:
bit-exact with the host restatement for the integer outputs, distribution
checks for the Gaussian, and a chain (keys + encryption from the samplers)
that decrypts."""
import numpy as np
import pytest

import oracle
from tests import philox_ref
from tests.gpu_util import require_gpu


def test_philox_known_answer():
    # Philox4x32-10 known-answer vectors of the Random123 distribution (counter, key -> output)
    x = philox_ref.philox(np.array([0], np.uint64), 0, 0)
    assert [int(v[0]) for v in x] == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    ctr = (0xFFFFFFFF << 32) | 0xFFFFFFFF
    x = philox_ref.philox(np.array([ctr], np.uint64), ctr, (0xFFFFFFFF << 32) | 0xFFFFFFFF)
    assert [int(v[0]) for v in x] == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]


def _setup(log_n=12):
    import aoa_b200
    ps = oracle.gen_ntt_primes(60, 2 << log_n, 7)
    # 4 special primes (B > Q); scale 2^50 keeps 2^40 after one rescale by a 60-bit prime
    E = aoa_b200.Engine(log_n, ps[:3], ps[3:], scale_bits=50)
    return aoa_b200, E, aoa_b200.Context(E)


@pytest.mark.gpu
def test_samplers_match_host_restatement():
    require_gpu()
    aoa, E, ctx = _setup()
    N = E.N
    u = aoa.sample_uniform(ctx, 1, 3, seed=2, stream=7).numpy()
    assert np.array_equal(u, philox_ref.uniform(E.primes[1:4], N, 2, 7))
    for hw in (64, N // 2, 0, N):
        t = aoa.sample_ternary(ctx, N, hw, seed=3, stream=hw).numpy()
        assert np.array_equal(t, philox_ref.ternary(N, hw, 3, hw)), hw
        assert np.count_nonzero(t) == hw and set(np.unique(t)) <= {-1, 0, 1}
    g = aoa.sample_gaussian(ctx, 1 << 16, seed=4, stream=1).numpy()
    want = philox_ref.gaussian(1 << 16, 4, 1)
    diff = g - want
    assert np.count_nonzero(diff) <= 8 and np.all(np.abs(diff) <= 1)   # last-ulp math differences only
    assert abs(g.mean()) < 0.05 and abs(g.std() - 3.2) < 0.05
    g2 = aoa.sample_gaussian(ctx, 1 << 16, seed=4, stream=1).numpy()
    assert np.array_equal(g, g2)                                       # reproducible
    assert not np.array_equal(g, aoa.sample_gaussian(ctx, 1 << 16, seed=4, stream=2).numpy())


@pytest.mark.gpu
def test_sampled_keys_and_encryption_decrypt():
    require_gpu()
    aoa, E, ctx = _setup(log_n=13)
    s, keys = aoa.ckks_keygen_sampled(ctx, seed=2)
    rng = np.random.default_rng(1)
    slots = E.N // 2
    va = rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots)
    vb = rng.uniform(-1, 1, slots) + 1j * rng.uniform(-1, 1, slots)
    ca = aoa.ckks_encrypt_sampled(ctx, va, keys["pk"], seed=3, stream=0)
    cb = aoa.ckks_encrypt_sampled(ctx, vb, keys["pk"], seed=3, stream=3)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_mul(ctx, out, ca, cb, keys["evk"])
    sk = ctx.alloc((E.k, E.N))
    aoa.capi.check(aoa.capi.load().aoa_memcpy_d2d(ctx.handle, sk.ptr, s.ptr, E.k * E.N * 8))
    dec = aoa.ckks_decrypt(ctx, out, sk)
    assert np.max(np.abs(dec - va * vb)) < 1e-5
