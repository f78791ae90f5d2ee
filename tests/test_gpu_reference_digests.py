"""The CUDA engine at the headline shape against the reference itself.

The digests of pdroalves/aoa's own ckks_mul and rotation at N = 2^16, 30 Q +
31 special primes (its 55-bit set, 63-bit q0; tests/test_oracle_reference_digests.py)
are compared with this engine's per-call and batched HMult + relinearise +
rescale and its per-call and batched rotation of the same seeded operands,
through the C ABI (63-bit q0 limbs on strict butterflies, the others lazy),
on an NTT context and on a DGT context (aoa-dgt's digests are the same)."""
import numpy as np
import pytest

from tests.gpu_util import require_gpu
from tests.test_oracle_reference_ckks import SCALE_A, SCALE_B, seeded_ct, seeded_key
from tests.test_oracle_reference_digests import digests, load

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", ["aoa-ntt", "aoa-dgt"])
def test_engine_digests_equal_reference(variant):
    require_gpu()
    import aoa_b200 as aoa
    d = load(variant)
    N, k = d["N"], d["k"]
    primes = d["primes"]
    E = aoa.Engine(16, primes[:k], primes[k:], scale_bits=55)
    ctx = aoa.Context(E)
    dgt = variant == "aoa-dgt"
    if dgt:                                     # roots derived from the primes' generators
        ctx.set_transform(aoa.AOA_DGT)
    evk = aoa.SwitchKey(ctx, *seeded_key(111, 112, primes, N), domain=aoa.AOA_COEF)
    rtk = aoa.SwitchKey(ctx, *seeded_key(123, 124, primes, N), domain=aoa.AOA_COEF)
    a_in, b_in, c_in = (seeded_ct(101, 102, primes[:k], N), seeded_ct(103, 104, primes[:k], N),
                        seeded_ct(105, 106, primes[:k], N))

    def ct(x, scale):
        return aoa.Ciphertext.from_residues(ctx, x[0], x[1], level=k - 1, slots=N // 2, scale=scale)

    out = aoa.Ciphertext(ctx)
    aoa.ckks_mul(ctx, out, ct(a_in, SCALE_A), ct(b_in, SCALE_B), evk)
    outs = [aoa.Ciphertext(ctx) for _ in range(2)]
    aoa.ckks_mul_batch(ctx, outs, [ct(a_in, SCALE_A), ct(a_in, SCALE_A)], [ct(b_in, SCALE_B), ct(b_in, SCALE_B)], evk)
    for o in [out] + outs:
        assert o.level == d["hmult"]["level"] and o.scale == d["hmult"]["scale"]
        g0, g1 = o.download(nlimbs=k - 1)
        assert digests(g0, g1, k - 1) == d["hmult"]["digests"]
    r = aoa.Ciphertext(ctx)
    aoa.ckks_rotate_left(ctx, r, ct(c_in, SCALE_A), 1, rtk)
    rs = []
    if not dgt:                                 # batched rotations run on NTT contexts
        rs = [aoa.Ciphertext(ctx) for _ in range(2)]
        aoa.ckks_rotate_batch(ctx, rs, [ct(c_in, SCALE_A), ct(c_in, SCALE_A)], 1, rtk)
    for o in [r] + rs:
        assert o.level == d["rotate1"]["level"] and o.scale == d["rotate1"]["scale"]
        g0, g1 = o.download(nlimbs=k)
        assert digests(g0, g1, k) == d["rotate1"]["digests"]
