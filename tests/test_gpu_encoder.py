"""GPU parity of encode / decode / encrypt / decrypt against the CPU oracle.

Encode residues and decrypt residues must be bit-exact; decoded doubles must be
the oracle's doubles bit for bit (the device FFT rounds every product and sum
separately, in the reference's order, on the same table of roots)."""
import numpy as np
import pytest

import oracle
from oracle import Oracle, ST_COEF, ST_NTT
from tests.ckks_inputs import make_keys, encryption_noise, signed_to_residues, uniform_residues
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


def _setup(log_n, nq=3, nb=2, bits=55, scale_bits=40):
    import aoa_b200
    ps = oracle.gen_ntt_primes(bits, 2 << log_n, nq + nb)
    Q, B = ps[:nq], ps[nq:]
    E = aoa_b200.Engine(log_n, Q, B, scale_bits=scale_bits)
    ctx = aoa_b200.Context(E)
    return aoa_b200, E, ctx, Oracle(1 << log_n, Q, B)


def _values(rng, n):
    return rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)


def _same_doubles(a, b):
    a = np.ascontiguousarray(a, dtype=np.complex128).view(np.uint64)
    b = np.ascontiguousarray(b, dtype=np.complex128).view(np.uint64)
    return np.array_equal(a, b)


@pytest.mark.parametrize("filled,empty", [(1, 0), (3, 1), (8, 0), (100, 28), (2048, 0), (1000, 1048)])
def test_encode_bit_exact(filled, empty):
    require_gpu()
    aoa, E, ctx, o = _setup(12)
    rng = np.random.default_rng(filled * 7 + empty)
    vals = _values(rng, filled)
    scale = 1 << 40
    want = o.encode(vals, scale, empty=empty)
    got, sc = aoa.ckks_encode(ctx, vals, empty_slots=empty, scale=scale)
    assert sc == scale
    assert np.array_equal(got.numpy(), want)
    got_ntt, _ = aoa.ckks_encode(ctx, vals, empty_slots=empty, scale=scale, domain=aoa.AOA_NTT)
    assert np.array_equal(got_ntt.numpy(), o.ntt_fwd(want))


@pytest.mark.parametrize("slots", [1, 2, 16, 2048])
def test_decode_bit_exact(slots):
    require_gpu()
    aoa, E, ctx, o = _setup(12)
    rng = np.random.default_rng(slots)
    scale = 1 << 40
    # an encoded message and uniform residues (both branches of the centring)
    m = o.encode(_values(rng, slots), scale)
    for msg in (m, uniform_residues(rng, o.primes[:o.k], o.N)):
        want = o.decode(msg[0], slots, scale)
        d = ctx.upload(msg)
        assert _same_doubles(aoa.ckks_decode(ctx, d, slots, scale), want)
        dn = ctx.upload(o.ntt_fwd(msg))
        assert _same_doubles(aoa.ckks_decode(ctx, dn, slots, scale, domain=aoa.AOA_NTT), want)


def test_encode_decode_full_size():
    """N = 2^16, 32768 slots: the FFT stages too wide for one CTA run as
    whole-vector launches."""
    require_gpu()
    aoa, E, ctx, o = _setup(16, nq=2, nb=1, bits=60, scale_bits=50)
    rng = np.random.default_rng(16)
    vals = _values(rng, E.N // 2)
    scale = 1 << 50
    want = o.encode(vals, scale)
    got, _ = aoa.ckks_encode(ctx, vals, scale=scale)
    assert np.array_equal(got.numpy(), want)
    dec = aoa.ckks_decode(ctx, got, E.N // 2, scale)
    assert _same_doubles(dec, o.decode(want[0], E.N // 2, scale))
    assert np.max(np.abs(dec - vals)) < 1e-9


def test_encrypt_decrypt_bit_exact():
    require_gpu()
    aoa, E, ctx, o = _setup(12, nq=4, nb=3)
    keys = make_keys(o, seed=5)
    rng = np.random.default_rng(9)
    slots = E.N // 2
    vals = _values(rng, slots)
    scale = 1 << 40
    u, e1, e2 = encryption_noise(o, seed=11)
    m = o.encode(vals, scale)
    w0, w1 = o.encrypt(m, signed_to_residues(u, o.primes[:o.k]), e1, e2, keys["pk"], pk_state=ST_NTT)
    pk = aoa.Ciphertext.from_residues(ctx, keys["pk"][0], keys["pk"][1], domain=aoa.AOA_NTT)
    ct = aoa.ckks_encrypt(ctx, vals, pk, u, e1, e2, scale=scale)
    assert (ct.level, ct.slots, ct.scale, ct.domain) == (E.k - 1, slots, scale, aoa.AOA_NTT)
    g0, g1 = ct.download(domain=aoa.AOA_NTT)
    assert np.array_equal(g0, w0) and np.array_equal(g1, w1)
    sk = ctx.upload(keys["s"][:E.k])
    m_got = aoa.ckks_decrypt_poly(ctx, ct, sk).numpy()
    assert np.array_equal(m_got, o.decrypt((w0, w1), keys["s"][:E.k], state=ST_NTT))
    dec = aoa.ckks_decrypt(ctx, ct, sk)
    assert _same_doubles(dec, o.decode(m_got[0], slots, scale))
    assert np.max(np.abs(dec - vals)) < 1e-5
    # secret given in the transform domain, ciphertext given in coefficients
    ct2 = aoa.Ciphertext.from_residues(ctx, o.ntt_inv(w0), o.ntt_inv(w1), slots=slots, scale=scale)
    sk_ntt = ctx.upload(o.ntt_fwd(keys["s"][:E.k]))
    assert np.array_equal(aoa.ckks_decrypt_poly(ctx, ct2, sk_ntt, sk_domain=aoa.AOA_NTT).numpy(), m_got)


def test_encrypt_multiply_decrypt_chain():
    """encode -> encrypt -> HMult + rescale -> decrypt -> decode, each stage on
    the GPU, equals the oracle's chain bit for bit."""
    require_gpu()
    aoa, E, ctx, o = _setup(12, nq=4, nb=3)
    keys = make_keys(o, seed=6)
    rng = np.random.default_rng(10)
    slots = 64
    va, vb = _values(rng, slots), _values(rng, slots)
    scale = 1 << 40
    pk = aoa.Ciphertext.from_residues(ctx, keys["pk"][0], keys["pk"][1], domain=aoa.AOA_NTT)
    evk = aoa.SwitchKey(ctx, keys["evk"][0], keys["evk"][1], domain=aoa.AOA_NTT)
    na, nb = encryption_noise(o, seed=12), encryption_noise(o, seed=13)
    ca = aoa.ckks_encrypt(ctx, va, pk, *na, scale=scale)
    cb = aoa.ckks_encrypt(ctx, vb, pk, *nb, scale=scale)
    out = aoa.Ciphertext(ctx)
    aoa.ckks_mul(ctx, out, ca, cb, evk)
    sk = ctx.upload(keys["s"][:E.k])
    dec = aoa.ckks_decrypt(ctx, out, sk)

    def oenc(v, n):
        m = o.encode(v, scale)
        return o.encrypt(m, signed_to_residues(n[0], o.primes[:o.k]), n[1], n[2], keys["pk"], pk_state=ST_NTT)
    ea, eb = oenc(va, na), oenc(vb, nb)
    r0, r1, rscale = o.hmult(ea, eb, keys["evk"], E.k - 1, scale, scale, rescale=True, a_state=ST_NTT,
                             b_state=ST_NTT)
    assert out.scale == rscale
    m = o.decrypt((r0, r1), keys["s"][:E.k], state=ST_COEF)
    want = o.decode(m[0], slots, rscale)
    assert _same_doubles(dec, want)
    assert np.max(np.abs(dec - va * vb)) < 1e-3


def test_encoder_rejects_bad_arguments():
    require_gpu()
    aoa, E, ctx, o = _setup(10)
    with pytest.raises(aoa.AoaError) as ei:
        aoa.ckks_encode(ctx, np.ones(3), empty_slots=0)
    assert ei.value.status == 1
    with pytest.raises(aoa.AoaError):
        aoa.ckks_encode(ctx, np.ones(E.N), empty_slots=0)
    d = ctx.alloc((E.k, E.N))
    with pytest.raises(aoa.AoaError):
        aoa.ckks_decode(ctx, d, 6, 1 << 40)
