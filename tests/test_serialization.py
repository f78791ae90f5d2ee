"""Ciphertext / key exchange: the reference's JSON text format (poly_export /
poly_import, aoa-ntt src/arithmetic/poly_t.cpp:426-473; cipher_export,
src/ckks/cipher_t.cpp:42-81; export_keys, src/ckks/ckkscontext.cpp:60-100)
and the binary wire format of the C ABI."""
import json

import numpy as np
import pytest

import oracle
from tests.ckks_inputs import make_keys, uniform_residues
from tests.gpu_util import require_gpu


def test_residue_text_format():
    from aoa_b200.serialization import residues_to_text, text_to_residues
    x = np.array([[0, 7, 2**63 + 5], [1, 2, 3]], dtype=np.uint64)
    t = residues_to_text(x)
    assert t == "0,7,%d,1,2,3," % (2**63 + 5)            # decimal, comma after every value, limb after limb
    assert np.array_equal(text_to_residues(t, 2, 3), x)
    assert np.array_equal(text_to_residues(t.rstrip(","), 2, 3), x)   # trailing comma optional
    assert np.array_equal(text_to_residues(" 0, 7," + t[4:], 2, 3), x)
    with pytest.raises(ValueError):
        text_to_residues(t, 2, 4)


def _setup(log_n=12, k=4, kl=3):
    import aoa_b200
    ps = oracle.gen_ntt_primes(60, 2 << log_n, k + kl)
    E = aoa_b200.Engine(log_n, ps[:k], ps[k:], scale_bits=40)
    return aoa_b200, E, aoa_b200.Context(E), oracle.Oracle(1 << log_n, ps[:k], ps[k:])


@pytest.mark.gpu
def test_wire_format_round_trip_and_rejections():
    require_gpu()
    aoa, E, ctx, o = _setup()
    from aoa_b200 import serialization as ser
    rng = np.random.default_rng(3)
    N, k = E.N, E.k
    c0, c1 = uniform_residues(rng, E.q_primes, N), uniform_residues(rng, E.q_primes, N)
    for dom in (aoa.AOA_COEF, aoa.AOA_NTT):
        ct = aoa.Ciphertext.from_residues(ctx, c0, c1, slots=64, scale=(1 << 40) + 3, domain=dom)
        ct.set(2, 64, (1 << 40) + 3, dom)
        data = ser.ct_to_bytes(ctx, ct)
        assert len(data) == 64 + 2 * 3 * N * 8 and data[:8] == b"AOACKKS1"
        back = ser.ct_from_bytes(ctx, data)
        assert (back.level, back.slots, back.scale, back.domain) == (2, 64, (1 << 40) + 3, dom)
        g = back.download(nlimbs=3, domain=dom)
        assert np.array_equal(g[0], c0[:3]) and np.array_equal(g[1], c1[:3])
    with pytest.raises(aoa.capi.AoaError):
        ser.ct_from_bytes(ctx, data[:-8])                 # truncated
    bad = bytearray(data)
    bad[0:8] = b"XXXXXXXX"
    with pytest.raises(aoa.capi.AoaError):
        ser.ct_from_bytes(ctx, bytes(bad))
    aoa2, E2, ctx2, _ = _setup(k=5, kl=2)                 # other prime set
    with pytest.raises(aoa.capi.AoaError):
        ser.ct_from_bytes(ctx2, data)
    # a residue >= its prime (last word of poly 1, limb 2), a slot count that
    # is not a power of two, one above N/2: each rejected with its reason
    body = np.frombuffer(data, dtype=np.uint64, offset=64).copy()
    body[-1] = E.q_primes[2]
    with pytest.raises(aoa.capi.AoaError) as ei:
        ser.ct_from_bytes(ctx, data[:64] + body.tobytes())
    assert "residue" in str(ei.value)
    for slots in (48, N):
        hdr = bytearray(data[:64])
        hdr[28:32] = int(slots).to_bytes(4, "little")     # slots field of the header
        with pytest.raises(aoa.capi.AoaError) as ei:
            ser.ct_from_bytes(ctx, bytes(hdr) + data[64:])
        assert "slot" in str(ei.value)
    # a key survives the trip and relinearises exactly as before
    keys = make_keys(o, seed=4)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    kdata = ser.key_to_bytes(ctx, evk)
    with pytest.raises(aoa.capi.AoaError):
        ser.ct_from_bytes(ctx, kdata)                     # a key is not a ciphertext
    evk2 = ser.key_from_bytes(ctx, kdata)
    a = aoa.Ciphertext.from_residues(ctx, c0, c1, slots=64, scale=1 << 40)
    b = aoa.Ciphertext.from_residues(ctx, c1, c0, slots=64, scale=1 << 40)
    outs = []
    for key in (evk, evk2):
        a.set(k - 1, 64, 1 << 40, a.domain)
        b.set(k - 1, 64, 1 << 40, b.domain)
        out = aoa.Ciphertext(ctx)
        aoa.ckks_mul(ctx, out, a, b, key)
        outs.append(out.download(nlimbs=k - 1))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


@pytest.mark.gpu
def test_reference_json_round_trip():
    require_gpu()
    aoa, E, ctx, o = _setup()
    from aoa_b200 import serialization as ser
    rng = np.random.default_rng(5)
    N, k = E.N, E.k
    c0, c1 = uniform_residues(rng, E.q_primes, N), uniform_residues(rng, E.q_primes, N)
    ct = aoa.Ciphertext.from_residues(ctx, c0, c1, slots=128, scale=1 << 40, domain=aoa.AOA_COEF)
    obj = json.loads(json.dumps(ser.cipher_export(ctx, ct)))
    assert set(obj) == {"ct", "props"} and set(obj["ct"]) == {"0", "1"}
    assert obj["props"] == {"level": k - 1, "scale": 1 << 40, "slots": 128}
    assert obj["ct"]["0"].endswith(",") and obj["ct"]["0"].count(",") == k * N
    assert obj["ct"]["0"].split(",")[N] == str(c0[1, 0])     # limb after limb
    back = ser.cipher_import(ctx, obj)
    g = back.download(nlimbs=k)
    assert np.array_equal(g[0], c0) and np.array_equal(g[1], c1)
    keys = make_keys(o, seed=6)
    pk = aoa.Ciphertext.from_residues(ctx, keys["pk"][0], keys["pk"][1], domain=aoa.AOA_NTT)
    evk = aoa.SwitchKey(ctx, *keys["evk"])
    kobj = json.loads(json.dumps(ser.export_keys(ctx, keys["s"], pk, evk)))
    assert set(kobj) == {"sk", "pk", "evk"} and set(kobj["evk"]) == {"a", "b"}
    sk2, pk2, evk2 = ser.load_keys(ctx, kobj)
    assert np.array_equal(sk2, keys["s"])
    b0, a0, _ = evk.numpy()
    b1, a1, _ = evk2.numpy()
    assert np.array_equal(b0, b1) and np.array_equal(a0, a1)
    g = pk2.download(nlimbs=k, domain=aoa.AOA_NTT)
    assert np.array_equal(g[0], keys["pk"][0]) and np.array_equal(g[1], keys["pk"][1])
