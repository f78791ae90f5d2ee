"""Ciphertext and key exchange formats.

JSON, the reference's format (cipher_export / cipher_import, aoa-ntt
src/ckks/cipher_t.cpp:42-81; CKKSContext::export_keys / load_keys,
src/ckks/ckkscontext.cpp:50-100; poly_export / poly_import,
src/arithmetic/poly_t.cpp:426-473): every residue of a poly in coefficients
as decimal text, each followed by a comma, limb after limb; a ciphertext is
{"ct": {"0": c0, "1": c1}, "props": {"level", "scale", "slots"}}, the keys
{"sk": {"s"}, "pk": {"a", "b"}, "evk": {"a", "b"}}.

Binary, for serving payloads: the C ABI's wire format (aoa_ct_serialize,
aoa_swk_serialize), a 64-byte header and the residues as u64.
"""
import ctypes

import numpy as np

from . import AOA_COEF, AOA_NTT, Ciphertext, SwitchKey, capi


# ---- JSON (reference format) ----------------------------------------------------

def residues_to_text(x):
    """[limbs][N] residues -> "r,r,...,r," (poly_residue_to_string)."""
    flat = np.ascontiguousarray(x, dtype=np.uint64).ravel()
    return "".join(v + "," for v in flat.astype(str))


def text_to_residues(s, nlimbs, n):
    """Inverse of residues_to_text (poly_import); spaces are ignored, the
    trailing comma is optional.  The value count must be nlimbs * n."""
    parts = [p for p in s.replace(" ", "").split(",") if p != ""]
    if len(parts) != nlimbs * n:
        raise ValueError("expected %d residues, found %d" % (nlimbs * n, len(parts)))
    return np.array([int(p) for p in parts], dtype=np.uint64).reshape(nlimbs, n)


def cipher_export(ctx, ct):
    """The reference's JSON object for a ciphertext (all k limbs, coefficients)."""
    E = ctx.engine
    c0, c1 = ct.download(nlimbs=E.k, domain=AOA_COEF)
    return {"ct": {"0": residues_to_text(c0), "1": residues_to_text(c1)},
            "props": {"level": int(ct.level), "scale": int(ct.scale), "slots": int(ct.slots)}}


def cipher_import(ctx, obj):
    """A ciphertext from the reference's JSON object."""
    E = ctx.engine
    c0 = text_to_residues(obj["ct"]["0"], E.k, E.N)
    c1 = text_to_residues(obj["ct"]["1"], E.k, E.N)
    p = obj["props"]
    ct = Ciphertext.from_residues(ctx, c0, c1, slots=int(p["slots"]), scale=int(p["scale"]), domain=AOA_COEF)
    ct.set(int(p["level"]), int(p["slots"]), int(p["scale"]), AOA_COEF)
    return ct


def _key_coef(ctx, key):
    b, a, dom = key.numpy()
    E = ctx.engine
    out = []
    for x in (b, a):
        d = ctx.upload(x)
        if dom != AOA_COEF:
            (ctx.ntt_inv if dom == AOA_NTT else ctx.dgt_inv)(d, 1, 0, len(E.primes))
        out.append(d.numpy())
    return out


def export_keys(ctx, sk, pk, evk):
    """The reference's key JSON: sk = [k+kl][N] secret residues (coefficients),
    pk a Ciphertext (b, a), evk a SwitchKey."""
    E = ctx.engine
    pb, pa = pk.download(nlimbs=E.k, domain=AOA_COEF)
    eb, ea = _key_coef(ctx, evk)
    return {"sk": {"s": residues_to_text(sk)}, "pk": {"a": residues_to_text(pa), "b": residues_to_text(pb)},
            "evk": {"a": residues_to_text(ea), "b": residues_to_text(eb)}}


def load_keys(ctx, obj):
    """(sk residues, pk Ciphertext, evk SwitchKey) from the reference's key JSON."""
    E = ctx.engine
    nqb = len(E.primes)
    sk = text_to_residues(obj["sk"]["s"], nqb, E.N)
    pk = Ciphertext.from_residues(ctx, text_to_residues(obj["pk"]["b"], E.k, E.N),
                                  text_to_residues(obj["pk"]["a"], E.k, E.N), domain=AOA_COEF)
    evk = SwitchKey(ctx, text_to_residues(obj["evk"]["b"], nqb, E.N), text_to_residues(obj["evk"]["a"], nqb, E.N),
                    domain=AOA_COEF)
    return sk, pk, evk


# ---- binary wire format -----------------------------------------------------------

def ct_to_bytes(ctx, ct):
    lib = capi.load()
    n = lib.aoa_ct_wire_size(ctx.handle, ct.handle)
    buf = ctypes.create_string_buffer(n)
    ln = ctypes.c_size_t()
    capi.check(lib.aoa_ct_serialize(ctx.handle, ct.handle, buf, n, ctypes.byref(ln)))
    return buf.raw[: ln.value]


def ct_from_bytes(ctx, data, out=None):
    ct = out if out is not None else Ciphertext(ctx)
    capi.check(capi.load().aoa_ct_deserialize(ctx.handle, ct.handle, data, len(data)))
    return ct


def key_to_bytes(ctx, key):
    lib = capi.load()
    n = lib.aoa_swk_wire_size(ctx.handle)
    buf = ctypes.create_string_buffer(n)
    ln = ctypes.c_size_t()
    capi.check(lib.aoa_swk_serialize(ctx.handle, key.handle, buf, n, ctypes.byref(ln)))
    return buf.raw[: ln.value]


def key_from_bytes(ctx, data):
    h = ctypes.c_void_p()
    capi.check(capi.load().aoa_swk_deserialize(ctx.handle, data, len(data), ctypes.byref(h)))
    return SwitchKey(ctx, None, None, handle=h)
