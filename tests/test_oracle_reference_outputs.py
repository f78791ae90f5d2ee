"""The oracle against outputs of the reference evaluator itself.

tests/golden/reference_outputs.npz holds what pdroalves/aoa's own aoa-ntt
kernels computed on a B200 through the reference's API (forward and inverse
hierarchical transforms, ModUp fast_conv_Q_to_B_opt, ModDown fast_conv_B_to_Q,
rescale; src/cuda/htrans/ntt.cu:321-460, src/cuda/manager.cu:90-118, 180-223,
312-341) with the reference's own prime choice and precompute
(oracle/ref/ref_harness.cu, built from the reference's sources by
oracle/ref/Makefile; fixture written by tests/golden/make_reference_outputs.py).
The inputs are regenerated here from the seeds the harness documents; every
oracle output must equal the reference's word for word."""
import os

import numpy as np
import pytest

from oracle import Oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_outputs.npz")
GAMMA = np.uint64(0x9E3779B97F4A7C15)


def splitmix_residues(seed, primes, N, max_=False):
    """Limb i, word j: the (i N + j)-th output of splitmix64 seeded with
    `seed`, reduced mod primes[i] (or primes[i] - 1 when max_)."""
    primes = [int(p) for p in primes]
    if max_:
        return np.array([np.full(N, p - 1, dtype=np.uint64) for p in primes])
    with np.errstate(over="ignore"):
        idx = np.arange(1, len(primes) * N + 1, dtype=np.uint64)
        z = np.uint64(seed) + idx * GAMMA
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    z = z.reshape(len(primes), N)
    return np.array([z[i] % np.uint64(p) for i, p in enumerate(primes)], dtype=np.uint64)


def _load():
    assert os.path.exists(GOLDEN), "missing fixture " + GOLDEN
    return np.load(GOLDEN)


def _configs(g):
    for key in sorted(g.files):
        if key.endswith("_params"):
            tag = key[: -len("_params")]
            N, k, kl, prec = (int(v) for v in g[key])
            yield tag, N, k, kl, prec, [int(p) for p in g[tag + "_primes"]]


def test_fixture_covers_the_reference_kernels():
    g = _load()
    names = set(g.files)
    for must in ("n1024_ntt_fwd_l0", "n1024_ntt_inv_l0", "n1024_ntt_fwd_max_l0", "n1024_modup_l3", "n1024_modup_l1",
                 "n1024_modup_max_l3", "n1024_moddown_l3", "n1024_moddown_l0", "n1024_rescale_l3",
                 "n1024_rescale_l1", "n4096_ntt_fwd_l0", "n4096_ntt_inv_l0"):
        assert must in names, must


def test_reference_primes_match_the_prime_table_fixture(ref_table):
    """The harness ran the reference's own prime selection: a 63-bit q0, then
    its prec-bit bucket; the special primes from its 55-bit bucket."""
    from oracle import reference_prime_set
    g = _load()
    for tag, N, k, kl, prec, primes in _configs(g):
        q, b = reference_prime_set(ref_table, k, kl, prec)
        assert primes == [int(v) for v in q + b], tag


@pytest.mark.parametrize("which", ["fwd", "fwd_max", "inv"])
def test_oracle_transforms_equal_reference(which):
    g = _load()
    for tag, N, k, kl, prec, primes in _configs(g):
        o = Oracle(N, primes[:k], primes[k:])
        if which == "inv":
            y = splitmix_residues(2, primes, N)
            got = o.ntt_inv(y)
        else:
            x = splitmix_residues(1, primes, N, max_=which == "fwd_max")
            got = o.ntt_fwd(x)
        want = g["%s_ntt_%s_l0" % (tag, which)].reshape(k + kl, N)
        assert np.array_equal(got, want), tag


def test_oracle_rns_kernels_equal_reference():
    g = _load()
    checked = 0
    for tag, N, k, kl, prec, primes in _configs(g):
        o = Oracle(N, primes[:k], primes[k:])
        for key in g.files:
            if not key.startswith(tag + "_") or "ntt" in key or key.endswith(("_params", "_primes")):
                continue
            name, level = key[len(tag) + 1:].rsplit("_l", 1)
            level = int(level)
            want = g[key]
            if name in ("modup", "modup_max"):
                x = splitmix_residues(2 + 1000 * level, primes[:k], N, max_=name == "modup_max")
                got = o.modup(x, level)
                assert np.array_equal(got, want.reshape(kl, N)), key
            elif name == "moddown":
                x = splitmix_residues(3 + 1000 * level, primes, N)
                got = o.moddown(x, level)[: level + 1]
                assert np.array_equal(got, want.reshape(level + 1, N)), key
            elif name == "rescale":
                x0 = splitmix_residues(4 + 1000 * level, primes[:k], N)
                x1 = splitmix_residues(5 + 1000 * level, primes[:k], N)
                w0, w1 = o.rescale(x0, x1, level)
                w = want.reshape(2, level, N)
                assert np.array_equal(w0[:level], w[0]) and np.array_equal(w1[:level], w[1]), key
            else:
                raise AssertionError("unknown record " + key)
            checked += 1
    assert checked >= 7
