"""The oracle's DGT and the RNS kernels on a DGT engine against outputs of the
reference's DGT evaluator itself.

tests/golden/reference_dgt_outputs.npz holds what pdroalves/aoa's aoa-dgt
computed on a B200 through its API (oracle/ref/ref_dgt_harness.cu, built from
aoa-dgt's sources by oracle/ref/Makefile; fixture written by
tests/golden/make_reference_outputs.py) on its own prime choice and root
tables: the single-kernel DGT at nphi = 2^10 (512 Gaussian integers) and the
hierarchical DGT at 2^13 (64 x 64), forward and inverse
(src/cuda/dgt.cu:860-1090); at 2^10 also poly_mul
(src/arithmetic/polynomial.cu:313-331), poly_modup / fast_conv_Q_to_B,
poly_moddown / fast_conv_B_to_Q and poly_ckks_rescale / ckks_rescale
(polynomial.cu:156-234, src/cuda/cudaengine.cu:264-460) at two levels.
The inputs are regenerated here from the seeds the harness documents; every
residue the oracle computes must equal the reference's."""
import json
import os

import numpy as np
import pytest

from oracle import DgtOracle, Oracle, dgt_prime_set, dgt_roots, fold, unfold
from tests.test_oracle_reference_outputs import splitmix_residues

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "reference_dgt_outputs.npz")


def load():
    assert os.path.exists(GOLDEN), "missing fixture " + GOLDEN
    return np.load(GOLDEN)


def configs(g):
    for key in sorted(g.files):
        if key.endswith("_params"):
            tag = key[: -len("_params")]
            nphi, k, kl, prec = (int(v) for v in g[key])
            yield tag, nphi, k, kl, prec, [int(p) for p in g[tag + "_primes"]]


@pytest.fixture(scope="module")
def dgt_table():
    with open(os.path.join(HERE, "golden", "dgt_roots.json")) as f:
        return json.load(f)


def _oracles(dgt_table, nphi, k, primes):
    g, r = dgt_roots(dgt_table, primes, nphi // 2)
    return DgtOracle(nphi // 2, primes, g, r), Oracle(nphi, primes[:k], primes[k:], proots=g)


def test_fixture_covers_the_reference_kernels():
    names = set(load().files)
    for must in ("n1024_dgt_fwd_l0", "n1024_dgt_inv_l0", "n1024_mul_l0", "n1024_modup_l2", "n1024_modup_l1",
                 "n1024_moddown_l2", "n1024_moddown_l1", "n1024_rescale_l2", "n1024_rescale_l1",
                 "n8192_dgt_fwd_l0", "n8192_dgt_inv_l0"):
        assert must in names, must


def test_reference_primes_are_the_dgt_prime_choice(dgt_table):
    """The harness ran aoa-dgt's own prime selection (fill_ckks_coprimes_bucket)."""
    for tag, nphi, k, kl, prec, primes in configs(load()):
        Q, B = dgt_prime_set(dgt_table, k, kl, prec)
        assert primes == [int(v) for v in Q + B], tag


def test_oracle_dgt_equals_reference(dgt_table):
    g = load()
    for tag, nphi, k, kl, prec, primes in configs(g):
        D, _ = _oracles(dgt_table, nphi, k, primes)
        n = nphi // 2
        x = splitmix_residues(1, primes, nphi)                 # coefficients, folded as the reference does
        got = D.fwd(fold(x))
        assert np.array_equal(got.reshape(-1), g[tag + "_dgt_fwd_l0"]), tag
        y = splitmix_residues(2, primes, nphi).reshape(len(primes), n, 2)   # raw transform-domain words
        got = D.inv(y)
        assert np.array_equal(got.reshape(-1), g[tag + "_dgt_inv_l0"]), tag


def test_oracle_product_and_rns_kernels_equal_reference(dgt_table):
    g = load()
    tag = "n1024"
    nphi, k, kl, prec = (int(v) for v in g[tag + "_params"])
    primes = [int(p) for p in g[tag + "_primes"]]
    D, o = _oracles(dgt_table, nphi, k, primes)
    a, b = splitmix_residues(3, primes[:k], nphi), splitmix_residues(4, primes[:k], nphi)
    prod = unfold(D.inv(D.gi_mul(D.fwd(fold(a)), D.fwd(fold(b)))))
    assert np.array_equal(prod.reshape(-1), g[tag + "_mul_l0"])
    for level in (k - 1, 1):
        x = splitmix_residues(10 + level, primes[:k], nphi)
        assert np.array_equal(o.modup(x, level).reshape(-1), g["%s_modup_l%d" % (tag, level)]), level
        x = splitmix_residues(20 + level, primes, nphi)
        got = o.moddown(x, level)[: level + 1]
        assert np.array_equal(got.reshape(-1), g["%s_moddown_l%d" % (tag, level)]), level
        c0 = splitmix_residues(30 + level, primes[:k], nphi)
        c1 = splitmix_residues(40 + level, primes[:k], nphi)
        r0, r1 = o.rescale(c0, c1, level)
        want = g["%s_rescale_l%d" % (tag, level)].reshape(2, level, nphi)
        assert np.array_equal(r0[:level], want[0]) and np.array_equal(r1[:level], want[1]), level
