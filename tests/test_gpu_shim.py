"""The drop-in boundary compiled: a C++ caller written against the reference
evaluator's signatures (aoa-ntt include/newckks/ckks/ckks.h:116-314; the
same names in aoa-dgt include/AOADGT/ckks.h) builds against the shim headers
include/newckks/ckks/ckks.h and include/AOADGT/ckks.h, links libaoa_b200.so and
runs ckks_mul, ckks_rotate_left / ckks_rotate_right, ckks_rescale,
ckks_add / ckks_sub and the reference's error cases on the GPU
(tests/shim/shim_check.cpp).  Its outputs must equal the oracle's."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from oracle import Oracle, ST_COEF
from tests.ckks_inputs import make_keys, uniform_residues
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path, dgt=False):
    lib = os.path.join(ROOT, "aoa_b200", "lib")
    exe = str(tmp_path / ("shim_check_dgt" if dgt else "shim_check"))
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", "-Werror"] + (["-DSHIM_DGT"] if dgt else []) +
                          ["-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "shim", "shim_check.cpp"), "-L", lib, "-laoa_b200",
                           "-Wl,-rpath," + lib, "-o", exe])
    return exe


@pytest.mark.parametrize("dgt", [False, True])
def test_reference_signature_caller_compiles_and_matches_oracle(tmp_path, dgt):
    """newckks callers (NTT) and, with -DSHIM_DGT, AOADGT callers (the same
    names on a DGT context, CUDAEngine::init, keys given in coefficients)."""
    require_gpu()
    exe = _build(tmp_path, dgt)
    log_n, k, kl, prec = 12, 5, 6, 40
    N = 1 << log_n
    ps = oracle.gen_ntt_primes(60, 1 << 13, k + kl)
    o = Oracle(N, ps[:k], ps[k:])
    r = 3
    keys = make_keys(o, seed=61, rotations=(r, N // 2 - r))
    rng = np.random.default_rng(62)
    c1 = (uniform_residues(rng, ps[:k], N), uniform_residues(rng, ps[:k], N))
    c2 = (uniform_residues(rng, ps[:k], N), uniform_residues(rng, ps[:k], N))
    slots, s1, s2 = 8, (1 << 40) + 5, (1 << 40) + 9
    words = [np.array([log_n, k, kl, prec, slots, r, s1, s2, 0 if dgt else 1] + ps, dtype=np.uint64)]
    for key in (keys["evk"], keys["rtk"][r], keys["rtk"][N // 2 - r]):
        kb, ka = (o.ntt_inv(key[0]), o.ntt_inv(key[1])) if dgt else key
        words += [kb.ravel(), ka.ravel()]
    words += [np.concatenate([c1[0], c1[1]]).ravel(), np.concatenate([c2[0], c2[1]]).ravel()]
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    np.concatenate(words).astype(np.uint64).tofile(src)
    res = subprocess.run([exe, str(src), str(dst)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    out = np.fromfile(dst, dtype=np.uint64)

    at = 0
    results = []
    while at < out.size:
        level, sl, sc = (int(v) for v in out[at:at + 3])
        n = 2 * (level + 1) * N
        body = out[at + 3:at + 3 + n].reshape(2, level + 1, N)
        results.append((level, sl, sc, body))
        at += 3 + n
    assert len(results) == 6

    w0, w1, wsc = o.hmult(c1, c2, keys["evk"], k - 1, s1, s2, rescale=True)
    lv, sl, sc, g = results[0]
    assert (lv, sl, sc) == (k - 2, slots, wsc)
    assert np.array_equal(g[0], w0[: k - 1]) and np.array_equal(g[1], w1[: k - 1])

    for (lv, sl, sc, g), step in zip(results[1:3], (r, N // 2 - r)):
        w0, w1 = o.rotate_left(c1, step, keys["rtk"][step], k - 1, state=ST_COEF)
        assert (lv, sl, sc) == (k - 1, slots, s1)
        assert np.array_equal(g[0], w0) and np.array_equal(g[1], w1), step

    w0, w1 = o.rescale(c1[0], c1[1], k - 1)
    lv, sl, sc, g = results[3]
    assert lv == k - 2 and np.array_equal(g[0], w0[: k - 1]) and np.array_equal(g[1], w1[: k - 1])

    for (lv, sl, sc, g), sub in zip(results[4:6], (False, True)):
        w0, w1, _ = o.add(c1, c2, subtract=sub, a_state=ST_COEF, b_state=ST_COEF)
        assert (lv, sl, sc) == (k - 1, slots, s1)
        assert np.array_equal(g[0], w0) and np.array_equal(g[1], w1), sub
