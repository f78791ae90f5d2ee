"""GPU transform parity against the oracle (bit-exact), through the C ABI."""
import os

import numpy as np
import pytest

import oracle
from oracle import Oracle, reference_prime_set
from tests.gpu_util import require_gpu

pytestmark = pytest.mark.gpu


def _engine_and_oracle(log_n, q, b):
    import aoa_b200
    E = aoa_b200.Engine(log_n, q, b)
    return E, aoa_b200.Context(E), Oracle(1 << log_n, q, b)


def _rand(rng, primes, n, npolys=1):
    return np.array([[rng.integers(0, p, n, dtype=np.uint64) for p in primes] for _ in range(npolys)],
                    dtype=np.uint64)


@pytest.mark.parametrize("log_n", [10, 11, 12, 13, 14, 15, 16, 17])
def test_ntt_reference_primes(ref_table, log_n):
    require_gpu()
    Q, B = reference_prime_set(ref_table, 3, 2, 55)
    if log_n == 17:   # 2N = 2^18 must divide q - 1: keep the table primes that allow it
        ok = [q for q in [ref_table["buckets"]["63"][0]] + ref_table["buckets"]["55"] if (q - 1) % (1 << 18) == 0]
        Q, B = ok[:3], ok[3:5]
    E, ctx, o = _engine_and_oracle(log_n, Q, B)
    rng = np.random.default_rng(log_n)
    x = _rand(rng, Q + B, 1 << log_n, npolys=2)
    d = ctx.upload(x)
    ctx.ntt_fwd(d, 2, 0, len(Q + B))
    X = d.numpy()
    for p in range(2):
        assert np.array_equal(X[p], o.ntt_fwd(x[p])), "forward mismatch"
    ctx.ntt_inv(d, 2, 0, len(Q + B))
    assert np.array_equal(d.numpy(), x), "inverse(forward(x)) != x"
    y = _rand(rng, Q + B, 1 << log_n)
    dy = ctx.upload(y)
    ctx.ntt_inv(dy, 1, 0, len(Q + B))
    assert np.array_equal(dy.numpy()[0], o.ntt_inv(y[0]))


@pytest.mark.parametrize("log_n", [12, 16])
def test_ntt_60bit_primes_strided(log_n):
    require_gpu()
    ps = oracle.gen_ntt_primes(60, 1 << 17, 6)
    E, ctx, o = _engine_and_oracle(log_n, ps[:4], ps[4:])
    rng = np.random.default_rng(5)
    n = 1 << log_n
    # 3 polys of stride 6 limbs; transform limbs 0..2 with primes 2..4
    x = np.array([[rng.integers(0, ps[min(l + 2, 5)], n, dtype=np.uint64) for l in range(6)] for _ in range(3)])
    d = ctx.upload(x)
    ctx.ntt_fwd(d, 3, 2, 3, poly_stride=6)
    X = d.numpy()
    for p in range(3):
        assert np.array_equal(X[p, :3], o.ntt_fwd(x[p, :3], first=2))
        assert np.array_equal(X[p, 3:], x[p, 3:])          # untouched limbs
    ctx.ntt_inv(d, 3, 2, 3, poly_stride=6)
    assert np.array_equal(d.numpy(), x)


def test_ntt_golden_vectors():
    require_gpu()
    import aoa_b200
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "ntt_n1024.npz"))
    primes = [int(v) for v in g["primes"]]
    E = aoa_b200.Engine(10, primes[:-1], primes[-1:])
    ctx = aoa_b200.Context(E)
    d = ctx.upload(g["x"])
    ctx.ntt_fwd(d, 1, 0, len(primes))
    assert np.array_equal(d.numpy(), g["X"])


def test_ntt_edge_values(ref_table):
    """All-zero, all (q-1) and single-impulse limbs."""
    require_gpu()
    Q, B = reference_prime_set(ref_table, 2, 1, 55)
    E, ctx, o = _engine_and_oracle(13, Q, B)
    n = 1 << 13
    x = np.zeros((3, n), dtype=np.uint64)
    x[1] = np.uint64(Q[1] - 1)
    x[2, 17] = 1
    d = ctx.upload(x)
    ctx.ntt_fwd(d, 1, 0, 3)
    assert np.array_equal(d.numpy(), o.ntt_fwd(x))


@pytest.mark.parametrize("log_n", [12, 15, 16])
@pytest.mark.parametrize("shape", [(s, c, r, k) for s in (-2, -1, 0, 1, 2) for c, r in ((0, 0), (1, 2), (2, 1))
                                   for k in (0, 1)])
def test_ntt_launch_shapes_bit_exact(log_n, shape):
    """Every split, tile shape and column-pass kind the autotuner may pick
    gives the oracle's transform."""
    require_gpu()
    split, cdiv, rdiv, kind = shape
    ps = oracle.gen_ntt_primes(60, 2 << log_n, 3)
    E, ctx, o = _engine_and_oracle(log_n, ps[:2], ps[2:])
    E.tune("ntt_split", split)
    E.tune("ntt_cols_div", cdiv)
    E.tune("ntt_rows_div", rdiv)
    E.tune("ntt_cols_kind", kind)
    rng = np.random.default_rng(log_n + 7 * (split + 2) + 100 * kind)
    x = _rand(rng, ps, 1 << log_n, npolys=3)
    d = ctx.upload(x)
    ctx.ntt_fwd(d, 3, 0, 3)
    X = d.numpy()
    assert np.array_equal(X[2], o.ntt_fwd(x[2])), "forward mismatch"
    ctx.ntt_inv(d, 3, 0, 3)
    assert np.array_equal(d.numpy(), x), "inverse(forward(x)) != x"


@pytest.mark.parametrize("bits", [60, 61, 62])
@pytest.mark.parametrize("shape", [(0, 0), (-1, 0), (1, 0), (0, 1), (1, 1)])
def test_ntt_prime_size_edges(bits, shape):
    """The largest primes below 2^60 (lazy butterflies: forward values up to
    16q just below 2^64, products from the three-product Shoup quotient up to
    4q), below 2^61 and below 2^62 (strict butterflies), with all-(q-1) and
    random inputs, for even and odd column-pass stage counts."""
    require_gpu()
    split, kind = shape
    log_n = 15
    ps = oracle.gen_ntt_primes(bits, 1 << 17, 4)
    E, ctx, o = _engine_and_oracle(log_n, ps[:2], ps[2:])
    E.tune("ntt_split", split)
    E.tune("ntt_cols_kind", kind)
    rng = np.random.default_rng(bits + 10 * (split + 2) + 100 * kind)
    x = _rand(rng, ps, 1 << log_n, npolys=2)
    x[0] = np.array([[p - 1] * (1 << log_n) for p in ps], dtype=np.uint64)
    d = ctx.upload(x)
    ctx.ntt_fwd(d, 2, 0, 4)
    X = d.numpy()
    for p in range(2):
        assert np.array_equal(X[p], o.ntt_fwd(x[p])), "forward mismatch"
    ctx.ntt_inv(d, 2, 0, 4)
    assert np.array_equal(d.numpy(), x), "inverse(forward(x)) != x"


@pytest.mark.parametrize("log_n,split", [(12, 0), (15, -1), (16, 0), (16, 1), (17, 0)])
@pytest.mark.parametrize("src", [False, True])
def test_column_tiles_by_tensor_map_equal_row_copies(log_n, split, src):
    """The column pass's 16-column tiles loaded by one tensor-map (TMA) load
    (knob ntt_cols_tma, the default) and by one bulk copy per tile row give
    the oracle's transforms, for strided polys in several launch chunks and
    for the out-of-place first pass of HMult's inverse of d2."""
    require_gpu()
    import aoa_b200 as aoa
    ps = oracle.gen_ntt_primes(60, 2 << log_n, 5)
    E, ctx, o = _engine_and_oracle(log_n, ps[:3], ps[3:])
    E.tune("ntt_split", split)
    E.tune("ntt_chunk_bytes", max(1 << 20, 2 * 4 * (8 << log_n)))   # two polys per launch pair from 2^15
    rng = np.random.default_rng(log_n + 3 * split)
    x = _rand(rng, ps, 1 << log_n, npolys=5)
    res = []
    for tma in (1, 0):
        E.tune("ntt_cols_tma", tma)
        d = ctx.upload(x)
        ctx.ntt_fwd(d, 5, 0, 4, poly_stride=5)                    # limbs 0..3 of stride-5 polys
        res.append(d.numpy())
        ctx.ntt_inv(d, 5, 0, 4, poly_stride=5)
        assert np.array_equal(d.numpy(), x), tma
    assert np.array_equal(res[0], res[1])
    for p in range(5):
        assert np.array_equal(res[0][p, :4], o.ntt_fwd(x[p, :4]))
        assert np.array_equal(res[0][p, 4], x[p, 4])              # untouched limb
    if src:                                                      # HMult with the out-of-place inverse
        keys_rng = np.random.default_rng(5)
        evk = aoa.SwitchKey(ctx, _rand(keys_rng, ps, 1 << log_n)[0], _rand(keys_rng, ps, 1 << log_n)[0])
        outs = []
        for tma in (1, 0):
            E.tune("ntt_cols_tma", tma)
            ca = aoa.Ciphertext.from_residues(ctx, x[0, :3], x[1, :3], slots=4, domain=aoa.AOA_NTT)
            cb = aoa.Ciphertext.from_residues(ctx, x[2, :3], x[3, :3], slots=4, domain=aoa.AOA_NTT)
            out = aoa.Ciphertext(ctx)
            aoa.ckks_mul(ctx, out, ca, cb, evk)
            outs.append(out.download(nlimbs=2))
        assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_autotune_keeps_results_bit_exact():
    require_gpu()
    ps = oracle.gen_ntt_primes(60, 1 << 15, 6)
    E, ctx, o = _engine_and_oracle(14, ps[:4], ps[4:])
    rep = E.autotune(limbs=64)
    ch = rep["choice"]
    assert -2 <= ch["ntt_split"] <= 2 and 0 <= ch["ntt_cols_div"] <= 2 and 0 <= ch["ntt_rows_div"] <= 2
    assert rep["best_ms"] <= rep["start_ms"] * 1.0001 and len(rep["trials"]) >= 10
    rng = np.random.default_rng(11)
    x = _rand(rng, ps, 1 << 14, npolys=2)
    d = ctx.upload(x)
    ctx.ntt_fwd(d, 2, 0, 6)
    assert np.array_equal(d.numpy()[1], o.ntt_fwd(x[1]))


def test_misaligned_device_pointer_is_rejected():
    """The transform passes copy tiles with bulk / tensor-map copies, which need
    16-byte aligned addresses: a pointer 8 bytes into an allocation is refused
    on the host (AOA_ERR_BAD_PARAM) before any kernel runs, and the context
    stays usable."""
    require_gpu()
    import ctypes
    import aoa_b200 as aoa
    ps = oracle.gen_ntt_primes(60, 1 << 13, 3)
    E, ctx, o = _engine_and_oracle(12, ps[:2], ps[2:])
    rng = np.random.default_rng(9)
    x = _rand(rng, ps, 1 << 12)
    d = ctx.upload(np.concatenate([np.zeros(1, np.uint64), x.ravel()]))
    lib = aoa.capi.load()
    for fn in (lib.aoa_ntt_fwd, lib.aoa_ntt_inv):
        st = fn(ctx.handle, ctypes.c_void_p(d.ptr.value + 8), 1, 0, 3, 3)
        assert st == 1 and "aligned" in lib.aoa_last_error().decode()
    ctx.sync()
    d2 = ctx.upload(x)
    ctx.ntt_fwd(d2, 1, 0, 3)
    assert np.array_equal(d2.numpy()[0], o.ntt_fwd(x[0]))


@pytest.mark.parametrize("log_n", [11, 13, 16])
@pytest.mark.parametrize("shape", [(0, 0, 0), (0, 1, 1), (1, 2, 2), (-1, 2, 0), (0, 0, 1, 1)])
def test_primes_one_mod_2_32_take_the_short_remainder(log_n, shape):
    """Primes q = 1 mod 2^32 below 2^60 run the lazy butterflies with the
    shorter Shoup remainder (t q = t + (t_0 q_1) 2^32 mod 2^64).  Interleaved
    with other lazy primes and with primes above 2^60, the limbs run in runs of
    all three butterfly kinds; with all-(q-1) and random inputs, for every
    column / row tile width and the warp-owned column pass, the transforms
    equal the oracle's."""
    require_gpu()
    split, cdiv, rdiv = shape[:3]
    cols_kind = shape[3] if len(shape) > 3 else 0
    n = 1 << log_n
    q1 = oracle.gen_ntt_primes(60, 1 << 32, 3)
    lazy = [q for q in oracle.gen_ntt_primes(59, 2 * n, 8) if q % (1 << 32) != 1][:2]
    big = oracle.gen_ntt_primes(62, 2 * n, 2)
    assert all(q % (1 << 32) == 1 and q < 1 << 60 for q in q1) and len(lazy) == 2
    ps = [q1[0], lazy[0], q1[1], big[0], q1[2], lazy[1], big[1]]
    E, ctx, o = _engine_and_oracle(log_n, ps[:5], ps[5:])
    E.tune("ntt_split", split)
    E.tune("ntt_cols_div", cdiv)
    E.tune("ntt_rows_div", rdiv)
    E.tune("ntt_cols_kind", cols_kind)
    rng = np.random.default_rng(log_n + 17 * (split + 2) + 3 * cdiv + rdiv)
    x = _rand(rng, ps, n, npolys=3)
    x[1] = np.array([[p - 1] * n for p in ps], dtype=np.uint64)
    d = ctx.upload(x)
    ctx.ntt_fwd(d, 3, 0, 7)
    X = d.numpy()
    for p in range(3):
        assert np.array_equal(X[p], o.ntt_fwd(x[p])), p
    ctx.ntt_inv(d, 3, 0, 7)
    assert np.array_equal(d.numpy(), x)
    y = _rand(rng, ps, n)
    dy = ctx.upload(y)
    ctx.ntt_inv(dy, 1, 0, 7)
    assert np.array_equal(dy.numpy()[0], o.ntt_inv(y[0]))
    # a set of such primes only (one run per pass, as in the benchmark)
    E1, ctx1, o1 = _engine_and_oracle(log_n, q1[:2], q1[2:])
    x1 = _rand(rng, q1, n, npolys=2)
    d1 = ctx1.upload(x1)
    ctx1.ntt_fwd(d1, 2, 0, 3)
    assert np.array_equal(d1.numpy()[1], o1.ntt_fwd(x1[1]))
    ctx1.ntt_inv(d1, 2, 0, 3)
    assert np.array_equal(d1.numpy(), x1)


@pytest.mark.parametrize("log_n", [11, 16])
def test_mixed_prime_sizes_run_lazy_and_strict_limbs(log_n):
    """Primes above and below 2^60 interleaved: the limbs run in alternating
    lazy and strict runs (several launches per pass), with a first prime other
    than 0 and strided polys, and equal the oracle's transforms."""
    require_gpu()
    n = 1 << log_n
    big = oracle.gen_ntt_primes(62, 2 * n, 3)
    small = oracle.gen_ntt_primes(59, 2 * n, 4)
    ps = [small[0], big[0], big[1], small[1], small[2], big[2], small[3]]
    E, ctx, o = _engine_and_oracle(log_n, ps[:5], ps[5:])
    rng = np.random.default_rng(log_n + 40)
    x = _rand(rng, ps, n, npolys=3)
    x[1] = np.array([[p - 1] * n for p in ps], dtype=np.uint64)
    d = ctx.upload(x)
    ctx.ntt_fwd(d, 3, 0, 7)
    X = d.numpy()
    for p in range(3):
        assert np.array_equal(X[p], o.ntt_fwd(x[p])), p
    ctx.ntt_inv(d, 3, 0, 7)
    assert np.array_equal(d.numpy(), x)
    import ctypes
    lib = __import__("aoa_b200").capi.load()
    d = ctx.upload(x)                                   # limbs 2..5 (primes 2..5) of each poly
    st = lib.aoa_ntt_fwd(ctx.handle, ctypes.c_void_p(d.ptr.value + 2 * n * 8), 3, 2, 4, 7)
    assert st == 0
    X = d.numpy()
    for p in range(3):
        assert np.array_equal(X[p, 2:6], o.ntt_fwd(x[p, 2:6], first=2)), p
        assert np.array_equal(X[p, :2], x[p, :2]) and np.array_equal(X[p, 6:], x[p, 6:])
