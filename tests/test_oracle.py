"""The CPU oracle checked against the reference's own tests.

Restates, against oracle/dnspir_oracle.cpp:
  * the N = 8 layout known-answer tests (crates/pir/src/base_pir.rs:1281-1411),
    from tests/golden/kat_layout_n8.json (extracted from the reference's test
    source by tests/golden/make_golden.py),
  * the decrypt-equality tests at N = 256 (base_pir.rs:1413-1537,
    double_pir.rs:328-451),
  * the codec round trip (pir_wrapper.rs:442-452),
  * the reduction test (simd_zn.rs:490-542) on a sampled range,
  * the shape rules (pir_wrapper.rs:166-241) against the reference's own run
    log (ARTIFACT-APPENDIX.md:141-142) and wire sizes (:163-165).
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as orc

Q1, T = orc.Q1, orc.T


def _lift(x, m):
    x %= m
    return x - m if x > m // 2 else x


def _check_layout(db, expected_rows, factor_den):
    """assert_correctly_preprocessed of base_pir.rs:1292-1304 (lane 0, q1)."""
    n = db.n
    te = db.array(0, 0, 0)
    assert te.shape[0] == len(expected_rows)
    zeta1 = pow(orc.zeta(db.log2n, 0), -1, Q1)
    factor = pow(factor_den, -1, T)
    for k, exp in enumerate(expected_rows):
        e = [_lift(factor * x, T) % Q1 for x in exp]
        for i in range(n):
            want = sum(e[j] * pow(zeta1, (2 * i + 1) * j, Q1) for j in range(n)) % Q1
            assert int(te[k, i, 0]) == want, (k, i)


def _unit(n, count, idx, poly):
    e = np.zeros((count, n), dtype=np.uint16)
    e[idx] = poly
    return e


ONE8 = [1, 0, 0, 0, 0, 0, 0, 0]
X8 = [0, 1, 0, 0, 0, 0, 0, 0]


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kat_layout_n8.json")
KAT = json.load(open(GOLDEN))


@pytest.mark.parametrize("name", sorted(KAT["tests"]))
def test_set_transformed_entries_known_answers(name):
    # base_pir.rs:1281-1411, the cases read from the reference's test source
    # by tests/golden/make_golden.py: full group, order-4 and order-2 subgroups
    kat = KAT["tests"][name]
    db = orc.Database(kat["log2n"], kat["order"])
    for case in kat["cases"]:
        poly = ONE8 if case["entry"] == "1" else X8
        db.set_transformed_entries(_unit(8, case["count"], case["index"], poly))
        rows = [[x % T for x in row] for row in case["rows"]]
        _check_layout(db, rows, kat["factor"])


def _monomial(n, e):
    m = np.zeros(n, dtype=np.int64)
    e %= 2 * n
    if e < n:
        m[e] = 1
    else:
        m[e - n] = T - 1
    return m


def test_base_pir_single():
    # base_pir.rs:1413-1452: N = 256, full group, data[i] = i, 32 indices
    n = 256
    db = orc.Database(8, n)
    data = np.array([[i % T] + [0] * (n - 1) for i in range(8 * n)], dtype=np.uint16)
    db.set_db(data)
    rng = orc.Rng(bytes(32))
    sk = orc.gen_sk(rng, 8)
    gk = orc.gen_gk_b(rng, 8, sk)
    a = db.get_a()
    for idx in range(0, 32, 3):
        qb = orc.enc_sym_b(rng, 8, 2, sk, _monomial(n, idx))
        qcb = orc.enc_sym_b(rng, 8, 3, sk, _monomial(n, 2 * n - idx))
        b = db.perform_pir(qb, qcb, gk)
        res = orc.dec(8, sk, a[0], b[0])
        assert np.array_equal(res, data[idx * 8].astype(np.int64))


def test_base_pir_nontrivial_quotient():
    # base_pir.rs:1454-1494: subgroup of order 32, no conjugate
    n, l = 256, 32
    db = orc.Database(8, l)
    data = np.array([[i % T] + [0] * (n - 1) for i in range(8 * l)], dtype=np.uint16)
    db.set_db(data)
    qbp = n // 2 // l
    rng = orc.Rng(bytes(32))
    sk = orc.gen_sk(rng, 8)
    gk = orc.gen_gk_b(rng, 8, sk)
    a = db.get_a()
    for idx in range(0, 32, 5):
        qb = orc.enc_sym_b(rng, 8, 2, sk, _monomial(n, idx * qbp))
        b = db.perform_pir(qb, None, gk)
        assert np.array_equal(orc.dec(8, sk, a[0], b[0]), data[idx * 8].astype(np.int64))


def test_base_pir_split():
    # base_pir.rs:1496-1537: 8 clients, one per lane, random data
    n = 256
    db = orc.Database(8, n)
    gen = np.random.default_rng(0)
    data = gen.integers(0, T, size=(8 * n, n), dtype=np.uint16)
    db.set_db(data)
    rng = orc.Rng(bytes(32))
    sks = [orc.gen_sk(rng, 8) for _ in range(8)]
    gks = np.stack([orc.gen_gk_b(rng, 8, sks[i]) for i in range(8)])
    a = db.get_a()
    for idx in (0, 7, 31):
        qbs = np.stack([orc.enc_sym_b(rng, 8, 2, sks[i], _monomial(n, idx)) for i in range(8)])
        qcbs = np.stack([orc.enc_sym_b(rng, 8, 3, sks[i], _monomial(n, 2 * n - idx)) for i in range(8)])
        b = db.perform_pir_split(qbs, qcbs, gks)
        for i in range(8):
            assert np.array_equal(orc.dec(8, sks[i], a[i], b[i]), data[idx * 8 + i].astype(np.int64))


def _fleet(n, l, count, seed):
    gen = np.random.default_rng(seed)
    data = gen.integers(0, T, size=(count, 8 * l, n), dtype=np.uint16)
    dbs = []
    for i in range(count):
        d = orc.Database(int(np.log2(n)), l)
        d.set_db(data[i])
        dbs.append(d)
    return data, dbs


def test_double_pir():
    # double_pir.rs:328-388: N = 256, full groups, one database, out-of-range shard -> 0
    n = 256
    data, dbs = _fleet(n, n, 1, 1)
    rng = orc.Rng(bytes(32))
    sk = orc.gen_sk(rng, 8)
    for (i, j) in [(0, 0), (1, 1), (2, 0), (2, 1)]:
        pq, pqc, sq, sqc, gk = orc.enc_double_pir(rng, 8, n, n, sk, i, j)
        reply = orc.perform_double_pir(dbs, n, pq, pqc, sq, sqc, gk)
        res = orc.dec_double_pir(8, sk, reply.reshape(6, n))
        want = data[j][i] if j < 1 else np.zeros(n)
        assert np.array_equal(res, np.asarray(want, dtype=np.int64)), (i, j)


def test_double_pir_primary_subgroup():
    # double_pir.rs:395-451: half-size primary, subgroup secondary, no conjugates
    n, count = 256, 2
    l1, l2 = n // 2, 8 * count
    data, dbs = _fleet(n, l1, count, 2)
    rng = orc.Rng(bytes([1] * 32))
    sk = orc.gen_sk(rng, 8)
    per = 8 * l1
    for (i, j) in [(0, 0), (1, 1), (2, 0), (9, 1), (per - 1, 0), (per - 1, 1)]:
        pq, pqc, sq, sqc, gk = orc.enc_double_pir(rng, 8, l1, l2, sk, i, j)
        assert pqc is None and sqc is None
        reply = orc.perform_double_pir(dbs, l2, pq, pqc, sq, sqc, gk)
        res = orc.dec_double_pir(8, sk, reply.reshape(6, n))
        assert np.array_equal(res, data[j][i].astype(np.int64)), (i, j)


@pytest.mark.parametrize("bits", [10, 11, 12, 13, 14, 15, 16, 17, 34, 50])
def test_condense_uncondense(bits):
    # pir_wrapper.rs:442-452 (10..16) plus the widths the wire uses
    data = np.arange(1000, dtype=np.uint64) % (1 << bits)
    packed = orc.condense(bits, data)
    assert len(packed) == 1000 // 8 * bits
    back, used = orc.uncondense(bits, 1000, packed)
    assert used == len(packed)
    assert np.array_equal(back, data)


def test_uncondense_not_enough_data():
    # pir_wrapper.rs:124: "not enough data"
    with pytest.raises(orc.OracleError, match="not enough data"):
        orc.uncondense(17, 2048, b"\x00" * 100)


@pytest.mark.parametrize("K", [26, 25])
def test_reduce_after_mul_sampled(K):
    # simd_zn.rs:490-542 on the low end, the top end and random windows of [0, 2^(2K+1)]
    p = (1 << K) - (1 << 12) + 1
    gen = np.random.default_rng(K)
    starts = [0, (1 << (2 * K + 1)) - 4095] + [int(x) for x in gen.integers(0, 1 << (2 * K + 1), 6)]
    for s in starts:
        lazy, full = orc.reduce_after_mul(K, s, 4096)
        x = np.arange(s, s + 4096, dtype=np.uint64)
        r = x % p
        ok = (lazy == r) | (lazy == r + p) | ((lazy == 2 * p) & (r == 0))
        assert ok.all()
        okf = (full == r) | ((full == p) & (r == 0))
        assert okf.all()


def test_database_shapes():
    # pir_wrapper.rs:166-241; ARTIFACT-APPENDIX.md:141 ("64 x 16384 entries" at 2^20)
    assert orc.get_database_shape(32768) == (1024, 32, 4)
    assert orc.get_database_shape(1 << 18) == (1024, 256, 32)
    assert orc.get_database_shape(1 << 20) == (2048, 512, 64)
    assert orc.get_database_shape(1 << 22) == (2048, 2048, 256)
    assert orc.get_database_shape(1) == (1024, 8, 1)
    assert orc.required_memory_general(11, 2048) * 32 == 805306368
    assert orc.required_memory_general(11, 1024) * 32 == 402653184
    with pytest.raises(orc.OracleError):
        orc.get_database_shape(0)
    with pytest.raises(orc.OracleError):
        orc.get_database_shape((1 << 22) + 1)


def test_mod_switch_roundtrip_and_range():
    gen = np.random.default_rng(5)
    x = gen.integers(0, orc.Q, 4096, dtype=np.int64)
    for bits in (12, 17, 34, 50):
        e = orc.mod_switch_encode(bits, x)
        assert int(e.max()) < (1 << bits)
        d = orc.mod_switch_decode(bits, e)
        # decode(encode(x)) is within q / 2^bits of x (centred distance)
        diff = (d.astype(object) - x.astype(object)) % orc.Q
        diff = np.array([int(v) if v <= orc.Q // 2 else int(v) - orc.Q for v in diff])
        assert np.abs(diff).max() <= orc.Q // (1 << bits) + 1


def test_rng_is_chacha12_stream():
    # the StdRng restatement: deterministic, next_u64 = two next_u32 words (lo, hi)
    a = orc.Rng(bytes(32))
    b = orc.Rng(bytes(32))
    lo, hi = b.next_u32(), b.next_u32()
    assert a.next_u64() == lo | (hi << 32)
    # crossing the 64-word buffer boundary with an odd offset
    for _ in range(61):
        a.next_u32()
        b.next_u32()
    b.next_u32()
    a.next_u32()
    x = a.next_u64()
    w1, w2 = b.next_u32(), b.next_u32()
    assert x == w1 | (w2 << 32)


@pytest.mark.skipif(not orc.cpu_has_avx512(), reason="the vectorised restatement needs AVX-512")
@pytest.mark.parametrize("log2n,l,used_seeds", [(8, 256, 1), (8, 32, 1), (8, 128, 0), (11, 2048, 1)])
def test_vectorised_restatement_equals_scalar_oracle(log2n, l, used_seeds):
    # the AVX-512 restatement the CPU arm times (8 lanes per vector, as the
    # reference's simd_zn.rs) builds the same arrays as the scalar oracle --
    # transformed entries, both key digits of every chain step, reply_a -- and
    # answers perform_pir_split identically
    n = 1 << log2n
    gen = np.random.default_rng(40 + l + log2n)
    data = gen.integers(0, orc.T, size=(8 * l, n), dtype=np.uint16)
    a = orc.Database(log2n, l, used_seeds)
    a.set_db(data)
    b = orc.Database(log2n, l, used_seeds)
    b.set_db_vec(data)
    for which in range(3):
        for conj in range(2 if l == n else 1):
            for prime in range(2):
                assert np.array_equal(a.array(which, conj, prime), b.array(which, conj, prime)), (which, conj, prime)
    assert np.array_equal(a.get_a(), b.get_a())
    qb = gen.integers(0, orc.Q, size=(8, n), dtype=np.int64)
    qc = gen.integers(0, orc.Q, size=(8, n), dtype=np.int64) if l == n else None
    gk = gen.integers(0, orc.Q, size=(8, 2, n), dtype=np.int64)
    assert np.array_equal(a.perform_pir_split(qb, qc, gk), b.perform_pir_split_vec(qb, qc, gk))
