"""GPU parity: the CUDA path, through the C ABI, against the CPU oracle.

Bit-exact equality of every output (integer arithmetic; no tolerance), plus the
client's decryption of every answer, on the cases of the reference's own tests
(N = 8 and 256, full group and subgroups; base_pir.rs:1281-1537,
double_pir.rs:328-451) and on the CPU-runnable bench configuration (2^15
entries of N = 2048, pir_wrapper.rs:493-615).
"""
import numpy as np
import pytest

import dnspir_b200 as dp
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
T = orc.T


def _data(seed, rows, n):
    return np.random.default_rng(seed).integers(0, T, size=(rows, n), dtype=np.uint16)


def _monomial(n, e):
    m = np.zeros(n, dtype=np.int64)
    e %= 2 * n
    if e < n:
        m[e] = 1
    else:
        m[e - n] = T - 1
    return m


@pytest.mark.parametrize("log2n,l", [(3, 8), (3, 4), (3, 2), (8, 256), (8, 128), (8, 32), (8, 8)])
def test_set_db_get_a_matches_oracle(log2n, l):
    # preprocessing (set_transformed_entries + the partial_gal chain) end to end:
    # get_a depends on every encoded entry and on every chain step
    n = 1 << log2n
    data = _data(l, 8 * l, n)
    ref = orc.Database(log2n, l)
    ref.set_db(data)
    db = dp.PIRDatabase(log2n, l)
    db.set_db(data)
    assert np.array_equal(db.get_a().astype(np.int64), ref.get_a())


@pytest.mark.parametrize("l", [256, 32])
def test_perform_pir_split_matches_oracle(l):
    # arbitrary ring elements as queries: checks the scan on every lane
    log2n, n = 8, 256
    data = _data(7 + l, 8 * l, n)
    ref = orc.Database(log2n, l)
    ref.set_db(data)
    db = dp.PIRDatabase(log2n, l)
    db.set_db(data)
    gen = np.random.default_rng(l)
    qb = gen.integers(0, orc.Q, size=(8, n), dtype=np.int64)
    qc = gen.integers(0, orc.Q, size=(8, n), dtype=np.int64) if l == n else None
    gk = gen.integers(0, orc.Q, size=(8, 2, n), dtype=np.int64)
    want = ref.perform_pir_split(qb, qc, gk)
    got = db.perform_pir_split(qb, qc, gk)
    assert np.array_equal(got.astype(np.int64), want)


def test_base_pir_split_decrypts():
    # base_pir.rs:1496-1537 on the GPU: 8 clients, one per lane
    n = 256
    data = _data(3, 8 * n, n)
    db = dp.PIRDatabase(8, n)
    db.set_db(data)
    rng = orc.Rng(bytes(32))
    sks = [orc.gen_sk(rng, 8) for _ in range(8)]
    gks = np.stack([orc.gen_gk_b(rng, 8, sks[i]) for i in range(8)])
    a = db.get_a().astype(np.int64)
    for idx in (0, 13, 255):
        qbs = np.stack([orc.enc_sym_b(rng, 8, 2, sks[i], _monomial(n, idx)) for i in range(8)])
        qcbs = np.stack([orc.enc_sym_b(rng, 8, 3, sks[i], _monomial(n, 2 * n - idx)) for i in range(8)])
        b = db.perform_pir_split(qbs, qcbs, gks).astype(np.int64)
        for i in range(8):
            assert np.array_equal(orc.dec(8, sks[i], a[i], b[i]), data[idx * 8 + i].astype(np.int64))


def _fleets(log2n, l1, l2, count, distinct, seed):
    n = 1 << log2n
    data = np.stack([_data(seed + i, 8 * l1, n) for i in range(distinct)])
    refs = []
    for i in range(distinct):
        d = orc.Database(log2n, l1)
        d.set_db(data[i])
        refs.append(d)
    fleet = dp.Fleet.general(log2n, l1, l2, count, distinct)
    fleet.set_shards(0, data)
    return data, [refs[k % distinct] for k in range(count)], fleet


@pytest.mark.parametrize("l1,l2,count,distinct", [(256, 256, 1, 1), (128, 16, 2, 2), (256, 32, 4, 2)])
def test_double_pir_matches_oracle_and_decrypts(l1, l2, count, distinct):
    # double_pir.rs:328-451 (full groups, half-size primary + subgroup secondary)
    log2n, n = 8, 256
    data, refs, fleet = _fleets(log2n, l1, l2, count, distinct, 40 + l1 + count)
    rng = orc.Rng(bytes([l2 % 256]) * 32)
    sk = orc.gen_sk(rng, log2n)
    per = 8 * l1
    cases = [(0, 0), (1, count - 1), (per - 1, 0), (9, count // 2), (per - 1, count - 1)]
    if count * 8 < l2:
        cases.append((2, count))  # a shard beyond the fleet answers zero (double_pir.rs:382-386)
    for (i, j) in cases:
        pq, pqc, sq, sqc, gk = orc.enc_double_pir(rng, log2n, l1, l2, sk, i, j)
        want = orc.perform_double_pir(refs, l2, pq, pqc, sq, sqc, gk)
        got = fleet.perform_double_pir(pq, pqc, sq, sqc, gk)
        assert np.array_equal(got.astype(np.int64), want), (i, j)
        res = orc.dec_double_pir(log2n, sk, got.astype(np.int64).reshape(6, n))
        expect = data[j % distinct][i] if j < count else np.zeros(n)
        assert np.array_equal(res, expect.astype(np.int64)), (i, j)


@pytest.fixture(scope="module")
def config1():
    # bench --db-entries 32768 --preprocessed-db-count 2 (pir_wrapper.rs:493-615)
    entries = 32768
    l1, l2, shards = dp.get_database_shape(entries)
    assert (l1, l2, shards) == (1024, 32, 4)
    data, refs, fleet = _fleets(11, l1, l2, shards, 2, 100)
    return data, refs, fleet, l1, l2, shards


def test_process_query_config1_bytes_match_oracle(config1):
    data, refs, fleet, l1, l2, shards = config1
    rng = orc.Rng(bytes([1]) + bytes(31))
    indices = [(0, 0), (1, 0), (0, 1), (2742, 3), (8191, 2), (4000, 1)]
    for (i, j) in indices:
        q, seed = orc.prepare_query(rng, i, j % shards, l1, l2)
        assert len(q) == 43008
        want = orc.process_query(refs, q)
        got = fleet.process_query(q)
        assert len(got) == 22272
        assert got == want, (i, j)
        res = orc.process_reply(got, seed)
        assert np.array_equal(res, data[(j % shards) % 2][i].astype(np.int64)), (i, j)


def test_process_queries_batch_equals_single(config1):
    data, refs, fleet, l1, l2, shards = config1
    rng = orc.Rng(bytes([2]) + bytes(31))
    qs = [orc.prepare_query(rng, 17 * k, k % shards, l1, l2) for k in range(4)]
    batch = fleet.process_queries([q for q, _ in qs])
    for (q, seed), r in zip(qs, batch):
        assert r == fleet.process_query(q)


def test_bad_query_length_is_rejected(config1):
    _, _, fleet, l1, l2, _ = config1
    rng = orc.Rng(bytes(32))
    q, _ = orc.prepare_query(rng, 0, 0, l1, l2)
    for bad in (q[:-1], q + b"\x00", b""):
        with pytest.raises(dp.DnspirError) as e:
            fleet.process_query(bad)
        assert e.value.code == 1


def test_unprepared_fleet_is_rejected():
    fleet = dp.Fleet(32768, 2)
    with pytest.raises(dp.DnspirError) as e:
        fleet.process_query(bytes(43008))
    assert e.value.code == 7


def test_conjugate_presence_is_checked():
    # double_pir.rs:160
    data, refs, fleet = _fleets(8, 256, 256, 1, 1, 5)
    z = np.zeros(256, dtype=np.uint64)
    with pytest.raises(dp.DnspirError) as e:
        fleet.perform_double_pir(z, None, z, z, np.zeros((2, 256), dtype=np.uint64))
    assert e.value.code == 2


@pytest.mark.parametrize("batch", [2, 4, 8, 16])
def test_batched_answers_equal_oracle(config1, batch):
    # one pass over the slabs per group of `batch` queries; every reply must be
    # the oracle's bytes (process_queries, pir_wrapper.rs:349)
    data, refs, fleet, l1, l2, shards = config1
    rng = orc.Rng(bytes([3, batch]) + bytes(30))
    qs = [orc.prepare_query(rng, (977 * k) % 8192, k % shards, l1, l2) for k in range(batch + 2)]
    fleet.set_batch(batch)
    try:
        got = fleet.process_queries([q for q, _ in qs])
    finally:
        fleet.set_batch(1)
    for k, ((q, seed), r) in enumerate(zip(qs, got)):
        assert r == orc.process_query(refs, q), k
        i, j = (977 * k) % 8192, k % shards
        assert np.array_equal(orc.process_reply(r, seed), data[j % 2][i].astype(np.int64))


def test_batched_group_with_rejected_query(config1):
    data, refs, fleet, l1, l2, shards = config1
    rng = orc.Rng(bytes([4]) + bytes(31))
    qs = [orc.prepare_query(rng, 5 * k, k % shards, l1, l2) for k in range(4)]
    queries = [qs[0][0], qs[1][0][:-3], qs[2][0], qs[3][0]]
    fleet.set_batch(4)
    try:
        with pytest.raises(dp.DnspirError) as e:
            fleet.process_queries(queries)
        assert e.value.code == 1
    finally:
        fleet.set_batch(1)
    # the valid queries are still answered correctly in the same call
    import ctypes
    L = dp.lib()
    bufs = [np.frombuffer(q, dtype=np.uint8) for q in queries]
    ptrs = (ctypes.c_void_p * 4)(*[b.ctypes.data for b in bufs])
    lens = (ctypes.c_uint64 * 4)(*[len(b) for b in bufs])
    out = np.zeros((4, dp.reply_bytes()), dtype=np.uint8)
    status = np.zeros(4, dtype=np.int32)
    fleet.set_batch(4)
    try:
        rc = L.dnspir_fleet_process_queries(fleet._h, ptrs, lens, 4, out.ctypes.data_as(ctypes.c_void_p),
                                            dp.reply_bytes(), status.ctypes.data_as(ctypes.c_void_p), 0)
    finally:
        fleet.set_batch(1)
    assert rc == 1 and list(status) == [0, 1, 0, 0]
    for k in (0, 2, 3):
        assert out[k].tobytes() == orc.process_query(refs, queries[k])


@pytest.mark.parametrize("batch", [32, 64])
def test_cuda_core_engine_large_groups(config1, batch):
    # groups beyond 16 on the CUDA-core engine: one launch, blocks of 16 (or
    # the tuned number of) queries on the second grid dimension
    data, refs, fleet, l1, l2, shards = config1
    rng = orc.Rng(bytes([5, batch]) + bytes(30))
    n = batch + 3
    qs = [orc.prepare_query(rng, (331 * k) % 8192, k % shards, l1, l2) for k in range(n)]
    fleet.set_batch(batch)
    try:
        got = fleet.process_queries([q for q, _ in qs])
        per_block, ms = fleet.tune_cuda_cores(batch)
        assert per_block in (1, 2, 4, 8, 16) and ms.max() > 0
        again = fleet.process_queries([q for q, _ in qs])
    finally:
        fleet.set_batch(1)
    for k, ((q, seed), r) in enumerate(zip(qs, got)):
        assert r == again[k]
        if k % 7 == 0:
            assert r == orc.process_query(refs, q), k
            i, j = (331 * k) % 8192, k % shards
            assert np.array_equal(orc.process_reply(r, seed), data[j % 2][i].astype(np.int64))


@pytest.fixture(scope="module")
def full_secondary():
    # the secondary database of 2^22 entries: the full group of order N = 2048
    # (both halves, 1024 chain steps per half), here under a small primary
    # group (l1 = 32, 256 shards on 2 distinct) so that the oracle answers in
    # seconds
    l1, l2, count, distinct = 32, 2048, 256, 2
    data, refs, fleet = _fleets(11, l1, l2, count, distinct, 700)
    return data, refs, fleet, l1, l2, count


@pytest.mark.parametrize("batch,nq", [(1, 1), (2, 3)])
def test_full_secondary_group_matches_oracle(full_secondary, batch, nq):
    data, refs, fleet, l1, l2, count = full_secondary
    rng = orc.Rng(bytes([6, batch]) + bytes(30))
    picks = [(17, 200), (8 * l1 - 1, 255), (0, 0)][:nq]
    qs = [orc.prepare_query(rng, i, j, l1, l2) for i, j in picks]
    fleet.set_batch(batch)
    try:
        got = fleet.process_queries([q for q, _ in qs])
    finally:
        fleet.set_batch(1)
    for (i, j), (q, seed), r in zip(picks, qs, got):
        assert r == orc.process_query(refs, q), (i, j)
        assert np.array_equal(orc.process_reply(r, seed), data[j % 2][i].astype(np.int64)), (i, j)


@pytest.mark.parametrize("schedule", [0, 1, 2, 6])
def test_group_schedules_keep_replies(full_secondary, schedule):
    # 64 queries answered as two groups of 32 in one call; each group's
    # secondary phase runs in two chunks (24 + 8 queries), and the second
    # group's primary phase overlaps the first group's secondary phase (0),
    # waits for all of it (1) or for its last chunk to start (2); 6 is 2 with
    # the 24-query chunk's chains as two-block clusters.  Every reply
    # decrypts; one per group is compared with the oracle byte for byte.
    data, refs, fleet, l1, l2, count = full_secondary
    rng = orc.Rng(bytes([9, schedule]) + bytes(30))
    picks = [((53 * k + 11 * schedule) % (8 * l1), (71 * k + schedule) % count) for k in range(64)]
    qs = [orc.prepare_query(rng, i, j, l1, l2) for i, j in picks]
    fleet.set_batch(32)
    fleet.set_schedule(32, schedule)
    try:
        got = fleet.process_queries([q for q, _ in qs])
    finally:
        fleet.set_schedule(32, -1)
        fleet.set_batch(1)
    for k, ((i, j), (q, seed), r) in enumerate(zip(picks, qs, got)):
        if k in (31, 63):
            assert r == orc.process_query(refs, q), k
        assert np.array_equal(orc.process_reply(r, seed), data[j % 2][i].astype(np.int64)), k


def test_full_secondary_group_large_chunk(full_secondary):
    # 16 queries: their secondary chains no longer fit one block per SM as
    # 2-block clusters, so the one-block-per-part kernel runs; three replies
    # are compared with the oracle byte for byte, all sixteen are decrypted
    data, refs, fleet, l1, l2, count = full_secondary
    rng = orc.Rng(bytes([7]) + bytes(31))
    picks = [((37 * k + 5) % (8 * l1), (29 * k + 3) % count) for k in range(16)]
    qs = [orc.prepare_query(rng, i, j, l1, l2) for i, j in picks]
    fleet.set_batch(16)
    try:
        got = fleet.process_queries([q for q, _ in qs])
    finally:
        fleet.set_batch(1)
    for k, ((i, j), (q, seed), r) in enumerate(zip(picks, qs, got)):
        if k in (0, 7, 15):
            assert r == orc.process_query(refs, q), k
        assert np.array_equal(orc.process_reply(r, seed), data[j % 2][i].astype(np.int64)), k


def _random_aparts(log2n, seed):
    return np.random.default_rng(seed).integers(0, orc.Q, size=(6, 1 << log2n), dtype=np.int64)


def test_installed_a_parts_follow_through_get_a_and_replies():
    # dnspir_set_a_parts (the hook for a-parts produced by the reference's own
    # expand, bfv.rs:46-49) and orc_set_aparts with the same six polynomials:
    # get_a (base_pir.rs:897) and the double-PIR reply follow them identically
    # on the GPU and in the oracle, differ from the default a-parts' results,
    # and the replies decrypt; a fleet preprocessed before the change answers
    # NOT_READY until its shards are set again
    log2n, n, l1, l2 = 8, 256, 256, 32
    data, refs, fleet = _fleets(log2n, l1, l2, 4, 2, 61)
    db = dp.PIRDatabase(log2n, l1)
    db.set_db(data[0])
    a_default = db.get_a().astype(np.int64)
    mine = _random_aparts(log2n, 62)
    try:
        dp.set_a_parts(log2n, mine.astype(np.uint64))
        orc.set_aparts(log2n, mine)
        with pytest.raises(dp.DnspirError) as e:
            db.get_a()
        assert e.value.code == 7
        rng = orc.Rng(bytes([63]) + bytes(31))
        sk = orc.gen_sk(rng, log2n)
        pq, pqc, sq, sqc, gk = orc.enc_double_pir(rng, log2n, l1, l2, sk, 77, 3)
        with pytest.raises(dp.DnspirError) as e:
            fleet.perform_double_pir(pq, pqc, sq, sqc, gk)
        assert e.value.code == 7
        db.set_db(data[0])
        ref0 = orc.Database(log2n, l1)
        ref0.set_db(data[0])
        a_mine = db.get_a().astype(np.int64)
        assert np.array_equal(a_mine, ref0.get_a())
        assert not np.array_equal(a_mine, a_default)
        fleet.set_shards(0, data)
        refs2 = []
        for k in range(2):
            d = orc.Database(log2n, l1)
            d.set_db(data[k])
            refs2.append(d)
        want = orc.perform_double_pir([refs2[k % 2] for k in range(4)], l2, pq, pqc, sq, sqc, gk)
        got = fleet.perform_double_pir(pq, pqc, sq, sqc, gk).astype(np.int64)
        assert np.array_equal(got, want)
        assert np.array_equal(orc.dec_double_pir(log2n, sk, got.reshape(6, n)), data[1][77].astype(np.int64))
    finally:
        dp.set_a_parts(log2n, None)
        orc.set_aparts(log2n, None)
    db.set_db(data[0])
    assert np.array_equal(db.get_a().astype(np.int64), a_default)
    fleet.close()


def test_installed_a_parts_wire_path_at_n2048():
    # the byte-level path (process_query, pir_wrapper.rs:328) at N = 2048 under
    # installed a-parts: the library's client writes the oracle client's bytes,
    # the GPU reply equals the oracle's and decrypts
    mine = _random_aparts(11, 64)
    l1, l2 = 1024, 32
    try:
        dp.set_a_parts(11, mine.astype(np.uint64))
        orc.set_aparts(11, mine)
        data, refs, fleet = _fleets(11, l1, l2, 4, 2, 65)
        for (i, j) in [(3, 0), (8000, 3)]:
            seed = bytes([66, i % 256, j]) + bytes(29)
            q, sk = dp.prepare_query(seed, i, j, l1, l2)
            q2, sk2 = orc.prepare_query(orc.Rng(seed), i, j, l1, l2)
            assert q == q2 and sk == sk2
            r = fleet.process_query(q)
            assert r == orc.process_query(refs, q)
            assert np.array_equal(dp.process_reply(r, sk), data[j % 2][i])
        fleet.close()
    finally:
        dp.set_a_parts(11, None)
        orc.set_aparts(11, None)
