"""The serving loop: every reply in the mix equals the reply to the same query
answered alone, and the oracle's.

Two resident databases of different sizes (2^15 and 2^16 entries of N = 2048,
half-size shards), queries submitted interleaved from several clients so that
groups form while others are on the device, some through device-resident
sessions (Galois keys sent once).  Each reply is compared byte for byte with
the fleet's own process_query run before the server started (the plain path,
process_query, pir_wrapper.rs:328) and with the oracle's, and decrypted.
"""
import time

import numpy as np
import pytest

import dnspir_b200 as dp
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
T = orc.T


def _data(seed, rows, n):
    return np.random.default_rng(seed).integers(0, T, size=(rows, n), dtype=np.uint16)


def _db(entries, distinct, seed, engine):
    l1, l2, shards = dp.get_database_shape(entries)
    data = np.stack([_data(seed + i, 8 * l1, 2048) for i in range(distinct)])
    f = dp.Fleet(entries, distinct)
    if engine:
        f.set_engine(dp.ENGINE_TENSOR)
    f.set_shards(0, data)
    refs = []
    for i in range(distinct):
        d = orc.Database(11, l1)
        d.set_db(data[i])
        refs.append(d)
    return f, data, [refs[k % distinct] for k in range(shards)], (l1, l2, shards)


@pytest.fixture(scope="module")
def two_dbs():
    a = _db(32768, 2, 300, True)
    b = _db(65536, 2, 400, False)
    return a, b


def _queries(shape, n, tag):
    l1, l2, shards = shape
    rng = orc.Rng(bytes([tag]) + bytes(31))
    out = []
    for k in range(n):
        i, j = (811 * k + 3 * tag) % (8 * l1), (5 * k + tag) % shards
        q, seed = orc.prepare_query(rng, i, j, l1, l2)
        out.append((q, seed, i, j))
    return out


def test_served_mix_equals_alone(two_dbs):
    (fa, da, ra, sa), (fb, db_, rb, sb) = two_dbs
    qa = _queries(sa, 10, 1)
    qb = _queries(sb, 9, 2)
    fb.set_batch(1)
    alone_a = [fa.process_query(q) for q, _, _, _ in qa]
    alone_b = [fb.process_query(q) for q, _, _, _ in qb]
    sv = dp.Server(max_sessions=4)
    ida = sv.add_db(fa, 8)
    idb = sv.add_db(fb, 4)
    sv.set_batching(ida, 3, 20.0)  # database a holds groups for up to 3 queries or 20 ms
    sv.start(graphs=True)
    try:
        # two clients of database a use sessions: keys sent once, then short queries
        gk = dp.GALOIS_KEY_BYTES
        s0 = sv.open_session(qa[0][0][:gk])
        s1 = sv.open_session(qa[1][0][:gk])
        tickets = []
        for wave in range(3):  # waves so that later groups replay captured graphs
            for k in range(wave, len(qa), 3):
                q = qa[k][0]
                if k in (0, 1):
                    tickets.append(("a", k, sv.submit(ida, q[gk:], session=(s0, s1)[k])))
                else:
                    tickets.append(("a", k, sv.submit(ida, q)))
            for k in range(wave, len(qb), 3):
                tickets.append(("b", k, sv.submit(idb, qb[k][0])))
            time.sleep(0.05)
        # database a again, with the same query repeated through its session
        tickets.append(("a", 0, sv.submit(ida, qa[0][0][gk:], session=s0)))
        got = [(w, k, sv.wait(t)) for w, k, t in tickets]
        sv.close_session(s0)
        sv.close_session(s1)
        st_a, st_b = sv.stats(ida), sv.stats(idb)
    finally:
        sv.stop()
        sv.close()
    for w, k, r in got:
        alone = (alone_a if w == "a" else alone_b)[k]
        assert r == alone, (w, k)
        q, seed, i, j = (qa if w == "a" else qb)[k]
        refs, data = (ra, da) if w == "a" else (rb, db_)
        assert r == orc.process_query(refs, q), (w, k)
        assert np.array_equal(orc.process_reply(r, seed), data[j % 2][i].astype(np.int64)), (w, k)
    assert st_a["completed"] == len(qa) + 1 and st_b["completed"] == len(qb)
    assert st_a["groups"] + st_b["groups"] >= 3
    assert len(st_a["latencies_ms"]) == st_a["completed"]


def test_server_rejects_and_detaches(two_dbs):
    (fa, da, ra, sa), _ = two_dbs
    sv = dp.Server(max_sessions=1)
    ida = sv.add_db(fa, 2)
    sv.start(graphs=False)
    try:
        q = _queries(sa, 1, 9)[0][0]
        with pytest.raises(dp.DnspirError) as e:
            sv.submit(ida, q[:-1])
        assert e.value.code == 1
        with pytest.raises(dp.DnspirError) as e:
            sv.submit(ida, q[dp.GALOIS_KEY_BYTES:], session=0)  # never opened
        assert e.value.code == 6
        with pytest.raises(dp.DnspirError):
            fa.process_query(q)  # attached to the server
        r = sv.wait(sv.submit(ida, q))
    finally:
        sv.stop()
        sv.close()
    assert r == fa.process_query(q)  # detached again


def test_wait_times_out_and_the_request_is_still_answered(two_dbs):
    # dnspir_server_wait's host timeout: a request held back by a long batching
    # window (16 queries or 300 ms) is not answered within 1 ms; the wait
    # returns DNSPIR_ERR_TIMEOUT and leaves the ticket in place, and a later
    # wait receives the reply (the oracle's bytes, decrypting to the entry)
    (fa, data, refs, shape), _ = two_dbs
    sv = dp.Server(device=0)
    try:
        db = sv.add_db(fa, 16)
        sv.set_batching(db, 16, 300.0)
        sv.start(graphs=False)
        q, seed, i, j = _queries(shape, 1, 91)[0]
        t0 = time.perf_counter()
        ticket = sv.submit(db, q)
        with pytest.raises(dp.DnspirError) as e:
            sv.wait(ticket, timeout_ms=1)
        assert e.value.code == 5
        r = sv.wait(ticket, timeout_ms=120000)
        assert time.perf_counter() - t0 >= 0.25  # it waited for the window
        assert r == orc.process_query(refs, q)
        assert np.array_equal(orc.process_reply(r, seed), data[j % 2][i].astype(np.int64))
    finally:
        sv.stop()
        sv.close()
