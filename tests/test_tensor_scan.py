"""The tensor-core scan (8-bit limbs on tcgen05, tensor layout) against the
CUDA-core scan and the oracle.

The scan outputs of both engines are compared word for word on the same
shards and decoded queries (main_pir_loop, base_pir.rs:1085-1247, reduced), and
full replies of the tensor engine are compared byte for byte with the oracle's
process_query (pir_wrapper.rs:349-409) and decrypted.
"""
import numpy as np
import pytest

import dnspir_b200 as dp
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
T = orc.T
P = (67104769, 33550337)


def _data(seed, rows, n):
    return np.random.default_rng(seed).integers(0, T, size=(rows, n), dtype=np.uint16)


def _qnat(torch, nq, n, seed):
    g = np.random.default_rng(seed)
    q = np.empty((nq, 6, 2, n), dtype=np.uint32)
    for p in range(2):
        q[:, :, p, :] = g.integers(0, P[p], size=(nq, 6, n), dtype=np.uint32)
    return torch.from_numpy(q.view(np.int32)).cuda()


def _pair(log2n, l1, l2, count, distinct, seed):
    n = 1 << log2n
    data = np.stack([_data(seed + i, 8 * l1, n) for i in range(distinct)])
    fa = dp.Fleet.general(log2n, l1, l2, count, distinct)
    fa.set_shards(0, data)
    fb = dp.Fleet.general(log2n, l1, l2, count, distinct)
    fb.set_engine(dp.ENGINE_TENSOR)
    fb.set_shards(0, data)
    return data, fa, fb


def _scan(torch, fleet, q, count, n):
    out = torch.zeros((q.shape[0], count, 2, n, 8), dtype=torch.int32, device="cuda")
    fleet.scan(q, out)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("l1,count,distinct", [(256, 1, 1), (128, 2, 2)])
def test_tensor_scan_equals_cuda_core_scan_n256(l1, count, distinct):
    torch = pytest.importorskip("torch")
    n = 256
    _, fa, fb = _pair(8, l1, 32 if count > 1 else 256, count, distinct, 11 + l1)
    q = _qnat(torch, 3, n, l1)
    a = _scan(torch, fa, q, count, n)
    b = _scan(torch, fb, q, count, n)
    assert np.array_equal(a, b)


@pytest.fixture(scope="module")
def config1_pair():
    # 32768 entries: half-size shards (l = 1024 = N/2), 4 shards on 2 distinct
    l1, l2, shards = dp.get_database_shape(32768)
    data, fa, fb = _pair(11, l1, l2, shards, 2, 100)
    refs = []
    for i in range(2):
        d = orc.Database(11, l1)
        d.set_db(data[i])
        refs.append(d)
    return data, fa, fb, [refs[k % 2] for k in range(shards)], l1, l2, shards


@pytest.mark.parametrize("batch,nq", [(1, 2), (4, 5), (16, 16), (37, 40)])
def test_tensor_scan_equals_cuda_core_scan_config1(config1_pair, batch, nq):
    torch = pytest.importorskip("torch")
    data, fa, fb, refs, l1, l2, shards = config1_pair
    q = _qnat(torch, nq, 2048, 1000 + batch)
    a = _scan(torch, fa, q, shards, 2048)
    fb.set_batch(batch)
    try:
        b = _scan(torch, fb, q, shards, 2048)
    finally:
        fb.set_batch(1)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("batch", [1, 3, 16])
def test_tensor_engine_replies_equal_oracle(config1_pair, batch):
    data, fa, fb, refs, l1, l2, shards = config1_pair
    rng = orc.Rng(bytes([7, batch]) + bytes(30))
    qs = [orc.prepare_query(rng, (613 * k + 5) % 8192, k % shards, l1, l2) for k in range(batch + 1)]
    fb.set_batch(batch)
    try:
        got = fb.process_queries([q for q, _ in qs])
    finally:
        fb.set_batch(1)
    for k, ((q, seed), r) in enumerate(zip(qs, got)):
        assert r == orc.process_query(refs, q), k
        i, j = (613 * k + 5) % 8192, k % shards
        assert np.array_equal(orc.process_reply(r, seed), data[j % 2][i].astype(np.int64))


def test_tensor_tune_keeps_results(config1_pair):
    torch = pytest.importorskip("torch")
    data, fa, fb, refs, l1, l2, shards = config1_pair
    chosen, ms, shapes = fb.tune(8)
    assert 0 <= chosen < len(shapes) and ms[chosen] > 0
    q = _qnat(torch, 8, 2048, 77)
    fb.set_batch(8)
    try:
        b = _scan(torch, fb, q, shards, 2048)
    finally:
        fb.set_batch(1)
    assert np.array_equal(_scan(torch, fa, q, shards, 2048), b)


def test_tensor_engine_shape_rules():
    # loop_len < N/2 has no tensor layout; an engine change unprepares the shards
    f = dp.Fleet.general(8, 32, 32, 2, 2)
    with pytest.raises(dp.DnspirError) as e:
        f.set_engine(dp.ENGINE_TENSOR)
    assert e.value.code == 2
    g = dp.Fleet.general(8, 256, 256, 1, 1)
    g.set_shards(0, _data(1, 8 * 256, 256)[None])
    g.set_engine(dp.ENGINE_TENSOR)
    with pytest.raises(dp.DnspirError) as e:
        g.perform_double_pir(*([np.zeros(256, dtype=np.uint64)] * 4), np.zeros((2, 256), dtype=np.uint64))
    assert e.value.code == 7
    with pytest.raises(dp.DnspirError):
        g.set_batch(257)


def test_tensor_tune_pipeline_keeps_replies(config1_pair):
    # the whole-group tuner times shapes with zero queries, then real replies
    # of the tuned group size still equal the oracle's
    data, fa, fb, refs, l1, l2, shards = config1_pair
    chosen, ms, shapes = fb.tune(6, pipeline=True)
    assert 0 <= chosen < len(shapes) and ms[chosen] > 0
    assert fb.get_schedule(6) in (0, 1, 2, 4, 5, 6)
    rng = orc.Rng(bytes([8]) + bytes(31))
    qs = [orc.prepare_query(rng, (97 * k) % 8192, k % shards, l1, l2) for k in range(6)]
    fb.set_batch(6)
    try:
        got = fb.process_queries([q for q, _ in qs])
    finally:
        fb.set_batch(1)
    for (q, seed), r in zip(qs, got):
        assert r == orc.process_query(refs, q)


def test_every_tile_shape_equals_cuda_core_scan(config1_pair):
    # each tile shape of the tensor scan, the persistent warp-specialised
    # kernel included, forced for a group of 10 queries
    torch = pytest.importorskip("torch")
    data, fa, fb, refs, l1, l2, shards = config1_pair
    q = _qnat(torch, 10, 2048, 4242)
    want = _scan(torch, fa, q, shards, 2048)
    fb.set_batch(10)
    try:
        for i, shape in enumerate(dp.tscan_shapes()):
            fb.set_tile(10, i)
            assert np.array_equal(_scan(torch, fb, q, shards, 2048), want), shape
    finally:
        fb.set_tile(10, -1)
        fb.set_batch(1)


def test_engines_agree_at_full_size():
    # the shape of 2^22 entries: 256 full shards of order 2048 (on 2 distinct
    # shards in HBM) and the full secondary group.  The oracle would take
    # minutes per query here, so two size-independent properties stand in:
    # the tensor engine's replies equal the CUDA-core engine's byte for byte
    # (one query at a time there, groups of 4 on the tensor cores), and every
    # reply decrypts to its entry.
    entries = 1 << 22
    l1, l2, shards = dp.get_database_shape(entries)
    assert (l1, l2, shards) == (2048, 2048, 256)
    data = np.stack([_data(900 + i, 8 * l1, 2048) for i in range(2)])
    fa = dp.Fleet(entries, 2)
    fa.set_shards(0, data)
    fb = dp.Fleet(entries, 2)
    fb.set_engine(dp.ENGINE_TENSOR)
    fb.set_shards(0, data)
    rng = orc.Rng(bytes([11]) + bytes(31))
    picks = [(0, 0), (8 * l1 - 1, 255), (4097, 128), (12345, 3), (777, 201)]
    qs = [orc.prepare_query(rng, i, j, l1, l2) for i, j in picks]
    ra = fa.process_queries([q for q, _ in qs])
    fb.set_batch(4)
    try:
        rb = fb.process_queries([q for q, _ in qs])
    finally:
        fb.set_batch(1)
    for (i, j), (q, seed), a, b in zip(picks, qs, ra, rb):
        assert a == b, (i, j)
        assert np.array_equal(orc.process_reply(a, seed), data[j % 2][i].astype(np.int64)), (i, j)


def test_empty_call_and_largest_group(config1_pair):
    # no queries: nothing to answer, no error; then the largest group the
    # tensor engine takes (256 queries in one pass over the slabs): every
    # reply decrypts, and a sample equals the oracle's bytes
    data, fa, fb, refs, l1, l2, shards = config1_pair
    assert fb.process_queries([]) == []
    rng = orc.Rng(bytes([12]) + bytes(31))
    picks = [((2897 * k + 1) % (8 * l1), k % shards) for k in range(256)]
    qs = [orc.prepare_query(rng, i, j, l1, l2) for i, j in picks]
    fb.set_batch(256)
    try:
        got = fb.process_queries([q for q, _ in qs])
    finally:
        fb.set_batch(1)
    for k, ((i, j), (q, seed), r) in enumerate(zip(picks, qs, got)):
        if k % 37 == 0 or k == 255:
            assert r == orc.process_query(refs, q), k
        assert np.array_equal(orc.process_reply(r, seed), data[j % 2][i].astype(np.int64)), k


@pytest.mark.parametrize("persistent", [0, 1, 2, 3])
def test_scan_wait_runs_out_and_the_device_stays_usable(persistent):
    # the timeout path of the tensor scan's bounded waits: with a 2 ms limit
    # and the first block's producer withholding one chunk, that block's MMA
    # thread gives up, the block drains its copies, frees its tensor memory and
    # returns; the call fails with DNSPIR_ERR_TIMEOUT.  The next call, with the
    # default limit and nothing withheld, answers correctly.
    torch = pytest.importorskip("torch")
    n = 256
    _, fa, fb = _pair(8, 256, 256, 1, 1, 77)
    if persistent:
        # the persistent one-CTA kernel, or a CTA-pair kernel (whose leader
        # then gives up and raises the pair's abort flag for its follower;
        # with tensor-map copies the follower's copies of the chunks its
        # leader never armed land on the leader's barrier regardless)
        shapes = dp.tscan_shapes()
        fb.set_tile(1, next(i for i, s in enumerate(shapes) if s[3] == persistent))
    q = _qnat(torch, 1, n, 78)
    want = _scan(torch, fa, q, 1, n)
    fb.set_wait_limit(2_000_000, withhold_chunk=2)
    with pytest.raises(dp.DnspirError) as e:
        _scan(torch, fb, q, 1, n)
    assert e.value.code == 5
    fb.set_wait_limit()
    assert np.array_equal(_scan(torch, fb, q, 1, n), want)
    fa.close()
    fb.close()
