"""GPU parity at the headline primary shape: full primary groups of order
N = 2048 (both halves of the scan, conjugate queries -- the shape every shard
of the 2^20 and 2^22 databases has, get_database_shape, pir_wrapper.rs:219),
reply bytes against the CPU oracle bit for bit and every reply decrypted.

Covered here and nowhere else byte for byte: the conjugate half of the
N = 2048 scan (base_pir.rs:1007-1064), the N = 2048 primary epilogue with
both halves (base_pir.rs:1066-1077), and the tensor layout with both signs at
K = 6144 (three arrays x two halves x 1024 rows), on both engines, alone and
in groups of 4 and 64 queries (and under the tuned tile).  The fleets hold
4 logical shards on 2 distinct full shards under a secondary group of order
512 (the 2^20 shapes with fewer shards), and 2 shards on 1 distinct under the
full secondary group of order 2048 (the 2^22 shapes), so that the oracle
answers each query in seconds.
"""
import numpy as np
import pytest

import dnspir_b200 as dp
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

L1 = 2048
PER = 8 * L1  # entries per shard


def _data(seed, rows, n):
    return np.random.default_rng(seed).integers(0, orc.T, size=(rows, n), dtype=np.uint16)


@pytest.fixture(scope="module")
def shards():
    data = np.stack([_data(900 + i, PER, dp.N) for i in range(2)])
    refs = []
    for i in range(2):
        d = orc.Database(11, L1)
        d.set_db(data[i])
        refs.append(d)
    return data, refs


def _fleet(data, l2, count, distinct, engine):
    fleet = dp.Fleet.general(11, L1, l2, count, distinct)
    if engine == dp.ENGINE_TENSOR:
        fleet.set_engine(dp.ENGINE_TENSOR)
    fleet.set_shards(0, data[:distinct])
    return fleet


@pytest.fixture(scope="module")
def fleets_512(shards):
    data, _ = shards
    out = {e: _fleet(data, 512, 4, 2, e) for e in (dp.ENGINE_CUDA_CORES, dp.ENGINE_TENSOR)}
    yield out
    for f in out.values():
        f.close()


# (primary index, shard): both halves of the shard's entries, first and last rows
PICKS = [(0, 0), (5, 1), (8191, 2), (8192, 3), (9000, 0), (PER - 1, 1), (12345, 2)]


def _check(data, refs, l2, count, distinct, picks, qs, got, compare):
    shard_refs = [refs[k % distinct] for k in range(count)]
    for k, ((i, j), (q, seed), r) in enumerate(zip(picks, qs, got)):
        if k in compare:
            assert r == orc.process_query(shard_refs, q, l2), (k, i, j)
        assert np.array_equal(orc.process_reply(r, seed), data[j % distinct][i].astype(np.int64)), (k, i, j)


@pytest.mark.parametrize("engine", [dp.ENGINE_CUDA_CORES, dp.ENGINE_TENSOR])
def test_full_primary_single_queries_match_oracle(shards, fleets_512, engine):
    data, refs = shards
    fleet = fleets_512[engine]
    rng = orc.Rng(bytes([11, engine]) + bytes(30))
    qs = [orc.prepare_query(rng, i, j, L1, 512) for i, j in PICKS]
    assert len(qs[0][0]) == dp.query_bytes(L1, 512) == 51712
    got = [fleet.process_query(q) for q, _ in qs]
    _check(data, refs, 512, 4, 2, PICKS, qs, got, compare=range(len(PICKS)))


@pytest.mark.parametrize("batch", [4, 64])
def test_full_primary_tensor_groups_match_oracle(shards, fleets_512, batch):
    # one pass of the tensor scan over the slabs per group of `batch`; replies
    # are the oracle's bytes (a sample) and every one decrypts
    data, refs = shards
    fleet = fleets_512[dp.ENGINE_TENSOR]
    nq = batch + 3
    picks = [((2731 * k + 17) % PER, (5 * k + 1) % 4) for k in range(nq)]
    rng = orc.Rng(bytes([12, batch]) + bytes(30))
    qs = [orc.prepare_query(rng, i, j, L1, 512) for i, j in picks]
    fleet.set_batch(batch)
    try:
        got = fleet.process_queries([q for q, _ in qs])
    finally:
        fleet.set_batch(1)
    compare = sorted({0, 1, batch // 2, batch - 1, batch, nq - 1})
    _check(data, refs, 512, 4, 2, picks, qs, got, compare)


def test_full_primary_tuned_tile_matches_oracle(shards, fleets_512):
    # the autotuner's tile for groups of 64, then a group under it
    data, refs = shards
    fleet = fleets_512[dp.ENGINE_TENSOR]
    chosen, ms, shapes = fleet.tune(64)
    assert ms[chosen] > 0
    picks = [((4099 * k + 3) % PER, (3 * k) % 4) for k in range(64)]
    rng = orc.Rng(bytes([13]) + bytes(31))
    qs = [orc.prepare_query(rng, i, j, L1, 512) for i, j in picks]
    fleet.set_batch(64)
    try:
        got = fleet.process_queries([q for q, _ in qs])
    finally:
        fleet.set_batch(1)
        fleet.set_tile(64, -1)
    _check(data, refs, 512, 4, 2, picks, qs, got, compare=[0, 21, 63])


def test_full_primary_cuda_core_group_matches_oracle(shards, fleets_512):
    data, refs = shards
    fleet = fleets_512[dp.ENGINE_CUDA_CORES]
    picks = [((977 * k + 8190) % PER, k % 4) for k in range(16)]
    rng = orc.Rng(bytes([14]) + bytes(31))
    qs = [orc.prepare_query(rng, i, j, L1, 512) for i, j in picks]
    fleet.set_batch(16)
    try:
        got = fleet.process_queries([q for q, _ in qs])
    finally:
        fleet.set_batch(1)
    _check(data, refs, 512, 4, 2, picks, qs, got, compare=[0, 7, 15])


def test_engines_scan_words_agree_at_full_primary(shards, fleets_512):
    # the scan alone (main_pir_loop outputs of every shard) on both engines,
    # word for word, for a group of 8 arbitrary query vectors
    torch = pytest.importorskip("torch")
    gen = np.random.default_rng(15)
    nq = 8
    qnat = np.zeros((nq, 6, 2, dp.N), dtype=np.uint32)
    qnat[:, :4, 0] = gen.integers(0, dp.Q1, size=(nq, 4, dp.N))
    qnat[:, :4, 1] = gen.integers(0, dp.Q2, size=(nq, 4, dp.N))
    q = torch.from_numpy(qnat.view(np.int32)).cuda()
    outs = []
    for e in (dp.ENGINE_CUDA_CORES, dp.ENGINE_TENSOR):
        f = fleets_512[e]
        f.set_batch(8)
        try:
            o = torch.zeros((nq, 4, 2, dp.N, 8), dtype=torch.int32, device="cuda")
            f.scan(q, o)
            outs.append(o.cpu().numpy())
        finally:
            f.set_batch(1)
    assert np.array_equal(outs[0], outs[1])


def test_cta_pair_tiles_at_full_primary(shards, fleets_512):
    # every CTA-pair tile of the tensor scan (tcgen05.mma.cta_group::2), both
    # load forms, at K = 6144 with both signs: scan words equal the CUDA-core
    # engine's for a group of 64 arbitrary query vectors
    torch = pytest.importorskip("torch")
    gen = np.random.default_rng(17)
    nq = 64
    qnat = np.zeros((nq, 6, 2, dp.N), dtype=np.uint32)
    qnat[:, :4, 0] = gen.integers(0, dp.Q1, size=(nq, 4, dp.N))
    qnat[:, :4, 1] = gen.integers(0, dp.Q2, size=(nq, 4, dp.N))
    q = torch.from_numpy(qnat.view(np.int32)).cuda()

    def scan(f):
        o = torch.zeros((nq, 4, 2, dp.N, 8), dtype=torch.int32, device="cuda")
        f.set_batch(nq)
        try:
            f.scan(q, o)
        finally:
            f.set_batch(1)
        return o.cpu().numpy()

    want = scan(fleets_512[dp.ENGINE_CUDA_CORES])
    ft = fleets_512[dp.ENGINE_TENSOR]
    # relayed bulk copies (2) and tensor-map copies on the leader's barrier (3)
    pairs = [i for i, s in enumerate(dp.tscan_shapes()) if s[3] in (2, 3)]
    assert pairs
    try:
        for i in pairs:
            ft.set_tile(nq, i)
            assert np.array_equal(scan(ft), want), dp.tscan_shapes()[i]
    finally:
        ft.set_tile(nq, -1)


def test_full_primary_full_secondary_matches_oracle(shards):
    # the 2^22 shapes: full primary and full secondary group (1024 chain steps
    # per half); tensor engine, alone and as one group of 3
    data, refs = shards
    fleet = _fleet(data, 2048, 2, 1, dp.ENGINE_TENSOR)
    try:
        picks = [(3, 0), (PER - 2, 1), (10000, 1)]
        rng = orc.Rng(bytes([16]) + bytes(31))
        qs = [orc.prepare_query(rng, i, j, L1, 2048) for i, j in picks]
        assert len(qs[0][0]) == 60416
        single = [fleet.process_query(q) for q, _ in qs]
        fleet.set_batch(3)
        group = fleet.process_queries([q for q, _ in qs])
        fleet.set_batch(1)
        assert group == single
        _check(data, refs, 2048, 2, 1, picks, qs, single, compare=range(3))
    finally:
        fleet.close()
