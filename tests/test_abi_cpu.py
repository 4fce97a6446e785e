"""C-ABI checks that need no GPU: the library loads, exports every symbol
include/dnspir.h declares, its host-side shape rules and seed expansion agree
with the oracle, and it refuses to run without a CUDA device (no CPU path)."""
import ctypes
import re
import os

import numpy as np
import pytest

import dnspir_b200 as dp
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "dnspir.h")).read()
    return sorted(set(re.findall(r"\b(dnspir_[a-z0-9_]+)\s*\(", src)))


def test_exports_every_declared_symbol():
    L = dp.lib()
    names = _declared()
    assert len(names) >= 20
    for name in names:
        assert hasattr(L, name), name


def test_version():
    assert b"sm_100a" in dp.lib().dnspir_version()


@pytest.mark.parametrize("entries", [1, 8192, 8193, 32768, 1 << 18, (1 << 18) + 1, 1 << 20, 3_000_000, 1 << 22])
def test_shape_rules_match_oracle(entries):
    assert dp.get_database_shape(entries) == orc.get_database_shape(entries)


def test_shape_rejects_out_of_range():
    for bad in (0, (1 << 22) + 1):
        with pytest.raises(dp.DnspirError) as e:
            dp.get_database_shape(bad)
        assert e.value.code == 2


def test_wire_sizes():
    # ARTIFACT-APPENDIX.md:163-165 (2^20: 25600 + 26112 B query, 22272 B reply)
    assert dp.reply_bytes() == 22272
    assert dp.query_bytes(2048, 512) == 51712
    assert dp.query_bytes(2048, 2048) == 60416
    assert dp.query_bytes(1024, 32) == 43008
    assert dp.required_memory_general(11, 2048) * 32 == 805306368


@pytest.mark.parametrize("log2n", [3, 8, 11])
def test_expand_matches_oracle(log2n):
    ref = orc.aparts(log2n)
    for which in range(6):
        got = dp.expand_seed(log2n, which)
        assert np.array_equal(got.astype(np.int64), ref[which])
        assert int(got.max()) < dp.Q


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_cuda(), reason="checks the behaviour without a CUDA device")
def test_no_cpu_fallback():
    with pytest.raises(dp.DnspirError) as e:
        dp.Fleet(32768, 2)
    assert e.value.code == 4
    with pytest.raises(dp.DnspirError) as e:
        dp.PIRDatabase(8, 256)
    assert e.value.code == 4
    with pytest.raises(dp.DnspirError) as e:
        dp.Server(max_sessions=4)
    assert e.value.code == 4


def test_null_handles_are_rejected():
    # every entry point checks its handle instead of crashing
    import ctypes
    L = dp.lib()
    t = ctypes.c_uint64()
    done = ctypes.c_int()
    assert L.dnspir_server_submit(None, 0, -1, b"x", 1, ctypes.byref(t)) == 6
    assert L.dnspir_server_poll(None, 1, None, 0, ctypes.byref(done)) == 6
    assert L.dnspir_server_start(None, 1) == 6
    assert L.dnspir_server_set_batching(None, 0, 1, 0) == 6
    assert L.dnspir_fleet_set_batch(None, 1) == 6
    assert L.dnspir_fleet_set_engine(None, 1) == 6
    assert L.dnspir_fleet_tune(None, 1, None, None) == 6
    assert L.dnspir_fleet_tune_pipeline(None, 1, None, None) == 6
    assert L.dnspir_fleet_tune_cuda_cores(None, 1, None, None) == 6
    assert L.dnspir_fleet_set_tile(None, 1, 0) == 6
    assert L.dnspir_fleet_set_schedule(None, 1, 0) == 6
    assert L.dnspir_fleet_get_schedule(None, 1, None) == 6
    assert L.dnspir_server_destroy(None) == 0 and L.dnspir_fleet_destroy(None) == 0


@pytest.mark.parametrize("entries,i,j", [(32768, 0, 0), (32768, 8191, 3), (1 << 20, 12345, 63), (1 << 22, 16383, 255)])
def test_client_query_matches_oracle_client(entries, i, j):
    # the library's client (prepare_query, pir_wrapper.rs:276) produces the
    # oracle client's bytes for the same StdRng seed
    l1, l2, _ = dp.get_database_shape(entries)
    seed = bytes([7, i % 256, j % 256]) + bytes(29)
    q, sk = dp.prepare_query(seed, i, j, l1, l2)
    q2, sk2 = orc.prepare_query(orc.Rng(seed), i, j, l1, l2)
    assert q == q2 and sk == sk2
    assert len(q) == dp.query_bytes(l1, l2)


def test_client_reads_oracle_reply():
    # process_reply (pir_wrapper.rs:420) of an oracle-made answer on a 1-shard 2^13 fleet
    gen = np.random.default_rng(9)
    data = gen.integers(0, orc.T, size=(8192, 2048), dtype=np.uint16)
    db = orc.Database(11, 1024)
    db.set_db(data)
    l1, l2, s = dp.get_database_shape(8192)
    for i in (0, 5000):
        q, sk = dp.prepare_query(bytes([i % 256]) * 32, i, 0, l1, l2)
        reply = orc.process_query([db], q)
        assert np.array_equal(dp.process_reply(reply, sk), data[i])
    with pytest.raises(dp.DnspirError):
        dp.process_reply(reply[:-10], sk)


def _random_aparts(log2n, seed):
    return np.random.default_rng(seed).integers(0, dp.Q, size=(6, 1 << log2n), dtype=np.int64).astype(np.uint64)


@pytest.mark.parametrize("log2n", [3, 8, 11])
def test_a_parts_hook_roundtrip(log2n):
    # dnspir_set_a_parts installs a-parts (e.g. vectors produced by the
    # reference's expand, bfv.rs:46-49); NULL restores the seed expansion
    default = dp.get_a_parts(log2n)
    assert np.array_equal(default, np.stack([dp.expand_seed(log2n, w) for w in range(6)]))
    mine = _random_aparts(log2n, 5)
    try:
        dp.set_a_parts(log2n, mine)
        assert np.array_equal(dp.get_a_parts(log2n), mine)
        # the seed expansion itself is unchanged
        assert np.array_equal(dp.expand_seed(log2n, 0), default[0])
    finally:
        dp.set_a_parts(log2n, None)
    assert np.array_equal(dp.get_a_parts(log2n), default)


def test_a_parts_hook_rejects_unreduced(tmp_path):
    bad = _random_aparts(8, 6)
    bad[3, 17] = dp.Q
    with pytest.raises(dp.DnspirError) as e:
        dp.set_a_parts(8, bad)
    assert e.value.code == 6
    assert np.array_equal(dp.get_a_parts(8), np.stack([dp.expand_seed(8, w) for w in range(6)]))
    # the file form: raw little-endian uint64, 6 x N
    mine = _random_aparts(8, 7)
    f = tmp_path / "aparts.bin"
    mine.astype("<u8").tofile(f)
    try:
        dp.load_a_parts_file(str(f), log2_n=8)
        assert np.array_equal(dp.get_a_parts(8), mine)
    finally:
        dp.set_a_parts(8, None)


def test_client_uses_installed_a_parts():
    # with the same a-parts installed in both, the library's client and the
    # oracle's client write the same query bytes, and those differ from the
    # default a-parts' query
    l1, l2, _ = dp.get_database_shape(32768)
    seed = bytes(range(32))
    q0, _ = dp.prepare_query(seed, 3, 1, l1, l2)
    mine = _random_aparts(11, 8)
    try:
        dp.set_a_parts(11, mine)
        orc.set_aparts(11, mine.astype(np.int64))
        q, sk = dp.prepare_query(seed, 3, 1, l1, l2)
        q2, sk2 = orc.prepare_query(orc.Rng(seed), 3, 1, l1, l2)
    finally:
        dp.set_a_parts(11, None)
        orc.set_aparts(11, None)
    assert q == q2 and sk == sk2
    assert q != q0
