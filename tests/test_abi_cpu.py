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
