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
