"""The no-allocation variant of perform_pir_split, through the C ABI.

Some callers of this library cannot allocate device memory while they answer
a query -- a server that has given all of HBM to shard slabs, or a request
handler that must not call cudaMalloc (it can fail under memory pressure and
it synchronizes the device).  dnspir_db_perform_pir_split_noalloc serves them
from a fixed region of device memory that dnspir_db_create reserves.  This
test checks, on two calls in a row per shard shape, that it returns exactly
what the allocating entry point (dnspir_db_perform_pir_split) returns -- the
path is integer arithmetic, so the tolerance is zero -- and, at N = 2048, what
the CPU oracle's perform_pir_split (base_pir.rs:958) returns; that no call,
the first one after the shard is created included, changes the device's free
memory; and that work queued on a caller's own stream is complete once that
stream alone is synchronized.  The file name sorts last so that a run
stopping at the first failure has run every other test before this one.
"""
import ctypes

import numpy as np
import pytest

import dnspir_b200 as dp
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _noalloc(db, d_qb, d_qc, d_gk, d_out, stream=None):
    L = dp.lib()
    rc = L.dnspir_db_perform_pir_split_noalloc(
        db._h, ctypes.c_void_p(d_qb.data_ptr()),
        None if d_qc is None else ctypes.c_void_p(d_qc.data_ptr()),
        ctypes.c_void_p(d_gk.data_ptr()), ctypes.c_void_p(d_out.data_ptr()),
        None if stream is None else ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, L.dnspir_last_error().decode()


@pytest.mark.parametrize("log2n,l", [(8, 256), (8, 32), (11, 2048)])
def test_noalloc_matches_allocating_entry_point(log2n, l):
    torch = pytest.importorskip("torch")
    n = 1 << log2n
    gen = np.random.default_rng(100 + l)
    data = gen.integers(0, dp.PLAIN_MODULUS, size=(8 * l, n), dtype=np.uint16)
    ref = None
    if log2n == 11:
        ref = orc.Database(log2n, l)
        ref.set_db(data)
    queries = []
    for call in range(2):
        qb = gen.integers(0, dp.Q, size=(8, n), dtype=np.int64)
        qc = gen.integers(0, dp.Q, size=(8, n), dtype=np.int64) if l == n else None
        gk = gen.integers(0, dp.Q, size=(8, 2, n), dtype=np.int64)
        d = (torch.from_numpy(qb).cuda(), None if qc is None else torch.from_numpy(qc).cuda(),
             torch.from_numpy(gk).cuda(), torch.full((8, n), -1, dtype=torch.int64, device="cuda"))
        queries.append(((qb, qc, gk), d))
    torch.cuda.synchronize()
    db = dp.PIRDatabase(log2n, l)
    db.set_db(data)
    for call, ((qb, qc, gk), (d_qb, d_qc, d_gk, d_out)) in enumerate(queries):
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        _noalloc(db, d_qb, d_qc, d_gk, d_out)
        torch.cuda.synchronize()
        # the first call after the shard was created included
        assert torch.cuda.mem_get_info()[0] == free_before, f"call {call} changed the free device memory"
        got = d_out.cpu().numpy().view(np.uint64)
        want = db.perform_pir_split(qb, qc, gk)
        assert np.array_equal(got, want), f"call {call}"
        if ref is not None:
            assert np.array_equal(got.astype(np.int64), ref.perform_pir_split(qb, qc, gk)), f"call {call}"
    db.close()


def test_noalloc_on_a_caller_stream():
    # work is queued on the caller's stream: synchronizing that stream alone
    # makes the answer visible; set_db afterwards waits for it
    torch = pytest.importorskip("torch")
    log2n, l, n = 8, 256, 256
    gen = np.random.default_rng(7)
    db = dp.PIRDatabase(log2n, l)
    db.set_db(gen.integers(0, dp.PLAIN_MODULUS, size=(8 * l, n), dtype=np.uint16))
    stream = torch.cuda.Stream()
    for call in range(2):
        qb = gen.integers(0, dp.Q, size=(8, n), dtype=np.int64)
        qc = gen.integers(0, dp.Q, size=(8, n), dtype=np.int64)
        gk = gen.integers(0, dp.Q, size=(8, 2, n), dtype=np.int64)
        with torch.cuda.stream(stream):
            d_qb, d_qc, d_gk = (torch.from_numpy(x).cuda() for x in (qb, qc, gk))
            d_out = torch.full((8, n), -1, dtype=torch.int64, device="cuda")
        _noalloc(db, d_qb, d_qc, d_gk, d_out, stream)
        stream.synchronize()
        got = d_out.cpu().numpy().view(np.uint64)
        assert np.array_equal(got, db.perform_pir_split(qb, qc, gk)), f"call {call}"
    db.close()
