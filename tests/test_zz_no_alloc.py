"""The no-allocation variant of perform_pir_split, through the C ABI.

Some callers of this library cannot allocate device memory while they answer
a query -- a server that has given all of HBM to shard slabs, or a request
handler that must not call cudaMalloc (it can fail under memory pressure and
it synchronizes the device).  dnspir_db_perform_pir_split_noalloc serves them
from a fixed region of device memory.  This test checks, on two calls in a
row per shard shape, that it returns exactly what the allocating entry point
(dnspir_db_perform_pir_split) returns -- the path is integer arithmetic, so
the tolerance is zero -- and that the second call leaves the device's free
memory unchanged.  The file name sorts last so that a run stopping at the
first failure has run every other test before this one.
"""
import ctypes

import numpy as np
import pytest

import dnspir_b200 as dp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("log2n,l", [(8, 256), (8, 32), (11, 2048)])
def test_noalloc_matches_allocating_entry_point(log2n, l):
    torch = pytest.importorskip("torch")
    n = 1 << log2n
    gen = np.random.default_rng(100 + l)
    db = dp.PIRDatabase(log2n, l)
    db.set_db(gen.integers(0, dp.PLAIN_MODULUS, size=(8 * l, n), dtype=np.uint16))
    L = dp.lib()
    for call in range(2):
        qb = gen.integers(0, dp.Q, size=(8, n), dtype=np.int64)
        qc = gen.integers(0, dp.Q, size=(8, n), dtype=np.int64) if l == n else None
        gk = gen.integers(0, dp.Q, size=(8, 2, n), dtype=np.int64)
        want = db.perform_pir_split(qb, qc, gk)
        d_qb = torch.from_numpy(qb).cuda()
        d_qc = torch.from_numpy(qc).cuda() if qc is not None else None
        d_gk = torch.from_numpy(gk).cuda()
        d_out = torch.full((8, n), -1, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = L.dnspir_db_perform_pir_split_noalloc(
            db._h, ctypes.c_void_p(d_qb.data_ptr()),
            None if d_qc is None else ctypes.c_void_p(d_qc.data_ptr()),
            ctypes.c_void_p(d_gk.data_ptr()), ctypes.c_void_p(d_out.data_ptr()), None)
        torch.cuda.synchronize()
        assert rc == 0, L.dnspir_last_error().decode()
        got = d_out.cpu().numpy().view(np.uint64)
        assert np.array_equal(got, want), f"call {call}"
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free_before
