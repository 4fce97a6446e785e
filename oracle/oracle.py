"""ctypes binding of the CPU oracle (liboracle_dnspir.so).

Test infrastructure only: imported by tests/, by ``__graft_entry__.smoke()``
as the checker, and by bench.py's CPU-baseline leg.  The product library in
``dnspir_b200`` never imports this module.

Every function mirrors a function of the reference's crates/pir; the C++ side
cites file:line for each.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_dnspir.so")

Q1 = (1 << 26) - (1 << 12) + 1
Q2 = (1 << 25) - (1 << 12) + 1
Q = Q1 * Q2
T = 1025
SIMD = 8
LOG2_N = 11
N = 1 << LOG2_N


def build():
    """Compile the oracle with its Makefile (g++ only)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _p(t):
    return ctypes.POINTER(t)


def _declare(L):
    c = ctypes
    L.orc_last_error.restype = c.c_char_p
    L.orc_num_threads.restype = c.c_int
    L.orc_set_num_threads.argtypes = [c.c_int]
    for f in ("orc_q1", "orc_q2", "orc_q"):
        getattr(L, f).restype = c.c_uint64
    L.orc_zeta.restype = c.c_uint64
    L.orc_zeta.argtypes = [c.c_int, c.c_int]
    L.orc_rng_new.restype = c.c_void_p
    L.orc_rng_new.argtypes = [c.c_char_p]
    L.orc_rng_free.argtypes = [c.c_void_p]
    L.orc_rng_next_u64.restype = c.c_uint64
    L.orc_rng_next_u64.argtypes = [c.c_void_p]
    L.orc_rng_next_u32.restype = c.c_uint32
    L.orc_rng_next_u32.argtypes = [c.c_void_p]
    L.orc_get_aparts.argtypes = [c.c_int, c.c_void_p]
    L.orc_set_aparts.argtypes = [c.c_int, c.c_void_p]
    L.orc_expand.argtypes = [c.c_int, c.c_char_p, c.c_void_p]
    L.orc_get_database_shape.argtypes = [c.c_uint64, _p(c.c_uint32), _p(c.c_uint32), _p(c.c_uint32)]
    L.orc_choose_secondary.argtypes = [c.c_uint32, _p(c.c_uint32)]
    L.orc_required_memory_general.restype = c.c_uint64
    L.orc_required_memory_general.argtypes = [c.c_uint32, c.c_uint32]
    L.orc_db_create.argtypes = [c.c_int, c.c_uint32, c.c_int, _p(c.c_void_p)]
    L.orc_db_free.argtypes = [c.c_void_p]
    L.orc_db_set_db.argtypes = [c.c_void_p, c.c_void_p]
    L.orc_db_set_transformed_entries.argtypes = [c.c_void_p, c.c_void_p]
    L.orc_db_loop_len.restype = c.c_uint32
    L.orc_db_loop_len.argtypes = [c.c_void_p]
    L.orc_db_array.argtypes = [c.c_void_p, c.c_int, c.c_int, c.c_int, c.c_void_p]
    L.orc_db_reply_a_ntt.argtypes = [c.c_void_p, c.c_int, c.c_void_p]
    L.orc_db_get_a.argtypes = [c.c_void_p, c.c_void_p]
    L.orc_db_perform_pir_split.argtypes = [c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p]
    L.orc_db_set_db_vec.argtypes = [c.c_void_p, c.c_void_p]
    L.orc_db_perform_pir_split_vec.argtypes = [c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p]
    L.orc_perform_double_pir.argtypes = [c.c_void_p, c.c_uint32, c.c_uint32] + [c.c_void_p] * 6
    L.orc_condense.argtypes = [c.c_int, c.c_void_p, c.c_uint64, c.c_void_p, _p(c.c_uint64)]
    L.orc_uncondense.argtypes = [c.c_int, c.c_uint64, c.c_void_p, c.c_uint64, c.c_void_p, _p(c.c_uint64)]
    L.orc_ms_encode.argtypes = [c.c_int, c.c_void_p, c.c_uint64, c.c_void_p]
    L.orc_ms_decode.argtypes = [c.c_int, c.c_void_p, c.c_uint64, c.c_void_p]
    L.orc_process_query.argtypes = [c.c_void_p, c.c_uint32, c.c_void_p, c.c_uint64, c.c_void_p, _p(c.c_uint64)]
    L.orc_process_query_general.argtypes = [c.c_void_p, c.c_uint32, c.c_uint32, c.c_void_p, c.c_uint64, c.c_void_p,
                                            _p(c.c_uint64)]
    L.orc_gen_sk.argtypes = [c.c_void_p, c.c_int, c.c_void_p]
    L.orc_enc_sym_b.argtypes = [c.c_void_p, c.c_int, c.c_int, c.c_void_p, c.c_void_p, c.c_void_p]
    L.orc_gen_gk_b.argtypes = [c.c_void_p, c.c_int, c.c_void_p, c.c_void_p]
    L.orc_dec.argtypes = [c.c_int, c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p]
    L.orc_enc_double_pir.argtypes = [c.c_void_p, c.c_int, c.c_uint32, c.c_uint32, c.c_void_p, c.c_uint64,
                                     c.c_uint64] + [c.c_void_p] * 5 + [_p(c.c_int), _p(c.c_int)]
    L.orc_dec_double_pir.argtypes = [c.c_int, c.c_void_p, c.c_void_p, c.c_void_p]
    L.orc_prepare_query.argtypes = [c.c_void_p, c.c_uint64, c.c_uint64, c.c_uint32, c.c_uint32, c.c_void_p,
                                    _p(c.c_uint64), c.c_void_p]
    L.orc_process_reply.argtypes = [c.c_void_p, c.c_uint64, c.c_void_p, c.c_void_p]
    L.orc_reduce_after_mul.argtypes = [c.c_int, c.c_uint64, c.c_uint64, c.c_void_p, c.c_void_p]
    if hasattr(L, "orc_scan_baseline"):
        L.orc_scan_baseline.restype = c.c_double
        L.orc_scan_baseline.argtypes = [c.c_int, c.c_uint32, c.c_uint32, c.c_int, c.c_int, _p(c.c_int)]
        L.orc_cpu_has_avx512.restype = c.c_int
        L.orc_time_secondary.restype = c.c_double
        L.orc_time_secondary.argtypes = [c.c_int, c.c_uint32]
        L.orc_bench_new.restype = c.c_void_p
        L.orc_bench_new.argtypes = [c.c_int, c.c_uint32, c.c_uint32, c.c_uint32, c.c_uint32]
        L.orc_bench_free.argtypes = [c.c_void_p]
        L.orc_bench_step.argtypes = [c.c_void_p, c.c_int, _p(c.c_double), _p(c.c_double), _p(c.c_int)]


class OracleError(RuntimeError):
    pass


def _check(rc):
    if rc != 0:
        raise OracleError(lib().orc_last_error().decode())


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def set_num_threads(n):
    lib().orc_set_num_threads(int(n))


def num_threads():
    return lib().orc_num_threads()


def zeta(log2n, prime):
    return lib().orc_zeta(log2n, prime)


class Rng:
    """StdRng (ChaCha12) restatement; seed is 32 bytes."""

    def __init__(self, seed):
        seed = bytes(seed)
        assert len(seed) == 32
        self._h = ctypes.c_void_p(lib().orc_rng_new(seed))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_rng_free(self._h)
            self._h = None

    def next_u64(self):
        return lib().orc_rng_next_u64(self._h)

    def next_u32(self):
        return lib().orc_rng_next_u32(self._h)


def aparts(log2n):
    out = np.zeros((6, 1 << log2n), dtype=np.int64)
    _check(lib().orc_get_aparts(log2n, _ptr(out)))
    return out


def set_aparts(log2n, parts):
    """Replace the six a-parts of dimension 2^log2n ((6, N) in [0, q)); None
    restores the seed expansion."""
    if parts is None:
        _check(lib().orc_set_aparts(log2n, None))
        return
    a = np.ascontiguousarray(parts, dtype=np.int64)
    assert a.shape == (6, 1 << log2n)
    _check(lib().orc_set_aparts(log2n, _ptr(a)))


def expand(log2n, seed):
    out = np.zeros(1 << log2n, dtype=np.int64)
    _check(lib().orc_expand(log2n, bytes(seed), _ptr(out)))
    return out


def get_database_shape(num_entries):
    a, b, s = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    _check(lib().orc_get_database_shape(num_entries, ctypes.byref(a), ctypes.byref(b), ctypes.byref(s)))
    return a.value, b.value, s.value


def choose_secondary(num_shards):
    v = ctypes.c_uint32()
    _check(lib().orc_choose_secondary(num_shards, ctypes.byref(v)))
    return v.value


def required_memory_general(log2n, l):
    return lib().orc_required_memory_general(log2n, l)


class Database:
    """PIRDatabase (base_pir.rs:229) restated on the CPU."""

    def __init__(self, log2n, group_order, used_seeds=0):
        self.log2n = log2n
        self.n = 1 << log2n
        self.l = group_order
        h = ctypes.c_void_p()
        _check(lib().orc_db_create(log2n, group_order, used_seeds, ctypes.byref(h)))
        self._h = h
        self.loop_len = lib().orc_db_loop_len(h)
        self.conj = group_order == self.n

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_db_free(self._h)
            self._h = None

    def set_db(self, entries):
        e = np.ascontiguousarray(entries, dtype=np.uint16)
        assert e.shape == (8 * self.l, self.n)
        _check(lib().orc_db_set_db(self._h, _ptr(e)))

    def set_db_vec(self, entries):
        """set_db through the AVX-512 restatement (8 lanes per vector, the
        reference's simd_zn.rs shape); the same arrays as set_db."""
        e = np.ascontiguousarray(entries, dtype=np.uint16)
        assert e.shape == (8 * self.l, self.n)
        _check(lib().orc_db_set_db_vec(self._h, _ptr(e)))

    def perform_pir_split_vec(self, qry_b, qry_conj_b, gk_b):
        """perform_pir_split with the AVX-512 scan."""
        qb = np.ascontiguousarray(qry_b, dtype=np.int64)
        qc = None if qry_conj_b is None else np.ascontiguousarray(qry_conj_b, dtype=np.int64)
        gk = np.ascontiguousarray(gk_b, dtype=np.int64)
        out = np.zeros((8, self.n), dtype=np.int64)
        _check(lib().orc_db_perform_pir_split_vec(self._h, _ptr(qb), None if qc is None else _ptr(qc), _ptr(gk),
                                                  _ptr(out)))
        return out

    def set_transformed_entries(self, entries):
        e = np.ascontiguousarray(entries, dtype=np.uint16)
        assert e.shape == (8 * self.l, self.n)
        _check(lib().orc_db_set_transformed_entries(self._h, _ptr(e)))

    def array(self, which, conj, prime):
        """which: 0 = transformed_entries, 1/2 = inner_prod_gk digit 0/1; shape (L, N, 8)."""
        out = np.zeros((self.loop_len, self.n, 8), dtype=np.uint64)
        _check(lib().orc_db_array(self._h, which, conj, prime, _ptr(out)))
        return out

    def reply_a_ntt(self, prime):
        out = np.zeros((self.n, 8), dtype=np.uint64)
        _check(lib().orc_db_reply_a_ntt(self._h, prime, _ptr(out)))
        return out

    def get_a(self):
        out = np.zeros((8, self.n), dtype=np.int64)
        _check(lib().orc_db_get_a(self._h, _ptr(out)))
        return out

    def perform_pir_split(self, qry_b, qry_conj_b, gk_b):
        """qry_b: (8, N); qry_conj_b: (8, N) or None; gk_b: (8, 2, N)."""
        qb = np.ascontiguousarray(qry_b, dtype=np.int64)
        qc = None if qry_conj_b is None else np.ascontiguousarray(qry_conj_b, dtype=np.int64)
        gk = np.ascontiguousarray(gk_b, dtype=np.int64)
        out = np.zeros((8, self.n), dtype=np.int64)
        _check(lib().orc_db_perform_pir_split(self._h, _ptr(qb), None if qc is None else _ptr(qc), _ptr(gk),
                                              _ptr(out)))
        return out

    def perform_pir(self, qry_b, qry_conj_b, gk_b):
        qb = np.broadcast_to(qry_b, (8, self.n))
        qc = None if qry_conj_b is None else np.broadcast_to(qry_conj_b, (8, self.n))
        gk = np.broadcast_to(np.asarray(gk_b), (8, 2, self.n))
        return self.perform_pir_split(qb, qc, gk)


def perform_double_pir(dbs, l2, pq, pqc, sq, sqc, gk):
    """perform_double_pir (double_pir.rs:104); returns (3, 2, N) = three (a, b) ciphertexts."""
    n = dbs[0].n
    arr = (ctypes.c_void_p * len(dbs))(*[d._h.value for d in dbs])
    out = np.zeros((3, 2, n), dtype=np.int64)
    a = [np.ascontiguousarray(x, dtype=np.int64) if x is not None else None for x in (pq, pqc, sq, sqc, gk)]
    _check(lib().orc_perform_double_pir(arr, len(dbs), l2, *[None if x is None else _ptr(x) for x in a],
                                        _ptr(out)))
    return out


def condense(bits, data):
    d = np.ascontiguousarray(data, dtype=np.uint64)
    out = np.zeros(len(d) * 8 + 8, dtype=np.uint8)
    n = ctypes.c_uint64()
    _check(lib().orc_condense(bits, _ptr(d), len(d), _ptr(out), ctypes.byref(n)))
    return out[: n.value].tobytes()


def uncondense(bits, count, data):
    b = np.frombuffer(bytes(data), dtype=np.uint8)
    out = np.zeros(count, dtype=np.uint64)
    used = ctypes.c_uint64()
    _check(lib().orc_uncondense(bits, count, _ptr(b) if len(b) else None, len(b), _ptr(out), ctypes.byref(used)))
    return out, used.value


def mod_switch_encode(bits, x):
    a = np.ascontiguousarray(x, dtype=np.int64)
    out = np.zeros(a.shape, dtype=np.uint64)
    _check(lib().orc_ms_encode(bits, _ptr(a), a.size, _ptr(out)))
    return out


def mod_switch_decode(bits, x):
    a = np.ascontiguousarray(x, dtype=np.uint64)
    out = np.zeros(a.shape, dtype=np.int64)
    _check(lib().orc_ms_decode(bits, _ptr(a), a.size, _ptr(out)))
    return out


def process_query(dbs, query, secondary_order=0):
    """process_query (pir_wrapper.rs:328) on a fleet whose shard k is dbs[k];
    secondary_order 0 follows the shape rule (choose_index_group_secondary),
    else the secondary group has that order (perform_double_pir allows any)."""
    arr = (ctypes.c_void_p * len(dbs))(*[d._h.value for d in dbs])
    q = np.frombuffer(bytes(query), dtype=np.uint8)
    out = np.zeros(1 << 16, dtype=np.uint8)
    n = ctypes.c_uint64()
    _check(lib().orc_process_query_general(arr, len(dbs), secondary_order, _ptr(q), len(q), _ptr(out),
                                           ctypes.byref(n)))
    return out[: n.value].tobytes()


# ---- client side (test only)
def gen_sk(rng, log2n):
    out = np.zeros(1 << log2n, dtype=np.int8)
    _check(lib().orc_gen_sk(rng._h, log2n, _ptr(out)))
    return out


def gen_gk_b(rng, log2n, sk):
    out = np.zeros((2, 1 << log2n), dtype=np.int64)
    _check(lib().orc_gen_gk_b(rng._h, log2n, _ptr(np.ascontiguousarray(sk, dtype=np.int8)), _ptr(out)))
    return out


def enc_sym_b(rng, log2n, apart_index, sk, m):
    out = np.zeros(1 << log2n, dtype=np.int64)
    mm = np.ascontiguousarray(m, dtype=np.int64)
    _check(lib().orc_enc_sym_b(rng._h, log2n, apart_index, _ptr(np.ascontiguousarray(sk, dtype=np.int8)),
                               _ptr(mm), _ptr(out)))
    return out


def dec(log2n, sk, a, b):
    out = np.zeros(1 << log2n, dtype=np.int64)
    _check(lib().orc_dec(log2n, _ptr(np.ascontiguousarray(sk, dtype=np.int8)),
                         _ptr(np.ascontiguousarray(a, dtype=np.int64)), _ptr(np.ascontiguousarray(b, dtype=np.int64)),
                         _ptr(out)))
    return out


def enc_double_pir(rng, log2n, l1, l2, sk, primary_idx, secondary_idx):
    n = 1 << log2n
    pq, pqc, sq, sqc = (np.zeros(n, dtype=np.int64) for _ in range(4))
    gk = np.zeros((2, n), dtype=np.int64)
    hp, hs = ctypes.c_int(), ctypes.c_int()
    _check(lib().orc_enc_double_pir(rng._h, log2n, l1, l2, _ptr(np.ascontiguousarray(sk, dtype=np.int8)),
                                    primary_idx, secondary_idx, _ptr(pq), _ptr(pqc), _ptr(sq), _ptr(sqc), _ptr(gk),
                                    ctypes.byref(hp), ctypes.byref(hs)))
    return pq, (pqc if hp.value else None), sq, (sqc if hs.value else None), gk


def dec_double_pir(log2n, sk, reply):
    out = np.zeros(1 << log2n, dtype=np.int64)
    r = np.ascontiguousarray(reply, dtype=np.int64)
    _check(lib().orc_dec_double_pir(log2n, _ptr(np.ascontiguousarray(sk, dtype=np.int8)), _ptr(r), _ptr(out)))
    return out


def prepare_query(rng, primary_idx, secondary_idx, l1, l2):
    """prepare_query_general (pir_wrapper.rs:276): returns (query bytes, sk seed)."""
    out = np.zeros(1 << 17, dtype=np.uint8)
    n = ctypes.c_uint64()
    seed = np.zeros(32, dtype=np.uint8)
    _check(lib().orc_prepare_query(rng._h, primary_idx, secondary_idx, l1, l2, _ptr(out), ctypes.byref(n),
                                   _ptr(seed)))
    return out[: n.value].tobytes(), seed.tobytes()


def process_reply(reply, sk_seed):
    """process_reply (pir_wrapper.rs:420): the N coefficients of the entry."""
    r = np.frombuffer(bytes(reply), dtype=np.uint8)
    out = np.zeros(N, dtype=np.int64)
    _check(lib().orc_process_reply(_ptr(r), len(r), bytes(sk_seed), _ptr(out)))
    return out


def reduce_after_mul(K, start, count):
    lazy = np.zeros(count, dtype=np.uint64)
    full = np.zeros(count, dtype=np.uint64)
    lib().orc_reduce_after_mul(K, start, count, _ptr(lazy), _ptr(full))
    return lazy, full


def scan_baseline(log2n, l, shards, threads, reps):
    """Times the restated main_pir_loop (AVX-512 where present); returns seconds per pass."""
    used = ctypes.c_int()
    t = lib().orc_scan_baseline(log2n, l, shards, threads, reps, ctypes.byref(used))
    return t, used.value


def time_secondary(log2n, l2):
    """Seconds of one oracle secondary phase (set_db + scan) at secondary order l2."""
    return lib().orc_time_secondary(log2n, l2)


def cpu_has_avx512():
    return bool(lib().orc_cpu_has_avx512())


class QueryBench:
    """One whole query answered on the CPU, timed for real: the AVX-512
    main_pir_loop restatement over every logical shard (distinct slabs in RAM
    reused as shard k mod distinct) plus the oracle's secondary phase."""

    def __init__(self, log2n, l1, l2, shards, distinct):
        self._h = ctypes.c_void_p(lib().orc_bench_new(log2n, l1, l2, shards, distinct))
        if not self._h.value:
            raise OracleError("out of host memory for the CPU bench slabs")

    def step(self, threads=0):
        """(scan seconds, secondary seconds, scan threads) of one query."""
        a, b, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        _check(lib().orc_bench_step(self._h, threads, ctypes.byref(a), ctypes.byref(b), ctypes.byref(t)))
        return a.value, b.value, t.value

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_bench_free(self._h)
            self._h = None

    __del__ = close
