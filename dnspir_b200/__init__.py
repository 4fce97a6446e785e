"""dnspir_b200 -- B200 (sm_100a) answer path of DNSPIR's two-level BFV PIR.

Python mirror of the server-side API of the reference's crates/pir, over the
C ABI of include/dnspir.h (libdnspir_b200.so, built in-tree by build.py):

    get_database_shape / num_databases     pir_wrapper.rs:219-241
    PIRDatabase (create, set_db, get_a,    base_pir.rs:229-1077
      perform_pir, perform_pir_split)
    Fleet.perform_double_pir               double_pir.rs:104-123
    Fleet.process_query / process_queries  pir_wrapper.rs:328-409

The product path is the CUDA library only.  Importing this package without the
built library, or using it without a CUDA device, raises; nothing here falls
back to a CPU implementation.
"""
import ctypes
import os

import numpy as np

__all__ = [
    "DnspirError", "lib", "get_database_shape", "num_databases", "required_memory_general",
    "choose_secondary_order", "expand_seed", "set_a_parts", "get_a_parts", "load_a_parts_file", "query_bytes", "prepare_query", "process_reply", "reply_bytes", "PIRDatabase", "Fleet", "pack_payloads",
    "LOG2_N", "N", "Q1", "Q2", "Q", "SIMD_COUNT", "PLAIN_MODULUS",
]

LOG2_N = 11
N = 1 << LOG2_N
Q1 = (1 << 26) - (1 << 12) + 1
Q2 = (1 << 25) - (1 << 12) + 1
Q = Q1 * Q2
SIMD_COUNT = 8
PLAIN_MODULUS = 1025

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdnspir_b200.so")

_ERRORS = {1: "BAD_SIZE", 2: "BAD_SHAPE", 3: "OOM", 4: "CUDA", 5: "TIMEOUT", 6: "BAD_ARG", 7: "NOT_READY"}


class DnspirError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"dnspir error {_ERRORS.get(code, code)}: {msg}")
        self.code = code


_lib = None
_vp = ctypes.c_void_p
_u32p = ctypes.POINTER(ctypes.c_uint32)
_u64p = ctypes.POINTER(ctypes.c_uint64)


def lib():
    """The loaded CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python dnspir_b200/build.py`")
        L = ctypes.CDLL(LIB_PATH)
        c = ctypes
        L.dnspir_last_error.restype = c.c_char_p
        L.dnspir_version.restype = c.c_char_p
        L.dnspir_get_database_shape.argtypes = [c.c_uint64, _u32p, _u32p, _u32p]
        L.dnspir_choose_secondary_order.argtypes = [c.c_uint32, _u32p]
        L.dnspir_required_memory_general.restype = c.c_uint64
        L.dnspir_required_memory_general.argtypes = [c.c_uint32, c.c_uint32]
        L.dnspir_query_bytes.restype = c.c_uint64
        L.dnspir_query_bytes.argtypes = [c.c_uint32, c.c_uint32]
        L.dnspir_reply_bytes.restype = c.c_uint64
        L.dnspir_db_create.argtypes = [c.c_int, c.c_uint32, c.c_uint32, c.c_int, c.POINTER(_vp)]
        L.dnspir_db_set_db.argtypes = [_vp, _vp, c.c_uint64, c.c_int]
        L.dnspir_db_get_a.argtypes = [_vp, _vp]
        L.dnspir_db_perform_pir_split.argtypes = [_vp, _vp, _vp, _vp, _vp]
        L.dnspir_db_destroy.argtypes = [_vp]
        L.dnspir_db_perform_pir_split_noalloc.argtypes = [_vp] * 6
        L.dnspir_fleet_create.argtypes = [c.c_int, c.c_uint64, c.c_uint32, c.POINTER(_vp)]
        L.dnspir_fleet_create_general.argtypes = [c.c_int, c.c_uint32, c.c_uint32, c.c_uint32, c.c_uint32,
                                                  c.c_uint32, c.POINTER(_vp)]
        L.dnspir_fleet_set_shards.argtypes = [_vp, c.c_uint32, c.c_uint32, _vp, c.c_int]
        L.dnspir_expand_seed.argtypes = [c.c_uint32, c.c_int, _vp]
        L.dnspir_set_a_parts.argtypes = [c.c_uint32, _vp]
        L.dnspir_get_a_parts.argtypes = [c.c_uint32, _vp]
        L.dnspir_pack_payloads.argtypes = [c.c_int, _vp, c.c_uint64, _vp]
        L.dnspir_fleet_process_queries.argtypes = [_vp, _vp, _vp, c.c_uint32, _vp, c.c_uint64, _vp, c.c_int]
        L.dnspir_fleet_process_query.argtypes = [_vp, _vp, c.c_uint64, _vp, _u64p]
        L.dnspir_fleet_perform_double_pir.argtypes = [_vp] * 7
        L.dnspir_fleet_last_timings.argtypes = [_vp] + [c.POINTER(c.c_double)] * 3
        L.dnspir_fleet_set_stream.argtypes = [_vp, _vp]
        L.dnspir_fleet_set_batch.argtypes = [_vp, c.c_uint32]
        L.dnspir_fleet_set_engine.argtypes = [_vp, c.c_int]
        L.dnspir_fleet_tune.argtypes = [_vp, c.c_uint32, _vp, _vp]
        L.dnspir_tscan_shapes.argtypes = [_vp, _vp, _vp, _vp, c.c_int]
        L.dnspir_fleet_scan.argtypes = [_vp, _vp, c.c_uint32, _vp]
        L.dnspir_fleet_set_tile.argtypes = [_vp, c.c_uint32, c.c_int]
        L.dnspir_fleet_set_schedule.argtypes = [_vp, c.c_uint32, c.c_int]
        L.dnspir_fleet_get_schedule.argtypes = [_vp, c.c_uint32, _vp]
        L.dnspir_fleet_tune_pipeline.argtypes = [_vp, c.c_uint32, _vp, _vp]
        L.dnspir_fleet_tune_cuda_cores.argtypes = [_vp, c.c_uint32, _vp, _vp]
        L.dnspir_fleet_set_wait_limit.argtypes = [_vp, c.c_uint64, c.c_int]
        L.dnspir_server_create.argtypes = [c.c_int, c.c_uint32, c.POINTER(_vp)]
        L.dnspir_server_add_db.argtypes = [_vp, _vp, c.c_uint32, _u32p]
        L.dnspir_server_start.argtypes = [_vp, c.c_int]
        L.dnspir_server_set_batching.argtypes = [_vp, c.c_uint32, c.c_uint32, c.c_uint32]
        L.dnspir_server_open_session.argtypes = [_vp, c.c_char_p, c.c_uint64, _u64p]
        L.dnspir_server_close_session.argtypes = [_vp, c.c_uint64]
        L.dnspir_server_submit.argtypes = [_vp, c.c_uint32, c.c_int64, c.c_char_p, c.c_uint64, _u64p]
        L.dnspir_server_poll.argtypes = [_vp, c.c_uint64, _vp, c.c_uint64, c.POINTER(c.c_int)]
        L.dnspir_server_wait.argtypes = [_vp, c.c_uint64, _vp, c.c_uint64, c.c_uint32]
        L.dnspir_server_db_stats.argtypes = [_vp, c.c_uint32, _u64p, _u32p, _u64p, _u64p, _vp, c.c_uint32, _u32p]
        L.dnspir_server_stop.argtypes = [_vp]
        L.dnspir_server_destroy.argtypes = [_vp]
        L.dnspir_fleet_batch_timings.argtypes = [_vp, c.c_uint32] + [_vp] * 4
        L.dnspir_fleet_launch_count.argtypes = [_vp, _u64p]
        L.dnspir_fleet_slab_bytes.restype = c.c_uint64
        L.dnspir_fleet_slab_bytes.argtypes = [_vp]
        L.dnspir_fleet_destroy.argtypes = [_vp]
        L.dnspir_client_prepare_query.argtypes = [c.c_char_p, c.c_uint64, c.c_uint64, c.c_uint32, c.c_uint32, _vp,
                                                  _u64p, _vp]
        L.dnspir_client_process_reply.argtypes = [_vp, c.c_uint64, c.c_char_p, _vp]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise DnspirError(rc, lib().dnspir_last_error().decode())


def _ptr(a):
    return a.ctypes.data_as(_vp)


def _dev_ptr(t):
    return _vp(int(t.data_ptr()))


def _is_cuda_tensor(x):
    return hasattr(x, "is_cuda") and x.is_cuda


def get_database_shape(num_entries):
    """(primary group order, secondary group order, number of shards) -- pir_wrapper.rs:219."""
    a, b, s = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
    _check(lib().dnspir_get_database_shape(num_entries, ctypes.byref(a), ctypes.byref(b), ctypes.byref(s)))
    return a.value, b.value, s.value


def num_databases(num_entries):
    """pir_wrapper.rs:238."""
    return get_database_shape(num_entries)[2]


def choose_secondary_order(num_shards):
    v = ctypes.c_uint32()
    _check(lib().dnspir_choose_secondary_order(num_shards, ctypes.byref(v)))
    return v.value


def required_memory_general(log2_n, group_order):
    """base_pir.rs:369 (in 32-byte elements)."""
    return lib().dnspir_required_memory_general(log2_n, group_order)


def query_bytes(primary_order, secondary_order):
    return lib().dnspir_query_bytes(primary_order, secondary_order)


def reply_bytes():
    return lib().dnspir_reply_bytes()


def expand_seed(log2_n, which):
    """expand (bfv.rs:46) of SEEDS[which] (base_pir.rs:64): N coefficients in [0, q)."""
    out = np.zeros(1 << log2_n, dtype=np.uint64)
    _check(lib().dnspir_expand_seed(log2_n, which, _ptr(out)))
    return out


def set_a_parts(log2_n, parts):
    """Install the six a-parts of ring dimension 2^log2_n process-wide
    ((6, N) coefficients in [0, q): gk0, gk1, FirstSet query and conjugate,
    SecondSet query and conjugate -- bfv.rs:46-49, base_pir.rs:104-107), or
    restore the seed expansion with parts=None.  Shards preprocessed before
    must be set again."""
    if parts is None:
        _check(lib().dnspir_set_a_parts(log2_n, None))
        return
    a = np.ascontiguousarray(parts, dtype=np.uint64)
    assert a.shape == (6, 1 << log2_n)
    _check(lib().dnspir_set_a_parts(log2_n, _ptr(a)))


def get_a_parts(log2_n):
    """The six a-parts in effect, (6, N) uint64."""
    out = np.zeros((6, 1 << log2_n), dtype=np.uint64)
    _check(lib().dnspir_get_a_parts(log2_n, _ptr(out)))
    return out


def load_a_parts_file(path, log2_n=LOG2_N):
    """Install a-parts from a file: a .npy array of shape (6, N), or raw
    little-endian uint64 (6 x N values)."""
    if str(path).endswith(".npy"):
        parts = np.load(path)
    else:
        parts = np.fromfile(path, dtype="<u8").reshape(6, 1 << log2_n)
    set_a_parts(log2_n, parts)


def pack_payloads(payload, out, device=0):
    """pack_bytes_into_coeffs (dns/bucket.rs:289) on the device: uint8 (E, 2560) -> uint16 (E, 2048)."""
    _check(lib().dnspir_pack_payloads(device, _dev_ptr(payload), payload.shape[0], _dev_ptr(out)))


def prepare_query(rng_seed, primary_idx, secondary_idx, primary_order, secondary_order):
    """Client side, pir_wrapper.rs:276: (query bytes, 32-byte secret-key seed)."""
    out = np.zeros(1 << 17, dtype=np.uint8)
    n = ctypes.c_uint64()
    sk = np.zeros(32, dtype=np.uint8)
    rc = lib().dnspir_client_prepare_query(bytes(rng_seed), primary_idx, secondary_idx, primary_order,
                                           secondary_order, _ptr(out), ctypes.byref(n), _ptr(sk))
    if rc:
        raise DnspirError(rc, "prepare_query: bad shape or index")
    return out[: n.value].tobytes(), sk.tobytes()


def process_reply(reply, sk_seed):
    """Client side, pir_wrapper.rs:420: the N coefficients of the entry (uint16)."""
    r = np.frombuffer(bytes(reply), dtype=np.uint8)
    out = np.zeros(N, dtype=np.uint16)
    rc = lib().dnspir_client_process_reply(_ptr(r), len(r), bytes(sk_seed), _ptr(out))
    if rc:
        raise DnspirError(rc, "process_reply: malformed reply")
    return out


def _zq(a, shape):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    if a.shape != shape:
        a = np.ascontiguousarray(np.broadcast_to(a, shape), dtype=np.uint64)
    return a


class PIRDatabase:
    """One preprocessed shard on the GPU (base_pir.rs:229)."""

    def __init__(self, log2_n, group_order, used_seeds=0, device=0):
        h = _vp()
        _check(lib().dnspir_db_create(device, log2_n, group_order, used_seeds, ctypes.byref(h)))
        self._h = h
        self.log2_n = log2_n
        self.n = 1 << log2_n
        self.group_order = group_order
        self.requires_conj = group_order == self.n

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.dnspir_db_destroy(self._h)
            self._h = None

    __del__ = close

    def set_db(self, entries):
        """entries: (8 l, N) plaintext coefficients in [0, 1025), numpy or a CUDA uint16 tensor."""
        want = (8 * self.group_order, self.n)
        if _is_cuda_tensor(entries):
            assert tuple(entries.shape) == want and entries.is_contiguous()
            _check(lib().dnspir_db_set_db(self._h, _dev_ptr(entries), entries.numel(), 1))
        else:
            e = np.ascontiguousarray(entries, dtype=np.uint16)
            _check(lib().dnspir_db_set_db(self._h, _ptr(e), e.size, 0))

    def get_a(self):
        out = np.zeros((8, self.n), dtype=np.uint64)
        _check(lib().dnspir_db_get_a(self._h, _ptr(out)))
        return out

    def perform_pir_split(self, qry_b, qry_conj_b, gk_b):
        n = self.n
        qb = _zq(qry_b, (8, n))
        qc = None if qry_conj_b is None else _zq(qry_conj_b, (8, n))
        gk = _zq(gk_b, (8, 2, n))
        out = np.zeros((8, n), dtype=np.uint64)
        _check(lib().dnspir_db_perform_pir_split(self._h, _ptr(qb), None if qc is None else _ptr(qc), _ptr(gk),
                                                 _ptr(out)))
        return out

    def perform_pir(self, qry_b, qry_conj_b, gk_b):
        """base_pir.rs:945: the same query on all 8 lanes."""
        n = self.n
        return self.perform_pir_split(_zq(qry_b, (8, n)), None if qry_conj_b is None else _zq(qry_conj_b, (8, n)),
                                      _zq(np.asarray(gk_b, dtype=np.uint64)[None], (8, 2, n)))


ENGINE_CUDA_CORES = 0
ENGINE_TENSOR = 1


def tscan_shapes():
    """The tensor scan's tile shapes: (query-operand rows, m-tiles, stages,
    kernel) per CTA; kernel 0 is one tile per CTA, 1 the persistent
    warp-specialised kernel, 2 and 3 the CTA pair (relayed bulk copies,
    tensor-map copies)."""
    n = lib().dnspir_tscan_shapes(None, None, None, None, 0)
    a = [np.zeros(n, dtype=np.int32) for _ in range(4)]
    lib().dnspir_tscan_shapes(*[_ptr(x) for x in a], n)
    return [tuple(int(x[i]) for x in a) for i in range(n)]


class Fleet:
    """The primary shards of one database plus the two-level answer path.

    Fleet(num_entries, num_distinct) follows get_database_shape (N = 2048);
    Fleet.general(log2_n, l1, l2, shards, distinct) takes the shape explicitly.
    Logical shard k is served by distinct shard k % num_distinct.
    """

    def __init__(self, num_entries=None, num_distinct=None, device=0, _shape=None):
        h = _vp()
        if _shape is None:
            l1, l2, s = get_database_shape(num_entries)
            d = s if num_distinct is None else num_distinct
            _check(lib().dnspir_fleet_create(device, num_entries, d, ctypes.byref(h)))
            self.log2_n, self.primary_order, self.secondary_order, self.num_shards, self.num_distinct = \
                LOG2_N, l1, l2, s, d
        else:
            log2_n, l1, l2, s, d = _shape
            _check(lib().dnspir_fleet_create_general(device, log2_n, l1, l2, s, d, ctypes.byref(h)))
            self.log2_n, self.primary_order, self.secondary_order, self.num_shards, self.num_distinct = _shape
        self._h = h
        self.device = device
        self.n = 1 << self.log2_n

    @classmethod
    def general(cls, log2_n, primary_order, secondary_order, num_shards, num_distinct=None, device=0):
        return cls(device=device, _shape=(log2_n, primary_order, secondary_order, num_shards,
                                          num_shards if num_distinct is None else num_distinct))

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.dnspir_fleet_destroy(self._h)
            self._h = None

    __del__ = close

    @property
    def entries_per_shard(self):
        return 8 * self.primary_order

    @property
    def query_len(self):
        return query_bytes(self.primary_order, self.secondary_order)

    def set_shards(self, first, entries):
        """entries: (count, 8 l, N) coefficients; numpy (host) or a CUDA uint16 tensor."""
        per = (8 * self.primary_order, self.n)
        if _is_cuda_tensor(entries):
            assert tuple(entries.shape[1:]) == per and entries.is_contiguous()
            _check(lib().dnspir_fleet_set_shards(self._h, first, entries.shape[0], _dev_ptr(entries), 1))
        else:
            e = np.ascontiguousarray(entries, dtype=np.uint16)
            if e.ndim == 2:
                e = e[None]
            assert e.shape[1:] == per
            _check(lib().dnspir_fleet_set_shards(self._h, first, e.shape[0], _ptr(e), 0))

    def process_queries(self, queries):
        """pir_wrapper.rs:349: list of query bytes -> list of reply bytes."""
        nq = len(queries)
        bufs = [np.frombuffer(bytes(q), dtype=np.uint8) for q in queries]
        ptrs = (_vp * nq)(*[b.ctypes.data for b in bufs])
        lens = (ctypes.c_uint64 * nq)(*[len(b) for b in bufs])
        rb = reply_bytes()
        out = np.zeros((nq, rb), dtype=np.uint8)
        status = np.zeros(nq, dtype=np.int32)
        _check(lib().dnspir_fleet_process_queries(self._h, ptrs, lens, nq, _ptr(out), rb, _ptr(status), 0))
        return [out[i].tobytes() for i in range(nq)]

    def process_query(self, query):
        """pir_wrapper.rs:328."""
        return self.process_queries([query])[0]

    def process_queries_device(self, queries, replies):
        """Device-resident variant: queries (nq, qlen) and replies (nq, reply_bytes) CUDA uint8 tensors."""
        nq = queries.shape[0]
        base = int(queries.data_ptr())
        stride = queries.stride(0)
        ptrs = (_vp * nq)(*[base + i * stride for i in range(nq)])
        lens = (ctypes.c_uint64 * nq)(*([queries.shape[1]] * nq))
        status = np.zeros(nq, dtype=np.int32)
        _check(lib().dnspir_fleet_process_queries(self._h, ptrs, lens, nq, _dev_ptr(replies), replies.stride(0),
                                                  _ptr(status), 1))

    def perform_double_pir(self, pq, pqc, sq, sqc, gk):
        """double_pir.rs:104: ring elements in, three (a, b) ciphertexts (3, 2, N) out."""
        n = self.n
        args = [None if x is None else _zq(x, s) for x, s in
                ((pq, (n,)), (pqc, (n,)), (sq, (n,)), (sqc, (n,)), (gk, (2, n)))]
        out = np.zeros((3, 2, n), dtype=np.uint64)
        _check(lib().dnspir_fleet_perform_double_pir(self._h, *[None if a is None else _ptr(a) for a in args],
                                                     _ptr(out)))
        return out

    def last_timings(self):
        """(primary ms, secondary ms, scan ms) of the last answered query (CUDA events)."""
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(lib().dnspir_fleet_last_timings(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def batch_timings(self, max_queries=1 << 16):
        """Per-query (latency, primary, secondary, scan) ms of the last call, from CUDA events."""
        out = np.full((4, max_queries), -1.0)
        n = lib().dnspir_fleet_batch_timings(self._h, max_queries, *[_ptr(out[i]) for i in range(4)])
        if n < 0:
            _check(-n)
        return out[:, :n]

    def set_batch(self, max_batch):
        """Queries per pass over the slabs (CUDA cores: a power of two up to 256; tensor
        cores: 1..256); replies do not depend on it."""
        _check(lib().dnspir_fleet_set_batch(self._h, max_batch))

    def scan(self, qnat, out):
        """Primary scan alone (torch cuda tensors): qnat uint32-as-int32
        [nq][6][2][N] natural NTT order, out [nq][shards][2][N][8]."""
        _check(lib().dnspir_fleet_scan(self._h, _dev_ptr(qnat), qnat.shape[0], _dev_ptr(out)))

    def set_tile(self, batch, shape_index):
        """Tensor engine: tile shape index for groups of `batch` (-1: default)."""
        _check(lib().dnspir_fleet_set_tile(self._h, batch, shape_index))

    def set_schedule(self, batch, schedule):
        """How groups of `batch` follow the previous group: 0 overlap its
        secondary phase, 1 wait for all of it, 2 wait for its last chunk to
        start; plus 4 for two-block-cluster chains at every chunk size; -1 the
        default."""
        _check(lib().dnspir_fleet_set_schedule(self._h, batch, schedule))

    def get_schedule(self, batch):
        """The schedule in force for groups of `batch` (set_schedule's encoding)."""
        s = ctypes.c_int()
        _check(lib().dnspir_fleet_get_schedule(self._h, batch, ctypes.byref(s)))
        return s.value

    def set_wait_limit(self, wait_ns=0, withhold_chunk=-1):
        """Tensor engine: limit of the scan's pipeline waits (0: default 2 s);
        withhold_chunk >= 0 is the timeout path's test hook."""
        _check(lib().dnspir_fleet_set_wait_limit(self._h, wait_ns, withhold_chunk))

    def set_engine(self, engine):
        """ENGINE_CUDA_CORES or ENGINE_TENSOR; marks every shard unprepared."""
        _check(lib().dnspir_fleet_set_engine(self._h, engine))
        self._engine = engine

    def tune_cuda_cores(self, batch):
        """CUDA-core engine: time 1, 2, 4, 8, 16 queries per block for groups of
        `batch` and keep the fastest.  Returns (queries per block, ms per tile)."""
        ms = np.full(5, -1.0)
        chosen = ctypes.c_int(-1)
        _check(lib().dnspir_fleet_tune_cuda_cores(self._h, batch, _ptr(ms), ctypes.byref(chosen)))
        return chosen.value, ms

    def tune(self, batch, pipeline=False):
        """Tensor engine: time each tile shape for groups of `batch` queries and
        keep the fastest (pipeline=True: whole groups through both phases
        instead of the scan alone).  Returns (chosen index, ms per shape, shapes)."""
        shapes = tscan_shapes()
        ms = np.full(len(shapes), -1.0)
        chosen = ctypes.c_int(-1)
        fn = lib().dnspir_fleet_tune_pipeline if pipeline else lib().dnspir_fleet_tune
        _check(fn(self._h, batch, _ptr(ms), ctypes.byref(chosen)))
        return chosen.value, ms, shapes

    def set_stream(self, stream_handle):
        _check(lib().dnspir_fleet_set_stream(self._h, _vp(stream_handle) if stream_handle else None))

    def launch_count(self):
        """Kernels the answer pipeline has launched so far."""
        v = ctypes.c_uint64()
        _check(lib().dnspir_fleet_launch_count(self._h, ctypes.byref(v)))
        return v.value

    @property
    def slab_bytes(self):
        return lib().dnspir_fleet_slab_bytes(self._h)


GALOIS_KEY_BYTES = 2 * N * 50 // 8


class Server:
    """Serving loop over resident fleets (continuous batching, CUDA graphs,
    device-resident client sessions).  Fleets stay attached until stop()."""

    def __init__(self, max_sessions=0, device=0):
        h = _vp()
        _check(lib().dnspir_server_create(device, max_sessions, ctypes.byref(h)))
        self._h = h
        self._fleets = []

    def add_db(self, fleet, max_batch):
        i = ctypes.c_uint32()
        _check(lib().dnspir_server_add_db(self._h, fleet._h, max_batch, ctypes.byref(i)))
        self._fleets.append(fleet)
        return i.value

    def set_batching(self, db, min_batch, max_wait_ms):
        """Hold a database's group until min_batch queries are pending or the
        oldest has waited max_wait_ms."""
        _check(lib().dnspir_server_set_batching(self._h, db, min_batch, int(max_wait_ms * 1000)))

    def start(self, graphs=True):
        _check(lib().dnspir_server_start(self._h, 1 if graphs else 0))

    def open_session(self, galois_key_bytes):
        s = ctypes.c_uint64()
        b = bytes(galois_key_bytes)
        _check(lib().dnspir_server_open_session(self._h, b, len(b), ctypes.byref(s)))
        return s.value

    def close_session(self, session):
        _check(lib().dnspir_server_close_session(self._h, session))

    def submit(self, db, query, session=-1):
        t = ctypes.c_uint64()
        b = bytes(query)
        _check(lib().dnspir_server_submit(self._h, db, session, b, len(b), ctypes.byref(t)))
        return t.value

    def poll(self, ticket):
        out = np.zeros(reply_bytes(), dtype=np.uint8)
        done = ctypes.c_int()
        _check(lib().dnspir_server_poll(self._h, ticket, _ptr(out), out.size, ctypes.byref(done)))
        return out.tobytes() if done.value else None

    def wait(self, ticket, timeout_ms=120000):
        out = np.zeros(reply_bytes(), dtype=np.uint8)
        _check(lib().dnspir_server_wait(self._h, ticket, _ptr(out), out.size, timeout_ms))
        return out.tobytes()

    def stats(self, db, max_latencies=1 << 20):
        comp, adm, grp, ggrp, n = (ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint64(),
                                   ctypes.c_uint32())
        lat = np.zeros(max_latencies)
        _check(lib().dnspir_server_db_stats(self._h, db, ctypes.byref(comp), ctypes.byref(adm), ctypes.byref(grp),
                                            ctypes.byref(ggrp), _ptr(lat), max_latencies, ctypes.byref(n)))
        return {"completed": comp.value, "admitted_batch": adm.value, "groups": grp.value,
                "graph_groups": ggrp.value, "latencies_ms": lat[:n.value].copy()}

    def stop(self):
        if getattr(self, "_h", None):
            _check(lib().dnspir_server_stop(self._h))

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.dnspir_server_destroy(self._h)
            self._h = None
            self._fleets = []

    __del__ = close
