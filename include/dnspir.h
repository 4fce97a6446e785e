/* dnspir.h -- C ABI of the B200 answer path of DNSPIR's two-level BFV PIR.
 *
 * Drop-in boundary for the server side of FeanorTheElf/dnspir's crates/pir:
 * the functions below replace the reference calls cited beside each one
 * (paths relative to crates/pir/src/).  Plain pointers and sizes only; every
 * function returns a status code (DNSPIR_OK = 0) and never aborts; the
 * message of the last failure on the calling thread is dnspir_last_error().
 * Host buffers belong to the caller, device memory to the library.  There is
 * no CPU fallback: without a CUDA device every constructor fails with
 * DNSPIR_ERR_CUDA.
 *
 * Ring elements cross the boundary as N coefficients in [0, q), q = q1 q2,
 * q1 = 2^26 - 2^12 + 1, q2 = 2^25 - 2^12 + 1 (base_pir.rs:75-77), uint64 each.
 * Plaintext entries are N coefficients in [0, 1025) (uint16), entry e of a
 * database of group order l being element e of its 8 l entries (set_db order,
 * base_pir.rs:612-637).
 */
#ifndef DNSPIR_H
#define DNSPIR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  DNSPIR_OK = 0,
  DNSPIR_ERR_BAD_SIZE = 1,  /* byte or entry count wrong: uncondense "not enough data" (pir_wrapper.rs:124), set_db length (base_pir.rs:693) */
  DNSPIR_ERR_BAD_SHAPE = 2, /* invalid group order / entry count / conjugate presence (base_pir.rs:150-154, pir_wrapper.rs:221-222, double_pir.rs:160) */
  DNSPIR_ERR_OOM = 3,       /* device memory exhausted */
  DNSPIR_ERR_CUDA = 4,      /* CUDA runtime error or no device */
  DNSPIR_ERR_TIMEOUT = 5,   /* a bounded wait gave up */
  DNSPIR_ERR_BAD_ARG = 6,   /* null pointer, index out of range, value not reduced */
  DNSPIR_ERR_NOT_READY = 7  /* shard used before it was preprocessed */
};

const char* dnspir_last_error(void);
const char* dnspir_version(void);

/* ---- shape rules ------------------------------------------------------- */

/* get_database_shape + num_databases (pir_wrapper.rs:219-241): group orders of
 * the primary and secondary databases and the number of primary shards for a
 * database of num_entries plaintext entries (N = 2048). */
int dnspir_get_database_shape(uint64_t num_entries, uint32_t* primary_order, uint32_t* secondary_order,
                              uint32_t* num_shards);
/* choose_index_group_secondary (pir_wrapper.rs:166-175) */
int dnspir_choose_secondary_order(uint32_t num_shards, uint32_t* secondary_order);
/* PIRDatabase::required_memory_general (base_pir.rs:369-371), in 32-byte elements */
uint64_t dnspir_required_memory_general(uint32_t log2_n, uint32_t group_order);
/* byte length of a query (prepare_query_general output, pir_wrapper.rs:304-316) and of a reply (:401-408) */
uint64_t dnspir_query_bytes(uint32_t primary_order, uint32_t secondary_order);
uint64_t dnspir_reply_bytes(void);

/* expand (bfv.rs:46-49) of SEEDS[which] (base_pir.rs:64-71) for ring dimension
 * 2^log2_n: out = N coefficients in [0, q).  Host only; needs no device.
 * Coefficient i is drawn in order i = 0..N-1 from the StdRng (ChaCha12) stream
 * keyed by the seed: the low ceil(log2 q) = 51 bits of one next_u64, drawn
 * again while >= q (the uniform-below-bound rule that feanor-math's
 * random_element applies per coefficient, as this library restates it). */
int dnspir_expand_seed(uint32_t log2_n, int which, uint64_t* out);
/* The six a-parts of ring dimension 2^log2_n, process-wide: the fixed `a`
 * polynomials every query ciphertext and Galois key shares (bfv.rs:46-49 via
 * UsedSeeds, base_pir.rs:104-107, 193-205; computed once in
 * PIRDatabase::create / preprocess, base_pir.rs:782-789).  coeffs = 6 x N
 * values in [0, q) in the order gk0, gk1, FirstSet query, FirstSet conjugate
 * query, SecondSet query, SecondSet conjugate query; NULL restores the seed
 * expansion (dnspir_expand_seed of SEEDS[0..5]).  This is the hook for a-parts
 * produced by the reference itself: with them installed, reply bytes are
 * comparable with the reference's.  Databases and fleets preprocessed under
 * other a-parts answer DNSPIR_ERR_NOT_READY until their set_db / set_shards
 * runs again; do not call it while a call on a database of that dimension is
 * running.  The client calls (dnspir_client_*) use the same a-parts. */
int dnspir_set_a_parts(uint32_t log2_n, const uint64_t* coeffs);
/* The six a-parts in effect for ring dimension 2^log2_n (6 x N coefficients,
 * order as dnspir_set_a_parts). */
int dnspir_get_a_parts(uint32_t log2_n, uint64_t* out);

/* ---- one preprocessed shard: PIRDatabase (base_pir.rs:229-255) --------- */

typedef struct dnspir_db dnspir_db;

/* PIRDatabase::create (base_pir.rs:280): used_seeds 0 = FirstSet, 1 = SecondSet
 * (:104-107); the slab is allocated on `device`. */
int dnspir_db_create(int device, uint32_t log2_n, uint32_t group_order, int used_seeds, dnspir_db** out);
/* PIRDatabase::set_db (base_pir.rs:632): count must equal 8 * group_order * N
 * coefficients; entries_on_device != 0 if `entries` is a device pointer. */
int dnspir_db_set_db(dnspir_db* db, const uint16_t* entries, uint64_t count, int entries_on_device);
/* PIRDatabase::get_a (base_pir.rs:897): out = 8 x N coefficients */
int dnspir_db_get_a(dnspir_db* db, uint64_t* out);
/* PIRDatabase::perform_pir_split (base_pir.rs:958): lane k answers query k.
 * qry_b: 8 x N, qry_conj_b: 8 x N (NULL iff group_order < N), gk_b: 8 x 2 x N,
 * out_b: 8 x N. */
int dnspir_db_perform_pir_split(dnspir_db* db, const uint64_t* qry_b, const uint64_t* qry_conj_b,
                                const uint64_t* gk_b, uint64_t* out_b);
int dnspir_db_destroy(dnspir_db* db);
/* No counterpart in the reference.  The same answer as
 * dnspir_db_perform_pir_split for callers that cannot allocate device memory
 * while answering (HBM fully committed to shard slabs; request paths that must
 * not call cudaMalloc, which can fail and synchronizes the device).  All five
 * arrays are DEVICE pointers with the layouts of dnspir_db_perform_pir_split;
 * coefficients must already be below q (not checked).  Work is queued on
 * cuda_stream (NULL = the default stream) and the call returns without waiting.
 * Intermediates live in a static 5 MiB region of device memory; nothing is
 * allocated.  The region (and the kernels this call launches) is loaded on a
 * device by the first dnspir_db_create there, which also looks its address up,
 * and the device holds it until exit.  Calls on one device share the region:
 * calls whose work overlaps on the GPU race.  dnspir_db_set_db and
 * dnspir_db_destroy wait for the work of earlier calls on their shard. */
int dnspir_db_perform_pir_split_noalloc(dnspir_db* db, const uint64_t* qry_b, const uint64_t* qry_conj_b,
                                        const uint64_t* gk_b, uint64_t* out_b, void* cuda_stream);

/* ---- a fleet of primary shards and the two-level answer ---------------- */

typedef struct dnspir_fleet dnspir_fleet;

/* A fleet laid out by get_database_shape(num_entries) (N = 2048).  Only
 * num_distinct shard slabs are stored; logical shard k is served by distinct
 * shard k % num_distinct, as bench_wrapped_pir's preprocessed-db-count does
 * (pir_wrapper.rs:578). */
int dnspir_fleet_create(int device, uint64_t num_entries, uint32_t num_distinct, dnspir_fleet** out);
/* The same with explicit shape (any N = 2^log2_n, 3 <= log2_n <= 11), as the
 * reference's perform_double_pir tests use (double_pir.rs:328-451). */
int dnspir_fleet_create_general(int device, uint32_t log2_n, uint32_t primary_order, uint32_t secondary_order,
                                uint32_t num_shards, uint32_t num_distinct, dnspir_fleet** out);
/* set_db of `count` distinct shards starting at first_distinct (base_pir.rs:632;
 * dns/server.rs:707-728).  entries: count x (8 primary_order N) coefficients. */
int dnspir_fleet_set_shards(dnspir_fleet* fleet, uint32_t first_distinct, uint32_t count, const uint16_t* entries,
                            int entries_on_device);
/* Queries answered per pass over the shard slabs (default 1): a power of two up
 * to 256 on the CUDA-core engine, 1..256 on the tensor engine.
 * dnspir_fleet_process_queries splits its queries into groups of this size;
 * every group reads each slab once.  Replies do not depend on it.  The
 * reference answers one query per pass (process_queries, pir_wrapper.rs:349
 * takes at most two, one per database); batching has no counterpart there. */
int dnspir_fleet_set_batch(dnspir_fleet* fleet, uint32_t max_batch);

/* Scan engine of a fleet.  CUDA_CORES (default): the slab in lane layout, 64-bit
 * multiply-accumulate per 32-bit residue.  TENSOR: the slab re-indexed by query
 * slot and stored as 8-bit limbs in tensor-core tiles; the scan is an exact
 * u8 x u8 -> s32 product on the tensor cores (needs loop_len = N/2, N >= 256).
 * Replies are identical.  Changing the engine marks every shard unprepared
 * (call dnspir_fleet_set_shards again) and resets the batch to 1.  Both replace
 * main_pir_loop (base_pir.rs:1085-1247); the engine choice has no counterpart
 * in the reference. */
#define DNSPIR_ENGINE_CUDA_CORES 0
#define DNSPIR_ENGINE_TENSOR 1
int dnspir_fleet_set_engine(dnspir_fleet* fleet, int engine);
/* Tensor engine: time every tile shape for groups of `batch` queries on the
 * fleet's own shards and keep the fastest for that group size.
 * ms_per_shape[dnspir_tscan_shapes()] receives each shape's scan time (-1 when
 * not run); *chosen its index.  No counterpart in the reference. */
int dnspir_fleet_tune(dnspir_fleet* fleet, uint32_t batch, double* ms_per_shape, int* chosen);
/* The primary scan alone: the main_pir_loop outputs (base_pir.rs:1085-1247,
 * reduced) of every shard for nq queries, in groups of the fleet's batch.
 * Device pointers.  qnat: per query [slot 0 gk0, 1 gk1, 2 query, 3 conjugate
 * query, 4, 5 unused][factor q1, q2][N] residues in natural NTT order (slot k
 * = evaluation at zeta^-(2k+1)); out: [query][shard][factor][slot u][lane]
 * with slot u = (sign, e) for 2k+1 = +-5^e mod 2N, u = sign * N/2 + e. */
int dnspir_fleet_scan(dnspir_fleet* fleet, const uint32_t* qnat, uint32_t nq, uint32_t* out);
/* The same, timing whole groups (decode, scan, epilogue, secondary phase,
 * replies; zero query bytes, two timed groups after one warm-up) instead of
 * the scan alone: the shape that maximises responses/s when the secondary
 * phase of one group overlaps the scan of the next.  ms_per_shape receives
 * milliseconds per group.  The schedule is tuned too: the three fastest shapes
 * are timed again with each group's primary phase waiting for the previous
 * group's secondary phase, and again waiting only until that phase starts its
 * last chunk; the fastest shape and schedule are kept for the group size, and
 * then the two-block-cluster form of the secondary chains is tried at every
 * chunk size (kept when faster; dnspir_fleet_set_schedule's +4). */
int dnspir_fleet_tune_pipeline(dnspir_fleet* fleet, uint32_t batch, double* ms_per_shape, int* chosen);
/* CUDA-core engine: time the scan of a group of `batch` queries (a power of two
 * up to 256, one launch) with 1, 2, 4, 8 and 16 queries per block and keep the
 * fastest; ms_per_tile[5] receives the times (-1 when not run), *chosen the
 * queries per block.  No counterpart in the reference. */
int dnspir_fleet_tune_cuda_cores(dnspir_fleet* fleet, uint32_t batch, double* ms_per_tile, int* chosen);
/* How a group of `batch` queries follows the previous group, overriding the
 * default or a previous tune: 0 its primary phase overlaps the previous
 * group's secondary phase, 1 it waits for all of that phase, 2 it waits until
 * that phase starts its last chunk; plus 4: its secondary chains run as
 * two-block clusters (one RNS factor per block) at every chunk size instead of
 * one block per part beyond one wave.  -1 returns to the default (0).  Either
 * engine.  No counterpart in the reference. */
int dnspir_fleet_set_schedule(dnspir_fleet* fleet, uint32_t batch, int schedule);
/* The schedule in force for groups of `batch` queries, in the encoding of
 * dnspir_fleet_set_schedule (what the pipeline tuner chose, or the default 0).
 * No counterpart in the reference. */
int dnspir_fleet_get_schedule(dnspir_fleet* fleet, uint32_t batch, int* schedule);
/* Tensor engine: use tile shape `shape_index` (dnspir_tscan_shapes order) for
 * groups of `batch` queries, overriding the table or a previous tune; -1
 * returns to the default.  No counterpart in the reference. */
int dnspir_fleet_set_tile(dnspir_fleet* fleet, uint32_t batch, int shape_index);
/* Tensor engine: limit of every wait in the scan's copy/MMA/epilogue pipeline
 * (wait_ns; 0 restores the default of 2 s).  A wait that runs out makes the
 * scan's blocks stop, wait (bounded) for their copies in flight, free their
 * tensor memory and return; the call then fails with DNSPIR_ERR_TIMEOUT and
 * the device stays usable.  withhold_chunk >= 0 is a test hook for that path:
 * the first block's producer stops before copying that chunk, so the block's
 * MMA thread waits for a copy that never comes (-1: off).  No counterpart in
 * the reference. */
int dnspir_fleet_set_wait_limit(dnspir_fleet* fleet, uint64_t wait_ns, int withhold_chunk);
/* The tensor scan's tile shapes (query-operand rows per CTA, m-tiles per CTA,
 * pipeline stages, kernel: 0 one tile per CTA, 1 persistent warp-specialised,
 * 2 CTA pair with relayed bulk copies, 3 CTA pair with tensor-map copies);
 * returns their count. */
int dnspir_tscan_shapes(int* nq, int* mtpc, int* stages, int* persistent, int max);

/* ---- Serving loop (no counterpart in the reference, whose server answers each
 * connection on its own thread with process_query, dns/server.rs:789).
 * One worker thread per server owns the device work of every database added
 * to it: submitted queries are queued per database and answered in groups
 * (continuous batching: each group takes every pending query up to the
 * database's admitted group size, while earlier groups are still on the
 * device); each group size's launch sequence is captured as CUDA graphs and
 * replayed.  Group sizes are admitted by free device memory at start.  A fleet
 * attached to a running server answers only through it (its other calls
 * return DNSPIR_ERR_BAD_ARG until dnspir_server_stop).
 * Sessions: a client's Galois keys (the first two polynomials of its query
 * bytes, 25,600 bytes) decoded once and held on the device; a query submitted
 * with a session omits those bytes.  max_sessions may be 0. */
typedef struct dnspir_server dnspir_server;
int dnspir_server_create(int device, uint32_t max_sessions, dnspir_server** out);
/* max_batch: 1..256 (tensor engine) or a power of two up to 256 (CUDA cores). */
int dnspir_server_add_db(dnspir_server* server, dnspir_fleet* fleet, uint32_t max_batch, uint32_t* db_id);
/* Batching window of a database (default 1 query, no wait): a group launches
 * once min_batch queries are pending or the oldest has waited max_wait_us. */
int dnspir_server_set_batching(dnspir_server* server, uint32_t db_id, uint32_t min_batch, uint32_t max_wait_us);
/* Databases are served on streams of their own, prioritised by database size
 * (smaller first); the fleets get their own streams back at stop. */
int dnspir_server_start(dnspir_server* server, int use_graphs);
int dnspir_server_open_session(dnspir_server* server, const uint8_t* galois_key_bytes, uint64_t len,
                               uint64_t* session);
/* Requests already submitted with the session still complete. */
int dnspir_server_close_session(dnspir_server* server, uint64_t session);
/* session: -1 for a full query (the reference's bytes). */
int dnspir_server_submit(dnspir_server* server, uint32_t db_id, int64_t session, const uint8_t* query, uint64_t len,
                         uint64_t* ticket);
/* *done = 0 while pending; once done the reply (22,272 bytes) is copied out,
 * the ticket is released and the request's status is returned. */
int dnspir_server_poll(dnspir_server* server, uint64_t ticket, uint8_t* reply, uint64_t reply_cap, int* done);
int dnspir_server_wait(dnspir_server* server, uint64_t ticket, uint8_t* reply, uint64_t reply_cap,
                       uint32_t timeout_ms);
/* Completed requests, admitted group size, groups launched (and of them,
 * replayed from graphs), and the submit-to-done latencies in completion order. */
int dnspir_server_db_stats(dnspir_server* server, uint32_t db_id, uint64_t* completed, uint32_t* admitted_batch,
                           uint64_t* groups, uint64_t* graph_groups, double* latencies_ms, uint32_t max_latencies,
                           uint32_t* n_latencies);
/* Answers every submitted request, then detaches the fleets. */
int dnspir_server_stop(dnspir_server* server);
int dnspir_server_destroy(dnspir_server* server);
/* Synthetic 2560-byte payloads packed into 10-bit coefficients
 * (pack_bytes_into_coeffs, dns/bucket.rs:289-303): bytes = entries x 2560 on
 * the device, coeffs = entries x 2048 on the device. */
int dnspir_pack_payloads(int device, const uint8_t* bytes, uint64_t entries, uint16_t* coeffs);

/* process_queries (pir_wrapper.rs:349-409) for nq independent queries.
 * queries[i] has query_lens[i] bytes; reply i is written at replies + i *
 * reply_stride (dnspir_reply_bytes() bytes).  status[i] receives each query's
 * status.  on_device != 0: query and reply buffers are device pointers. */
int dnspir_fleet_process_queries(dnspir_fleet* fleet, const uint8_t* const* queries, const uint64_t* query_lens,
                                 uint32_t nq, uint8_t* replies, uint64_t reply_stride, int32_t* status,
                                 int on_device);
/* process_query (pir_wrapper.rs:328) */
int dnspir_fleet_process_query(dnspir_fleet* fleet, const uint8_t* query, uint64_t query_len, uint8_t* reply,
                               uint64_t* reply_len);
/* perform_double_pir (double_pir.rs:104-123) on ring elements: pq, pqc (NULL
 * iff the primary group needs no conjugate), sq, sqc (likewise), gk (2 x N);
 * out = 3 ciphertexts x (a, b) x N. */
int dnspir_fleet_perform_double_pir(dnspir_fleet* fleet, const uint64_t* pq, const uint64_t* pqc, const uint64_t* sq,
                                    const uint64_t* sqc, const uint64_t* gk, uint64_t* out);
/* Device time of the last answered query, from CUDA events: primary phase
 * (copy-in + decode + scan + epilogue), secondary phase, and the scan kernel
 * alone (PRIMARY_PHASE_MICROS / SECONDARY_PHASE_MICROS, double_pir.rs:230-242). */
int dnspir_fleet_last_timings(dnspir_fleet* fleet, double* primary_ms, double* secondary_ms, double* scan_ms);
/* Per-query device times of the last process_queries / perform_double_pir
 * call, from CUDA events, for up to `max` queries: latency (start of the
 * query's copy-in to its reply), primary phase, secondary phase, scan kernel.
 * Consecutive queries overlap (the primary phase of query k+1 runs during the
 * secondary phase of query k).  Entries of rejected queries are -1.  Returns
 * the number of entries written, or minus a status code. */
int dnspir_fleet_batch_timings(dnspir_fleet* fleet, uint32_t max, double* latency_ms, double* primary_ms,
                               double* secondary_ms, double* scan_ms);
/* Launch on a caller-owned cudaStream_t (NULL restores the fleet's own stream). */
int dnspir_fleet_set_stream(dnspir_fleet* fleet, void* cuda_stream);
/* Kernels the fleet's answer pipeline has launched so far (counted at each
 * launch: decode, query operand and scan, epilogue, and per secondary chunk the
 * encoder's three kernels, the chains and the replies).  No counterpart in the
 * reference. */
int dnspir_fleet_launch_count(dnspir_fleet* fleet, uint64_t* count);
/* Bytes of slab memory the fleet holds on its device. */
uint64_t dnspir_fleet_slab_bytes(dnspir_fleet* fleet);
int dnspir_fleet_destroy(dnspir_fleet* fleet);

/* ---- client side (host only; load generation and answer checks) -------- */

/* prepare_query_general (pir_wrapper.rs:276-317) with rng = StdRng(rng_seed):
 * writes dnspir_query_bytes(primary_order, secondary_order) bytes and the
 * 32-byte secret-key seed needed to read the reply. */
int dnspir_client_prepare_query(const uint8_t* rng_seed, uint64_t primary_idx, uint64_t secondary_idx,
                                uint32_t primary_order, uint32_t secondary_order, uint8_t* query,
                                uint64_t* query_len, uint8_t* sk_seed_out);
/* process_reply (pir_wrapper.rs:420-440): the N = 2048 coefficients of the entry. */
int dnspir_client_process_reply(const uint8_t* reply, uint64_t reply_len, const uint8_t* sk_seed, uint16_t* coeffs);

#ifdef __cplusplus
}
#endif

#endif /* DNSPIR_H */
