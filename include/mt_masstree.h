/*
 * C ABI of the B200 masstree (libmt_b200.so).
 *
 * Drop-in boundary for IndexinGPU's gpu_masstree host API
 * (include/gpu_masstree.hpp:84-191 of the reference).  Every entry point takes
 * plain pointers and sizes; key and value buffers are flat uint32 "slice"
 * arrays of stride max_key_length / max_value_length (reference README.md:43-50)
 * and may live in device memory or in pinned host memory mapped into the
 * device address space.  A NULL length array means "every item has the maximum
 * length".  value_lengths[i] == 0 after a find means "not found".
 *
 * Calls are asynchronous on `stream` (a cudaStream_t passed as void*).  A tree
 * must be driven from one stream at a time (the reference has the same rule:
 * kernels on one reclaimer must not overlap, simple_debra_reclaim.hpp:189,226).
 * Device-side failures (pool exhausted, lock timeout, corruption) are recorded
 * on the device and returned by mt_sync().
 */
#ifndef MT_MASSTREE_H_
#define MT_MASSTREE_H_

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mt_masstree mt_masstree;

/* Status codes. */
enum {
  MT_OK = 0,
  MT_ERR_OOM = 1,          /* slab pool exhausted */
  MT_ERR_LOCK_TIMEOUT = 2, /* a node lock was not obtained within the bound */
  MT_ERR_CORRUPT = 3,      /* an invalid slab index or a runaway traversal was seen */
  MT_ERR_INVALID_ARG = 4,
  MT_ERR_CUDA = 5,
  MT_ERR_RETRY_LIMIT = 6,  /* an insert restarted its descent too often */
  MT_ERR_KEY_TOO_LONG = 7, /* a scan's layer stack could not grow (device API scans without an allocator) */
  MT_ERR_BATCH_TOO_LARGE = 8 /* batch larger than mt_mixed_batch_noalloc's fixed scratch */
};

/* Request kinds of mt_mixed_batch (reference macros.hpp:51-57). */
enum { MT_REQ_INSERT = 0, MT_REQ_ERASE = 1, MT_REQ_FIND = 2, MT_REQ_UPDATE = 3 };

/* Flags. */
#define MT_FLAG_CONCURRENT 1u       /* find/scan may run beside writers (reference template `concurrent`) */
#define MT_FLAG_UPDATE_IF_EXISTS 2u /* insert overwrites an existing key (reference `update_if_exists`) */
#define MT_FLAG_USE_UPPER_KEY 4u    /* scan stops after upper_keys (reference `use_upper_key`) */
#define MT_FLAG_SINGLE_PASS 8u      /* mixed_batch: one kernel for every kind instead of
                                       finds-then-writes passes (comparison switch) */
#define MT_FLAG_BUCKET_KEYS 16u     /* mixed_batch(es): serve short keys before long keys in
                                       every request class */
#define MT_FLAG_PERSISTENT 32u      /* mixed_batches: one cooperative persistent launch for all
                                       sub-batches instead of three class kernels per sub-batch */
#define MT_FLAG_MERGE 64u           /* erase, mixed_batch: after the call's erases, fold nodes
                                       left with 4 entries or fewer into a neighbour under the same
                                       parent, border nodes and then their sparse ancestors, and
                                       fold a layer root left with one child into its slab
                                       (reference erase merge levels 2-4; space only, results are
                                       the same) */
#define MT_FLAG_GROUP_BY_KEY 512u   /* mixed_batches: serve all sub-batches at once, the requests on one key
                                       resolved in sub-batch order (one tree read and at most one write per
                                       key that several requests touch) */
#define MT_FLAG_INPUTS_ON_STREAM 256u /* mixed_batch_host: the uploads wait for the work queued on `stream`
                                       before the call (for host inputs that work produces, e.g. a copy
                                       queued just before); without it the uploads start at once */
#define MT_FLAG_REMOVE_EMPTY_LAYERS 128u /* erase, mixed_batch: after the call's erases (and merges),
                                       remove every trie layer (1 or deeper, reached by at most 15
                                       key slices) whose only node they left empty (with
                                       MT_FLAG_MERGE: whose nodes all folded into an empty root),
                                       and the parent layers this empties in turn (reference erase
                                       merge level 4,
                                       do_remove_empty_root, include/gpu_masstree.hpp:914-960;
                                       space only, results are the same) */

/* One sub-batch of mt_mixed_batches: the buffers of one mt_mixed_batch call
 * (device pointers; max lengths are common to all sub-batches). */
typedef struct mt_subbatch {
  const uint8_t* request_types;
  const uint32_t* keys;
  const uint32_t* key_lengths; /* may be NULL */
  uint32_t* values;
  uint32_t* value_lengths;
  bool* results;               /* may be NULL */
  uint32_t num_requests;
  uint32_t reserved;
} mt_subbatch;

typedef struct mt_stats_t {
  uint64_t total_slabs;     /* slabs in the pool (128 bytes each) */
  uint64_t used_slabs;      /* handed out and not yet returned */
  uint64_t free_slabs;      /* never used or returned */
  uint64_t limbo_slabs;     /* retired, returned at the next call on the tree */
  uint32_t num_shards;
  uint32_t tile_size;
  uint32_t device_error;    /* first device error since the last mt_sync */
  uint32_t device_error_count;
  uint32_t device_error_site; /* where that error (or, if none is pending, the one the last mt_sync
                                 returned) was detected: source file number << 16 | line (diagnostics) */
  uint32_t reserved;
} mt_stats_t;

/* Construction.  Replaces gpu_masstree(allocator(pool_ratio), reclaimer())
 * (reference gpu_masstree.hpp:67-72, simple_slab_alloc.hpp:56-69): the slab
 * pool takes pool_ratio of the currently free device memory.  tile_size is the
 * number of lanes serving one request (4, 8, 16 or 32). */
int mt_create(mt_masstree** out, float pool_ratio, uint32_t tile_size);
/* Same, with the pool size given in bytes. */
int mt_create_bytes(mt_masstree** out, uint64_t pool_bytes, uint32_t tile_size);
/* Reference ~gpu_masstree / ~simple_slab_allocator (gpu_masstree.hpp:80-82). */
int mt_destroy(mt_masstree* tree);

/* Launch shape: lanes per request (4/8/16/32) and resident blocks per SM
 * (0 = as many as fit).  New in this library. */
int mt_set_tile_size(mt_masstree* tree, uint32_t tile_size);
/* Lanes per request for inserts, updates and erases only (mt_set_tile_size
 * sets both widths). */
int mt_set_write_tile_size(mt_masstree* tree, uint32_t tile_size);
int mt_set_blocks_per_sm(mt_masstree* tree, uint32_t blocks_per_sm);
/* Lanes per update or erase request of mixed batches (4/8/16/32; 0 = the
 * write width, the default).  Under skewed key choice most of them miss (the
 * key was erased) and end in a lock-free check, which narrow tiles serve many
 * at a time.  New in this library. */
int mt_set_upderase_tile_size(mt_masstree* tree, uint32_t tile_size);
/* Lanes per scan query (4/8/16/32; 0 = the find width, the default).  Scans
 * read many independent suffix lines per query and run fastest with narrow
 * tiles (more queries in flight).  New in this library. */
int mt_set_scan_tile_size(mt_masstree* tree, uint32_t tile_size);

/* Bound of every node-lock wait: lock attempts (each followed by a backoff of
 * 64 ns to 1 us) before the waiting request gives up and the call reports
 * MT_ERR_LOCK_TIMEOUT (default 2^20, about one second).  The reference spins
 * without a bound (masstree_node_subwarp.hpp:217-219).  New in this library. */
int mt_set_lock_wait(mt_masstree* tree, uint32_t attempts);

/* Fault injection for tests of the bounded lock wait: set (locked != 0) or
 * clear the LOCK bit of tree node `slab` (slab 0 is the root of trie layer 0)
 * from the host, as a writer that never releases its lock would leave it.
 * Synchronous; the caller must not run other work on the tree meanwhile.
 * New in this library. */
int mt_inject_node_lock(mt_masstree* tree, uint32_t slab, int locked);

/* Reference gpu_masstree::find (gpu_masstree.hpp:86-99). */
int mt_find(mt_masstree* tree, const uint32_t* keys, uint32_t max_key_length, const uint32_t* key_lengths,
            uint32_t* values, uint32_t max_value_length, uint32_t* value_lengths, uint32_t num_keys,
            uint32_t flags, void* stream);

/* Reference gpu_masstree::insert (gpu_masstree.hpp:101-115).  results may be
 * NULL (the reference has none); else results[i] = inserted (or updated).
 * An insert of at least 1,024 keys into a tree that holds nothing
 * bulk-builds the tree's first layer (same results and contents); that call
 * waits for the device and allocates temporary scratch, and so does the
 * emptiness check of every insert of 1,024+ keys until one finds keys in the
 * tree. */
int mt_insert(mt_masstree* tree, const uint32_t* keys, uint32_t max_key_length, const uint32_t* key_lengths,
              const uint32_t* values, uint32_t max_value_length, const uint32_t* value_lengths,
              uint32_t num_keys, bool* results, uint32_t flags, void* stream);

/* Reference gpu_masstree::update (gpu_masstree.hpp:117-130). */
int mt_update(mt_masstree* tree, const uint32_t* keys, uint32_t max_key_length, const uint32_t* key_lengths,
              const uint32_t* values, uint32_t max_value_length, const uint32_t* value_lengths,
              uint32_t num_keys, bool* results, uint32_t flags, void* stream);

/* Reference gpu_masstree::erase (gpu_masstree.hpp:132-145).  flags may hold
 * MT_FLAG_MERGE and MT_FLAG_REMOVE_EMPTY_LAYERS (as may mt_mixed_batch's): they
 * change only the space the tree holds afterwards.  The first call with each
 * allocates that flag's log on the device (about 32 MB and 16 MB, kept by the
 * tree); when it does not fit, the call erases without that pass. */
int mt_erase(mt_masstree* tree, const uint32_t* keys, uint32_t max_key_length, const uint32_t* key_lengths,
             uint32_t num_keys, bool* results, uint32_t flags, void* stream);

/* Reference gpu_masstree::scan (gpu_masstree.hpp:147-171).  Query q writes
 * counts[q], values[q][max_count][max_value_length], value_lengths[q][max_count],
 * out_keys[q][max_count][max_key_length], out_key_lengths[q][max_count]; every
 * output pointer may be NULL.  Both bounds are inclusive. */
int mt_scan(mt_masstree* tree, const uint32_t* lower_keys, const uint32_t* lower_key_lengths,
            uint32_t max_key_length, uint32_t max_count_per_query, uint32_t num_queries,
            const uint32_t* upper_keys, const uint32_t* upper_key_lengths, uint32_t* counts,
            uint32_t* values, uint32_t max_value_length, uint32_t* value_lengths,
            uint32_t* out_keys, uint32_t* out_key_lengths, uint32_t flags, void* stream);

/* Reference gpu_masstree::mixed_batch (gpu_masstree.hpp:173-191): request_types
 * uses MT_REQ_*; values / value_lengths are inputs for insert and update and
 * outputs for find; results[i] (may be NULL) is written for insert, update and
 * erase. */
int mt_mixed_batch(mt_masstree* tree, const uint8_t* request_types, const uint32_t* keys,
                   uint32_t max_key_length, const uint32_t* key_lengths, uint32_t* values,
                   uint32_t max_value_length, uint32_t* value_lengths, bool* results,
                   uint32_t num_requests, uint32_t flags, void* stream);

/* mt_mixed_batch with every buffer in HOST memory (pinned for the copies to
 * overlap): the batch is cut into chunks of `chunk` requests (0 = 262,144)
 * that go through a ring of device staging slots kept by the tree; the
 * uploads, the work and the downloads of consecutive chunks overlap, also
 * across consecutive calls on one tree.  Each chunk is served as one
 * mt_mixed_batch (one of the orders a mixed batch allows).  Asynchronous:
 * the input buffers are read from the moment of the call on (they must hold
 * the requests then, and the uploads do not wait for earlier work on
 * `stream`, unless flags hold MT_FLAG_INPUTS_ON_STREAM, which makes them wait
 * for it at the cost of the overlap with the previous call's work), the work
 * and the results are ordered on `stream`, and all host
 * buffers must stay untouched until the stream reaches the end of the call
 * (results are in host memory then).  The first call, and a
 * call with longer rows or larger chunks than before, allocates the staging
 * (not during graph capture).  New in this library: the reference's caller
 * copies around each device-buffer call itself. */
int mt_mixed_batch_host(mt_masstree* tree, const uint8_t* request_types, const uint32_t* keys,
                        uint32_t max_key_length, const uint32_t* key_lengths, uint32_t* values,
                        uint32_t max_value_length, uint32_t* value_lengths, bool* results,
                        uint32_t num_requests, uint32_t chunk, uint32_t flags, void* stream);

/* Size the scratch of mt_mixed_batches for up to max_subbatches sub-batches
 * and max_total_requests requests in one call (allocates; call it before any
 * graph capture).  New in this library. */
int mt_batches_reserve(mt_masstree* tree, uint32_t max_subbatches, uint64_t max_total_requests);

/* Serve num_subbatches mixed batches in order, with the results of one
 * mt_mixed_batch call per sub-batch: sub-batch k+1 sees every effect of
 * sub-batch k.  One partition pass files every request of every sub-batch
 * under its class; then, by default, each sub-batch runs its three class
 * kernels side by side on forked streams (3 launches per sub-batch), or, with
 * MT_FLAG_PERSISTENT, one cooperative persistent launch serves all
 * sub-batches with a grid barrier between them.  `subbatches` is a DEVICE
 * array of descriptors; nothing is read back to the host and the number of
 * launches depends only on num_subbatches, so the call can be captured in a
 * CUDA graph and replayed after the descriptors' contents change.  Needs
 * mt_batches_reserve; flags may hold MT_FLAG_BUCKET_KEYS and
 * MT_FLAG_PERSISTENT.  Find tile width: mt_set_tile_size (4/8/16/32); write
 * tile width: mt_set_write_tile_size (16 or 32).  With MT_FLAG_GROUP_BY_KEY
 * all sub-batches are served at once: the requests are sorted by a hash of
 * their key, each key's requests resolved in sub-batch order (and, inside a
 * sub-batch, in buffer order) by a segmented scan, the tree read once and
 * written at most once per key that several requests touch; results and the
 * final contents are those of one call per sub-batch.  Its first call (and
 * one after a larger mt_batches_reserve) allocates about 100 bytes per
 * reserved request plus 4 per reserved request and value slice (outside
 * graph capture; when that does not fit, the call is served in the default
 * form), later calls launch a fixed sequence.  The batched
 * counterpart of the reference's per-call mixed_batch
 * (gpu_masstree.hpp:173-191). */
int mt_mixed_batches(mt_masstree* tree, const mt_subbatch* subbatches, uint32_t num_subbatches,
                     uint32_t max_key_length, uint32_t max_value_length, uint32_t flags, void* stream);

/* Diagnostic for MT_FLAG_GROUP_BY_KEY: its sort uses `bits` bits of the key
 * hash (1..64, default 64).  With fewer, different keys share hashes; the form
 * finds them when it checks each run key by key and serves such a run one
 * request after the other (the path tests reach this way).  New in this
 * library. */
int mt_set_group_hash_bits(mt_masstree* tree, uint32_t bits);

/* Serving (mt_serve). */
#define MT_SERVE_SERVED 0u /* device-resident request loop with continuous admission */
#define MT_SERVE_PLAIN 1u  /* one synchronous mt_mixed_batch call per request, in arrival order */
#define MT_SERVE_ONLINE 2u /* the plan's op buffers are HOST memory: each request is submitted at its
                              arrival time through mt_server_submit (its upload and the download of
                              its results are part of its latency) and polled to completion */

typedef struct mt_serve_plan {
  /* Ops of every request, concatenated (device pointers; request r owns ops
   * [request_first_op[r], request_first_op[r] + request_num_ops[r])). */
  const uint8_t* types;
  const uint32_t* keys;
  const uint32_t* key_lengths; /* may be NULL */
  uint32_t* values;
  uint32_t* value_lengths;
  bool* results;               /* may be NULL */
  uint32_t max_key_length;
  uint32_t max_value_length;
  /* Host arrays, one entry per request, in arrival order; the op ranges of
   * different requests must not overlap. */
  const uint32_t* request_first_op;
  const uint32_t* request_num_ops;
  const uint64_t* arrival_ns;  /* arrival time after the start of the run */
  uint32_t num_requests;
  uint32_t mode;               /* MT_SERVE_SERVED, MT_SERVE_PLAIN or MT_SERVE_ONLINE */
  uint32_t chunk_ops;          /* ops per device work item (0 = chosen per request from the backlog) */
  uint32_t epoch_us;           /* device time per launch of the serving loop (0 = 20000) */
  float memory_budget;         /* admit while slabs in use stay under this share of the pool (0 = 0.9) */
  uint32_t reserved;
} mt_serve_plan;

typedef struct mt_serve_stats {
  uint64_t wall_ns;          /* host time from start to the last completion */
  uint64_t requests_done;
  uint64_t ops_done;
  uint64_t admission_waits;  /* times an arrived request waited for slab memory */
  uint64_t stage_ns[4];      /* MT_SERVE_ONLINE: the server's queued / upload / device /
                                deliver sums (mt_server_stats_t); 0 otherwise */
} mt_serve_stats;

/* Serve an open-loop stream of requests: each request is admitted when its
 * arrival time has come (and memory allows), served by the device-resident
 * loop together with whatever else is in flight, and completed by a flag the
 * device writes to host memory.  latency_ns[r] (host array) receives
 * completion - arrival for request r.  Synchronous; runs on its own stream.
 * Requests in flight together have no defined order among each other, as the
 * requests of one reference mixed_batch.  No counterpart in the reference
 * (its host API serves one batch per call). */
int mt_serve(mt_masstree* tree, const mt_serve_plan* plan, uint64_t* latency_ns, mt_serve_stats* stats);

/* Online serving (mt_server_*): a device-resident request loop that clients
 * feed with requests from host memory while it runs.  mt_server_submit takes
 * one request (num_ops ops of any kind, the buffers of one mt_mixed_batch call,
 * in HOST memory, pinned for the copies to overlap) and returns at once with a
 * ticket; a host thread of the server admits queued requests in submission
 * order while the staging space and the memory budget allow, uploads their ops
 * (the upload is part of the request's latency), publishes them as work items
 * to the device loop (the persistent kernel of mt_serve), downloads each
 * request's results into its host buffers when the device completes it, and
 * then marks the ticket done.  Requests in flight together have no order among
 * each other, as the requests of one mixed batch; a request's buffers must stay
 * untouched until mt_server_poll reports it done.  Submit and poll may be
 * called from any host thread; while a server runs, nothing else may be called
 * on its tree.  No counterpart in the reference (its host API serves one batch
 * per call, gpu_masstree.hpp:173-191). */
typedef struct mt_server mt_server;

typedef struct mt_server_config {
  uint32_t max_key_length;
  uint32_t max_value_length;
  uint32_t max_ops_in_flight;      /* device staging for admitted ops (0 = 1 << 20) */
  uint32_t max_requests_in_flight; /* admitted and not yet done (0 = 65536) */
  uint32_t chunk_ops;              /* ops per device work item (0 = chosen per request from the backlog) */
  uint32_t epoch_us;               /* device time per launch of the loop (0 = 20000) */
  float memory_budget;             /* admit while slabs in use stay under this share of the pool (0 = 0.9) */
  uint32_t reserved;
} mt_server_config;

/* Start serving `tree` (allocates the staging and starts the host thread and
 * the device loop). */
int mt_server_start(mt_masstree* tree, const mt_server_config* config, mt_server** out);
/* Queue one request of num_ops ops (1 .. max_ops_in_flight); *ticket receives
 * its ticket.  key_lengths and results may be NULL, as for mt_mixed_batch. */
int mt_server_submit(mt_server* server, const uint8_t* request_types, const uint32_t* keys,
                     const uint32_t* key_lengths, uint32_t* values, uint32_t* value_lengths, bool* results,
                     uint32_t num_ops, uint64_t* ticket);
/* *done = 1 once the request's results are in its host buffers (then
 * *latency_ns, if not NULL, receives the time from submit to done, kept for
 * the last 65,536 tickets or max_requests_in_flight, whichever is more; 0
 * for older ones), else 0. */
int mt_server_poll(mt_server* server, uint64_t ticket, int* done, uint64_t* latency_ns);
/* Where completed requests spent their time: sums over the requests completed
 * so far (divide by `requests` for means) of the time from submit to
 * admission (queued behind earlier requests, staging space or the memory
 * budget), admission to publication (the copy into the staging and its upload),
 * publication to the device's completion flag as the host thread saw it, and
 * flag to results in the caller's buffers; and the largest submit-to-done
 * time. */
typedef struct mt_server_stats_t {
  uint64_t requests;
  uint64_t ops;
  uint64_t queued_ns;
  uint64_t upload_ns;
  uint64_t device_ns;
  uint64_t deliver_ns;
  uint64_t max_latency_ns;
  uint64_t reserved;
} mt_server_stats_t;
int mt_server_stats(mt_server* server, mt_server_stats_t* out);
/* Serve every submitted request, stop the loop and free the server (the tree
 * stays).  Returns the first device error of the run (as mt_sync), or
 * MT_ERR_LOCK_TIMEOUT if the queued work did not drain within 60 s. */
int mt_server_stop(mt_server* server);

/* mt_mixed_batch for callers that cannot allocate device memory at call time:
 * request loops that must never wait on the driver's allocator (mt_mixed_batch,
 * given a batch larger than any before, waits for its stream and cudaMallocs
 * new partition scratch), and programs that hand the whole device to the slab
 * pool or to another allocator up front, where a cudaMalloc in the middle of
 * serving fails.  This variant never calls cudaMalloc, cudaFree or any
 * allocating routine.  Its scratch is one fixed array of 2 MiB + 128 B in the
 * library, present on every GPU that loads it until the process exits, so
 * num_requests is limited to 262144 (1 << 18); larger batches return
 * MT_ERR_BATCH_TOO_LARGE and launch nothing.  It takes the arguments of
 * mt_mixed_batch without flags and behaves as mt_mixed_batch with flags = 0
 * (same results and error reporting; the finds and then the writes are served
 * as two passes on `stream`).
 * The tree's device must be current (else MT_ERR_INVALID_ARG).  The first call
 * on a device looks up the array's device address there (once per device);
 * make that first call before any stream capture.  All calls on one GPU share
 * the array and it keeps the last call's contents: calls whose work overlaps on
 * the GPU (different streams, or different trees, without ordering between
 * them) race on it and must be serialised by the caller.
 * No counterpart in the reference. */
int mt_mixed_batch_noalloc(mt_masstree* tree, const uint8_t* request_types, const uint32_t* keys,
                           uint32_t max_key_length, const uint32_t* key_lengths, uint32_t* values,
                           uint32_t max_value_length, uint32_t* value_lengths, bool* results,
                           uint32_t num_requests, void* stream);

/* Device view of the tree for kernels that call the device API
 * (include/mt/device.cuh, gpu_masstree_device::from): copies the view, a
 * plain struct of view_bytes bytes (checked), to *view.  The view stays valid
 * until mt_destroy.  New in this library (the reference's kernels take the
 * host object itself by value, include/gpu_masstree.hpp:194-971). */
int mt_device_view(mt_masstree* tree, void* view, size_t view_bytes);

/* Wait for `stream`, then return (and clear) the first device error recorded
 * since the previous mt_sync (MT_OK if none). */
int mt_sync(mt_masstree* tree, void* stream);

/* Pool statistics (synchronous; reference simple_slab_allocator::print_stats,
 * simple_slab_alloc.hpp:82-89). */
int mt_stats(mt_masstree* tree, mt_stats_t* out);

/* Return retired slabs to the free lists now (normally done at the start of
 * every call).  Retired slabs are those unlinked by earlier calls. */
int mt_reclaim(mt_masstree* tree, void* stream);

/* Structural check of the whole index from a device snapshot (synchronous):
 * node counts, key order inside and across nodes, separators equal to child
 * high keys, suffix chain lengths, no node left locked.  num_keys receives the
 * number of stored keys; msg (may be NULL) a one-line report.  Returns MT_OK
 * or MT_ERR_CORRUPT.  Reference gpu_masstree::validate (gpu_masstree.hpp:1421-1472). */
int mt_validate(mt_masstree* tree, uint64_t* num_keys, char* msg, size_t msg_len);

/* Self-test of the assumption that one tile's 128-byte node load observes a
 * node store atomically, at the given tile width: writer tiles publish lines
 * of identical words while reader tiles count lines whose words disagree.
 * Allocates its own buffers; bounded by iters.  New in this library (the
 * reference states the assumption in README.md:168-172 without a test). */
int mt_selftest_line_atomicity(uint32_t tile_size, uint32_t nlines, uint32_t iters, uint64_t* reads,
                               uint64_t* torn);

/* Human-readable name of a status code. */
const char* mt_status_string(int status);

#ifdef __cplusplus
}
#endif

#endif /* MT_MASSTREE_H_ */
