// Internal declarations shared by the translation units of libmt_b200.so.
#pragma once
#include <cuda_runtime.h>

#include "mt_tree.cuh"
#include "../../include/mt_masstree.h"

namespace mtb {

constexpr int kBlock = 128;
constexpr uint32_t kShards = 64;
constexpr uint32_t kScanDepth = 32;   // scan layer frames per tile in scratch (deeper ones spill to slabs)
// In the persistent launch of mt_mixed_batches, sub-batches of at least this
// many requests serve their classes one after the other with a grid barrier
// between them (all warps in the same code at a time, faster on large
// sub-batches); smaller ones let tiles flow from class to class.
constexpr uint32_t kClassBarrierMin = 1u << 17;

#ifndef MT_MIN_BLOCKS_PER_SM
#define MT_MIN_BLOCKS_PER_SM 8  // occupancy hint for the batch kernels: caps registers at 64
#endif
#ifndef MT_WRITE_MIN_BLOCKS_PER_SM
#define MT_WRITE_MIN_BLOCKS_PER_SM MT_MIN_BLOCKS_PER_SM  // the same for kernels that insert
#endif

// Kernel flavours.  OP_PASS_* serve one class of a partitioned mixed batch and
// compile only that class's code (smaller kernels, fewer instruction-cache
// misses than OP_MIXED, which handles every kind).
enum op_kind : int {
  OP_FIND = 0, OP_INSERT = 1, OP_UPSERT = 2, OP_UPDATE = 3, OP_ERASE = 4, OP_MIXED = 5,
  OP_PASS_INSERT = 6, OP_PASS_UPDERASE = 7
};
template <int OP> constexpr bool op_finds = OP == OP_FIND || OP == OP_MIXED;
// Occupancy hint of a batch kernel of kind OP.
template <int OP> constexpr int min_blocks_for =
    (OP == OP_INSERT || OP == OP_UPSERT || OP == OP_PASS_INSERT) ? MT_WRITE_MIN_BLOCKS_PER_SM : MT_MIN_BLOCKS_PER_SM;
template <int OP> constexpr bool op_inserts = OP == OP_INSERT || OP == OP_UPSERT || OP == OP_MIXED || OP == OP_PASS_INSERT;
template <int OP> constexpr bool op_updates = OP == OP_UPDATE || OP == OP_MIXED || OP == OP_PASS_UPDERASE;
template <int OP> constexpr bool op_erases = OP == OP_ERASE || OP == OP_MIXED || OP == OP_PASS_UPDERASE;

struct batch_args {
  const uint8_t* types;
  const uint32_t* keys;
  const uint32_t* key_lengths;
  uint32_t* values;              // insert/update: input, find: output
  const uint32_t* value_lengths_in;
  uint32_t* value_lengths_out;
  bool* results;
  uint32_t* values_out;          // optional: find outputs go here instead of `values` (same row stride)
  const uint32_t* leader_of;     // optional: per request, the request it was combined into (kInvalid: none);
                                 // combined requests are not served here (combine_results_kernel copies results)
  const uint32_t* index;       // optional request subset
  const uint32_t* n_dev;       // optional device-side request count (with index)
  const uint32_t* n_back_dev;  // optional: further indices at the END of the index region
  uint32_t region;             // size of the index region (with n_back_dev)
  uint32_t max_key_length;
  uint32_t max_value_length;
  uint32_t n;
};

struct scan_args {
  const uint32_t* lower;
  const uint32_t* lower_lengths;
  const uint32_t* upper;
  const uint32_t* upper_lengths;
  uint32_t* counts;
  uint32_t* values;
  uint32_t* value_lengths;
  uint32_t* out_keys;
  uint32_t* out_key_lengths;
  scan_frame* frames;
  uint32_t max_key_length;
  uint32_t max_value_length;
  uint32_t max_count;
  uint32_t n;
  uint32_t use_upper;
};

// One request of any kind, executed by the whole tile.
template <int T, int OP, bool CONC>
MT_DEV void run_request(const tile<T>& t, const tree_view& tv, slab_cache<T>& cache, const batch_args& a,
                        uint32_t j, uint32_t kind, uint32_t klen, uint32_t vlen, uint32_t& res, uint32_t& vout) {
  const uint32_t* key = a.keys + (size_t)j * a.max_key_length;
  if constexpr (op_finds<OP>) {
    if (kind == MT_REQ_FIND) {
      uint32_t* vo = a.values_out ? a.values_out : a.values;
      uint32_t* out = vo ? vo + (size_t)j * a.max_value_length : nullptr;
      vout = coop_find<T, CONC>(t, tv, key, klen, out, a.max_value_length);
      return;
    }
  }
  if constexpr (op_inserts<OP>) {
    if (kind == MT_REQ_INSERT) {
      const uint32_t* val = a.values + (size_t)j * a.max_value_length;
      const int r = (OP == OP_UPSERT) ? coop_insert<T, true>(t, tv, cache, key, klen, val, vlen)
                                      : coop_insert<T, false>(t, tv, cache, key, klen, val, vlen);
      res = (r == RES_OK) ? 1u : 0u;
      return;
    }
  }
  if constexpr (op_updates<OP>) {
    if (kind == MT_REQ_UPDATE) {
      const uint32_t* val = a.values + (size_t)j * a.max_value_length;
      res = (coop_update<T>(t, tv, cache, key, klen, val, vlen) == RES_OK) ? 1u : 0u;
      return;
    }
  }
  if constexpr (op_erases<OP>) {
    if (kind == MT_REQ_ERASE) res = (coop_erase<T>(t, tv, key, klen) == RES_OK) ? 1u : 0u;
  }
}

// Serve requests of one batch (all, or the subset a.index[0 .. *a.n_dev)) with
// the tiles tile_id, tile_id + num_tiles, ... of the launch.
template <int T, int OP, bool CONC>
MT_DEV void serve_requests(const tile<T>& t, const tree_view& tv, slab_cache<T>& cache, const batch_args& a,
                           uint32_t tile_id, uint32_t num_tiles) {
  // With a.index the kernel serves requests a.index[0 .. *a.n_dev) (a subset
  // produced by partition_kernel); otherwise requests 0 .. a.n.
  // With n_back_dev the subset is index[0 .. nf) followed by
  // index[region - nb .. region) (two buckets filled from both ends).
  const uint32_t nf = a.n_dev ? *a.n_dev : a.n;
  const uint32_t nb = a.n_back_dev ? *a.n_back_dev : 0u;
  const uint32_t n = nf + nb;
  // A tile takes `per` consecutive requests per round (one per lane, served in
  // turn).  per = T keeps the metadata loads coalesced on large batches; on
  // small ones per shrinks so that every tile gets work and the batch ends
  // after one request latency instead of T of them.
  const uint32_t per = max(1u, min((uint32_t)T, (n + num_tiles - 1u) / num_tiles));
  for (uint32_t base = tile_id * per; base < n; base += num_tiles * per) {
    if (t.shfl((uint32_t)(t.leader() && fatal_error(tv.pool)), 0)) break;
    const uint32_t pos = base + t.rank;
    const bool valid = t.rank < per && pos < n;
    const uint32_t i = (valid && a.index) ? a.index[pos < nf ? pos : a.region - nb + (pos - nf)] : pos;
    uint32_t kind = 0, klen = 0, vlen = 0;
    if (valid) {
      if constexpr (OP == OP_MIXED || OP == OP_PASS_UPDERASE) kind = a.types[i];
      else if constexpr (OP == OP_FIND) kind = MT_REQ_FIND;
      else if constexpr (OP == OP_INSERT || OP == OP_UPSERT || OP == OP_PASS_INSERT) kind = MT_REQ_INSERT;
      else if constexpr (OP == OP_UPDATE) kind = MT_REQ_UPDATE;
      else kind = MT_REQ_ERASE;
      klen = a.key_lengths ? a.key_lengths[i] : a.max_key_length;
      if (kind == MT_REQ_INSERT || kind == MT_REQ_UPDATE)
        vlen = a.value_lengths_in ? a.value_lengths_in[i] : a.max_value_length;
    }
    // Lengths beyond the row stride (or unknown kinds) would read outside the
    // caller's buffers: such requests are skipped and reported.
    const bool bad = valid && (klen > a.max_key_length || vlen > a.max_value_length || kind > MT_REQ_UPDATE);
    if (t.any(bad) && bad) record_error(tv.pool, ERR_INVALID_ARG);
    const bool combined = valid && a.leader_of != nullptr && a.leader_of[i] != kInvalid;
    uint32_t res = 0, vout = 0;
    const uint32_t nreq = min(per, n - base);
    for (uint32_t r = 0; r < nreq; ++r) {
      if (t.shfl((uint32_t)(bad || combined), (int)r)) continue;
      const uint32_t j = t.shfl(i, (int)r);
      const uint32_t k = t.shfl(kind, (int)r);
      const uint32_t kl = t.shfl(klen, (int)r);
      const uint32_t vl = t.shfl(vlen, (int)r);
      uint32_t rr = 0, vo = 0;
      run_request<T, OP, CONC>(t, tv, cache, a, j, k, kl, vl, rr, vo);
      if (t.rank == r) { res = rr; vout = vo; }
    }
    if (valid && !combined) {
      if (kind == MT_REQ_FIND) {
        if (a.value_lengths_out) a.value_lengths_out[i] = vout;
      } else if (a.results) {
        a.results[i] = res != 0u;
      }
    }
  }
}

}  // namespace mtb

namespace mtb {

// mt_mixed_batches (mt_batches.cu, mt_grouped.cu): the call's sub-batches and scratch.
constexpr uint32_t kCountStride = 8;  // per sub-batch: 3 classes x (front, back), padded

struct batches_view {
  const mt_subbatch* sub;   // device descriptors
  uint32_t nsub;
  uint32_t* offsets;        // [nsub + 1] first request of every sub-batch in the flat order
  uint32_t* counts;         // [nsub][kCountStride]
  uint32_t* lists;          // [3][max_total] class index regions
  uint32_t* status;         // [0] = 1 when the list exceeds the reserved scratch
  uint32_t max_total;
  uint32_t max_key_length;
  uint32_t max_value_length;
  uint32_t bucket_keys;     // 1: short keys first, long keys last in every class
};

// Sub-batch holding flat request g (binary search over the prefix sums).
MT_DEV uint32_t find_subbatch(const uint32_t* offsets, uint32_t nsub, uint32_t g) {
  uint32_t lo = 0, hi = nsub;  // offsets[lo] <= g < offsets[hi]
  while (hi - lo > 1u) {
    const uint32_t mid = (lo + hi) >> 1;
    if (offsets[mid] <= g) lo = mid;
    else hi = mid;
  }
  return lo;
}

}  // namespace mtb

struct mt_host_pipe;  // staging of mt_mixed_batch_host (mt_host.cu)

struct mt_masstree {
  // Host-side state of one tree.
  int device = 0;
  int sms = 0;
  uint32_t tile_size = 8;        // finds and scans
  uint32_t write_tile_size = 8;  // inserts, updates, erases
  uint32_t upderase_tile_size = 0;  // updates and erases of mixed batches (0: the write width)
  uint32_t scan_tile_size = 0;   // scans (0: the find width)
  uint32_t blocks_per_sm = 0;    // 0 = occupancy limit
  uint32_t* split_idx = nullptr; // mixed-batch partition scratch
  uint32_t split_cap = 0;
  // Streams and events of the forked class launches of large mixed batches
  // (created on first use).
  cudaStream_t side[2] = {nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr;
  cudaEvent_t ev_join[2] = {nullptr, nullptr};
  mt_host_pipe* host_pipe = nullptr;
  void* mem = nullptr;
  mtb::tree_view tv{};
  mtb::scan_frame* frames = nullptr;
  size_t frames_tiles = 0;
  uint32_t* h_err = nullptr;  // pinned: code, count, fatal flag, site of the first device error
  uint32_t last_error_site = 0;  // site of the error the last mt_sync returned
  // Sub-batch scratch of mt_mixed_batches (see mt_batches.cu).
  void* batches_mem = nullptr;
  void* grouped_mem = nullptr;  // mt_mixed_batches with MT_FLAG_GROUP_BY_KEY (mt_grouped.cu)
  uint32_t grouped_m = 0, grouped_max_v = 0;
  size_t grouped_temp = 0;
  uint32_t group_hash_bits = 64;
  uint32_t batches_max_sub = 0;
  uint64_t batches_max_total = 0;
  // Merge log of MT_FLAG_MERGE calls and layer log of
  // MT_FLAG_REMOVE_EMPTY_LAYERS calls (see mt_merge.cu; created on first use).
  bool maybe_empty = true;  // no insert call has found the tree holding keys yet (bulk build candidate)
  uint32_t* merge_log = nullptr;
  uint32_t* layer_log = nullptr;
};

namespace mtb {
// MT_FLAG_MERGE and MT_FLAG_REMOVE_EMPTY_LAYERS (mt_merge.cu): begin logs the
// call's sparse border nodes and emptied layers as `flags` ask, end (given the
// call's status) merges and removes them after the call's erase kernels.
int host_merge_begin(mt_masstree* t, cudaStream_t s, uint32_t flags);
int host_merge_end(mt_masstree* t, cudaStream_t s, int rc);
// Host helpers implemented in mt_capi.cu.
int host_max_blocks_per_sm(const void* fn, int block, size_t smem);
int host_launch_reclaim(mt_masstree* t, cudaStream_t s);
int host_fork(mt_masstree* t, cudaStream_t s);
int host_join(mt_masstree* t, cudaStream_t s, int rc);
void host_pipe_free(mt_masstree* t);  // mt_host.cu
// mt_grouped.cu; kGroupedUnavailable: its scratch does not fit, nothing launched.
constexpr int kGroupedUnavailable = -1001;
int launch_grouped(mt_masstree* t, const batches_view& b, cudaStream_t s);
int host_launch_insert(mt_masstree* t, const batch_args& a, bool upsert, cudaStream_t s);
// Bulk build of a new tree's first layer (mt_bulk.cu): MT_OK, an error, or
// kBulkDeclined when the batch does not suit it (insert it as usual).
constexpr int kBulkDeclined = -1000;
constexpr uint32_t kBulkMin = 1u << 10;  // smallest insert call that may bulk-build
int host_bulk_insert(mt_masstree* t, const batch_args& a, bool upsert, cudaStream_t s);
bool host_valid_tile(uint32_t ts);
}  // namespace mtb

namespace mtb {

// The three request classes of one mixed batch, served by every tile of the
// launch in turn with no barrier between them: finds with TF-lane tiles, then
// inserts, then updates and erases with TW-lane tiles.  Requests of one mixed
// batch have no defined order, so a tile may start on inserts while others
// still serve finds; only the tail of the whole batch is waited for.
template <int TF, int TW>
MT_DEV void serve_mixed_classes(const tree_view& tv, slab_cache<TW>& wcache, const batch_args& finds,
                                const batch_args& inserts, const batch_args& upderases) {
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  {
    tile<TF> t;
    slab_cache<TF> unused;  // finds never allocate
    serve_requests<TF, OP_FIND, true>(t, tv, unused, finds, gtid / TF, nthreads / TF);
  }
  tile<TW> t;
  serve_requests<TW, OP_PASS_INSERT, true>(t, tv, wcache, inserts, gtid / TW, nthreads / TW);
  serve_requests<TW, OP_PASS_UPDERASE, true>(t, tv, wcache, upderases, gtid / TW, nthreads / TW);
}

}  // namespace mtb
