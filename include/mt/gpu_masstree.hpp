// C++ host mirror of IndexinGPU's GpuMasstree::gpu_masstree over the C ABI in
// mt_masstree.h.  Method names, argument order, defaults and meaning follow the
// reference's host API (include/gpu_masstree.hpp:84-191); the reference's
// allocator and reclaimer objects become the pool_ratio constructor argument
// (simple_slab_alloc.hpp:56-69).  The template switches are kept for source
// compatibility:
//   * concurrent (find/scan): selects loads that tolerate concurrent writers;
//   * update_if_exists (insert): upsert;
//   * use_upper_key (scan): stop after the upper key;
//   * do_merge (erase) and erase_do_merge (mixed_batch): merge sparse border
//     nodes after the call's erases (MT_FLAG_MERGE; space only, results are
//     the same);
//   * do_remove_empty_root (erase) and erase_do_remove_empty_root
//     (mixed_batch), together with the merge switch as the reference requires:
//     remove the trie layers that the call's erases empty
//     (MT_FLAG_REMOVE_EMPTY_LAYERS; space only, results are the same);
//   * enable_suffix, use_shmem_key and the other erase switches are accepted
//     and do not change results (this library always stores key tails in
//     suffix chains).
// Device-side failures surface through last_error() (which synchronises the
// stream) instead of std::terminate.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>

#include "../mt_masstree.h"

namespace GpuMasstreeB200 {

enum request_type : uint8_t {
  request_type_insert = MT_REQ_INSERT,
  request_type_erase = MT_REQ_ERASE,
  request_type_find = MT_REQ_FIND,
  request_type_update = MT_REQ_UPDATE
};

class gpu_masstree {
 public:
  using size_type = uint32_t;
  using key_slice_type = uint32_t;
  using value_slice_type = uint32_t;

  explicit gpu_masstree(float pool_ratio = 0.9f, uint32_t tile_size = 16, uint32_t write_tile_size = 32) {
    check(mt_create(&h_, pool_ratio, tile_size), "mt_create");
    check(mt_set_write_tile_size(h_, write_tile_size), "mt_set_write_tile_size");
  }
  gpu_masstree(const gpu_masstree&) = delete;
  gpu_masstree& operator=(const gpu_masstree&) = delete;
  ~gpu_masstree() {
    if (h_) mt_destroy(h_);
  }

  template <bool concurrent = false, bool use_shmem_key = false>
  void find(const key_slice_type* keys, const size_type max_key_length, const size_type* key_lengths,
            value_slice_type* values, const size_type max_value_length, size_type* value_lengths,
            const size_type num_keys, cudaStream_t stream = 0) {
    check(mt_find(h_, keys, max_key_length, key_lengths, values, max_value_length, value_lengths, num_keys,
                  concurrent ? MT_FLAG_CONCURRENT : 0u, stream),
          "mt_find");
  }

  template <bool update_if_exists = false, bool enable_suffix = true, bool use_shmem_key = false>
  void insert(const key_slice_type* keys, const size_type max_key_length, const size_type* key_lengths,
              const value_slice_type* values, const size_type max_value_length, const size_type* value_lengths,
              const size_type num_keys, cudaStream_t stream = 0) {
    check(mt_insert(h_, keys, max_key_length, key_lengths, values, max_value_length, value_lengths, num_keys,
                    nullptr, update_if_exists ? MT_FLAG_UPDATE_IF_EXISTS : 0u, stream),
          "mt_insert");
  }

  template <bool enable_suffix = true, bool use_shmem_key = false>
  void update(const key_slice_type* keys, const size_type max_key_length, const size_type* key_lengths,
              const value_slice_type* values, const size_type max_value_length, const size_type* value_lengths,
              const size_type num_keys, cudaStream_t stream = 0) {
    check(mt_update(h_, keys, max_key_length, key_lengths, values, max_value_length, value_lengths, num_keys,
                    nullptr, 0u, stream),
          "mt_update");
  }

  template <bool do_remove_empty_root = true, bool pessimistic_merge = true, bool do_merge = true,
            bool concurrent = true, bool use_shmem_key = false>
  void erase(const key_slice_type* keys, const size_type max_key_length, const size_type* key_lengths,
             const size_type num_keys, cudaStream_t stream = 0) {
    const uint32_t flags =
        (do_merge ? MT_FLAG_MERGE : 0u) | (do_merge && do_remove_empty_root ? MT_FLAG_REMOVE_EMPTY_LAYERS : 0u);
    check(mt_erase(h_, keys, max_key_length, key_lengths, num_keys, nullptr, flags, stream), "mt_erase");
  }

  template <bool use_upper_key = true, bool concurrent = false, bool use_shmem_key = false>
  void scan(const key_slice_type* lower_keys, const size_type* lower_key_lengths, const size_type max_key_length,
            const size_type max_count_per_query, const size_type num_queries,
            const key_slice_type* upper_keys = nullptr, const size_type* upper_key_lengths = nullptr,
            size_type* counts = nullptr, value_slice_type* values = nullptr, const size_type max_value_length = 1,
            size_type* value_lengths = nullptr, key_slice_type* out_keys = nullptr,
            size_type* out_key_lengths = nullptr, cudaStream_t stream = 0) {
    const uint32_t flags = (use_upper_key ? MT_FLAG_USE_UPPER_KEY : 0u) | (concurrent ? MT_FLAG_CONCURRENT : 0u);
    check(mt_scan(h_, lower_keys, lower_key_lengths, max_key_length, max_count_per_query, num_queries, upper_keys,
                  upper_key_lengths, counts, values, max_value_length, value_lengths, out_keys, out_key_lengths,
                  flags, stream),
          "mt_scan");
  }

  template <bool enable_suffix = true, bool erase_do_remove_empty_root = true, bool erase_pessimistic_merge = true,
            bool erase_do_merge = true, bool use_shmem_key = false>
  void mixed_batch(const request_type* request_types, const key_slice_type* keys, const size_type max_key_length,
                   const size_type* key_lengths, value_slice_type* values, const size_type max_value_length,
                   size_type* value_lengths, bool* results, const size_type num_requests,
                   cudaStream_t stream = 0) {
    check(mt_mixed_batch(h_, reinterpret_cast<const uint8_t*>(request_types), keys, max_key_length, key_lengths,
                         values, max_value_length, value_lengths, results, num_requests,
                         (erase_do_merge ? MT_FLAG_MERGE : 0u) |
                             (erase_do_merge && erase_do_remove_empty_root ? MT_FLAG_REMOVE_EMPTY_LAYERS : 0u),
                         stream),
          "mt_mixed_batch");
  }

  // ---- additions of this library (no counterpart in the reference) ----------

  // Lanes per scan query (4/8/16/32; 0 = the find width).
  void set_scan_tile_size(const size_type tile_size) {
    check(mt_set_scan_tile_size(h_, tile_size), "mt_set_scan_tile_size");
  }

  // mixed_batch with every buffer in pinned host memory; uploads, work and
  // downloads of consecutive chunks overlap (mt_mixed_batch_host).
  void mixed_batch_host(const request_type* request_types, const key_slice_type* keys,
                        const size_type max_key_length, const size_type* key_lengths, value_slice_type* values,
                        const size_type max_value_length, size_type* value_lengths, bool* results,
                        const size_type num_requests, cudaStream_t stream = 0, const size_type chunk = 0) {
    check(mt_mixed_batch_host(h_, reinterpret_cast<const uint8_t*>(request_types), keys, max_key_length,
                              key_lengths, values, max_value_length, value_lengths, results, num_requests, chunk,
                              0u, stream),
          "mt_mixed_batch_host");
  }

  // Many mixed sub-batches in order in one call (mt_mixed_batches; device
  // descriptors, sized beforehand by reserve_batches).
  void reserve_batches(const size_type max_subbatches, const uint64_t max_total_requests) {
    check(mt_batches_reserve(h_, max_subbatches, max_total_requests), "mt_batches_reserve");
  }
  void mixed_batches(const mt_subbatch* subbatches, const size_type num_subbatches, const size_type max_key_length,
                     const size_type max_value_length, const uint32_t flags = 0u, cudaStream_t stream = 0) {
    check(mt_mixed_batches(h_, subbatches, num_subbatches, max_key_length, max_value_length, flags, stream),
          "mt_mixed_batches");
  }

  // Open-loop request stream served by the device-resident loop (mt_serve).
  void serve(const mt_serve_plan& plan, uint64_t* latency_ns, mt_serve_stats* stats = nullptr) {
    check(mt_serve(h_, &plan, latency_ns, stats), "mt_serve");
  }

  // Waits for `stream`; returns the first device-side error since the last call.
  int last_error(cudaStream_t stream = 0) { return mt_sync(h_, stream); }

  // Structural check (reference gpu_masstree::validate).
  bool validate(std::string* report = nullptr) {
    char msg[512];
    uint64_t n = 0;
    const int rc = mt_validate(h_, &n, msg, sizeof(msg));
    if (report) *report = msg;
    return rc == MT_OK;
  }

  mt_stats_t stats() {
    mt_stats_t s{};
    check(mt_stats(h_, &s), "mt_stats");
    return s;
  }

  mt_masstree* handle() const { return h_; }

 private:
  static void check(int rc, const char* what) {
    if (rc != MT_OK) throw std::runtime_error(std::string(what) + ": " + mt_status_string(rc));
  }
  mt_masstree* h_ = nullptr;
};

}  // namespace GpuMasstreeB200
