// Universal-bench adapter over this library: the same struct, members and
// command-line configuration as IndexinGPU's gpu_masstree_adapter
// (evaluation/gpu_masstree_adapter.hpp:26-243), so the reference's
// evaluation/universal_bench.cu (phases insert, lookup, scan, update, insdel,
// space, mixed; :213-537) runs unchanged against libmt_b200.so when this
// directory comes first on its include path.
//
// Configuration arguments (`-name=value` or `--name=value`, parsed like the
// reference's get_arg_value, include/cmd.hpp):
//   allocator_pool_ratio (0.9)  fraction of free device memory for the slab pool
//   tile_size (16)              lanes per find/scan request: 4, 8, 16 or 32
//                               (the reference accepts 16 or 32)
//   lookup_concurrent (false)   find/scan loads that tolerate concurrent writers
//   enable_suffix (true)        accepted; key tails always live in suffix chains
//   merge_level (4)             0-4; 2 and above merge sparse border nodes after
//                               erases (MT_FLAG_MERGE), 4 also removes the trie
//                               layers they empty (MT_FLAG_REMOVE_EMPTY_LAYERS);
//                               results are the same at every level
//   use_shmem_key (false)       accepted; no effect
// and two of this library's own:
//   write_tile_size (32)        lanes per insert/update/erase request
//   scan_tile_size (0)          lanes per scan request (0 = tile_size)
//
// print_stats() prints the reference allocator's line
// (simple_slab_alloc.hpp:82-89), "simple_slab_allocator(128B slabs): A/T slabs
// allocated (P%)", which evaluation/scripts/evaluate.py reads for the space
// test.  A counts the slabs the index holds: retired slabs (unreachable, back
// in the free lists at the next call) are not counted, as the reference's
// reclaimer has freed them by the end of the call that retired them.
//
// A malformed argument throws std::invalid_argument (the reference prints a
// message and calls std::terminate); an unsupported value throws as well.
#pragma once

#include <cctype>
#include <cstdint>
#include <cstdlib>
#include <iostream>
#include <optional>
#include <stdexcept>
#include <string>
#include <string_view>
#include <type_traits>
#include <vector>

#include "../mt/gpu_masstree.hpp"

namespace mt_adapter_detail {

// Value of `-name=value` / `--name=value` among arguments[1..]; every argument
// must have that form.
template <typename T>
std::optional<T> arg_value(const std::vector<std::string>& arguments, std::string_view name) {
  for (std::size_t i = 1; i < arguments.size(); ++i) {
    const std::string_view a(arguments[i]);
    const std::size_t dashes = a.find_first_not_of('-');
    const std::size_t eq = a.find('=');
    if (a.empty() || dashes == std::string_view::npos || dashes > 2 || eq == std::string_view::npos ||
        eq == dashes || eq + 1 == a.size()) {
      throw std::invalid_argument("argument '" + std::string(a) + "' is not -flag=value");
    }
    if (a.substr(dashes, eq - dashes) != name) continue;
    const std::string v(a.substr(eq + 1));
    if constexpr (std::is_same_v<T, bool>) {
      std::string lower = v;
      for (char& c : lower) c = (char)std::tolower((unsigned char)c);
      return lower == "true" || lower == "1";
    } else if constexpr (std::is_same_v<T, float>) {
      return std::strtof(v.c_str(), nullptr);
    } else if constexpr (std::is_same_v<T, uint32_t>) {
      return (uint32_t)std::strtoul(v.c_str(), nullptr, 10);
    } else {
      static_assert(std::is_same_v<T, std::string>, "unsupported argument type");
      return v;
    }
  }
  return std::nullopt;
}

}  // namespace mt_adapter_detail

struct gpu_masstree_adapter {
  static constexpr bool is_ordered = true;
  static constexpr bool support_mixed = true;
  using key_slice_type = uint32_t;
  using value_slice_type = uint32_t;
  using size_type = uint32_t;
  using index_type = GpuMasstreeB200::gpu_masstree;

  void parse(std::vector<std::string>& arguments) { configs_ = configs(arguments); }
  void print_args() const { configs_.print(); }

  void initialize() {
    delete index_;
    index_ = new index_type(configs_.allocator_pool_ratio, configs_.tile_size, configs_.write_tile_size);
    if (configs_.scan_tile_size) index_->set_scan_tile_size(configs_.scan_tile_size);
  }
  void destroy() {
    delete index_;
    index_ = nullptr;
  }
  ~gpu_masstree_adapter() { destroy(); }

  void insert(const key_slice_type* keys, uint32_t keylen_max, const size_type* key_lengths,
              const value_slice_type* values, uint32_t valuelen_max, const size_type* value_lengths,
              std::size_t num_keys) {
    tree().insert(keys, keylen_max, key_lengths, values, valuelen_max, value_lengths, count(num_keys));
  }
  void update(const key_slice_type* keys, uint32_t keylen_max, const size_type* key_lengths,
              const value_slice_type* values, uint32_t valuelen_max, const size_type* value_lengths,
              std::size_t num_keys) {
    tree().update(keys, keylen_max, key_lengths, values, valuelen_max, value_lengths, count(num_keys));
  }
  void erase(const key_slice_type* keys, uint32_t keylen_max, const size_type* key_lengths, std::size_t num_keys) {
    if (configs_.merge_level >= 4) {
      tree().erase<true, true, true>(keys, keylen_max, key_lengths, count(num_keys));
    } else if (configs_.merge_level >= 2) {
      tree().erase<false, true, true>(keys, keylen_max, key_lengths, count(num_keys));
    } else {
      tree().erase<false, false, false>(keys, keylen_max, key_lengths, count(num_keys));
    }
  }
  void find(const key_slice_type* keys, uint32_t keylen_max, const size_type* key_lengths,
            value_slice_type* results, uint32_t valuelen_max, size_type* result_lengths, std::size_t num_keys) {
    if (configs_.lookup_concurrent) {
      tree().find<true>(keys, keylen_max, key_lengths, results, valuelen_max, result_lengths, count(num_keys));
    } else {
      tree().find<false>(keys, keylen_max, key_lengths, results, valuelen_max, result_lengths, count(num_keys));
    }
  }
  // Up to `count` values from each lower bound, no upper bound; the reference
  // ignores upper_keys_for_btree as well (gpu_masstree_adapter.hpp:124-141).
  void scan(const key_slice_type* keys, uint32_t keylen_max, const size_type* key_lengths, uint32_t count_per_query,
            value_slice_type* results, uint32_t valuelen_max, size_type* result_lengths, std::size_t num_keys,
            const key_slice_type* upper_keys_for_btree) {
    (void)upper_keys_for_btree;
    if (configs_.lookup_concurrent) {
      tree().scan<false, true>(keys, key_lengths, keylen_max, count_per_query, count(num_keys), nullptr, nullptr,
                               nullptr, results, valuelen_max, result_lengths, nullptr, nullptr);
    } else {
      tree().scan<false, false>(keys, key_lengths, keylen_max, count_per_query, count(num_keys), nullptr, nullptr,
                                nullptr, results, valuelen_max, result_lengths, nullptr, nullptr);
    }
  }
  // `request_type` is the reference's kernels::request_type or this library's
  // GpuMasstreeB200::request_type: one byte, 0 insert, 1 erase, 2 find, 3 update.
  template <typename request_type>
  void mixed_batch(const request_type* types, const key_slice_type* keys, uint32_t keylen_max,
                   const size_type* key_lengths, value_slice_type* values, uint32_t valuelen_max,
                   size_type* value_lengths, std::size_t num_keys) {
    static_assert(sizeof(request_type) == 1, "request types are one byte");
    const auto* rt = reinterpret_cast<const GpuMasstreeB200::request_type*>(types);
    if (configs_.merge_level >= 4) {
      tree().mixed_batch<true, true, true, true>(rt, keys, keylen_max, key_lengths, values, valuelen_max,
                                                 value_lengths, nullptr, count(num_keys));
    } else if (configs_.merge_level >= 2) {
      tree().mixed_batch<true, false, true, true>(rt, keys, keylen_max, key_lengths, values, valuelen_max,
                                                  value_lengths, nullptr, count(num_keys));
    } else {
      tree().mixed_batch<true, false, false, false>(rt, keys, keylen_max, key_lengths, values, valuelen_max,
                                                    value_lengths, nullptr, count(num_keys));
    }
  }
  void print_stats() {
    const mt_stats_t s = tree().stats();
    const uint64_t allocated = s.used_slabs;
    std::cout << "simple_slab_allocator(128B slabs): " << allocated << "/" << s.total_slabs << " slabs allocated ("
              << (float)allocated / (float)s.total_slabs * 100.0f << "%)" << std::endl;
  }
  void ht_print_load_factor(std::size_t max_keys, uint32_t key_length, uint32_t value_length) {
    (void)max_keys;
    (void)key_length;
    (void)value_length;
  }

  // This library's own: the first device error since the last call, after
  // waiting for the default stream.
  int last_error() { return tree().last_error(); }
  index_type* index() { return index_; }

 private:
  struct configs {
    float allocator_pool_ratio = 0.9f;
    uint32_t tile_size = 16;
    bool lookup_concurrent = false;
    bool enable_suffix = true;
    uint32_t merge_level = 4;
    bool use_shmem_key = false;
    uint32_t write_tile_size = 32;
    uint32_t scan_tile_size = 0;

    configs() = default;
    explicit configs(const std::vector<std::string>& a) {
      using mt_adapter_detail::arg_value;
      allocator_pool_ratio = arg_value<float>(a, "allocator_pool_ratio").value_or(allocator_pool_ratio);
      tile_size = arg_value<uint32_t>(a, "tile_size").value_or(tile_size);
      lookup_concurrent = arg_value<bool>(a, "lookup_concurrent").value_or(lookup_concurrent);
      enable_suffix = arg_value<bool>(a, "enable_suffix").value_or(enable_suffix);
      merge_level = arg_value<uint32_t>(a, "merge_level").value_or(merge_level);
      use_shmem_key = arg_value<bool>(a, "use_shmem_key").value_or(use_shmem_key);
      write_tile_size = arg_value<uint32_t>(a, "write_tile_size").value_or(write_tile_size);
      scan_tile_size = arg_value<uint32_t>(a, "scan_tile_size").value_or(scan_tile_size);
      if (!lanes_ok(tile_size) || !lanes_ok(write_tile_size) || (scan_tile_size && !lanes_ok(scan_tile_size))) {
        throw std::invalid_argument("tile sizes must be 4, 8, 16 or 32");
      }
      if (merge_level > 4) throw std::invalid_argument("merge_level must be 0-4");
      if (!(allocator_pool_ratio > 0.0f && allocator_pool_ratio <= 1.0f)) {
        throw std::invalid_argument("allocator_pool_ratio must be in (0, 1]");
      }
    }
    static bool lanes_ok(uint32_t t) { return t == 4 || t == 8 || t == 16 || t == 32; }
    void print() const {
      std::cout << "    allocator_pool_ratio=" << allocator_pool_ratio << "\n"
                << "    tile_size=" << tile_size << "\n"
                << "    lookup_concurrent=" << lookup_concurrent << "\n"
                << "    enable_suffix=" << enable_suffix << "\n"
                << "    merge_level=" << merge_level << "\n"
                << "    use_shmem_key=" << use_shmem_key << "\n"
                << "    write_tile_size=" << write_tile_size << "\n"
                << "    scan_tile_size=" << scan_tile_size << std::endl;
    }
  };

  index_type& tree() {
    if (!index_) throw std::logic_error("gpu_masstree_adapter: initialize() was not called");
    return *index_;
  }
  static uint32_t count(std::size_t n) {
    if (n > UINT32_MAX) throw std::invalid_argument("gpu_masstree_adapter: more than 2^32-1 keys in one call");
    return (uint32_t)n;
  }

  configs configs_;
  index_type* index_ = nullptr;
};
