// Device API of the B200 masstree: tile-cooperative find / insert / update /
// erase / scan for use inside the caller's own CUDA kernels.
//
// Drop-in for the reference's device-side API (GpuMasstree::gpu_masstree::
// cooperative_find / cooperative_insert / cooperative_update /
// cooperative_erase / cooperative_scan, include/gpu_masstree.hpp:194-971; usage
// pattern in README.md:114-166): same member names, template switches,
// argument order and return values.  A kernel receives the index by value,
// builds a tile with cooperative_groups::tiled_partition<Index::tile_size_>,
// an allocator context from `index.allocator_` and, for writes, a reclaimer
// context from `index.reclaimer_`, then calls the cooperative functions with
// every lane of the tile:
//
//   using Index = GpuMasstreeB200::gpu_masstree_device<16>;
//   __global__ void probe(Index index, const uint32_t* keys, ...) {
//     auto tile = cg::tiled_partition<Index::tile_size_>(cg::this_thread_block());
//     typename Index::device_allocator_context_type allocator{index.allocator_, tile};
//     uint32_t vlen = index.template cooperative_find<false>(key, klen, value, maxV, tile, allocator);
//   }
//   // host: Index index = Index::from(tree);  probe<<<...>>>(index, ...);
//
// Differences from the reference, all kept out of the call signatures:
//   * tile_size_ may be 4, 8, 16 or 32 (the reference: 16 or 32);
//   * keys and values are plain uint32 slice pointers (the reference also
//     accepts its key-store wrappers);
//   * reclamation is per launch, not DEBRA epochs: slabs that a kernel's
//     updates, erases and suffix splits unlink are put on a limbo list and
//     return to the free lists at the next mt_reclaim (or any host call on the
//     tree, which starts with that pass).  That pass must be ordered after the
//     kernel on a stream, and no kernel using the device API may run while a
//     host call on the same tree runs.  The allocator context returns the
//     slabs its tile cached but did not use when it goes out of scope;
//   * erase never merges nodes from the device API (do_merge and the other
//     erase switches are accepted; results are the same, only space differs);
//   * failures (pool exhausted, a lock wait that ran out, corruption) make the
//     call return 0 / false and are recorded on the device; mt_sync(tree,
//     stream) returns them;
//   * cooperative_find<false> and cooperative_scan<..., false> read without
//     checks against concurrent writers (as the reference's non-concurrent
//     forms): use them only in kernels and at times when no writer runs.
#pragma once

#include <cooperative_groups.h>

#include "../../indexingpu_b200/csrc/mt_tree.cuh"
#include "../mt_masstree.h"

namespace GpuMasstreeB200 {

namespace detail {
template <class Tile>
struct tile_width;
template <unsigned N, class Parent>
struct tile_width<cooperative_groups::thread_block_tile<N, Parent>> {
  static constexpr int value = (int)N;
};
template <int N>
struct tile_width<mtb::tile<N>> {
  static constexpr int value = N;
};
}  // namespace detail

template <uint32_t tile_size = 16>
struct gpu_masstree_device {
  static_assert(tile_size == 4 || tile_size == 8 || tile_size == 16 || tile_size == 32,
                "tile_size must be 4, 8, 16 or 32");
  static constexpr uint32_t tile_size_ = tile_size;
  static constexpr int T = (int)tile_size;
  using size_type = uint32_t;
  using key_slice_type = uint32_t;
  using value_slice_type = uint32_t;

  mtb::tree_view tree_;
  mtb::pool_view allocator_;  // pass to device_allocator_context_type (reference member allocator_)
  mtb::pool_view reclaimer_;  // pass to device_reclaimer_context_type (reference member reclaimer_)

  // Device view of a tree (host side; a plain copy to pass to kernels by value).
  static gpu_masstree_device from(mt_masstree* tree) {
    gpu_masstree_device d{};
    if (mt_device_view(tree, &d.tree_, sizeof(d.tree_)) != MT_OK) {
      d.tree_.pool.num_slabs = 0;  // every slab index is then invalid: calls fail as corrupt
    }
    d.allocator_ = d.tree_.pool;
    d.reclaimer_ = d.tree_.pool;
    return d;
  }

  // Per-tile slab cache (reference device_allocator_context{index.allocator_, tile}).
  struct device_allocator_context_type {
    mtb::pool_view pool;
    mtb::tile<T> t;
    mtb::slab_cache<T> cache;
    template <class Tile>
    __device__ device_allocator_context_type(const mtb::pool_view& p, const Tile&) : pool(p), t(mtb::lane_id()) {
      static_assert(detail::tile_width<Tile>::value == T, "tile width differs from the index's tile_size_");
      const uint32_t tid = (blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)) *
                               (blockDim.x * blockDim.y * blockDim.z) +
                           threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
      cache.init(p, tid / T);
    }
    __device__ ~device_allocator_context_type() { cache.release(t, pool); }
    device_allocator_context_type(const device_allocator_context_type&) = delete;
    device_allocator_context_type& operator=(const device_allocator_context_type&) = delete;
  };

  // Retirement needs no per-tile state here (see the reclamation note above);
  // the type keeps the reference's call signatures.
  struct device_reclaimer_context_type {
    template <class Tile>
    __device__ device_reclaimer_context_type(const mtb::pool_view&, const Tile&) {}
  };

  // Reference cooperative_find (gpu_masstree.hpp:194-248): the full value
  // length (0 = not found); writes min(length, max_value_length) slices.
  template <bool concurrent, class Tile>
  __device__ size_type cooperative_find(const key_slice_type* key, const size_type key_length,
                                        value_slice_type* value, const size_type max_value_length, const Tile&,
                                        device_allocator_context_type& allocator) const {
    return mtb::coop_find<T, concurrent>(allocator.t, tree_, key, key_length, value, max_value_length);
  }

  // Reference cooperative_insert (gpu_masstree.hpp:397-627): true if inserted
  // (or, with update_if_exists, updated).  Keys always keep their tails in
  // suffix chains (enable_suffix is accepted).
  template <bool update_if_exists = false, bool enable_suffix = true, class Tile>
  __device__ bool cooperative_insert(const key_slice_type* key, const size_type key_length,
                                     const value_slice_type* value, const size_type value_length, const Tile&,
                                     device_allocator_context_type& allocator,
                                     device_reclaimer_context_type&) const {
    return mtb::coop_insert<T, update_if_exists>(allocator.t, tree_, allocator.cache, key, key_length, value,
                                                 value_length) == mtb::RES_OK;
  }

  // Reference cooperative_update (gpu_masstree.hpp:629-749): false on a miss.
  template <bool enable_suffix = true, class Tile>
  __device__ bool cooperative_update(const key_slice_type* key, const size_type key_length,
                                     const value_slice_type* value, const size_type value_length, const Tile&,
                                     device_allocator_context_type& allocator,
                                     device_reclaimer_context_type&) const {
    return mtb::coop_update<T>(allocator.t, tree_, allocator.cache, key, key_length, value, value_length) ==
           mtb::RES_OK;
  }

  // Reference cooperative_erase (gpu_masstree.hpp:751-971): whether the key
  // was present.
  template <bool concurrent = true, bool do_merge = false, bool pessimistic_merge = false,
            bool do_remove_empty_root = false, class Tile>
  __device__ bool cooperative_erase(const key_slice_type* key, const size_type key_length, const Tile&,
                                    device_allocator_context_type& allocator,
                                    device_reclaimer_context_type&) const {
    mtb::tree_view tv = tree_;
    tv.merge_log = nullptr;
    tv.layer_log = nullptr;
    return mtb::coop_erase<T>(allocator.t, tv, key, key_length) == mtb::RES_OK;
  }

  // Reference cooperative_scan (gpu_masstree.hpp:250-395): up to out_max_count
  // keys from lower_key (inclusive) in key order, stopping after upper_key
  // (inclusive) when use_upper_key; returns the number written.  Result c goes
  // to out_values[c * out_value_max_length ...], out_value_lengths[c],
  // out_keys[c * out_key_max_length ...] and out_key_lengths[c] (each may be
  // null).  The layer stack lives in slabs of the allocator context.
  template <bool use_upper_key, bool concurrent, class Tile>
  __device__ size_type cooperative_scan(const key_slice_type* lower_key, const size_type lower_key_length,
                                        const Tile&, device_allocator_context_type& allocator,
                                        const key_slice_type* upper_key = nullptr,
                                        const size_type upper_key_length = 1, size_type out_max_count = 1,
                                        value_slice_type* out_values = nullptr,
                                        size_type* out_value_lengths = nullptr,
                                        const size_type out_value_max_length = 1,
                                        key_slice_type* out_keys = nullptr, size_type* out_key_lengths = nullptr,
                                        const size_type out_key_max_length = 1) const {
    mtb::scan_out o;
    o.values = out_values;
    o.value_lengths = out_value_lengths;
    o.maxV = out_values ? out_value_max_length : 0u;
    o.keys = out_keys;
    o.key_lengths = out_key_lengths;
    o.maxK = out_key_max_length;
    mtb::scan_frames<T> frames(nullptr, 0u, &allocator.cache);
    return mtb::coop_scan<T, concurrent>(allocator.t, tree_, lower_key, lower_key_length,
                                         use_upper_key && upper_key != nullptr, upper_key, upper_key_length,
                                         out_max_count, o, frames);
  }
};

}  // namespace GpuMasstreeB200
