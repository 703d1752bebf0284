// TEST INFRASTRUCTURE: user kernels written against the device API
// (include/mt/device.cuh) the way the reference's README shows it for
// gpu_masstree (README.md:114-166): one cooperative_groups tile per request,
// an allocator context from index.allocator_, a reclaimer context from
// index.reclaimer_, every lane of the tile calling the cooperative function.
// Built into tests/cpp/build/libmt_device_check.so and driven from
// tests/test_gpu_device_api.py through the extern "C" launchers below.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "mt/device.cuh"

namespace cg = cooperative_groups;

namespace {

constexpr int kBlock = 128;

template <class Index>
__device__ uint32_t request_of(const cg::thread_block_tile<Index::tile_size_, cg::thread_block>&) {
  return (blockIdx.x * blockDim.x + threadIdx.x) / Index::tile_size_;
}

template <class Index, bool concurrent>
__global__ void find_kernel(Index index, const uint32_t* keys, const uint32_t* key_lengths, uint32_t* values,
                            uint32_t* value_lengths, uint32_t max_key_length, uint32_t max_value_length,
                            uint32_t num_keys) {
  auto block = cg::this_thread_block();
  auto tile = cg::tiled_partition<Index::tile_size_>(block);
  const uint32_t i = request_of<Index>(tile);
  if (i >= num_keys) return;
  typename Index::device_allocator_context_type allocator{index.allocator_, tile};
  const uint32_t* key = &keys[(size_t)i * max_key_length];
  uint32_t* value = &values[(size_t)i * max_value_length];
  const uint32_t key_length = key_lengths ? key_lengths[i] : max_key_length;
  const uint32_t value_length =
      index.template cooperative_find<concurrent>(key, key_length, value, max_value_length, tile, allocator);
  if (tile.thread_rank() == 0) value_lengths[i] = value_length;
}

// kind: 0 insert, 1 upsert, 2 update, 3 erase.
template <class Index>
__global__ void write_kernel(Index index, int kind, const uint32_t* keys, const uint32_t* key_lengths,
                             const uint32_t* values, const uint32_t* value_lengths, uint32_t max_key_length,
                             uint32_t max_value_length, uint32_t num_keys, uint8_t* results) {
  auto block = cg::this_thread_block();
  auto tile = cg::tiled_partition<Index::tile_size_>(block);
  const uint32_t i = request_of<Index>(tile);
  if (i >= num_keys) return;
  typename Index::device_allocator_context_type allocator{index.allocator_, tile};
  typename Index::device_reclaimer_context_type reclaimer{index.reclaimer_, tile};
  const uint32_t* key = &keys[(size_t)i * max_key_length];
  const uint32_t key_length = key_lengths ? key_lengths[i] : max_key_length;
  const uint32_t* value = values ? &values[(size_t)i * max_value_length] : nullptr;
  const uint32_t value_length = value_lengths ? value_lengths[i] : max_value_length;
  bool ok = false;
  switch (kind) {
    case 0:
      ok = index.template cooperative_insert<false, true>(key, key_length, value, value_length, tile, allocator,
                                                          reclaimer);
      break;
    case 1:
      ok = index.template cooperative_insert<true, true>(key, key_length, value, value_length, tile, allocator,
                                                         reclaimer);
      break;
    case 2:
      ok = index.template cooperative_update<true>(key, key_length, value, value_length, tile, allocator, reclaimer);
      break;
    default:
      ok = index.template cooperative_erase<true, false, false, false>(key, key_length, tile, allocator, reclaimer);
      break;
  }
  if (tile.thread_rank() == 0 && results) results[i] = ok ? 1 : 0;
}

// One kernel that inserts request i and then looks it up again (a fused use of
// the device API: writer and concurrent reader in the same launch).
template <class Index>
__global__ void insert_then_find_kernel(Index index, const uint32_t* keys, const uint32_t* key_lengths,
                                        const uint32_t* values, const uint32_t* value_lengths,
                                        uint32_t max_key_length, uint32_t max_value_length, uint32_t num_keys,
                                        uint8_t* results, uint32_t* found_lengths) {
  auto block = cg::this_thread_block();
  auto tile = cg::tiled_partition<Index::tile_size_>(block);
  const uint32_t i = request_of<Index>(tile);
  if (i >= num_keys) return;
  typename Index::device_allocator_context_type allocator{index.allocator_, tile};
  typename Index::device_reclaimer_context_type reclaimer{index.reclaimer_, tile};
  const uint32_t* key = &keys[(size_t)i * max_key_length];
  const uint32_t key_length = key_lengths ? key_lengths[i] : max_key_length;
  const uint32_t* value = &values[(size_t)i * max_value_length];
  const bool ok = index.template cooperative_insert<false, true>(key, key_length, value, value_lengths[i], tile,
                                                                 allocator, reclaimer);
  uint32_t scratch[1];
  const uint32_t vl = index.template cooperative_find<true>(key, key_length, scratch, 0u, tile, allocator);
  if (tile.thread_rank() == 0) {
    results[i] = ok ? 1 : 0;
    found_lengths[i] = vl;
  }
}

template <class Index, bool use_upper>
__global__ void scan_kernel(Index index, const uint32_t* lower, const uint32_t* lower_lengths,
                            const uint32_t* upper, const uint32_t* upper_lengths, uint32_t max_key_length,
                            uint32_t max_count, uint32_t num_queries, uint32_t* counts, uint32_t* values,
                            uint32_t max_value_length, uint32_t* value_lengths, uint32_t* out_keys,
                            uint32_t* out_key_lengths) {
  auto block = cg::this_thread_block();
  auto tile = cg::tiled_partition<Index::tile_size_>(block);
  const uint32_t q = request_of<Index>(tile);
  if (q >= num_queries) return;
  typename Index::device_allocator_context_type allocator{index.allocator_, tile};
  const size_t mc = max_count;
  const uint32_t c = index.template cooperative_scan<use_upper, true>(
      &lower[(size_t)q * max_key_length], lower_lengths[q], tile, allocator,
      use_upper ? &upper[(size_t)q * max_key_length] : nullptr, use_upper ? upper_lengths[q] : 1u, max_count,
      &values[q * mc * max_value_length], &value_lengths[q * mc], max_value_length,
      &out_keys[q * mc * max_key_length], &out_key_lengths[q * mc], max_key_length);
  if (tile.thread_rank() == 0) counts[q] = c;
}

uint32_t grid_for(uint32_t n, uint32_t tile) {
  const uint64_t threads = (uint64_t)n * tile;
  return (uint32_t)((threads + kBlock - 1) / kBlock);
}

int launched() { return cudaGetLastError() == cudaSuccess ? 0 : MT_ERR_CUDA; }

template <uint32_t T>
int find_t(mt_masstree* tree, const uint32_t* keys, uint32_t maxK, const uint32_t* klens, uint32_t* vals,
           uint32_t maxV, uint32_t* vlens, uint32_t n, int concurrent, cudaStream_t s) {
  using Index = GpuMasstreeB200::gpu_masstree_device<T>;
  const Index index = Index::from(tree);
  if (n == 0) return 0;
  if (concurrent)
    find_kernel<Index, true><<<grid_for(n, T), kBlock, 0, s>>>(index, keys, klens, vals, vlens, maxK, maxV, n);
  else
    find_kernel<Index, false><<<grid_for(n, T), kBlock, 0, s>>>(index, keys, klens, vals, vlens, maxK, maxV, n);
  return launched();
}

template <uint32_t T>
int write_t(mt_masstree* tree, int kind, const uint32_t* keys, uint32_t maxK, const uint32_t* klens,
            const uint32_t* vals, uint32_t maxV, const uint32_t* vlens, uint32_t n, uint8_t* results,
            cudaStream_t s) {
  using Index = GpuMasstreeB200::gpu_masstree_device<T>;
  const Index index = Index::from(tree);
  if (n == 0) return 0;
  write_kernel<Index><<<grid_for(n, T), kBlock, 0, s>>>(index, kind, keys, klens, vals, vlens, maxK, maxV, n,
                                                         results);
  return launched();
}

template <uint32_t T>
int insert_find_t(mt_masstree* tree, const uint32_t* keys, uint32_t maxK, const uint32_t* klens,
                  const uint32_t* vals, uint32_t maxV, const uint32_t* vlens, uint32_t n, uint8_t* results,
                  uint32_t* found, cudaStream_t s) {
  using Index = GpuMasstreeB200::gpu_masstree_device<T>;
  const Index index = Index::from(tree);
  if (n == 0) return 0;
  insert_then_find_kernel<Index><<<grid_for(n, T), kBlock, 0, s>>>(index, keys, klens, vals, vlens, maxK, maxV, n,
                                                                    results, found);
  return launched();
}

template <uint32_t T>
int scan_t(mt_masstree* tree, const uint32_t* lower, const uint32_t* lower_lens, uint32_t maxK, uint32_t max_count,
           uint32_t nq, const uint32_t* upper, const uint32_t* upper_lens, int use_upper, uint32_t* counts,
           uint32_t* vals, uint32_t maxV, uint32_t* vlens, uint32_t* out_keys, uint32_t* out_klens,
           cudaStream_t s) {
  using Index = GpuMasstreeB200::gpu_masstree_device<T>;
  const Index index = Index::from(tree);
  if (nq == 0) return 0;
  if (use_upper)
    scan_kernel<Index, true><<<grid_for(nq, T), kBlock, 0, s>>>(index, lower, lower_lens, upper, upper_lens, maxK,
                                                                 max_count, nq, counts, vals, maxV, vlens,
                                                                 out_keys, out_klens);
  else
    scan_kernel<Index, false><<<grid_for(nq, T), kBlock, 0, s>>>(index, lower, lower_lens, nullptr, nullptr, maxK,
                                                                  max_count, nq, counts, vals, maxV, vlens,
                                                                  out_keys, out_klens);
  return launched();
}

}  // namespace

// Run f<T>() for the tile width given at run time.
template <class F>
int by_tile(uint32_t tile, F f) {
  switch (tile) {
    case 8: return f(std::integral_constant<uint32_t, 8>{});
    case 16: return f(std::integral_constant<uint32_t, 16>{});
    case 32: return f(std::integral_constant<uint32_t, 32>{});
    default: return MT_ERR_INVALID_ARG;
  }
}

extern "C" {

int dev_find(mt_masstree* tree, uint32_t tile, const uint32_t* keys, uint32_t maxK, const uint32_t* klens,
             uint32_t* vals, uint32_t maxV, uint32_t* vlens, uint32_t n, int concurrent, void* stream) {
  return by_tile(tile, [&](auto T) {
    return find_t<decltype(T)::value>(tree, keys, maxK, klens, vals, maxV, vlens, n, concurrent, (cudaStream_t)stream);
  });
}

int dev_write(mt_masstree* tree, uint32_t tile, int kind, const uint32_t* keys, uint32_t maxK,
              const uint32_t* klens, const uint32_t* vals, uint32_t maxV, const uint32_t* vlens, uint32_t n,
              uint8_t* results, void* stream) {
  return by_tile(tile, [&](auto T) {
    return write_t<decltype(T)::value>(tree, kind, keys, maxK, klens, vals, maxV, vlens, n, results,
                                       (cudaStream_t)stream);
  });
}

int dev_insert_then_find(mt_masstree* tree, uint32_t tile, const uint32_t* keys, uint32_t maxK,
                         const uint32_t* klens, const uint32_t* vals, uint32_t maxV, const uint32_t* vlens,
                         uint32_t n, uint8_t* results, uint32_t* found, void* stream) {
  return by_tile(tile, [&](auto T) {
    return insert_find_t<decltype(T)::value>(tree, keys, maxK, klens, vals, maxV, vlens, n, results, found,
                                             (cudaStream_t)stream);
  });
}

int dev_scan(mt_masstree* tree, uint32_t tile, const uint32_t* lower, const uint32_t* lower_lens, uint32_t maxK,
             uint32_t max_count, uint32_t nq, const uint32_t* upper, const uint32_t* upper_lens, int use_upper,
             uint32_t* counts, uint32_t* vals, uint32_t maxV, uint32_t* vlens, uint32_t* out_keys,
             uint32_t* out_klens, void* stream) {
  return by_tile(tile, [&](auto T) {
    return scan_t<decltype(T)::value>(tree, lower, lower_lens, maxK, max_count, nq, upper, upper_lens, use_upper,
                                      counts, vals, maxV, vlens, out_keys, out_klens, (cudaStream_t)stream);
  });
}

}  // extern "C"
