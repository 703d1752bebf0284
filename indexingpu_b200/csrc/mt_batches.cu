// Many mixed sub-batches in one call (mt_mixed_batches).
//
// The reference serves one host call per batch (include/kernels.hpp:81-103):
// each call pays host launch overhead, an occupancy query, a partition pass
// and the tail of its slowest request.  Here a list of sub-batches (device
// descriptors) is served by
//   1. batches_prepare_kernel: prefix sums of the sub-batch sizes, counters reset;
//   2. batches_partition_kernel: every request of every sub-batch is filed
//      under (sub-batch, class) with class = find / insert / update+erase,
//      optionally split into short and long keys (filled from the two ends of
//      the class's index region, so each class is served short keys first);
//   3. either (default) for every sub-batch its three batches_class_kernel
//      launches side by side on forked streams, joined before the next
//      sub-batch, or (MT_FLAG_PERSISTENT) batches_persistent_kernel: a
//      cooperative grid walks the sub-batches in order with one grid barrier
//      between sub-batches.
// Sub-batch k+1 observes every effect of sub-batch k, as with one host call per
// sub-batch; inside a sub-batch the classes have no order among each other
// (as inside one mixed batch).  Nothing in the call allocates once
// mt_batches_reserve has sized the scratch, and no host value depends on the
// sub-batch contents, so the call can be captured in a CUDA graph and replayed
// with new descriptor contents.
#include <cooperative_groups.h>

#include <algorithm>

#include "mt_internal.cuh"

namespace cg = cooperative_groups;

namespace mtb {

__global__ void batches_prepare_kernel(batches_view b, pool_view p) {
  if (threadIdx.x == 0) {
    uint64_t acc = 0;
    for (uint32_t s = 0; s < b.nsub; ++s) {
      b.offsets[s] = (uint32_t)min(acc, (uint64_t)0xFFFFFFFFu);
      acc += b.sub[s].num_requests;
    }
    b.offsets[b.nsub] = (uint32_t)min(acc, (uint64_t)0xFFFFFFFFu);
    b.status[0] = acc > b.max_total ? 1u : 0u;
    if (acc > b.max_total) record_error(p, ERR_INVALID_ARG);
  }
  for (uint32_t i = threadIdx.x; i < b.nsub * kCountStride; i += blockDim.x) b.counts[i] = 0u;
}

__global__ void batches_partition_kernel(batches_view b) {
  if (b.status[0]) return;
  const uint32_t total = b.offsets[b.nsub];
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < total;
       base += gridDim.x * blockDim.x) {
    const uint32_t g = base + lane;
    const bool valid = g < total;
    uint32_t sb = 0, i = 0, cls = 0, bucket = 0;
    if (valid) {
      sb = find_subbatch(b.offsets, b.nsub, g);
      i = g - b.offsets[sb];
      const mt_subbatch& d = b.sub[sb];
      const uint32_t k = d.request_types[i];
      cls = k == MT_REQ_FIND ? 0u : (k == MT_REQ_INSERT ? 1u : 2u);
      if (b.bucket_keys) {
        const uint32_t kl = d.key_lengths ? d.key_lengths[i] : b.max_key_length;
        bucket = (2u * kl > b.max_key_length) ? 1u : 0u;
      }
    }
    // Lanes filing into the same counter share one atomic.
    const uint32_t key = valid ? (sb * kCountStride + cls * 2u + bucket) : 0xFFFFFFFFu;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key);
    const uint32_t leader = __ffs(peers) - 1u;
    uint32_t first = 0;
    if (valid && lane == leader) first = atomicAdd(b.counts + key, (uint32_t)__popc(peers));
    first = __shfl_sync(0xFFFFFFFFu, first, (int)leader);
    if (valid) {
      const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
      const uint32_t n = b.sub[sb].num_requests;
      uint32_t* region = b.lists + (size_t)cls * b.max_total + b.offsets[sb];
      const uint32_t slot = bucket ? (n - 1u - (first + rank)) : (first + rank);
      region[slot] = i;
    }
  }
}

// Arguments of class cls of sub-batch sb (index region filled from both ends).
MT_DEV batch_args class_args(const batches_view& b, uint32_t sb, uint32_t cls) {
  const mt_subbatch d = b.sub[sb];
  batch_args a{};
  a.types = d.request_types;
  a.keys = d.keys;
  a.key_lengths = d.key_lengths;
  a.values = d.values;
  a.value_lengths_in = d.value_lengths;
  a.value_lengths_out = d.value_lengths;
  a.results = d.results;
  a.index = b.lists + (size_t)cls * b.max_total + b.offsets[sb];
  a.n_dev = b.counts + sb * kCountStride + cls * 2u;
  a.n_back_dev = a.n_dev + 1;
  a.region = d.num_requests;
  a.max_key_length = b.max_key_length;
  a.max_value_length = b.max_value_length;
  return a;
}

// One grid barrier per sub-batch: sub-batch sb+1 starts after every request of
// sub-batch sb has finished; inside a sub-batch the classes flow without one.
template <int TF, int TW>
__global__ void __launch_bounds__(kBlock, MT_MIN_BLOCKS_PER_SM) batches_persistent_kernel(tree_view tv,
                                                                                          batches_view b) {
  if (b.status[0]) return;  // uniform over the grid: no barrier is skipped by a subset
  cg::grid_group grid = cg::this_grid();
  slab_cache<TW> wcache;
  wcache.init(tv.pool, (blockIdx.x * blockDim.x + threadIdx.x) / TW);
  const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  for (uint32_t sb = 0; sb < b.nsub; ++sb) {
    if (b.sub[sb].num_requests >= kClassBarrierMin) {
      // Large sub-batch: one class at a time.
      {
        tile<TF> tf;
        slab_cache<TF> unused;
        serve_requests<TF, OP_FIND, true>(tf, tv, unused, class_args(b, sb, 0u), gtid / TF, nthreads / TF);
      }
      grid.sync();
      tile<TW> tw;
      serve_requests<TW, OP_PASS_INSERT, true>(tw, tv, wcache, class_args(b, sb, 1u), gtid / TW, nthreads / TW);
      grid.sync();
      serve_requests<TW, OP_PASS_UPDERASE, true>(tw, tv, wcache, class_args(b, sb, 2u), gtid / TW, nthreads / TW);
    } else {
      serve_mixed_classes<TF, TW>(tv, wcache, class_args(b, sb, 0u), class_args(b, sb, 1u), class_args(b, sb, 2u));
    }
    grid.sync();
  }
  tile<TW> tw;
  wcache.release(tw, tv.pool);
}

// One class of one sub-batch (the forked form): the class kernels of a
// sub-batch run side by side, each compiled for its class only.
template <int T, int OP>
__global__ void __launch_bounds__(kBlock, min_blocks_for<OP>) batches_class_kernel(tree_view tv, batches_view b,
                                                                                     uint32_t sb) {
  if (b.status[0]) return;
  constexpr uint32_t cls = OP == OP_FIND ? 0u : (OP == OP_PASS_INSERT ? 1u : 2u);
  tile<T> t;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / T;
  const uint32_t num_tiles = (gridDim.x * blockDim.x) / T;
  slab_cache<T> cache;
  cache.init(tv.pool, tile_id);
  serve_requests<T, OP, true>(t, tv, cache, class_args(b, sb, cls), tile_id, num_tiles);
  cache.release(t, tv.pool);
}

}  // namespace mtb

using namespace mtb;

namespace {

template <int T, int OP>
int launch_class(mt_masstree* t, const batches_view& b, uint32_t sb, cudaStream_t s) {
  const void* fn = (const void*)batches_class_kernel<T, OP>;
  int bps = host_max_blocks_per_sm(fn, kBlock, 0);
  if (t->blocks_per_sm > 0) bps = std::min<int>(bps, (int)t->blocks_per_sm);
  batches_class_kernel<T, OP><<<std::max(bps, 1) * t->sms, kBlock, 0, s>>>(t->tv, b, sb);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_CUDA;
}

template <int OP>
int launch_class_tile(mt_masstree* t, uint32_t tile, const batches_view& b, uint32_t sb, cudaStream_t s) {
  switch (tile) {
    case 4: return launch_class<4, OP>(t, b, sb, s);
    case 8: return launch_class<8, OP>(t, b, sb, s);
    case 16: return launch_class<16, OP>(t, b, sb, s);
    default: return launch_class<32, OP>(t, b, sb, s);
  }
}

// Forked form: per sub-batch, the insert class on the caller's stream and the
// find and update/erase classes on the tree's two side streams, joined before
// the next sub-batch starts.
int launch_forked(mt_masstree* t, const batches_view& b, cudaStream_t s) {
  const uint32_t tw = t->write_tile_size <= 16 ? 16u : 32u;
  const uint32_t tu = t->upderase_tile_size ? t->upderase_tile_size : tw;
  for (uint32_t sb = 0; sb < b.nsub; ++sb) {
    int rc = host_fork(t, s);
    if (rc) return rc;
    rc = launch_class_tile<OP_PASS_INSERT>(t, tw, b, sb, s);
    if (!rc) rc = launch_class_tile<OP_FIND>(t, t->tile_size, b, sb, t->side[0]);
    if (!rc) rc = launch_class_tile<OP_PASS_UPDERASE>(t, tu, b, sb, t->side[1]);
    rc = host_join(t, s, rc);
    if (rc) return rc;
  }
  return MT_OK;
}

template <int TF, int TW>
int launch_persistent(mt_masstree* t, const batches_view& b, cudaStream_t s) {
  const void* fn = (const void*)batches_persistent_kernel<TF, TW>;
  int bps = host_max_blocks_per_sm(fn, kBlock, 0);
  if (t->blocks_per_sm > 0) bps = std::min<int>(bps, (int)t->blocks_per_sm);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(bps * t->sms));
  cfg.blockDim = dim3(kBlock);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, batches_persistent_kernel<TF, TW>, t->tv, b);
  return e == cudaSuccess ? MT_OK : MT_ERR_CUDA;
}

template <int TF>
int launch_persistent_tf(mt_masstree* t, const batches_view& b, cudaStream_t s) {
  switch (t->write_tile_size <= 16 ? 16u : 32u) {
    case 16: return launch_persistent<TF, 16>(t, b, s);
    case 32: return launch_persistent<TF, 32>(t, b, s);
    default: return MT_ERR_INVALID_ARG;
  }
}

}  // namespace

extern "C" int mt_batches_reserve(mt_masstree* t, uint32_t max_subbatches, uint64_t max_total_requests) {
  if (!t || max_subbatches == 0 || max_total_requests == 0 || max_total_requests >= 0xFFFFFFFFull)
    return MT_ERR_INVALID_ARG;
  if (max_subbatches <= t->batches_max_sub && max_total_requests <= t->batches_max_total) return MT_OK;
  const uint32_t ms = std::max(max_subbatches, t->batches_max_sub);
  const uint64_t mt = std::max<uint64_t>(max_total_requests, t->batches_max_total);
  if (cudaDeviceSynchronize() != cudaSuccess) return MT_ERR_CUDA;
  if (t->batches_mem) cudaFree(t->batches_mem);
  t->batches_mem = nullptr;
  t->batches_max_sub = 0;
  t->batches_max_total = 0;
  // [status: 32 words][offsets: ms+1][counts: ms*8][lists: 3*mt]
  const size_t words = 32u + (ms + 1u) + (size_t)ms * kCountStride + 3u * mt;
  if (cudaMalloc(&t->batches_mem, words * sizeof(uint32_t)) != cudaSuccess) return MT_ERR_OOM;
  t->batches_max_sub = ms;
  t->batches_max_total = mt;
  return MT_OK;
}

extern "C" int mt_mixed_batches(mt_masstree* t, const mt_subbatch* subbatches, uint32_t num_subbatches,
                                uint32_t max_key_length, uint32_t max_value_length, uint32_t flags, void* stream) {
  if (!t || (num_subbatches && !subbatches) || max_key_length == 0 || max_value_length == 0)
    return MT_ERR_INVALID_ARG;
  if (num_subbatches == 0) return MT_OK;
  if (num_subbatches > t->batches_max_sub || !t->batches_mem) return MT_ERR_INVALID_ARG;
  if (t->tile_size != 4 && t->tile_size != 8 && t->tile_size != 16 && t->tile_size != 32) return MT_ERR_INVALID_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  uint32_t* base = static_cast<uint32_t*>(t->batches_mem);
  batches_view b{};
  b.sub = subbatches;
  b.nsub = num_subbatches;
  b.status = base;
  b.offsets = base + 32;
  b.counts = b.offsets + t->batches_max_sub + 1;
  b.lists = b.counts + (size_t)t->batches_max_sub * kCountStride;
  b.max_total = (uint32_t)t->batches_max_total;
  b.max_key_length = max_key_length;
  b.max_value_length = max_value_length;
  b.bucket_keys = (flags & MT_FLAG_BUCKET_KEYS) ? 1u : 0u;
  int rc = host_launch_reclaim(t, s);
  if (rc) return rc;
  batches_prepare_kernel<<<1, 256, 0, s>>>(b, t->tv.pool);
  if (cudaGetLastError() != cudaSuccess) return MT_ERR_CUDA;
  if (flags & MT_FLAG_GROUP_BY_KEY) {
    const int grc = launch_grouped(t, b, s);
    if (grc != kGroupedUnavailable) return grc;
  }
  batches_partition_kernel<<<t->sms * 4, 256, 0, s>>>(b);
  if (cudaGetLastError() != cudaSuccess) return MT_ERR_CUDA;
  if (!(flags & MT_FLAG_PERSISTENT)) return launch_forked(t, b, s);
  switch (t->tile_size) {
    case 4: return launch_persistent_tf<4>(t, b, s);
    case 8: return launch_persistent_tf<8>(t, b, s);
    case 16: return launch_persistent_tf<16>(t, b, s);
    default: return launch_persistent_tf<32>(t, b, s);
  }
}
