// Batch kernels and the C ABI of libmt_b200.so.
//
// Every host call is one stream-ordered launch of a persistent grid-stride
// kernel (the reference's batch_kernel, include/kernels.hpp:31-103), preceded by
// the reclaim pass that returns slabs retired by earlier calls.  Differences:
//   * the launch shape (blocks per SM from the occupancy API, SM count) is
//     computed once per kernel and cached, not on every call (the reference
//     queries it per call, kernels.hpp:91-99);
//   * a tile serves T requests per round, loading their metadata coalesced
//     (one request per lane) and writing results coalesced;
//   * there is no block-wide barrier per round: reclamation is launch-granular
//     (see mt_pool.cuh).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "mt_internal.cuh"

namespace mtb {

// Split a mixed batch into its finds and its writes (insert/update/erase):
// one atomic per warp and class.  Order inside a class is arbitrary (requests
// of one mixed batch have no defined order).  counts = {finds, writes}.
__global__ void partition_kernel(const uint8_t* types, uint32_t n, uint32_t* find_idx, uint32_t* write_idx,
                                 uint32_t* counts) {
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < n;
       base += gridDim.x * blockDim.x) {
    const uint32_t i = base + lane;
    const bool valid = i < n;
    const bool is_find = valid && types[i] == MT_REQ_FIND;
    const bool is_write = valid && !is_find;
    const uint32_t fm = __ballot_sync(0xFFFFFFFFu, is_find);
    const uint32_t wm = __ballot_sync(0xFFFFFFFFu, is_write);
    uint32_t fb = 0, wb = 0;
    if (lane == 0) {
      if (fm) fb = atomicAdd(counts, (uint32_t)__popc(fm));
      if (wm) wb = atomicAdd(counts + 1, (uint32_t)__popc(wm));
    }
    fb = __shfl_sync(0xFFFFFFFFu, fb, 0);
    wb = __shfl_sync(0xFFFFFFFFu, wb, 0);
    const uint32_t below = (1u << lane) - 1u;
    if (is_find) find_idx[fb + __popc(fm & below)] = i;
    if (is_write) write_idx[wb + __popc(wm & below)] = i;
  }
}

// Split a mixed batch into finds, inserts and updates+erases (one atomic per
// warp and counter).  Each class has an index region of n entries; with
// bucketing, keys longer than half the maximum length fill it from the back,
// so that the tiles of a warp serve keys of similar length (similar paths)
// side by side.  counts[2c] / counts[2c+1] = entries from the front / back of
// class c's region (c = finds, inserts, updates+erases).
__global__ void partition3_kernel(const uint8_t* types, const uint32_t* key_lengths, uint32_t max_key_length,
                                  uint32_t bucket_keys, uint32_t n, uint32_t* find_idx, uint32_t* insert_idx,
                                  uint32_t* upderase_idx, uint32_t* counts) {
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < n;
       base += gridDim.x * blockDim.x) {
    const uint32_t i = base + lane;
    const bool valid = i < n;
    const uint32_t k = valid ? types[i] : 0xFFu;
    const uint32_t c = k == MT_REQ_FIND ? 0u : (k == MT_REQ_INSERT ? 1u : 2u);
    uint32_t bucket = 0;
    if (valid && bucket_keys && key_lengths) bucket = (2u * key_lengths[i] > max_key_length) ? 1u : 0u;
    const uint32_t slot = valid ? c * 2u + bucket : 0xFFu;
    uint32_t m[6], b[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) m[q] = __ballot_sync(0xFFFFFFFFu, slot == (uint32_t)q);
    if (lane == 0) {
#pragma unroll
      for (int q = 0; q < 6; ++q) b[q] = m[q] ? atomicAdd(counts + q, (uint32_t)__popc(m[q])) : 0u;
    }
#pragma unroll
    for (int q = 0; q < 6; ++q) b[q] = __shfl_sync(0xFFFFFFFFu, b[q], 0);
    if (valid) {
      const uint32_t r = reg_select(b, slot) + __popc(reg_select(m, slot) & ((1u << lane) - 1u));
      uint32_t* dst = c == 0 ? find_idx : (c == 1 ? insert_idx : upderase_idx);
      dst[bucket ? n - 1u - r : r] = i;
    }
  }
}

// Update combining.  Updates of one key in one call have no order among each
// other, so all but one of them can be linearised right before the one that
// runs, and report its result: the final value is one of theirs either way.
// Under skewed key choice this turns thousands of serialised updates of a hot
// key (each taking the node lock) into one.  combine_kernel files every valid
// update of the class (or of the whole call) in an open-addressing table keyed
// by a hash of the key; the first request of a key owns its slot, the others
// compare keys and record that request in leader_of.  The batch kernel skips
// them, and combine_results_kernel copies the leader's result.
MT_DEV uint64_t key_hash(const uint32_t* k, uint32_t klen) {
  uint64_t h = 0x9E3779B97F4A7C15ull ^ klen;
  for (uint32_t q = 0; q < klen; ++q) {
    h = (h ^ k[q]) * 0xFF51AFD7ED558CCDull;
    h ^= h >> 32;
  }
  h *= 0xC4CEB9FE1A85EC53ull;
  return h ^ (h >> 29);
}

MT_DEV uint32_t class_request(const batch_args& a, uint32_t pos, uint32_t nf, uint32_t nb) {
  return a.index ? a.index[pos < nf ? pos : a.region - nb + (pos - nf)] : pos;
}

__global__ void combine_kernel(batch_args a, uint32_t* table, uint32_t mask, uint32_t* leader_of) {
  const uint32_t nf = a.n_dev ? *a.n_dev : a.n;
  const uint32_t nb = a.n_back_dev ? *a.n_back_dev : 0u;
  for (uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x; pos < nf + nb; pos += gridDim.x * blockDim.x) {
    const uint32_t i = class_request(a, pos, nf, nb);
    if (a.types && a.types[i] != MT_REQ_UPDATE) continue;
    const uint32_t klen = a.key_lengths ? a.key_lengths[i] : a.max_key_length;
    const uint32_t vlen = a.value_lengths_in ? a.value_lengths_in[i] : a.max_value_length;
    if (klen == 0u || klen > a.max_key_length || vlen > a.max_value_length) continue;  // reported when served
    const uint32_t* k = a.keys + (size_t)i * a.max_key_length;
    uint32_t slot = (uint32_t)key_hash(k, klen) & mask;
    for (uint32_t probe = 0; probe <= mask; ++probe) {
      const uint32_t j = atomicCAS(table + slot, kInvalid, i);
      if (j == kInvalid) break;  // i leads its key
      const uint32_t jl = a.key_lengths ? a.key_lengths[j] : a.max_key_length;
      bool same = jl == klen;
      const uint32_t* kj = a.keys + (size_t)j * a.max_key_length;
      for (uint32_t q = 0; same && q < klen; ++q) same = kj[q] == k[q];
      if (same) {
        leader_of[i] = j;
        break;
      }
      slot = (slot + 1u) & mask;
    }
  }
}

__global__ void combine_results_kernel(batch_args a, const uint32_t* leader_of) {
  const uint32_t nf = a.n_dev ? *a.n_dev : a.n;
  const uint32_t nb = a.n_back_dev ? *a.n_back_dev : 0u;
  for (uint32_t pos = blockIdx.x * blockDim.x + threadIdx.x; pos < nf + nb; pos += gridDim.x * blockDim.x) {
    const uint32_t i = class_request(a, pos, nf, nb);
    const uint32_t j = leader_of[i];
    if (j != kInvalid) a.results[i] = a.results[j];
  }
}

template <int T, int OP, bool CONC>
__global__ void __launch_bounds__(kBlock, min_blocks_for<OP>) batch_kernel(tree_view tv, batch_args a) {
  tile<T> t;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / T;
  const uint32_t num_tiles = (gridDim.x * blockDim.x) / T;
  slab_cache<T> cache;
  cache.init(tv.pool, tile_id);
  serve_requests<T, OP, CONC>(t, tv, cache, a, tile_id, num_tiles);
  cache.release(t, tv.pool);
}

template <int T, bool CONC>
__global__ void __launch_bounds__(kBlock, MT_MIN_BLOCKS_PER_SM) scan_kernel(tree_view tv, scan_args a) {
  tile<T> t;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / T;
  const uint32_t num_tiles = (gridDim.x * blockDim.x) / T;
  // Layer frames: kScanDepth per tile in the tree's scratch, deeper ones
  // spill to slabs from the tile's cache.
  slab_cache<T> cache;
  cache.init(tv.pool, tile_id);
  scan_frames<T> frames(a.frames + (size_t)tile_id * kScanDepth, kScanDepth, &cache);
  // Queries per tile and round: T on large batches, fewer on small ones so that
  // every tile gets work (as in serve_requests).
  const uint32_t per = max(1u, min((uint32_t)T, (a.n + num_tiles - 1u) / num_tiles));
  for (uint32_t base = tile_id * per; base < a.n; base += num_tiles * per) {
    if (t.shfl((uint32_t)(t.leader() && fatal_error(tv.pool)), 0)) break;
    const uint32_t i = base + t.rank;
    const bool valid = t.rank < per && i < a.n;
    uint32_t llen = 0, ulen = 0, cnt = 0;
    if (valid) {
      llen = a.lower_lengths ? a.lower_lengths[i] : a.max_key_length;
      ulen = a.upper_lengths ? a.upper_lengths[i] : a.max_key_length;
    }
    const bool bad = valid && (llen > a.max_key_length || (a.use_upper && ulen > a.max_key_length));
    if (t.any(bad) && bad) record_error(tv.pool, ERR_INVALID_ARG, MT_AT(SRC_CAPI));
    const uint32_t nreq = min(per, a.n - base);
    for (uint32_t r = 0; r < nreq; ++r) {
      if (t.shfl((uint32_t)bad, (int)r)) continue;
      const uint32_t q = base + r;
      const uint32_t ll = t.shfl(llen, (int)r);
      const uint32_t ul = t.shfl(ulen, (int)r);
      scan_out o;
      const size_t mc = a.max_count;
      o.values = a.values ? a.values + (size_t)q * mc * a.max_value_length : nullptr;
      o.value_lengths = a.value_lengths ? a.value_lengths + (size_t)q * mc : nullptr;
      o.maxV = a.max_value_length;
      o.keys = a.out_keys ? a.out_keys + (size_t)q * mc * a.max_key_length : nullptr;
      o.key_lengths = a.out_key_lengths ? a.out_key_lengths + (size_t)q * mc : nullptr;
      o.maxK = a.max_key_length;
      const uint32_t* lower = a.lower + (size_t)q * a.max_key_length;
      const uint32_t* upper = a.upper ? a.upper + (size_t)q * a.max_key_length : nullptr;
      const uint32_t c = coop_scan<T, CONC>(t, tv, lower, ll, a.use_upper != 0u && upper != nullptr, upper, ul,
                                           a.max_count, o, frames);
      if (t.rank == r) cnt = c;
    }
    if (valid && a.counts) a.counts[i] = cnt;
  }
  cache.release(t, tv.pool);
}


// Line-atomicity self-test: writer tiles publish whole 128-byte lines whose
// words all carry one stamp, reader tiles load lines the way node loads do
// and count lines whose words disagree (a torn read).  Both loops are bounded.
template <int T>
__global__ void line_atomicity_kernel(uint32_t* lines, uint32_t nlines, uint32_t iters,
                                      unsigned long long* reads, unsigned long long* torn) {
  tile<T> t;
  constexpr int W = 32 / T;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / T;
  const bool writer = (tile_id & 1u) == 0u;
  unsigned long long my_reads = 0, my_torn = 0;
  uint32_t x = tile_id * 0x9E3779B1u + 1u;
  for (uint32_t it = 0; it < iters; ++it) {
    x ^= x << 13; x ^= x >> 17; x ^= x << 5;
    const uint32_t line = t.shfl(x, 0) % nlines;
    uint32_t* base = lines + (size_t)line * 32u + t.rank * W;
    uint32_t w[W];
    if (writer) {
      const uint32_t stamp = (tile_id << 12) ^ it;
#pragma unroll
      for (int k = 0; k < W; ++k) w[k] = stamp;
      t.sync();
      store_words<W, st_order::RELEASE>(base, w);
    } else {
      load_words<W, kConc>(base, w);
      uint32_t lo = w[0], hi = w[0];
#pragma unroll
      for (int k = 1; k < W; ++k) { lo = min(lo, w[k]); hi = max(hi, w[k]); }
      lo = t.min_all(lo);
      hi = __reduce_max_sync(t.mask, hi);
      my_reads += 1;
      my_torn += (lo != hi) ? 1 : 0;
    }
  }
  if (t.leader() && !writer) {
    atomicAdd(reads, my_reads);
    atomicAdd(torn, my_torn);
  }
}

// Return slabs retired by earlier launches to their shard's free stack.
__global__ void reclaim_kernel(pool_view p) {
  for (uint32_t s = blockIdx.x; s < p.num_shards; s += gridDim.x) {
    __shared__ int top, n;
    if (threadIdx.x == 0) {
      top = max(*p.top(s), 0);
      n = *p.limbo_count(s);
      if (top + n > (int)p.shard_slabs) {
        record_error(p, ERR_CORRUPT, MT_AT(SRC_CAPI));
        n = 0;
      }
    }
    __syncthreads();
    uint32_t* stack = p.free_stack + (size_t)s * p.shard_slabs;
    const uint32_t* limbo = p.limbo + (size_t)s * p.shard_slabs;
    for (int i = threadIdx.x; i < n; i += blockDim.x) stack[top + i] = limbo[i];
    __syncthreads();
    if (threadIdx.x == 0) {
      *p.top(s) = top + n;
      *p.limbo_count(s) = 0;
    }
    __syncthreads();
  }
}

}  // namespace mtb

namespace mtb {
bool host_valid_tile(uint32_t ts) { return ts == 4 || ts == 8 || ts == 16 || ts == 32; }
int host_max_blocks_per_sm(const void* fn, int block, size_t smem) {
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, block, smem) != cudaSuccess || b <= 0) b = 1;
  return b;
}
// Make the tree's two side streams wait for the work queued so far on s.
int host_fork(mt_masstree* t, cudaStream_t s) {
  if (!t->ev_fork) {
    bool ok = cudaEventCreateWithFlags(&t->ev_fork, cudaEventDisableTiming) == cudaSuccess;
    for (int k = 0; k < 2 && ok; ++k)
      ok = cudaStreamCreateWithFlags(&t->side[k], cudaStreamNonBlocking) == cudaSuccess &&
           cudaEventCreateWithFlags(&t->ev_join[k], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) return MT_ERR_CUDA;
  }
  if (cudaEventRecord(t->ev_fork, s) != cudaSuccess) return MT_ERR_CUDA;
  for (int k = 0; k < 2; ++k)
    if (cudaStreamWaitEvent(t->side[k], t->ev_fork, 0) != cudaSuccess) return MT_ERR_CUDA;
  return MT_OK;
}

// Make s wait for the side streams.  Called after a fork even when a launch
// failed (rc != MT_OK, returned unchanged), so that the side streams never run
// ahead of the caller's stream.
int host_join(mt_masstree* t, cudaStream_t s, int rc) {
  for (int k = 0; k < 2; ++k) {
    if (cudaEventRecord(t->ev_join[k], t->side[k]) != cudaSuccess ||
        cudaStreamWaitEvent(s, t->ev_join[k], 0) != cudaSuccess)
      rc = rc ? rc : MT_ERR_CUDA;
  }
  return rc;
}

int host_launch_reclaim(mt_masstree* t, cudaStream_t s) {
  reclaim_kernel<<<kShards, 256, 0, s>>>(t->tv.pool);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_CUDA;
}
}  // namespace mtb

// ------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------

using namespace mtb;

namespace {

struct launch_cache {
  std::mutex mu;
  std::unordered_map<const void*, int> bps;
};
launch_cache& lcache() {
  static launch_cache c;
  return c;
}

int max_blocks_per_sm(const void* fn) {
  auto& c = lcache();
  std::lock_guard<std::mutex> g(c.mu);
  auto it = c.bps.find(fn);
  if (it != c.bps.end()) return it->second;
  int b = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, kBlock, 0) != cudaSuccess || b <= 0) b = 1;
  c.bps.emplace(fn, b);
  return b;
}

int grid_for(const mt_masstree* t, const void* fn) {
  int b = max_blocks_per_sm(fn);
  if (t->blocks_per_sm > 0) b = std::min<int>(b, (int)t->blocks_per_sm);
  return b * t->sms;
}

int cuda_status(cudaError_t e) { return e == cudaSuccess ? MT_OK : MT_ERR_CUDA; }

int launch_reclaim(mt_masstree* t, cudaStream_t s) {
  reclaim_kernel<<<kShards, 256, 0, s>>>(t->tv.pool);
  return cuda_status(cudaGetLastError());
}

template <int T, int OP, bool CONC>
int launch_batch_t(mt_masstree* t, const batch_args& a, cudaStream_t s) {
  const void* fn = (const void*)batch_kernel<T, OP, CONC>;
  batch_kernel<T, OP, CONC><<<grid_for(t, fn), kBlock, 0, s>>>(t->tv, a);
  return cuda_status(cudaGetLastError());
}

template <int OP, bool CONC>
int launch_batch_tile(mt_masstree* t, uint32_t tile, const batch_args& a, cudaStream_t s) {
  switch (tile) {
    case 4: return launch_batch_t<4, OP, CONC>(t, a, s);
    case 8: return launch_batch_t<8, OP, CONC>(t, a, s);
    case 16: return launch_batch_t<16, OP, CONC>(t, a, s);
    case 32: return launch_batch_t<32, OP, CONC>(t, a, s);
    default: return MT_ERR_INVALID_ARG;
  }
}

template <int OP, bool CONC>
int launch_batch(mt_masstree* t, const batch_args& a, cudaStream_t s) {
  if (a.n == 0) return MT_OK;
  int rc = launch_reclaim(t, s);
  if (rc) return rc;
  return launch_batch_tile<OP, CONC>(t, OP == OP_FIND ? t->tile_size : t->write_tile_size, a, s);
}

// Slots of the update-combining table for n requests: a power of two of at
// least 2n (load factor at most one half).
uint32_t combine_slots(uint32_t n) {
  uint32_t p = 64;
  while (p < 2u * n && p < (1u << 31)) p <<= 1;
  return p;
}

// Index scratch for split mixed batches (grown on demand, kept).
int ensure_split_scratch(mt_masstree* t, uint32_t n, cudaStream_t s) {
  if (n <= t->split_cap) return MT_OK;
  if (cudaStreamSynchronize(s) != cudaSuccess) return MT_ERR_CUDA;
  if (t->split_idx) cudaFree(t->split_idx);
  t->split_idx = nullptr;
  t->split_cap = 0;
  // [counts(32 words, one line)] [find indices n] [insert indices n] [update/erase indices n]
  // [leader_of n] [combining table combine_slots(n)]
  if (cudaMalloc(&t->split_idx, (32u + 4ull * n + combine_slots(n)) * sizeof(uint32_t)) != cudaSuccess)
    return MT_ERR_OOM;
  t->split_cap = n;
  return MT_OK;
}

// Combine the updates among the requests `a` describes (a class of a mixed
// batch, or a whole update call) on stream s; returns a.leader_of for the batch
// kernel (nullptr when there is nothing to combine into).
int launch_combine(mt_masstree* t, batch_args& a, uint32_t n, cudaStream_t s) {
  uint32_t* leader_of = t->split_idx + 32 + 3ull * t->split_cap;
  uint32_t* table = leader_of + t->split_cap;
  const uint32_t slots = combine_slots(n);
  if (cudaMemsetAsync(leader_of, 0xFF, (size_t)n * sizeof(uint32_t), s) != cudaSuccess ||
      cudaMemsetAsync(table, 0xFF, (size_t)slots * sizeof(uint32_t), s) != cudaSuccess)
    return MT_ERR_CUDA;
  combine_kernel<<<std::max(1, std::min(t->sms * 8, (int)((n + 255) / 256))), 256, 0, s>>>(a, table, slots - 1u,
                                                                                           leader_of);
  if (cudaGetLastError() != cudaSuccess) return MT_ERR_CUDA;
  a.leader_of = leader_of;
  return MT_OK;
}

int launch_combine_results(mt_masstree* t, const batch_args& a, uint32_t n, cudaStream_t s) {
  if (!a.results || !a.leader_of) return MT_OK;
  combine_results_kernel<<<std::max(1, std::min(t->sms * 8, (int)((n + 255) / 256))), 256, 0, s>>>(a, a.leader_of);
  return cuda_status(cudaGetLastError());
}

int launch_mixed_split(mt_masstree* t, batch_args a, bool bucket_keys, cudaStream_t s) {
  if (a.n == 0) return MT_OK;
  int rc = ensure_split_scratch(t, a.n, s);
  if (rc) return rc;
  rc = launch_reclaim(t, s);
  if (rc) return rc;
  uint32_t* counts = t->split_idx;
  uint32_t* find_idx = t->split_idx + 32;
  uint32_t* insert_idx = find_idx + a.n;
  uint32_t* upderase_idx = insert_idx + a.n;
  if (cudaMemsetAsync(counts, 0, 6 * sizeof(uint32_t), s) != cudaSuccess) return MT_ERR_CUDA;
  partition3_kernel<<<std::max(1, std::min(t->sms * 8, (int)((a.n + 255) / 256))), 256, 0, s>>>(
      a.types, a.key_lengths, a.max_key_length, bucket_keys ? 1u : 0u, a.n, find_idx, insert_idx, upderase_idx,
      counts);
  if (cudaGetLastError() != cudaSuccess) return MT_ERR_CUDA;
  batch_args f = a, i = a, u = a;
  uint32_t* idx[3] = {find_idx, insert_idx, upderase_idx};
  batch_args* cls[3] = {&f, &i, &u};
  for (int c = 0; c < 3; ++c) {
    cls[c]->index = idx[c];
    cls[c]->n_dev = counts + 2 * c;
    cls[c]->n_back_dev = counts + 2 * c + 1;
    cls[c]->region = a.n;
  }
  // One launch per class, each compiled for its class only.
  // The classes of one mixed batch have no order among each other, so they
  // go to three streams (the caller's and two of the tree's, forked and
  // joined by events): the blocks of one class fill the SMs that another
  // class's tail leaves idle.
  rc = host_fork(t, s);
  if (rc) return rc;
  // Write classes run with 16- or 32-lane tiles (narrower write tiles, allowed
  // for plain insert/update/erase calls, are widened to 16 here).
  const uint32_t tw = t->write_tile_size <= 16 ? 16u : 32u;
  const uint32_t tu = t->upderase_tile_size ? t->upderase_tile_size : tw;
  rc = launch_batch_tile<OP_PASS_INSERT, true>(t, tw, i, s);
  if (!rc) rc = launch_batch_tile<OP_FIND, true>(t, t->tile_size, f, t->side[0]);
  if (!rc) rc = launch_combine(t, u, a.n, t->side[1]);
  if (!rc) rc = launch_batch_tile<OP_PASS_UPDERASE, true>(t, tu, u, t->side[1]);
  if (!rc) rc = launch_combine_results(t, u, a.n, t->side[1]);
  return host_join(t, s, rc);
}

template <int T, bool CONC>
int launch_scan_t(mt_masstree* t, scan_args a, cudaStream_t s) {
  const void* fn = (const void*)scan_kernel<T, CONC>;
  const int grid = grid_for(t, fn);
  const size_t tiles = (size_t)grid * kBlock / T;
  if (tiles > t->frames_tiles) {
    // Scan frames: grown on demand, kept for later calls.
    cudaStreamSynchronize(s);
    if (t->frames) cudaFree(t->frames);
    t->frames = nullptr;
    t->frames_tiles = 0;
    if (cudaMalloc(&t->frames, tiles * kScanDepth * sizeof(scan_frame)) != cudaSuccess) return MT_ERR_CUDA;
    t->frames_tiles = tiles;
  }
  a.frames = t->frames;
  scan_kernel<T, CONC><<<grid, kBlock, 0, s>>>(t->tv, a);
  return cuda_status(cudaGetLastError());
}

template <bool CONC>
int launch_scan(mt_masstree* t, const scan_args& a, cudaStream_t s) {
  switch (t->scan_tile_size ? t->scan_tile_size : t->tile_size) {
    case 4: return launch_scan_t<4, CONC>(t, a, s);
    case 8: return launch_scan_t<8, CONC>(t, a, s);
    case 16: return launch_scan_t<16, CONC>(t, a, s);
    case 32: return launch_scan_t<32, CONC>(t, a, s);
    default: return MT_ERR_INVALID_ARG;
  }
}

bool valid_tile(uint32_t ts) { return host_valid_tile(ts); }

int create_impl(mt_masstree** out, uint64_t pool_bytes, uint32_t tile_size) {
  if (!out || !valid_tile(tile_size)) return MT_ERR_INVALID_ARG;
  *out = nullptr;
  auto* t = new (std::nothrow) mt_masstree();
  if (!t) return MT_ERR_OOM;
  t->tile_size = tile_size;
  t->write_tile_size = tile_size;
  if (cudaGetDevice(&t->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&t->sms, cudaDevAttrMultiProcessorCount, t->device) != cudaSuccess) {
    delete t;
    return MT_ERR_CUDA;
  }
  // Per slab: 128 B node + 4 B free-stack entry + 4 B limbo entry.
  uint64_t slabs = pool_bytes / (128u + 8u);
  slabs = std::min<uint64_t>(slabs, 0xFFFFFF00ull);
  const uint32_t shard_slabs = (uint32_t)(slabs / kShards);
  if (shard_slabs < 64) { delete t; return MT_ERR_INVALID_ARG; }
  const uint64_t nslabs = (uint64_t)shard_slabs * kShards;
  const size_t slab_bytes = nslabs * 128u;
  const size_t stack_bytes = nslabs * 4u;
  const size_t ctr_bytes = (size_t)kShards * 3u * kCtrStride * sizeof(int);
  const size_t err_bytes = 128;
  const size_t total = slab_bytes + 2 * stack_bytes + ctr_bytes + err_bytes;
  if (cudaMalloc(&t->mem, total) != cudaSuccess) { delete t; return MT_ERR_OOM; }
  char* base = (char*)t->mem;
  pool_view& p = t->tv.pool;
  p.slabs = (uint32_t*)base;
  p.free_stack = (uint32_t*)(base + slab_bytes);
  p.limbo = (uint32_t*)(base + slab_bytes + stack_bytes);
  p.ctr = (int*)(base + slab_bytes + 2 * stack_bytes);
  p.err = (uint32_t*)(base + slab_bytes + 2 * stack_bytes + ctr_bytes);
  p.num_slabs = (uint32_t)nslabs;
  p.num_shards = kShards;
  p.shard_slabs = shard_slabs;
  p.lock_spins = kLockSpins;
  cudaError_t e = cudaMemset(p.ctr, 0, ctr_bytes + err_bytes);
  // Root of trie layer 0 = slab 0 (shard 0's bump pointer starts past it).
  uint32_t root_img[32] = {0};
  root_img[WORD_HIGH] = 0xFFFFFFFFu;
  root_img[WORD_SIB] = kInvalid;
  root_img[WORD_META] = META_BORDER | META_ROOT;
  root_img[WORD_KS] = 0u;
  root_img[WORD_CSUM] = node_checksum(root_img);
  const int one = 1;
  if (e == cudaSuccess) e = cudaMemcpy(p.slabs, root_img, sizeof(root_img), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(p.bump(0), &one, sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMallocHost(&t->h_err, 4 * sizeof(uint32_t));
  if (e != cudaSuccess) {
    cudaFree(t->mem);
    delete t;
    return MT_ERR_CUDA;
  }
  t->tv.root = 0;
  *out = t;
  return MT_OK;
}

}  // namespace

namespace mtb {
int host_launch_insert(mt_masstree* t, const batch_args& a, bool upsert, cudaStream_t s) {
  return upsert ? launch_batch<OP_UPSERT, true>(t, a, s) : launch_batch<OP_INSERT, true>(t, a, s);
}
}  // namespace mtb

namespace {
// Whether the tree holds nothing: one slab in use (the root) and a root
// without entries (waits for the device).
bool tree_is_empty(mt_masstree* t) {
  mt_stats_t st{};
  if (mt_stats(t, &st) != MT_OK || st.used_slabs != 1u || st.limbo_slabs != 0u) return false;
  uint32_t meta = 0;
  if (cudaMemcpy(&meta, t->tv.pool.addr(t->tv.root) + WORD_META, sizeof(meta), cudaMemcpyDeviceToHost) !=
      cudaSuccess)
    return false;
  return (meta & META_COUNT) == 0u;
}
}  // namespace

extern "C" {

int mt_create(mt_masstree** out, float pool_ratio, uint32_t tile_size) {
  if (!(pool_ratio > 0.0f && pool_ratio <= 1.0f)) return MT_ERR_INVALID_ARG;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return MT_ERR_CUDA;
  return create_impl(out, (uint64_t)((double)free_b * (double)pool_ratio), tile_size);
}

int mt_create_bytes(mt_masstree** out, uint64_t pool_bytes, uint32_t tile_size) {
  return create_impl(out, pool_bytes, tile_size);
}

int mt_destroy(mt_masstree* t) {
  if (!t) return MT_ERR_INVALID_ARG;
  cudaDeviceSynchronize();
  if (t->frames) cudaFree(t->frames);
  if (t->split_idx) cudaFree(t->split_idx);
  if (t->batches_mem) cudaFree(t->batches_mem);
  if (t->grouped_mem) cudaFree(t->grouped_mem);
  if (t->merge_log) cudaFree(t->merge_log);
  if (t->layer_log) cudaFree(t->layer_log);
  host_pipe_free(t);
  if (t->mem) cudaFree(t->mem);
  if (t->h_err) cudaFreeHost(t->h_err);
  for (int k = 0; k < 2; ++k) {
    if (t->side[k]) cudaStreamDestroy(t->side[k]);
    if (t->ev_join[k]) cudaEventDestroy(t->ev_join[k]);
  }
  if (t->ev_fork) cudaEventDestroy(t->ev_fork);
  delete t;
  return MT_OK;
}

int mt_set_tile_size(mt_masstree* t, uint32_t ts) {
  if (!t || !valid_tile(ts)) return MT_ERR_INVALID_ARG;
  t->tile_size = ts;
  t->write_tile_size = ts;
  return MT_OK;
}

int mt_set_write_tile_size(mt_masstree* t, uint32_t ts) {
  if (!t || !valid_tile(ts)) return MT_ERR_INVALID_ARG;
  t->write_tile_size = ts;
  return MT_OK;
}

int mt_set_scan_tile_size(mt_masstree* t, uint32_t ts) {
  if (!t || (ts != 0 && !valid_tile(ts))) return MT_ERR_INVALID_ARG;
  t->scan_tile_size = ts;
  return MT_OK;
}

int mt_set_lock_wait(mt_masstree* t, uint32_t attempts) {
  if (!t || attempts == 0) return MT_ERR_INVALID_ARG;
  t->tv.pool.lock_spins = attempts;
  return MT_OK;
}

int mt_inject_node_lock(mt_masstree* t, uint32_t slab, int locked) {
  if (!t || !t->tv.pool.valid(slab)) return MT_ERR_INVALID_ARG;
  if (cudaDeviceSynchronize() != cudaSuccess) return MT_ERR_CUDA;
  uint32_t* mw = t->tv.pool.addr(slab) + WORD_META;
  uint32_t meta = 0;
  if (cudaMemcpy(&meta, mw, sizeof(meta), cudaMemcpyDeviceToHost) != cudaSuccess) return MT_ERR_CUDA;
  // The LOCK bit is outside the node checksum, so the image stays valid.
  meta = locked ? (meta | META_LOCK) : (meta & ~META_LOCK);
  return cuda_status(cudaMemcpy(mw, &meta, sizeof(meta), cudaMemcpyHostToDevice));
}

int mt_set_upderase_tile_size(mt_masstree* t, uint32_t ts) {
  if (!t || (ts != 0 && !valid_tile(ts))) return MT_ERR_INVALID_ARG;
  t->upderase_tile_size = ts;
  return MT_OK;
}

int mt_set_blocks_per_sm(mt_masstree* t, uint32_t b) {
  if (!t) return MT_ERR_INVALID_ARG;
  t->blocks_per_sm = b;
  return MT_OK;
}

int mt_find(mt_masstree* t, const uint32_t* keys, uint32_t maxK, const uint32_t* klens, uint32_t* values,
            uint32_t maxV, uint32_t* vlens, uint32_t n, uint32_t flags, void* stream) {
  if (!t || (n && (!keys || !vlens || maxK == 0))) return MT_ERR_INVALID_ARG;
  batch_args a{};
  a.keys = keys; a.key_lengths = klens; a.values = values; a.value_lengths_out = vlens;
  a.max_key_length = maxK; a.max_value_length = values ? maxV : 0u; a.n = n;
  cudaStream_t s = (cudaStream_t)stream;
  return (flags & MT_FLAG_CONCURRENT) ? launch_batch<OP_FIND, true>(t, a, s) : launch_batch<OP_FIND, false>(t, a, s);
}

int mt_insert(mt_masstree* t, const uint32_t* keys, uint32_t maxK, const uint32_t* klens, const uint32_t* values,
              uint32_t maxV, const uint32_t* vlens, uint32_t n, bool* results, uint32_t flags, void* stream) {
  if (!t || (n && (!keys || !values || maxK == 0))) return MT_ERR_INVALID_ARG;
  batch_args a{};
  a.keys = keys; a.key_lengths = klens; a.values = const_cast<uint32_t*>(values); a.value_lengths_in = vlens;
  a.results = results; a.max_key_length = maxK; a.max_value_length = maxV; a.n = n;
  cudaStream_t s = (cudaStream_t)stream;
  const bool upsert = (flags & MT_FLAG_UPDATE_IF_EXISTS) != 0;
  // The emptiness check waits for the device: only until an insert call
  // finds the tree holding keys (erasing every key later forgoes the build).
  if (n >= kBulkMin && t->maybe_empty) {
    const bool empty = tree_is_empty(t);
    t->maybe_empty = false;
    if (empty) {
      const int rc = host_bulk_insert(t, a, upsert, s);
      if (rc != kBulkDeclined) return rc;
    }
  }
  if (n) t->maybe_empty = false;
  return upsert ? launch_batch<OP_UPSERT, true>(t, a, s) : launch_batch<OP_INSERT, true>(t, a, s);
}

int mt_update(mt_masstree* t, const uint32_t* keys, uint32_t maxK, const uint32_t* klens, const uint32_t* values,
              uint32_t maxV, const uint32_t* vlens, uint32_t n, bool* results, uint32_t flags, void* stream) {
  (void)flags;
  if (!t || (n && (!keys || !values || maxK == 0))) return MT_ERR_INVALID_ARG;
  batch_args a{};
  a.keys = keys; a.key_lengths = klens; a.values = const_cast<uint32_t*>(values); a.value_lengths_in = vlens;
  a.results = results; a.max_key_length = maxK; a.max_value_length = maxV; a.n = n;
  const cudaStream_t s = (cudaStream_t)stream;
  if (n < 2) return launch_batch<OP_UPDATE, true>(t, a, s);
  int rc = ensure_split_scratch(t, n, s);
  if (!rc) rc = launch_combine(t, a, n, s);
  if (!rc) rc = launch_batch<OP_UPDATE, true>(t, a, s);
  if (!rc) rc = launch_combine_results(t, a, n, s);
  return rc;
}

int mt_erase(mt_masstree* t, const uint32_t* keys, uint32_t maxK, const uint32_t* klens, uint32_t n,
             bool* results, uint32_t flags, void* stream) {
  if (!t || (n && (!keys || maxK == 0))) return MT_ERR_INVALID_ARG;
  batch_args a{};
  a.keys = keys; a.key_lengths = klens; a.results = results; a.max_key_length = maxK; a.n = n;
  const cudaStream_t s = (cudaStream_t)stream;
  if (!(flags & (MT_FLAG_MERGE | MT_FLAG_REMOVE_EMPTY_LAYERS))) return launch_batch<OP_ERASE, true>(t, a, s);
  const int rc = host_merge_begin(t, s, flags);
  if (rc) return rc;
  return host_merge_end(t, s, launch_batch<OP_ERASE, true>(t, a, s));
}

int mt_mixed_batch(mt_masstree* t, const uint8_t* types, const uint32_t* keys, uint32_t maxK,
                   const uint32_t* klens, uint32_t* values, uint32_t maxV, uint32_t* vlens, bool* results,
                   uint32_t n, uint32_t flags, void* stream) {
  if (!t || (n && (!types || !keys || !values || !vlens || maxK == 0 || maxV == 0))) return MT_ERR_INVALID_ARG;
  batch_args a{};
  a.types = types; a.keys = keys; a.key_lengths = klens; a.values = values;
  a.value_lengths_in = vlens; a.value_lengths_out = vlens; a.results = results;
  a.max_key_length = maxK; a.max_value_length = maxV; a.n = n;
  const cudaStream_t s = (cudaStream_t)stream;
  auto run = [&] {
    if (flags & MT_FLAG_SINGLE_PASS) return launch_batch<OP_MIXED, true>(t, a, s);
    return launch_mixed_split(t, a, (flags & MT_FLAG_BUCKET_KEYS) != 0, s);
  };
  if (!(flags & (MT_FLAG_MERGE | MT_FLAG_REMOVE_EMPTY_LAYERS))) return run();
  const int rc = host_merge_begin(t, s, flags);
  if (rc) return rc;
  return host_merge_end(t, s, run());
}

int mt_scan(mt_masstree* t, const uint32_t* lower, const uint32_t* lower_lens, uint32_t maxK, uint32_t max_count,
            uint32_t nq, const uint32_t* upper, const uint32_t* upper_lens, uint32_t* counts, uint32_t* values,
            uint32_t maxV, uint32_t* vlens, uint32_t* out_keys, uint32_t* out_klens, uint32_t flags,
            void* stream) {
  if (!t || (nq && (!lower || maxK == 0))) return MT_ERR_INVALID_ARG;
  if ((flags & MT_FLAG_USE_UPPER_KEY) && nq && !upper) return MT_ERR_INVALID_ARG;
  if (nq == 0) return MT_OK;
  cudaStream_t s = (cudaStream_t)stream;
  int rc = launch_reclaim(t, s);
  if (rc) return rc;
  scan_args a{};
  a.lower = lower; a.lower_lengths = lower_lens; a.upper = upper; a.upper_lengths = upper_lens;
  a.counts = counts; a.values = values; a.value_lengths = vlens; a.out_keys = out_keys;
  a.out_key_lengths = out_klens; a.max_key_length = maxK; a.max_value_length = values ? maxV : 0u;
  a.max_count = max_count; a.n = nq; a.use_upper = (flags & MT_FLAG_USE_UPPER_KEY) ? 1u : 0u;
  return (flags & MT_FLAG_CONCURRENT) ? launch_scan<true>(t, a, s) : launch_scan<false>(t, a, s);
}

int mt_sync(mt_masstree* t, void* stream) {
  if (!t) return MT_ERR_INVALID_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(t->h_err, t->tv.pool.err, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return MT_ERR_CUDA;
  const uint32_t code = t->h_err[0];
  if (code != 0u) {
    t->last_error_site = t->h_err[3];
    e = cudaMemsetAsync(t->tv.pool.err, 0, 4 * sizeof(uint32_t), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return MT_ERR_CUDA;
  }
  return (int)code;
}

int mt_device_view(mt_masstree* t, void* view, size_t view_bytes) {
  if (!t || !view || view_bytes != sizeof(tree_view)) return MT_ERR_INVALID_ARG;
  tree_view v = t->tv;
  v.merge_log = nullptr;  // the device API never logs merges
  v.merge_cap = 0;
  v.layer_log = nullptr;
  v.layer_cap = 0;
  std::memcpy(view, &v, sizeof(v));
  return MT_OK;
}

int mt_reclaim(mt_masstree* t, void* stream) {
  if (!t) return MT_ERR_INVALID_ARG;
  return launch_reclaim(t, (cudaStream_t)stream);
}

int mt_stats(mt_masstree* t, mt_stats_t* out) {
  if (!t || !out) return MT_ERR_INVALID_ARG;
  if (cudaDeviceSynchronize() != cudaSuccess) return MT_ERR_CUDA;
  const pool_view& p = t->tv.pool;
  const size_t nctr = (size_t)p.num_shards * 3u * kCtrStride;
  int* h = new (std::nothrow) int[nctr];
  if (!h) return MT_ERR_OOM;
  uint32_t err[4] = {0, 0, 0, 0};
  cudaError_t e = cudaMemcpy(h, p.ctr, nctr * sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(err, p.err, sizeof(err), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) { delete[] h; return MT_ERR_CUDA; }
  uint64_t handed = 0, stacked = 0, limbo = 0;
  for (uint32_t s = 0; s < p.num_shards; ++s) {
    const int top = h[(3 * s + 0) * kCtrStride];
    const int bump = h[(3 * s + 1) * kCtrStride];
    const int lim = h[(3 * s + 2) * kCtrStride];
    handed += (uint64_t)std::min<int>(std::max(bump, 0), (int)p.shard_slabs);
    stacked += (uint64_t)std::max(top, 0);
    limbo += (uint64_t)std::max(lim, 0);
  }
  delete[] h;
  out->total_slabs = p.num_slabs;
  out->used_slabs = handed - stacked - limbo;
  out->limbo_slabs = limbo;
  out->free_slabs = (uint64_t)p.num_slabs - out->used_slabs - limbo;
  out->num_shards = p.num_shards;
  out->tile_size = t->tile_size;
  out->device_error = err[0];
  out->device_error_count = err[1];
  out->device_error_site = err[0] ? err[3] : t->last_error_site;
  out->reserved = 0;
  return MT_OK;
}

const char* mt_status_string(int s) {
  switch (s) {
    case MT_OK: return "ok";
    case MT_ERR_OOM: return "slab pool exhausted";
    case MT_ERR_LOCK_TIMEOUT: return "node lock timeout";
    case MT_ERR_CORRUPT: return "corrupt index structure";
    case MT_ERR_INVALID_ARG: return "invalid argument";
    case MT_ERR_CUDA: return "CUDA error";
    case MT_ERR_RETRY_LIMIT: return "retry limit reached";
    case MT_ERR_KEY_TOO_LONG: return "scan layer stack could not grow";
    case MT_ERR_BATCH_TOO_LARGE: return "batch larger than the fixed no-allocation scratch";
    default: return "unknown status";
  }
}

}  // extern "C"

// ---- validation (host walk over a device snapshot) ----------------------------------

namespace {

struct validator {
  // Used prefix of every shard (slabs past a shard's bump pointer were never
  // handed out).
  std::vector<std::vector<uint32_t>> img;
  std::vector<uint32_t> used;
  uint32_t shard_slabs = 1;
  std::vector<bool> seen;  // slab reached from the root (each at most once)
  uint64_t keys = 0, nodes = 0, chains = 0;
  std::string err;
  int depth_limit = 1 << 16;

  bool ok(uint32_t i) const {
    const uint32_t s = i / shard_slabs;
    return s < used.size() && (i % shard_slabs) < used[s];
  }
  const uint32_t* slab(uint32_t i) const { return img[i / shard_slabs].data() + (size_t)(i % shard_slabs) * 32u; }
  bool fail(const std::string& m) {
    if (err.empty()) err = m;
    return false;
  }
  bool mark(uint32_t i) {
    if (seen[i]) return fail("slab reachable twice (handed out twice)");
    seen[i] = true;
    return true;
  }

  bool chain(uint32_t head) {
    if (!ok(head)) return fail("suffix chain head out of range");
    const uint32_t hdr = slab(head)[SUF_WORD_HDR];
    const uint32_t kl = hdr & kMaxLen16, vl = hdr >> 16;
    const uint32_t need = suf_nodes(kl, vl);
    uint32_t c = head;
    if (!mark(c)) return false;
    for (uint32_t n = 1; n < need; ++n) {
      c = slab(c)[SUF_WORD_NEXT];
      if (!ok(c)) return fail("suffix chain shorter than its header");
      if (!mark(c)) return false;
    }
    if (slab(c)[SUF_WORD_NEXT] != kInvalid) return fail("suffix chain longer than its header");
    ++chains;
    return true;
  }

  // Validate the subtree at idx covering (lo, hi] (lo exclusive unless first).
  // last[level] is the node met before at that level of the layer (in key
  // order), whose sibling link must lead to this one.
  bool subtree(uint32_t idx, uint64_t lo_excl, uint32_t hi, int level, int& border_level, int layer_depth,
               std::vector<uint32_t>& last) {
    if (!ok(idx)) return fail("node index out of range");
    if (!mark(idx)) return false;
    const uint32_t* w = slab(idx);
    const uint32_t meta = w[WORD_META], ks = w[WORD_KS], n = meta & META_COUNT;
    ++nodes;
    if (meta & META_LOCK) return fail("node left locked");
    if (meta & META_DEAD) return fail("merged-away node still linked");
    if ((size_t)level >= last.size()) last.resize((size_t)level + 1u, kInvalid);
    if (last[level] != kInvalid) {
      const uint32_t* pw = slab(last[level]);
      if (!(pw[WORD_META] & META_SIB) || pw[WORD_SIB] != idx) return fail("sibling link does not lead to the next node");
    }
    last[level] = idx;
    if (n > (uint32_t)kMaxEntries) return fail("count above the node capacity");
    if (node_checksum(w) != w[WORD_CSUM]) return fail("node checksum mismatch");
    if (w[WORD_HIGH] != hi) return fail("high key differs from the parent's separator");
    const bool border = (meta & META_BORDER) != 0;
    if (border) {
      if (border_level < 0) border_level = level;
      else if (border_level != level) return fail("border nodes at different depths");
      uint64_t prev = 0;
      bool have = false;
      for (uint32_t e = 0; e < n; ++e) {
        const uint32_t k = w[2 * e], v = w[2 * e + 1], st = ks_get(ks, e);
        const uint64_t pos = ((uint64_t)k << 1) | (ks_more(st) ? 1u : 0u);
        if (have && pos <= prev) return fail("border entries out of order");
        if (lo_excl != ~0ull && (uint64_t)k <= lo_excl) return fail("border key below its range");
        if (k > hi) return fail("border key above its high key");
        prev = pos;
        have = true;
        if (st == KS_LINK) {
          if (!layer(v, layer_depth + 1)) return false;
        } else if (st == KS_VALUE) {
          ++keys;
        } else {
          if (!chain(v)) return false;
          ++keys;
        }
      }
      return true;
    }
    if (n == 0) return fail("empty interior node");
    uint64_t lo = lo_excl;
    for (uint32_t e = 0; e < n; ++e) {
      const uint32_t sep = w[2 * e];
      if (lo != ~0ull && (uint64_t)sep <= lo) return fail("interior separators out of order");
      if (!subtree(w[2 * e + 1], lo, sep, level + 1, border_level, layer_depth, last)) return false;
      lo = sep;
    }
    if (w[2 * (n - 1)] != hi) return fail("last separator differs from the high key");
    return true;
  }

  bool layer(uint32_t root, int depth) {
    if (depth > depth_limit) return fail("trie deeper than the limit");
    if (!ok(root)) return fail("layer root out of range");
    if (!(slab(root)[WORD_META] & META_ROOT)) return fail("layer root without ROOT flag");
    int border_level = -1;
    std::vector<uint32_t> last;
    if (!subtree(root, ~0ull, 0xFFFFFFFFu, 0, border_level, depth, last)) return false;
    for (uint32_t i : last)
      if (slab(i)[WORD_META] & META_SIB) return fail("rightmost node of a level with a sibling link");
    return true;
  }
};

}  // namespace

extern "C" int mt_validate(mt_masstree* t, uint64_t* num_keys, char* msg, size_t msg_len) {
  if (!t) return MT_ERR_INVALID_ARG;
  if (cudaDeviceSynchronize() != cudaSuccess) return MT_ERR_CUDA;
  const pool_view& p = t->tv.pool;
  const size_t nctr = (size_t)p.num_shards * 3u * kCtrStride;
  std::vector<int> h(nctr);
  if (cudaMemcpy(h.data(), p.ctr, nctr * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return MT_ERR_CUDA;
  validator v;
  v.shard_slabs = p.shard_slabs;
  v.img.resize(p.num_shards);
  v.used.resize(p.num_shards);
  v.seen.assign(p.num_slabs, false);
  std::vector<uint32_t> freed;  // free-stack and limbo entries
  for (uint32_t s = 0; s < p.num_shards; ++s) {
    const int bump = std::min<int>(std::max(h[(3 * s + 1) * kCtrStride], 0), (int)p.shard_slabs);
    v.used[s] = (uint32_t)bump;
    if (bump > 0) {
      v.img[s].resize((size_t)bump * 32u);
      const size_t off = (size_t)s * p.shard_slabs * 32u;
      if (cudaMemcpy(v.img[s].data(), p.slabs + off, (size_t)bump * 128u, cudaMemcpyDeviceToHost) != cudaSuccess)
        return MT_ERR_CUDA;
    }
    const int top = std::max(h[(3 * s + 0) * kCtrStride], 0);
    const int lim = std::max(h[(3 * s + 2) * kCtrStride], 0);
    const size_t base = freed.size();
    freed.resize(base + top + lim);
    if (top > 0 && cudaMemcpy(freed.data() + base, p.free_stack + (size_t)s * p.shard_slabs, (size_t)top * 4u,
                              cudaMemcpyDeviceToHost) != cudaSuccess)
      return MT_ERR_CUDA;
    if (lim > 0 && cudaMemcpy(freed.data() + base + top, p.limbo + (size_t)s * p.shard_slabs, (size_t)lim * 4u,
                              cudaMemcpyDeviceToHost) != cudaSuccess)
      return MT_ERR_CUDA;
  }
  bool good = v.layer(t->tv.root, 0);
  // Allocator invariant: a free or retired slab is neither reachable nor listed twice.
  if (good) {
    std::vector<bool> listed(p.num_slabs, false);
    for (uint32_t f : freed) {
      if (f >= p.num_slabs) { good = v.fail("free list holds an out-of-range slab"); break; }
      if (v.seen[f]) { good = v.fail("reachable slab is on a free list"); break; }
      if (listed[f]) { good = v.fail("slab listed twice on the free lists"); break; }
      listed[f] = true;
    }
  }
  if (num_keys) *num_keys = v.keys;
  if (msg && msg_len) {
    std::snprintf(msg, msg_len, "%s (keys %llu, nodes %llu, chains %llu, free+limbo %zu)",
                  good ? "ok" : v.err.c_str(), (unsigned long long)v.keys, (unsigned long long)v.nodes,
                  (unsigned long long)v.chains, freed.size());
  }
  return good ? MT_OK : MT_ERR_CORRUPT;
}

extern "C" int mt_selftest_line_atomicity(uint32_t tile_size, uint32_t nlines, uint32_t iters, uint64_t* reads,
                                          uint64_t* torn) {
  if (!valid_tile(tile_size) || nlines == 0 || !reads || !torn) return MT_ERR_INVALID_ARG;
  uint32_t* lines = nullptr;
  unsigned long long* ctr = nullptr;
  if (cudaMalloc(&lines, (size_t)nlines * 128u) != cudaSuccess) return MT_ERR_CUDA;
  if (cudaMalloc(&ctr, 2 * sizeof(unsigned long long)) != cudaSuccess) { cudaFree(lines); return MT_ERR_CUDA; }
  cudaMemset(lines, 0, (size_t)nlines * 128u);
  cudaMemset(ctr, 0, 2 * sizeof(unsigned long long));
  int sms = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int grid = sms * 8;
  switch (tile_size) {
    case 4: line_atomicity_kernel<4><<<grid, kBlock>>>(lines, nlines, iters, ctr, ctr + 1); break;
    case 8: line_atomicity_kernel<8><<<grid, kBlock>>>(lines, nlines, iters, ctr, ctr + 1); break;
    case 16: line_atomicity_kernel<16><<<grid, kBlock>>>(lines, nlines, iters, ctr, ctr + 1); break;
    default: line_atomicity_kernel<32><<<grid, kBlock>>>(lines, nlines, iters, ctr, ctr + 1); break;
  }
  unsigned long long hctr[2] = {0, 0};
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(hctr, ctr, sizeof(hctr), cudaMemcpyDeviceToHost);
  cudaFree(lines);
  cudaFree(ctr);
  if (e != cudaSuccess) return MT_ERR_CUDA;
  *reads = hctr[0];
  *torn = hctr[1];
  return MT_OK;
}

// ---- mixed batch that allocates nothing -------------------------------------------
//
// mt_mixed_batch keeps its partition scratch in memory it allocates with
// cudaMalloc the first time a batch is larger than any before.  Some callers
// cannot allocate at that point: latency-critical request loops that must never
// wait for the driver's allocator, and hosts that hand the whole device budget
// to the slab pool (or to another allocator) up front, where a late cudaMalloc
// fails.  mt_mixed_batch_noalloc serves them: its partition scratch is the fixed
// file-scope array below, sized for kNoAllocMaxRequests requests (2 MiB plus
// one line, held on every GPU that loads this library until the process exits).

namespace {
constexpr uint32_t kNoAllocMaxRequests = 1u << 18;
constexpr int kNoAllocMaxDevices = 64;
}  // namespace

// [0, 32): find / write counters (one line); then find indices, write indices.
static __device__ __align__(256) uint32_t g_noalloc_scratch[32u + 2u * kNoAllocMaxRequests];

namespace {
std::mutex g_noalloc_mu;
uint32_t* g_noalloc_addr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_scratch on device `dev`, which must be current.
// In host code the array's name is only a host-side stand-in, so the address
// is looked up once per device with that device current and kept.
int noalloc_scratch(int dev, uint32_t** out) {
  if (dev < 0 || dev >= kNoAllocMaxDevices) return MT_ERR_CUDA;
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return MT_ERR_CUDA;
    g_noalloc_addr[dev] = static_cast<uint32_t*>(p);
  }
  *out = g_noalloc_addr[dev];
  return MT_OK;
}
}  // namespace

extern "C" int mt_mixed_batch_noalloc(mt_masstree* t, const uint8_t* types, const uint32_t* keys, uint32_t maxK,
                                      const uint32_t* klens, uint32_t* values, uint32_t maxV, uint32_t* vlens,
                                      bool* results, uint32_t n, void* stream) {
  if (!t || (n && (!types || !keys || !values || !vlens || maxK == 0 || maxV == 0))) return MT_ERR_INVALID_ARG;
  if (n > kNoAllocMaxRequests) return MT_ERR_BATCH_TOO_LARGE;
  if (n == 0) return MT_OK;
  // The scratch address belongs to the current device: it must be the tree's.
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return MT_ERR_CUDA;
  if (dev != t->device) return MT_ERR_INVALID_ARG;
  uint32_t* scratch = nullptr;
  int rc = noalloc_scratch(dev, &scratch);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  batch_args a{};
  a.types = types; a.keys = keys; a.key_lengths = klens; a.values = values;
  a.value_lengths_in = vlens; a.value_lengths_out = vlens; a.results = results;
  a.max_key_length = maxK; a.max_value_length = maxV; a.n = n;
  rc = launch_reclaim(t, s);
  if (rc) return rc;
  uint32_t* counts = scratch;
  uint32_t* find_idx = scratch + 32;
  uint32_t* write_idx = find_idx + n;
  // The array keeps the previous call's contents: the counters must restart at 0.
  if (cudaMemsetAsync(counts, 0, 2 * sizeof(uint32_t), s) != cudaSuccess) return MT_ERR_CUDA;
  partition_kernel<<<std::max(1, std::min(t->sms * 8, (int)((n + 255) / 256))), 256, 0, s>>>(types, n, find_idx,
                                                                                             write_idx, counts);
  if (cudaGetLastError() != cudaSuccess) return MT_ERR_CUDA;
  batch_args f = a;
  f.index = find_idx;
  f.n_dev = counts;
  rc = launch_batch_tile<OP_MIXED, true>(t, t->tile_size, f, s);
  if (rc) return rc;
  batch_args w = a;
  w.index = write_idx;
  w.n_dev = counts + 1;
  return launch_batch_tile<OP_MIXED, true>(t, t->write_tile_size, w, s);
}
