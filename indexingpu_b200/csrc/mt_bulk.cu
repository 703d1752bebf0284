// Bulk build of a new tree's first layer (the first large insert into a tree
// that holds nothing yet).
//
// Inserted one by one, such a batch starts every tile on the single root node,
// and node splits serialise there until the tree has thousands of leaves.  The
// reference inserts one by one as well (include/gpu_masstree.hpp:101-115).  Here
// the batch is ordered by its first slice on the device; every key whose first
// slice no other key of the batch shares becomes a layer-0 entry directly (its
// value, or a suffix chain of its key rest and value, built by one tile each),
// the entries are packed into border nodes in key order, and the interior
// levels are written bottom-up, the top node into the root slab.  The other
// keys (a first slice shared with another key, invalid lengths) are then
// inserted by the ordinary insert kernel, which also reports their results.
// Nodes are packed to kBulkFill entries so that later inserts find room.
#include <algorithm>

#include "mt_internal.cuh"

namespace mtb {

constexpr uint32_t kBuckets = 1u << 16;  // ordered by the top 16 bits of the first slice, then sorted
constexpr uint32_t kBulkFill = 10;       // entries per built node (of kMaxEntries)

struct bulk_view {
  const uint32_t* keys;
  const uint32_t* klens;
  const uint32_t* values;
  const uint32_t* vlens;
  bool* results;
  uint32_t max_key_length, max_value_length, n;
  uint32_t* counts;          // [kBuckets] keys per bucket, then fill cursors
  uint32_t* offsets;         // [kBuckets] first position of every bucket
  uint32_t* ctl;             // [0] valid keys, [1] largest bucket, [2] rest count, [3] unique count,
                             // [4] buckets holding keys
  unsigned long long* order; // [n] (first slice << 32 | request) in key order
  uint32_t* rest;            // [n] requests left to the ordinary insert
  uint32_t* block_uniques;   // [blocks of the classify pass] unique keys per block, then their offsets
  uint32_t* e_slice;         // [n] per unique entry: slice, value word, key state, request
  uint32_t* e_val;
  uint32_t* e_state;
  uint32_t* e_src;
};

MT_DEV bool bulk_valid(const bulk_view& b, uint32_t i) {
  const uint32_t kl = b.klens ? b.klens[i] : b.max_key_length;
  const uint32_t vl = b.vlens ? b.vlens[i] : b.max_value_length;
  return kl >= 1u && kl <= b.max_key_length && vl <= b.max_value_length && kl <= kMaxLen16 && vl <= kMaxLen16;
}

__global__ void bulk_count_kernel(bulk_view b) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.n; i += gridDim.x * blockDim.x) {
    if (!bulk_valid(b, i)) {
      b.rest[atomicAdd(&b.ctl[2], 1u)] = i;
      continue;
    }
    const uint32_t bucket = b.keys[(size_t)i * b.max_key_length] >> 16;
    const uint32_t c = atomicAdd(&b.counts[bucket], 1u) + 1u;
    if (c == 1u) atomicAdd(&b.ctl[4], 1u);
    atomicMax(&b.ctl[1], c);
    atomicAdd(&b.ctl[0], 1u);
  }
}

// Exclusive prefix sums of the bucket sizes (one block of 1024 threads).
__global__ void bulk_scan_kernel(bulk_view b) {
  __shared__ uint32_t part[1024];
  constexpr uint32_t per = kBuckets / 1024u;
  const uint32_t base = threadIdx.x * per;
  uint32_t s = 0;
  for (uint32_t k = 0; k < per; ++k) s += b.counts[base + k];
  part[threadIdx.x] = s;
  __syncthreads();
  for (uint32_t d = 1; d < 1024u; d <<= 1) {
    const uint32_t v = threadIdx.x >= d ? part[threadIdx.x - d] : 0u;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  uint32_t run = part[threadIdx.x] - s;
  for (uint32_t k = 0; k < per; ++k) {
    const uint32_t c = b.counts[base + k];
    b.offsets[base + k] = run;
    b.counts[base + k] = run;  // fill cursor
    run += c;
  }
}

__global__ void bulk_scatter_kernel(bulk_view b) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.n; i += gridDim.x * blockDim.x) {
    if (!bulk_valid(b, i)) continue;
    const uint32_t s0 = b.keys[(size_t)i * b.max_key_length];
    const uint32_t pos = atomicAdd(&b.counts[s0 >> 16], 1u);
    b.order[pos] = ((unsigned long long)s0 << 32) | i;
  }
}

// Sort inside every bucket (insertion sort; buckets are small, the host checks).
__global__ void bulk_sort_kernel(bulk_view b) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < kBuckets; k += gridDim.x * blockDim.x) {
    const uint32_t lo = b.offsets[k], hi = b.counts[k];  // counts: end of the bucket after the scatter
    for (uint32_t x = lo + 1; x < hi; ++x) {
      const unsigned long long v = b.order[x];
      uint32_t y = x;
      while (y > lo && b.order[y - 1] > v) {
        b.order[y] = b.order[y - 1];
        --y;
      }
      b.order[y] = v;
    }
  }
}

// Whether position j of the ordered keys holds a first slice no other key has.
MT_DEV bool bulk_unique(const bulk_view& b, uint32_t j, uint32_t m) {
  const uint32_t s = (uint32_t)(b.order[j] >> 32);
  return (j == 0 || (uint32_t)(b.order[j - 1] >> 32) != s) && (j + 1 >= m || (uint32_t)(b.order[j + 1] >> 32) != s);
}

// Pass 1: unique keys per block of 256 positions; the others go to the rest.
__global__ void bulk_classify_kernel(bulk_view b, uint32_t m) {
  const uint32_t j = blockIdx.x * 256u + threadIdx.x;
  const bool u = j < m && bulk_unique(b, j, m);
  if (j < m && !u) b.rest[atomicAdd(&b.ctl[2], 1u)] = (uint32_t)b.order[j];
  const uint32_t c = __syncthreads_count(u);
  if (threadIdx.x == 0) b.block_uniques[blockIdx.x] = c;
}

// Exclusive sums of the per-block counts (one block); ctl[3] = total.
__global__ void bulk_block_scan_kernel(bulk_view b, uint32_t nblocks) {
  if (threadIdx.x != 0) return;
  uint32_t run = 0;
  for (uint32_t k = 0; k < nblocks; ++k) {
    const uint32_t c = b.block_uniques[k];
    b.block_uniques[k] = run;
    run += c;
  }
  b.ctl[3] = run;
}

// Pass 2: unique keys, in key order, to the entry arrays.
__global__ void bulk_compact_kernel(bulk_view b, uint32_t m) {
  __shared__ uint32_t warp_base[8];
  const uint32_t j = blockIdx.x * 256u + threadIdx.x;
  const bool u = j < m && bulk_unique(b, j, m);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t bal = __ballot_sync(0xFFFFFFFFu, u);
  if (lane == 0) warp_base[warp] = __popc(bal);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (int w = 0; w < 8; ++w) {
      const uint32_t c = warp_base[w];
      warp_base[w] = run;
      run += c;
    }
  }
  __syncthreads();
  if (u) {
    const uint32_t pos = b.block_uniques[blockIdx.x] + warp_base[warp] + __popc(bal & ((1u << lane) - 1u));
    b.e_slice[pos] = (uint32_t)(b.order[j] >> 32);
    b.e_src[pos] = (uint32_t)b.order[j];
  }
}

// The value word and key state of every unique entry (a 32-lane tile each:
// chains are written cooperatively); its request reports success.
__global__ void __launch_bounds__(kBlock, MT_MIN_BLOCKS_PER_SM) bulk_entry_kernel(tree_view tv, bulk_view b,
                                                                                  uint32_t nu) {
  tile<32> t;
  slab_cache<32> cache;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / 32u;
  const uint32_t num_tiles = (gridDim.x * blockDim.x) / 32u;
  cache.init(tv.pool, tile_id);
  const pool_view& p = tv.pool;
  for (uint32_t u = tile_id; u < nu; u += num_tiles) {
    if (t.shfl((uint32_t)(t.leader() && fatal_error(p)), 0)) break;
    const uint32_t i = b.e_src[u];
    const uint32_t klen = b.klens ? b.klens[i] : b.max_key_length;
    const uint32_t vlen = b.vlens ? b.vlens[i] : b.max_value_length;
    const uint32_t* key = b.keys + (size_t)i * b.max_key_length;
    const uint32_t* val = b.values + (size_t)i * b.max_value_length;
    uint32_t nv = kInvalid, ns = KS_VALUE;
    bool ok;
    if (klen > 1u) {
      slice_src ks, vs;
      ks.ptr = key + 1;
      ks.len = klen - 1u;
      vs.ptr = val;
      vs.len = vlen;
      nv = suffix_create<32, kConcSuffix>(t, p, cache, ks, vs);
      ns = KS_SUFFIX;
      ok = nv != kInvalid;
    } else {
      ok = make_value(t, p, cache, val, vlen, nv, ns);
    }
    if (t.leader()) {
      b.e_val[u] = nv;
      b.e_state[u] = ok ? ns : 0xFFFFFFFFu;
      if (b.results) b.results[i] = ok;
    }
  }
  cache.release(t, p);
}

// Slabs of the nodes of one level (the root slab when the level has one node).
__global__ void __launch_bounds__(kBlock, MT_MIN_BLOCKS_PER_SM) bulk_alloc_kernel(tree_view tv, uint32_t* ids,
                                                                                  uint32_t count, uint32_t root) {
  tile<32> t;
  slab_cache<32> cache;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / 32u;
  const uint32_t num_tiles = (gridDim.x * blockDim.x) / 32u;
  cache.init(tv.pool, tile_id);
  for (uint32_t k = tile_id; k < count; k += num_tiles) {
    const uint32_t s = count == 1u ? root : cache.allocate(t, tv.pool);
    if (t.leader()) ids[k] = s;
  }
  cache.release(t, tv.pool);
}

// Write node k of a level: entries [k*F, min((k+1)*F, count)) of
// (key[], val[], state[]); border nodes carry key states, interior nodes route
// to children (key = the child's high key).  high[k] receives the node's high
// key for the level above.
__global__ void __launch_bounds__(kBlock, MT_MIN_BLOCKS_PER_SM) bulk_node_kernel(
    tree_view tv, const uint32_t* key, const uint32_t* val, const uint32_t* state, uint32_t count, const uint32_t* ids,
    uint32_t* high_out, uint32_t nodes, bool border) {
  tile<32> t;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / 32u;
  const uint32_t num_tiles = (gridDim.x * blockDim.x) / 32u;
  const pool_view& p = tv.pool;
  for (uint32_t k = tile_id; k < nodes; k += num_tiles) {
    const uint32_t first = k * kBulkFill;
    const uint32_t cnt = min(kBulkFill, count - first);
    const bool last = k + 1u == nodes;
    node<32> nd;
    nd.idx = ids[k];
    if (!p.valid(nd.idx)) {
      if (t.leader()) record_error(p, ERR_OOM, MT_AT(SRC_BULK));
      continue;
    }
    const uint32_t g = t.rank;  // one word per lane
    const uint32_t e = g >> 1;
    nd.w[0] = (e < cnt && g < 2u * kMaxEntries) ? ((g & 1u) ? val[first + e] : key[first + e]) : 0u;
    uint32_t ks = 0;
    if (border) {
      const uint32_t st = (t.rank < cnt) ? (state[first + t.rank] & 3u) << (2u * t.rank) : 0u;
      ks = t.or_all(st);
    }
    const uint32_t hk = last ? 0xFFFFFFFFu : key[first + cnt - 1u];
    nd.meta = cnt | (border ? META_BORDER : 0u) | (last ? 0u : META_SIB) | (nodes == 1u ? META_ROOT : 0u);
    nd.ks = ks;
    nd.high = hk;
    nd.sib = last ? kInvalid : ids[k + 1u];
    nd.encode_header(t);
    nd.seal(t);
    nd.template store<st_order::WEAK>(t, p);
    if (t.leader()) high_out[k] = hk;
  }
}

}  // namespace mtb

using namespace mtb;

namespace {

int cu(cudaError_t e) { return e == cudaSuccess ? MT_OK : MT_ERR_CUDA; }

template <typename X>
int dalloc(X** p, size_t n) {
  return cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(X)) == cudaSuccess ? MT_OK
                                                                                                    : MT_ERR_OOM;
}

}  // namespace

namespace mtb {

// Returns MT_OK after building (and inserting the rest), or kBulkDeclined when
// the batch does not suit a bulk build or its scratch does not fit in device
// memory (the caller inserts it as usual).
int host_bulk_insert(mt_masstree* t, const batch_args& a, bool upsert, cudaStream_t s) {
  const uint32_t n = a.n;
  bulk_view b{};
  b.keys = a.keys;
  b.klens = a.key_lengths;
  b.values = a.values;
  b.vlens = a.value_lengths_in;
  b.results = a.results;
  b.max_key_length = a.max_key_length;
  b.max_value_length = a.max_value_length;
  b.n = n;
  const uint32_t cblocks = (n + 255u) / 256u;
  int rc = dalloc(&b.counts, kBuckets);
  if (!rc) rc = dalloc(&b.offsets, kBuckets);
  if (!rc) rc = dalloc(&b.ctl, 8);
  if (!rc) rc = dalloc(&b.order, n);
  if (!rc) rc = dalloc(&b.rest, n);
  if (!rc) rc = dalloc(&b.block_uniques, cblocks);
  if (!rc) rc = dalloc(&b.e_slice, n);
  if (!rc) rc = dalloc(&b.e_val, n);
  if (!rc) rc = dalloc(&b.e_state, n);
  if (!rc) rc = dalloc(&b.e_src, n);
  uint32_t* ids = nullptr;
  uint32_t* highs[2] = {nullptr, nullptr};
  const uint32_t max_nodes = n / kBulkFill + 2u;
  if (!rc) rc = dalloc(&ids, max_nodes);
  if (!rc) rc = dalloc(&highs[0], max_nodes);
  if (!rc) rc = dalloc(&highs[1], max_nodes);
  uint32_t* ids2 = nullptr;
  if (!rc) rc = dalloc(&ids2, max_nodes);
  auto release = [&] {
    for (void* q : {(void*)b.counts, (void*)b.offsets, (void*)b.ctl, (void*)b.order, (void*)b.rest,
                    (void*)b.block_uniques, (void*)b.e_slice, (void*)b.e_val, (void*)b.e_state, (void*)b.e_src,
                    (void*)ids, (void*)ids2, (void*)highs[0], (void*)highs[1]})
      if (q) cudaFree(q);
  };
  if (rc) {
    // No room for the scratch beside the slab pool: the ordinary insert needs
    // none.  Clear the failed allocation's error so later launch checks do
    // not report it.
    cudaGetLastError();
    release();
    return kBulkDeclined;
  }
  uint32_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int grid = std::max(1, t->sms * 8);
  if (!rc) rc = cu(cudaMemsetAsync(b.counts, 0, kBuckets * sizeof(uint32_t), s));
  if (!rc) rc = cu(cudaMemsetAsync(b.ctl, 0, 8 * sizeof(uint32_t), s));
  if (!rc) {
    bulk_count_kernel<<<grid, 256, 0, s>>>(b);
    rc = cu(cudaGetLastError());
  }
  if (!rc) rc = cu(cudaMemcpyAsync(h, b.ctl, sizeof(h), cudaMemcpyDeviceToHost, s));
  if (!rc) rc = cu(cudaStreamSynchronize(s));
  const uint32_t m = h[0];
  // Decline when one bucket is large, or the keys crowd into few buckets
  // (first slices shared by many keys: little to build, and the in-bucket
  // sort would be slow), or fewer than half the keys are valid.
  bool declined = !rc && (h[1] > 2048u || h[4] < std::min<uint32_t>(m, kBuckets) / 64u || m < n / 2u);
  if (!rc && !declined) {
    bulk_scan_kernel<<<1, 1024, 0, s>>>(b);
    bulk_scatter_kernel<<<grid, 256, 0, s>>>(b);
    bulk_sort_kernel<<<(kBuckets + 255u) / 256u, 256, 0, s>>>(b);
    const uint32_t mblocks = std::max(1u, (m + 255u) / 256u);
    bulk_classify_kernel<<<mblocks, 256, 0, s>>>(b, m);
    bulk_block_scan_kernel<<<1, 32, 0, s>>>(b, mblocks);
    bulk_compact_kernel<<<mblocks, 256, 0, s>>>(b, m);
    rc = cu(cudaGetLastError());
    if (!rc) rc = cu(cudaMemcpyAsync(h, b.ctl, sizeof(h), cudaMemcpyDeviceToHost, s));
    if (!rc) rc = cu(cudaStreamSynchronize(s));
  }
  const uint32_t nu = h[3];
  if (!rc && !declined && nu == 0u) declined = true;
  if (!rc && !declined) {
    // Entries, then (unless building them failed: pool exhausted) the levels
    // bottom-up.
    bulk_entry_kernel<<<grid, kBlock, 0, s>>>(t->tv, b, nu);
    rc = cu(cudaGetLastError());
    uint32_t err = 0;
    if (!rc) rc = cu(cudaMemcpyAsync(&err, t->tv.pool.err, sizeof(err), cudaMemcpyDeviceToHost, s));
    if (!rc) rc = cu(cudaStreamSynchronize(s));
    if (!rc && err != 0u) rc = (int)err;
    uint32_t count = nu;
    const uint32_t* key = b.e_slice;
    const uint32_t* val = b.e_val;
    bool border = true;
    uint32_t* cur_ids = ids;
    uint32_t* next_ids = ids2;
    int hi = 0;
    while (!rc) {
      const uint32_t nodes = (count + kBulkFill - 1u) / kBulkFill;
      bulk_alloc_kernel<<<std::min<uint32_t>(grid, (nodes + 3u) / 4u), kBlock, 0, s>>>(t->tv, cur_ids, nodes,
                                                                                           t->tv.root);
      bulk_node_kernel<<<std::min<uint32_t>(grid, (nodes + 3u) / 4u), kBlock, 0, s>>>(
          t->tv, key, val, b.e_state, count, cur_ids, highs[hi], nodes, border);
      rc = cu(cudaGetLastError());
      if (nodes == 1u) break;
      // The level above routes to these nodes by their high keys.
      key = highs[hi];
      val = cur_ids;
      count = nodes;
      border = false;
      hi ^= 1;
      std::swap(cur_ids, next_ids);
    }
    if (!rc) rc = cu(cudaStreamSynchronize(s));
  }
  if (!rc && !declined) {
    // The rest through the ordinary insert kernel.
    if (!rc) rc = cu(cudaMemcpyAsync(h, b.ctl, sizeof(h), cudaMemcpyDeviceToHost, s));
    if (!rc) rc = cu(cudaStreamSynchronize(s));
    if (!rc && h[2] > 0u) {
      batch_args r = a;
      r.index = b.rest;
      r.n_dev = b.ctl + 2;
      r.n = h[2];
      rc = host_launch_insert(t, r, upsert, s);
      if (!rc) rc = cu(cudaStreamSynchronize(s));
    }
  }
  cudaStreamSynchronize(s);
  release();
  if (rc) return rc;
  return declined ? kBulkDeclined : MT_OK;
}

}  // namespace mtb
