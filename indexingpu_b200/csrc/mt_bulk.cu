// Bulk build of a new tree's first layer (an insert into a tree that holds
// nothing yet).
//
// Inserted one by one, such a batch starts every tile on the single root node,
// and node splits serialise there until the tree has thousands of leaves (a
// few thousand keys took milliseconds).  The reference inserts one by one as
// well (include/gpu_masstree.hpp:101-115).  Here the batch is sorted on the
// device by (first slice, whether the key continues past it), the key-order
// position of a layer-0 entry (a key ending at a slice sorts before one that
// continues with it).  Each run of one such position becomes one layer-0
// entry:
//   * a run of one key: the key's entry itself (its value, or a suffix chain of
//     its key rest and value), built by one tile each;
//   * a run of keys that continue past one first slice: a LINK entry to a new,
//     empty layer-1 root, and the keys are inserted afterwards;
//   * a run of keys ending at one first slice (the same key more than once):
//     no entry, the keys are inserted afterwards (one of them wins).
// The entries are packed into border nodes in key order, and the interior
// levels are written bottom-up, the top node into the root slab.  The keys
// left over (and invalid ones) then go through the ordinary insert kernel,
// which also reports their results: they meet in their own layer-1 roots, one
// per shared first slice, instead of all in the root.  Nodes are packed to
// kBulkFill entries so that later inserts find room.
#include <algorithm>

#include <cub/device/device_radix_sort.cuh>

#include "mt_internal.cuh"

namespace mtb {

constexpr uint32_t kBulkFill = 10;                    // entries per built node (of kMaxEntries)
constexpr unsigned long long kBulkInvalid = 1ull << 33;  // sort key of an invalid request (after all valid ones)
constexpr int kBulkSortBits = 34;

struct bulk_view {
  const uint32_t* keys;
  const uint32_t* klens;
  const uint32_t* values;
  const uint32_t* vlens;
  bool* results;
  uint32_t max_key_length, max_value_length, n;
  uint32_t* ctl;                  // [0] valid keys, [2] rest count, [3] entries
  unsigned long long* sort_key;   // [n] (first slice << 1 | continues) in key order (after the sort)
  uint32_t* sort_req;             // [n] the request at each sorted position
  uint32_t* rest;                 // [n] requests left to the ordinary insert
  uint32_t* block_entries;        // [blocks of the classify pass] entries per block, then their offsets
  uint32_t* e_slice;              // [n] per entry: slice, value word, key state, request (kInvalid: LINK)
  uint32_t* e_val;
  uint32_t* e_state;
  uint32_t* e_src;
};

MT_DEV bool bulk_valid(const bulk_view& b, uint32_t i) {
  const uint32_t kl = b.klens ? b.klens[i] : b.max_key_length;
  const uint32_t vl = b.vlens ? b.vlens[i] : b.max_value_length;
  return kl >= 1u && kl <= b.max_key_length && vl <= b.max_value_length && kl <= kMaxLen16 && vl <= kMaxLen16;
}

// Sort keys of all requests; invalid requests go to the rest at once.
__global__ void bulk_keys_kernel(bulk_view b, unsigned long long* key_out, uint32_t* req_out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.n; i += gridDim.x * blockDim.x) {
    unsigned long long k = kBulkInvalid;
    if (bulk_valid(b, i)) {
      const uint32_t kl = b.klens ? b.klens[i] : b.max_key_length;
      k = ((unsigned long long)b.keys[(size_t)i * b.max_key_length] << 1) | (kl > 1u ? 1ull : 0ull);
      atomicAdd(&b.ctl[0], 1u);
    } else {
      b.rest[atomicAdd(&b.ctl[2], 1u)] = i;
    }
    key_out[i] = k;
    req_out[i] = i;
  }
}

// What sorted position j (of m valid ones) becomes: an entry of its own
// (alone in its run), the LINK entry of a run of continuing keys (its first
// position), and / or a request for the ordinary insert (every position of a
// run of two or more).
MT_DEV void bulk_position(const bulk_view& b, uint32_t j, uint32_t m, bool& entry, bool& to_rest) {
  const unsigned long long k = b.sort_key[j];
  const bool first = j == 0 || b.sort_key[j - 1] != k;
  const bool last = j + 1 >= m || b.sort_key[j + 1] != k;
  const bool alone = first && last;
  entry = alone || (first && (k & 1ull) != 0ull);
  to_rest = !alone;
}

// Pass 1: entries per block of 256 positions; the others go to the rest.
__global__ void bulk_classify_kernel(bulk_view b) {
  const uint32_t m = b.ctl[0];
  const uint32_t j = blockIdx.x * 256u + threadIdx.x;
  bool entry = false, to_rest = false;
  if (j < m) bulk_position(b, j, m, entry, to_rest);
  if (to_rest) b.rest[atomicAdd(&b.ctl[2], 1u)] = b.sort_req[j];
  const uint32_t c = __syncthreads_count(entry);
  if (threadIdx.x == 0) b.block_entries[blockIdx.x] = c;
}

// Exclusive sums of the per-block counts (one thread); ctl[3] = total.
__global__ void bulk_block_scan_kernel(bulk_view b, uint32_t nblocks) {
  if (threadIdx.x != 0) return;
  uint32_t run = 0;
  for (uint32_t k = 0; k < nblocks; ++k) {
    const uint32_t c = b.block_entries[k];
    b.block_entries[k] = run;
    run += c;
  }
  b.ctl[3] = run;
}

// Pass 2: the entries, in key order, to the entry arrays.
__global__ void bulk_compact_kernel(bulk_view b) {
  __shared__ uint32_t warp_base[8];
  const uint32_t m = b.ctl[0];
  const uint32_t j = blockIdx.x * 256u + threadIdx.x;
  bool entry = false, to_rest = false;
  if (j < m) bulk_position(b, j, m, entry, to_rest);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t bal = __ballot_sync(0xFFFFFFFFu, entry);
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
  if (entry) {
    const uint32_t pos = b.block_entries[blockIdx.x] + warp_base[warp] + __popc(bal & ((1u << lane) - 1u));
    b.e_slice[pos] = (uint32_t)(b.sort_key[j] >> 1);
    b.e_src[pos] = to_rest ? kInvalid : b.sort_req[j];
  }
}

// The value word and key state of every entry (a 32-lane tile each: chains
// are written cooperatively); the request of a key's own entry reports
// success.
__global__ void __launch_bounds__(kBlock, MT_MIN_BLOCKS_PER_SM) bulk_entry_kernel(tree_view tv, bulk_view b,
                                                                                  uint32_t nu) {
  tile<32> t;
  slab_cache<32> cache;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / 32u;
  const uint32_t num_tiles = (gridDim.x * blockDim.x) / 32u;
  cache.init(tv.pool, tile_id);
  const pool_view& p = tv.pool;
  nu = min(nu, b.ctl[3]);  // entries found by the compaction (nu: capacity)
  for (uint32_t u = tile_id; u < nu; u += num_tiles) {
    if (t.shfl((uint32_t)(t.leader() && fatal_error(p)), 0)) break;
    const uint32_t i = b.e_src[u];
    if (i == kInvalid) {
      // A LINK entry: a new, empty root for the layer below this first slice.
      const uint32_t r = cache.allocate(t, p);
      if (r != kInvalid) {
        node<32> nd;
        make_layer_root(t, nd, r);
        publish_new(t, p, nd);
      }
      if (t.leader()) {
        b.e_val[u] = r;
        b.e_state[u] = r != kInvalid ? KS_LINK : 0xFFFFFFFFu;
      }
      continue;
    }
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
  // Node k takes entries [k*F, (k+1)*F), each bound moved one up when it
  // would part the two entries of one slice (a key ending there and one
  // continuing), which must share a node: lookups of the slice go to the
  // node whose high key it is.
  auto bound = [&](uint32_t x) {
    return (x == 0u || x >= count) ? min(x, count) : x + (key[x - 1u] == key[x] ? 1u : 0u);
  };
  for (uint32_t k = tile_id; k < nodes; k += num_tiles) {
    const uint32_t first = bound(k * kBulkFill);
    const bool last = k + 1u == nodes;
    const uint32_t cnt = (last ? count : bound((k + 1u) * kBulkFill)) - first;
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
  const uint32_t max_nodes = n / kBulkFill + 2u;
  // One allocation for all scratch: the sort's input and output, its own
  // temporary storage, and the arrays of the build.
  size_t sort_bytes = 0;
  if (cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (unsigned long long*)nullptr,
                                      (unsigned long long*)nullptr, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)n, 0,
                                      kBulkSortBits, s) != cudaSuccess)
    return kBulkDeclined;
  auto up = [](size_t x) { return (x + 255u) & ~size_t(255); };
  const size_t n64 = up((size_t)n * 8u), n32 = up((size_t)n * 4u), nodes32 = up((size_t)max_nodes * 4u);
  const size_t total = 2 * n64 + 2 * n32 + up(sort_bytes) + up(8 * 4u) + 5 * n32 + up((size_t)cblocks * 4u) +
                       4 * nodes32;
  char* mem = nullptr;
  if (cudaMalloc(&mem, total) != cudaSuccess) {
    // No room for the scratch beside the slab pool: the ordinary insert needs
    // none.  Clear the failed allocation's error so later launch checks do
    // not report it.
    cudaGetLastError();
    return kBulkDeclined;
  }
  char* q = mem;
  auto carve = [&](size_t bytes) {
    char* r = q;
    q += bytes;
    return r;
  };
  auto* key_in = reinterpret_cast<unsigned long long*>(carve(n64));
  b.sort_key = reinterpret_cast<unsigned long long*>(carve(n64));
  auto* req_in = reinterpret_cast<uint32_t*>(carve(n32));
  b.sort_req = reinterpret_cast<uint32_t*>(carve(n32));
  void* sort_tmp = carve(up(sort_bytes));
  b.ctl = reinterpret_cast<uint32_t*>(carve(up(8 * 4u)));
  b.rest = reinterpret_cast<uint32_t*>(carve(n32));
  b.e_slice = reinterpret_cast<uint32_t*>(carve(n32));
  b.e_val = reinterpret_cast<uint32_t*>(carve(n32));
  b.e_state = reinterpret_cast<uint32_t*>(carve(n32));
  b.e_src = reinterpret_cast<uint32_t*>(carve(n32));
  b.block_entries = reinterpret_cast<uint32_t*>(carve(up((size_t)cblocks * 4u)));
  uint32_t* ids = reinterpret_cast<uint32_t*>(carve(nodes32));
  uint32_t* ids2 = reinterpret_cast<uint32_t*>(carve(nodes32));
  uint32_t* highs[2] = {reinterpret_cast<uint32_t*>(carve(nodes32)), reinterpret_cast<uint32_t*>(carve(nodes32))};

  uint32_t h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  uint32_t err = 0;
  const int grid = std::max(1, t->sms * 8);
  int rc = cu(cudaMemsetAsync(b.ctl, 0, 8 * sizeof(uint32_t), s));
  if (!rc) {
    bulk_keys_kernel<<<std::min<uint32_t>(grid, cblocks), 256, 0, s>>>(b, key_in, req_in);
    rc = cu(cudaGetLastError());
  }
  size_t sb = sort_bytes;
  if (!rc)
    rc = cu(cub::DeviceRadixSort::SortPairs(sort_tmp, sb, key_in, b.sort_key, req_in, b.sort_req, (int)n, 0,
                                            kBulkSortBits, s));
  if (!rc) {
    bulk_classify_kernel<<<cblocks, 256, 0, s>>>(b);
    bulk_block_scan_kernel<<<1, 32, 0, s>>>(b, cblocks);
    bulk_compact_kernel<<<cblocks, 256, 0, s>>>(b);
    rc = cu(cudaGetLastError());
  }
  // Every entry's value word and key state (capacity: all positions), then
  // the counts and the error word.
  if (!rc) {
    bulk_entry_kernel<<<grid, kBlock, 0, s>>>(t->tv, b, n);
    rc = cu(cudaGetLastError());
  }
  if (!rc) rc = cu(cudaMemcpyAsync(h, b.ctl, sizeof(h), cudaMemcpyDeviceToHost, s));
  if (!rc) rc = cu(cudaMemcpyAsync(&err, t->tv.pool.err, sizeof(err), cudaMemcpyDeviceToHost, s));
  if (!rc) rc = cu(cudaStreamSynchronize(s));
  if (!rc && err != 0u) rc = (int)err;
  const uint32_t nu = h[3];
  if (!rc && nu > 0u) {
    // The levels bottom-up.
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
  }
  if (!rc && h[2] > 0u) {
    // The rest through the ordinary insert kernel.
    batch_args r = a;
    r.index = b.rest;
    r.n_dev = b.ctl + 2;
    r.n = h[2];
    rc = host_launch_insert(t, r, upsert, s);
  }
  cudaStreamSynchronize(s);
  cudaFree(mem);
  return rc;
}

}  // namespace mtb
