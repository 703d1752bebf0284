// Sub-batches grouped by key (mt_mixed_batches with MT_FLAG_GROUP_BY_KEY).
//
// mt_mixed_batches serves sub-batch k+1 after every request of sub-batch k;
// inside one sub-batch requests have no order.  Requests on different keys
// commute (their results do not depend on each other), so the whole list can
// be served at once as long as the requests on one key take effect in
// sub-batch order.  This form:
//   1. hashes every request's key and radix-sorts (hash, flat request id): the
//      requests on one key become one run, in sub-batch order (the sort is
//      stable and the ids grow with the sub-batch);
//   2. gives every request a transfer function on its key's state (absent,
//      present with the value the tree holds, present with the value of
//      request x) and takes the exclusive scan of their compositions per run
//      (a segmented scan: the state each request sees, relative to the state
//      before the call);
//   3. reads the tree once per key that two or more requests touch (present?
//      value?), derives every request's result from the scanned state (a find
//      copies the tree's value or the value of the write it sees), and writes
//      the key's final state back with one insert, update or erase;
//   4. serves a key that only one request touches as that request, directly.
// The result of every request is the one the per-sub-batch order gives with
// the requests of one sub-batch taken in their buffer order, and the tree ends
// in the same state.  A hot key that thousands of requests touch costs one
// read and at most one write instead of thousands of tree operations on one
// node.  Two different keys with one hash are caught when the run is checked
// key by key against its neighbours; such a run is served one request after
// the other, in order, by one tile.
#include <algorithm>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "mt_internal.cuh"

namespace mtb {

// A key's state as a request sees it: kGAbsent, kGKeep (present with the value
// the tree held before the call) or the flat id of the insert / update whose
// value the key holds.  The transfer function of a run of requests maps
// "absent before" to a and "present before" to p.
constexpr uint32_t kGAbsent = 0xFFFFFFFEu;
constexpr uint32_t kGKeep = 0xFFFFFFFFu;
constexpr uint32_t kGNoFirst = 0xFFFFFFFFu;

struct gfn {
  uint32_t a, p;
  uint32_t first;  // sorted position of the earliest request in the composition
};

MT_HD uint32_t gfn_apply(uint32_t s, const gfn& g) {
  if (s == kGAbsent) return g.a;
  return g.p == kGKeep ? s : g.p;
}

// f, then g (the scan's operator; its left operand is the earlier prefix).
struct gfn_compose {
  MT_HD gfn operator()(const gfn& f, const gfn& g) const {
    gfn r;
    r.a = gfn_apply(f.a, g);
    r.p = gfn_apply(f.p, g);
    r.first = f.first != kGNoFirst ? f.first : g.first;
    return r;
  }
};

constexpr unsigned long long kGPad = ~0ull;                            // positions past the call's requests
constexpr unsigned long long kGBad = ~0ull - 1ull;                     // requests rejected (error recorded)
constexpr unsigned long long kGMaxHash = ~0ull - (1ull << 32) - 2ull;  // key hashes stay below; above: one-offs

struct grouped_view {
  batches_view b;
  uint32_t m;                // positions (the reserved total)
  unsigned long long* hash;  // [m] sorted hashes
  uint32_t* gid;             // [m] flat request id at each sorted position
  gfn* fn;                   // [m] each request's own transfer function
  gfn* pre;                  // [m] composition of the earlier requests of its run
  uint32_t* flags;           // [m] bit 0 (at a run head): serve the run one by one; bit 1: key differs from the previous
  uint32_t* init;            // [m] at a run head: kGAbsent or the value length the tree held
  uint32_t* act;             // [m] at a run head: final write (kGKeep none, kGAbsent erase, else insert/update id)
  uint32_t* vals;            // [m][max_value_length] at a run head: the value the tree held
  uint32_t* heads;           // run heads of keys touched more than once (count: counts[0])
  uint32_t* singles;         // inserts on keys touched once (count: counts[1])
  uint32_t* singles_ue;      // updates and erases on keys touched once (count: counts[4])
  uint32_t* serial;          // heads of runs served one by one (count: counts[2])
  uint32_t* finds;           // finds on keys touched once (count: counts[3])
  uint32_t* counts;          // [5], zeroed at the start of the call
  unsigned long long hash_mask;  // bits of the key hash used (mt_set_group_hash_bits)
};

struct greq {
  const mt_subbatch* d;
  uint32_t i;
  uint32_t kind, klen, vlen;
};

MT_DEV greq group_req(const grouped_view& g, uint32_t id) {
  greq r;
  const uint32_t sb = find_subbatch(g.b.offsets, g.b.nsub, id);
  r.d = g.b.sub + sb;
  r.i = id - g.b.offsets[sb];
  r.kind = r.d->request_types[r.i];
  r.klen = r.d->key_lengths ? r.d->key_lengths[r.i] : g.b.max_key_length;
  r.vlen = (r.kind == MT_REQ_INSERT || r.kind == MT_REQ_UPDATE) ? r.d->value_lengths[r.i] : 0u;
  return r;
}
template <int T>
MT_DEV greq greq_shfl(const tile<T>& t, const greq& r, int src) {
  greq q;
  q.d = reinterpret_cast<const mt_subbatch*>(t.shfl64(reinterpret_cast<uint64_t>(r.d), src));
  q.i = t.shfl(r.i, src);
  q.kind = t.shfl(r.kind, src);
  q.klen = t.shfl(r.klen, src);
  q.vlen = t.shfl(r.vlen, src);
  return q;
}
// Warp-aggregated append of j to `list` (count at *count) by the lanes where want holds.
MT_DEV void list_append(bool want, uint32_t* list, uint32_t* count, uint32_t j) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t act = __activemask();
  const uint32_t bal = __ballot_sync(act, want);
  if (!bal) return;
  const uint32_t leader = __ffs(bal) - 1u;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(bal));
  base = __shfl_sync(act, base, (int)leader);
  if (want) list[base + __popc(bal & ((1u << lane) - 1u))] = j;
}
MT_DEV const uint32_t* greq_key(const grouped_view& g, const greq& r) {
  return r.d->keys + (size_t)r.i * g.b.max_key_length;
}
MT_DEV uint32_t* greq_val(const grouped_view& g, const greq& r) {
  return r.d->values + (size_t)r.i * g.b.max_value_length;
}
// Requests the per-call path rejects (lengths beyond the rows, unknown kinds).
MT_DEV bool greq_bad(const grouped_view& g, const greq& r) {
  return r.klen > g.b.max_key_length || r.vlen > g.b.max_value_length || r.kind > MT_REQ_UPDATE;
}

MT_DEV unsigned long long key_hash64(const uint32_t* key, uint32_t klen) {
  unsigned long long h = 0x9E3779B97F4A7C15ull ^ ((unsigned long long)klen * 0xD6E8FEB86659FD93ull);
  for (uint32_t s = 0; s < klen; ++s) {
    h ^= key[s];
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 31;
  }
  h ^= h >> 33;
  h *= 0x94D049BB133111EBull;
  h ^= h >> 29;
  return h % kGMaxHash;
}

// 1. Sort keys: the key's hash; a one-off value for a request served on its
// own (an empty key), kGBad for a rejected request, kGPad past the last one.
__global__ void group_hash_kernel(tree_view tv, grouped_view g, unsigned long long* hash_in, uint32_t* gid_in) {
  const uint32_t total = g.b.status[0] ? 0u : g.b.offsets[g.b.nsub];
  for (uint32_t id = blockIdx.x * blockDim.x + threadIdx.x; id < g.m; id += gridDim.x * blockDim.x) {
    unsigned long long h = kGPad;
    if (id < total) {
      const greq r = group_req(g, id);
      if (greq_bad(g, r)) {
        h = kGBad;
        record_error(tv.pool, ERR_INVALID_ARG);
      } else if (r.klen == 0u) {
        h = kGMaxHash + 1ull + id;
      } else {
        h = key_hash64(greq_key(g, r), r.klen) & g.hash_mask;
      }
    }
    hash_in[id] = h;
    gid_in[id] = id;
  }
}

// 2. Each request's transfer function; a key that differs from its
// neighbour's under the same hash is flagged.
__global__ void group_fn_kernel(grouped_view g) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < g.m; j += gridDim.x * blockDim.x) {
    const unsigned long long h = g.hash[j];
    gfn f{kGAbsent, kGKeep, j};
    uint32_t fl = 0;
    if (h < kGBad) {
      const uint32_t id = g.gid[j];
      const greq r = group_req(g, id);
      if (r.kind == MT_REQ_INSERT) f.a = id;
      else if (r.kind == MT_REQ_UPDATE) f.p = id;
      else if (r.kind == MT_REQ_ERASE) f.p = kGAbsent;
      if (j > 0u && h <= kGMaxHash && g.hash[j - 1u] == h) {
        const greq q = group_req(g, g.gid[j - 1u]);
        bool same = q.klen == r.klen;
        const uint32_t* a = greq_key(g, r);
        const uint32_t* b = greq_key(g, q);
        for (uint32_t s = 0; same && s < r.klen; ++s) same = a[s] == b[s];
        if (!same) fl = 2u;
      }
    }
    g.fn[j] = f;
    g.flags[j] = fl;
  }
}

MT_DEV uint32_t run_head(const grouped_view& g, uint32_t j) {
  const uint32_t f = g.pre[j].first;
  return f == kGNoFirst ? j : f;
}
MT_DEV bool run_last(const grouped_view& g, uint32_t j) {
  return j + 1u >= g.m || g.hash[j + 1u] != g.hash[j];
}

// 3. A run holding two different keys is served one by one (flag at its head,
// head listed once).
__global__ void group_mark_kernel(grouped_view g) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < g.m; j += gridDim.x * blockDim.x) {
    if (!(g.flags[j] & 2u)) continue;
    const uint32_t head = g.pre[j].first;
    if (!(atomicOr(&g.flags[head], 1u) & 1u)) g.serial[atomicAdd(&g.counts[2], 1u)] = head;
  }
}

// 4. Work lists: heads of keys touched more than once, writes and finds on
// keys touched once.
__global__ void group_list_kernel(grouped_view g) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = blockIdx.x * blockDim.x; base < g.m; base += stride) {
    const uint32_t j = base + threadIdx.x;
    bool head = false, multi = false, ins = false, find = false;
    if (j < g.m && g.hash[j] < kGBad && g.pre[j].first == kGNoFirst && !(g.flags[j] & 1u)) {
      head = true;
      multi = !run_last(g, j);
      ins = g.fn[j].a != kGAbsent;
      find = !ins && g.fn[j].p == kGKeep;
    }
    const bool single = head && !multi;
    list_append(head && multi, g.heads, &g.counts[0], j);
    list_append(single && ins, g.singles, &g.counts[1], j);
    list_append(single && !ins && !find, g.singles_ue, &g.counts[4], j);
    list_append(single && find, g.finds, &g.counts[3], j);
  }
}

// Find that also tells a present key with an empty value from an absent one.
template <int T>
MT_DEV bool group_lookup(const tile<T>& t, const tree_view& tv, const uint32_t* key, uint32_t klen, uint32_t* out,
                         uint32_t maxV, uint32_t& vlen) {
  const pool_view& p = tv.pool;
  uint32_t root = tv.root, hops = 0;
  node<T> nd;
  vlen = 0;
  for (uint32_t layer = 0; layer < klen; ++layer) {
    const uint32_t slice = key[layer];
    const bool more = layer + 1u < klen;
    if (!descend<T, kConc>(t, p, root, slice, nd, hops)) return false;
    const int e = nd.match(t, slice, more);
    if (e < 0) return false;
    const uint32_t st = ks_get(nd.ks, (uint32_t)e);
    const uint32_t v = nd.val_at(t, (uint32_t)e);
    if (st == KS_LINK) { root = v; continue; }
    if (st == KS_VALUE) {
      if (maxV > 0u && t.leader()) out[0] = v;
      vlen = 1u;
      return true;
    }
    if (!p.valid(v)) { if (t.leader()) record_error(p, ERR_CORRUPT, MT_AT(SRC_TREE)); return false; }
    suffix_head<T> h;
    h.template load<kConcSuffix>(t, p, v);
    if (st == KS_SUFFIX) {
      const uint32_t lk = klen - layer - 1u;
      if (h.klen != lk) return false;
      if (suffix_compare<T, kConcSuffix>(t, p, h, key + layer + 1u, lk).sign != 0) return false;
    }
    vlen = suffix_get_value<T, kConcSuffix>(t, p, h, out, maxV);
    return true;
  }
  return false;
}

// 5. Run heads of keys touched more than once: the tree's state of the key;
// and the finds on keys touched once.
template <int T>
__global__ void __launch_bounds__(kBlock, MT_MIN_BLOCKS_PER_SM) group_head_kernel(tree_view tv, grouped_view g) {
  tile<T> t;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / T;
  const uint32_t num_tiles = (gridDim.x * blockDim.x) / T;
  const uint32_t maxV = g.b.max_value_length;
  const uint32_t nh = g.counts[0], n = nh + g.counts[3];
  // As in the batch kernels: each lane fetches one entry's request, then the
  // tile serves the entries one after the other.
  for (uint32_t base = tile_id * T; base < n; base += num_tiles * T) {
    if (t.shfl((uint32_t)(t.leader() && fatal_error(tv.pool)), 0)) break;
    const uint32_t mine = base + t.rank;
    uint32_t j = 0;
    greq rq{};
    if (mine < n) {
      j = mine < nh ? g.heads[mine] : g.finds[mine - nh];
      rq = group_req(g, g.gid[j]);
    }
    const uint32_t cnt = min((uint32_t)T, n - base);
    for (uint32_t q = 0; q < cnt; ++q) {
      const greq r = greq_shfl(t, rq, (int)q);
      const uint32_t jj = t.shfl(j, (int)q);
      if (base + q >= nh) {  // a find on a key touched once: served directly
        const uint32_t vo = coop_find<T, true>(t, tv, greq_key(g, r), r.klen, greq_val(g, r), maxV);
        if (t.leader()) r.d->value_lengths[r.i] = vo;
        continue;
      }
      uint32_t vl = 0;
      const bool found = group_lookup<T>(t, tv, greq_key(g, r), r.klen, g.vals + (size_t)jj * maxV, maxV, vl);
      if (t.leader()) {
        g.init[jj] = found ? vl : kGAbsent;
        g.act[jj] = kGKeep;
      }
    }
  }
}

// 6. Results of the requests on keys touched more than once, from the scanned
// state (one thread per request: a find copies at most max_value_length
// slices), and the final write of each such key (at its head).
__global__ void group_result_kernel(grouped_view g) {
  const uint32_t maxV = g.b.max_value_length;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < g.m; j += gridDim.x * blockDim.x) {
    if (g.hash[j] >= kGBad) continue;
    const gfn pf = g.pre[j];
    const uint32_t head = pf.first == kGNoFirst ? j : pf.first;
    const bool last = run_last(g, j);
    if ((head == j && last) || (g.flags[head] & 1u)) continue;  // touched once, or served one by one
    const greq r = group_req(g, g.gid[j]);
    const uint32_t init = g.init[head];
    const uint32_t s0 = init == kGAbsent ? kGAbsent : kGKeep;
    const uint32_t before = gfn_apply(s0, pf);
    if (r.kind == MT_REQ_FIND) {
      uint32_t vo = 0;
      const uint32_t* src = nullptr;
      if (before == kGKeep) {
        vo = init;
        src = g.vals + (size_t)head * maxV;
      } else if (before != kGAbsent) {
        const greq w = group_req(g, before);
        vo = w.vlen;
        src = greq_val(g, w);
      }
      uint32_t* out = greq_val(g, r);
      const uint32_t c = min(vo, maxV);
      for (uint32_t s = 0; s < c; ++s) out[s] = src[s];
      r.d->value_lengths[r.i] = vo;
    } else if (r.d->results) {
      r.d->results[r.i] = r.kind == MT_REQ_INSERT ? before == kGAbsent : before != kGAbsent;
    }
    if (last) {
      const uint32_t fin = gfn_apply(s0, gfn_compose()(pf, g.fn[j]));
      g.act[head] = fin == s0 ? kGKeep : fin;  // kGAbsent here: present before, erased
    }
  }
}

// 7. Writes: the requests on keys touched once, or the final write of every
// key touched more than once.
// MODE kGWInsert / kGWUpdErase: the inserts / the updates and erases on keys
// touched once (they need nothing from the other passes and run beside them,
// each kernel compiled for its kinds only); kGWHeads: the final writes.
constexpr int kGWInsert = 0, kGWUpdErase = 1, kGWHeads = 2;
template <int T, int MODE>
__global__ void __launch_bounds__(kBlock, MT_WRITE_MIN_BLOCKS_PER_SM) group_write_kernel(tree_view tv, grouped_view g) {
  tile<T> t;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / T;
  const uint32_t num_tiles = (gridDim.x * blockDim.x) / T;
  slab_cache<T> cache;
  cache.init(tv.pool, tile_id);
  constexpr bool HEADS = MODE == kGWHeads;
  const uint32_t n = HEADS ? g.counts[0] : (MODE == kGWInsert ? g.counts[1] : g.counts[4]);
  for (uint32_t base = tile_id * T; base < n; base += num_tiles * T) {
    if (t.shfl((uint32_t)(t.leader() && fatal_error(tv.pool)), 0)) break;
    // Each lane fetches one entry: its request and, for a key touched more
    // than once, the final write and the request whose value it writes.
    const uint32_t mine = base + t.rank;
    greq rq{}, wq{};
    uint32_t act = kGKeep, init = kGAbsent;
    if (mine < n) {
      const uint32_t j = HEADS ? g.heads[mine] : (MODE == kGWInsert ? g.singles[mine] : g.singles_ue[mine]);
      rq = group_req(g, g.gid[j]);
      if (HEADS) {
        act = g.act[j];
        init = g.init[j];
        if (act != kGKeep && act != kGAbsent) wq = group_req(g, act);
      }
    }
    const uint32_t cnt = min((uint32_t)T, n - base);
    for (uint32_t q = 0; q < cnt; ++q) {
      const greq r = greq_shfl(t, rq, (int)q);
      const uint32_t* key = greq_key(g, r);
      if constexpr (MODE == kGWInsert) {
        const int res = coop_insert<T, false>(t, tv, cache, key, r.klen, greq_val(g, r), r.vlen);
        if (t.leader() && r.d->results) r.d->results[r.i] = res == RES_OK;
      } else if constexpr (MODE == kGWUpdErase) {
        int res;
        if (r.kind == MT_REQ_UPDATE) res = coop_update<T>(t, tv, cache, key, r.klen, greq_val(g, r), r.vlen);
        else res = coop_erase<T>(t, tv, key, r.klen);
        if (t.leader() && r.d->results) r.d->results[r.i] = res == RES_OK;
      } else {
        const uint32_t a = t.shfl(act, (int)q);
        if (a == kGKeep) continue;
        if (a == kGAbsent) {
          coop_erase<T>(t, tv, key, r.klen);
          continue;
        }
        const greq w = greq_shfl(t, wq, (int)q);
        if (t.shfl(init, (int)q) == kGAbsent) coop_insert<T, false>(t, tv, cache, key, r.klen, greq_val(g, w), w.vlen);
        else coop_update<T>(t, tv, cache, key, r.klen, greq_val(g, w), w.vlen);
      }
    }
  }
  cache.release(t, tv.pool);
}

// 8. Runs holding two keys under one hash: every request in order.
template <int T>
__global__ void __launch_bounds__(kBlock, MT_WRITE_MIN_BLOCKS_PER_SM) group_serial_kernel(tree_view tv, grouped_view g) {
  tile<T> t;
  const uint32_t tile_id = (blockIdx.x * blockDim.x + threadIdx.x) / T;
  const uint32_t num_tiles = (gridDim.x * blockDim.x) / T;
  slab_cache<T> cache;
  cache.init(tv.pool, tile_id);
  const uint32_t maxV = g.b.max_value_length;
  const uint32_t n = g.counts[2];
  for (uint32_t q = tile_id; q < n; q += num_tiles) {
    const uint32_t j = g.serial[q];
    for (uint32_t k = j; k < g.m && g.hash[k] == g.hash[j]; ++k) {
      if (t.shfl((uint32_t)(t.leader() && fatal_error(tv.pool)), 0)) break;
      const greq r = group_req(g, g.gid[k]);
      const uint32_t* key = greq_key(g, r);
      if (r.kind == MT_REQ_FIND) {
        const uint32_t vo = coop_find<T, true>(t, tv, key, r.klen, greq_val(g, r), maxV);
        if (t.leader()) r.d->value_lengths[r.i] = vo;
        continue;
      }
      int res = RES_FAIL;
      if (r.kind == MT_REQ_INSERT) res = coop_insert<T, false>(t, tv, cache, key, r.klen, greq_val(g, r), r.vlen);
      else if (r.kind == MT_REQ_UPDATE) res = coop_update<T>(t, tv, cache, key, r.klen, greq_val(g, r), r.vlen);
      else res = coop_erase<T>(t, tv, key, r.klen);
      if (t.leader() && r.d->results) r.d->results[r.i] = res == RES_OK;
    }
  }
  cache.release(t, tv.pool);
}

}  // namespace mtb

using namespace mtb;

namespace {

struct hash_equal {
  __host__ __device__ bool operator()(unsigned long long a, unsigned long long b) const { return a == b; }
};

size_t up256(size_t x) { return (x + 255u) & ~size_t(255); }

// Scratch for m positions and rows of max_v value slices (grown on demand).
int ensure_grouped(mt_masstree* t, uint32_t m, uint32_t max_v, cudaStream_t s) {
  if (t->grouped_mem && t->grouped_m >= m && t->grouped_max_v >= max_v) return MT_OK;
  m = std::max(m, t->grouped_m);
  max_v = std::max(max_v, t->grouped_max_v);
  size_t sort_bytes = 0, scan_bytes = 0;
  if (cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (unsigned long long*)nullptr,
                                      (unsigned long long*)nullptr, (uint32_t*)nullptr, (uint32_t*)nullptr, (int)m, 0,
                                      64, s) != cudaSuccess ||
      cub::DeviceScan::ExclusiveScanByKey(nullptr, scan_bytes, (unsigned long long*)nullptr, (gfn*)nullptr,
                                          (gfn*)nullptr, gfn_compose(), gfn{kGAbsent, kGKeep, kGNoFirst}, (int)m,
                                          hash_equal(), s) != cudaSuccess)
    return MT_ERR_CUDA;
  const size_t temp = std::max(sort_bytes, scan_bytes);
  const size_t bytes = 4 * up256((size_t)m * 8u) + 2 * up256((size_t)m * sizeof(gfn)) + 8 * up256((size_t)m * 4u) +
                       up256((size_t)m * max_v * 4u) + up256(temp);
  if (cudaDeviceSynchronize() != cudaSuccess) return MT_ERR_CUDA;
  if (t->grouped_mem) cudaFree(t->grouped_mem);
  t->grouped_mem = nullptr;
  t->grouped_m = 0;
  t->grouped_max_v = 0;
  if (cudaMalloc(&t->grouped_mem, bytes) != cudaSuccess) {
    cudaGetLastError();
    return MT_ERR_OOM;
  }
  t->grouped_m = m;
  t->grouped_max_v = max_v;
  t->grouped_temp = temp;
  return MT_OK;
}

template <int T>
int launch_tile_kernel(mt_masstree* t, void (*fn)(tree_view, grouped_view), const grouped_view& g, cudaStream_t s) {
  int bps = host_max_blocks_per_sm((const void*)fn, kBlock, 0);
  if (t->blocks_per_sm > 0) bps = std::min<int>(bps, (int)t->blocks_per_sm);
  fn<<<std::max(bps, 1) * t->sms, kBlock, 0, s>>>(t->tv, g);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_CUDA;
}

template <int TF>
int launch_find_side(mt_masstree* t, const grouped_view& g, cudaStream_t s) {
  int rc = launch_tile_kernel<TF>(t, group_head_kernel<TF>, g, s);
  if (rc) return rc;
  const int grid = std::max(1, std::min<int>(t->sms * 8, (int)((g.m + 255u) / 256u)));
  group_result_kernel<<<grid, 256, 0, s>>>(g);
  return cudaGetLastError() == cudaSuccess ? MT_OK : MT_ERR_CUDA;
}

template <int TW>
int launch_singles(mt_masstree* t, const grouped_view& g, cudaStream_t s_ins, cudaStream_t s_ue) {
  int rc = launch_tile_kernel<TW>(t, group_write_kernel<TW, kGWInsert>, g, s_ins);
  if (!rc) rc = launch_tile_kernel<TW>(t, group_write_kernel<TW, kGWUpdErase>, g, s_ue);
  if (!rc) rc = launch_tile_kernel<TW>(t, group_serial_kernel<TW>, g, s_ue);
  return rc;
}
template <int TW>
int launch_heads(mt_masstree* t, const grouped_view& g, cudaStream_t s) {
  return launch_tile_kernel<TW>(t, group_write_kernel<TW, kGWHeads>, g, s);
}

}  // namespace

namespace mtb {

int launch_grouped(mt_masstree* t, const batches_view& b, cudaStream_t s) {
  const uint32_t m = (uint32_t)t->batches_max_total;
  // CUB counts items in int; without room for the scratch the caller serves
  // the call in the forked form instead (nothing has been launched yet).
  if (m > 0x7FFFFFFFu) return kGroupedUnavailable;
  int rc = ensure_grouped(t, m, b.max_value_length, s);
  if (rc == MT_ERR_OOM) return kGroupedUnavailable;
  if (rc) return rc;
  grouped_view g{};
  g.b = b;
  g.m = m;
  g.hash_mask = t->group_hash_bits >= 64u ? ~0ull : ((1ull << t->group_hash_bits) - 1ull);
  char* p = static_cast<char*>(t->grouped_mem);
  auto carve = [&](size_t bytes) {
    char* r = p;
    p += up256(bytes);
    return r;
  };
  const size_t M = t->grouped_m;
  auto* hash_in = reinterpret_cast<unsigned long long*>(carve(M * 8u));
  g.hash = reinterpret_cast<unsigned long long*>(carve(M * 8u));
  auto* gid_in = reinterpret_cast<uint32_t*>(carve(M * 8u));  // 8-byte slots keep the carving simple
  g.gid = reinterpret_cast<uint32_t*>(carve(M * 8u));
  g.fn = reinterpret_cast<gfn*>(carve(M * sizeof(gfn)));
  g.pre = reinterpret_cast<gfn*>(carve(M * sizeof(gfn)));
  g.flags = reinterpret_cast<uint32_t*>(carve(M * 4u));
  g.init = reinterpret_cast<uint32_t*>(carve(M * 4u));
  g.act = reinterpret_cast<uint32_t*>(carve(M * 4u));
  g.vals = reinterpret_cast<uint32_t*>(carve(M * t->grouped_max_v * 4u));
  g.heads = reinterpret_cast<uint32_t*>(carve(M * 4u));
  g.singles = reinterpret_cast<uint32_t*>(carve(M * 4u));
  g.serial = reinterpret_cast<uint32_t*>(carve(M * 4u));
  g.finds = reinterpret_cast<uint32_t*>(carve(M * 4u));
  g.singles_ue = reinterpret_cast<uint32_t*>(carve(M * 4u));
  void* temp = carve(t->grouped_temp);
  g.counts = b.status + 2;
  if (cudaMemsetAsync(g.counts, 0, 5 * sizeof(uint32_t), s) != cudaSuccess) return MT_ERR_CUDA;
  const int grid = std::max(1, std::min<int>(t->sms * 8, (int)((m + 255u) / 256u)));
  group_hash_kernel<<<grid, 256, 0, s>>>(t->tv, g, hash_in, gid_in);
  if (cudaGetLastError() != cudaSuccess) return MT_ERR_CUDA;
  size_t tb = t->grouped_temp;
  if (cub::DeviceRadixSort::SortPairs(temp, tb, hash_in, g.hash, gid_in, g.gid, (int)m, 0, 64, s) != cudaSuccess)
    return MT_ERR_CUDA;
  group_fn_kernel<<<grid, 256, 0, s>>>(g);
  if (cudaGetLastError() != cudaSuccess) return MT_ERR_CUDA;
  tb = t->grouped_temp;
  if (cub::DeviceScan::ExclusiveScanByKey(temp, tb, g.hash, g.fn, g.pre, gfn_compose(),
                                          gfn{kGAbsent, kGKeep, kGNoFirst}, (int)m, hash_equal(),
                                          s) != cudaSuccess)
    return MT_ERR_CUDA;
  group_mark_kernel<<<grid, 256, 0, s>>>(g);
  group_list_kernel<<<grid, 256, 0, s>>>(g);
  if (cudaGetLastError() != cudaSuccess) return MT_ERR_CUDA;
  // Keys touched once (and runs served one by one) on a side stream, beside
  // the reads, results and final writes of the keys touched more than once:
  // no key is in both.
  rc = host_fork(t, s);
  if (rc) return rc;
  const bool w16 = t->write_tile_size <= 16;
  rc = w16 ? launch_singles<16>(t, g, t->side[0], t->side[1]) : launch_singles<32>(t, g, t->side[0], t->side[1]);
  if (!rc) {
    switch (t->tile_size) {
      case 4: rc = launch_find_side<4>(t, g, s); break;
      case 8: rc = launch_find_side<8>(t, g, s); break;
      case 16: rc = launch_find_side<16>(t, g, s); break;
      default: rc = launch_find_side<32>(t, g, s); break;
    }
  }
  if (!rc) rc = w16 ? launch_heads<16>(t, g, s) : launch_heads<32>(t, g, s);
  return host_join(t, s, rc);
}

}  // namespace mtb

extern "C" int mt_set_group_hash_bits(mt_masstree* t, uint32_t bits) {
  if (!t || bits == 0u || bits > 64u) return MT_ERR_INVALID_ARG;
  t->group_hash_bits = bits;
  return MT_OK;
}
